# Builds the xtcore side of the GPU path: the GPU integrator and Scene
# flattener (gpu_integrator.cc) and the xtgpu-xtcore front end, linked with
# XTracer's own host code (xtcore + lib/*), compiled from the XTracer source
# tree where it lies, and with libxtgpu.so.
#
#   make -f xtracer_b200/xtcore/xtcore.mk REF=<XTracer source tree> -j8
#
# Outputs go to xtracer_b200/_build/: xtcore_obj/ (the host objects) and
# xtgpu-xtcore (rpath $ORIGIN, next to libxtgpu.so, which must be built first).

ifndef REF
$(error REF must name the XTracer source tree: make -f xtracer_b200/xtcore/xtcore.mk REF=<dir>)
endif
HERE     := $(dir $(lastword $(MAKEFILE_LIST)))
BUILD    := $(HERE)../_build
OBJDIR   := $(BUILD)/xtcore_obj

SRCS_CC  := $(sort $(wildcard $(REF)/src/xtcore/*.cc $(REF)/src/xtcore/*/*.cc \
                              $(REF)/src/xtcore/*/*/*.cc $(REF)/lib/*/*.cc))
SRCS_C   := $(sort $(wildcard $(REF)/lib/*/*.c))

# the include directories of XTracer's CMake build (CMakeLists.txt:24-33)
HDR_DIRS := $(sort $(dir $(shell find $(REF)/src/xtcore $(REF)/lib $(REF)/ext -name '*.h')))
INCS     := -I$(REF)/lib -I$(REF)/src -I$(REF)/ext $(addprefix -I,$(HDR_DIRS))
SYSINCS  := -isystem $(REF)/lib -isystem $(REF)/src -isystem $(REF)/ext $(addprefix -isystem ,$(HDR_DIRS))

CXX      := /usr/bin/g++
CC       := /usr/bin/gcc
HOSTFLAGS := -O2 -fopenmp -std=c++11 -fPIC -w -DXTCORE_VERSION='"xtgpu-host"' $(INCS)
HOSTCFLAGS := -O2 -fopenmp -std=gnu99 -fPIC -w $(INCS)
OWNFLAGS := -O2 -fopenmp -std=c++11 -fPIC -Wall -Wextra -DXTCORE_VERSION='"xtgpu-host"' \
            -I$(HERE)../../include $(SYSINCS)

OBJS     := $(patsubst $(REF)/%.cc,$(OBJDIR)/%.o,$(SRCS_CC)) \
            $(patsubst $(REF)/%.c,$(OBJDIR)/%.o,$(SRCS_C))
OWN      := $(OBJDIR)/own/gpu_integrator.o $(OBJDIR)/own/xtgpu_xtcore.o

all: $(BUILD)/xtgpu-xtcore

$(OBJDIR)/%.o: $(REF)/%.cc
	@mkdir -p $(dir $@)
	$(CXX) $(HOSTFLAGS) -c $< -o $@

$(OBJDIR)/%.o: $(REF)/%.c
	@mkdir -p $(dir $@)
	$(CC) $(HOSTCFLAGS) -c $< -o $@

$(OBJDIR)/own/%.o: $(HERE)%.cc $(HERE)gpu_integrator.h $(HERE)../../include/xtgpu.h
	@mkdir -p $(dir $@)
	$(CXX) $(OWNFLAGS) -c $< -o $@

$(BUILD)/xtgpu-xtcore: $(OWN) $(OBJS) $(BUILD)/libxtgpu.so
	$(CXX) -fopenmp $(OWN) $(OBJS) -L$(BUILD) -lxtgpu -Wl,-rpath,'$$ORIGIN' -o $@ -lpthread

clean:
	rm -rf $(OBJDIR) $(BUILD)/xtgpu-xtcore

.PHONY: all clean
