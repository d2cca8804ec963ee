# Builds the reference renderer (XTracer's xtcore + lib/*) from its own sources,
# where they lie, plus the harness driver in this folder, into oracle/_ref/.
#
# This is test infrastructure: the binary it makes is the checker (golden
# fixtures, pinning of the C restatement) and the timed CPU baseline.  It never
# feeds the GPU product path.
#
#   make -f oracle/ref.mk REF=<XTracer source tree> -j8
#
# Flags: -O2 -fopenmp.  The reference's own CMake "Release" flags are -O0
# (CMakeLists.txt:157); -O2 is used so the CPU baseline is not handicapped.

ifndef REF
$(error REF must name the XTracer source tree: make -f oracle/ref.mk REF=<dir>)
endif
HERE     := $(dir $(lastword $(MAKEFILE_LIST)))
OUT      := $(HERE)_ref
OBJDIR   := $(OUT)/obj

SRCS_CC  := $(sort $(wildcard $(REF)/src/xtcore/*.cc $(REF)/src/xtcore/*/*.cc \
                              $(REF)/src/xtcore/*/*/*.cc $(REF)/lib/*/*.cc))
SRCS_C   := $(sort $(wildcard $(REF)/lib/*/*.c))

HDR_DIRS := $(sort $(dir $(shell find $(REF)/src/xtcore $(REF)/lib $(REF)/ext -name '*.h')))
INCS     := -I$(REF)/lib -I$(REF)/src -I$(REF)/ext $(addprefix -I,$(HDR_DIRS))

# The image exports CXX/CC pointing at a wrapper whose driver cannot find
# libgomp.spec when linking with -fopenmp; the system compiler is used instead.
CXX      := /usr/bin/g++
CC       := /usr/bin/gcc
CXXFLAGS := -O2 -fopenmp -std=c++11 -fPIC -w -DXTCORE_VERSION='"ref-harness"' $(INCS)
CFLAGS   := -O2 -fopenmp -std=gnu99 -fPIC -w $(INCS)

OBJS     := $(patsubst $(REF)/%.cc,$(OBJDIR)/%.o,$(SRCS_CC)) \
            $(patsubst $(REF)/%.c,$(OBJDIR)/%.o,$(SRCS_C))

# The driver counts every Scene::intersection call (rays) and fixes time() so the
# reference's srand(time(NULL)) seeding is reproducible; both through --wrap, so
# no reference source is modified.
WRAPS    := -Wl,--wrap=_ZN6xtcore5Scene12intersectionERKNS_3RayERNS_12hit_record_tE \
            -Wl,--wrap=time

all: $(OUT)/xtref

$(OBJDIR)/%.o: $(REF)/%.cc
	@mkdir -p $(dir $@)
	$(CXX) $(CXXFLAGS) -c $< -o $@

$(OBJDIR)/%.o: $(REF)/%.c
	@mkdir -p $(dir $@)
	$(CC) $(CFLAGS) -c $< -o $@

$(OUT)/xtref: $(HERE)ref_driver.cc $(OBJS)
	$(CXX) $(CXXFLAGS) $(HERE)ref_driver.cc $(OBJS) $(WRAPS) -o $@ -lpthread

clean:
	rm -rf $(OUT)

.PHONY: all clean
