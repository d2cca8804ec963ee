"""B200 (sm_100a) backend for XTracer's ray-scene intersection and integrator
hot path.  The compute lives in libxtgpu.so (xtracer_b200/csrc, C ABI in
include/xtgpu.h); this package holds its Python binding and the seeded scene
generators used by the tests and the benchmark."""
