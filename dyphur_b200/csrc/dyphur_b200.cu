// Single translation unit of the native library: the kernels share device
// symbols (the sticky error word) and inline helpers without relocatable
// device code.
#include "integrate.cu"
#include "sort.cu"
#include "broadphase.cu"
#include "narrowphase.cu"
#include "solver.cu"
#include "hash.cu"
#include "ray_query.cu"
#include "world.cu"
