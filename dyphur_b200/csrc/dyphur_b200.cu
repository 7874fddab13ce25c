// Main translation unit of the native library: the kernels share device
// symbols (the sticky error word) and inline helpers without relocatable
// device code. The adjoint's reverse kernel is the one kernel built apart
// (reverse.cu, with its own numerics flags); it shares no device symbol.
#include "integrate.cu"
#include "sort.cu"
#include "broadphase.cu"
#include "narrowphase.cu"
#include "solver.cu"
#include "hash.cu"
#include "ray_query.cu"
#include "world.cu"
