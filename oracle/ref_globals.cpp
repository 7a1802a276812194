/* ref_globals.cpp -- the emulated CUDA built-in indices of ref_shim.h.
 * TEST INFRASTRUCTURE ONLY. */
#include "ref_shim.h"
thread_local ref_dim3 threadIdx, blockIdx, blockDim;
