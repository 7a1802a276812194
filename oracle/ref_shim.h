/*
 * ref_shim.h -- lets the reference's CUDA kernel sources compile as plain
 * host C++ so that they can serve as the parity oracle's anchor.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle/cpab_oracle.c).  The reference files
 * are #included from the reference checkout at build time (oracle/Makefile,
 * REF_ROOT); nothing of them is copied into this repository.
 *
 * Emulation model: one CUDA block is run by one host thread, thread by
 * thread.  __shared__ arrays become per-host-thread statics.  Because the
 * reference's kernels fill shared memory and then __syncthreads(), the
 * wrappers in ref_shim.cpp first run every thread of a block once with a
 * block index past the data (fill only), then run the block for real.
 */
#pragma once
#include <cmath>
#include <algorithm>

using std::min;
using std::max;

struct ref_dim3 { unsigned x, y, z; };
extern thread_local ref_dim3 threadIdx, blockIdx, blockDim;

#define __device__
#define __global__
#define __shared__ static thread_local
#define __syncthreads() ((void)0)
