// cpab_ctx.h -- the context behind the opaque cpab_ctx handle and the
// error helpers shared by the C ABI files.
#pragma once

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cstdint>
#include <initializer_list>
#include <vector>

#include "../../include/cpab_b200.h"
#include "cpab_internal.h"
#include "cpab_launch.h"

struct cpab_ctx {
    cpab::Tess t;
    int nCs[3];
    int clamp = 0;
    double clamp_lo = 0, clamp_hi = 0;
    cpab::LaunchCfg cfg;
    // Cancellation: a flag in device memory that the persistent kernels poll
    // (an L2 read), written by a 4-byte DMA from a pinned {0, 1} pair on a
    // private non-blocking stream -- no SM is needed to set it while kernels
    // occupy the GPU, and the kernels never read host memory over PCIe.
    int *cancel_dev = nullptr;
    int *cancel_src = nullptr;         // pinned host {0, 1}
    cudaStream_t cancel_stream = nullptr;
    int cancel_state = 0;              // host mirror (atomic)
    int device = -1;                   // the device the flag lives on
    // facet tables for the 2D/3D exact scheme, on the same device
    double *facets_dev = nullptr;
    int *nbr_dev = nullptr;
    int nF = 0;
    char err[512] = {0};
};

namespace cpab {

extern thread_local char g_thread_err[512];

inline int fail(cpab_ctx *ctx, int status, const char *fmt, ...)
{
    char *buf = ctx ? ctx->err : g_thread_err;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, 512, fmt, ap);
    va_end(ap);
    return status;
}

inline int cuda_status(cpab_ctx *ctx, cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return CPAB_OK;
    return fail(ctx, CPAB_CUDA_ERROR, "%s: %s", what, cudaGetErrorString(e));
}

inline int cell_len(const cpab_ctx *c) { return c->t.dim * (c->t.dim + 1); }

inline bool overlaps(const void *a, size_t na, const void *b, size_t nb)
{
    const char *pa = (const char *)a, *pb = (const char *)b;
    return pa < pb + nb && pb < pa + na;
}

// Device arrays must be aligned to their element size (a misaligned access
// faults the kernel).  Returns the name of the first offender, or nullptr.
struct AlignReq {
    const void *p;
    size_t bytes;
    const char *name;
};
inline const char *misaligned(std::initializer_list<AlignReq> reqs)
{
    for (const AlignReq &r : reqs)
        if (r.p && (reinterpret_cast<uintptr_t>(r.p) % r.bytes) != 0) return r.name;
    return nullptr;
}

#define CPAB_CHECK_ALIGN(ctx, ...)                                                                          \
    do {                                                                                                    \
        if (const char *m_ = ::cpab::misaligned({__VA_ARGS__}))                                             \
            return fail(ctx, CPAB_BAD_ARG, "%s is not aligned to its element size", m_);                   \
    } while (0)

// The cancel flag to hand to a launch: the context's device flag when the
// launch goes to the device the flag lives on, else none (no polling).
inline const volatile int *cancel_ptr(const cpab_ctx *c)
{
    int d = -1;
    return (c->cancel_dev && cudaGetDevice(&d) == cudaSuccess && d == c->device) ? c->cancel_dev : nullptr;
}

int max_smem_optin();
int build_facets(const Tess &t, const int *nCs, std::vector<double> &F, std::vector<int> &nbr);

}  // namespace cpab
