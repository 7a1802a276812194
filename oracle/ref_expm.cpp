/*
 * ref_expm.cpp -- host wrapper around the reference's affine-expm kernel
 * strings (cpab/gpu/expm/expm_affine_by_series_{2D,3D}.py, the `krnl`
 * variable), extracted to oracle/_ref/ by oracle/extract_krnl.py at build
 * time and included here.
 *
 * TEST INFRASTRUCTURE ONLY.  Compiled twice by oracle/Makefile with
 *   -DREF_EXPM_SRC="<extracted file>" -Dexpm=<unique kernel name>
 *   -DREF_EXPM_WRAPPER=<exported name>
 * The launch mirrors gpu_expm (expm_affine_by_series_2D.py:246-258): 512
 * threads per block, one thread per cell, series order p.
 */
#include "ref_shim.h"

#include REF_EXPM_SRC

extern "C" void REF_EXPM_WRAPPER(double *As, double *Ts, int N, int p)
{
    const unsigned bd = 512;
    const unsigned nb = (unsigned)((N + bd - 1) / bd);
    blockDim = ref_dim3{bd, 1, 1};
    for (unsigned b = 0; b < nb; ++b) {
        blockIdx = ref_dim3{b, 0, 0};
        for (unsigned t = 0; t < bd; ++t) {
            threadIdx = ref_dim3{t, 0, 0};
            expm(As, Ts, N, p);
        }
    }
}
