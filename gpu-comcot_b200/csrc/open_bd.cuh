/*
 * OPEN radiation boundary on one perimeter cell of the outermost layer
 * (boundaries.f90:42-200), shared by the fused step kernels.
 *
 * The square root and the division run on every lane that evaluates the
 * cell, including lanes whose cell is still water or dry (the two-step
 * kernel evaluates the perimeter column on all lanes to stay convergent).
 * An exact zero is answered without calling sqrtf or dividing, and a dry
 * cell's depth is replaced before its square root, so no lane takes the
 * special-case path of either operation for those inputs; every result is
 * the bits sqrtf and '/' give: sqrt(+0) = +0, and 0 / c = 0 with the sign of
 * the zero for c > 0.
 */
#ifndef GC_OPEN_BD_CUH
#define GC_OPEN_BD_CUH

#include "gc_internal.h"

namespace gcopen {

/* sqrtf(x) for x >= 0 or NaN */
__device__ __forceinline__ float sqrt_nz(float x) {
    const bool z = x == 0.0f;
    const float r = sqrtf(z ? 1.0f : x);
    return z ? x : r;
}

/* x / y for y > 0 */
__device__ __forceinline__ float div_nz(float x, float y) {
    const bool z = x == 0.0f;
    const float q = (z ? 1.0f : x) / y;
    return z ? x : q;
}

/* OPEN at (i,j): h, m, n at (i,j); hs, ns at (i,j-1); mw at (i-1,j) */
__device__ __forceinline__ float open_cell(int i, int j, int nx, int ny, float h, float hs, float m, float mw,
                                           float n, float ns) {
    const bool wet = h > CC_GX;
    const float cc = sqrtf(CC_GRAV * (wet ? h : 1.0f));
    const bool corner = (i == 0 || i == nx - 1) && (j == 0 || j == ny - 1);
    /* the flux along the boundary (a) and across it (b), as the reference
     * forms UH and the normal flux; neg: the outgoing direction */
    float a, b;
    bool neg;
    if (!corner) {
        if (j == 0) {
            a = 0.5f * (m + mw);
            b = n;
            neg = n > 0.0f;
        } else if (j == ny - 1) {
            a = 0.5f * (m + mw);
            b = ns;
            neg = ns < 0.0f;
        } else if (i == 0) {
            a = (hs > CC_GX) ? 0.5f * (n + ns) : n;
            b = m;
            neg = m > 0.0f;
        } else {
            a = 0.5f * (n + ns);
            b = mw;
            neg = mw < 0.0f;
        }
    } else {
        a = (i == 0) ? m : mw; /* QX */
        b = (j == 0) ? n : ns; /* QY */
        if (i == 0 && j == 0) neg = (a > 0.0f || b > 0.0f);
        else if (j == 0) neg = (a < 0.0f || b > 0.0f);
        else if (i == 0) neg = (a > 0.0f || b < 0.0f);
        else neg = (a < 0.0f || b < 0.0f);
    }
    float zz = div_nz(sqrt_nz(a * a + b * b), cc);
    if (neg) zz = -zz;
    if (fabsf(zz) > CC_UB) zz = 0.0f;
    return wet ? zz : 0.0f;
}

} // namespace gcopen

#endif
