// site_rows.cuh: one site's row of block (a)'s least squares, Z = [phi | 1 | t], in registers, for the two
// normal-equation kernels (decoder.cu's FP64 tensor-core form and gram_tc.cu's tcgen05 form).
//
// The row has a fixed layout whatever the channel counts, so that every slot is a compile-time register: slots 0..3
// the level-1 sample c_b, 4..7 the level-0 sample s_i, 8..23 the products s_i c_b (i * 4 + b), 24 the constant 1,
// 25.. the targets, zeros in every slot a layout with fewer channels does not use and after the targets. The system's
// own (compact) column order, [c_b (c1)] [s_i (c0)] [s_i c_b] [1] [t] (src/sample.cuh:74-85), maps onto it by
// z_slot(). The arithmetic is the solver's: the samples by blend_u, the products rounded once, the fractional sites'
// targets from the per-model target cache (k_site_targets, the same blend of the source's four level-0 taps), so the
// FP64 form's sums are of the same floats as before.
#pragma once

#include "device.cuh"

namespace nb
{

constexpr int ZS_C = 0, ZS_S = 4, ZS_SC = 8, ZS_ONE = 24, ZS_T = 25, ZS_WIDTH = 48;

// The fixed slot of column a of the compact [phi (nin) | 1 | t (nout)].
__host__ __device__ __forceinline__ int z_slot(int a, int c0, int c1)
{
    const int nin = c1 + c0 + c0 * c1;
    if (a < c1)
        return ZS_C + a;
    if (a < c1 + c0)
        return ZS_S + (a - c1);
    if (a < nin)
    {
        const int q = a - c1 - c0;
        return ZS_SC + (q / c1) * 4 + q % c1;
    }
    return a == nin ? ZS_ONE : ZS_T + (a - nin - 1);
}

// Where the fractional sites' float targets of each plane start in the per-model cache ([site][NOUT]).
struct SiteTargetView
{
    const float* t;
    long long site0[MAX_PLANES + 1];
};

// Site j (0 the centre, 1..K fractional) of pixel (px, py) of plane V, as the fixed-layout row z.
template <int NOUT>
__device__ __forceinline__ void site_z(const Planes& P, const PlaneView& V, const float* tgt, long long pixel, int px,
                                       int py, int j, float (&z)[ZS_WIDTH])
{
    const int c0 = P.c0, c1 = P.c1;
    float dx, dy;
    site_offset(P.kc, j, px, py, dx, dy);
    float s[MAX_CH], c[MAX_CH];
    blend_u<MAX_CH>(V.v1, V.w1, c1, tap_at(px, py, dx, dy, V.w0, V.h0, V.w1, V.h1), c);
    const float* t;
    if (j == 0)
    {
#pragma unroll
        for (int i = 0; i < MAX_CH; i++)
            if (i < c0)
                s[i] = __ldg(V.v0 + pixel * c0 + i);
        t = V.src + (size_t)pixel * NOUT;
    }
    else
    {
        blend_u<MAX_CH>(V.v0, V.w0, c0, tap_at(px, py, dx, dy, V.w0, V.h0, V.w0, V.h0), s);
        t = tgt + (size_t)(pixel * P.kc + (j - 1)) * NOUT;
    }
#pragma unroll
    for (int b = 0; b < MAX_CH; b++)
        z[ZS_C + b] = b < c1 ? c[b] : 0.0f;
#pragma unroll
    for (int i = 0; i < MAX_CH; i++)
        z[ZS_S + i] = i < c0 ? s[i] : 0.0f;
#pragma unroll
    for (int i = 0; i < MAX_CH; i++)
#pragma unroll
        for (int b = 0; b < MAX_CH; b++)
            z[ZS_SC + i * 4 + b] = i < c0 && b < c1 ? s[i] * c[b] : 0.0f;
    z[ZS_ONE] = 1.0f;
#pragma unroll
    for (int r = 0; r < NOUT; r++)
        z[ZS_T + r] = __ldg(t + r);
#pragma unroll
    for (int q = ZS_T + NOUT; q < ZS_WIDTH; q++)
        z[q] = 0.0f;
}

}   // namespace nb
