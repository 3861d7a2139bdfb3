// footprint.cuh: which sites of a plane reach a texel of the unknown latent, and with what weight - shared by the
// stencil assembly (assemble.cu) and the matrix-free operator of the adjoint form (adjoint_cg.cu).
#pragma once

#include "common.cuh"

namespace nb
{

// The pixels whose bilinear footprint into an n1-wide plane can reach texel ti (src/solve_level1.cu:246-257).
__host__ __device__ __forceinline__ void reach(int ti, int n0, int n1, int& lo, int& hi)
{
    const double r = (double)n0 / (double)n1;
    lo = (int)ceil(((double)ti - 0.5) * r - 1.0);
    hi = (int)ceil(((double)ti + 1.5) * r) - 1;
    lo = lo < 0 ? 0 : lo;
    hi = hi > n0 - 1 ? n0 - 1 : hi;
}

// Whether site (px, py, j) touches both texel (tx, ty) and texel (nbx, nby) of the unknown latent (w x h, its pixels
// w0 x h0), and with which weights. A merged tap's weight is the sum, in corner order, of the corner weights that
// landed on that texel (src/solve_level1.cu:287-316, 466-498): accumulating the corners of the self texel and of the
// neighbour from zero gives the same two weights.
template <bool LEVEL0>
__host__ __device__ __forceinline__ bool site_touches(int px, int py, int j, int kc, int tx, int ty, int nbx, int nby,
                                                      int w0, int h0, int w, int h, float& w_self, float& w_other)
{
    float dx, dy;
    site_offset(kc, j, px, py, dx, dy);
    w_self = 0.0f;
    w_other = 0.0f;
    bool has_self = false, has_other = false;
    if (LEVEL0 && j == 0)
    {
        has_self = px == tx && py == ty;
        has_other = px == nbx && py == nby;
        w_self = has_self ? 1.0f : 0.0f;
        w_other = has_other ? 1.0f : 0.0f;
    }
    else
    {
        const Tap tq = tap_at(px, py, dx, dy, w0, h0, w, h);
        float cw4[4];
        tap_weights(tq, cw4);
        const int cx4[4] = { tq.x0, tq.x1, tq.x0, tq.x1 };
        const int cy4[4] = { tq.y0, tq.y0, tq.y1, tq.y1 };
#pragma unroll
        for (int q = 0; q < 4; q++)
        {
            if (cx4[q] == tx && cy4[q] == ty)
            {
                w_self += cw4[q];
                has_self = true;
            }
            if (cx4[q] == nbx && cy4[q] == nby)
            {
                w_other += cw4[q];
                has_other = true;
            }
        }
    }
    return has_self && has_other;
}

}   // namespace nb
