// adjoint_cg.cu: the adjoint form's conjugate-gradient product for blocks (b) and (c'): (H + lambda I) p applied
// matrix-free, in FP32, from the decode's forward pass and its adjoint, with the inner products in FP64.
//
// H = sum over sites s of J_s^T diag(cw) J_s, where J_s maps the unknown latent to the site's decode: the bilinear
// sample of the unknown at the site's taps (weights w_sk), then the site's Jacobian G_s (block b: nout x C1,
// G = A + sum_i s_i M_i from level 0's sample s) or Q_s (block c': nout x C0, Q = B + sum_q c_q N_q from level 1's
// sample c). The stencil form (stencil.cu) stores H's 5 C x C blocks per texel in FP64; this form stores nothing but
// the site's sample of the other latent, which the assembly's site pass already keeps (4 floats per site):
//
//   pass 1, one thread per site:     u_s = G_s^T diag(cw) G_s (sum_k w_sk p_{t_k})              FP32, FMA
//   pass 2, one thread per texel t:  (H p)_t = sum_{sites s reaching t} w_st u_s + lambda p_t   FP64 sums
//                                    and the block's partial of p . H p, FP64
//
// Pass 2 gathers in a fixed site order (no atomics), so the product is deterministic; its partials feed the same
// alpha / beta kernels as the stencil form. The decoder rides as a launch parameter (constant-bank operands). The
// gradient, the diagonal blocks (the preconditioner and the ridge) come from the assembly's site pass and a gather of
// slot 0 alone.

#include "device.cuh"
#include "footprint.cuh"

namespace nb
{

constexpr int MF_SITE_THREADS = 256;

// The decoder in the 24-slot row layout [c_q (4)][s_i (4)][s_i c_q (4 x 4)], with the objective's weights.
struct MfDecoder
{
    float w[MAX_NOUT * 24];
    float cw[MAX_NOUT];
};

struct MfArgs
{
    const float4* y;                  // [site]: the site's sample of the other latent (the assembly's site pass)
    float* u;                         // [site][c]: pass 1's product
    const double* scalars;            // [plane][S_COUNT]
    long long site0[MAX_PLANES + 1];  // each plane's first site
};

template <bool LEVEL0, int NOUT>
__global__ void __launch_bounds__(MF_SITE_THREADS) k_mf_sites(Planes S, MfArgs A, MfDecoder W)
{
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(S, base);
    if (A.scalars[(size_t)pl * S_COUNT + S_ACTIVE] == 0.0)
        return;
    const PlaneView& V = S.p[pl];
    const int per = 1 + S.kc;
    const long long si = base - S.start[pl] + threadIdx.x;
    if (si >= (long long)V.w0 * V.h0 * per)
        return;
    const long long pixel = si / per;
    const int j = (int)(si % per);
    const int px = (int)(pixel % V.w0), py = (int)(pixel / V.w0);
    const int c = LEVEL0 ? S.c0 : S.c1;
    const int uw = LEVEL0 ? V.w0 : V.w1, uh = LEVEL0 ? V.h0 : V.h1;
    // forward: the unknown's sample of the direction at the site
    float dc[MAX_CH] = { 0.0f, 0.0f, 0.0f, 0.0f };
    if (LEVEL0 && j == 0)
    {
#pragma unroll
        for (int a = 0; a < MAX_CH; a++)
            if (a < c)
                dc[a] = (float)V.p[(size_t)pixel * c + a];
    }
    else
    {
        float dx, dy;
        site_offset(S.kc, j, px, py, dx, dy);
        const Tap t = tap_at(px, py, dx, dy, V.w0, V.h0, uw, uh);
        float wk[4];
        tap_weights(t, wk);
        const size_t q4[4] = { (size_t)t.y0 * uw + t.x0, (size_t)t.y0 * uw + t.x1, (size_t)t.y1 * uw + t.x0,
                               (size_t)t.y1 * uw + t.x1 };
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
            for (int a = 0; a < MAX_CH; a++)
                if (a < c)
                    dc[a] = __fmaf_rn(wk[k], (float)V.p[q4[k] * c + a], dc[a]);
    }
    const float4 y4 = A.y[A.site0[pl] + si];
    const float y[4] = { y4.x, y4.y, y4.z, y4.w };
    // the site's Jacobian row by row: dout_r = J_r . dc, then u += J_r^T cw_r dout_r
    float u[MAX_CH] = { 0.0f, 0.0f, 0.0f, 0.0f };
#pragma unroll
    for (int r = 0; r < NOUT; r++)
    {
        const float* wr = W.w + r * 24;
        float g[MAX_CH];
        float dout = 0.0f;
#pragma unroll
        for (int a = 0; a < MAX_CH; a++)
        {
            float ga = LEVEL0 ? wr[4 + a] : wr[a];
#pragma unroll
            for (int b = 0; b < MAX_CH; b++)
                ga = __fmaf_rn(y[b], LEVEL0 ? wr[8 + a * 4 + b] : wr[8 + b * 4 + a], ga);
            g[a] = a < c ? ga : 0.0f;
            dout = __fmaf_rn(g[a], dc[a], dout);
        }
        const float wd = W.cw[r] * dout;
#pragma unroll
        for (int a = 0; a < MAX_CH; a++)
            u[a] = __fmaf_rn(g[a], wd, u[a]);
    }
    float* out = A.u + (size_t)(A.site0[pl] + si) * c;
#pragma unroll
    for (int a = 0; a < MAX_CH; a++)
        if (a < c)
            out[a] = u[a];
}

__device__ __forceinline__ double mf_warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

template <bool LEVEL0>
__global__ void __launch_bounds__(THREADS) k_mf_gather(Planes P, MfArgs A, double* partial)
{
    __shared__ double sh[THREADS / 32];
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const double* s = A.scalars + (size_t)pl * S_COUNT;
    if (s[S_ACTIVE] == 0.0)
        return;   // the whole block: one plane per block
    const PlaneView& V = P.p[pl];
    const long long t = base - P.start[pl] + threadIdx.x;
    const int w = V.w, h = V.h, c = P.c, kc = P.kc, per = 1 + kc;
    double dot = 0.0;
    if (t < (long long)w * h)
    {
        const int tx = (int)(t % w), ty = (int)(t / w);
        int xl, xh, yl, yh;
        reach(tx, V.w0, w, xl, xh);
        reach(ty, V.h0, h, yl, yh);
        double acc[MAX_CH] = { 0.0, 0.0, 0.0, 0.0 };
        for (int py = yl; py <= yh; py++)
            for (int px = xl; px <= xh; px++)
                for (int j = 0; j < per; j++)
                {
                    float ws, wo;
                    if (!site_touches<LEVEL0>(px, py, j, kc, tx, ty, tx, ty, V.w0, V.h0, w, h, ws, wo))
                        continue;
                    const float* us = A.u + (size_t)(A.site0[pl] + ((long long)py * V.w0 + px) * per + j) * c;
#pragma unroll
                    for (int a = 0; a < MAX_CH; a++)
                        if (a < c)
                            acc[a] += (double)ws * (double)__ldg(us + a);
                }
        const double lambda = s[S_LAMBDA];
#pragma unroll
        for (int a = 0; a < MAX_CH; a++)
            if (a < c)
            {
                const size_t q = (size_t)t * c + a;
                const double pq = V.p[q];
                const double y = acc[a] + lambda * pq;
                V.ap[q] = y;
                dot += pq * y;
            }
    }
    dot = mf_warp_sum(dot);
    if ((threadIdx.x & 31) == 0)
        sh[threadIdx.x >> 5] = dot;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double sum = 0.0;
        for (int q = 0; q < THREADS / 32; q++)
            sum += sh[q];
        partial[blockIdx.x] = sum;
    }
}

// (H + lambda I) p of every active plane into ap, and the per-block partials of p . ap (row 0 of the reduction
// partials, one per THREADS texels): the matrix-free stand-in for the stencil product, same outputs, same shape.
int matvec_free(nntc_b200_device* d, const Planes& P, double* partial, int level0)
{
    Planes S = planes_for(d, level0, [&](int i) {
        const DevPlane& p = d->planes[(size_t)i];
        return (size_t)p.w0 * p.h0 * (size_t)(1 + P.kc);
    });
    S.kc = P.kc;
    MfArgs A{};
    A.y = (const float4*)d->site_y;
    A.u = reinterpret_cast<float*>(d->site_terms);   // the site terms are spent once the gather has run
    A.scalars = d->scalars;
    long long at = 0;
    for (int i = 0; i < S.n; i++)
    {
        A.site0[i] = at;
        at += (long long)d->planes[(size_t)i].w0 * d->planes[(size_t)i].h0 * (1 + P.kc);
    }
    A.site0[S.n] = at;
    MfDecoder W{};
    const int nin = d->nin, c0 = d->c0, c1 = d->c1;
    for (int r = 0; r < d->nout; r++)
    {
        for (int q = 0; q < c1; q++)
            W.w[r * 24 + q] = d->host_weights[(size_t)r * nin + q];
        for (int i = 0; i < c0; i++)
            W.w[r * 24 + 4 + i] = d->host_weights[(size_t)r * nin + c1 + i];
        for (int i = 0; i < c0; i++)
            for (int q = 0; q < c1; q++)
                W.w[r * 24 + 8 + i * 4 + q] = d->host_weights[(size_t)r * nin + c1 + c0 + i * c1 + q];
        W.cw[r] = d->m.cw[r];
    }
    const unsigned sblocks = (unsigned)(S.start[S.n] / MF_SITE_THREADS);
#define NB_MF(NO)                                                                                                     \
    case NO:                                                                                                          \
        if (level0)                                                                                                   \
            k_mf_sites<true, NO><<<sblocks, MF_SITE_THREADS, 0, d->stream>>>(S, A, W);                                \
        else                                                                                                          \
            k_mf_sites<false, NO><<<sblocks, MF_SITE_THREADS, 0, d->stream>>>(S, A, W);                               \
        break;
    switch (d->nout)
    {
        NB_MF(3)
        NB_MF(6)
        NB_MF(9)
        NB_MF(12)
        NB_MF(15)
        NB_MF(18)
    default:
        set_error(NNTC_B200_ERR_STATE, "a material holds 1..6 RGB textures");
        return NNTC_B200_ERR_STATE;
    }
#undef NB_MF
    NB_LAUNCHED();
    const unsigned tblocks = (unsigned)(P.start[P.n] / THREADS);
    if (level0)
        k_mf_gather<true><<<tblocks, THREADS, 0, d->stream>>>(P, A, partial);
    else
        k_mf_gather<false><<<tblocks, THREADS, 0, d->stream>>>(P, A, partial);
    NB_LAUNCHED();
    return NNTC_B200_OK;
}

}   // namespace nb
