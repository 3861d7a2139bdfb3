// adjoint.cu: the Gauss-Newton operator of block (b) applied matrix-free, from the decode and its adjoint.
//
// Block (b) minimises E over one plane's level-1 values v. At a site s the decode is out = W phi(s_bar, c) + b with
// c = sum_k w_k v[t_k] the bilinear sample of level 1 over the site's four taps, so the site's Jacobian with respect
// to c is G = A + sum_i s_bar_i M_i (nout x C1: A the decoder's columns of c, M_i those of s_i c) and the stencil the
// assembly builds is H = sum_sites (w w^T) kron (G^T diag(cw) G) (src/solve_level1.cu:259-438). This kernel applies
// H to a vector without assembling it: per site, the forward pass dc = sum_k w_k x[t_k] and dout = G dc, then the
// adjoint pass u = G^T diag(cw) dout scattered back as y[t_k] += w_k u - the fused forward/adjoint form of the same
// operator. Everything is FP64 from the float samples the assembly uses, so H x agrees with the assembled stencil's
// product to rounding (the scatter adds in hardware order). It is a check of the assembly, not a path of the encode.

#include "device.cuh"

namespace nb
{

struct JtjArgs
{
    const float* weights;   // nout x nin
    const float* cw;
    const double* x;        // plane texels x C1
    double* y;
};

__global__ void k_jtj_level1(PlaneView V, int c0, int c1, int nin, int nout, int kc, JtjArgs A)
{
    const long long si = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int per = 1 + kc;
    if (si >= (long long)V.w0 * V.h0 * per)
        return;
    const long long pixel = si / per;
    const int j = (int)(si % per);
    const int px = (int)(pixel % V.w0), py = (int)(pixel / V.w0);
    float dx, dy;
    site_offset(kc, j, px, py, dx, dy);
    // the site's sample of level 0, as the assembly takes it
    float sbar[MAX_CH];
    if (j == 0)
    {
        for (int i = 0; i < c0; i++)
            sbar[i] = V.v0[pixel * c0 + i];
    }
    else
    {
        const Tap t0 = tap_at(px, py, dx, dy, V.w0, V.h0, V.w0, V.h0);
        blend<MAX_CH>(V.v0, V.w0, c0, t0, sbar);
    }
    // the site's four taps on level 1 and their weights
    const Tap t1 = tap_at(px, py, dx, dy, V.w0, V.h0, V.w1, V.h1);
    float c4[4];
    tap_weights(t1, c4);
    const int tx[4] = { t1.x0, t1.x1, t1.x0, t1.x1 };
    const int ty[4] = { t1.y0, t1.y0, t1.y1, t1.y1 };
    // a texel two corners landed on (a clamped tap) weighs the float sum of their weights in corner order, as the
    // assembly merges them (src/solve_level1.cu:287-316); it is then visited once
    float w4[4] = { 0.0f, 0.0f, 0.0f, 0.0f };
    bool first[4];
    for (int k = 0; k < 4; k++)
    {
        int owner = k;
        for (int e = 0; e < k; e++)
            if (tx[e] == tx[k] && ty[e] == ty[k])
            {
                owner = e;
                break;
            }
        first[k] = owner == k;
        w4[owner] += c4[k];
    }
    // forward: dc = sum_k w_k x[t_k]
    double dc[MAX_CH] = { 0.0, 0.0, 0.0, 0.0 };
    for (int k = 0; k < 4; k++)
    {
        if (!first[k])
            continue;
        const double* xk = A.x + ((size_t)ty[k] * V.w1 + tx[k]) * c1;
        for (int q = 0; q < c1; q++)
            dc[q] += (double)w4[k] * xk[q];
    }
    // dout = G dc, then u = G^T diag(cw) dout
    double u[MAX_CH] = { 0.0, 0.0, 0.0, 0.0 };
    for (int r = 0; r < nout; r++)
    {
        const float* row = A.weights + (size_t)r * nin;
        double g[MAX_CH];
        double dout = 0.0;
        for (int q = 0; q < c1; q++)
        {
            double gq = (double)row[q];
            for (int i = 0; i < c0; i++)
                gq += (double)sbar[i] * (double)row[c1 + c0 + i * c1 + q];
            g[q] = gq;
            dout += gq * dc[q];
        }
        const double wd = (double)A.cw[r] * dout;
        for (int q = 0; q < c1; q++)
            u[q] += g[q] * wd;
    }
    // adjoint scatter: y[t_k] += w_k u
    for (int k = 0; k < 4; k++)
    {
        if (!first[k])
            continue;
        double* yk = A.y + ((size_t)ty[k] * V.w1 + tx[k]) * c1;
        for (int q = 0; q < c1; q++)
            atomicAdd(yk + q, (double)w4[k] * u[q]);
    }
}

}   // namespace nb

using namespace nb;

extern "C" int nntc_b200_probe_jtj_level1(nntc_b200_device* d, int k, int plane, const double* x, double* y, size_t n)
{
    NB_TRY(check_plane(d, plane));
    if (k < 0 || k > 4 || k == 3)
    {
        set_error(NNTC_B200_ERR_ARG, "k must be 0, 1, 2 or 4");
        return NNTC_B200_ERR_ARG;
    }
    DevPlane& p = d->planes[(size_t)plane];
    const size_t want = (size_t)p.w1 * p.h1 * d->c1;
    if (n < want)
    {
        set_error(NNTC_B200_ERR_ARG, "vector buffer too small");
        return NNTC_B200_ERR_ARG;
    }
    // the plane's CG direction and product vectors serve as the device copies of x and y
    Work& w = p.work[0];
    NB_TRY(upload(d, w.p, x, want * sizeof(double)));
    NB_CUDA(cudaMemsetAsync(w.ap, 0, want * sizeof(double), d->stream));
    PlaneView V{};
    V.w0 = p.w0;
    V.h0 = p.h0;
    V.w1 = p.w1;
    V.h1 = p.h1;
    V.src = p.src;
    V.v0 = p.v0;
    V.v1 = p.v1;
    const size_t sites = (size_t)p.w0 * p.h0 * (size_t)(1 + k);
    k_jtj_level1<<<grid_for(sites, 256), 256, 0, d->stream>>>(V, d->c0, d->c1, d->nin, d->nout, k,
                                                             JtjArgs{ d->weights, d->cw, w.p, w.ap });
    NB_LAUNCHED();
    return download(d, y, w.ap, want * sizeof(double));
}
