// adjoint.cu: the Gauss-Newton operators of blocks (b) and (c') applied matrix-free, from the decode and its adjoint.
//
// Block (b) minimises E over one plane's level-1 values v. At a site s the decode is out = W phi(s_bar, c) + b with
// c = sum_k w_k v[t_k] the bilinear sample of level 1 over the site's four taps, so the site's Jacobian with respect
// to c is G = A + sum_i s_bar_i M_i (nout x C1: A the decoder's columns of c, M_i those of s_i c) and the stencil the
// assembly builds is H = sum_sites (w w^T) kron (G^T diag(cw) G) (src/solve_level1.cu:259-438). This kernel applies
// H to a vector without assembling it: per site, the forward pass dc = sum_k w_k x[t_k] and dout = G dc, then the
// adjoint pass u = G^T diag(cw) dout scattered back as y[t_k] += w_k u - the fused forward/adjoint form of the same
// operator. Everything is FP64 from the float samples the assembly uses, so H x agrees with the assembled stencil's
// product to rounding (the scatter adds in hardware order). Block (c') is the same with the roles of the latents
// swapped. It is a check of the assembly, not a path of the encode.

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

// LEVEL0 = false: block (b), the unknown level 1 (taps on level 1, G from level 0's sample s).
// LEVEL0 = true: block (c'), the unknown level 0 (the centre site's own pixel with weight 1, the fractional sites'
// bilinear taps on level 0; Q = B + sum_q c_q N_q from level 1's sample c), src/solve_level1.cu:440-581.
template <bool LEVEL0>
__global__ void k_jtj(PlaneView V, int c0, int c1, int nin, int nout, int kc, JtjArgs A)
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
    const int c = LEVEL0 ? c0 : c1;          // the unknown's channels
    const int uw = LEVEL0 ? V.w0 : V.w1;     // the unknown's width
    // the other latent's sample at the site, as the assembly takes it
    float other[MAX_CH];
    if (LEVEL0)
    {
        const Tap t1 = tap_at(px, py, dx, dy, V.w0, V.h0, V.w1, V.h1);
        blend<MAX_CH>(V.v1, V.w1, c1, t1, other);
    }
    else if (j == 0)
    {
        for (int i = 0; i < c0; i++)
            other[i] = V.v0[pixel * c0 + i];
    }
    else
    {
        const Tap t0 = tap_at(px, py, dx, dy, V.w0, V.h0, V.w0, V.h0);
        blend<MAX_CH>(V.v0, V.w0, c0, t0, other);
    }
    // the site's taps on the unknown and their weights; a texel two corners landed on (a clamped tap) weighs the float
    // sum of their weights in corner order, as the assembly merges them (src/solve_level1.cu:287-316, 466-498)
    int tx[4], ty[4];
    float w4[4] = { 0.0f, 0.0f, 0.0f, 0.0f };
    bool first[4] = { true, false, false, false };
    if (LEVEL0 && j == 0)
    {
        tx[0] = px;
        ty[0] = py;
        w4[0] = 1.0f;
    }
    else
    {
        const Tap tq = LEVEL0 ? tap_at(px, py, dx, dy, V.w0, V.h0, V.w0, V.h0)
                              : tap_at(px, py, dx, dy, V.w0, V.h0, V.w1, V.h1);
        float c4[4];
        tap_weights(tq, c4);
        const int cx4[4] = { tq.x0, tq.x1, tq.x0, tq.x1 };
        const int cy4[4] = { tq.y0, tq.y0, tq.y1, tq.y1 };
        for (int k = 0; k < 4; k++)
        {
            tx[k] = cx4[k];
            ty[k] = cy4[k];
            int owner = k;
            for (int e = 0; e < k; e++)
                if (cx4[e] == cx4[k] && cy4[e] == cy4[k])
                {
                    owner = e;
                    break;
                }
            first[k] = owner == k;
            w4[owner] += c4[k];
        }
    }
    // forward: d = sum_k w_k x[t_k]
    double dc[MAX_CH] = { 0.0, 0.0, 0.0, 0.0 };
    for (int k = 0; k < 4; k++)
    {
        if (!first[k])
            continue;
        const double* xk = A.x + ((size_t)ty[k] * uw + tx[k]) * c;
        for (int q = 0; q < c; q++)
            dc[q] += (double)w4[k] * xk[q];
    }
    // dout = J_site d, then u = J_site^T diag(cw) dout; J_site's column a: level 1 (b): G[r][q] = W[r][q] +
    // sum_i s_i W[r][c1 + c0 + i c1 + q]; level 0 (c'): Q[r][i] = W[r][c1 + i] + sum_q c_q W[r][c1 + c0 + i c1 + q]
    double u[MAX_CH] = { 0.0, 0.0, 0.0, 0.0 };
    for (int r = 0; r < nout; r++)
    {
        const float* row = A.weights + (size_t)r * nin;
        double g[MAX_CH];
        double dout = 0.0;
        for (int a = 0; a < c; a++)
        {
            double ga = LEVEL0 ? (double)row[c1 + a] : (double)row[a];
            if (LEVEL0)
                for (int q = 0; q < c1; q++)
                    ga += (double)other[q] * (double)row[c1 + c0 + a * c1 + q];
            else
                for (int i = 0; i < c0; i++)
                    ga += (double)other[i] * (double)row[c1 + c0 + i * c1 + a];
            g[a] = ga;
            dout += ga * dc[a];
        }
        const double wd = (double)A.cw[r] * dout;
        for (int a = 0; a < c; a++)
            u[a] += g[a] * wd;
    }
    // adjoint scatter: y[t_k] += w_k u
    for (int k = 0; k < 4; k++)
    {
        if (!first[k])
            continue;
        double* yk = A.y + ((size_t)ty[k] * uw + tx[k]) * c;
        for (int q = 0; q < c; q++)
            atomicAdd(yk + q, (double)w4[k] * u[q]);
    }
}

}   // namespace nb

using namespace nb;

static int probe_jtj(nntc_b200_device* d, int level0, int k, int plane, const double* x, double* y, size_t n)
{
    NB_TRY(check_plane(d, plane));
    if (k < 0 || k > 4 || k == 3)
    {
        set_error(NNTC_B200_ERR_ARG, "k must be 0, 1, 2 or 4");
        return NNTC_B200_ERR_ARG;
    }
    if (level0 && !d->l0_bc8)
    {
        set_error(NNTC_B200_ERR_STATE, "block (c') runs only under --l0 bc8");
        return NNTC_B200_ERR_STATE;
    }
    DevPlane& p = d->planes[(size_t)plane];
    const size_t want = level0 ? (size_t)p.w0 * p.h0 * d->c0 : (size_t)p.w1 * p.h1 * d->c1;
    if (n < want)
    {
        set_error(NNTC_B200_ERR_ARG, "vector buffer too small");
        return NNTC_B200_ERR_ARG;
    }
    // the unknown's CG direction and product vectors serve as the device copies of x and y
    Work& w = p.work[level0 ? 1 : 0];
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
    const JtjArgs A{ d->weights, d->cw, w.p, w.ap };
    if (level0)
        k_jtj<true><<<grid_for(sites, 256), 256, 0, d->stream>>>(V, d->c0, d->c1, d->nin, d->nout, k, A);
    else
        k_jtj<false><<<grid_for(sites, 256), 256, 0, d->stream>>>(V, d->c0, d->c1, d->nin, d->nout, k, A);
    NB_LAUNCHED();
    return download(d, y, w.ap, want * sizeof(double));
}

extern "C" int nntc_b200_probe_jtj_level1(nntc_b200_device* d, int k, int plane, const double* x, double* y, size_t n)
{
    return probe_jtj(d, 0, k, plane, x, y, n);
}

extern "C" int nntc_b200_probe_jtj_level0(nntc_b200_device* d, int k, int plane, const double* x, double* y, size_t n)
{
    return probe_jtj(d, 1, k, plane, x, y, n);
}
