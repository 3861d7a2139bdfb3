// palette.cu: block (c) of --l0 palette, the exact per-texel palette search (the method of src/solve_level0.cu), and
// the dense direct twin of block (b) that the reference's check harness compares the conjugate gradients against
// (the contract of src/solve_level1.cu:1502-1688).
//
// Block (c). With level 1, the decoder and every other level-0 texel held, E is a C0-dimensional quadratic in one
// texel's values x, E(x) = a0 + 2 x.a1 + x^T a2 x, collected from the texel's own centre site (level 0 read nearest,
// weight 1) and every fractional site of its 3x3 pixel neighbourhood whose bilinear taps reach it (weight alpha, the
// sum of the taps that land on the texel). The texel takes the exact argmin over its palette states: a joint
// enumeration when the channels' bits add up to at most 8, coordinate sweeps over each channel's alphabet beyond, a
// strict decrease to move. Four colour passes ((x & 1, y & 1) classes) make the texels of one pass independent.
//
// Shape on the B200: ONE WARP PER TEXEL. The texel's candidate sites (9 pixels x (K + 1) site slots, at most 45) are
// spread over the lanes, each lane forming its site's residual and slope columns and the site's contributions to the
// quadratic; the contributions are then folded one coefficient per lane, in site order, through shared memory; and the
// palette states (at most 256 in a joint enumeration, one channel's alphabet in a sweep) are spread over the lanes and
// reduced by a warp argmin whose tie rule (lowest energy, then first state in enumeration order, the current state
// before all) is the sequential scan's. The warp design keeps each lane's state to one site, where a thread-per-texel
// kernel carries the whole 37-site walk and a 256-state loop in one thread.
//
// What has to match the reference bit for bit, and why: the moved texels are bytes (level 0's indices), and a state's
// energy can tie another's to the last bit, so the float arithmetic of a site (sample, decode slope and residual, in
// the decode's own operation order), the double products of its contributions, the order in which sites are added
// into each coefficient, and the order of the terms of a state's energy are the method's (src/solve_level0.cu:62-73,
// 104-180). Everything else - which thread does what, how the work is split and reduced - is this file's.

#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "device.cuh"

namespace nb
{

constexpr int PS_WARPS = 2;                      // texels (warps) per block
constexpr int PS_CANDIDATES = 9 * 5;             // 3x3 pixels x (K + 1) site slots at K = 4
constexpr int PS_COEFFS = MAX_CH + MAX_CH * MAX_CH;   // a1 then a2, row-major

struct SearchArgs
{
    const float* weights;
    const float* bias;
    const float* cw;
    const float* palette;
    int bits[MAX_CH];
    int cx, cy, joint, sweeps;
    unsigned int* moved;   // [plane][4]
    int colour;
};

// One warp's staging: per candidate site, whether it contributes, its a0 terms (one per output, added one by one in
// output order) and its a1 / a2 contributions (alpha g_i, alpha^2 s_ij).
struct SearchStage
{
    double a0t[PS_CANDIDATES][MAX_NOUT];
    double coef[PS_CANDIDATES][PS_COEFFS];
    int live[PS_CANDIDATES];
    double q[1 + PS_COEFFS];   // the folded quadratic: a0, a1, a2
};

// The energy of a state x: a0, then channel by channel the linear term and the channel's row of the quadratic term.
__device__ __forceinline__ double state_energy(const double* q, const float* x, int c0)
{
    double e = q[0];
    for (int i = 0; i < c0; i++)
    {
        const double xi = (double)x[i];
        e += 2.0 * xi * q[1 + i];
        for (int j = 0; j < c0; j++)
            e += xi * (double)x[j] * q[1 + MAX_CH + i * MAX_CH + j];
    }
    return e;
}

// The warp's argmin of (energy, state index): lower energy first, then the lower index. Every lane returns the winner.
__device__ __forceinline__ void warp_argmin(double& e, int& n)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        const double oe = __shfl_xor_sync(0xffffffffu, e, off);
        const int on = __shfl_xor_sync(0xffffffffu, n, off);
        if (oe < e || (oe == e && on < n))
        {
            e = oe;
            n = on;
        }
    }
}

// Candidate `cand` of texel (tx, ty): pixel (tx + ox, ty + oy) with ox, oy in -1..1 and site slot j; only the texel's
// own pixel has a centre site (j = 0). Writes the candidate's staging row; `live` says whether it contributes.
__device__ void search_site(const Planes& P, const PlaneView& V, const SearchArgs& A, int tx, int ty, int cand,
                            SearchStage& S)
{
    const int c0 = P.c0, c1 = P.c1, nin = P.nin, nout = P.nout, kc = P.kc, w0 = V.w0, h0 = V.h0;
    const int slot = cand % (kc + 1), pix = cand / (kc + 1);
    const int px = tx + pix % 3 - 1, py = ty + pix / 3 - 1;
    const bool own = pix == 4;
    int live = pix < 9 && px >= 0 && py >= 0 && px < w0 && py < h0 && (slot > 0 || own);
    float alpha = 0.0f, beta[MAX_CH] = { 0.0f, 0.0f, 0.0f, 0.0f }, cbar[MAX_CH], target[MAX_NOUT];
    if (live)
    {
        float dx, dy;
        site_offset(kc, slot, px, py, dx, dy);
        blend<MAX_CH>(V.v1, V.w1, c1, tap_at(px, py, dx, dy, w0, h0, V.w1, V.h1), cbar);
        if (slot == 0)
        {
            // level 0 read nearest: the site's sample is the texel itself
            alpha = 1.0f;
            const float* s = V.src + ((size_t)ty * w0 + tx) * nout;
            for (int r = 0; r < nout; r++)
                target[r] = s[r];
        }
        else
        {
            const Tap t0 = tap_at(px, py, dx, dy, w0, h0, w0, h0);
            blend<MAX_NOUT>(V.src, w0, nout, t0, target);
            float wt[4];
            tap_weights(t0, wt);
            for (int q = 0; q < 4; q++)
            {
                const int qx = (q & 1) ? t0.x1 : t0.x0, qy = (q & 2) ? t0.y1 : t0.y0;
                if (qx == tx && qy == ty)
                    alpha += wt[q];   // a tap the clamp folded onto the texel adds its weight
                else
                {
                    const float* nv = V.v0 + ((size_t)qy * w0 + qx) * c0;
                    for (int i = 0; i < c0; i++)
                        beta[i] += wt[q] * nv[i];
                }
            }
            live = alpha > 0.0f;
        }
    }
    S.live[cand] = live;
    if (!live)
        return;
    // output by output: the decode's slope in each channel of the texel at this site (the s-columns of W plus the
    // sc-columns weighted by cbar), the decode with the texel at zero, the residual, and the double products
    double g[MAX_CH] = { 0.0, 0.0, 0.0, 0.0 }, s2[MAX_CH * MAX_CH];
    for (int e = 0; e < MAX_CH * MAX_CH; e++)
        s2[e] = 0.0;
    for (int r = 0; r < nout; r++)
    {
        const float* wr = A.weights + (size_t)r * nin;
        float dec = A.bias[r];
        for (int q = 0; q < c1; q++)
            dec += wr[q] * cbar[q];
        float slope[MAX_CH];
        for (int i = 0; i < c0; i++)
        {
            float sl = wr[c1 + i];
            for (int q = 0; q < c1; q++)
                sl += wr[c1 + c0 + i * c1 + q] * cbar[q];
            slope[i] = sl;
            dec += sl * beta[i];
        }
        const double res = (double)(dec - target[r]);
        const double wgt = (double)A.cw[r];
        S.a0t[cand][r] = wgt * res * res;
        for (int i = 0; i < c0; i++)
        {
            const double wq = wgt * (double)slope[i];
            g[i] += wq * res;
            for (int j = 0; j < c0; j++)
                s2[i * MAX_CH + j] += wq * (double)slope[j];
        }
    }
    const double al = (double)alpha;
    for (int i = 0; i < c0; i++)
    {
        S.coef[cand][i] = al * g[i];
        for (int j = 0; j < c0; j++)
            S.coef[cand][MAX_CH + i * MAX_CH + j] = al * al * s2[i * MAX_CH + j];
    }
}

__global__ void __launch_bounds__(32 * PS_WARPS) k_palette_search(Planes P, SearchArgs A)
{
    __shared__ SearchStage stage[PS_WARPS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    SearchStage& S = stage[wid];
    const long long item = (long long)blockIdx.x * PS_WARPS + wid;   // the texel of this pass, over every plane
    const int pl = plane_of(P, item);
    const PlaneView& V = P.p[pl];
    const long long ci = item - P.start[pl];
    const int cw0 = (V.w0 - A.cx + 1) / 2, ch0 = (V.h0 - A.cy + 1) / 2;
    if (ci >= (long long)cw0 * ch0)
        return;   // the whole warp leaves together
    const int c0 = P.c0;
    const int tx = A.cx + 2 * (int)(ci % cw0), ty = A.cy + 2 * (int)(ci / cw0);
    const size_t t = (size_t)ty * V.w0 + tx;
    const int ncand = 9 * (P.kc + 1);

    for (int cand = lane; cand < ncand; cand += 32)
        search_site(P, V, A, tx, ty, cand, S);
    __syncwarp();
    // the fold: one coefficient per lane over the live sites in order; the last lane walks a0's terms
    if (lane < PS_COEFFS)
    {
        const int i = lane < MAX_CH ? lane : (lane - MAX_CH) / MAX_CH, j = lane < MAX_CH ? 0 : (lane - MAX_CH) % MAX_CH;
        if (i < c0 && j < c0)
        {
            double acc = 0.0;
            for (int cand = 0; cand < ncand; cand++)
                if (S.live[cand])
                    acc += S.coef[cand][lane];
            S.q[1 + lane] = acc;
        }
    }
    else if (lane == 31)
    {
        double acc = 0.0;
        for (int cand = 0; cand < ncand; cand++)
            if (S.live[cand])
                for (int r = 0; r < P.nout; r++)
                    acc += S.a0t[cand][r];
        S.q[0] = acc;
    }
    __syncwarp();

    int levels[MAX_CH], cur[MAX_CH], best[MAX_CH];
    float x[MAX_CH];
    for (int i = 0; i < c0; i++)
    {
        levels[i] = (1 << A.bits[i]) - 1;
        cur[i] = best[i] = (int)V.k0[t * c0 + i];
        x[i] = A.palette[i * 16 + cur[i]];
    }
    double best_e = state_energy(S.q, x, c0);
    if (A.joint)
    {
        // mixed radix, channel 0 fastest; the current state stays unless something is strictly lower
        int total = 1, cur_n = 0, stride = 1;
        for (int i = 0; i < c0; i++)
        {
            cur_n += cur[i] * stride;
            stride *= levels[i] + 1;
        }
        total = stride;
        double e_min = DBL_MAX;
        int n_min = INT_MAX;
        for (int n = lane; n < total; n += 32)
        {
            if (n == cur_n)
                continue;
            int rest = n;
            for (int i = 0; i < c0; i++)
            {
                x[i] = A.palette[i * 16 + rest % (levels[i] + 1)];
                rest /= levels[i] + 1;
            }
            const double e = state_energy(S.q, x, c0);
            if (e < e_min)
            {
                e_min = e;
                n_min = n;
            }
        }
        warp_argmin(e_min, n_min);
        if (n_min != INT_MAX && e_min < best_e)
        {
            int rest = n_min;
            for (int i = 0; i < c0; i++)
            {
                best[i] = rest % (levels[i] + 1);
                rest /= levels[i] + 1;
            }
        }
    }
    else
    {
        for (int sw = 0; sw < A.sweeps; sw++)
        {
            bool changed = false;
            for (int i = 0; i < c0; i++)
            {
                for (int q = 0; q < c0; q++)
                    x[q] = A.palette[q * 16 + best[q]];
                double e_min = DBL_MAX;
                int k_min = INT_MAX;
                for (int k = lane; k <= levels[i]; k += 32)
                {
                    if (k == best[i])
                        continue;
                    x[i] = A.palette[i * 16 + k];
                    const double e = state_energy(S.q, x, c0);
                    if (e < e_min)
                    {
                        e_min = e;
                        k_min = k;
                    }
                }
                warp_argmin(e_min, k_min);
                if (k_min != INT_MAX && e_min < best_e)
                {
                    best_e = e_min;
                    best[i] = k_min;
                    changed = true;
                }
            }
            if (!changed)
                break;   // a sweep that moves nothing is followed by none that does
        }
    }
    bool moved = false;
    for (int i = 0; i < c0; i++)
        moved = moved || best[i] != cur[i];
    if (moved && lane == 0)
    {
        for (int i = 0; i < c0; i++)
        {
            V.v0[t * c0 + i] = A.palette[i * 16 + best[i]];
            V.k0[t * c0 + i] = (uint8_t)best[i];
        }
        atomicAdd(A.moved + pl * 4 + A.colour, 1u);
    }
}

}   // namespace nb

using namespace nb;

extern "C"
{

int nntc_b200_solve_level0_all(nntc_b200_device* d, const nntc_b200_model* m, int k, int sweeps,
                               nntc_b200_level0_report* rep, double* ms)
{
    if (k < 0 || k > 4 || k == 3)
    {
        set_error(NNTC_B200_ERR_ARG, "k must be 0, 1, 2 or 4");
        return NNTC_B200_ERR_ARG;
    }
    const int np = (int)d->planes.size();
    SearchArgs A{};
    A.weights = d->weights;
    A.bias = d->bias;
    A.cw = d->cw;
    A.palette = d->palette;
    long long states = 1;
    int total_bits = 0;
    for (int c = 0; c < d->c0; c++)
    {
        A.bits[c] = m->bits0[c];
        states *= (long long)1 << m->bits0[c];
        total_bits += m->bits0[c];
    }
    A.joint = total_bits <= 8 ? 1 : 0;
    A.sweeps = sweeps;
    A.moved = d->counters + CNT_SEARCH;   // [plane][4]
    NB_CUDA(cudaMemsetAsync(A.moved, 0, (size_t)MAX_PLANES * 4 * sizeof(unsigned int), d->stream));
    NB_TRY(block_begin(d));
    for (int colour = 0; colour < 4; colour++)
    {
        const int cx = colour & 1, cy = colour >> 1;
        Planes P = planes_for(d, 0, [&](int i) {
            const DevPlane& p = d->planes[(size_t)i];
            return (size_t)((p.w0 - cx + 1) / 2) * (size_t)((p.h0 - cy + 1) / 2);
        });
        P.kc = k;
        if (P.start[P.n] == 0)
            continue;
        A.cx = cx;
        A.cy = cy;
        A.colour = colour;
        // one warp per texel; planes_for pads each plane's range to THREADS texels, a multiple of PS_WARPS
        k_palette_search<<<(unsigned)(P.start[P.n] / PS_WARPS), 32 * PS_WARPS, 0, d->stream>>>(P, A);
        NB_LAUNCHED();
    }
    double t = 0.0;
    std::vector<unsigned int> moved((size_t)MAX_PLANES * 4);
    NB_CUDA(cudaMemcpyAsync(moved.data(), A.moved, moved.size() * sizeof(unsigned int), cudaMemcpyDeviceToHost,
                            d->stream));
    NB_TRY(block_end(d, &t));
    for (int i = 0; i < np; i++)
    {
        rep[i] = nntc_b200_level0_report{};
        rep[i].joint = A.joint;
        rep[i].states = states;
        rep[i].ms = t;
        for (int c = 0; c < 4; c++)
        {
            rep[i].moved[c] = moved[(size_t)i * 4 + c];
            rep[i].moved_total += rep[i].moved[c];
        }
    }
    if (ms)
        *ms = t;
    return NNTC_B200_OK;
}

// The dense direct twin of block (b) on one small plane, on the host, for the check harness: the Gauss-Newton system of
// level 1 built independently of the device path - every site's Jacobian rows formed explicitly in double (double
// u-space addressing, the two level-1 taps per axis merged by texel), H = sum_rows cw J^T J and g = sum_rows cw J^T res
// accumulated as outer products - and solved exactly, (H + lambda I) delta = -g, by a dense Cholesky factorisation.
// c_prev is level 1 as the caller holds it. Returns NNTC_B200_ERR_STATE when the plane has more than max_unknowns
// unknowns or H + lambda I is not positive definite.
int nntc_b200_solve_level1_dense_host(nntc_b200_device* d, const nntc_b200_model* m, int k, int plane, double lambda,
                                      const float* c_prev, size_t n_prev, double* delta, int max_unknowns)
{
    NB_TRY(check_plane(d, plane));
    const DevPlane& p = d->planes[(size_t)plane];
    const int w0 = p.w0, h0 = p.h0, w1 = p.w1, h1 = p.h1, c0 = m->c0, c1 = m->c1, nout = m->nout, nin = m->nin;
    const int n = w1 * h1 * c1;
    if (n > max_unknowns || n_prev < (size_t)n)
        return NNTC_B200_ERR_STATE;
    std::vector<float> v0((size_t)w0 * h0 * c0), src((size_t)w0 * h0 * nout);
    NB_TRY(download(d, v0.data(), p.v0, v0.size() * sizeof(float)));
    NB_TRY(download(d, src.data(), p.src, src.size() * sizeof(float)));
    std::vector<double> H((size_t)n * n, 0.0), g((size_t)n, 0.0);

    // The bilinear taps of a position in a w x h plane, in double, merged by texel: up to four (texel, weight) pairs.
    struct Taps
    {
        int n = 0;
        int id[4];
        double w[4];
        void add(int i, double wt)
        {
            for (int e = 0; e < n; e++)
                if (id[e] == i)
                {
                    w[e] += wt;
                    return;
                }
            id[n] = i;
            w[n++] = wt;
        }
    };
    auto taps_of = [](double u, double v, int w, int h) {
        const double gx = u * w - 0.5, gy = v * h - 0.5;
        const double fx = std::floor(gx), fy = std::floor(gy);
        const double ax = gx - fx, ay = gy - fy;
        auto cl = [](double i, int n) { return i < 0 ? 0 : (i > n - 1 ? n - 1 : (int)i); };
        Taps t;
        for (int b = 0; b < 2; b++)
            for (int a = 0; a < 2; a++)
                t.add(cl(fy + b, h) * w + cl(fx + a, w), (a ? ax : 1.0 - ax) * (b ? ay : 1.0 - ay));
        return t;
    };

    std::vector<double> row((size_t)MAX_NOUT * 4 * MAX_CH);   // per output: the Jacobian's entries, tap-major
    for (int py = 0; py < h0; py++)
        for (int px = 0; px < w0; px++)
            for (int j = 0; j <= k; j++)
            {
                float fdx = 0.0f, fdy = 0.0f;
                site_offset(k, j, px, py, fdx, fdy);
                const double u = ((double)px + 0.5 + fdx) / w0, v = ((double)py + 0.5 + fdy) / h0;
                const Taps t1 = taps_of(u, v, w1, h1);
                double c[MAX_CH] = { 0, 0, 0, 0 }, s[MAX_CH] = { 0, 0, 0, 0 }, tgt[MAX_NOUT] = {};
                for (int e = 0; e < t1.n; e++)
                    for (int q = 0; q < c1; q++)
                        c[q] += t1.w[e] * c_prev[(size_t)t1.id[e] * c1 + q];
                if (j == 0)
                {
                    const size_t pi = (size_t)py * w0 + px;
                    for (int i = 0; i < c0; i++)
                        s[i] = v0[pi * c0 + i];
                    for (int r = 0; r < nout; r++)
                        tgt[r] = src[pi * nout + r];
                }
                else
                {
                    const Taps t0 = taps_of(u, v, w0, h0);
                    for (int e = 0; e < t0.n; e++)
                    {
                        for (int i = 0; i < c0; i++)
                            s[i] += t0.w[e] * v0[(size_t)t0.id[e] * c0 + i];
                        for (int r = 0; r < nout; r++)
                            tgt[r] += t0.w[e] * src[(size_t)t0.id[e] * nout + r];
                    }
                }
                // output r is affine in c: out_r = b_r + W_s s + sum_q G_rq c_q, G_rq = W_c,q + sum_i s_i W_sc,iq
                for (int r = 0; r < nout; r++)
                {
                    const float* wr = m->dec_w + (size_t)r * nin;
                    double out = m->dec_b[r];
                    for (int i = 0; i < c0; i++)
                        out += wr[c1 + i] * s[i];
                    double G[MAX_CH];
                    for (int q = 0; q < c1; q++)
                    {
                        G[q] = wr[q];
                        for (int i = 0; i < c0; i++)
                            G[q] += s[i] * wr[c1 + c0 + i * c1 + q];
                        out += G[q] * c[q];
                    }
                    const double res = out - tgt[r], cw = m->cw[r];
                    // the Jacobian row of output r: d out_r / d c_q at tap e is w_e G_rq
                    for (int e = 0; e < t1.n; e++)
                        for (int q = 0; q < c1; q++)
                            row[(size_t)e * c1 + q] = t1.w[e] * G[q];
                    for (int e = 0; e < t1.n; e++)
                        for (int q = 0; q < c1; q++)
                        {
                            const size_t a = (size_t)t1.id[e] * c1 + q;
                            const double ja = row[(size_t)e * c1 + q];
                            g[a] += cw * ja * res;
                            for (int f = 0; f < t1.n; f++)
                                for (int q2 = 0; q2 < c1; q2++)
                                    H[a * n + (size_t)t1.id[f] * c1 + q2] += cw * ja * row[(size_t)f * c1 + q2];
                        }
                }
            }

    // (H + lambda I) = L L^T, then two triangular solves for -g
    for (int i = 0; i < n; i++)
        H[(size_t)i * n + i] += lambda;
    for (int c = 0; c < n; c++)
    {
        double piv = H[(size_t)c * n + c];
        for (int q = 0; q < c; q++)
            piv -= H[(size_t)c * n + q] * H[(size_t)c * n + q];
        if (!(piv > 0.0) || !std::isfinite(piv))
            return NNTC_B200_ERR_STATE;
        const double lcc = std::sqrt(piv);
        H[(size_t)c * n + c] = lcc;
        for (int r = c + 1; r < n; r++)
        {
            double v = H[(size_t)r * n + c];
            for (int q = 0; q < c; q++)
                v -= H[(size_t)r * n + q] * H[(size_t)c * n + q];
            H[(size_t)r * n + c] = v / lcc;
        }
    }
    for (int i = 0; i < n; i++)
    {
        double v = -g[(size_t)i];
        for (int q = 0; q < i; q++)
            v -= H[(size_t)i * n + q] * delta[q];
        delta[i] = v / H[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; i--)
    {
        double v = delta[i];
        for (int q = i + 1; q < n; q++)
            v -= H[(size_t)q * n + i] * delta[q];
        delta[i] = v / H[(size_t)i * n + i];
    }
    return NNTC_B200_OK;
}

}   // extern "C"
