// palette.cu: block (c) of --l0 palette, the exact per-texel palette search (src/solve_level0.cu), and the dense
// direct twin of block (b) behind --check (src/solve_level1.cu:1502-1688).
//
// Block (c): with level 1 and the decoder held and every other level-0 texel fixed, E is a C0-dimensional quadratic
// in one texel's values, E(x) = a0 + 2 x.a1 + x^T a2 x, gathered from the texel's own centre site and every fractional
// site of its 3x3 neighbourhood whose bilinear taps reach it; the texel takes the exact argmin over its palette
// states (a joint enumeration up to 8 bits in total, coordinate sweeps beyond), in four colour passes so that no two
// texels of a pass share a site. One thread per texel of the colour; every plane of the chain in one launch.

#include <cmath>
#include <cstring>
#include <vector>

#include "device.cuh"

namespace nb
{

constexpr int SEARCH_THREADS = 128;

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

__device__ __forceinline__ double search_energy(double a0, const double* a1, const double* a2, const float* x, int c0)
{
    double e = a0;
    for (int i = 0; i < c0; i++)
    {
        e += 2.0 * (double)x[i] * a1[i];
        for (int j = 0; j < c0; j++)
            e += (double)x[i] * (double)x[j] * a2[i * c0 + j];
    }
    return e;
}

__global__ void __launch_bounds__(SEARCH_THREADS) k_level0_search(Planes P, SearchArgs A)
{
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long ci = base - P.start[pl] + threadIdx.x;
    const int cw0 = (V.w0 - A.cx + 1) / 2, ch0 = (V.h0 - A.cy + 1) / 2;
    if (ci >= (long long)cw0 * ch0)
        return;
    const int c0 = P.c0, c1 = P.c1, nin = P.nin, nout = P.nout, kc = P.kc;
    const int w0 = V.w0, h0 = V.h0;
    const int tx = A.cx + 2 * (int)(ci % cw0);
    const int ty = A.cy + 2 * (int)(ci / cw0);
    const size_t t = (size_t)ty * w0 + tx;

    double a0 = 0.0, a1[MAX_CH], a2[MAX_CH * MAX_CH];
    for (int i = 0; i < c0; i++)
        a1[i] = 0.0;
    for (int i = 0; i < c0 * c0; i++)
        a2[i] = 0.0;
    for (int oy = -1; oy <= 1; oy++)
        for (int ox = -1; ox <= 1; ox++)
        {
            const int px = tx + ox, py = ty + oy;
            if (px < 0 || py < 0 || px >= w0 || py >= h0)
                continue;
            const int first = (ox == 0 && oy == 0) ? 0 : 1;
            for (int j = first; j <= kc; j++)
            {
                float dx, dy;
                site_offset(kc, j, px, py, dx, dy);
                float alpha = 0.0f, beta[MAX_CH], cbar[MAX_CH], target[MAX_NOUT];
                const Tap t1 = tap_at(px, py, dx, dy, w0, h0, V.w1, V.h1);
                blend<MAX_CH>(V.v1, V.w1, c1, t1, cbar);
                for (int i = 0; i < c0; i++)
                    beta[i] = 0.0f;
                if (j == 0)
                {
                    alpha = 1.0f;
                    for (int r = 0; r < nout; r++)
                        target[r] = V.src[t * nout + r];
                }
                else
                {
                    const Tap t0 = tap_at(px, py, dx, dy, w0, h0, w0, h0);
                    blend<MAX_NOUT>(V.src, w0, nout, t0, target);
                    const int qx[4] = { t0.x0, t0.x1, t0.x0, t0.x1 };
                    const int qy[4] = { t0.y0, t0.y0, t0.y1, t0.y1 };
                    float cwt[4];
                    tap_weights(t0, cwt);
                    for (int q = 0; q < 4; q++)
                    {
                        if (qx[q] == tx && qy[q] == ty)
                            alpha += cwt[q];
                        else
                        {
                            const float* nv = V.v0 + ((size_t)qy[q] * w0 + qx[q]) * c0;
                            for (int i = 0; i < c0; i++)
                                beta[i] += cwt[q] * nv[i];
                        }
                    }
                    if (!(alpha > 0.0f))
                        continue;
                }
                float qcol[MAX_NOUT * MAX_CH], resid[MAX_NOUT];
                for (int r = 0; r < nout; r++)
                {
                    const float* row = A.weights + (size_t)r * nin;
                    float out = A.bias[r];
                    for (int q = 0; q < c1; q++)
                        out += row[q] * cbar[q];
                    for (int i = 0; i < c0; i++)
                    {
                        float slope = row[c1 + i];
                        for (int q = 0; q < c1; q++)
                            slope += row[c1 + c0 + i * c1 + q] * cbar[q];
                        qcol[r * c0 + i] = slope;
                        out += slope * beta[i];
                    }
                    resid[r] = out - target[r];
                }
                for (int i = 0; i < nout; i++)
                    a0 += (double)A.cw[i] * (double)resid[i] * (double)resid[i];
                for (int i = 0; i < c0; i++)
                {
                    double g = 0.0;
                    for (int r = 0; r < nout; r++)
                        g += (double)A.cw[r] * (double)qcol[r * c0 + i] * (double)resid[r];
                    a1[i] += (double)alpha * g;
                    for (int j2 = 0; j2 < c0; j2++)
                    {
                        double s = 0.0;
                        for (int r = 0; r < nout; r++)
                            s += (double)A.cw[r] * (double)qcol[r * c0 + i] * (double)qcol[r * c0 + j2];
                        a2[i * c0 + j2] += (double)alpha * (double)alpha * s;
                    }
                }
            }
        }

    int cur[MAX_CH], best[MAX_CH], levels[MAX_CH];
    float x[MAX_CH];
    for (int i = 0; i < c0; i++)
    {
        levels[i] = (1 << A.bits[i]) - 1;
        cur[i] = (int)V.k0[t * c0 + i];
        best[i] = cur[i];
        x[i] = A.palette[(size_t)i * 16 + cur[i]];
    }
    double best_e = search_energy(a0, a1, a2, x, c0);
    if (A.joint)
    {
        long long total = 1;
        for (int i = 0; i < c0; i++)
            total *= (long long)(levels[i] + 1);
        for (long long n = 0; n < total; n++)
        {
            long long rest = n;
            bool same = true;
            int state[MAX_CH];
            for (int i = 0; i < c0; i++)
            {
                state[i] = (int)(rest % (long long)(levels[i] + 1));
                rest /= (long long)(levels[i] + 1);
                if (state[i] != cur[i])
                    same = false;
                x[i] = A.palette[(size_t)i * 16 + state[i]];
            }
            if (same)
                continue;
            const double e = search_energy(a0, a1, a2, x, c0);
            if (e < best_e)
            {
                best_e = e;
                for (int i = 0; i < c0; i++)
                    best[i] = state[i];
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
                    x[q] = A.palette[(size_t)q * 16 + best[q]];
                const int hold = best[i];
                for (int k = 0; k <= levels[i]; k++)
                {
                    if (k == best[i])
                        continue;
                    x[i] = A.palette[(size_t)i * 16 + k];
                    const double e = search_energy(a0, a1, a2, x, c0);
                    if (e < best_e)
                    {
                        best_e = e;
                        best[i] = k;
                    }
                }
                if (best[i] != hold)
                    changed = true;
            }
            if (!changed)
                break;
        }
    }
    bool moved_here = false;
    for (int i = 0; i < c0; i++)
        moved_here = moved_here || best[i] != cur[i];
    if (moved_here)
    {
        for (int i = 0; i < c0; i++)
        {
            V.v0[t * c0 + i] = A.palette[(size_t)i * 16 + best[i]];
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
        // the planes_for padding is in THREADS; the search uses SEARCH_THREADS, which divides it
        k_level0_search<<<(int)(P.start[P.n] / SEARCH_THREADS), SEARCH_THREADS, 0, d->stream>>>(P, A);
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

// The dense direct twin of block (b) on one small plane, on the host: the same H and gradient scattered into a dense
// matrix by a plain double loop over every site, then solved exactly (src/solve_level1.cu:1502-1688). Check-only.
int nntc_b200_solve_level1_dense_host(nntc_b200_device* d, const nntc_b200_model* m, int k, int plane, double lambda,
                                      const float* c_prev, size_t n_prev, double* delta, int max_unknowns)
{
    NB_TRY(check_plane(d, plane));
    const DevPlane& p = d->planes[(size_t)plane];
    const int w0 = p.w0, h0 = p.h0, w1 = p.w1, h1 = p.h1, c0 = m->c0, c1 = m->c1, nout = m->nout, nin = m->nin;
    const int nunk = w1 * h1 * c1;
    if (nunk > max_unknowns || n_prev < (size_t)nunk)
        return NNTC_B200_ERR_STATE;
    std::vector<float> v0((size_t)w0 * h0 * c0), src((size_t)w0 * h0 * nout);
    NB_TRY(download(d, v0.data(), p.v0, v0.size() * sizeof(float)));
    NB_TRY(download(d, src.data(), p.src, src.size() * sizeof(float)));
    std::vector<double> hm((size_t)nunk * nunk, 0.0), gv((size_t)nunk, 0.0);
    auto clampd = [](int i, int n) { return i < 0 ? 0 : (i > n - 1 ? n - 1 : i); };
    for (int py = 0; py < h0; py++)
        for (int px = 0; px < w0; px++)
            for (int j = 0; j <= k; j++)
            {
                double dx = 0.0, dy = 0.0;
                if (j > 0)
                {
                    float fx = 0.0f, fy = 0.0f;
                    subtexel(k, j - 1, px, py, fx, fy);
                    dx = fx;
                    dy = fy;
                }
                const double u = ((double)px + 0.5 + dx) / (double)w0;
                const double v = ((double)py + 0.5 + dy) / (double)h0;
                const double gx = u * (double)w1 - 0.5, gy = v * (double)h1 - 0.5;
                const int ix = (int)std::floor(gx), iy = (int)std::floor(gy);
                const double ax = gx - (double)ix, ay = gy - (double)iy;
                const int xs[2] = { clampd(ix, w1), clampd(ix + 1, w1) };
                const int ys[2] = { clampd(iy, h1), clampd(iy + 1, h1) };
                const double wx[2] = { 1.0 - ax, ax }, wy[2] = { 1.0 - ay, ay };
                int tid[4];
                double tws[4];
                int taps = 0;
                for (int b = 0; b < 2; b++)
                    for (int a = 0; a < 2; a++)
                    {
                        const int id = ys[b] * w1 + xs[a];
                        const double weight = wx[a] * wy[b];
                        int found = -1;
                        for (int e = 0; e < taps; e++)
                            if (tid[e] == id)
                                found = e;
                        if (found >= 0)
                            tws[found] += weight;
                        else
                        {
                            tid[taps] = id;
                            tws[taps] = weight;
                            taps++;
                        }
                    }
                double sbar[MAX_CH] = { 0, 0, 0, 0 }, cbar[MAX_CH] = { 0, 0, 0, 0 }, target[MAX_NOUT];
                for (int e = 0; e < taps; e++)
                    for (int q = 0; q < c1; q++)
                        cbar[q] += tws[e] * (double)c_prev[(size_t)tid[e] * c1 + q];
                if (j == 0)
                {
                    const size_t pi = (size_t)py * w0 + px;
                    for (int i = 0; i < c0; i++)
                        sbar[i] = v0[pi * c0 + i];
                    for (int r = 0; r < nout; r++)
                        target[r] = src[pi * nout + r];
                }
                else
                {
                    const double bx = u * (double)w0 - 0.5, by = v * (double)h0 - 0.5;
                    const int jx = (int)std::floor(bx), jy = (int)std::floor(by);
                    const double bfx = bx - (double)jx, bfy = by - (double)jy;
                    const int qx[2] = { clampd(jx, w0), clampd(jx + 1, w0) };
                    const int qy[2] = { clampd(jy, h0), clampd(jy + 1, h0) };
                    const double bwx[2] = { 1.0 - bfx, bfx }, bwy[2] = { 1.0 - bfy, bfy };
                    for (int r = 0; r < nout; r++)
                        target[r] = 0.0;
                    for (int b = 0; b < 2; b++)
                        for (int a = 0; a < 2; a++)
                        {
                            const size_t pi = (size_t)qy[b] * w0 + qx[a];
                            const double weight = bwx[a] * bwy[b];
                            for (int i = 0; i < c0; i++)
                                sbar[i] += weight * (double)v0[pi * c0 + i];
                            for (int r = 0; r < nout; r++)
                                target[r] += weight * (double)src[pi * nout + r];
                        }
                }
                std::vector<double> gmat((size_t)nout * c1), res((size_t)nout);
                for (int r = 0; r < nout; r++)
                {
                    const float* row = m->dec_w + (size_t)r * nin;
                    double out = (double)m->dec_b[r];
                    for (int i = 0; i < c0; i++)
                        out += (double)row[c1 + i] * sbar[i];
                    for (int q = 0; q < c1; q++)
                    {
                        double gg = (double)row[q];
                        for (int i = 0; i < c0; i++)
                            gg += sbar[i] * (double)row[c1 + c0 + i * c1 + q];
                        gmat[(size_t)r * c1 + q] = gg;
                        out += gg * cbar[q];
                    }
                    res[(size_t)r] = out - target[r];
                }
                for (int e = 0; e < taps; e++)
                {
                    for (int a = 0; a < c1; a++)
                    {
                        double ga = 0.0;
                        for (int r = 0; r < nout; r++)
                            ga += (double)m->cw[r] * gmat[(size_t)r * c1 + a] * res[(size_t)r];
                        gv[(size_t)tid[e] * c1 + a] += tws[e] * ga;
                    }
                    for (int f = 0; f < taps; f++)
                        for (int a = 0; a < c1; a++)
                            for (int b = 0; b < c1; b++)
                            {
                                double s = 0.0;
                                for (int r = 0; r < nout; r++)
                                    s += (double)m->cw[r] * gmat[(size_t)r * c1 + a] * gmat[(size_t)r * c1 + b];
                                hm[((size_t)tid[e] * c1 + a) * nunk + (size_t)tid[f] * c1 + b] += tws[e] * tws[f] * s;
                            }
                }
            }
    const int cols = nunk + 1;
    std::vector<double> aug((size_t)nunk * cols, 0.0);
    for (int i = 0; i < nunk; i++)
    {
        for (int j = 0; j < nunk; j++)
            aug[(size_t)i * cols + j] = hm[(size_t)i * nunk + j];
        aug[(size_t)i * cols + i] += lambda;
        aug[(size_t)i * cols + nunk] = -gv[(size_t)i];
    }
    for (int kk = 0; kk < nunk; kk++)
    {
        int pivot = kk;
        double best = std::fabs(aug[(size_t)kk * cols + kk]);
        for (int i = kk + 1; i < nunk; i++)
            if (std::fabs(aug[(size_t)i * cols + kk]) > best)
            {
                best = std::fabs(aug[(size_t)i * cols + kk]);
                pivot = i;
            }
        if (!(best > 0.0))
            return NNTC_B200_ERR_STATE;
        if (pivot != kk)
            for (int j = 0; j < cols; j++)
                std::swap(aug[(size_t)kk * cols + j], aug[(size_t)pivot * cols + j]);
        const double s = 1.0 / aug[(size_t)kk * cols + kk];
        for (int j = 0; j < cols; j++)
            aug[(size_t)kk * cols + j] *= s;
        for (int i = 0; i < nunk; i++)
        {
            if (i == kk)
                continue;
            const double f = aug[(size_t)i * cols + kk];
            if (f == 0.0)
                continue;
            for (int j = 0; j < cols; j++)
                aug[(size_t)i * cols + j] -= f * aug[(size_t)kk * cols + j];
        }
    }
    for (int i = 0; i < nunk; i++)
        delta[i] = aug[(size_t)i * cols + nunk];
    return NNTC_B200_OK;
}

}   // extern "C"
