// init.cu: the initial state of both latents and their grids (src/init.cu:384-1400).
//
// - level 0: luma into channel 0 snapped to the palette, or continuous under --l0 bc8 (src/init.cu:389-482);
// - level 1: the block mean of the source per level-1 texel, by source channel (box) or projected onto the base
//   plane's principal directions (pca), fitted onto one min/max grid over the whole chain (src/init.cu:484-967);
// - --init0 residual: one level-0 channel from the leading principal direction of the decode's residual, divided by
//   its peak (bc8) or its 99th percentile (palette) over the chain (src/init.cu:969-1400);
// - the grid fits: minmax or the 0.1 / 99.9 percentiles over every plane of the chain, then the snap onto the grid
//   through the one definition of the grid value (src/init.cu:520-750).
//
// The per-element kernels are the reference's arithmetic; the covariance sums are fixed-order two-stage reductions;
// the eigenproblems, the sorts of the percentile fit and the histogram walk are small host work, as in the reference.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "device.cuh"

namespace nb
{


struct ChannelBits
{
    int b[MAX_CH];
};

__global__ void k_init_level0(const float* src, int w, int h, int nout, int c0, ChannelBits bits, const float* palette,
                              float lr, float lg, float lb, int luma_channel0, float* v0, uint8_t* k0)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)w * h)
        return;
    const float* s = src + i * nout;
    const float luma = lr * s[0] + lg * s[1] + lb * s[2];
    for (int c = 0; c < c0; c++)
    {
        const float value = (c == 0 && luma_channel0) ? 2.0f * luma - 1.0f : 0.0f;
        const int levels = (1 << bits.b[c]) - 1;
        int k = 0;
        float best = fabsf(palette[(size_t)c * 16] - value);
        for (int j = 1; j <= levels; j++)
        {
            const float dist = fabsf(palette[(size_t)c * 16 + j] - value);
            if (dist < best)
            {
                best = dist;
                k = j;
            }
        }
        v0[i * c0 + c] = palette[(size_t)c * 16 + k];
        k0[i * c0 + c] = (uint8_t)k;
    }
}

__global__ void k_init_level0_cont(const float* src, int w, int h, int nout, int c0, float lr, float lg, float lb,
                                   int luma_channel0, float* v0)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)w * h)
        return;
    const float* s = src + i * nout;
    const float luma = lr * s[0] + lg * s[1] + lb * s[2];
    for (int c = 0; c < c0; c++)
        v0[i * c0 + c] = (c == 0 && luma_channel0) ? 2.0f * luma - 1.0f : 0.0f;
}

// The footprint of level-1 texel (x, y): source pixels [x w0 / w1, (x + 1) w0 / w1) and the same in y.
__device__ __forceinline__ void block_span(int x, int w0, int w1, int& a, int& b)
{
    a = (int)((long long)x * w0 / w1);
    b = (int)((long long)(x + 1) * w0 / w1);
    if (b <= a)
        b = a + 1;
    b = b > w0 ? w0 : b;
}

__global__ void k_init_level1_box(const float* src, int w0, int h0, int nout, int w1, int h1, int c1, float* out)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)w1 * h1)
        return;
    const int x = (int)(i % (size_t)w1), y = (int)(i / (size_t)w1);
    int xa, xb, ya, yb;
    block_span(x, w0, w1, xa, xb);
    block_span(y, h0, h1, ya, yb);
    float acc[MAX_CH];
    for (int c = 0; c < c1; c++)
        acc[c] = 0.0f;
    int n = 0;
    for (int sy = ya; sy < yb; sy++)
        for (int sx = xa; sx < xb; sx++)
        {
            const float* s = src + ((size_t)sy * w0 + sx) * nout;
            for (int c = 0; c < c1; c++)
                acc[c] += c < nout ? s[c] : 0.0f;
            n++;
        }
    const float inv = n > 0 ? 1.0f / (float)n : 0.0f;
    for (int c = 0; c < c1; c++)
        out[i * c1 + c] = c < nout ? 2.0f * acc[c] * inv - 1.0f : 0.0f;
}

__global__ void k_block_means(const float* src, int w0, int h0, int nout, int w1, int h1, float* means)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)w1 * h1)
        return;
    const int x = (int)(i % (size_t)w1), y = (int)(i / (size_t)w1);
    int xa, xb, ya, yb;
    block_span(x, w0, w1, xa, xb);
    block_span(y, h0, h1, ya, yb);
    float acc[MAX_NOUT];
    for (int c = 0; c < nout; c++)
        acc[c] = 0.0f;
    int n = 0;
    for (int sy = ya; sy < yb; sy++)
        for (int sx = xa; sx < xb; sx++)
        {
            const float* s = src + ((size_t)sy * w0 + sx) * nout;
            for (int c = 0; c < nout; c++)
                acc[c] += s[c];
            n++;
        }
    const float inv = n > 0 ? 1.0f / (float)n : 0.0f;
    for (int c = 0; c < nout; c++)
        means[i * (size_t)nout + c] = acc[c] * inv;
}

// Entry e < nout: the sum of channel e; entry nout + r nout + s: the sum of channel r times channel s. Block
// (b, r) makes the partial b of the entries of channel r - its sum and its nout products - from ONE read of each row:
// every entry's sum runs over the same texels in the same grid-stride order as one block per entry would, and is
// folded by the same tree, so the partials do not depend on how entries share a block.
__global__ void k_cov_partial(const float* v, size_t count, int nout, double* cov)
{
    __shared__ double sh[256];
    const int r = (int)blockIdx.y;
    double acc[1 + MAX_NOUT];
#pragma unroll
    for (int q = 0; q <= MAX_NOUT; q++)
        acc[q] = 0.0;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < count; t += (size_t)gridDim.x * blockDim.x)
    {
        const float* row = v + t * (size_t)nout;
        const double a = (double)row[r];
        acc[0] += a;
#pragma unroll
        for (int q = 0; q < MAX_NOUT; q++)
            if (q < nout)
                acc[1 + q] += a * (double)row[q];
    }
#pragma unroll
    for (int q = 0; q <= MAX_NOUT; q++)
    {
        if (q > nout)
            break;
        __syncthreads();
        sh[threadIdx.x] = acc[q];
        __syncthreads();
        for (int half = (int)blockDim.x / 2; half > 0; half >>= 1)
        {
            if ((int)threadIdx.x < half)
                sh[threadIdx.x] += sh[threadIdx.x + half];
            __syncthreads();
        }
        if (threadIdx.x == 0)
        {
            const int e = q == 0 ? r : nout + r * nout + (q - 1);
            cov[(size_t)e * COV_GRID + blockIdx.x] = sh[0];
        }
    }
}

__global__ void k_quantise(const float* in, size_t n, int c, int bits, const float* lo, const float* hi, float* v,
                           uint8_t* k)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int ch = (int)(i % (size_t)c);
    const int kk = grid_index(lo[ch], hi[ch], bits, in[i]);
    v[i] = grid_value(lo[ch], hi[ch], bits, kk);
    k[i] = (uint8_t)kk;
}

__global__ void k_residual(const float* v0, const float* v1, const float* src, int w0, int h0, int w1, int h1, int c0,
                           int c1, int nin, int nout, const float* weights, const float* bias, float* resid)
{
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)w0 * h0)
        return;
    const int px = (int)(idx % (size_t)w0), py = (int)(idx / (size_t)w0);
    float s[MAX_CH], c[MAX_CH], phi[MAX_NIN];
    for (int i = 0; i < c0; i++)
        s[i] = v0[idx * c0 + i];
    const Tap t = tap_at(px, py, 0.0f, 0.0f, w0, h0, w1, h1);
    blend<MAX_CH>(v1, w1, c1, t, c);
    features(s, c0, c, c1, phi);
    for (int r = 0; r < nout; r++)
    {
        float acc = bias[r];
        const float* row = weights + (size_t)r * nin;
        for (int i = 0; i < nin; i++)
            acc += row[i] * phi[i];
        resid[idx * (size_t)nout + r] = acc - src[idx * (size_t)nout + r];
    }
}

struct ProjDir
{
    double e[MAX_NOUT];
    double mu[MAX_NOUT];
};

__device__ __forceinline__ double proj_value(const float* resid, size_t t, int nout, const ProjDir& dir)
{
    double acc = 0.0;
    for (int r = 0; r < nout; r++)
        acc += dir.e[r] * ((double)resid[t * (size_t)nout + r] - dir.mu[r]);
    return acc;
}

__global__ void k_proj_peak(const float* resid, size_t texels, int nout, ProjDir dir, double* partial)
{
    __shared__ double sh[256];
    double acc = 0.0;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < texels; t += (size_t)gridDim.x * blockDim.x)
    {
        const double v = fabs(proj_value(resid, t, nout, dir));
        acc = v > acc ? v : acc;
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int half = (int)blockDim.x / 2; half > 0; half >>= 1)
    {
        if ((int)threadIdx.x < half)
            sh[threadIdx.x] = sh[threadIdx.x] > sh[threadIdx.x + half] ? sh[threadIdx.x] : sh[threadIdx.x + half];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        partial[blockIdx.x] = sh[0];
}

__global__ void k_proj_hist(const float* resid, size_t texels, int nout, ProjDir dir, double inv_peak, int bins,
                            unsigned long long* hist)
{
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < texels; t += (size_t)gridDim.x * blockDim.x)
    {
        const double v = fabs(proj_value(resid, t, nout, dir)) * inv_peak;
        int b = (int)(v * (double)bins);
        b = b < 0 ? 0 : (b >= bins ? bins - 1 : b);
        atomicAdd(hist + b, 1ull);
    }
}

__global__ void k_seed_channel(const float* resid, size_t texels, int nout, ProjDir dir, double inv, int c0,
                               int channel, int levels, const float* palette, int palette_mode, float* v0, uint8_t* k0)
{
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= texels)
        return;
    const double p = proj_value(resid, t, nout, dir) * inv;
    const float value = (float)(p < -1.0 ? -1.0 : (p > 1.0 ? 1.0 : p));
    if (palette_mode)
    {
        int k = (int)lroundf((value + 1.0f) * 0.5f * (float)levels);
        k = k < 0 ? 0 : (k > levels ? levels : k);
        v0[t * (size_t)c0 + channel] = palette[(size_t)channel * 16 + k];
        k0[t * (size_t)c0 + channel] = (uint8_t)k;
    }
    else
        v0[t * (size_t)c0 + channel] = value;
}

// ---- host helpers -------------------------------------------------------------------------------------------------

static void fit_range(const std::vector<std::vector<float>>& cont, int nc, bool pct, std::vector<float>& lo,
                      std::vector<float>& hi)
{
    lo.assign((size_t)nc, 1e30f);
    hi.assign((size_t)nc, -1e30f);
    if (!pct)
    {
        for (size_t i = 0; i < cont.size(); i++)
            for (size_t t = 0; t < cont[i].size(); t++)
            {
                const int c = (int)(t % (size_t)nc);
                lo[(size_t)c] = std::min(lo[(size_t)c], cont[i][t]);
                hi[(size_t)c] = std::max(hi[(size_t)c], cont[i][t]);
            }
        return;
    }
    std::vector<float> v;
    for (int c = 0; c < nc; c++)
    {
        v.clear();
        for (size_t i = 0; i < cont.size(); i++)
            for (size_t t = (size_t)c; t < cont[i].size(); t += (size_t)nc)
                v.push_back(cont[i][t]);
        if (v.empty())
            continue;
        const size_t last = v.size() - 1;
        const size_t a = (size_t)(0.001 * (double)last + 0.5);
        const size_t b = (size_t)(0.999 * (double)last + 0.5);
        // the two order statistics of the sorted values, by selection
        std::nth_element(v.begin(), v.begin() + (long)a, v.end());
        lo[(size_t)c] = v[a];
        std::nth_element(v.begin(), v.begin() + (long)b, v.end());
        hi[(size_t)c] = v[b];
    }
}

static void jacobi_eigen(std::vector<double>& a, int n, std::vector<double>& vec, std::vector<double>& val)
{
    vec.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++)
        vec[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; sweep++)
    {
        double off = 0.0;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++)
                off += a[(size_t)p * n + q] * a[(size_t)p * n + q];
        if (off <= 1e-30)
            break;
        for (int p = 0; p < n; p++)
            for (int q = p + 1; q < n; q++)
            {
                const double apq = a[(size_t)p * n + q];
                if (std::fabs(apq) <= 1e-300)
                    continue;
                const double theta = (a[(size_t)q * n + q] - a[(size_t)p * n + p]) / (2.0 * apq);
                const double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; k++)
                {
                    const double akp = a[(size_t)k * n + p], akq = a[(size_t)k * n + q];
                    a[(size_t)k * n + p] = c * akp - s * akq;
                    a[(size_t)k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; k++)
                {
                    const double apk = a[(size_t)p * n + k], aqk = a[(size_t)q * n + k];
                    a[(size_t)p * n + k] = c * apk - s * aqk;
                    a[(size_t)q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; k++)
                {
                    const double vkp = vec[(size_t)k * n + p], vkq = vec[(size_t)k * n + q];
                    vec[(size_t)k * n + p] = c * vkp - s * vkq;
                    vec[(size_t)k * n + q] = s * vkp + c * vkq;
                }
            }
    }
    val.assign((size_t)n, 0.0);
    for (int i = 0; i < n; i++)
        val[(size_t)i] = a[(size_t)i * n + i];
}

// The covariance sums of `count` rows of nout floats on the device, added on the host in block order.
static int cov_sums(nntc_b200_device* d, const float* rows, size_t count, int nout, std::vector<double>& raw)
{
    const int entries = nout + nout * nout;
    dim3 grid((unsigned)COV_GRID, (unsigned)nout);
    k_cov_partial<<<grid, 256, 0, d->stream>>>(rows, count, nout, d->cov);
    NB_LAUNCHED();
    std::vector<double> partial((size_t)entries * COV_GRID);
    NB_TRY(download(d, partial.data(), d->cov, partial.size() * sizeof(double)));
    raw.assign((size_t)entries, 0.0);
    for (int e = 0; e < entries; e++)
        for (int b = 0; b < COV_GRID; b++)
            raw[(size_t)e] += partial[(size_t)e * COV_GRID + b];
    return NNTC_B200_OK;
}

int fit_grid_device(nntc_b200_device* d, int level0, bool pct, float* lo, float* hi);

// Fit the grid (when `fit`) and snap every plane onto it. With `cont` empty both read the planes where the device holds
// them; with a host copy (the pca init's projections) the fit is the host's and the snap reads the copy.
static int fit_and_snap(nntc_b200_device* d, nntc_b200_model* m, int level0,
                        const std::vector<std::vector<float>>& cont, bool pct, uint8_t* const* k_out, bool fit)
{
    const int nc = level0 ? d->c0 : d->c1;
    if (fit)
    {
        std::vector<float> lo(MAX_CH), hi(MAX_CH);
        if (cont.empty())
            NB_TRY(fit_grid_device(d, level0, pct, lo.data(), hi.data()));   // the planes as the device holds them
        else
            fit_range(cont, nc, pct, lo, hi);
        for (int c = 0; c < nc; c++)
            if (!(hi[(size_t)c] > lo[(size_t)c]))
            {
                lo[(size_t)c] = -1.0f;
                hi[(size_t)c] = 1.0f;
            }
        for (int c = 0; c < nc; c++)
        {
            if (level0)
            {
                m->lo0[c] = lo[(size_t)c];
                m->hi0[c] = hi[(size_t)c];
            }
            else
            {
                m->lo1[c] = lo[(size_t)c];
                m->hi1[c] = hi[(size_t)c];
            }
        }
        if (level0)
            m->has_lo0 = 1;
        else
            m->has_lo1 = 1;
        NB_TRY(upload_grids(d, m));
    }
    for (size_t i = 0; i < d->planes.size(); i++)
    {
        const DevPlane& p = d->planes[i];
        const size_t n = level0 ? (size_t)p.w0 * p.h0 * d->c0 : (size_t)p.w1 * p.h1 * d->c1;
        float* v = level0 ? p.v0 : p.v1;
        uint8_t* k = level0 ? p.k0 : p.k1;
        const float* in = v;   // snap in place (each thread reads and writes one value)
        if (!cont.empty())
        {
            NB_TRY(upload(d, d->scratch, cont[i].data(), n * sizeof(float)));
            in = d->scratch;
        }
        k_quantise<<<grid_for(n, 256), 256, 0, d->stream>>>(in, n, nc, level0 ? 8 : m->bits1, level0 ? d->lo0 : d->lo1,
                                                           level0 ? d->hi0 : d->hi1, v, k);
        NB_LAUNCHED();
        if (k_out && k_out[i])
            NB_TRY(download(d, k_out[i], k, n));
    }
    NB_CUDA(cudaStreamSynchronize(d->stream));
    return NNTC_B200_OK;
}

static int residual_pass(nntc_b200_device* d, size_t plane)
{
    const DevPlane& p = d->planes[plane];
    const size_t n = (size_t)p.w0 * p.h0;
    k_residual<<<grid_for(n, 256), 256, 0, d->stream>>>(p.v0, p.v1, p.src, p.w0, p.h0, p.w1, p.h1, d->c0, d->c1,
                                                       d->nin, d->nout, d->weights, d->bias, d->resid);
    NB_LAUNCHED();
    return NNTC_B200_OK;
}

}   // namespace nb

using namespace nb;

extern "C"
{

int nntc_b200_init_level0(nntc_b200_device* d, const nntc_b200_model* m, const float luma[3], int luma_channel0,
                          uint8_t* const* k0_out)
{
    NB_TRY(upload_grids(d, m));
    ChannelBits bits{};
    for (int c = 0; c < d->c0; c++)
        bits.b[c] = m->bits0[c];
    for (size_t i = 0; i < d->planes.size(); i++)
    {
        const DevPlane& p = d->planes[i];
        const size_t n = (size_t)p.w0 * p.h0;
        if (m->l0_bc8)
        {
            k_init_level0_cont<<<grid_for(n, 256), 256, 0, d->stream>>>(p.src, p.w0, p.h0, d->nout, d->c0, luma[0],
                                                                        luma[1], luma[2], luma_channel0 ? 1 : 0,
                                                                        p.v0);
            NB_LAUNCHED();
            NB_CUDA(cudaMemsetAsync(p.k0, 0, n * d->c0, d->stream));
            if (k0_out && k0_out[i])
                std::memset(k0_out[i], 0, n * d->c0);
        }
        else
        {
            k_init_level0<<<grid_for(n, 256), 256, 0, d->stream>>>(p.src, p.w0, p.h0, d->nout, d->c0, bits,
                                                                   d->palette, luma[0], luma[1], luma[2],
                                                                   luma_channel0 ? 1 : 0, p.v0, p.k0);
            NB_LAUNCHED();
            if (k0_out && k0_out[i])
                NB_TRY(download(d, k0_out[i], p.k0, n * d->c0));
        }
    }
    NB_CUDA(cudaStreamSynchronize(d->stream));
    return NNTC_B200_OK;
}

int nntc_b200_init_level1(nntc_b200_device* d, nntc_b200_model* m, int pca, nntc_b200_init1_report* rep,
                          uint8_t* const* k1_out)
{
    *rep = nntc_b200_init1_report{};
    rep->pca = pca;
    std::vector<std::vector<float>> cont(d->planes.size());
    const int c1 = d->c1, nout = d->nout;
    if (!pca)
    {
        for (size_t i = 0; i < d->planes.size(); i++)
        {
            const DevPlane& p = d->planes[i];
            const size_t n = (size_t)p.w1 * p.h1;
            k_init_level1_box<<<grid_for(n, 256), 256, 0, d->stream>>>(p.src, p.w0, p.h0, nout, p.w1, p.h1, c1, p.v1);
            NB_LAUNCHED();
        }
        const std::vector<std::vector<float>> on_device;
        return fit_and_snap(d, m, 0, on_device, false, k1_out, true);
    }
    // The basis: the base plane's block means, their covariance, the host eigenproblem.
    std::vector<double> raw;
    {
        const DevPlane& p = d->planes[0];
        const size_t texels = (size_t)p.w1 * p.h1;
        k_block_means<<<grid_for(texels, 256), 256, 0, d->stream>>>(p.src, p.w0, p.h0, nout, p.w1, p.h1, d->means);
        NB_LAUNCHED();
        NB_TRY(cov_sums(d, d->means, texels, nout, raw));
    }
    const DevPlane& base = d->planes[0];
    const double count = (double)((size_t)base.w1 * base.h1);
    std::vector<double> mu((size_t)nout, 0.0), cov((size_t)nout * nout, 0.0);
    for (int r = 0; r < nout; r++)
        mu[(size_t)r] = count > 0.0 ? raw[(size_t)r] / count : 0.0;
    for (int r = 0; r < nout; r++)
        for (int s = 0; s < nout; s++)
            cov[(size_t)r * nout + s] =
                (count > 0.0 ? raw[(size_t)(nout + r * nout + s)] / count : 0.0) - mu[(size_t)r] * mu[(size_t)s];
    for (int r = 0; r < nout; r++)
        rep->total_variance += cov[(size_t)r * nout + r];
    std::vector<double> work = cov, vec, val;
    jacobi_eigen(work, nout, vec, val);
    std::vector<int> order((size_t)nout);
    for (int i = 0; i < nout; i++)
        order[(size_t)i] = i;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return val[(size_t)a] > val[(size_t)b]; });
    rep->components = c1 < nout ? c1 : nout;
    for (int j = 0; j < rep->components && j < MAX_CH; j++)
        rep->eigenvalue[j] = val[(size_t)order[(size_t)j]];
    std::vector<float> means;
    std::vector<double> peak((size_t)c1, 0.0);
    for (size_t i = 0; i < d->planes.size(); i++)
    {
        const DevPlane& p = d->planes[i];
        const size_t texels = (size_t)p.w1 * p.h1;
        k_block_means<<<grid_for(texels, 256), 256, 0, d->stream>>>(p.src, p.w0, p.h0, nout, p.w1, p.h1, d->means);
        NB_LAUNCHED();
        means.resize(texels * (size_t)nout);
        NB_TRY(download(d, means.data(), d->means, means.size() * sizeof(float)));
        cont[i].assign(texels * (size_t)c1, 0.0f);
        for (size_t t = 0; t < texels; t++)
            for (int j = 0; j < rep->components; j++)
            {
                const int col = order[(size_t)j];
                double acc = 0.0;
                for (int r = 0; r < nout; r++)
                    acc += vec[(size_t)r * nout + col] * ((double)means[t * (size_t)nout + r] - mu[(size_t)r]);
                cont[i][t * (size_t)c1 + j] = (float)acc;
                peak[(size_t)j] = std::max(peak[(size_t)j], std::fabs(acc));
            }
    }
    for (int j = 0; j < c1; j++)
    {
        rep->peak[j] = peak[(size_t)j];
        if (!(peak[(size_t)j] > 0.0))
            continue;
        const double inv = 1.0 / peak[(size_t)j];
        for (size_t i = 0; i < cont.size(); i++)
            for (size_t t = (size_t)j; t < cont[i].size(); t += (size_t)c1)
            {
                const double v = (double)cont[i][t] * inv;
                cont[i][t] = (float)(v < -1.0 ? -1.0 : (v > 1.0 ? 1.0 : v));
            }
    }
    return fit_and_snap(d, m, 0, cont, false, k1_out, true);
}

int nntc_b200_init0_residual_channel(nntc_b200_device* d, const nntc_b200_model* m, int channel,
                                     const double* plane_weight, nntc_b200_init0_report* rep, uint8_t* const* k0_io)
{
    if (!d->resid)
    {
        set_error(NNTC_B200_ERR_STATE, "the residual seed needs a model created with init0_residual");
        return NNTC_B200_ERR_STATE;
    }
    const int nout = d->nout;
    *rep = nntc_b200_init0_report{};
    rep->nout = nout;
    rep->texture = -1;
    const int entries = nout + nout * nout;
    std::vector<double> raw((size_t)entries, 0.0);
    double count = 0.0;
    {
        const size_t nplanes = m->init0_chain ? d->planes.size() : 1;
        for (size_t i = 0; i < nplanes; i++)
        {
            const DevPlane& p = d->planes[i];
            const size_t texels = (size_t)p.w0 * p.h0;
            const double w = m->init0_chain ? plane_weight[i] : 1.0;
            if (!(w > 0.0))
                continue;
            NB_TRY(residual_pass(d, i));
            std::vector<double> part;
            NB_TRY(cov_sums(d, d->resid, texels, nout, part));
            for (int e = 0; e < entries; e++)
                raw[(size_t)e] += w * part[(size_t)e];
            count += w * (double)texels;
        }
    }
    std::vector<double> mu((size_t)nout, 0.0), cov((size_t)nout * nout, 0.0);
    for (int r = 0; r < nout; r++)
        mu[(size_t)r] = count > 0.0 ? raw[(size_t)r] / count : 0.0;
    for (int r = 0; r < nout; r++)
        for (int s = 0; s < nout; s++)
            cov[(size_t)r * nout + s] =
                (count > 0.0 ? raw[(size_t)(nout + r * nout + s)] / count : 0.0) - mu[(size_t)r] * mu[(size_t)s];
    for (int r = 0; r < nout; r++)
        rep->total_variance += cov[(size_t)r * nout + r];
    std::vector<double> u((size_t)nout, 0.0);
    if (m->init0_texture)
    {
        int best = 0;
        double best_value = -1.0;
        std::vector<double> best_vec(3, 0.0);
        for (int t = 0; t < m->textures; t++)
        {
            std::vector<double> block(9, 0.0);
            for (int r = 0; r < 3; r++)
                for (int s = 0; s < 3; s++)
                    block[(size_t)r * 3 + s] = cov[(size_t)(3 * t + r) * nout + (3 * t + s)];
            std::vector<double> work = block, vec, val;
            jacobi_eigen(work, 3, vec, val);
            int top = 0;
            for (int i = 1; i < 3; i++)
                if (val[(size_t)i] > val[(size_t)top])
                    top = i;
            if (val[(size_t)top] > best_value)
            {
                best_value = val[(size_t)top];
                best = t;
                for (int r = 0; r < 3; r++)
                    best_vec[(size_t)r] = vec[(size_t)r * 3 + top];
            }
        }
        rep->texture = best;
        rep->eigenvalue = best_value > 0.0 ? best_value : 0.0;
        for (int r = 0; r < 3; r++)
            u[(size_t)(3 * best + r)] = best_vec[(size_t)r];
    }
    else
    {
        std::vector<double> work = cov, vec, val;
        jacobi_eigen(work, nout, vec, val);
        int top = 0;
        for (int i = 1; i < nout; i++)
            if (val[(size_t)i] > val[(size_t)top])
                top = i;
        rep->eigenvalue = val[(size_t)top];
        for (int r = 0; r < nout; r++)
            u[(size_t)r] = vec[(size_t)r * nout + top];
    }
    rep->share = rep->total_variance > 0.0 ? rep->eigenvalue / rep->total_variance : 0.0;
    ProjDir dir{};
    for (int r = 0; r < nout; r++)
    {
        dir.e[r] = u[(size_t)r];
        dir.mu[r] = mu[(size_t)r];
    }
    int biggest = 0;
    for (int r = 1; r < nout; r++)
        if (std::fabs(dir.e[r]) > std::fabs(dir.e[biggest]))
            biggest = r;
    if (dir.e[biggest] < 0.0)
        for (int r = 0; r < nout; r++)
            dir.e[r] = -dir.e[r];
    for (int r = 0; r < nout && r < MAX_NOUT; r++)
        rep->dir[r] = dir.e[r];

    double peak = 0.0;
    std::vector<double> partial((size_t)COV_GRID, 0.0);
    for (size_t i = 0; i < d->planes.size(); i++)
    {
        const DevPlane& p = d->planes[i];
        const size_t texels = (size_t)p.w0 * p.h0;
        NB_TRY(residual_pass(d, i));
        k_proj_peak<<<COV_GRID, 256, 0, d->stream>>>(d->resid, texels, nout, dir, d->cov);
        NB_LAUNCHED();
        NB_TRY(download(d, partial.data(), d->cov, partial.size() * sizeof(double)));
        for (int b = 0; b < COV_GRID; b++)
            peak = std::max(peak, partial[(size_t)b]);
    }
    rep->peak = peak;
    rep->divisor = peak;
    double divisor = peak;
    const int BINS = HIST_BINS;
    if (!m->l0_bc8 && peak > 0.0)
    {
        NB_CUDA(cudaMemsetAsync(d->hist, 0, BINS * sizeof(unsigned long long), d->stream));
        unsigned long long total = 0ull;
        for (size_t i = 0; i < d->planes.size(); i++)
        {
            const DevPlane& p = d->planes[i];
            const size_t texels = (size_t)p.w0 * p.h0;
            NB_TRY(residual_pass(d, i));
            k_proj_hist<<<COV_GRID, 256, 0, d->stream>>>(d->resid, texels, nout, dir, 1.0 / peak, BINS, d->hist);
            NB_LAUNCHED();
            total += (unsigned long long)texels;
        }
        std::vector<unsigned long long> hist((size_t)BINS);
        NB_TRY(download(d, hist.data(), d->hist, hist.size() * sizeof(unsigned long long)));
        const unsigned long long want = (unsigned long long)(0.99 * (double)total);
        unsigned long long cum = 0ull;
        int bin = BINS - 1;
        for (int b = 0; b < BINS; b++)
        {
            cum += hist[(size_t)b];
            if (cum >= want)
            {
                bin = b;
                break;
            }
        }
        divisor = peak * (double)(bin + 1) / (double)BINS;
        if (!(divisor > 0.0))
            divisor = peak;
        rep->divisor = divisor;
    }
    const double inv = divisor > 0.0 ? 1.0 / divisor : 0.0;
    const int levels = m->l0_bc8 ? 255 : (1 << m->bits0[channel]) - 1;
    for (size_t i = 0; i < d->planes.size(); i++)
    {
        const DevPlane& p = d->planes[i];
        const size_t texels = (size_t)p.w0 * p.h0;
        NB_TRY(residual_pass(d, i));
        k_seed_channel<<<grid_for(texels, 256), 256, 0, d->stream>>>(d->resid, texels, nout, dir, inv, d->c0, channel,
                                                                     levels, d->palette, m->l0_bc8 ? 0 : 1, p.v0,
                                                                     p.k0);
        NB_LAUNCHED();
        if (!m->l0_bc8 && k0_io && k0_io[i])
            NB_TRY(download(d, k0_io[i], p.k0, texels * d->c0));
    }
    NB_CUDA(cudaStreamSynchronize(d->stream));
    return NNTC_B200_OK;
}

int nntc_b200_quantise_level1(nntc_b200_device* d, nntc_b200_model* m, int range_pct, uint8_t* const* k1_out)
{
    const std::vector<std::vector<float>> on_device;
    return fit_and_snap(d, m, 0, on_device, range_pct != 0, k1_out, true);
}

int nntc_b200_freeze_level1_grid(nntc_b200_device* d, nntc_b200_model* m, int range_pct, uint8_t* const* k1_out)
{
    const std::vector<std::vector<float>> on_device;
    return fit_and_snap(d, m, 0, on_device, range_pct != 0, k1_out, true);
}

static int level0_grid(nntc_b200_device* d, nntc_b200_model* m, int range_pct, uint8_t* const* k0_out)
{
    if (!d->l0_bc8)
    {
        set_error(NNTC_B200_ERR_STATE, "level 0 has a grid only under --l0 bc8");
        return NNTC_B200_ERR_STATE;
    }
    const std::vector<std::vector<float>> on_device;
    return fit_and_snap(d, m, 1, on_device, range_pct != 0, k0_out, true);
}

int nntc_b200_quantise_level0(nntc_b200_device* d, nntc_b200_model* m, int range_pct, uint8_t* const* k0_out)
{
    return level0_grid(d, m, range_pct, k0_out);
}

int nntc_b200_freeze_level0_grid(nntc_b200_device* d, nntc_b200_model* m, int range_pct, uint8_t* const* k0_out)
{
    return level0_grid(d, m, range_pct, k0_out);
}

int nntc_b200_snap_level0_on_grid(nntc_b200_device* d, const nntc_b200_model* m, uint8_t* const* k0_out)
{
    if (!d->l0_bc8)
    {
        set_error(NNTC_B200_ERR_STATE, "level 0 has a grid only under --l0 bc8");
        return NNTC_B200_ERR_STATE;
    }
    nntc_b200_model copy = *m;
    std::vector<std::vector<float>> none;
    return fit_and_snap(d, &copy, 1, none, false, k0_out, false);
}

}   // extern "C"
