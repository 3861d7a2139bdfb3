// grid.cu: the per-channel range of a latent over every plane of the chain, on the device (src/init.cu:520-563).
//
// minmax: the smallest and largest value of each channel. pct: the order statistics at ranks round(0.001 last) and
// round(0.999 last) of the channel's values over every plane - the values the reference reads off std::sort (and this
// library once read off std::nth_element on the host, after downloading the planes). Here they are found by an exact
// three-pass radix select on the values' order-preserving 32-bit keys (11 + 11 + 10 bits): each pass histograms the
// next digit of the keys that share the digits found so far, and the host walks the 2048-bin histogram to the bucket
// holding the rank. Integer counts, so the answer does not depend on scheduling; the value is the same k-th smallest
// value the sort gives (two zeros of opposite sign are the one value either way).
//
// Also here: the duplicate-channel test of the box init (src/main.cpp:1938-1960) - which source channels are exact
// copies of an earlier one over every texel of every plane - without the source leaving the device.

#include <algorithm>
#include <cstring>
#include <vector>

#include "device.cuh"

namespace nb
{

constexpr int RADIX_BINS = 2048;

__device__ __forceinline__ unsigned order_key(float f)
{
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__host__ __device__ inline float key_value(unsigned k)
{
    const unsigned b = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
#ifdef __CUDA_ARCH__
    return __uint_as_float(b);
#else
    float f;
    std::memcpy(&f, &b, sizeof(f));
    return f;
#endif
}

struct RadixPass
{
    int c;                          // channels
    int shift, width;               // this pass's digit
    int prefix_bits;                // digits already fixed (0 on the first pass)
    unsigned prefix[2 * MAX_CH];    // per (channel, target) the key's fixed high digits
};

// Histogram of this pass's digit over the values whose fixed digits match, per (channel, target).
__global__ void k_radix_hist(const float* v, size_t n, RadixPass R, unsigned int* hist)
{
    extern __shared__ unsigned int sh_hist[];   // [2 c][RADIX_BINS]
    const int bins = 1 << R.width;
    for (int i = threadIdx.x; i < 2 * R.c * bins; i += blockDim.x)
        sh_hist[i] = 0;
    __syncthreads();
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    {
        const int ch = (int)(i % (size_t)R.c);
        const unsigned k = order_key(v[i]);
        const unsigned digit = (k >> R.shift) & (unsigned)(bins - 1);
        for (int t = 0; t < 2; t++)
        {
            const bool match = R.prefix_bits == 0 || (k >> (32 - R.prefix_bits)) == R.prefix[2 * ch + t];
            if (match)
                atomicAdd(sh_hist + (2 * ch + t) * bins + digit, 1u);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * R.c * bins; i += blockDim.x)
        if (sh_hist[i])
            atomicAdd(hist + i, sh_hist[i]);
}

// Per-channel min and max as order keys (an integer atomic min / max is order-independent and exact).
__global__ void k_minmax_keys(const float* v, size_t n, int c, unsigned int* keys)
{
    unsigned lo[MAX_CH], hi[MAX_CH];
#pragma unroll
    for (int q = 0; q < MAX_CH; q++)
    {
        lo[q] = 0xFFFFFFFFu;
        hi[q] = 0u;
    }
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    {
        const int ch = (int)(i % (size_t)c);
        const unsigned k = order_key(v[i]);
#pragma unroll
        for (int q = 0; q < MAX_CH; q++)
            if (q == ch)
            {
                lo[q] = k < lo[q] ? k : lo[q];
                hi[q] = k > hi[q] ? k : hi[q];
            }
    }
#pragma unroll
    for (int q = 0; q < MAX_CH; q++)
        if (q < c)
        {
            atomicMin(keys + 2 * q, lo[q]);
            atomicMax(keys + 2 * q + 1, hi[q]);
        }
}

// flags[s nout + e] = 1 when source channel s differs from channel e (e < s) at any texel.
__global__ void k_channel_differs(const float* src, size_t texels, int nout, unsigned int* flags)
{
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < texels; t += (size_t)gridDim.x * blockDim.x)
    {
        const float* p = src + t * nout;
        for (int s = 1; s < nout; s++)
            for (int e = 0; e < s; e++)
                if (p[s] != p[e] && !flags[s * nout + e])
                    flags[s * nout + e] = 1u;
    }
}

// The range of every channel of one latent over every plane (level0: level 0's planes, else level 1's).
int fit_grid_device(nntc_b200_device* d, int level0, bool pct, float* lo, float* hi)
{
    const int c = level0 ? d->c0 : d->c1;
    auto values = [&](const DevPlane& p) {
        return level0 ? (size_t)p.w0 * p.h0 * c : (size_t)p.w1 * p.h1 * c;
    };
    unsigned int* scratch = d->radix;
    if (!pct)
    {
        std::vector<unsigned int> init(2 * MAX_CH);
        for (int q = 0; q < MAX_CH; q++)
        {
            init[2 * q] = 0xFFFFFFFFu;
            init[2 * q + 1] = 0u;
        }
        NB_TRY(upload(d, scratch, init.data(), init.size() * sizeof(unsigned)));
        for (const DevPlane& p : d->planes)
        {
            const size_t n = values(p);
            k_minmax_keys<<<std::min(grid_for(n, 256), 148 * 8), 256, 0, d->stream>>>(level0 ? p.v0 : p.v1, n, c,
                                                                                       scratch);
            NB_LAUNCHED();
        }
        std::vector<unsigned int> keys(2 * MAX_CH);
        NB_TRY(download(d, keys.data(), scratch, keys.size() * sizeof(unsigned)));
        for (int q = 0; q < c; q++)
        {
            lo[q] = key_value(keys[2 * q]);
            hi[q] = key_value(keys[2 * q + 1]);
        }
        return NNTC_B200_OK;
    }
    size_t count = 0;
    for (const DevPlane& p : d->planes)
        count += values(p) / (size_t)c;
    if (count == 0)
    {
        for (int q = 0; q < c; q++)
        {
            lo[q] = 1e30f;
            hi[q] = -1e30f;
        }
        return NNTC_B200_OK;
    }
    const size_t last = count - 1;
    size_t rank[2 * MAX_CH];
    for (int q = 0; q < c; q++)
    {
        rank[2 * q] = (size_t)(0.001 * (double)last + 0.5);
        rank[2 * q + 1] = (size_t)(0.999 * (double)last + 0.5);
    }
    RadixPass R{};
    R.c = c;
    const int widths[3] = { 11, 11, 10 };
    int done = 0;
    std::vector<unsigned int> hist;
    for (int pass = 0; pass < 3; pass++)
    {
        R.width = widths[pass];
        R.shift = 32 - done - R.width;
        R.prefix_bits = done;
        const int bins = 1 << R.width;
        NB_CUDA(cudaMemsetAsync(scratch, 0, (size_t)2 * c * bins * sizeof(unsigned), d->stream));
        const size_t shared = (size_t)2 * c * bins * sizeof(unsigned);
        NB_CUDA(cudaFuncSetAttribute(k_radix_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shared));
        for (const DevPlane& p : d->planes)
        {
            const size_t n = values(p);
            k_radix_hist<<<std::min(grid_for(n, 256), 148 * 4), 256, shared, d->stream>>>(level0 ? p.v0 : p.v1, n, R,
                                                                                          scratch);
            NB_LAUNCHED();
        }
        hist.assign((size_t)2 * c * bins, 0);
        NB_TRY(download(d, hist.data(), scratch, hist.size() * sizeof(unsigned)));
        for (int t = 0; t < 2 * c; t++)
        {
            size_t cum = 0;
            int b = 0;
            for (; b < bins; b++)
            {
                const size_t h = hist[(size_t)t * bins + b];
                if (rank[t] < cum + h)
                    break;
                cum += h;
            }
            rank[t] -= cum;
            R.prefix[t] = (done == 0 ? 0u : (R.prefix[t] << R.width)) | (unsigned)b;
        }
        done += R.width;
    }
    for (int q = 0; q < c; q++)
    {
        lo[q] = key_value(R.prefix[2 * q]);
        hi[q] = key_value(R.prefix[2 * q + 1]);
    }
    return NNTC_B200_OK;
}

// Which source channels repeat an earlier one exactly over every texel of every plane: same[s nout + e] for e < s.
int channel_copies(nntc_b200_device* d, std::vector<unsigned char>& same)
{
    const int nout = d->nout;
    unsigned int* flags = d->radix;
    NB_CUDA(cudaMemsetAsync(flags, 0, (size_t)nout * nout * sizeof(unsigned), d->stream));
    for (const DevPlane& p : d->planes)
    {
        const size_t n = (size_t)p.w0 * p.h0;
        k_channel_differs<<<std::min(grid_for(n, 256), 148 * 8), 256, 0, d->stream>>>(p.src, n, nout, flags);
        NB_LAUNCHED();
    }
    std::vector<unsigned int> f((size_t)nout * nout);
    NB_TRY(download(d, f.data(), flags, f.size() * sizeof(unsigned)));
    same.assign((size_t)nout * nout, 0);
    for (int s = 0; s < nout; s++)
        for (int e = 0; e < s; e++)
            same[(size_t)s * nout + e] = f[(size_t)s * nout + e] == 0;
    return NNTC_B200_OK;
}

}   // namespace nb
