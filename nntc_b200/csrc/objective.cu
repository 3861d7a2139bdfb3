// objective.cu: the objective E over every site of every plane, and the encoder's own 8-bit decode of a level.
//
// Follows src/objective.cu:53-279: E = sum_m w_m sum_sites sum_c cw_c (W phi + b - t)_c^2 with phi and the target
// sampled in double at u = (px + 0.5 + dx) / w0 (src/objective.cu:97-118), plus the unweighted centre-site and
// fractional-site sums per plane, normalised on the host (src/objective.cu:224-250).
//
// B200 shape: one thread per pixel handles that pixel's 1 + K sites, every plane of the chain in ONE launch (the
// per-plane pixel ranges are padded to whole blocks, so a block belongs to one plane); the decoder sits in shared
// memory as doubles; each block writes one partial per sum, and a second kernel adds a plane's partials in block
// order. The dot products use DFMA: the per-site value differs from the reference's separately-rounded multiply-add
// in the last bits only, and E is a measurement held to 1e-9 relative of the host twin (src/objective.cu:317-380).

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "device.cuh"

namespace nb
{

constexpr int OBJ_THREADS = 256;
constexpr int OBJ_P_THREADS = 128;   // k_objective_p's blocks: smaller blocks fit five per SM at its register count

struct ObjArgs
{
    const float* weights;
    const float* bias;
    const float* cw;
    double* partial;   // [3][total blocks]
};

// The bilinear rule in double at u, v (src/objective.cu:97-118), the channel loop unrolled to MAXC and guarded so
// the result stays in registers.
template <int MAXC>
__device__ __forceinline__ void obj_sample(const float* plane, int w, int h, int c, double u, double v, double* out)
{
    const double x = u * (double)w - 0.5, y = v * (double)h - 0.5;
    const double xf = floor(x), yf = floor(y);
    const double fx = x - xf, fy = y - yf;
    const int x0 = clampi((int)xf, w), x1 = clampi((int)xf + 1, w);
    const int y0 = clampi((int)yf, h), y1 = clampi((int)yf + 1, h);
    const float* a = plane + ((size_t)y0 * w + x0) * c;
    const float* b = plane + ((size_t)y0 * w + x1) * c;
    const float* e = plane + ((size_t)y1 * w + x0) * c;
    const float* f = plane + ((size_t)y1 * w + x1) * c;
    const double w00 = (1.0 - fx) * (1.0 - fy), w10 = fx * (1.0 - fy), w01 = (1.0 - fx) * fy, w11 = fx * fy;
#pragma unroll
    for (int k = 0; k < MAXC; k++)
        if (k < c)
            out[k] = w00 * (double)__ldg(a + k) + w10 * (double)__ldg(b + k) + w01 * (double)__ldg(e + k) +
                     w11 * (double)__ldg(f + k);
}

__device__ __forceinline__ double block_sum(double v, double* sh)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0)
        sh[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); i++)
            s += sh[i];
    return s;   // valid on thread 0
}

// One thread per pixel, its 1 + K sites in turn; each output row r formed in phi's order, b + sum of W[r][.] phi,
// with phi = [c_q][s_i][s_i c_q] never stored: the row walks the three groups itself.
__global__ void __launch_bounds__(OBJ_THREADS) k_objective(Planes P, ObjArgs A)
{
    // The decoder at a fixed row stride of 24 feature slots, [c_q (4)][s_i (4)][s_i c_q (4 x 4)], whatever C0 and C1
    // are: a channel the layout does not use has weight zero, whose product adds an exact zero to the row, so each row
    // is the reference's sum over phi in phi's order and loads as twelve 16-byte pairs.
    __shared__ __align__(16) double sw[MAX_NOUT * 24];
    __shared__ double sb[MAX_NOUT];
    __shared__ double scw[MAX_NOUT];
    __shared__ double red[32];
    const int nin = P.nin, nout = P.nout, c0 = P.c0, c1 = P.c1, kc = P.kc;
    for (int i = threadIdx.x; i < nout * 24; i += blockDim.x)
    {
        const int r = i / 24, slot = i % 24;
        int col = -1;
        if (slot < 4)
            col = slot < c1 ? slot : -1;
        else if (slot < 8)
            col = slot - 4 < c0 ? c1 + slot - 4 : -1;
        else
        {
            const int ii = (slot - 8) / 4, q = (slot - 8) % 4;
            col = ii < c0 && q < c1 ? c1 + c0 + ii * c1 + q : -1;
        }
        sw[i] = col >= 0 ? (double)A.weights[(size_t)r * nin + col] : 0.0;
    }
    for (int i = threadIdx.x; i < nout; i += blockDim.x)
    {
        sb[i] = (double)A.bias[i];
        scw[i] = (double)A.cw[i];
    }
    __syncthreads();

    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long local = base - P.start[pl] + threadIdx.x;
    double weighted = 0.0, centre = 0.0, fractional = 0.0;
    if (local < (long long)V.w0 * V.h0)
    {
        const int px = (int)(local % V.w0), py = (int)(local / V.w0);
        for (int j = 0; j <= kc; j++)
        {
            float dx = 0.0f, dy = 0.0f;
            if (j > 0)
                subtexel(kc, j - 1, px, py, dx, dy);
            const double u = ((double)px + 0.5 + (double)dx) / (double)V.w0;
            const double v = ((double)py + 0.5 + (double)dy) / (double)V.h0;
            double s[MAX_CH], c[MAX_CH];
#pragma unroll
            for (int q = 0; q < MAX_CH; q++)
            {
                s[q] = 0.0;
                c[q] = 0.0;
            }
            obj_sample<MAX_CH>(V.v1, V.w1, V.h1, c1, u, v, c);
            // the source's taps at this site (the centre site reads the pixel itself)
            size_t ta = (size_t)local * nout, tb = ta, te = ta, tf = ta;
            double w00 = 1.0, w10 = 0.0, w01 = 0.0, w11 = 0.0;
            if (j == 0)
            {
#pragma unroll
                for (int i = 0; i < MAX_CH; i++)
                    if (i < c0)
                        s[i] = (double)V.v0[local * c0 + i];
            }
            else
            {
                obj_sample<MAX_CH>(V.v0, V.w0, V.h0, c0, u, v, s);
                const double x = u * (double)V.w0 - 0.5, y = v * (double)V.h0 - 0.5;
                const double xf = floor(x), yf = floor(y);
                const double fx = x - xf, fy = y - yf;
                const int x0 = clampi((int)xf, V.w0), x1 = clampi((int)xf + 1, V.w0);
                const int y0 = clampi((int)yf, V.h0), y1 = clampi((int)yf + 1, V.h0);
                ta = ((size_t)y0 * V.w0 + x0) * nout;
                tb = ((size_t)y0 * V.w0 + x1) * nout;
                te = ((size_t)y1 * V.w0 + x0) * nout;
                tf = ((size_t)y1 * V.w0 + x1) * nout;
                w00 = (1.0 - fx) * (1.0 - fy);
                w10 = fx * (1.0 - fy);
                w01 = (1.0 - fx) * fy;
                w11 = fx * fy;
            }
            double sc[16];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int q = 0; q < 4; q++)
                    sc[i * 4 + q] = s[i] * c[q];
            for (int r = 0; r < nout; r++)
            {
                const double t = j == 0 ? (double)__ldg(V.src + ta + r)
                                        : w00 * (double)__ldg(V.src + ta + r) + w10 * (double)__ldg(V.src + tb + r) +
                                              w01 * (double)__ldg(V.src + te + r) + w11 * (double)__ldg(V.src + tf + r);
                const double2* row = (const double2*)(sw + r * 24);
                double acc = sb[r];
#pragma unroll
                for (int h = 0; h < 2; h++)
                {
                    const double2 wv = row[h];
                    acc = fma(wv.x, c[2 * h], acc);
                    acc = fma(wv.y, c[2 * h + 1], acc);
                }
#pragma unroll
                for (int h = 0; h < 2; h++)
                {
                    const double2 wv = row[2 + h];
                    acc = fma(wv.x, s[2 * h], acc);
                    acc = fma(wv.y, s[2 * h + 1], acc);
                }
#pragma unroll
                for (int h = 0; h < 8; h++)
                {
                    const double2 wv = row[4 + h];
                    acc = fma(wv.x, sc[2 * h], acc);
                    acc = fma(wv.y, sc[2 * h + 1], acc);
                }
                const double e = acc - t;
                weighted = fma(scw[r] * e, e, weighted);
                if (j == 0)
                    centre = fma(e, e, centre);
                else
                    fractional = fma(e, e, fractional);
            }
        }
    }
    const double a = block_sum(weighted, red);
    const double b = block_sum(centre, red);
    const double c = block_sum(fractional, red);
    if (threadIdx.x == 0)
    {
        const size_t nb = gridDim.x;
        A.partial[blockIdx.x] = a;
        A.partial[nb + blockIdx.x] = b;
        A.partial[2 * nb + blockIdx.x] = c;
    }
}

// The decoder as a launch parameter, in k_objective's fixed 24-slot row layout: with the row loop unrolled every
// weight is an immediate constant-bank operand of its DFMA, so the dot products issue no shared-memory loads.
struct ObjDecoder
{
    double w[MAX_NOUT * 24];
    double b[MAX_NOUT];
    double cw[MAX_NOUT];
};

// The target of every fractional site (j > 0) in double: the source's bilinear sample at the site as k_objective_p
// took it inline, a chain of fused multiply-adds (a measurement: its last bits move, within the objective's 1e-12). It
// depends on nothing but the source and K, neither of which an encode changes, so it is formed once per device model
// and K and read by every later objective pass.
struct ObjTargets
{
    const double* t;                   // [fractional site][NOUT]
    long long site0[MAX_PLANES + 1];   // the first fractional site of each plane
};

template <int NOUT>
__global__ void __launch_bounds__(OBJ_THREADS) k_objective_targets(Planes P, double* tgt, const __grid_constant__ ObjTargets O)
{
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long fi = base - P.start[pl] + threadIdx.x;
    const int kc = P.kc;
    if (fi >= (long long)V.w0 * V.h0 * kc)
        return;
    const long long local = fi / kc;
    const int j = 1 + (int)(fi % kc);
    const int px = (int)(local % V.w0), py = (int)(local / V.w0);
    float dx = 0.0f, dy = 0.0f;
    subtexel(kc, j - 1, px, py, dx, dy);
    const double u = ((double)px + 0.5 + (double)dx) / (double)V.w0;
    const double v = ((double)py + 0.5 + (double)dy) / (double)V.h0;
    const double x = u * (double)V.w0 - 0.5, y = v * (double)V.h0 - 0.5;
    const double xf = floor(x), yf = floor(y);
    const double fx = x - xf, fy = y - yf;
    const int x0 = clampi((int)xf, V.w0), x1 = clampi((int)xf + 1, V.w0);
    const int y0 = clampi((int)yf, V.h0), y1 = clampi((int)yf + 1, V.h0);
    const size_t ta = ((size_t)y0 * V.w0 + x0) * NOUT, tb = ((size_t)y0 * V.w0 + x1) * NOUT;
    const size_t te = ((size_t)y1 * V.w0 + x0) * NOUT, tf = ((size_t)y1 * V.w0 + x1) * NOUT;
    const double w00 = (1.0 - fx) * (1.0 - fy), w10 = fx * (1.0 - fy), w01 = (1.0 - fx) * fy, w11 = fx * fy;
    double* out = tgt + (size_t)(O.site0[pl] + fi) * NOUT;
#pragma unroll
    for (int r = 0; r < NOUT; r++)
        out[r] = fma(w11, (double)__ldg(V.src + tf + r),
                     fma(w01, (double)__ldg(V.src + te + r),
                         fma(w10, (double)__ldg(V.src + tb + r), w00 * (double)__ldg(V.src + ta + r))));
}

// k_objective for a material of NOUT outputs (3 per texture), the decoder in the launch's parameters, the fractional
// sites' targets from k_objective_targets. The same sites, the same operations in the same order as k_objective,
// whose bits it matches but for the targets' fused multiply-adds.
template <int NOUT>
__global__ void __launch_bounds__(OBJ_P_THREADS, 5)
    k_objective_p(Planes P, ObjDecoder W, double* partial, const __grid_constant__ ObjTargets T)
{
    __shared__ double red[32];
    const int c0 = P.c0, c1 = P.c1, kc = P.kc;
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long local = base - P.start[pl] + threadIdx.x;
    double weighted = 0.0, centre = 0.0, fractional = 0.0;
    if (local < (long long)V.w0 * V.h0)
    {
        const int px = (int)(local % V.w0), py = (int)(local / V.w0);
        for (int j = 0; j <= kc; j++)
        {
            float dx = 0.0f, dy = 0.0f;
            if (j > 0)
                subtexel(kc, j - 1, px, py, dx, dy);
            const double u = ((double)px + 0.5 + (double)dx) / (double)V.w0;
            const double v = ((double)py + 0.5 + (double)dy) / (double)V.h0;
            double s[MAX_CH], c[MAX_CH];
#pragma unroll
            for (int q = 0; q < MAX_CH; q++)
            {
                s[q] = 0.0;
                c[q] = 0.0;
            }
            obj_sample<MAX_CH>(V.v1, V.w1, V.h1, c1, u, v, c);
            if (j == 0)
            {
#pragma unroll
                for (int i = 0; i < MAX_CH; i++)
                    if (i < c0)
                        s[i] = (double)V.v0[local * c0 + i];
            }
            else
                obj_sample<MAX_CH>(V.v0, V.w0, V.h0, c0, u, v, s);
            // every row's dot product advanced together, feature by feature (each row's own sum keeps phi's order),
            // so that NOUT independent chains of DFMAs are in flight at once; a product feature s_i c_q is formed
            // once, when its turn comes, instead of being held for the whole site
            double acc[NOUT];
#pragma unroll
            for (int r = 0; r < NOUT; r++)
                acc[r] = W.b[r];
#pragma unroll
            for (int h = 0; h < 4; h++)
#pragma unroll
                for (int r = 0; r < NOUT; r++)
                    acc[r] = fma(W.w[r * 24 + h], c[h], acc[r]);
#pragma unroll
            for (int h = 0; h < 4; h++)
#pragma unroll
                for (int r = 0; r < NOUT; r++)
                    acc[r] = fma(W.w[r * 24 + 4 + h], s[h], acc[r]);
#pragma unroll
            for (int h = 0; h < 16; h++)
            {
                const double sc = s[h / 4] * c[h % 4];
#pragma unroll
                for (int r = 0; r < NOUT; r++)
                    acc[r] = fma(W.w[r * 24 + 8 + h], sc, acc[r]);
            }
            // the pixel's own source at the centre site, else the fractional site's sample from k_objective_targets
            const float* t_centre = V.src + (size_t)local * NOUT;
            const double* t_frac = j > 0 ? T.t + (size_t)(T.site0[pl] + local * kc + (j - 1)) * NOUT : nullptr;
#pragma unroll
            for (int r = 0; r < NOUT; r++)
            {
                const double t = j == 0 ? (double)__ldg(t_centre + r) : __ldg(t_frac + r);
                const double e = acc[r] - t;
                weighted = fma(W.cw[r] * e, e, weighted);
                if (j == 0)
                    centre = fma(e, e, centre);
                else
                    fractional = fma(e, e, fractional);
            }
        }
    }
    const double a = block_sum(weighted, red);
    const double b = block_sum(centre, red);
    const double c = block_sum(fractional, red);
    if (threadIdx.x == 0)
    {
        const size_t nb = gridDim.x;
        partial[blockIdx.x] = a;
        partial[nb + blockIdx.x] = b;
        partial[2 * nb + blockIdx.x] = c;
    }
}

// The mixed-precision objective (the adjoint form): the sites' samples with the float tap rule of the assembly
// (tap_at, blend), every output row's dot product in FP32 fused multiply-adds with the decoder as a launch parameter,
// the fractional sites' float targets of the assembly (d->site_tgt), each site's squared residuals summed over its
// outputs in FP32 (a few positive terms) and the sites' sums in FP64. E agrees with the FP64 objective to about 1e-7
// relative; what decides on E (the stops, the acceptance of a repack pass)
// sees the same E within tolerances four orders coarser.
struct ObjDecoderF
{
    float w[MAX_NOUT * 24];
    float b[MAX_NOUT];
    float cw[MAX_NOUT];
};

struct ObjTargetsF
{
    const float* t;                    // [fractional site][NOUT]
    long long site0[MAX_PLANES + 1];
};

template <int NOUT>
__global__ void __launch_bounds__(OBJ_P_THREADS, 8)
    k_objective_f32(Planes P, ObjDecoderF W, double* partial, const __grid_constant__ ObjTargetsF T)
{
    __shared__ double red[32];
    const int c0 = P.c0, c1 = P.c1, kc = P.kc;
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long local = base - P.start[pl] + threadIdx.x;
    double weighted = 0.0, centre = 0.0, fractional = 0.0;
    if (local < (long long)V.w0 * V.h0)
    {
        const int px = (int)(local % V.w0), py = (int)(local / V.w0);
        for (int j = 0; j <= kc; j++)
        {
            float dx, dy;
            site_offset(kc, j, px, py, dx, dy);
            float s[MAX_CH] = { 0.0f, 0.0f, 0.0f, 0.0f }, c[MAX_CH] = { 0.0f, 0.0f, 0.0f, 0.0f };
            blend_u<MAX_CH>(V.v1, V.w1, c1, tap_at(px, py, dx, dy, V.w0, V.h0, V.w1, V.h1), c);
            if (j == 0)
            {
#pragma unroll
                for (int i = 0; i < MAX_CH; i++)
                    if (i < c0)
                        s[i] = __ldg(V.v0 + local * c0 + i);
            }
            else
                blend_u<MAX_CH>(V.v0, V.w0, c0, tap_at(px, py, dx, dy, V.w0, V.h0, V.w0, V.h0), s);
            float acc[NOUT];
#pragma unroll
            for (int r = 0; r < NOUT; r++)
                acc[r] = W.b[r];
#pragma unroll
            for (int h = 0; h < 4; h++)
#pragma unroll
                for (int r = 0; r < NOUT; r++)
                    acc[r] = __fmaf_rn(W.w[r * 24 + h], c[h], acc[r]);
#pragma unroll
            for (int h = 0; h < 4; h++)
#pragma unroll
                for (int r = 0; r < NOUT; r++)
                    acc[r] = __fmaf_rn(W.w[r * 24 + 4 + h], s[h], acc[r]);
#pragma unroll
            for (int h = 0; h < 16; h++)
            {
                const float sc = s[h / 4] * c[h % 4];
#pragma unroll
                for (int r = 0; r < NOUT; r++)
                    acc[r] = __fmaf_rn(W.w[r * 24 + 8 + h], sc, acc[r]);
            }
            const float* tg = j == 0 ? V.src + (size_t)local * NOUT
                                     : T.t + (size_t)(T.site0[pl] + local * kc + (j - 1)) * NOUT;
            // the site's two sums over its outputs in FP32 (NOUT positive terms), each added to the FP64 totals once
            float sw = 0.0f, ss = 0.0f;
#pragma unroll
            for (int r = 0; r < NOUT; r++)
            {
                const float e = acc[r] - __ldg(tg + r);
                sw = __fmaf_rn(W.cw[r] * e, e, sw);
                ss = __fmaf_rn(e, e, ss);
            }
            weighted += (double)sw;
            if (j == 0)
                centre += (double)ss;
            else
                fractional += (double)ss;
        }
    }
    const double a = block_sum(weighted, red);
    const double b = block_sum(centre, red);
    const double c = block_sum(fractional, red);
    if (threadIdx.x == 0)
    {
        const size_t nb = gridDim.x;
        partial[blockIdx.x] = a;
        partial[nb + blockIdx.x] = b;
        partial[2 * nb + blockIdx.x] = c;
    }
}

int ensure_site_targets(nntc_b200_device* d, int k, int level0);

// One block per plane: the plane's block partials added in a fixed order (a strided pass, then a fixed tree).
__global__ void k_objective_reduce(Planes P, const double* partial, int nblocks, double* out, int bthreads)
{
    __shared__ double red[32];
    const int pl = blockIdx.x;
    const long long b0 = P.start[pl] / bthreads, b1 = P.start[pl + 1] / bthreads;
    for (int row = 0; row < 3; row++)
    {
        double s = 0.0;
        for (long long b = b0 + threadIdx.x; b < b1; b += blockDim.x)
            s += partial[(size_t)row * nblocks + b];
        const double t = block_sum(s, red);
        if (threadIdx.x == 0)
            out[3 * pl + row] = t;
        __syncthreads();
    }
}

// The recon decode at texel centres: saturate, then lroundf(acc * 255) (src/objective.cu:53-75).
__global__ void k_decode(const float* v0, const float* v1, int w0, int h0, int w1, int h1, int c0, int c1, int nin,
                         int nout, const float* weights, const float* bias, uint8_t* out)
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
        acc = acc < 0.0f ? 0.0f : (acc > 1.0f ? 1.0f : acc);
        out[idx * nout + r] = (uint8_t)lroundf(acc * 255.0f);
    }
}

// The per-texture squared error of the 8-bit decode against the source bytes round(255 src) (src/main.cpp:3000-3060),
// as exact integer sums: one 64-bit total per texture, added with integer atomics, so the order does not matter.
__global__ void k_psnr_sums(const uint8_t* rgb, const float* src, size_t n, int nout, unsigned long long* se)
{
    unsigned long long acc[6] = { 0, 0, 0, 0, 0, 0 };
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    {
#pragma unroll
        for (int t = 0; t < 6; t++)
#pragma unroll
            for (int c = 0; c < 3; c++)
            {
                const int k = 3 * t + c;
                if (k >= nout)
                    continue;
                const long long want = llround((double)src[i * nout + k] * 255.0);
                const long long e = (long long)rgb[i * nout + k] - want;
                acc[t] += (unsigned long long)(e * e);
            }
    }
#pragma unroll
    for (int t = 0; t < 6; t++)
    {
        unsigned long long v = acc[t];
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v)
            atomicAdd(se + t, v);
    }
}

int psnr_base(nntc_b200_device* d, const nntc_b200_model* m, double* psnr)
{
    const DevPlane& p = d->planes[0];
    const size_t n = (size_t)p.w0 * p.h0;
    k_decode<<<grid_for(n, 256), 256, 0, d->stream>>>(p.v0, p.v1, p.w0, p.h0, p.w1, p.h1, d->c0, d->c1, d->nin,
                                                      d->nout, d->weights, d->bias, d->rgb8);
    NB_LAUNCHED();
    unsigned long long* se = (unsigned long long*)d->radix;
    NB_CUDA(cudaMemsetAsync(se, 0, 6 * sizeof(unsigned long long), d->stream));
    k_psnr_sums<<<std::min(grid_for(n, 256), 148 * 8), 256, 0, d->stream>>>(d->rgb8, p.src, n, d->nout, se);
    NB_LAUNCHED();
    unsigned long long h[6];
    NB_TRY(download(d, h, se, sizeof(h)));
    for (int t = 0; t < m->textures && t < 6; t++)
    {
        const double mse = (double)h[t] / (double)(n * 3);
        psnr[t] = mse > 0.0 ? 10.0 * std::log10(255.0 * 255.0 / mse) : 99.0;
    }
    return NNTC_B200_OK;
}

// The reported numbers from the three raw sums per plane (src/objective.cu:224-250).
static void normalise(const nntc_b200_model& m, int k, const double* per_site, const std::vector<double>& acc,
                      nntc_b200_objective* r)
{
    double sum_cw = 0.0;
    for (int c = 0; c < m.nout; c++)
        sum_cw += (double)m.cw[c];
    double num = 0.0, den = 0.0;
    for (int p = 0; p < m.nplanes; p++)
    {
        const double pixels = (double)m.w0[p] * (double)m.h0[p];
        const double sites = pixels * (double)(1 + k);
        r->e_plane[p] = acc[3 * p] / (sum_cw * sites);
        r->centre_plane[p] = acc[3 * p + 1] / (pixels * (double)m.nout);
        num += per_site[p] * acc[3 * p];
        den += per_site[p] * sites;
    }
    r->e = den > 0.0 ? num / (sum_cw * den) : 0.0;
    const double base = (double)m.w0[0] * (double)m.h0[0] * (double)m.nout;
    r->centre_mse = acc[1] / base;
    r->sampled_mse = k > 0 ? acc[2] / (base * (double)k) : 0.0;
}

// The reported numbers from three raw sums per plane formed elsewhere (the tensor-core normal equations' pass).
void objective_from_sums(const nntc_b200_model& m, int k, const double* per_site, const std::vector<double>& acc,
                         nntc_b200_objective* r)
{
    *r = nntc_b200_objective{};
    normalise(m, k, per_site, acc, r);
}

static double g_objective_ms = 0.0;
static long long g_objective_calls = 0;

// The raw sums of every plane, three per plane, into host memory (acc has 3 nplanes entries).
int objective_sums(nntc_b200_device* d, int k, std::vector<double>& acc, double* ms)
{
    Planes P = planes_for(d, 0, [&](int i) { return (size_t)d->planes[(size_t)i].w0 * d->planes[(size_t)i].h0; });
    P.kc = k;
    const int bthreads = d->nout % 3 == 0 && d->nout <= 18 ? OBJ_P_THREADS : OBJ_THREADS;
    const int nblocks = (int)(P.start[P.n] / bthreads);
    // device_create sized obj_partial for this layout: 3 doubles per pixel block, then 3 sums per plane.
    double* sums = d->obj_partial + (size_t)nblocks * 3;
    // the decoder as the device holds it, in the 24-slot row layout (a channel the layout does not use has weight 0)
    ObjDecoder W{};
    const int nin = d->nin, nout = d->nout, c0 = d->c0, c1 = d->c1;
    for (int r = 0; r < nout; r++)
    {
        for (int slot = 0; slot < 24; slot++)
        {
            int col = -1;
            if (slot < 4)
                col = slot < c1 ? slot : -1;
            else if (slot < 8)
                col = slot - 4 < c0 ? c1 + slot - 4 : -1;
            else
            {
                const int ii = (slot - 8) / 4, q = (slot - 8) % 4;
                col = ii < c0 && q < c1 ? c1 + c0 + ii * c1 + q : -1;
            }
            W.w[r * 24 + slot] = col >= 0 ? (double)d->host_weights[(size_t)r * nin + col] : 0.0;
        }
        W.b[r] = (double)d->host_bias[r];
        W.cw[r] = (double)d->m.cw[r];
    }
    NB_TRY(block_begin(d));
    // the fractional sites' targets, formed on the first pass at this K
    ObjTargets T{};
    T.t = d->obj_tgt;
    {
        long long ft = 0;
        for (int i = 0; i < P.n; i++)
        {
            T.site0[i] = ft;
            ft += (long long)d->planes[(size_t)i].w0 * d->planes[(size_t)i].h0 * k;
        }
        T.site0[P.n] = ft;
    }
    if (d->obj_tgt_kc != k && k > 0 && bthreads == OBJ_P_THREADS && !d->mixed_objective)
    {
        Planes F = planes_for(d, 0, [&](int i) {
            const DevPlane& p = d->planes[(size_t)i];
            return (size_t)p.w0 * p.h0 * (size_t)k;
        });
        F.kc = k;
        const int fblocks = (int)(F.start[F.n] / OBJ_THREADS);
        switch (nout)
        {
        case 3: k_objective_targets<3><<<fblocks, OBJ_THREADS, 0, d->stream>>>(F, d->obj_tgt, T); break;
        case 6: k_objective_targets<6><<<fblocks, OBJ_THREADS, 0, d->stream>>>(F, d->obj_tgt, T); break;
        case 9: k_objective_targets<9><<<fblocks, OBJ_THREADS, 0, d->stream>>>(F, d->obj_tgt, T); break;
        case 12: k_objective_targets<12><<<fblocks, OBJ_THREADS, 0, d->stream>>>(F, d->obj_tgt, T); break;
        case 15: k_objective_targets<15><<<fblocks, OBJ_THREADS, 0, d->stream>>>(F, d->obj_tgt, T); break;
        case 18: k_objective_targets<18><<<fblocks, OBJ_THREADS, 0, d->stream>>>(F, d->obj_tgt, T); break;
        }
        NB_LAUNCHED();
        d->obj_tgt_kc = k;
    }
    if (d->mixed_objective && bthreads == OBJ_P_THREADS)
    {
        NB_TRY(ensure_site_targets(d, k, 0));
        ObjDecoderF F{};
        for (int i = 0; i < nout * 24; i++)
            F.w[i] = (float)W.w[i];
        for (int r = 0; r < nout; r++)
        {
            F.b[r] = d->host_bias[r];
            F.cw[r] = d->m.cw[r];
        }
        ObjTargetsF TF{};
        TF.t = d->site_tgt;
        for (int i = 0; i <= P.n; i++)
            TF.site0[i] = T.site0[i];
        NB_TRY(ktimer_begin(d, NNTC_B200_K_OBJECTIVE));
        switch (nout)
        {
        case 3: k_objective_f32<3><<<nblocks, OBJ_P_THREADS, 0, d->stream>>>(P, F, d->obj_partial, TF); break;
        case 6: k_objective_f32<6><<<nblocks, OBJ_P_THREADS, 0, d->stream>>>(P, F, d->obj_partial, TF); break;
        case 9: k_objective_f32<9><<<nblocks, OBJ_P_THREADS, 0, d->stream>>>(P, F, d->obj_partial, TF); break;
        case 12: k_objective_f32<12><<<nblocks, OBJ_P_THREADS, 0, d->stream>>>(P, F, d->obj_partial, TF); break;
        case 15: k_objective_f32<15><<<nblocks, OBJ_P_THREADS, 0, d->stream>>>(P, F, d->obj_partial, TF); break;
        default: k_objective_f32<18><<<nblocks, OBJ_P_THREADS, 0, d->stream>>>(P, F, d->obj_partial, TF); break;
        }
        NB_TRY(ktimer_end(d));
        NB_LAUNCHED();
        k_objective_reduce<<<P.n, 256, 0, d->stream>>>(P, d->obj_partial, nblocks, sums, bthreads);
        NB_LAUNCHED();
        NB_TRY(block_end(d, ms));
        acc.assign((size_t)3 * P.n, 0.0);
        return download(d, acc.data(), sums, acc.size() * sizeof(double));
    }
    NB_TRY(ktimer_begin(d, NNTC_B200_K_OBJECTIVE));
    switch (nout)
    {
    case 3: k_objective_p<3><<<nblocks, OBJ_P_THREADS, 0, d->stream>>>(P, W, d->obj_partial, T); break;
    case 6: k_objective_p<6><<<nblocks, OBJ_P_THREADS, 0, d->stream>>>(P, W, d->obj_partial, T); break;
    case 9: k_objective_p<9><<<nblocks, OBJ_P_THREADS, 0, d->stream>>>(P, W, d->obj_partial, T); break;
    case 12: k_objective_p<12><<<nblocks, OBJ_P_THREADS, 0, d->stream>>>(P, W, d->obj_partial, T); break;
    case 15: k_objective_p<15><<<nblocks, OBJ_P_THREADS, 0, d->stream>>>(P, W, d->obj_partial, T); break;
    case 18: k_objective_p<18><<<nblocks, OBJ_P_THREADS, 0, d->stream>>>(P, W, d->obj_partial, T); break;
    default:
        k_objective<<<nblocks, OBJ_THREADS, 0, d->stream>>>(P, ObjArgs{ d->weights, d->bias, d->cw, d->obj_partial });
    }
    NB_TRY(ktimer_end(d));
    NB_LAUNCHED();
    k_objective_reduce<<<P.n, 256, 0, d->stream>>>(P, d->obj_partial, nblocks, sums, bthreads);
    NB_LAUNCHED();
    NB_TRY(block_end(d, ms));
    acc.assign((size_t)3 * P.n, 0.0);
    return download(d, acc.data(), sums, acc.size() * sizeof(double));
}

}   // namespace nb

using namespace nb;

extern "C"
{

int nntc_b200_objective_eval(nntc_b200_device* d, const nntc_b200_model* m, int k, const double* per_site,
                             nntc_b200_objective* r)
{
    std::vector<double> acc;
    double ms = 0.0;
    NB_TRY(objective_sums(d, k, acc, &ms));
    *r = nntc_b200_objective{};
    normalise(*m, k, per_site, acc, r);
    r->ms = ms;
    g_objective_ms += ms;
    g_objective_calls++;
    return NNTC_B200_OK;
}

double nntc_b200_objective_total_ms(void)
{
    return g_objective_ms;
}

long long nntc_b200_objective_passes(void)
{
    return g_objective_calls;
}

int nntc_b200_decode_plane(nntc_b200_device* d, const nntc_b200_model* m, int plane, uint8_t* rgb8, size_t n)
{
    NB_TRY(check_plane(d, plane));
    const DevPlane& p = d->planes[(size_t)plane];
    const size_t px = (size_t)p.w0 * p.h0;
    if (n < px * m->nout)
    {
        set_error(NNTC_B200_ERR_ARG, "decode buffer too small");
        return NNTC_B200_ERR_ARG;
    }
    k_decode<<<grid_for(px, 256), 256, 0, d->stream>>>(p.v0, p.v1, p.w0, p.h0, p.w1, p.h1, d->c0, d->c1, d->nin,
                                                      d->nout, d->weights, d->bias, d->rgb8);
    NB_LAUNCHED();
    return download(d, rgb8, d->rgb8, px * m->nout);
}

// The brute-force host twin (src/objective.cu:317-380): every plane downloaded and walked site by site in double.
int nntc_b200_objective_check_host(nntc_b200_device* d, const nntc_b200_model* m, int k, const double* per_site,
                                   nntc_b200_objective* r)
{
    const int c0 = m->c0, c1 = m->c1, nout = m->nout, nin = m->nin;
    std::vector<double> acc((size_t)3 * m->nplanes, 0.0);
    auto sample = [](const std::vector<float>& plane, int w, int h, int c, double u, double v, double* out) {
        const double x = u * (double)w - 0.5, y = v * (double)h - 0.5;
        const double xf = std::floor(x), yf = std::floor(y);
        const double fx = x - xf, fy = y - yf;
        const int x0 = clampi((int)xf, w), x1 = clampi((int)xf + 1, w);
        const int y0 = clampi((int)yf, h), y1 = clampi((int)yf + 1, h);
        for (int q = 0; q < c; q++)
        {
            const double a = plane[((size_t)y0 * w + x0) * c + q], b = plane[((size_t)y0 * w + x1) * c + q];
            const double e = plane[((size_t)y1 * w + x0) * c + q], f = plane[((size_t)y1 * w + x1) * c + q];
            out[q] = (1.0 - fx) * (1.0 - fy) * a + fx * (1.0 - fy) * b + (1.0 - fx) * fy * e + fx * fy * f;
        }
    };
    for (int pl = 0; pl < m->nplanes; pl++)
    {
        const DevPlane& dp = d->planes[(size_t)pl];
        std::vector<float> v0((size_t)dp.w0 * dp.h0 * c0), v1((size_t)dp.w1 * dp.h1 * c1),
            src((size_t)dp.w0 * dp.h0 * nout);
        NB_TRY(download(d, v0.data(), dp.v0, v0.size() * sizeof(float)));
        NB_TRY(download(d, v1.data(), dp.v1, v1.size() * sizeof(float)));
        NB_TRY(download(d, src.data(), dp.src, src.size() * sizeof(float)));
        for (int py = 0; py < dp.h0; py++)
            for (int px = 0; px < dp.w0; px++)
                for (int j = 0; j <= k; j++)
                {
                    float dx = 0.0f, dy = 0.0f;
                    if (j > 0)
                        subtexel(k, j - 1, px, py, dx, dy);
                    const double u = ((double)px + 0.5 + (double)dx) / (double)dp.w0;
                    const double v = ((double)py + 0.5 + (double)dy) / (double)dp.h0;
                    double s[MAX_CH], c[MAX_CH], t[MAX_NOUT], phi[MAX_NIN];
                    sample(v1, dp.w1, dp.h1, c1, u, v, c);
                    if (j == 0)
                    {
                        const size_t idx = (size_t)py * dp.w0 + px;
                        for (int i = 0; i < c0; i++)
                            s[i] = v0[idx * c0 + i];
                        for (int i = 0; i < nout; i++)
                            t[i] = src[idx * nout + i];
                    }
                    else
                    {
                        sample(v0, dp.w0, dp.h0, c0, u, v, s);
                        sample(src, dp.w0, dp.h0, nout, u, v, t);
                    }
                    features(s, c0, c, c1, phi);
                    for (int row = 0; row < nout; row++)
                    {
                        double y = (double)m->dec_b[row];
                        for (int i = 0; i < nin; i++)
                            y += (double)m->dec_w[(size_t)row * nin + i] * phi[i];
                        const double e = y - t[row];
                        acc[3 * pl] += (double)m->cw[row] * e * e;
                        acc[3 * pl + (j == 0 ? 1 : 2)] += e * e;
                    }
                }
    }
    *r = nntc_b200_objective{};
    normalise(*m, k, per_site, acc, r);
    return NNTC_B200_OK;
}

}   // extern "C"

// ---- the objective of one caller-owned plane, with no device allocation -------------------------------------------
//
// Who calls this: a host that keeps a plane in device memory it manages itself - the reference's own device model,
// which owns every plane buffer of its chain, or a process whose device memory is already committed to its own arena
// - and wants E of that plane without building a device model. nntc_b200_device_create allocates the whole encode
// workspace of a chain (stencils, CG vectors, partials: tens of GB at 4096 x 4096), and cudaMalloc both blocks the
// device and may simply fail under such a budget. Here the inputs and the three sums are the caller's memory; the only
// scratch is the per-block partials of k_objective, held in a fixed static device array of NOALLOC_MAX_BLOCKS * 3
// doubles (1.5 MiB), which bounds one call at NNTC_B200_NOALLOC_MAX_PIXELS pixels.

namespace nb
{

constexpr long long NOALLOC_MAX_BLOCKS = NNTC_B200_NOALLOC_MAX_PIXELS / OBJ_THREADS;

// Every word a call reads is written earlier in the same call (k_objective writes each block's three partials,
// k_objective_reduce reads only those), so nothing here needs to start at zero.
static __device__ __align__(256) double g_noalloc_partial[3 * NOALLOC_MAX_BLOCKS];

// The scratch's device address on the current device, looked up on every call with that device current: a stored
// address could outlive the context it belongs to (a device reset, another context on the same ordinal), and the
// lookup allocates nothing.
static int noalloc_scratch(double** out)
{
    void* p = nullptr;
    NB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_partial));
    *out = (double*)p;
    return NNTC_B200_OK;
}

// A pointer the kernels may read or write on the current device: device memory of this device, or managed memory.
static int noalloc_pointer(const void* p, const char* name)
{
    if (!p)
    {
        set_error(NNTC_B200_ERR_ARG, std::string("objective_plane_noalloc: ") + name + " is null");
        return NNTC_B200_ERR_ARG;
    }
    cudaPointerAttributes a{};
    NB_CUDA(cudaPointerGetAttributes(&a, p));
    int dev = -1;
    NB_CUDA(cudaGetDevice(&dev));
    const bool ok = a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == dev);
    if (!ok)
    {
        set_error(NNTC_B200_ERR_ARG,
                  std::string("objective_plane_noalloc: ") + name + " is not device memory of the current device");
        return NNTC_B200_ERR_ARG;
    }
    return NNTC_B200_OK;
}

}   // namespace nb

extern "C" int nntc_b200_objective_plane_noalloc(const float* v0, int w0, int h0, int c0, const float* v1, int w1,
                                                 int h1, int c1, const float* src, int nout, const float* weights,
                                                 const float* bias, const float* cw, int nin, int k, double* sums,
                                                 void* stream)
{
    auto bad = [](const std::string& what) {
        set_error(NNTC_B200_ERR_ARG, "objective_plane_noalloc: " + what);
        return (int)NNTC_B200_ERR_ARG;
    };
    if (w0 < 1 || h0 < 1 || w1 < 1 || h1 < 1)
        return bad("plane sizes must be positive");
    if ((long long)w0 * h0 > NNTC_B200_NOALLOC_MAX_PIXELS)
        return bad(std::to_string((long long)w0 * h0) + " pixels is above the limit of " +
                   std::to_string((long long)NNTC_B200_NOALLOC_MAX_PIXELS) + " (its static scratch holds " +
                   std::to_string(NOALLOC_MAX_BLOCKS) + " blocks of " + std::to_string(OBJ_THREADS) + ")");
    if (c0 < 1 || c0 > MAX_CH || c1 < 1 || c1 > MAX_CH)
        return bad("channel counts must be 1.." + std::to_string(MAX_CH));
    if (nout < 1 || nout > MAX_NOUT)
        return bad("nout must be 1.." + std::to_string(MAX_NOUT));
    if (nin != c1 + c0 + c0 * c1)
        return bad("nin must be c1 + c0 + c0 c1");
    if (k != 0 && k != 1 && k != 2 && k != 4)
        return bad("k must be 0, 1, 2 or 4");
    NB_TRY(noalloc_pointer(v0, "v0"));
    NB_TRY(noalloc_pointer(v1, "v1"));
    NB_TRY(noalloc_pointer(src, "src"));
    NB_TRY(noalloc_pointer(weights, "weights"));
    NB_TRY(noalloc_pointer(bias, "bias"));
    NB_TRY(noalloc_pointer(cw, "cw"));
    NB_TRY(noalloc_pointer(sums, "sums"));
    double* partial = nullptr;
    NB_TRY(noalloc_scratch(&partial));

    Planes P{};
    P.n = 1;
    P.c0 = c0;
    P.c1 = c1;
    P.nin = nin;
    P.nout = nout;
    P.kc = k;
    P.c = c0;
    PlaneView& v = P.p[0];
    v.w0 = w0;
    v.h0 = h0;
    v.w1 = w1;
    v.h1 = h1;
    v.src = src;
    v.v0 = const_cast<float*>(v0);   // read only: k_objective writes nothing but its partials
    v.v1 = const_cast<float*>(v1);
    const long long pixels = (long long)w0 * h0;
    P.start[0] = 0;
    P.start[1] = (pixels + OBJ_THREADS - 1) / OBJ_THREADS * OBJ_THREADS;
    const int nblocks = (int)(P.start[1] / OBJ_THREADS);
    const cudaStream_t s = (cudaStream_t)stream;
    k_objective<<<nblocks, OBJ_THREADS, 0, s>>>(P, ObjArgs{ weights, bias, cw, partial });
    NB_LAUNCHED();
    k_objective_reduce<<<1, 256, 0, s>>>(P, partial, nblocks, sums, OBJ_THREADS);
    NB_LAUNCHED();
    return NNTC_B200_OK;
}
