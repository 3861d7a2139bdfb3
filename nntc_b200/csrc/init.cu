// init.cu: the initial state of both latents and their grids (the method of src/init.cu:384-1400), on the device.
//
// - level 0: luma into channel 0 (2 luma - 1), the other channels zero; snapped to the nearest palette entry, or kept
//   continuous under --l0 bc8;
// - level 1, box: each texel the mean of its block of source pixels, channel c from source channel c (2 mean - 1);
//   pca: the block means projected onto the leading principal directions of the base plane's block means, each
//   component divided by its peak over the chain; then one min/max grid over the chain and the snap;
// - --init0 residual: one level-0 channel from the leading principal direction of the decode's residual at the pixel
//   centres (over the base plane, or the chain with each plane's site weight; by texture, the texture whose 3x3 block
//   has the largest leading eigenvalue), divided by the projection's peak (bc8) or its 99th percentile (palette).
//
// Shape on the B200. Nothing of the init leaves the device but the report's few numbers:
// - moments (means and covariance sums) by k_moments: a block stages a tile of rows - block means or decode residuals,
//   formed on the fly, never stored - in shared memory, and each thread owns one entry (a channel sum or one product
//   of the upper triangle) over all of the block's tiles; one partial per block and entry, added in block order;
// - the eigenproblem by k_basis, one block: a parallel (round-robin) Jacobi on the <= 18 x 18 covariance, every
//   disjoint pair of a round rotated at once;
// - projections, peaks (an integer max on the bits of non-negative doubles), the percentile histogram (integer
//   counts) and the seeds by fused kernels that form each pixel's residual in registers; every plane of the chain in
//   one launch where the work is per texel.
//
// What has to be alike, and why: the per-element arithmetic of the seeds (luma weights, block means in row order, the
// decode at the pixel centre, the projection sum, the clamps and roundings) decides quantised values the reference's
// check harness compares; the percentile rule (4096 bins of |p| / peak, the first bin whose running count reaches
// 0.99 of all texels) and the sign rule of init0's direction (its largest entry positive) are the method's. A
// principal direction's sign is not fixed by the method for level 1's pca components (the reference keeps whatever its
// eigen solver returns); here each component gets the same rule as init0's direction.

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "device.cuh"

namespace nb
{

constexpr int MOM_TILE = 128;                                        // rows per staged tile
constexpr int MOM_ENTRIES = MAX_NOUT + MAX_NOUT * (MAX_NOUT + 1) / 2;   // sums, then the upper triangle
constexpr int JM = MAX_NOUT + 1;                                     // the eigen solver's padded order (even)

// What k_basis hands to the projection kernels and back to the host.
struct Basis
{   // 808 bytes; the arena's slice is 1 KB
    double mu[MAX_NOUT];
    double dir[MAX_CH][MAX_NOUT];
    double eig[MAX_CH];
    double total_variance;
    unsigned long long peak_bits[MAX_CH];   // max |projection| per component, as the bits of a non-negative double
    double divisor;
    int texture;
    int bin;
};

static_assert(sizeof(Basis) <= 1024, "the arena's basis slice holds one Basis");

// ---- level 0 -----------------------------------------------------------------------------------------------------

struct SeedArgs
{
    float luma[3];
    int luma_channel0;
    int palette_mode;
    int levels[MAX_CH];
    const float* palette;
};

__global__ void k_seed_level0(Planes P, SeedArgs A)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int pl = plane_of(P, i);
    const PlaneView& V = P.p[pl];
    const long long t = i - P.start[pl];
    if (t >= (long long)V.w0 * V.h0)
        return;
    const float* s = V.src + t * P.nout;
    const float luma = A.luma[0] * s[0] + A.luma[1] * s[1] + A.luma[2] * s[2];
    for (int c = 0; c < P.c0; c++)
    {
        const float want = (c == 0 && A.luma_channel0) ? 2.0f * luma - 1.0f : 0.0f;
        int k = 0;
        float v = want;
        if (A.palette_mode)
        {
            // the nearest entry of the channel's palette, the first of equals
            const float* pal = A.palette + c * 16;
            float gap = fabsf(pal[0] - want);
            for (int j = 1; j <= A.levels[c]; j++)
            {
                const float g = fabsf(pal[j] - want);
                k = g < gap ? j : k;
                gap = g < gap ? g : gap;
            }
            v = pal[k];
        }
        V.v0[t * P.c0 + c] = v;
        V.k0[t * P.c0 + c] = (uint8_t)k;
    }
}

// ---- level 1: block means ----------------------------------------------------------------------------------------

// Source pixels [x w0 / w1, (x + 1) w0 / w1) of level-1 column x (at least one), and the same in y.
__host__ __device__ __forceinline__ void block_span(int x, int w0, int w1, int& a, int& b)
{
    a = (int)((long long)x * w0 / w1);
    b = (int)((long long)(x + 1) * w0 / w1);
    if (b <= a)
        b = a + 1;
    b = b > w0 ? w0 : b;
}

// The mean of the first n source channels over level-1 texel t's block, summed in row order.
__device__ __forceinline__ void block_mean(const float* src, int w0, int h0, int nout, int w1, int h1, size_t t,
                                           int n, float* out)
{
    int xa, xb, ya, yb;
    block_span((int)(t % (size_t)w1), w0, w1, xa, xb);
    block_span((int)(t / (size_t)w1), h0, h1, ya, yb);
    for (int c = 0; c < n; c++)
        out[c] = 0.0f;
    for (int y = ya; y < yb; y++)
        for (int x = xa; x < xb; x++)
        {
            const float* s = src + ((size_t)y * w0 + x) * nout;
            for (int c = 0; c < n; c++)
                out[c] += s[c];
        }
    const int count = (xb - xa) * (yb - ya);
    const float inv = count > 0 ? 1.0f / (float)count : 0.0f;
    for (int c = 0; c < n; c++)
        out[c] *= inv;
}

__global__ void k_box_level1(Planes P)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int pl = plane_of(P, i);
    const PlaneView& V = P.p[pl];
    const long long t = i - P.start[pl];
    if (t >= (long long)V.w1 * V.h1)
        return;
    const int c1 = P.c1, n = c1 < P.nout ? c1 : P.nout;
    float m[MAX_CH];
    block_mean(V.src, V.w0, V.h0, P.nout, V.w1, V.h1, (size_t)t, n, m);
    for (int c = 0; c < c1; c++)
        V.v1[t * c1 + c] = c < n ? 2.0f * m[c] - 1.0f : 0.0f;
}

// ---- rows for the moments -----------------------------------------------------------------------------------------

struct MeanRows
{
    const float* src;
    int w0, h0, w1, h1, nout;
    __device__ void row(size_t t, float* out) const { block_mean(src, w0, h0, nout, w1, h1, t, nout, out); }
};

// The decode's residual at pixel t's centre: level 0 read nearest, level 1 bilinear at the centre, minus the source.
struct ResidualRows
{
    float* v0;
    uint8_t* k0;
    const float *v1, *src, *weights, *bias;
    int w0, h0, w1, h1, c0, c1, nin, nout;
    __device__ void row(size_t t, float* out) const
    {
        const int px = (int)(t % (size_t)w0), py = (int)(t / (size_t)w0);
        float s[MAX_CH], c[MAX_CH], phi[MAX_NIN];
        for (int i = 0; i < c0; i++)
            s[i] = v0[t * c0 + i];
        blend<MAX_CH>(v1, w1, c1, tap_at(px, py, 0.0f, 0.0f, w0, h0, w1, h1), c);
        features(s, c0, c, c1, phi);
        for (int r = 0; r < nout; r++)
        {
            const float* wr = weights + (size_t)r * nin;
            float dec = bias[r];
            for (int i = 0; i < nin; i++)
                dec += wr[i] * phi[i];
            out[r] = dec - src[t * nout + r];
        }
    }
};

// Entry e of the moments: e < nout the sum of channel e, then the products (a, b), a <= b, row by row.
__host__ __device__ inline void moment_pair(int e, int nout, int& a, int& b)
{
    int k = e - nout;
    a = 0;
    while (k >= nout - a)
    {
        k -= nout - a;
        a++;
    }
    b = a + k;
}

// partial[e][block] (COV_GRID blocks) = weight x the block's sum of entry e, added to what is there when `accumulate`.
template <class Rows>
__global__ void __launch_bounds__(256) k_moments(Rows R, size_t count, int nout, double weight, int accumulate,
                                                 double* partial)
{
    __shared__ float rows[MOM_TILE][MAX_NOUT + 1];
    const int entries = nout + nout * (nout + 1) / 2;
    const int e = threadIdx.x;
    int a = 0, b = 0;
    if (e >= nout && e < entries)
        moment_pair(e, nout, a, b);
    double acc = 0.0;
    for (size_t start = (size_t)blockIdx.x * MOM_TILE; start < count; start += (size_t)gridDim.x * MOM_TILE)
    {
        __syncthreads();
        for (int r = threadIdx.x; r < MOM_TILE; r += blockDim.x)
        {
            if (start + r < count)
                R.row(start + r, rows[r]);
            else
                for (int c = 0; c < nout; c++)
                    rows[r][c] = 0.0f;   // a padded row adds exact zeros
        }
        __syncthreads();
        if (e < nout)
            for (int r = 0; r < MOM_TILE; r++)
                acc += (double)rows[r][e];
        else if (e < entries)
            for (int r = 0; r < MOM_TILE; r++)
                acc += (double)rows[r][a] * (double)rows[r][b];
    }
    if (e < entries)
    {
        double* slot = partial + (size_t)e * COV_GRID + blockIdx.x;
        *slot = accumulate ? *slot + weight * acc : weight * acc;
    }
}

// ---- the basis: covariance, eigenproblem, choice of directions ---------------------------------------------------

// Parallel Jacobi on the symmetric n x n matrix A (shared, padded to an even order m with zero rows): every round
// rotates m / 2 disjoint pairs at once, the pairs of a round-robin tournament, m - 1 rounds a sweep. V accumulates the
// rotations. Every thread of the block calls it.
__device__ void jacobi_block(double (*A)[JM], double (*V)[JM], int n, double* cs, double* sn, double* red)
{
    const int m = n + (n & 1), half = m / 2, tid = threadIdx.x;
    for (int e = tid; e < JM * JM; e += blockDim.x)
    {
        const int i = e / JM, j = e % JM;
        V[i][j] = i == j ? 1.0 : 0.0;
        if (i >= n || j >= n)
            A[i][j] = 0.0;
    }
    __syncthreads();
    for (int sweep = 0; sweep < 64; sweep++)
    {
        if (tid == 0)
        {
            double off = 0.0, diag = 0.0;
            for (int p = 0; p < n; p++)
            {
                diag += A[p][p] * A[p][p];
                for (int q = p + 1; q < n; q++)
                    off += A[p][q] * A[p][q];
            }
            red[0] = off <= 1e-30 * diag || off == 0.0 ? 1.0 : 0.0;
        }
        __syncthreads();
        if (red[0] != 0.0)
            break;
        for (int round = 0; round < m - 1; round++)
        {
            // pair k of this round: the fixed player m - 1 meets player `round`; the others meet symmetrically
            if (tid < half)
            {
                int p = tid == 0 ? m - 1 : (round + tid) % (m - 1);
                int q = tid == 0 ? round : (round - tid + (m - 1)) % (m - 1);
                if (p > q)
                {
                    const int x = p;
                    p = q;
                    q = x;
                }
                double c = 1.0, s = 0.0;
                const double apq = A[p][q];
                if (apq != 0.0)
                {
                    const double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
                    const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    c = 1.0 / sqrt(t * t + 1.0);
                    s = t * c;
                }
                cs[tid] = c;
                sn[tid] = s;
                red[2 + 2 * tid] = p;
                red[3 + 2 * tid] = q;
            }
            __syncthreads();
            // columns: A <- A G, V <- V G
            for (int w = tid; w < half * m; w += blockDim.x)
            {
                const int k = w / half, pr = w % half;
                const int p = (int)red[2 + 2 * pr], q = (int)red[3 + 2 * pr];
                const double c = cs[pr], s = sn[pr];
                const double akp = A[k][p], akq = A[k][q];
                A[k][p] = c * akp - s * akq;
                A[k][q] = s * akp + c * akq;
                const double vkp = V[k][p], vkq = V[k][q];
                V[k][p] = c * vkp - s * vkq;
                V[k][q] = s * vkp + c * vkq;
            }
            __syncthreads();
            // rows: A <- G^T A
            for (int w = tid; w < half * m; w += blockDim.x)
            {
                const int k = w / half, pr = w % half;
                const int p = (int)red[2 + 2 * pr], q = (int)red[3 + 2 * pr];
                const double c = cs[pr], s = sn[pr];
                const double apk = A[p][k], aqk = A[q][k];
                A[p][k] = c * apk - s * aqk;
                A[q][k] = s * apk + c * aqk;
            }
            __syncthreads();
        }
    }
}

struct BasisArgs
{
    int nout;
    int mode;         // 0: level 1's leading `components` directions; 1: init0's leading direction; 2: init0 by texture
    int components;
    int textures;
    double count;     // the (weighted) number of rows the moments summed
};

// A direction with its largest entry (the first of equals in magnitude) made positive.
__device__ void sign_rule(double* u, int n)
{
    int big = 0;
    for (int r = 1; r < n; r++)
        if (fabs(u[r]) > fabs(u[big]))
            big = r;
    if (u[big] < 0.0)
        for (int r = 0; r < n; r++)
            u[r] = -u[r];
}

__global__ void __launch_bounds__(256) k_basis(const double* partial, BasisArgs a, Basis* out)
{
    __shared__ double raw[MOM_ENTRIES];
    __shared__ double C[JM][JM], A[JM][JM], V[JM][JM];
    __shared__ double cs[JM / 2 + 1], sn[JM / 2 + 1], red[2 + JM + 2];
    __shared__ double mu[MAX_NOUT];
    const int nout = a.nout, tid = threadIdx.x;
    const int entries = nout + nout * (nout + 1) / 2;
    for (int e = tid; e < entries; e += blockDim.x)
    {
        double s = 0.0;
        for (int b = 0; b < COV_GRID; b++)
            s += partial[(size_t)e * COV_GRID + b];
        raw[e] = s;
    }
    __syncthreads();
    if (tid < nout)
        mu[tid] = a.count > 0.0 ? raw[tid] / a.count : 0.0;
    __syncthreads();
    for (int e = nout + tid; e < entries; e += blockDim.x)
    {
        int p, q;
        moment_pair(e, nout, p, q);
        const double v = (a.count > 0.0 ? raw[e] / a.count : 0.0) - mu[p] * mu[q];
        C[p][q] = v;
        C[q][p] = v;
    }
    for (int e = tid; e < MAX_NOUT; e += blockDim.x)
        out->mu[e] = e < nout ? mu[e] : 0.0;
    __syncthreads();
    if (tid == 0)
    {
        double tv = 0.0;
        for (int r = 0; r < nout; r++)
            tv += C[r][r];
        out->total_variance = tv;
        out->texture = -1;
        for (int j = 0; j < MAX_CH; j++)
            out->peak_bits[j] = 0ull;
    }
    if (a.mode < 2)
    {
        for (int e = tid; e < JM * JM; e += blockDim.x)
            A[e / JM][e % JM] = C[e / JM][e % JM];
        __syncthreads();
        jacobi_block(A, V, nout, cs, sn, red);
        if (tid == 0)
        {
            // the leading directions by eigenvalue, largest first (the first index of equals)
            bool used[JM] = {};
            const int take = a.mode == 0 ? a.components : 1;
            for (int j = 0; j < take; j++)
            {
                int top = -1;
                for (int i = 0; i < nout; i++)
                    if (!used[i] && (top < 0 || A[i][i] > A[top][top]))
                        top = i;
                used[top] = true;
                double u[MAX_NOUT];
                for (int r = 0; r < nout; r++)
                    u[r] = V[r][top];
                sign_rule(u, nout);
                for (int r = 0; r < MAX_NOUT; r++)
                    out->dir[j][r] = r < nout ? u[r] : 0.0;
                out->eig[j] = A[top][top];
            }
        }
    }
    else
    {
        // by texture: the 3x3 block of each texture's own channels, the texture whose leading eigenvalue is largest
        __shared__ double best_value, best_vec[3];
        __shared__ int best_t;
        if (tid == 0)
        {
            best_value = -1.0;
            best_t = 0;
        }
        for (int t = 0; t < a.textures; t++)
        {
            __syncthreads();
            for (int e = tid; e < JM * JM; e += blockDim.x)
            {
                const int i = e / JM, j = e % JM;
                A[i][j] = i < 3 && j < 3 ? C[3 * t + i][3 * t + j] : 0.0;
            }
            __syncthreads();
            jacobi_block(A, V, 3, cs, sn, red);
            if (tid == 0)
            {
                int top = 0;
                for (int i = 1; i < 3; i++)
                    if (A[i][i] > A[top][top])
                        top = i;
                if (A[top][top] > best_value)
                {
                    best_value = A[top][top];
                    best_t = t;
                    for (int r = 0; r < 3; r++)
                        best_vec[r] = V[r][top];
                }
            }
        }
        __syncthreads();
        if (tid == 0)
        {
            double u[MAX_NOUT];
            for (int r = 0; r < nout; r++)
                u[r] = 0.0;
            for (int r = 0; r < 3; r++)
                u[3 * best_t + r] = best_vec[r];
            sign_rule(u, nout);
            for (int r = 0; r < MAX_NOUT; r++)
                out->dir[0][r] = r < nout ? u[r] : 0.0;
            out->eig[0] = best_value > 0.0 ? best_value : 0.0;
            out->texture = best_t;
        }
    }
}

__device__ __forceinline__ double project(const float* row, const Basis& B, int j, int nout)
{
    double acc = 0.0;
    for (int r = 0; r < nout; r++)
        acc += B.dir[j][r] * ((double)row[r] - B.mu[r]);
    return acc;
}

__device__ __forceinline__ void peak_max(unsigned long long* bits, double v)
{
    atomicMax(bits, (unsigned long long)__double_as_longlong(v));   // v >= 0: the bits order as the values
}

// ---- level 1 pca: projections, peaks, normalisation ---------------------------------------------------------------

__global__ void k_pca_project(Planes P, Basis* B, int components)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int pl = plane_of(P, i);
    const PlaneView& V = P.p[pl];
    const long long t = i - P.start[pl];
    if (t >= (long long)V.w1 * V.h1)
        return;
    float m[MAX_NOUT];
    block_mean(V.src, V.w0, V.h0, P.nout, V.w1, V.h1, (size_t)t, P.nout, m);
    for (int j = 0; j < P.c1; j++)
    {
        const double p = j < components ? project(m, *B, j, P.nout) : 0.0;
        V.v1[t * P.c1 + j] = (float)p;
        if (j < components)
            peak_max(&B->peak_bits[j], fabs(p));
    }
}

__global__ void k_pca_normalise(Planes P, const Basis* __restrict__ B)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int pl = plane_of(P, i);
    const PlaneView& V = P.p[pl];
    const long long t = i - P.start[pl];
    if (t >= (long long)V.w1 * V.h1)
        return;
    for (int j = 0; j < P.c1; j++)
    {
        const double peak = __longlong_as_double((long long)B->peak_bits[j]);
        if (!(peak > 0.0))
            continue;
        const double v = (double)V.v1[t * P.c1 + j] * (1.0 / peak);
        V.v1[t * P.c1 + j] = (float)(v < -1.0 ? -1.0 : (v > 1.0 ? 1.0 : v));
    }
}

// ---- init0: peak, percentile histogram, divisor, seed -------------------------------------------------------------

enum ResidualPass
{
    RP_PEAK = 0,
    RP_HIST,
    RP_SEED
};

struct ResidualPassArgs
{
    int channel, levels, palette_mode;
    const float* palette;
    unsigned long long* hist;
};

template <int PASS>
__global__ void k_residual_pass(ResidualRows R, size_t texels, Basis* B, ResidualPassArgs a)
{
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (PASS == RP_PEAK)
    {
        // the largest |projection|: each warp's maximum first (a maximum is the same whatever the order), then one
        // atomic per warp - one per texel had every texel of the chain contend for one address
        unsigned long long bits = 0ull;   // |p| >= 0: the bits order as the values
        if (t < texels)
        {
            float row[MAX_NOUT];
            R.row(t, row);
            bits = (unsigned long long)__double_as_longlong(fabs(project(row, *B, 0, R.nout)));
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
        {
            const unsigned long long x = __shfl_xor_sync(0xffffffffu, bits, o);
            bits = x > bits ? x : bits;
        }
        if ((threadIdx.x & 31) == 0 && bits != 0ull)
            atomicMax(&B->peak_bits[0], bits);
        return;
    }
    if (t >= texels)
        return;
    float row[MAX_NOUT];
    R.row(t, row);
    const double p = project(row, *B, 0, R.nout);
    if (PASS == RP_HIST)
    {
        const double peak = __longlong_as_double((long long)B->peak_bits[0]);
        if (!(peak > 0.0))
            return;
        int b = (int)(fabs(p) * (1.0 / peak) * (double)HIST_BINS);
        b = b < 0 ? 0 : (b >= HIST_BINS ? HIST_BINS - 1 : b);
        atomicAdd(a.hist + b, 1ull);
    }
    else
    {
        const double inv = B->divisor > 0.0 ? 1.0 / B->divisor : 0.0;
        const double q = p * inv;
        const float value = (float)(q < -1.0 ? -1.0 : (q > 1.0 ? 1.0 : q));
        float* v0 = R.v0;
        if (a.palette_mode)
        {
            int k = (int)lroundf((value + 1.0f) * 0.5f * (float)a.levels);
            k = k < 0 ? 0 : (k > a.levels ? a.levels : k);
            v0[t * R.c0 + a.channel] = a.palette[a.channel * 16 + k];
            R.k0[t * R.c0 + a.channel] = (uint8_t)k;
        }
        else
            v0[t * R.c0 + a.channel] = value;
    }
}

// The divisor: the peak under bc8; under palette the peak scaled to the first histogram bin whose running count
// reaches 0.99 of every texel of the chain (the peak again if that is not positive).
__global__ void __launch_bounds__(256) k_divisor(Basis* B, const unsigned long long* hist, unsigned long long total,
                                                 int use_hist)
{
    __shared__ unsigned long long part[256];
    __shared__ int first;
    const int tid = threadIdx.x, per = HIST_BINS / 256;
    const double peak = __longlong_as_double((long long)B->peak_bits[0]);
    if (!use_hist || !(peak > 0.0))
    {
        if (tid == 0)
        {
            B->divisor = peak;
            B->bin = HIST_BINS - 1;
        }
        return;
    }
    unsigned long long s = 0ull;
    for (int b = 0; b < per; b++)
        s += hist[tid * per + b];
    part[tid] = s;
    if (tid == 0)
        first = HIST_BINS - 1;
    __syncthreads();
    if (tid == 0)
    {
        unsigned long long run = 0ull;
        for (int i = 0; i < 256; i++)
        {
            const unsigned long long x = part[i];
            part[i] = run;   // exclusive prefix
            run += x;
        }
    }
    __syncthreads();
    const unsigned long long want = (unsigned long long)(0.99 * (double)total);
    unsigned long long run = part[tid];
    for (int b = 0; b < per; b++)
    {
        run += hist[tid * per + b];
        if (run >= want)
        {
            atomicMin(&first, tid * per + b);
            break;
        }
    }
    __syncthreads();
    if (tid == 0)
    {
        double d = peak * (double)(first + 1) / (double)HIST_BINS;
        B->divisor = d > 0.0 ? d : peak;
        B->bin = first;
    }
}

// ---- grids --------------------------------------------------------------------------------------------------------

__global__ void k_snap(float* v, uint8_t* k, size_t n, int c, int bits, const float* lo, const float* hi)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int ch = (int)(i % (size_t)c);
    const int q = grid_index(lo[ch], hi[ch], bits, v[i]);
    v[i] = grid_value(lo[ch], hi[ch], bits, q);
    k[i] = (uint8_t)q;
}

int fit_grid_device(nntc_b200_device* d, int level0, bool pct, float* lo, float* hi);

// Fit the latent's grid over the chain where the device holds it (when `fit`), then snap every plane onto it.
static int fit_and_snap(nntc_b200_device* d, nntc_b200_model* m, int level0, bool pct, uint8_t* const* k_out, bool fit)
{
    const int nc = level0 ? d->c0 : d->c1;
    if (fit)
    {
        float lo[MAX_CH], hi[MAX_CH];
        NB_TRY(fit_grid_device(d, level0, pct, lo, hi));
        for (int c = 0; c < nc; c++)
        {
            if (!(hi[c] > lo[c]))
            {
                lo[c] = -1.0f;
                hi[c] = 1.0f;
            }
            (level0 ? m->lo0 : m->lo1)[c] = lo[c];
            (level0 ? m->hi0 : m->hi1)[c] = hi[c];
        }
        (level0 ? m->has_lo0 : m->has_lo1) = 1;
        NB_TRY(upload_grids(d, m));
    }
    for (size_t i = 0; i < d->planes.size(); i++)
    {
        const DevPlane& p = d->planes[i];
        const size_t n = level0 ? (size_t)p.w0 * p.h0 * d->c0 : (size_t)p.w1 * p.h1 * d->c1;
        uint8_t* k = level0 ? p.k0 : p.k1;
        k_snap<<<grid_for(n, 256), 256, 0, d->stream>>>(level0 ? p.v0 : p.v1, k, n, nc, level0 ? 8 : m->bits1,
                                                        level0 ? d->lo0 : d->lo1, level0 ? d->hi0 : d->hi1);
        NB_LAUNCHED();
        if (k_out && k_out[i])
            NB_CUDA(cudaMemcpyAsync(k_out[i], k, n, cudaMemcpyDeviceToHost, d->stream));
    }
    NB_CUDA(cudaStreamSynchronize(d->stream));
    return NNTC_B200_OK;
}

static ResidualRows residual_rows(const nntc_b200_device* d, const DevPlane& p)
{
    ResidualRows R{};
    R.v0 = p.v0;
    R.k0 = p.k0;
    R.v1 = p.v1;
    R.src = p.src;
    R.weights = d->weights;
    R.bias = d->bias;
    R.w0 = p.w0;
    R.h0 = p.h0;
    R.w1 = p.w1;
    R.h1 = p.h1;
    R.c0 = d->c0;
    R.c1 = d->c1;
    R.nin = d->nin;
    R.nout = d->nout;
    return R;
}

}   // namespace nb

using namespace nb;

extern "C"
{

int nntc_b200_init_level0(nntc_b200_device* d, const nntc_b200_model* m, const float luma[3], int luma_channel0,
                          uint8_t* const* k0_out)
{
    NB_TRY(upload_grids(d, m));
    SeedArgs A{};
    for (int i = 0; i < 3; i++)
        A.luma[i] = luma[i];
    A.luma_channel0 = luma_channel0 ? 1 : 0;
    A.palette_mode = m->l0_bc8 ? 0 : 1;
    for (int c = 0; c < d->c0; c++)
        A.levels[c] = (1 << m->bits0[c]) - 1;
    A.palette = d->palette;
    Planes P = planes_for(d, 1, [&](int i) { return (size_t)d->planes[(size_t)i].w0 * d->planes[(size_t)i].h0; });
    k_seed_level0<<<(unsigned)(P.start[P.n] / THREADS), THREADS, 0, d->stream>>>(P, A);
    NB_LAUNCHED();
    for (size_t i = 0; i < d->planes.size(); i++)
        if (k0_out && k0_out[i])
            NB_CUDA(cudaMemcpyAsync(k0_out[i], d->planes[i].k0, (size_t)d->planes[i].w0 * d->planes[i].h0 * d->c0,
                                    cudaMemcpyDeviceToHost, d->stream));
    NB_CUDA(cudaStreamSynchronize(d->stream));
    return NNTC_B200_OK;
}

int nntc_b200_init_level1(nntc_b200_device* d, nntc_b200_model* m, int pca, nntc_b200_init1_report* rep,
                          uint8_t* const* k1_out)
{
    *rep = nntc_b200_init1_report{};
    rep->pca = pca;
    const int nout = d->nout;
    Planes P = planes_for(d, 0, [&](int i) { return (size_t)d->planes[(size_t)i].w1 * d->planes[(size_t)i].h1; });
    const unsigned blocks = (unsigned)(P.start[P.n] / THREADS);
    if (!pca)
    {
        k_box_level1<<<blocks, THREADS, 0, d->stream>>>(P);
        NB_LAUNCHED();
        return fit_and_snap(d, m, 0, false, k1_out, true);
    }
    // the basis from the base plane's block means, then every plane projected onto it, on the device
    const DevPlane& base = d->planes[0];
    const size_t count = (size_t)base.w1 * base.h1;
    MeanRows R{ base.src, base.w0, base.h0, base.w1, base.h1, nout };
    k_moments<MeanRows><<<COV_GRID, 256, 0, d->stream>>>(R, count, nout, 1.0, 0, d->cov);
    NB_LAUNCHED();
    BasisArgs a{};
    a.nout = nout;
    a.mode = 0;
    a.components = d->c1 < nout ? d->c1 : nout;
    a.textures = m->textures;
    a.count = (double)count;
    Basis* B = reinterpret_cast<Basis*>(d->basis);
    k_basis<<<1, 256, 0, d->stream>>>(d->cov, a, B);
    NB_LAUNCHED();
    k_pca_project<<<blocks, THREADS, 0, d->stream>>>(P, B, a.components);
    NB_LAUNCHED();
    k_pca_normalise<<<blocks, THREADS, 0, d->stream>>>(P, B);
    NB_LAUNCHED();
    Basis h;
    NB_TRY(download(d, &h, B, sizeof(h)));
    rep->components = a.components;
    rep->total_variance = h.total_variance;
    for (int j = 0; j < a.components && j < MAX_CH; j++)
    {
        rep->eigenvalue[j] = h.eig[j];
        double peak;
        std::memcpy(&peak, &h.peak_bits[j], sizeof(peak));
        rep->peak[j] = peak;
    }
    return fit_and_snap(d, m, 0, false, k1_out, true);
}

int nntc_b200_init0_residual_channel(nntc_b200_device* d, const nntc_b200_model* m, int channel,
                                     const double* plane_weight, nntc_b200_init0_report* rep, uint8_t* const* k0_io)
{
    if (channel < 0 || channel >= d->c0)
    {
        set_error(NNTC_B200_ERR_ARG, "init0 channel out of range");
        return NNTC_B200_ERR_ARG;
    }
    const int nout = d->nout;
    *rep = nntc_b200_init0_report{};
    rep->nout = nout;
    rep->texture = -1;
    // the residual's moments: the base plane, or every plane of the chain with its site weight
    double count = 0.0;
    int used = 0;
    const size_t scope = m->init0_chain ? d->planes.size() : 1;
    for (size_t i = 0; i < scope; i++)
    {
        const DevPlane& p = d->planes[i];
        const double w = m->init0_chain ? plane_weight[i] : 1.0;
        if (!(w > 0.0))
            continue;
        const size_t texels = (size_t)p.w0 * p.h0;
        k_moments<ResidualRows><<<COV_GRID, 256, 0, d->stream>>>(residual_rows(d, p), texels, nout, w, used ? 1 : 0,
                                                                 d->cov);
        NB_LAUNCHED();
        count += w * (double)texels;
        used++;
    }
    if (!used)
        NB_CUDA(cudaMemsetAsync(d->cov, 0, (size_t)MOM_ENTRIES * COV_GRID * sizeof(double), d->stream));
    BasisArgs a{};
    a.nout = nout;
    a.mode = m->init0_texture ? 2 : 1;
    a.components = 1;
    a.textures = m->textures;
    a.count = count;
    Basis* B = reinterpret_cast<Basis*>(d->basis);
    k_basis<<<1, 256, 0, d->stream>>>(d->cov, a, B);
    NB_LAUNCHED();
    // the projection's peak, the percentile (palette), then the seed, every plane of the chain
    ResidualPassArgs ra{};
    ra.channel = channel;
    ra.levels = m->l0_bc8 ? 255 : (1 << m->bits0[channel]) - 1;
    ra.palette_mode = m->l0_bc8 ? 0 : 1;
    ra.palette = d->palette;
    ra.hist = d->hist;
    unsigned long long total = 0ull;
    for (const DevPlane& p : d->planes)
    {
        const size_t texels = (size_t)p.w0 * p.h0;
        k_residual_pass<RP_PEAK><<<grid_for(texels, 256), 256, 0, d->stream>>>(residual_rows(d, p), texels, B, ra);
        NB_LAUNCHED();
        total += texels;
    }
    if (!m->l0_bc8)
    {
        NB_CUDA(cudaMemsetAsync(d->hist, 0, HIST_BINS * sizeof(unsigned long long), d->stream));
        for (const DevPlane& p : d->planes)
        {
            const size_t texels = (size_t)p.w0 * p.h0;
            k_residual_pass<RP_HIST><<<grid_for(texels, 256), 256, 0, d->stream>>>(residual_rows(d, p), texels, B,
                                                                                     ra);
            NB_LAUNCHED();
        }
    }
    k_divisor<<<1, 256, 0, d->stream>>>(B, d->hist, total, m->l0_bc8 ? 0 : 1);
    NB_LAUNCHED();
    for (size_t i = 0; i < d->planes.size(); i++)
    {
        const DevPlane& p = d->planes[i];
        const size_t texels = (size_t)p.w0 * p.h0;
        k_residual_pass<RP_SEED><<<grid_for(texels, 256), 256, 0, d->stream>>>(residual_rows(d, p), texels, B, ra);
        NB_LAUNCHED();
        if (!m->l0_bc8 && k0_io && k0_io[i])
            NB_CUDA(cudaMemcpyAsync(k0_io[i], p.k0, texels * d->c0, cudaMemcpyDeviceToHost, d->stream));
    }
    Basis h;
    NB_TRY(download(d, &h, B, sizeof(h)));
    rep->eigenvalue = h.eig[0];
    rep->total_variance = h.total_variance;
    rep->share = h.total_variance > 0.0 ? h.eig[0] / h.total_variance : 0.0;
    std::memcpy(&rep->peak, &h.peak_bits[0], sizeof(double));
    rep->divisor = h.divisor;
    rep->texture = h.texture;
    for (int r = 0; r < nout; r++)
        rep->dir[r] = h.dir[0][r];
    return NNTC_B200_OK;
}

int nntc_b200_quantise_level1(nntc_b200_device* d, nntc_b200_model* m, int range_pct, uint8_t* const* k1_out)
{
    return fit_and_snap(d, m, 0, range_pct != 0, k1_out, true);
}

int nntc_b200_freeze_level1_grid(nntc_b200_device* d, nntc_b200_model* m, int range_pct, uint8_t* const* k1_out)
{
    return fit_and_snap(d, m, 0, range_pct != 0, k1_out, true);
}

static int level0_grid(nntc_b200_device* d, nntc_b200_model* m, int range_pct, uint8_t* const* k0_out, bool fit)
{
    if (!d->l0_bc8)
    {
        set_error(NNTC_B200_ERR_STATE, "level 0 has a grid only under --l0 bc8");
        return NNTC_B200_ERR_STATE;
    }
    return fit_and_snap(d, m, 1, range_pct != 0, k0_out, fit);
}

int nntc_b200_quantise_level0(nntc_b200_device* d, nntc_b200_model* m, int range_pct, uint8_t* const* k0_out)
{
    return level0_grid(d, m, range_pct, k0_out, true);
}

int nntc_b200_freeze_level0_grid(nntc_b200_device* d, nntc_b200_model* m, int range_pct, uint8_t* const* k0_out)
{
    return level0_grid(d, m, range_pct, k0_out, true);
}

int nntc_b200_snap_level0_on_grid(nntc_b200_device* d, const nntc_b200_model* m, uint8_t* const* k0_out)
{
    nntc_b200_model copy = *m;
    return level0_grid(d, &copy, 0, k0_out, false);
}

}   // extern "C"
