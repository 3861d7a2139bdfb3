// decoder.cu: block (a), the decoder as one global least squares (src/solve_decoder.cu:1-458).
//
// With v = [phi ; 1] (mm = nin + 1) and the target t, the normal equations are A = sum omega v v^T (upper triangle)
// and rhs_c = sum omega v t_c; W and b follow by Gauss-Jordan with the ridge ladder {1e-9, 1e-12, 0} mean(diag A)
// and the acceptance test on the objective's own quadratic Q (src/solve_decoder.cu:184-458), on the host.
//
// The accumulation, B200 shape: every product is a float times a float, exact in double, and the entries needed are
// blocks of the Gram of Z = [phi | 1 | t] over all sites, so they run on the FP64 tensor cores (k_ls_accumulate_mma
// below). Every plane of the chain is in the one launch (grid.y is the plane); each block writes one partial per
// entry, and a second kernel adds, per entry, the planes in index order with their site weight omega and the blocks
// in index order (src/solve_decoder.cu:165-180): deterministic.

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "device.cuh"

namespace nb
{


__host__ __device__ inline int tri_index(int i, int j, int mm)
{
    return i * mm - i * (i - 1) / 2 + (j - i);
}

struct LsArgs
{
    double* partial;   // [plane][entry][LS_GRID]
    int entries;
};

// ---- the accumulation on the FP64 tensor cores
//
// Z = [phi (nin) | 1 | t (nout) | 0 ...] per site, 48 columns in six blocks of eight, and every product the normal
// equations need is an entry of the 48 x 48 Gram Z^T Z: A from its upper-left mm x mm corner, the right-hand sides
// from the columns after it. The 18 upper block pairs (I <= J, I < 4) of the Gram are accumulated with the FP64
// tensor-core MMA (m8n8k4: an 8x4 slice of Z_I^T times a 4x8 slice of Z_J, four sites per step, every product exact
// in double since both factors are floats). One block stages 128 sites' rows of Z; each of its four warps
// takes 32 of them and keeps all 18 tiles in registers over all of its chunks; the warps' tiles are added in warp
// order and each block writes one partial per entry, folded across blocks by k_ls_reduce in block order:
// deterministic.

constexpr int NE_THREADS = 128;
constexpr int NE_WARPS = NE_THREADS / 32;
constexpr int NE_STRIDE = 57;    // floats per staged site: 48 columns; an odd stride keeps the staging stores (one
                                 // row per lane) conflict-free, and 57 = 25 (mod 32) spreads the four sites of one
                                 // fragment load over the banks
constexpr int NE_TILES = 18;     // block pairs I <= J of six blocks with I <= 3: the rows a < mm <= 25 the system
                                 // reads (pairs of two target blocks are never needed)

__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

__host__ __device__ constexpr int tile_i(int t)
{
    return t < 6 ? 0 : (t < 11 ? 1 : (t < 15 ? 2 : (t < 18 ? 3 : (t < 20 ? 4 : 5))));
}
__host__ __device__ constexpr int tile_j(int t)
{
    return t < 6 ? t : (t < 11 ? t - 5 : (t < 15 ? t - 9 : (t < 18 ? t - 12 : (t < 20 ? t - 14 : 5))));
}

__global__ void __launch_bounds__(NE_THREADS, 4) k_ls_accumulate_mma(Planes P, LsArgs A)
{
    extern __shared__ double ne_sh[];
    float* sz = (float*)ne_sh;   // [site][NE_STRIDE] floats; after the chunks, the warps' tiles as doubles
    const int pl = blockIdx.y;
    const PlaneView& V = P.p[pl];
    const int c0 = P.c0, c1 = P.c1, nin = P.nin, nout = P.nout, kc = P.kc, mm = nin + 1;
    const int per_pixel = 1 + kc;
    const size_t sites = (size_t)V.w0 * V.h0 * per_pixel;
    const size_t chunks = (sites + NE_THREADS - 1) / NE_THREADS;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double acc[NE_TILES][2];
#pragma unroll
    for (int t = 0; t < NE_TILES; t++)
    {
        acc[t][0] = 0.0;
        acc[t][1] = 0.0;
    }

    for (size_t chunk = blockIdx.x; chunk < chunks; chunk += gridDim.x)
    {
        const size_t si = chunk * NE_THREADS + tid;
        __syncthreads();   // the previous chunk's fragments have been read
        float* row = sz + tid * NE_STRIDE;
        // the site's row of Z with the solver's arithmetic (src/sample.cuh:154-178); a site outside the plane stages
        // zeros
        int q = 0;
        if (si < sites)
        {
            const size_t pixel = si / (size_t)per_pixel;
            const int j = (int)(si % (size_t)per_pixel);
            const int px = (int)(pixel % (size_t)V.w0), py = (int)(pixel / (size_t)V.w0);
            float dx, dy;
            site_offset(kc, j, px, py, dx, dy);
            float s[MAX_CH], c[MAX_CH];
            const Tap t1 = tap_at(px, py, dx, dy, V.w0, V.h0, V.w1, V.h1);
            blend_u<MAX_CH>(V.v1, V.w1, c1, t1, c);
            Tap t0{};
            float w4[4];
            if (j == 0)
            {
#pragma unroll
                for (int i = 0; i < MAX_CH; i++)
                    if (i < c0)
                        s[i] = __ldg(V.v0 + pixel * c0 + i);
            }
            else
            {
                t0 = tap_at(px, py, dx, dy, V.w0, V.h0, V.w0, V.h0);
                blend_u<MAX_CH>(V.v0, V.w0, c0, t0, s);
                tap_weights(t0, w4);
            }
#pragma unroll
            for (int jj = 0; jj < MAX_CH; jj++)
                if (jj < c1)
                    row[q++] = c[jj];
#pragma unroll
            for (int i = 0; i < MAX_CH; i++)
                if (i < c0)
                    row[q++] = s[i];
#pragma unroll
            for (int i = 0; i < MAX_CH; i++)
#pragma unroll
                for (int jj = 0; jj < MAX_CH; jj++)
                    if (i < c0 && jj < c1)
                        row[q++] = s[i] * c[jj];
            row[q++] = 1.0f;
            for (int r = 0; r < nout; r++)
            {
                float t;
                if (j == 0)
                    t = __ldg(V.src + pixel * nout + r);
                else
                    t = w4[0] * __ldg(V.src + ((size_t)t0.y0 * V.w0 + t0.x0) * nout + r) +
                        w4[1] * __ldg(V.src + ((size_t)t0.y0 * V.w0 + t0.x1) * nout + r) +
                        w4[2] * __ldg(V.src + ((size_t)t0.y1 * V.w0 + t0.x0) * nout + r) +
                        w4[3] * __ldg(V.src + ((size_t)t0.y1 * V.w0 + t0.x1) * nout + r);
                row[q++] = t;
            }
        }
        for (; q < 48; q++)
            row[q] = 0.0f;
        __syncthreads();
        // this warp's 32 sites, four per step
        const float* base = sz + (size_t)(warp * 32 + (lane & 3)) * NE_STRIDE + (lane >> 2);
#pragma unroll 2
        for (int step = 0; step < 8; step++)
        {
            const float* f = base + (size_t)step * 4 * NE_STRIDE;
            double frag[6];
#pragma unroll
            for (int b = 0; b < 6; b++)
                frag[b] = (double)f[8 * b];
#pragma unroll
            for (int t = 0; t < NE_TILES; t++)
                dmma_8x8x4(acc[t][0], acc[t][1], frag[tile_i(t)], frag[tile_j(t)]);
        }
    }

    // the warps' tiles, added in warp order; each block writes the entries the system needs
    __syncthreads();
    double* red = ne_sh;   // [warp][tile][64]
#pragma unroll
    for (int t = 0; t < NE_TILES; t++)
    {
        const int r = lane >> 2, cidx = (lane & 3) * 2;
        red[((size_t)warp * NE_TILES + t) * 64 + r * 8 + cidx] = acc[t][0];
        red[((size_t)warp * NE_TILES + t) * 64 + r * 8 + cidx + 1] = acc[t][1];
    }
    __syncthreads();
    for (int x = tid; x < NE_TILES * 64; x += NE_THREADS)
    {
        const int t = x / 64, r = (x % 64) / 8, cc = x % 8;
        const int a = 8 * tile_i(t) + r, b = 8 * tile_j(t) + cc;
        int e = -1;
        if (a <= b && b < mm)
            e = tri_index(a, b, mm);
        else if (a < mm && b >= mm && b < mm + nout)
            e = mm * (mm + 1) / 2 + (b - mm) * mm + a;   // rhs of output b - mm (t sits at column mm + c)
        if (e < 0)
            continue;
        double sum = 0.0;
        for (int w = 0; w < NE_WARPS; w++)
            sum += red[((size_t)w * NE_TILES + t) * 64 + r * 8 + cc];
        A.partial[((size_t)pl * A.entries + e) * LS_GRID + blockIdx.x] = sum;
    }
}

__global__ void k_ls_reduce(const double* partial, int entries, int planes, const double* omega, double* out)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= entries)
        return;
    double total = 0.0;
    for (int p = 0; p < planes; p++)
    {
        const double* row = partial + ((size_t)p * entries + e) * LS_GRID;
        double sum = 0.0;
        for (int b = 0; b < LS_GRID; b++)
            sum += row[b];
        total += omega[p] * sum;
    }
    out[e] = total;
}

int normal_equations(nntc_b200_device* d, int k, const double* per_site, double* ms)
{
    const int mm = d->nin + 1;
    const int entries = mm * (mm + 1) / 2 + d->nout * mm;
    double* omega = d->ls_partial + (size_t)d->planes.size() * entries * LS_GRID;
    NB_CUDA(cudaMemcpyAsync(omega, per_site, d->planes.size() * sizeof(double), cudaMemcpyHostToDevice, d->stream));
    Planes P = planes_for(d, 0, [&](int) { return (size_t)0; });
    P.kc = k;
    NB_TRY(block_begin(d));
    dim3 grid(LS_GRID, (unsigned)P.n);
    const size_t shared = std::max((size_t)NE_THREADS * NE_STRIDE * sizeof(float),
                                   (size_t)NE_WARPS * NE_TILES * 64 * sizeof(double));
    NB_CUDA(cudaFuncSetAttribute(k_ls_accumulate_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shared));
    NB_TRY(ktimer_begin(d, NNTC_B200_K_NORMAL_EQ));
    k_ls_accumulate_mma<<<grid, NE_THREADS, shared, d->stream>>>(P, LsArgs{ d->ls_partial, entries });
    NB_TRY(ktimer_end(d));
    NB_LAUNCHED();
    k_ls_reduce<<<grid_for((size_t)entries, 128), 128, 0, d->stream>>>(d->ls_partial, entries, P.n, omega,
                                                                      d->reduction);
    NB_LAUNCHED();
    return block_end(d, ms);
}

// ---- the host solve (src/solve_decoder.cu:184-458) -----------------------------------------------------------------

static bool gauss_jordan(std::vector<double>& g, int m, int nrhs)
{
    const int cols = m + nrhs;
    for (int k = 0; k < m; k++)
    {
        int pivot = k;
        double best = std::fabs(g[(size_t)k * cols + k]);
        for (int i = k + 1; i < m; i++)
        {
            const double a = std::fabs(g[(size_t)i * cols + k]);
            if (a > best)
            {
                best = a;
                pivot = i;
            }
        }
        if (best == 0.0)
            return false;
        if (pivot != k)
            for (int j = 0; j < cols; j++)
                std::swap(g[(size_t)k * cols + j], g[(size_t)pivot * cols + j]);
        const double inv = 1.0 / g[(size_t)k * cols + k];
        for (int j = 0; j < cols; j++)
            g[(size_t)k * cols + j] *= inv;
        for (int i = 0; i < m; i++)
        {
            if (i == k)
                continue;
            const double f = g[(size_t)i * cols + k];
            if (f == 0.0)
                continue;
            for (int j = 0; j < cols; j++)
                g[(size_t)i * cols + j] -= f * g[(size_t)k * cols + j];
        }
    }
    return true;
}

static const double RIDGE_LADDER[] = { 1e-9, 1e-12, 0.0 };
static const double LS_ACCEPT_RISE = 1e-12;
static long long g_ridge_tally[4] = { 0, 0, 0, 0 };

// The decoder from the normal equations in acc (the ladder, the acceptance test and the fallbacks). Returns the rung
// taken (0..2), or 3 when every rung was refused.
int decoder_from_normal_equations(nntc_b200_model& m, int k, const double* per_site, const std::vector<double>& acc)
{
    const int nin = m.nin, nout = m.nout, mm = nin + 1;
    const int tri = mm * (mm + 1) / 2;
    double trace = 0.0;
    for (int i = 0; i < mm; i++)
        trace += acc[(size_t)tri_index(i, i, mm)];
    const double mean_diag = trace > 0.0 ? trace / mm : 1.0;

    const bool had_previous = m.has_decoder != 0;
    std::vector<double> x_prev((size_t)nout * mm, 0.0);
    if (had_previous)
        for (int c = 0; c < nout; c++)
        {
            for (int i = 0; i < nin; i++)
                x_prev[(size_t)c * mm + i] = (double)m.dec_w[(size_t)c * nin + i];
            x_prev[(size_t)c * mm + nin] = (double)m.dec_b[c];
        }
    double sum_cw = 0.0;
    for (int c = 0; c < nout; c++)
        sum_cw += (double)m.cw[c];
    double den = 0.0;
    for (int i = 0; i < m.nplanes; i++)
        den += per_site[i] * (double)m.w0[i] * (double)m.h0[i] * (double)(1 + k);
    const bool norm_ok = sum_cw * den > 0.0;
    const double inv_norm = norm_ok ? 1.0 / (sum_cw * den) : 0.0;

    auto qform = [&](const std::vector<double>& x, double& err) {
        double q = 0.0, e = 0.0;
        for (int c = 0; c < nout; c++)
        {
            double qc = 0.0, ec = 0.0;
            for (int i = 0; i < mm; i++)
            {
                for (int j = 0; j < mm; j++)
                {
                    const double a = i <= j ? acc[(size_t)tri_index(i, j, mm)] : acc[(size_t)tri_index(j, i, mm)];
                    qc += x[(size_t)c * mm + i] * a * x[(size_t)c * mm + j];
                    ec += std::fabs(x[(size_t)c * mm + i]) * std::fabs(a) * std::fabs(x[(size_t)c * mm + j]);
                }
                qc -= 2.0 * x[(size_t)c * mm + i] * acc[(size_t)tri + (size_t)c * mm + i];
                ec += 2.0 * std::fabs(x[(size_t)c * mm + i]) * std::fabs(acc[(size_t)tri + (size_t)c * mm + i]);
            }
            q += (double)m.cw[c] * qc;
            e += (double)m.cw[c] * ec;
        }
        err = DBL_EPSILON * (double)mm * e * inv_norm;
        return q;
    };

    double err_prev = 0.0;
    const double q_prev = had_previous ? qform(x_prev, err_prev) : 0.0;
    const int cols = mm + nout;
    std::vector<double> g((size_t)mm * cols, 0.0);
    std::vector<double> x_new((size_t)nout * mm, 0.0);
    bool accepted = false;
    int taken = 0;
    for (int step = 0; step < 3 && !accepted; step++)
    {
        const double ridge = RIDGE_LADDER[step] * mean_diag;
        std::fill(g.begin(), g.end(), 0.0);
        for (int i = 0; i < mm; i++)
        {
            for (int j = i; j < mm; j++)
            {
                const double a = acc[(size_t)tri_index(i, j, mm)];
                g[(size_t)i * cols + j] = a;
                g[(size_t)j * cols + i] = a;
            }
            g[(size_t)i * cols + i] += ridge;
            for (int c = 0; c < nout; c++)
                g[(size_t)i * cols + mm + c] = acc[(size_t)tri + (size_t)c * mm + i];
        }
        if (!gauss_jordan(g, mm, nout))
            continue;
        bool finite = true;
        for (int c = 0; c < nout; c++)
            for (int i = 0; i < mm; i++)
            {
                const double v = (double)(float)g[(size_t)i * cols + mm + c];
                x_new[(size_t)c * mm + i] = v;
                finite = finite && std::isfinite(v);
            }
        if (!finite)
            continue;
        double err_cand = 0.0;
        const double q_cand = qform(x_new, err_cand);
        if (!had_previous || (norm_ok && (q_cand - q_prev) * inv_norm + err_prev + err_cand <= LS_ACCEPT_RISE))
        {
            accepted = true;
            taken = step;
        }
    }
    g_ridge_tally[accepted ? taken : 3]++;
    if (accepted)
    {
        for (int c = 0; c < nout; c++)
        {
            for (int i = 0; i < nin; i++)
                m.dec_w[(size_t)c * nin + i] = (float)x_new[(size_t)c * mm + i];
            m.dec_b[c] = (float)x_new[(size_t)c * mm + nin];
        }
        m.has_decoder = 1;
    }
    else if (!had_previous)
    {
        for (int i = 0; i < nout * nin; i++)
            m.dec_w[i] = 0.0f;
        const double count = acc[(size_t)tri_index(nin, nin, mm)];
        for (int c = 0; c < nout; c++)
            m.dec_b[c] = count > 0.0 ? (float)(acc[(size_t)tri + (size_t)c * mm + nin] / count) : 0.0f;
        m.has_decoder = 1;
    }
    return accepted ? taken : 3;
}

}   // namespace nb

using namespace nb;

extern "C"
{

int nntc_b200_solve_decoder(nntc_b200_device* d, nntc_b200_model* m, int k, const double* per_site, double* ms)
{
    double t = 0.0;
    NB_TRY(normal_equations(d, k, per_site, &t));
    const int mm = d->nin + 1;
    std::vector<double> acc((size_t)(mm * (mm + 1) / 2 + d->nout * mm));
    NB_TRY(download(d, acc.data(), d->reduction, acc.size() * sizeof(double)));
    decoder_from_normal_equations(*m, k, per_site, acc);
    NB_TRY(upload_decoder(d, m));
    if (ms)
        *ms = t;
    return NNTC_B200_OK;
}

void nntc_b200_decoder_ridge_tally(long long out[4])
{
    for (int i = 0; i < 4; i++)
        out[i] = g_ridge_tally[i];
}

}   // extern "C"
