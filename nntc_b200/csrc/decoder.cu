// decoder.cu: block (a), the decoder as one global least squares (src/solve_decoder.cu:1-458).
//
// With v = [phi ; 1] (mm = nin + 1) and the target t, the normal equations are A = sum omega v v^T (upper triangle)
// and rhs_c = sum omega v t_c; W and b follow from an FP64 Cholesky solve on the device with one refinement step,
// under the ridge ladder {1e-9, 1e-12, 0} mean(diag A) and the acceptance test on the objective's own quadratic Q
// (the semantics of src/solve_decoder.cu:184-458; the solver is this file's own, see k_decoder_solve).
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
#include "site_rows.cuh"

namespace nb
{

int launch_ls_accumulate_tc(nntc_b200_device* d, const Planes& P, double* partial, int entries,
                            const SiteTargetView& tgt, cudaStream_t stream, double* obj_partial);
int ensure_site_targets(nntc_b200_device* d, int k, int level0);

struct LsArgs
{
    double* partial;   // [plane][entry][LS_GRID]
    int entries;
    SiteTargetView tgt;
};

// ---- the accumulation on the FP64 tensor cores
//
// Z = [phi | 1 | t] per site in site_z()'s fixed 48-slot layout (six blocks of eight: slots 0..24 the columns of the
// system, 25.. the targets), and every product the normal equations need is an entry of the 48 x 48 Gram Z^T Z: A from
// the rows and columns of phi and 1, the right-hand sides from the rows of phi and 1 against the target columns. The
// 18 upper block pairs (I <= J, I < 4) of the Gram are accumulated with the FP64 tensor-core MMA (m8n8k4: an 8x4 slice
// of Z_I^T times a 4x8 slice of Z_J, four sites per step, every product exact in double since both factors are
// floats). A block takes 128 texels at a time, one per thread, and stages their rows site by site (the centre, then
// each fractional site: every lane of a warp takes the same branch); each of its four warps multiplies 32 of the
// staged rows and keeps all 18 tiles in registers over all of its chunks; the warps' tiles are added in warp order
// and each block writes one partial per entry, folded across blocks by k_ls_reduce in block order: deterministic.

constexpr int NE_THREADS = 128;
constexpr int NE_WARPS = NE_THREADS / 32;
constexpr int NE_STRIDE = 57;    // floats per staged site: 48 columns; an odd stride keeps the staging stores (one
                                 // row per lane) conflict-free, and 57 = 25 (mod 32) spreads the four sites of one
                                 // fragment load over the banks
constexpr int NE_TILES = 18;     // block pairs I <= J of six blocks with I <= 3: the rows a < 32 the system reads
                                 // (pairs of two target blocks are never needed)

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

template <int NOUT>
__global__ void __launch_bounds__(NE_THREADS, 4) k_ls_accumulate_mma(Planes P, const __grid_constant__ LsArgs A)
{
    extern __shared__ double ne_sh[];
    float* sz = (float*)ne_sh;   // [site][NE_STRIDE] floats; after the chunks, the warps' tiles as doubles
    const int pl = blockIdx.y;
    const PlaneView& V = P.p[pl];
    const int nin = P.nin, mm = nin + 1, kc = P.kc;
    const long long texels = (long long)V.w0 * V.h0;
    const long long chunks = (texels + NE_THREADS - 1) / NE_THREADS;
    const float* tgt = A.tgt.t + (size_t)A.tgt.site0[pl] * NOUT;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double acc[NE_TILES][2];
#pragma unroll
    for (int t = 0; t < NE_TILES; t++)
    {
        acc[t][0] = 0.0;
        acc[t][1] = 0.0;
    }

    for (long long chunk = blockIdx.x; chunk < chunks; chunk += gridDim.x)
    {
        const long long pixel = chunk * NE_THREADS + tid;
        const bool valid = pixel < texels;
        const int px = valid ? (int)(pixel % V.w0) : 0, py = valid ? (int)(pixel / V.w0) : 0;
        for (int j = 0; j <= kc; j++)
        {
            float z[ZS_WIDTH];
            if (valid)
                site_z<NOUT>(P, V, tgt, pixel, px, py, j, z);
            else
            {
#pragma unroll
                for (int q = 0; q < ZS_WIDTH; q++)
                    z[q] = 0.0f;
            }
            __syncthreads();   // the previous stage's fragments have been read
            float* row = sz + tid * NE_STRIDE;
#pragma unroll
            for (int q = 0; q < ZS_WIDTH; q++)
                row[q] = z[q];
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
    // entry (a, b) of the compact system sits at slots (z_slot(a), z_slot(b)) of the Gram, a <= b read from the upper
    // block triangle (slot order follows column order, so z_slot(a) <= z_slot(b))
    for (int e = tid; e < A.entries; e += NE_THREADS)
    {
        const int tri = mm * (mm + 1) / 2;
        int a, b;
        if (e < tri)
        {
            a = 0;
            while (e >= tri_index(a, mm - 1, mm) + 1)
                a++;
            b = a + (e - tri_index(a, a, mm));
        }
        else
        {
            a = (e - tri) % mm;
            b = mm + (e - tri) / mm;
        }
        const int sa = z_slot(a, P.c0, P.c1), sb = z_slot(b, P.c0, P.c1);
        int t = 0;
        while (!(tile_i(t) == sa / 8 && tile_j(t) == sb / 8))
            t++;
        const int r = sa % 8, cc = sb % 8;
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

// Each plane's three objective sums from the normal equations' pass, its CTAs' partials added in block order.
__global__ void k_ls_obj_reduce(const double* partial, int planes, double* out)
{
    const int pl = blockIdx.x, q = threadIdx.x;
    if (pl >= planes || q >= 3)
        return;
    double t = 0.0;
    for (int b = 0; b < LS_GRID; b++)
        t += partial[((size_t)pl * 3 + q) * LS_GRID + b];
    out[3 * pl + q] = t;
}

// obj_sums (the mixed-precision Gram only): also the objective's three raw sums per plane of the decoder on the device,
// at the same sites, into host memory (3 per plane).
int normal_equations(nntc_b200_device* d, int k, const double* per_site, double* ms, std::vector<double>* obj_sums)
{
    const int mm = d->nin + 1;
    const int entries = mm * (mm + 1) / 2 + d->nout * mm;
    double* omega = d->ls_partial + (size_t)d->planes.size() * entries * LS_GRID;
    NB_CUDA(cudaMemcpyAsync(omega, per_site, d->planes.size() * sizeof(double), cudaMemcpyHostToDevice, d->stream));
    Planes P = planes_for(d, 0, [&](int) { return (size_t)0; });
    P.kc = k;
    NB_TRY(block_begin(d));
    NB_TRY(ensure_site_targets(d, k, 0));
    LsArgs A{ d->ls_partial, entries, {} };
    A.tgt.t = d->site_tgt;
    long long ft = 0;
    for (int i = 0; i < P.n; i++)
    {
        A.tgt.site0[i] = ft;
        ft += (long long)P.p[i].w0 * P.p[i].h0 * k;
    }
    A.tgt.site0[P.n] = ft;
    dim3 grid(LS_GRID, (unsigned)P.n);
    if (d->mixed_gram)
    {
        NB_CUDA(cudaMemsetAsync(d->counters + CNT_STATUS, 0, sizeof(unsigned int), d->stream));
        NB_TRY(ktimer_begin(d, NNTC_B200_K_NORMAL_EQ));
        NB_TRY(launch_ls_accumulate_tc(d, P, d->ls_partial, entries, A.tgt, d->stream, obj_sums ? d->ls_obj : nullptr));
        NB_TRY(ktimer_end(d));
    }
    else
    {
        const size_t shared = std::max((size_t)NE_THREADS * NE_STRIDE * sizeof(float),
                                       (size_t)NE_WARPS * NE_TILES * 64 * sizeof(double));
        NB_TRY(ktimer_begin(d, NNTC_B200_K_NORMAL_EQ));
#define NB_NE(NO)                                                                                                     \
    case NO:                                                                                                          \
        NB_CUDA(cudaFuncSetAttribute(k_ls_accumulate_mma<NO>, cudaFuncAttributeMaxDynamicSharedMemorySize,           \
                                     (int)shared));                                                                   \
        k_ls_accumulate_mma<NO><<<grid, NE_THREADS, shared, d->stream>>>(P, A);                                       \
        break;
        switch (d->nout)
        {
            NB_NE(3)
            NB_NE(6)
            NB_NE(9)
            NB_NE(12)
            NB_NE(15)
            NB_NE(18)
        default:
            set_error(NNTC_B200_ERR_STATE, "a material holds 1..6 RGB textures");
            return NNTC_B200_ERR_STATE;
        }
#undef NB_NE
        NB_TRY(ktimer_end(d));
        NB_LAUNCHED();
    }
    k_ls_reduce<<<grid_for((size_t)entries, 128), 128, 0, d->stream>>>(d->ls_partial, entries, P.n, omega,
                                                                      d->reduction);
    NB_LAUNCHED();
    const bool with_obj = obj_sums && d->mixed_gram;
    double* obj_out = d->ls_obj + (size_t)P.n * 3 * LS_GRID;
    if (with_obj)
    {
        k_ls_obj_reduce<<<P.n, 32, 0, d->stream>>>(d->ls_obj, P.n, obj_out);
        NB_LAUNCHED();
    }
    NB_TRY(block_end(d, ms));
    if (with_obj)
    {
        obj_sums->assign((size_t)3 * P.n, 0.0);
        NB_TRY(download(d, obj_sums->data(), obj_out, obj_sums->size() * sizeof(double)));
    }
    else if (obj_sums)
    {
        set_error(NNTC_B200_ERR_STATE, "the objective rides only on the tensor-core normal equations");
        return NNTC_B200_ERR_STATE;
    }
    if (d->mixed_gram)
    {
        unsigned int status = 0;
        NB_TRY(download(d, &status, d->counters + CNT_STATUS, sizeof(status)));
        if (status)
        {
            set_error(NNTC_B200_ERR_TIMEOUT, "the tensor-core normal equations gave up waiting on their MMAs");
            return NNTC_B200_ERR_TIMEOUT;
        }
    }
    return NNTC_B200_OK;
}

// ---- the solve, on the device ---------------------------------------------------------------------------------------
//
// The system is tiny (mm <= 25 unknowns, nout <= 18 right-hand sides), so one block of 128 threads does all of it in
// shared memory, with no host round trip between the accumulation and the decision:
//
//   for each ridge r of the ladder {1e-9, 1e-12, 0} x mean(diag A), until one is accepted:
//     L L^T = A + r I                       FP64 Cholesky, right-looking, a non-positive or non-finite pivot refuses
//                                           the rung;
//     X = (L L^T)^-1 R                      one forward and one backward substitution per output;
//     X += (L L^T)^-1 (R - (A + r I) X)     one step of iterative refinement, the residual with fused multiply-adds;
//     X rounded to float                    the decoder that would ship; a non-finite value refuses the rung;
//     accept X if Q(X) does not exceed Q(previous decoder) by more than 1e-12 in E's units once both quadratics'
//     rounding bounds are charged against the difference (or if there is no previous decoder).
//
// Q(x) = sum_c cw_c (x_c^T A x_c - 2 x_c . R_c) is E's numerator up to a constant, so the test costs no objective pass;
// its rounding bound is eps mm sum_c cw_c (|x_c|^T |A| |x_c| + 2 |x_c| . |R_c|). These semantics - the rungs, the float
// rounding before judging, the bound and the 1e-12 tolerance, keeping the previous decoder when every rung is refused
// and the weighted mean target when there is none - are the reference's (src/solve_decoder.cu:267-458); the solver is
// not (the reference runs Gauss-Jordan with partial pivoting on the host). A Cholesky pivot that is not positive
// refuses a rung where Gauss-Jordan would have pivoted on, which the acceptance test would refuse in any case: such a
// system's ridge-free solution is not a minimiser of Q.

constexpr int DS_THREADS = 128;
constexpr int DS_MM = MAX_NIN + 1;

struct DecoderSolveArgs
{
    int nin, nout;
    int had_previous;   // the model arrives with a decoder
    int norm_ok;        // sum(cw) x the weighted site count > 0
    double inv_norm;    // 1 / (sum(cw) x the weighted site count): Q in E's units
    float cw[MAX_NOUT];
    float w[MAX_NOUT * MAX_NIN];
    float b[MAX_NOUT];
};

// What the solve hands back: the rung taken (0..2), 3 with a fallback fit (no previous decoder), 4 when the previous
// decoder stays; then, unless 4, the decoder as nout rows of [w_c (nin) | b_c].
struct DecoderSolveOut
{
    int rung;
    int pad[3];
    float x[MAX_NOUT * DS_MM];
};

// The quadratic and its rounding bound at the solution rows X (shared), in E's units for the bound. Every thread
// calls it; thread c < nout forms output c's terms, thread 0 adds the outputs in index order.
__device__ void ds_quadratic(const double (*A)[DS_MM + 1], const double (*R)[DS_MM], const double (*X)[DS_MM],
                             const DecoderSolveArgs& a, int mm, double* qc, double* ec, double& q, double& err)
{
    const int c = threadIdx.x;
    if (c < a.nout)
    {
        double qs = 0.0, es = 0.0;
        for (int i = 0; i < mm; i++)
        {
            double ax = 0.0, aax = 0.0;
            for (int j = 0; j < mm; j++)
            {
                ax = fma(A[i][j], X[c][j], ax);
                aax = fma(fabs(A[i][j]), fabs(X[c][j]), aax);
            }
            qs = fma(X[c][i], ax - 2.0 * R[c][i], qs);
            es = fma(fabs(X[c][i]), aax + 2.0 * fabs(R[c][i]), es);
        }
        qc[c] = qs;
        ec[c] = es;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double qt = 0.0, et = 0.0;
        for (int o = 0; o < a.nout; o++)
        {
            qt += (double)a.cw[o] * qc[o];
            et += (double)a.cw[o] * ec[o];
        }
        q = qt;
        err = DBL_EPSILON * (double)mm * et * a.inv_norm;
    }
    __syncthreads();
}

// Solve (L L^T) y = rhs in place for output row c (one thread).
__device__ void ds_substitute(const double (*L)[DS_MM + 1], double* y, int mm)
{
    for (int i = 0; i < mm; i++)
    {
        double s = y[i];
        for (int j = 0; j < i; j++)
            s = fma(-L[i][j], y[j], s);
        y[i] = s / L[i][i];
    }
    for (int i = mm - 1; i >= 0; i--)
    {
        double s = y[i];
        for (int j = i + 1; j < mm; j++)
            s = fma(-L[j][i], y[j], s);
        y[i] = s / L[i][i];
    }
}

__global__ void __launch_bounds__(DS_THREADS) k_decoder_solve(const double* __restrict__ ne, DecoderSolveArgs a,
                                                               DecoderSolveOut* out)
{
    __shared__ double A[DS_MM][DS_MM + 1], L[DS_MM][DS_MM + 1];
    __shared__ double R[MAX_NOUT][DS_MM], X[MAX_NOUT][DS_MM], D[MAX_NOUT][DS_MM];
    __shared__ double qc[MAX_NOUT], ec[MAX_NOUT];
    __shared__ double q_prev, err_prev, q_new, err_new, mean_diag;
    __shared__ int refused, accepted;
    const int tid = threadIdx.x, nin = a.nin, nout = a.nout, mm = nin + 1;
    const int tri = mm * (mm + 1) / 2;

    // A from its upper triangle, R from the right-hand-side rows (output c's rhs is the c-th run of mm entries)
    for (int e = tid; e < mm * mm; e += DS_THREADS)
    {
        const int i = e / mm, j = e % mm, lo = min(i, j), hi = max(i, j);
        A[i][j] = ne[tri_index(lo, hi, mm)];
    }
    for (int e = tid; e < nout * mm; e += DS_THREADS)
        R[e / mm][e % mm] = ne[tri + e];
    // the previous decoder as solution rows, for its quadratic
    for (int e = tid; e < nout * mm; e += DS_THREADS)
    {
        const int c = e / mm, i = e % mm;
        X[c][i] = a.had_previous ? (double)(i < nin ? a.w[c * nin + i] : a.b[c]) : 0.0;
    }
    __syncthreads();
    if (tid == 0)
    {
        double trace = 0.0;
        for (int i = 0; i < mm; i++)
            trace += A[i][i];
        mean_diag = trace > 0.0 ? trace / mm : 1.0;
        accepted = -1;
    }
    __syncthreads();
    if (a.had_previous)
        ds_quadratic(A, R, X, a, mm, qc, ec, q_prev, err_prev);

    const double ladder[3] = { 1e-9, 1e-12, 0.0 };
    for (int rung = 0; rung < 3; rung++)
    {
        const double ridge = ladder[rung] * mean_diag;
        for (int e = tid; e < mm * mm; e += DS_THREADS)
        {
            const int i = e / mm, j = e % mm;
            L[i][j] = i == j ? A[i][j] + ridge : A[i][j];
        }
        if (tid == 0)
            refused = 0;
        __syncthreads();
        // right-looking Cholesky on the lower triangle
        for (int k = 0; k < mm; k++)
        {
            if (tid == 0)
            {
                const double p = L[k][k];
                if (p > 0.0 && isfinite(p))
                    L[k][k] = sqrt(p);
                else
                    refused = 1;
            }
            __syncthreads();
            if (refused)
                break;
            for (int i = k + 1 + tid; i < mm; i += DS_THREADS)
                L[i][k] /= L[k][k];
            __syncthreads();
            const int n = mm - k - 1;
            for (int e = tid; e < n * n; e += DS_THREADS)
            {
                const int i = k + 1 + e / n, j = k + 1 + e % n;
                if (j <= i)
                    L[i][j] = fma(-L[i][k], L[j][k], L[i][j]);
            }
            __syncthreads();
        }
        if (refused)
            continue;
        // solve, then one refinement step against A + ridge I
        if (tid < nout)
        {
            for (int i = 0; i < mm; i++)
                D[tid][i] = R[tid][i];
            ds_substitute(L, D[tid], mm);
        }
        __syncthreads();
        for (int e = tid; e < nout * mm; e += DS_THREADS)
            X[e / mm][e % mm] = D[e / mm][e % mm];
        __syncthreads();
        for (int e = tid; e < nout * mm; e += DS_THREADS)
        {
            const int c = e / mm, i = e % mm;
            double r = fma(-ridge, X[c][i], R[c][i]);
            for (int j = 0; j < mm; j++)
                r = fma(-A[i][j], X[c][j], r);
            D[c][i] = r;
        }
        __syncthreads();
        if (tid < nout)
            ds_substitute(L, D[tid], mm);
        __syncthreads();
        int finite = 1;
        for (int e = tid; e < nout * mm; e += DS_THREADS)
        {
            const int c = e / mm, i = e % mm;
            const double v = (double)(float)(X[c][i] + D[c][i]);
            X[c][i] = v;
            finite &= isfinite(v) ? 1 : 0;
        }
        if (!__syncthreads_and(finite))
            continue;
        ds_quadratic(A, R, X, a, mm, qc, ec, q_new, err_new);
        if (tid == 0 && (!a.had_previous ||
                         (a.norm_ok && (q_new - q_prev) * a.inv_norm + err_prev + err_new <= 1e-12)))
            accepted = rung;
        __syncthreads();
        if (accepted >= 0)
            break;
    }

    if (accepted >= 0)
    {
        for (int e = tid; e < nout * mm; e += DS_THREADS)
            out->x[e] = (float)X[e / mm][e % mm];
        if (tid == 0)
            out->rung = accepted;
    }
    else if (!a.had_previous)
    {
        // nothing usable and nothing to keep: the constant fit, each output's weighted mean target
        const double count = A[nin][nin];
        for (int e = tid; e < nout * mm; e += DS_THREADS)
        {
            const int c = e / mm, i = e % mm;
            out->x[e] = i < nin ? 0.0f : (count > 0.0 ? (float)(R[c][nin] / count) : 0.0f);
        }
        if (tid == 0)
            out->rung = 3;
    }
    else if (tid == 0)
        out->rung = 4;
}

static_assert(sizeof(DecoderSolveOut) <= 2048, "the arena's dec_solve slice holds one DecoderSolveOut");

static long long g_rung_tally[4] = { 0, 0, 0, 0 };

void objective_from_sums(const nntc_b200_model& m, int k, const double* per_site, const std::vector<double>& acc,
                         nntc_b200_objective* r);

int solve_decoder_on_device(nntc_b200_device* d, nntc_b200_model& m, int k, const double* per_site)
{
    DecoderSolveArgs a{};
    a.nin = m.nin;
    a.nout = m.nout;
    a.had_previous = m.has_decoder != 0;
    double sum_cw = 0.0, sites = 0.0;
    for (int c = 0; c < m.nout; c++)
    {
        a.cw[c] = m.cw[c];
        sum_cw += (double)m.cw[c];
        a.b[c] = m.dec_b[c];
    }
    for (int i = 0; i < m.nout * m.nin; i++)
        a.w[i] = m.dec_w[i];
    for (int i = 0; i < m.nplanes; i++)
        sites += per_site[i] * (double)m.w0[i] * (double)m.h0[i] * (double)(1 + k);
    a.norm_ok = sum_cw * sites > 0.0;
    a.inv_norm = a.norm_ok ? 1.0 / (sum_cw * sites) : 0.0;
    DecoderSolveOut* dev_out = reinterpret_cast<DecoderSolveOut*>(d->dec_solve);
    k_decoder_solve<<<1, DS_THREADS, 0, d->stream>>>(d->reduction, a, dev_out);
    NB_LAUNCHED();
    DecoderSolveOut o;
    NB_TRY(download(d, &o, dev_out, sizeof(o)));
    const int mm = m.nin + 1;
    g_rung_tally[o.rung < 3 ? o.rung : 3]++;
    if (o.rung <= 3)
    {
        for (int c = 0; c < m.nout; c++)
        {
            for (int i = 0; i < m.nin; i++)
                m.dec_w[c * m.nin + i] = o.x[c * mm + i];
            m.dec_b[c] = o.x[c * mm + m.nin];
        }
        m.has_decoder = 1;
    }
    return NNTC_B200_OK;
}

}   // namespace nb

using namespace nb;

extern "C"
{

int nntc_b200_solve_decoder(nntc_b200_device* d, nntc_b200_model* m, int k, const double* per_site, double* ms)
{
    double t = 0.0;
    NB_TRY(normal_equations(d, k, per_site, &t, nullptr));
    NB_TRY(solve_decoder_on_device(d, *m, k, per_site));
    NB_TRY(upload_decoder(d, m));
    if (ms)
        *ms = t;
    return NNTC_B200_OK;
}

}   // extern "C"

namespace nb
{

// The adjoint form's closing pass of a round: block (a)'s normal equations at the current latents (kept on the device
// for the next round's solve) and E of the current decoder at the same sites, from one pass over the sites.
int normal_equations_and_objective(nntc_b200_device* d, const nntc_b200_model* m, int k, const double* per_site,
                                   nntc_b200_objective* e, double* ms)
{
    std::vector<double> sums;
    NB_TRY(normal_equations(d, k, per_site, ms, &sums));
    objective_from_sums(*m, k, per_site, sums, e);
    if (ms)
        e->ms = *ms;
    return NNTC_B200_OK;
}

// Block (a) from the normal equations already on the device (normal_equations_and_objective at the same latents).
int solve_decoder_prepared(nntc_b200_device* d, nntc_b200_model* m, int k, const double* per_site)
{
    NB_TRY(solve_decoder_on_device(d, *m, k, per_site));
    return upload_decoder(d, m);
}

}   // namespace nb

extern "C"
{

int nntc_b200_probe_objective_with_normal_equations(nntc_b200_device* d, const nntc_b200_model* m, int k,
                                                    const double* per_site, nntc_b200_objective* r)
{
    if (!d->mixed_gram)
    {
        set_error(NNTC_B200_ERR_STATE, "the objective rides only on the tensor-core normal equations");
        return NNTC_B200_ERR_STATE;
    }
    double ms = 0.0;
    return normal_equations_and_objective(d, m, k, per_site, r, &ms);
}

void nntc_b200_decoder_ridge_tally(long long out[4])
{
    for (int i = 0; i < 4; i++)
        out[i] = g_rung_tally[i];
}

}   // extern "C"
