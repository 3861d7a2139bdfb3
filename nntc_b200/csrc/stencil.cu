// stencil.cu: blocks (b) and (c'), the latent planes as sparse weighted least squares (src/solve_level1.cu).
//
// Block (b) holds level 0 and the decoder and solves level 1; block (c') (--l0 bc8) holds level 1 and the decoder and
// solves level 0 as a continuous 8-bit plane. Both assemble a 9-point block stencil H (five owned C x C blocks per
// texel, the other four read as the neighbours' transposes) and a gradient by GATHER, one thread per texel of the
// unknown, exactly as src/solve_level1.cu:259-581 derives it; then either preconditioned conjugate gradients on
// (H + lambda I) d = -grad (src/solve_level1.cu:1222-1338) or four-colour quantised Gauss-Seidel sweeps with the exact
// per-value grid argmin (src/solve_level1.cu:1023-1098, 1343-1403).
//
// Per-texel arithmetic is the reference's, operation for operation, compiled without FMA contraction: given the same
// planes and decoder the stencil, the gradient, the preconditioner and every sweep decision are the same bits as the
// reference's. What differs is the B200 shape:
//
// - every plane of the chain in ONE launch (nb::Planes), one stream, no per-plane fan-out;
// - the stencil stored structure-of-arrays [slot][i][j][texel], coalesced for a warp of consecutive texels;
// - the gather's 5 x nmono monomial sums live in shared memory (registers spill at C = 4);
// - the conjugate-gradient iteration is 5 launches (matvec + <p,Ap>, alpha, update + preconditioner + <r,r> +
//   <r,z>, beta, direction) instead of 13, all planes in lockstep, and the stop is decided ON THE DEVICE with the
//   reference's rule (a plane leaves at an iteration that is a multiple of CG_PROBE once its residual is below the
//   tolerance); the host reads one active-plane count every CG_PROBE iterations, the reference's probe cadence.
// - every dot product is a fixed-order two-stage reduction: one partial per 256-texel block, added per plane in
//   block order.

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "device.cuh"

namespace nb
{

constexpr int ASM_THREADS = 128;

// ---- the gather (src/solve_level1.cu:259-581) ----------------------------------------------------------------------

struct AsmArgs
{
    const float* weights;
    const float* bias;
    const float* cw;
    const double* mono;   // nmono matrices of c x c
    int nmono;
};

// The monomials of a form in y: 1, y_i, y_i y_j (i <= j), in double (src/solve_level1.cu:142-152).
__device__ __forceinline__ void monomials(const float* y, int n, double* out)
{
    int k = 0;
    out[k++] = 1.0;
    for (int i = 0; i < n; i++)
        out[k++] = (double)y[i];
    for (int i = 0; i < n; i++)
        for (int j = i; j < n; j++)
            out[k++] = (double)y[i] * (double)y[j];
}

// The four corners of a tap merged by texel index, so a clamped duplicate adds its weight to one texel.
__device__ __forceinline__ int merge_taps(const Tap& t, int* nx, int* ny, float* tw)
{
    const int cx[4] = { t.x0, t.x1, t.x0, t.x1 };
    const int cy[4] = { t.y0, t.y0, t.y1, t.y1 };
    float cwt[4];
    tap_weights(t, cwt);
    int taps = 0;
    for (int q = 0; q < 4; q++)
    {
        int found = -1;
        for (int e = 0; e < taps; e++)
            if (nx[e] == cx[q] && ny[e] == cy[q])
                found = e;
        if (found >= 0)
            tw[found] += cwt[q];
        else
        {
            nx[taps] = cx[q];
            ny[taps] = cy[q];
            tw[taps] = cwt[q];
            taps++;
        }
    }
    return taps;
}

// The pixels whose bilinear footprint into an n1-wide plane can reach texel ti (src/solve_level1.cu:246-257).
__device__ __forceinline__ void footprint(int ti, int n0, int n1, int& lo, int& hi)
{
    const double r = (double)n0 / (double)n1;
    lo = (int)ceil(((double)ti - 0.5) * r - 1.0);
    hi = (int)ceil(((double)ti + 1.5) * r) - 1;
    lo = lo < 0 ? 0 : lo;
    hi = hi > n0 - 1 ? n0 - 1 : hi;
}

template <bool LEVEL0>
__global__ void __launch_bounds__(ASM_THREADS) k_assemble(Planes P, AsmArgs A)
{
    extern __shared__ double sums_sh[];   // [slot * nmono + i][thread]
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long ti = base - P.start[pl] + threadIdx.x;
    const int c0 = P.c0, c1 = P.c1, nin = P.nin, nout = P.nout, kc = P.kc, nmono = A.nmono;
    const int c = LEVEL0 ? c0 : c1;
    const int tw_ = V.w, th_ = V.h;
    if (ti >= (long long)tw_ * th_)
        return;
    const int tx = (int)(ti % tw_), ty = (int)(ti / tw_);
    double* sums = sums_sh + threadIdx.x;
    const int S = blockDim.x;
    for (int i = 0; i < SLOTS * nmono; i++)
        sums[i * S] = 0.0;
    double g[MAX_CH];
    for (int i = 0; i < c; i++)
        g[i] = 0.0;

    int px_lo, px_hi, py_lo, py_hi;
    if (LEVEL0)
    {
        footprint(tx, V.w0, V.w0, px_lo, px_hi);
        footprint(ty, V.h0, V.h0, py_lo, py_hi);
    }
    else
    {
        footprint(tx, V.w0, V.w1, px_lo, px_hi);
        footprint(ty, V.h0, V.h1, py_lo, py_hi);
    }

    for (int py = py_lo; py <= py_hi; py++)
        for (int px = px_lo; px <= px_hi; px++)
            for (int j = 0; j <= kc; j++)
            {
                float dx, dy;
                site_offset(kc, j, px, py, dx, dy);
                int nx[4], ny[4];
                float tw[4];
                int taps = 0;
                float sbar[MAX_CH], cbar[MAX_CH], target[MAX_NOUT];
                const Tap tp = tap_at(px, py, dx, dy, V.w0, V.h0, V.w1, V.h1);
                if (!LEVEL0)
                {
                    taps = merge_taps(tp, nx, ny, tw);
                    int self = -1;
                    for (int e = 0; e < taps; e++)
                        if (nx[e] == tx && ny[e] == ty)
                            self = e;
                    if (self < 0)
                        continue;
                    blend<MAX_CH>(V.v1, V.w1, c1, tp, cbar);
                    if (j == 0)
                    {
                        const size_t pi = (size_t)py * V.w0 + px;
                        for (int i = 0; i < c0; i++)
                            sbar[i] = V.v0[pi * c0 + i];
                        for (int r = 0; r < nout; r++)
                            target[r] = __ldg(V.src + pi * nout + r);
                    }
                    else
                    {
                        const Tap t0 = tap_at(px, py, dx, dy, V.w0, V.h0, V.w0, V.h0);
                        blend<MAX_CH>(V.v0, V.w0, c0, t0, sbar);
                        blend<MAX_NOUT>(V.src, V.w0, nout, t0, target);
                    }
                    // G = A + sum_i sbar_i M_i, residual r = b + B sbar + G cbar - t (src/solve_level1.cu:335-352)
                    float gmat[MAX_NOUT * MAX_CH], res[MAX_NOUT];
                    for (int r = 0; r < nout; r++)
                    {
                        const float* row = A.weights + (size_t)r * nin;
                        float out = A.bias[r];
                        for (int i = 0; i < c0; i++)
                            out += row[c1 + i] * sbar[i];
                        for (int q = 0; q < c1; q++)
                        {
                            float gg = row[q];
                            for (int i = 0; i < c0; i++)
                                gg += sbar[i] * row[c1 + c0 + i * c1 + q];
                            gmat[r * c1 + q] = gg;
                            out += gg * cbar[q];
                        }
                        res[r] = out - target[r];
                    }
                    double mono[MAX_MONO];
                    monomials(sbar, c0, mono);
                    const float w_self = tw[self];
                    for (int a = 0; a < c1; a++)
                    {
                        double acc = 0.0;
                        for (int r = 0; r < nout; r++)
                            acc += (double)A.cw[r] * (double)gmat[r * c1 + a] * (double)res[r];
                        g[a] += (double)w_self * acc;
                    }
                    for (int e = 0; e < taps; e++)
                    {
                        const int slot = slot_of(nx[e] - tx, ny[e] - ty);
                        if (slot < 0)
                            continue;
                        const double scale = (double)w_self * (double)tw[e];
                        double* dst = sums + (size_t)slot * nmono * S;
                        for (int i = 0; i < nmono; i++)
                            dst[i * S] += scale * mono[i];
                    }
                }
                else
                {
                    blend<MAX_CH>(V.v1, V.w1, c1, tp, cbar);
                    if (j == 0)
                    {
                        const size_t pi = (size_t)py * V.w0 + px;
                        nx[0] = px;
                        ny[0] = py;
                        tw[0] = 1.0f;
                        taps = 1;
                        for (int i = 0; i < c0; i++)
                            sbar[i] = V.v0[pi * c0 + i];
                        for (int r = 0; r < nout; r++)
                            target[r] = __ldg(V.src + pi * nout + r);
                    }
                    else
                    {
                        const Tap t0 = tap_at(px, py, dx, dy, V.w0, V.h0, V.w0, V.h0);
                        blend<MAX_CH>(V.v0, V.w0, c0, t0, sbar);
                        blend<MAX_NOUT>(V.src, V.w0, nout, t0, target);
                        taps = merge_taps(t0, nx, ny, tw);
                    }
                    int self = -1;
                    for (int e = 0; e < taps; e++)
                        if (nx[e] == tx && ny[e] == ty)
                            self = e;
                    if (self < 0)
                        continue;
                    // Q = B + sum_q cbar_q N_q, residual r = b + A cbar + Q sbar - t (src/solve_level1.cu:518-536)
                    float qmat[MAX_NOUT * MAX_CH], res[MAX_NOUT];
                    for (int r = 0; r < nout; r++)
                    {
                        const float* row = A.weights + (size_t)r * nin;
                        float out = A.bias[r];
                        for (int q = 0; q < c1; q++)
                            out += row[q] * cbar[q];
                        for (int i = 0; i < c0; i++)
                        {
                            float qq = row[c1 + i];
                            for (int q = 0; q < c1; q++)
                                qq += cbar[q] * row[c1 + c0 + i * c1 + q];
                            qmat[r * c0 + i] = qq;
                            out += qq * sbar[i];
                        }
                        res[r] = out - target[r];
                    }
                    double mono[MAX_MONO];
                    monomials(cbar, c1, mono);
                    const float w_self = tw[self];
                    for (int a = 0; a < c0; a++)
                    {
                        double acc = 0.0;
                        for (int r = 0; r < nout; r++)
                            acc += (double)A.cw[r] * (double)qmat[r * c0 + a] * (double)res[r];
                        g[a] += (double)w_self * acc;
                    }
                    for (int e = 0; e < taps; e++)
                    {
                        const int slot = slot_of(nx[e] - tx, ny[e] - ty);
                        if (slot < 0)
                            continue;
                        const double scale = (double)w_self * (double)tw[e];
                        double* dst = sums + (size_t)slot * nmono * S;
                        for (int i = 0; i < nmono; i++)
                            dst[i * S] += scale * mono[i];
                    }
                }
            }

    // The five blocks expanded once against the monomial matrices (src/solve_level1.cu:382-399), stored SoA.
    const size_t T = (size_t)tw_ * th_;
    const int cc = c * c;
    for (int slot = 0; slot < SLOTS; slot++)
    {
        double blk[MAX_CH * MAX_CH];
        for (int e = 0; e < cc; e++)
            blk[e] = 0.0;
        for (int i = 0; i < nmono; i++)
        {
            const double s = sums[(size_t)(slot * nmono + i) * S];
            if (s == 0.0)
                continue;
            const double* mat = A.mono + (size_t)i * cc;
            for (int e = 0; e < cc; e++)
                blk[e] += s * __ldg(mat + e);
        }
        for (int e = 0; e < cc; e++)
            V.stencil[(size_t)(slot * cc + e) * T + stencil_pos(tx, ty, tw_, th_)] = blk[e];
    }
    for (int i = 0; i < c; i++)
        V.grad[ti * c + i] = g[i];
}

// ---- reductions --------------------------------------------------------------------------------------------------

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_min(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide reduction of up to 3 values with a fixed shape (warp trees, then warps in order). kind: 0 sum, 1 min,
// 2 max. The result lands on thread 0.
template <int N>
__device__ __forceinline__ void block_reduce(double (&v)[N], const int (&kind)[N], double* sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int q = 0; q < N; q++)
        v[q] = kind[q] == 0 ? warp_sum(v[q]) : (kind[q] == 1 ? warp_min(v[q]) : warp_max(v[q]));
    __syncthreads();
    if (lane == 0)
        for (int q = 0; q < N; q++)
            sh[q * 32 + warp] = v[q];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int q = 0; q < N; q++)
        {
            double s = sh[q * 32];
            for (int w = 1; w < nw; w++)
                s = kind[q] == 0 ? s + sh[q * 32 + w] : (kind[q] == 1 ? fmin(s, sh[q * 32 + w]) : fmax(s, sh[q * 32 + w]));
            v[q] = s;
        }
}

// One warp per plane: the plane's block partials of `rows` rows added in block order (strided by lane, then a tree).
__device__ __forceinline__ double plane_total(const double* partial, size_t nblocks, long long b0, long long b1,
                                              int row, int kind)
{
    const int lane = threadIdx.x & 31;
    double s = kind == 0 ? 0.0 : (kind == 1 ? 1e300 : -1e300);
    for (long long b = b0 + lane; b < b1; b += 32)
    {
        const double x = partial[(size_t)row * nblocks + b];
        s = kind == 0 ? s + x : (kind == 1 ? fmin(s, x) : fmax(s, x));
    }
    return kind == 0 ? warp_sum(s) : (kind == 1 ? warp_min(s) : warp_max(s));
}

struct Red
{
    double* partial;      // [row][block]
    size_t nblocks;       // blocks of the launch (the row stride)
    double* scalars;      // [plane][S_COUNT]
};

// One coefficient of the stencil as stored: FP64 (the plain form) or FP32 (the adjoint form's quantised sweeps read a
// single-precision stencil, half the bytes), widened to double for the sums that read it.
template <typename TS>
__device__ __forceinline__ double sten(const PlaneView& V, size_t idx)
{
    return (double)reinterpret_cast<const TS*>(V.stencil)[idx];
}

// A texel's C x C block of slot `slot` (the texel at stencil position sp). An FP32 block of 16 (or 4) coefficients is
// read at once as 16-byte vector loads into registers; an FP64 block (and any other) is read a coefficient at a time
// where it is used, as the plain form always has (holding 16 doubles would cost its kernels occupancy).
template <int C, typename TS>
struct StenBlock
{
    static constexpr int cc = C * C;
    static constexpr bool vec = sizeof(TS) == sizeof(float) && cc % 4 == 0;
    float f[vec ? cc : 1];
    const TS* base;
    size_t T, sp;
    int slot;
    __device__ __forceinline__ StenBlock(const PlaneView& V, int slot_, size_t T_, size_t sp_)
        : base(reinterpret_cast<const TS*>(V.stencil)), T(T_), sp(sp_), slot(slot_)
    {
        if constexpr (vec)
        {
            const float4* q = reinterpret_cast<const float4*>(base + ((size_t)slot * T + sp) * cc);
#pragma unroll
            for (int v = 0; v < cc / 4; v++)
            {
                const float4 x = __ldg(q + v);
                f[4 * v] = x.x;
                f[4 * v + 1] = x.y;
                f[4 * v + 2] = x.z;
                f[4 * v + 3] = x.w;
            }
        }
    }
    __device__ __forceinline__ double operator[](int e) const
    {
        if constexpr (vec)
            return (double)f[e];
        else
            return (double)base[sten_index<TS>(slot, e, cc, T, sp)];
    }
};

// ---- ridge, preconditioner ----------------------------------------------------------------------------------------

template <typename TS>
__global__ void __launch_bounds__(THREADS) k_diag(Planes P, Red R)
{
    __shared__ double sh[3 * 32];
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long t = base - P.start[pl] + threadIdx.x;
    const size_t T = (size_t)V.w * V.h;
    const int c = P.c;
    double v[3] = { 0.0, 1e300, -1e300 };
    const int kind[3] = { 0, 1, 2 };
    if (t < (long long)T)
        for (int a = 0; a < c; a++)
        {
            const double x = sten<TS>(V, sten_index<TS>(0, a * c + a, c * c, T, stencil_pos((int)(t % V.w), (int)(t / V.w), V.w, V.h)));
            v[0] += x;
            v[1] = x < v[1] ? x : v[1];
            v[2] = x > v[2] ? x : v[2];
        }
    block_reduce(v, kind, sh);
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; q++)
            R.partial[(size_t)q * R.nblocks + blockIdx.x] = v[q];
}

__global__ void k_diag_reduce(Planes P, Red R, double ridge)
{
    const int pl = blockIdx.x;
    const long long b0 = P.start[pl] / THREADS, b1 = P.start[pl + 1] / THREADS;
    const double sum = plane_total(R.partial, R.nblocks, b0, b1, 0, 0);
    const double lo = plane_total(R.partial, R.nblocks, b0, b1, 1, 1);
    const double hi = plane_total(R.partial, R.nblocks, b0, b1, 2, 2);
    if (threadIdx.x == 0)
    {
        double* s = R.scalars + (size_t)pl * S_COUNT;
        const size_t unknowns = (size_t)P.p[pl].w * P.p[pl].h * P.c;
        s[S_DIAG_SUM] = sum;
        s[S_DIAG_MIN] = lo;
        s[S_DIAG_MAX] = hi;
        s[S_LAMBDA] = unknowns > 0 ? ridge * sum / (double)unknowns : 0.0;
    }
}

// Gauss-Jordan with partial pivoting on [a | I], n <= 4, in double (src/solve_level1.cu:689-740).
__device__ __forceinline__ bool invert(double* a, int n, double* inv)
{
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            inv[i * n + j] = i == j ? 1.0 : 0.0;
    for (int k = 0; k < n; k++)
    {
        int pivot = k;
        double best = fabs(a[k * n + k]);
        for (int i = k + 1; i < n; i++)
            if (fabs(a[i * n + k]) > best)
            {
                best = fabs(a[i * n + k]);
                pivot = i;
            }
        if (!(best > 0.0))
            return false;
        if (pivot != k)
            for (int j = 0; j < n; j++)
            {
                double t = a[k * n + j];
                a[k * n + j] = a[pivot * n + j];
                a[pivot * n + j] = t;
                t = inv[k * n + j];
                inv[k * n + j] = inv[pivot * n + j];
                inv[pivot * n + j] = t;
            }
        const double s = 1.0 / a[k * n + k];
        for (int j = 0; j < n; j++)
        {
            a[k * n + j] *= s;
            inv[k * n + j] *= s;
        }
        for (int i = 0; i < n; i++)
        {
            if (i == k)
                continue;
            const double f = a[i * n + k];
            if (f == 0.0)
                continue;
            for (int j = 0; j < n; j++)
            {
                a[i * n + j] -= f * a[k * n + j];
                inv[i * n + j] -= f * inv[k * n + j];
            }
        }
    }
    return true;
}

__device__ __forceinline__ void apply_precond(const float* minv, const double* r, int c, double* z)
{
    for (int i = 0; i < c; i++)
    {
        double acc = 0.0;
        for (int j = 0; j < c; j++)
            acc += (double)minv[i * c + j] * r[j];
        z[i] = acc;
    }
}

// y_t = (H_tt + lambda I) x_t + sum of the owned slots' blocks times the forward neighbours + the transposes of the
// backward neighbours' blocks (src/solve_level1.cu:781-828), in the reference's order of accumulation.
template <int C, typename TS>
__device__ __forceinline__ void stencil_apply(const PlaneView& V, size_t T, long long t, double lambda, const double* x,
                                              double* acc)
{
    constexpr int cc = C * C;
    const int tx = (int)(t % V.w), ty = (int)(t / V.w);
    const size_t sp = stencil_pos(tx, ty, V.w, V.h);
    const double* xt = x + (size_t)t * C;
    const StenBlock<C, TS> self(V, 0, T, sp);
#pragma unroll
    for (int i = 0; i < C; i++)
    {
        double s = lambda * xt[i];
#pragma unroll
        for (int j = 0; j < C; j++)
            s += self[i * C + j] * xt[j];
        acc[i] = s;
    }
    // Every neighbour's loads are issued whether or not the neighbour exists (from a clamped, in-range texel), and a
    // missing neighbour's products are replaced by -0.0, which leaves any sum, a signed zero included, exactly as it
    // was: the same bits as skipping those terms.
#pragma unroll
    for (int slot = 1; slot < SLOTS; slot++)
    {
        int dx, dy;
        slot_offset(slot, dx, dy);
        const int fx = tx + dx, fy = ty + dy;
        const bool fwd = fx >= 0 && fx < V.w && fy >= 0 && fy < V.h;
        const int gx = fwd ? fx : tx, gy = fwd ? fy : ty;
        const double* xn = x + ((size_t)gy * V.w + gx) * C;
        const StenBlock<C, TS> blk(V, slot, T, sp);
#pragma unroll
        for (int i = 0; i < C; i++)
#pragma unroll
            for (int j = 0; j < C; j++)
            {
                const double e = blk[i * C + j] * xn[j];
                acc[i] += fwd ? e : -0.0;
            }
        const int bx = tx - dx, by = ty - dy;
        const bool bwd = bx >= 0 && bx < V.w && by >= 0 && by < V.h;
        const int hx = bwd ? bx : tx, hy = bwd ? by : ty;
        const size_t nt = (size_t)hy * V.w + hx, np = stencil_pos(hx, hy, V.w, V.h);
        const double* xb = x + nt * C;
        const StenBlock<C, TS> nbk(V, slot, T, np);
#pragma unroll
        for (int i = 0; i < C; i++)
#pragma unroll
            for (int j = 0; j < C; j++)
            {
                const double e = nbk[j * C + i] * xb[j];
                acc[i] += bwd ? e : -0.0;
            }
    }
}

template <typename TS>
__global__ void __launch_bounds__(THREADS) k_precondition_init(Planes P, Red R)
{
    __shared__ double sh[2 * 32];
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long t = base - P.start[pl] + threadIdx.x;
    const size_t T = (size_t)V.w * V.h;
    const int c = P.c;
    double v[2] = { 0.0, 0.0 };
    const int kind[2] = { 0, 0 };
    if (t < (long long)T)
    {
        const double lambda = R.scalars[(size_t)pl * S_COUNT + S_LAMBDA];
        double a[MAX_CH * MAX_CH], inv[MAX_CH * MAX_CH];
        for (int i = 0; i < c; i++)
            for (int j = 0; j < c; j++)
                a[i * c + j] = sten<TS>(V, sten_index<TS>(0, i * c + j, c * c, T, stencil_pos((int)(t % V.w), (int)(t / V.w), V.w, V.h))) +
                               (i == j ? lambda : 0.0);
        if (!invert(a, c, inv))
            for (int i = 0; i < c; i++)
                for (int j = 0; j < c; j++)
                    inv[i * c + j] = i == j ? 1.0 : 0.0;
        float minv[MAX_CH * MAX_CH];
        for (int i = 0; i < c * c; i++)
        {
            minv[i] = (float)inv[i];
            V.precond[(size_t)t * c * c + i] = minv[i];
        }
        // CG from d = 0: r = -grad, z = M r, p = z.
        double r[MAX_CH], z[MAX_CH];
        for (int i = 0; i < c; i++)
        {
            r[i] = -V.grad[(size_t)t * c + i];
            V.x[(size_t)t * c + i] = 0.0;
            V.r[(size_t)t * c + i] = r[i];
        }
        apply_precond(minv, r, c, z);
        for (int i = 0; i < c; i++)
        {
            V.z[(size_t)t * c + i] = z[i];
            V.p[(size_t)t * c + i] = z[i];
            v[0] += r[i] * r[i];
            v[1] += r[i] * z[i];
        }
    }
    block_reduce(v, kind, sh);
    if (threadIdx.x == 0)
    {
        R.partial[blockIdx.x] = v[0];
        R.partial[R.nblocks + blockIdx.x] = v[1];
    }
}

__global__ void k_cg_start(Planes P, Red R)
{
    const int pl = blockIdx.x;
    const long long b0 = P.start[pl] / THREADS, b1 = P.start[pl + 1] / THREADS;
    const double rr = plane_total(R.partial, R.nblocks, b0, b1, 0, 0);
    const double rz = plane_total(R.partial, R.nblocks, b0, b1, 1, 0);
    if (threadIdx.x == 0)
    {
        double* s = R.scalars + (size_t)pl * S_COUNT;
        s[S_RHS2] = rr;
        s[S_RZ] = rz;
        s[S_ACTIVE] = 1.0;
        s[S_ITER] = 0.0;
        s[S_RESID] = 0.0;
    }
}

template <int C, typename TS>
__global__ void __launch_bounds__(THREADS) k_cg_matvec(Planes P, Red R)
{
    __shared__ double sh[32];
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const double* s = R.scalars + (size_t)pl * S_COUNT;
    if (s[S_ACTIVE] == 0.0)
        return;
    const PlaneView& V = P.p[pl];
    const long long t = base - P.start[pl] + threadIdx.x;
    const size_t T = (size_t)V.w * V.h;
    constexpr int c = C;
    double v[1] = { 0.0 };
    const int kind[1] = { 0 };
    if (t < (long long)T)
    {
        double acc[MAX_CH];
        stencil_apply<C, TS>(V, T, t, s[S_LAMBDA], V.p, acc);
#pragma unroll
        for (int i = 0; i < c; i++)
        {
            V.ap[(size_t)t * c + i] = acc[i];
            v[0] += V.p[(size_t)t * c + i] * acc[i];
        }
    }
    block_reduce(v, kind, sh);
    if (threadIdx.x == 0)
        R.partial[blockIdx.x] = v[0];
}

__global__ void k_cg_alpha(Planes P, Red R)
{
    const int pl = blockIdx.x;
    double* s = R.scalars + (size_t)pl * S_COUNT;
    if (s[S_ACTIVE] == 0.0)
        return;
    const long long b0 = P.start[pl] / THREADS, b1 = P.start[pl + 1] / THREADS;
    const double pap = plane_total(R.partial, R.nblocks, b0, b1, 0, 0);
    if (threadIdx.x == 0)
    {
        s[S_PAP] = pap;
        s[S_ALPHA] = pap > 0.0 ? s[S_RZ] / pap : 0.0;
    }
}

template <int C>
__global__ void __launch_bounds__(THREADS) k_cg_update(Planes P, Red R)
{
    __shared__ double sh[2 * 32];
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const double* s = R.scalars + (size_t)pl * S_COUNT;
    if (s[S_ACTIVE] == 0.0)
        return;
    const PlaneView& V = P.p[pl];
    const long long t = base - P.start[pl] + threadIdx.x;
    const size_t T = (size_t)V.w * V.h;
    constexpr int c = C;   // the channel count as a constant: r, z and the preconditioner stay in registers
    double v[2] = { 0.0, 0.0 };
    const int kind[2] = { 0, 0 };
    if (t < (long long)T)
    {
        const double alpha = s[S_ALPHA];
        double r[MAX_CH], z[MAX_CH];
#pragma unroll
        for (int i = 0; i < c; i++)
        {
            const size_t q = (size_t)t * c + i;
            V.x[q] += 1.0 * alpha * V.p[q];
            r[i] = V.r[q] + -1.0 * alpha * V.ap[q];
            V.r[q] = r[i];
        }
        float minv[MAX_CH * MAX_CH];
#pragma unroll
        for (int i = 0; i < c * c; i++)
            minv[i] = V.precond[(size_t)t * c * c + i];
#pragma unroll
        for (int i = 0; i < c; i++)
        {
            double acc = 0.0;
#pragma unroll
            for (int j = 0; j < c; j++)
                acc += (double)minv[i * c + j] * r[j];
            z[i] = acc;
        }
#pragma unroll
        for (int i = 0; i < c; i++)
        {
            V.z[(size_t)t * c + i] = z[i];
            v[0] += r[i] * r[i];
            v[1] += r[i] * z[i];
        }
    }
    block_reduce(v, kind, sh);
    if (threadIdx.x == 0)
    {
        R.partial[blockIdx.x] = v[0];
        R.partial[R.nblocks + blockIdx.x] = v[1];
    }
}

// beta, the residual, and the device-side stop: at an iteration that is a multiple of CG_PROBE a plane whose residual
// is not at or above the tolerance leaves (the reference's host probe, src/solve_level1.cu:1288-1302).
__global__ void k_cg_beta(Planes P, Red R, int it, unsigned int* active_count, double tol)
{
    const int pl = blockIdx.x;
    double* s = R.scalars + (size_t)pl * S_COUNT;
    if (s[S_ACTIVE] == 0.0)
        return;
    const long long b0 = P.start[pl] / THREADS, b1 = P.start[pl + 1] / THREADS;
    const double rr = plane_total(R.partial, R.nblocks, b0, b1, 0, 0);
    const double rz_new = plane_total(R.partial, R.nblocks, b0, b1, 1, 0);
    if (threadIdx.x == 0)
    {
        const double rz = s[S_RZ];
        s[S_RR] = rr;
        s[S_RZ_NEW] = rz_new;
        s[S_BETA] = rz != 0.0 ? rz_new / rz : 0.0;
        s[S_RZ] = rz_new;
        const double rhs2 = s[S_RHS2];
        s[S_RESID] = rhs2 > 0.0 ? sqrt((rr > 0.0 ? rr : 0.0) / rhs2) : 0.0;
        s[S_ITER] = (double)(it + 1);
        if ((it + 1) % CG_PROBE == 0 && !(s[S_RESID] >= tol))
            s[S_ACTIVE] = 0.5;   // leaves after this iteration's direction update (which no longer matters)
        else
            atomicAdd(active_count, 1u);
    }
}

__global__ void __launch_bounds__(THREADS) k_cg_direction(Planes P, Red R)
{
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const double* s = R.scalars + (size_t)pl * S_COUNT;
    if (s[S_ACTIVE] == 0.0)
        return;
    const PlaneView& V = P.p[pl];
    const long long t = base - P.start[pl] + threadIdx.x;
    const size_t T = (size_t)V.w * V.h;
    if (t >= (long long)T)
        return;
    const double beta = s[S_BETA];
    for (int i = 0; i < P.c; i++)
    {
        const size_t q = (size_t)t * P.c + i;
        V.p[q] = V.z[q] + beta * V.p[q];
    }
}

__global__ void k_cg_retire(Planes P, double* scalars)
{
    const int pl = threadIdx.x;
    if (pl < P.n && scalars[(size_t)pl * S_COUNT + S_ACTIVE] == 0.5)
        scalars[(size_t)pl * S_COUNT + S_ACTIVE] = 0.0;
}

// ---- the correction and the movement probe (src/solve_level1.cu:872-979) -------------------------------------------

__global__ void __launch_bounds__(THREADS) k_correct_range(Planes P, Red R)
{
    __shared__ double sh[2 * MAX_CH * 32];
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long t = base - P.start[pl] + threadIdx.x;
    const size_t T = (size_t)V.w * V.h;
    const int c = P.c;
    double v[2 * MAX_CH];
    int kind[2 * MAX_CH];
    for (int q = 0; q < MAX_CH; q++)
    {
        v[q] = 1e300;
        v[MAX_CH + q] = -1e300;
        kind[q] = 1;
        kind[MAX_CH + q] = 2;
    }
    if (t < (long long)T)
        for (int i = 0; i < c; i++)
        {
            const size_t q = (size_t)t * c + i;
            const float nv = (float)((double)V.v[q] + V.x[q]);
            V.v[q] = nv;
            v[i] = (double)nv;
            v[MAX_CH + i] = (double)nv;
        }
    block_reduce(v, kind, sh);
    if (threadIdx.x == 0)
        for (int q = 0; q < c; q++)
        {
            R.partial[(size_t)(3 + q) * R.nblocks + blockIdx.x] = v[q];
            R.partial[(size_t)(3 + MAX_CH + q) * R.nblocks + blockIdx.x] = v[MAX_CH + q];
        }
}

__global__ void k_range_reduce(Planes P, Red R)
{
    const int pl = blockIdx.x;
    const long long b0 = P.start[pl] / THREADS, b1 = P.start[pl + 1] / THREADS;
    for (int q = 0; q < P.c; q++)
    {
        const double lo = plane_total(R.partial, R.nblocks, b0, b1, 3 + q, 1);
        const double hi = plane_total(R.partial, R.nblocks, b0, b1, 3 + MAX_CH + q, 2);
        if (threadIdx.x == 0)
        {
            R.scalars[(size_t)pl * S_COUNT + S_LO + q] = lo;
            R.scalars[(size_t)pl * S_COUNT + S_HI + q] = hi;
        }
    }
}

__global__ void __launch_bounds__(THREADS) k_movement(Planes P, Red R, int levels)
{
    __shared__ double sh[3 * 32];
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const double* s = R.scalars + (size_t)pl * S_COUNT;
    const long long t = base - P.start[pl] + threadIdx.x;
    const size_t T = (size_t)V.w * V.h;
    const int c = P.c;
    double v[3] = { 0.0, 0.0, 0.0 };
    const int kind[3] = { 0, 0, 0 };
    if (t < (long long)T)
        for (int i = 0; i < c; i++)
        {
            const size_t q = (size_t)t * c + i;
            const double step = (s[S_HI + i] - s[S_LO + i]) / (double)levels;
            const double dq = V.x[q];
            if (fabs(dq) > 0.5 * step)
                v[0] += 1.0;
            v[1] += dq * dq;
            v[2] += (double)V.v[q] * (double)V.v[q];
        }
    block_reduce(v, kind, sh);
    if (threadIdx.x == 0)
        for (int q = 0; q < 3; q++)
            R.partial[(size_t)q * R.nblocks + blockIdx.x] = v[q];
}

__global__ void k_movement_reduce(Planes P, Red R)
{
    const int pl = blockIdx.x;
    const long long b0 = P.start[pl] / THREADS, b1 = P.start[pl + 1] / THREADS;
    const double moved = plane_total(R.partial, R.nblocks, b0, b1, 0, 0);
    const double d2 = plane_total(R.partial, R.nblocks, b0, b1, 1, 0);
    const double p2 = plane_total(R.partial, R.nblocks, b0, b1, 2, 0);
    if (threadIdx.x == 0)
    {
        double* s = R.scalars + (size_t)pl * S_COUNT;
        s[S_MOVED] = moved;
        s[S_DELTA2] = d2;
        s[S_PLANE2] = p2;
    }
}

// ---- the quantised phase (src/solve_level1.cu:1023-1098) ----------------------------------------------------------

struct SweepArgs
{
    const double* scalars;
    const float* lo;
    const float* hi;
    int bits;
    int cx, cy;
    unsigned int* moved;   // [plane]
};

template <int C, typename TS>
__global__ void __launch_bounds__(THREADS) k_quant_sweep(Planes P, SweepArgs A)
{
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long ci = base - P.start[pl] + threadIdx.x;
    const int cwn = (V.w - A.cx + 1) / 2, chn = (V.h - A.cy + 1) / 2;
    if (ci >= (long long)cwn * chn)
        return;
    const int tx = A.cx + 2 * (int)(ci % cwn);
    const int ty = A.cy + 2 * (int)(ci / cwn);
    const size_t t = (size_t)ty * V.w + tx;
    const size_t sp = stencil_pos(tx, ty, V.w, V.h);
    const size_t T = (size_t)V.w * V.h;
    constexpr int c = C, cc = C * C;
    const double lambda = A.scalars[(size_t)pl * S_COUNT + S_LAMBDA];
    double nb[MAX_CH];
#pragma unroll
    for (int i = 0; i < c; i++)
        nb[i] = 0.0;
    // as in stencil_apply: every load issued, a missing neighbour's products replaced by -0.0 (an exact no-op)
#pragma unroll
    for (int slot = 1; slot < SLOTS; slot++)
    {
        int dx, dy;
        slot_offset(slot, dx, dy);
        const int fx = tx + dx, fy = ty + dy;
        const bool fwd = fx >= 0 && fx < V.w && fy >= 0 && fy < V.h;
        const int gx = fwd ? fx : tx, gy = fwd ? fy : ty;
        const double* xn = V.x + ((size_t)gy * V.w + gx) * c;
        const StenBlock<C, TS> blk(V, slot, T, sp);
#pragma unroll
        for (int i = 0; i < c; i++)
#pragma unroll
            for (int j = 0; j < c; j++)
            {
                const double e = blk[i * c + j] * xn[j];
                nb[i] += fwd ? e : -0.0;
            }
        const int bx = tx - dx, by = ty - dy;
        const bool bwd = bx >= 0 && bx < V.w && by >= 0 && by < V.h;
        const int hx = bwd ? bx : tx, hy = bwd ? by : ty;
        const size_t nt = (size_t)hy * V.w + hx, np = stencil_pos(hx, hy, V.w, V.h);
        const double* xb = V.x + nt * c;
        const StenBlock<C, TS> nbk(V, slot, T, np);
#pragma unroll
        for (int i = 0; i < c; i++)
#pragma unroll
            for (int j = 0; j < c; j++)
            {
                const double e = nbk[j * c + i] * xb[j];
                nb[i] += bwd ? e : -0.0;
            }
    }
    const StenBlock<C, TS> self(V, 0, T, sp);
    unsigned int changed = 0;
#pragma unroll
    for (int q = 0; q < c; q++)
    {
        const size_t idx = t * c + q;
        const float l = A.lo[q], span = A.hi[q] - A.lo[q];
        const double a = self[q * c + q] + lambda;
        if (!(a > 0.0) || !(span > 0.0f))
            continue;
        double rest = nb[q];
#pragma unroll
        for (int j = 0; j < c; j++)
            if (j != q)
                rest += self[q * c + j] * V.x[t * c + j];
        const double b = V.grad[idx] + rest;
        const double want = (double)V.prev[idx] - b / a;
        const int kk = grid_index(l, A.hi[q], A.bits, (float)want);
        const float value = grid_value(l, A.hi[q], A.bits, kk);
        if ((int)V.k[idx] != kk)
        {
            V.k[idx] = (uint8_t)kk;
            changed++;
        }
        V.v[idx] = value;
        V.x[idx] = (double)value - (double)V.prev[idx];
    }
    if (changed)
        atomicAdd(A.moved + pl, changed);
}

// prev = v, x = 0 (the quantised path and the refinement measure the correction from the plane as assembled).
__global__ void k_snapshot(Planes P)
{
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long t = base - P.start[pl] + threadIdx.x;
    if (t >= (long long)V.w * V.h)
        return;
    for (int i = 0; i < P.c; i++)
    {
        const size_t q = (size_t)t * P.c + i;
        V.prev[q] = V.v[q];
        V.x[q] = 0.0;
    }
}

// ---- host drivers ---------------------------------------------------------------------------------------------------

static Planes texel_planes(nntc_b200_device* d, int level0, int k)
{
    Planes P = planes_for(d, level0, [&](int i) { return d->planes[(size_t)i].work[level0 ? 1 : 0].texels(); });
    P.kc = k;
    return P;
}

static Red red_for(nntc_b200_device* d, const Planes& P)
{
    return Red{ d->partial, (size_t)(P.start[P.n] / THREADS), d->scalars };
}

int assemble_split(nntc_b200_device* d, int k, int level0, const Planes& P_texels, int nmono, const double* mono,
                   int slots, bool f32);
int matvec_free(nntc_b200_device* d, const Planes& P, double* partial, int level0);

// diag_only: the gradient and the diagonal blocks (slot 0) alone, what the matrix-free conjugate gradients of the
// adjoint form need (their products come from adjoint_cg.cu, not from the other four slots).
int assemble(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge, int level0, bool diag_only = false)
{
    if (level0 && !d->l0_bc8)
    {
        set_error(NNTC_B200_ERR_STATE, "block (c') runs only under --l0 bc8");
        return NNTC_B200_ERR_STATE;
    }
    std::vector<double> mono;
    build_monomials(*m, level0, mono);
    NB_TRY(upload(d, d->mono[level0], mono.data(), mono.size() * sizeof(double)));
    Planes P = texel_planes(d, level0, k);
    const int nmono = monomial_count(level0 ? d->c1 : d->c0);
    const int blocks = (int)(P.start[P.n] / ASM_THREADS);
    const size_t shared = (size_t)SLOTS * nmono * ASM_THREADS * sizeof(double);
    AsmArgs A{ d->weights, d->bias, d->cw, d->mono[level0], nmono };
    NB_TRY(ktimer_begin(d, level0 ? NNTC_B200_K_ASSEMBLE0 : NNTC_B200_K_ASSEMBLE1));
    const bool split = diag_only || (!d->reference_shaped_assembly && k <= 4);
    // the adjoint form stores the stencil in FP32 (the split form only; the reference-shaped kernel is FP64)
    d->sten_f32[level0] = split && d->mixed_stencil != 0;
    if (split)
        NB_TRY(assemble_split(d, k, level0, P, nmono, mono.data(), diag_only ? 1 : SLOTS, d->sten_f32[level0]));
    else if (level0)
    {
        NB_CUDA(cudaFuncSetAttribute(k_assemble<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shared));
        k_assemble<true><<<blocks, ASM_THREADS, shared, d->stream>>>(P, A);
    }
    else
    {
        NB_CUDA(cudaFuncSetAttribute(k_assemble<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shared));
        k_assemble<false><<<blocks, ASM_THREADS, shared, d->stream>>>(P, A);
    }
    NB_TRY(ktimer_end(d));
    if (!diag_only && (d->reference_shaped_assembly || k > 4))
        NB_LAUNCHED();
    const Red R = red_for(d, P);
    const int tblocks = (int)(P.start[P.n] / THREADS);
    if (d->sten_f32[level0])
        k_diag<float><<<tblocks, THREADS, 0, d->stream>>>(P, R);
    else
        k_diag<double><<<tblocks, THREADS, 0, d->stream>>>(P, R);
    NB_LAUNCHED();
    k_diag_reduce<<<P.n, 32, 0, d->stream>>>(P, R, ridge);
    NB_LAUNCHED();
    return NNTC_B200_OK;
}

static void fill_report(const nntc_b200_device* d, int i, int channels, nntc_b200_plane_report& rep)
{
    const double* s = d->host_scalars + (size_t)i * S_COUNT;
    rep.lambda = s[S_LAMBDA];
    rep.min_diag = s[S_DIAG_MIN];
    rep.max_diag = s[S_DIAG_MAX];
    rep.residual = s[S_RESID];
    rep.moved_values = (long long)s[S_MOVED];
    rep.delta2 = s[S_DELTA2];
    rep.plane2 = s[S_PLANE2];
    for (int c = 0; c < channels; c++)
    {
        rep.lo[c] = (float)s[S_LO + c];
        rep.hi[c] = (float)s[S_HI + c];
    }
}

int solve_block(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge, int level0,
                nntc_b200_plane_report* rep, double* ms)
{
    const int np = (int)d->planes.size();
    const int nc = level0 ? d->c0 : d->c1;
    for (int i = 0; i < np; i++)
        rep[i] = nntc_b200_plane_report{};
    // the adjoint form: the gradient and the diagonal blocks assembled, the products matrix-free (adjoint_cg.cu)
    const bool adjoint = d->adjoint_cg != 0 && k <= 4;
    NB_TRY(block_begin(d));
    NB_TRY(assemble(d, m, k, ridge, level0, adjoint));
    NB_CUDA(cudaEventRecord(d->ev[2], d->stream));
    Planes P = texel_planes(d, level0, k);
    const Red R = red_for(d, P);
    const int tblocks = (int)(P.start[P.n] / THREADS);
    if (d->sten_f32[level0])
        k_precondition_init<float><<<tblocks, THREADS, 0, d->stream>>>(P, R);
    else
        k_precondition_init<double><<<tblocks, THREADS, 0, d->stream>>>(P, R);
    NB_LAUNCHED();
    k_cg_start<<<P.n, 32, 0, d->stream>>>(P, R);
    NB_LAUNCHED();
    NB_CUDA(cudaEventRecord(d->ev[3], d->stream));
    unsigned int* active = d->counters + CNT_ACTIVE;
    for (int it = 0; it < CG_MAX_IT; it++)
    {
        NB_CUDA(cudaMemsetAsync(active + (it % CG_PROBE), 0, sizeof(unsigned int), d->stream));
        NB_TRY(ktimer_begin(d, level0 ? NNTC_B200_K_MATVEC0 : NNTC_B200_K_MATVEC));
        if (adjoint)
            NB_TRY(matvec_free(d, P, R.partial, level0));
        else
        {
#define NB_MATVEC(TS)                                                                                                 \
    switch (P.c)                                                                                                      \
    {                                                                                                                 \
    case 1: k_cg_matvec<1, TS><<<tblocks, THREADS, 0, d->stream>>>(P, R); break;                                      \
    case 2: k_cg_matvec<2, TS><<<tblocks, THREADS, 0, d->stream>>>(P, R); break;                                      \
    case 3: k_cg_matvec<3, TS><<<tblocks, THREADS, 0, d->stream>>>(P, R); break;                                      \
    default: k_cg_matvec<4, TS><<<tblocks, THREADS, 0, d->stream>>>(P, R); break;                                     \
    }
            if (d->sten_f32[level0])
            {
                NB_MATVEC(float)
            }
            else
            {
                NB_MATVEC(double)
            }
#undef NB_MATVEC
            NB_LAUNCHED();
        }
        NB_TRY(ktimer_end(d));
        k_cg_alpha<<<P.n, 32, 0, d->stream>>>(P, R);
        NB_LAUNCHED();
        switch (P.c)
        {
        case 1: k_cg_update<1><<<tblocks, THREADS, 0, d->stream>>>(P, R); break;
        case 2: k_cg_update<2><<<tblocks, THREADS, 0, d->stream>>>(P, R); break;
        case 3: k_cg_update<3><<<tblocks, THREADS, 0, d->stream>>>(P, R); break;
        default: k_cg_update<4><<<tblocks, THREADS, 0, d->stream>>>(P, R); break;
        }
        NB_LAUNCHED();
        k_cg_beta<<<P.n, 32, 0, d->stream>>>(P, R, it, active + (it % CG_PROBE),
                                             adjoint || d->sten_f32[level0] ? CG_TOL_FP32 : CG_TOL);
        NB_LAUNCHED();
        k_cg_direction<<<tblocks, THREADS, 0, d->stream>>>(P, R);
        NB_LAUNCHED();
        k_cg_retire<<<1, 32, 0, d->stream>>>(P, d->scalars);
        NB_LAUNCHED();
        if ((it + 1) % CG_PROBE != 0)
            continue;
        unsigned int still = 0;
        NB_CUDA(cudaMemcpyAsync(&still, active + (it % CG_PROBE), sizeof(unsigned int), cudaMemcpyDeviceToHost,
                                d->stream));
        NB_CUDA(cudaStreamSynchronize(d->stream));
        if (still == 0)
            break;
    }
    k_correct_range<<<tblocks, THREADS, 0, d->stream>>>(P, R);
    NB_LAUNCHED();
    k_range_reduce<<<P.n, 32, 0, d->stream>>>(P, R);
    NB_LAUNCHED();
    const int levels = level0 ? 255 : (1 << m->bits1) - 1;
    k_movement<<<tblocks, THREADS, 0, d->stream>>>(P, R, levels);
    NB_LAUNCHED();
    k_movement_reduce<<<P.n, 32, 0, d->stream>>>(P, R);
    NB_LAUNCHED();
    NB_CUDA(cudaMemcpyAsync(d->host_scalars, d->scalars, (size_t)np * S_COUNT * sizeof(double),
                            cudaMemcpyDeviceToHost, d->stream));
    double t = 0.0;
    NB_TRY(block_end(d, &t));
    float a_ms = 0.0f, p_ms = 0.0f, c_ms = 0.0f;
    NB_CUDA(cudaEventElapsedTime(&a_ms, d->ev[0], d->ev[2]));
    NB_CUDA(cudaEventElapsedTime(&p_ms, d->ev[2], d->ev[3]));
    NB_CUDA(cudaEventElapsedTime(&c_ms, d->ev[3], d->ev[1]));
    for (int i = 0; i < np; i++)
    {
        fill_report(d, i, nc, rep[i]);
        rep[i].iterations = (int)d->host_scalars[(size_t)i * S_COUNT + S_ITER];
        rep[i].quantised = 0;
        rep[i].ms_assemble = a_ms;
        rep[i].ms_precond = p_ms;
        rep[i].ms_cg = c_ms;
    }
    if (ms)
        *ms = t;
    return NNTC_B200_OK;
}

int sweep_block(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge, int sweeps, int level0,
                nntc_b200_plane_report* rep, double* ms)
{
    const int np = (int)d->planes.size();
    const int nc = level0 ? d->c0 : d->c1;
    for (int i = 0; i < np; i++)
        rep[i] = nntc_b200_plane_report{};
    // every slot assembled whatever the conjugate gradients' operator: a sweep step reads the texel's coupling to its
    // eight neighbours from the stencil (with the matrix-free option on, an assembly of the diagonal blocks alone
    // would leave the sweeps reading another block's off-diagonal slots)
    NB_TRY(block_begin(d));
    NB_TRY(assemble(d, m, k, ridge, level0, false));
    NB_CUDA(cudaEventRecord(d->ev[2], d->stream));
    Planes P = texel_planes(d, level0, k);
    k_snapshot<<<(int)(P.start[P.n] / THREADS), THREADS, 0, d->stream>>>(P);
    NB_LAUNCHED();
    NB_CUDA(cudaMemsetAsync(d->counters + CNT_SWEEP, 0, MAX_PLANES * sizeof(unsigned int), d->stream));
    const int bits = level0 ? 8 : m->bits1;
    for (int s = 0; s < sweeps; s++)
        for (int colour = 0; colour < 4; colour++)
        {
            const int cx = colour & 1, cy = colour >> 1;
            Planes C = planes_for(d, level0, [&](int i) {
                const Work& w = d->planes[(size_t)i].work[level0 ? 1 : 0];
                return (size_t)((w.w - cx + 1) / 2) * (size_t)((w.h - cy + 1) / 2);
            });
            C.kc = k;
            if (C.start[C.n] == 0)
                continue;
            SweepArgs A{ d->scalars, level0 ? d->lo0 : d->lo1, level0 ? d->hi0 : d->hi1, bits, cx, cy, d->counters + CNT_SWEEP };
            NB_TRY(ktimer_begin(d, NNTC_B200_K_SWEEP));
            const int sblocks = (int)(C.start[C.n] / THREADS);
#define NB_SWEEP(TS)                                                                                                  \
    switch (C.c)                                                                                                      \
    {                                                                                                                 \
    case 1: k_quant_sweep<1, TS><<<sblocks, THREADS, 0, d->stream>>>(C, A); break;                                    \
    case 2: k_quant_sweep<2, TS><<<sblocks, THREADS, 0, d->stream>>>(C, A); break;                                    \
    case 3: k_quant_sweep<3, TS><<<sblocks, THREADS, 0, d->stream>>>(C, A); break;                                    \
    default: k_quant_sweep<4, TS><<<sblocks, THREADS, 0, d->stream>>>(C, A); break;                                   \
    }
            if (d->sten_f32[level0])
            {
                NB_SWEEP(float)
            }
            else
            {
                NB_SWEEP(double)
            }
#undef NB_SWEEP
            NB_TRY(ktimer_end(d));
            NB_LAUNCHED();
        }
    NB_CUDA(cudaEventRecord(d->ev[3], d->stream));
    NB_CUDA(cudaMemcpyAsync(d->host_scalars, d->scalars, (size_t)np * S_COUNT * sizeof(double),
                            cudaMemcpyDeviceToHost, d->stream));
    NB_CUDA(cudaMemcpyAsync(d->host_counters, d->counters, MAX_PLANES * sizeof(unsigned int),
                            cudaMemcpyDeviceToHost, d->stream));
    double t = 0.0;
    NB_TRY(block_end(d, &t));
    float a_ms = 0.0f, s_ms = 0.0f;
    NB_CUDA(cudaEventElapsedTime(&a_ms, d->ev[0], d->ev[2]));
    NB_CUDA(cudaEventElapsedTime(&s_ms, d->ev[2], d->ev[3]));
    for (int i = 0; i < np; i++)
    {
        fill_report(d, i, nc, rep[i]);
        rep[i].quantised = 1;
        rep[i].sweeps = sweeps;
        rep[i].ms_assemble = a_ms;
        rep[i].ms_sweeps = s_ms;
        // the fields only the continuous path writes are cleared (src/solve_level1.cu:1388-1397)
        rep[i].iterations = 0;
        rep[i].residual = 0.0;
        rep[i].moved_values = 0;
        rep[i].delta2 = 0.0;
        rep[i].plane2 = 0.0;
        rep[i].moved = (long long)d->host_counters[i];
    }
    if (ms)
        *ms = t;
    return NNTC_B200_OK;
}

// The gradient, the diagonal blocks and the preconditioned descent direction of one latent at its current plane:
// grad, z = -(H_tt + lambda I)^-1 grad texel by texel, prev = v (what the joint pass steps from).
int descent_direction(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge, int level0)
{
    NB_TRY(assemble(d, m, k, ridge, level0, true));
    Planes P = texel_planes(d, level0, k);
    const Red R = red_for(d, P);
    const int tblocks = (int)(P.start[P.n] / THREADS);
    if (d->sten_f32[level0])
        k_precondition_init<float><<<tblocks, THREADS, 0, d->stream>>>(P, R);
    else
        k_precondition_init<double><<<tblocks, THREADS, 0, d->stream>>>(P, R);
    NB_LAUNCHED();
    k_snapshot<<<tblocks, THREADS, 0, d->stream>>>(P);
    NB_LAUNCHED();
    return NNTC_B200_OK;
}

// Level 0's stencil copied into the BC refinement's block-major layout (bc_sten: [block][slot][i][j][texel of the
// block]), one thread per texel; used when the assembly did not write the copy itself.
__global__ void k_bc_sten_copy(Planes P)
{
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long t = base - P.start[pl] + threadIdx.x;
    if (t >= (long long)V.w * V.h)
        return;
    const int x = (int)(t % V.w), y = (int)(t / V.w), cc = P.c * P.c;
    const size_t T = (size_t)V.w * V.h, sp = stencil_pos(x, y, V.w, V.h);
    const size_t blk = (size_t)(y >> 2) * (size_t)((V.w + 3) >> 2) + (size_t)(x >> 2);
    const int in = (y & 3) * 4 + (x & 3);
    for (int slot = 0; slot < SLOTS; slot++)
        for (int e = 0; e < cc; e++)
            V.bc_sten[((blk * SLOTS + slot) * cc + e) * 16 + in] = V.stencil[(size_t)(slot * cc + e) * T + sp];
}

// Block (c')'s assembly alone with no ridge, the correction measured from the plane as it stands (for refine_bc). The
// refinement's decisions are the reference's on an FP64 stencil, so this assembly is FP64 in either form.
int assemble_for_refine(nntc_b200_device* d, const nntc_b200_model* m, int k, double* ms)
{
    struct Fp64Scope
    {
        nntc_b200_device* d;
        int was;
        ~Fp64Scope()
        {
            d->mixed_stencil = was;
            d->bc_copy = 0;
        }
    } fp64{ d, d->mixed_stencil };
    d->mixed_stencil = 0;
    d->bc_copy = 1;   // the refinement reads the block-major copy the gather writes beside the stencil
    d->bc_copied = 0;
    NB_TRY(block_begin(d));
    NB_TRY(assemble(d, m, k, 0.0, 1));
    Planes P = texel_planes(d, 1, k);
    if (!d->bc_copied)
    {
        // the reference-shaped assembly wrote the stencil alone: the copy from it
        k_bc_sten_copy<<<(int)(P.start[P.n] / THREADS), THREADS, 0, d->stream>>>(P);
        NB_LAUNCHED();
    }
    k_snapshot<<<(int)(P.start[P.n] / THREADS), THREADS, 0, d->stream>>>(P);
    NB_LAUNCHED();
    return block_end(d, ms);
}

}   // namespace nb

using namespace nb;

extern "C"
{

int nntc_b200_set_option(nntc_b200_device* d, int option, int value)
{
    if (option == NNTC_B200_OPT_REFERENCE_SHAPED_ASSEMBLY)
    {
        d->reference_shaped_assembly = value != 0;
        return NNTC_B200_OK;
    }
    if (option == NNTC_B200_OPT_MIXED_PRECISION_GRAM)
    {
        d->mixed_gram = value != 0;
        return NNTC_B200_OK;
    }
    if (option == NNTC_B200_OPT_ADJOINT_CG)
    {
        d->adjoint_cg = value != 0;
        return NNTC_B200_OK;
    }
    if (option == NNTC_B200_OPT_MIXED_OBJECTIVE)
    {
        d->mixed_objective = value != 0;
        return NNTC_B200_OK;
    }
    if (option == NNTC_B200_OPT_FP32_STENCIL)
    {
        d->mixed_stencil = value != 0;
        return NNTC_B200_OK;
    }
    set_error(NNTC_B200_ERR_ARG, "no such option");
    return NNTC_B200_ERR_ARG;
}

int nntc_b200_solve_level1_all(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge,
                               nntc_b200_plane_report* rep, double* ms)
{
    return solve_block(d, m, k, ridge, 0, rep, ms);
}

int nntc_b200_sweep_level1_all(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge, int sweeps,
                               nntc_b200_plane_report* rep, double* ms)
{
    return sweep_block(d, m, k, ridge, sweeps, 0, rep, ms);
}

int nntc_b200_solve_level0_cont_all(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge,
                                    nntc_b200_plane_report* rep, double* ms)
{
    return solve_block(d, m, k, ridge, 1, rep, ms);
}

int nntc_b200_sweep_level0_cont_all(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge, int sweeps,
                                    nntc_b200_plane_report* rep, double* ms)
{
    return sweep_block(d, m, k, ridge, sweeps, 1, rep, ms);
}

int nntc_b200_assemble_level0_for_refine(nntc_b200_device* d, const nntc_b200_model* m, int k, double* ms)
{
    return assemble_for_refine(d, m, k, ms);
}

}   // extern "C"
