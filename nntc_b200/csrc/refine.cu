// refine.cu: the BC4/BC5 pack of level 0 and its refinement by analysis by synthesis (src/refine_bc.cu).
//
// With level 1 and the decoder held, E is an exact quadratic in level 0's values; restricted to one 4x4 block with
// every texel outside it held it is E_blk(d) = const + 2 A1.d + d^T A2 d (src/refine_bc.cu:15-45). Per block and
// channel the endpoints move by a 2x2 least squares with its nine rounded candidates, then two Gauss-Seidel passes
// of exact 8-way selector argmins; a step is taken only on a strict decrease weighed in the float arithmetic the
// file decodes in (src/refine_bc.cu:47-95). Four colours over the block grid keep every block's neighbourhood frozen.
//
// B200 shape: ONE WARP PER 4x4 BLOCK, with the block's A2 (up to 64 x 64 doubles) in shared memory, read from a
// block-major copy of the FP64 stencil that the refinement's own assembly writes (a block's coefficients contiguous,
// so the warp's reads are whole lines instead of scattered doubles of the colour-major stencil). Every value is
// computed with the arithmetic of the reference's CPU transcription (src/cpu/cpu_refine_bc.cpp:134-400), including
// its order of summation: each block sum is a SERIAL fold over the sixteen texels in increasing order, which a warp
// reproduces exactly by shuffling the sixteen per-lane terms to every lane and folding them in texel order. The
// selector argmin evaluates its eight candidates on eight lanes and scans them in candidate order. Given the same
// stencil, gradient and planes the endpoints and selectors are therefore the same bytes as the reference's.
//
// The seed pack (src/export.cpp:294-328 over shared/bc_pack.h:95-188) runs here on the device as well: one thread
// per block-channel, integer arithmetic and the same float palette distances.

#include <cmath>
#include <cstring>
#include <vector>

#include "bc.cuh"
#include "device.cuh"

namespace nb
{

constexpr int REFINE_WARPS = 2;   // 4x4 blocks per CTA

__host__ __device__ __forceinline__ double bc4_weight8(int sel)
{
    return sel == 0 ? 1.0 : (sel == 1 ? 0.0 : (double)(8 - sel) / 7.0);
}

__host__ __device__ __forceinline__ float bc4_entry(int r0, int r1, int sel)
{
    if (sel == 0)
        return (float)r0;
    if (sel == 1)
        return (float)r1;
    return (float)((8 - sel) * r0 + (sel - 1) * r1) / 7.0f;
}

__host__ __device__ __forceinline__ float bc0_value(float lo, float hi, float byte)
{
    const double frac = (double)byte / 255.0;
    const double span = (double)hi - (double)lo;
#ifdef __CUDA_ARCH__
    return (float)__dadd_rn((double)lo, __dmul_rn(frac, span));
#else
    return (float)((double)lo + frac * span);
#endif
}

__host__ __device__ __forceinline__ uint8_t bc0_index(float byte)
{
    return (uint8_t)(byte < 0.0f ? 0 : (byte > 255.0f ? 255 : (int)(byte + 0.5f)));
}

struct BcPlane
{
    int w0, h0, bx;
    uint8_t* ep;
    uint8_t* sel;
    const uint8_t* k0src;   // the indices the seed pack reads
    float* v0;
    uint8_t* k0;
    double* delta;
    const float* prev;
    const double* bsten;    // level 0's FP64 stencil, block-major: [block][slot][i][j][texel of the block]
    const double* grad;
};

struct BcPlanes
{
    int n, c0;
    int bits[MAX_CH];
    long long start[MAX_PLANES + 1];
    BcPlane p[MAX_PLANES];
};

__device__ __forceinline__ int bc_plane_of(const BcPlanes& P, long long i)
{
    int lo = 0;
    while (lo + 1 < P.n && P.start[lo + 1] <= i)
        lo++;
    return lo;
}

// One thread per block-channel: the stb_dxt-style seed (src/export.cpp:294-328).
__global__ void k_bc_seed(BcPlanes P)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.start[P.n])
        return;
    const int pl = bc_plane_of(P, i);
    const BcPlane& B = P.p[pl];
    const long long local = i - P.start[pl];
    const int c0 = P.c0;
    const long long blk = local / c0;
    const int c = (int)(local % c0);
    if (blk >= (long long)B.bx * ((B.h0 + 3) / 4))
        return;
    const int gx = (int)(blk % B.bx), gy = (int)(blk / B.bx);
    const int bits = P.bits[c];
    uint8_t v[16];
    for (int t = 0; t < 16; t++)
    {
        const int px = min(B.w0 - 1, gx * 4 + t % 4), py = min(B.h0 - 1, gy * 4 + t / 4);
        v[t] = (uint8_t)rep_index((int)B.k0src[((size_t)py * B.w0 + px) * c0 + c], bits);
    }
    int r0, r1;
    uint8_t sel[16];
    bc4_seed_block(v, bits, r0, r1, sel);
    const size_t slot = (size_t)blk * c0 + c;
    B.ep[slot * 2] = (uint8_t)r0;
    B.ep[slot * 2 + 1] = (uint8_t)r1;
    for (int t = 0; t < 16; t++)
        B.sel[slot * 16 + t] = sel[t];
}

// Endpoints and selectors to the plane, its indices and the correction (src/refine_bc.cu:155-174).
__global__ void k_bc_decode(BcPlanes P, const float* lo0, const float* hi0)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.start[P.n])
        return;
    const int pl = bc_plane_of(P, i);
    const BcPlane& B = P.p[pl];
    const long long ti = i - P.start[pl];
    if (ti >= (long long)B.w0 * B.h0)
        return;
    const int px = (int)(ti % B.w0), py = (int)(ti / B.w0);
    const size_t gi = (size_t)(py / 4) * B.bx + (px / 4);
    const int t = (py % 4) * 4 + (px % 4);
    const int c0 = P.c0;
    for (int c = 0; c < c0; c++)
    {
        const size_t b = gi * c0 + c;
        const float byte = bc4_entry(B.ep[b * 2], B.ep[b * 2 + 1], B.sel[b * 16 + t]);
        const float value = bc0_value(lo0[c], hi0[c], byte);
        const size_t idx = (size_t)ti * c0 + c;
        B.v0[idx] = value;
        B.k0[idx] = bc0_index(byte);
        B.delta[idx] = (double)value - (double)B.prev[idx];
    }
}

// The layout of one warp's block in shared memory, per level-0 channel count.
//
// A2 couples a texel only with itself and its eight neighbours (the 9-point stencil), so it is held as the sixteen
// texels' five OWNED stencil blocks, S[texel][slot][i][j] (the texel stride padded to an odd number of doubles), and
// an entry A2[(t, i)][(u, j)] is read from t's block when u sits at one of t's owned offsets, else from u's block,
// transposed. Every sum over a row of A2 visits only the entries that can be nonzero, in column order: such a sum
// starts at +0.0 and so never holds -0.0, and adding the product of a structural zero would leave it bit-for-bit
// unchanged. The vector u = A2 d lives in registers, R rows per lane.
template <int C0>
struct RefineShape
{
    static constexpr int N = 16 * C0;              // unknowns of the block: (texel, channel), texel-major
    static constexpr int R = (N + 31) / 32;        // rows of u per lane: row r = lane + 32 q
    static constexpr int CC = C0 * C0;
    static constexpr int TS = (5 * CC) | 1;        // doubles per texel of S
    static constexpr int PER_WARP = 16 * TS + 2 * N + 16 + 8 + 16;   // S, a1, d, dlt, the weights, ep and sel
};

// The entry of A2 at row (t, i), column (u, j), where u is t's neighbour number k (k = (dy + 1) 3 + (dx + 1), the
// neighbours' order by texel index).
template <int C0>
__device__ __forceinline__ double a2_entry(const double* S, int t, int i, int u, int j, int k)
{
    using Sh = RefineShape<C0>;
    return k >= 4 ? S[t * Sh::TS + (k - 4) * Sh::CC + i * C0 + j] : S[u * Sh::TS + (4 - k) * Sh::CC + j * C0 + i];
}

// Neighbour k of in-block texel t, or -1 outside the block.
__device__ __forceinline__ int block_neighbour(int t, int k)
{
    const int x = (t & 3) + k % 3 - 1, y = (t >> 2) + k / 3 - 1;
    return x >= 0 && x < 4 && y >= 0 && y < 4 ? y * 4 + x : -1;
}

// Which neighbour of texel t texel u is, or -1.
__device__ __forceinline__ int neighbour_index(int t, int u)
{
    const int dx = (u & 3) - (t & 3), dy = (u >> 2) - (t >> 2);
    return dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 ? (dy + 1) * 3 + (dx + 1) : -1;
}

// Row idx of u, from the lane that holds it (every lane takes part; the value is meaningful on every lane).
template <int R>
__device__ __forceinline__ double row_of(const double (&uv)[R], int idx)
{
    double v = 0.0;
#pragma unroll
    for (int q = 0; q < R; q++)
    {
        const double x = __shfl_sync(0xffffffffu, uv[q], idx & 31);
        if ((idx >> 5) == q)
            v = x;
    }
    return v;
}

// The sixteen lanes' terms folded serially in texel order, the same on every lane.
__device__ __forceinline__ double fold16(double v)
{
    double s = 0.0;
    for (int t = 0; t < 16; t++)
        s += __shfl_sync(0xffffffffu, v, t);
    return s;
}

struct RefineArgs
{
    const float* lo0;
    const float* hi0;
    int cx, cy;
    double* stats;   // [plane][2]
};

// One warp per 4x4 block of the colour; the blocks of every plane of the chain in one launch (start[] counts blocks
// of the colour per plane).
template <int C0>
__global__ void __launch_bounds__(32 * REFINE_WARPS, 8) k_bc_refine(BcPlanes P, RefineArgs R)
{
    using Sh = RefineShape<C0>;
    constexpr int N = Sh::N, RR = Sh::R, TS = Sh::TS, CC = Sh::CC;
    extern __shared__ double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* S = smem + warp * Sh::PER_WARP;
    double* a1 = S + 16 * TS;
    double* dv = a1 + N;
    double* dlt = dv + N;
    double* w8 = dlt + 16;
    int* s_ep = (int*)(w8 + 8);                          // 8 ints
    unsigned char* s_sel = (unsigned char*)(s_ep + 8);   // 64 bytes

    const long long bi = (long long)blockIdx.x * REFINE_WARPS + warp;
    if (bi >= P.start[P.n])
        return;
    const int pl = bc_plane_of(P, bi);
    const BcPlane& B = P.p[pl];
    const long long local = bi - P.start[pl];
    const int by = (B.h0 + 3) / 4;
    const int cbx = (B.bx - R.cx + 1) / 2, cby = (by - R.cy + 1) / 2;
    if (local >= (long long)cbx * cby)
        return;
    const int gx = R.cx + 2 * (int)(local % cbx);
    const int gy = R.cy + 2 * (int)(local / cbx);
    const int w0 = B.w0, h0 = B.h0;

    // The block's quadratic (src/cpu/cpu_refine_bc.cpp:152-205), one lane per row (texel, channel): the row's owned
    // stencil blocks whose partner lies in the block go to S, the rest of the stencil meets the neighbours'
    // corrections in the row's share of A1, summed in the reference's order (per slot: the owned block, then the
    // neighbour's transposed one). The stencil is read from its block-major copy: the block's own coefficients are one
    // contiguous run (the lanes of one coefficient read consecutive texels), a neighbouring block's transposed ones
    // the same layout one block over.
    const size_t gi = (size_t)gy * B.bx + gx;
    const double* own = B.bsten + gi * (SLOTS * CC * 16);
#pragma unroll
    for (int q = 0; q < RR; q++)
    {
        const int r = lane + 32 * q;
        if (r >= N)
            continue;
        const int t = r / C0, i = r % C0;
        const int px = gx * 4 + (t & 3), py = gy * 4 + (t >> 2);
        const bool in = px < w0 && py < h0;
        const size_t ti = in ? (size_t)py * w0 + px : 0;
        double acc = in ? B.grad[ti * C0 + i] : 0.0;
#pragma unroll
        for (int slot = 0; slot < SLOTS; slot++)
        {
            int dx, dy;
            slot_offset(slot, dx, dy);
            const int fx = px + dx, fy = py + dy;
            const bool f_img = in && fx >= 0 && fx < w0 && fy >= 0 && fy < h0;
            const int lx = fx - gx * 4, ly = fy - gy * 4;
            const bool f_blk = lx >= 0 && lx < 4 && ly >= 0 && ly < 4;
            const double* row = own + (size_t)(slot * CC + i * C0) * 16 + t;   // coefficient j at row[16 j]
            double* s_row = S + t * TS + slot * CC + i * C0;
#pragma unroll
            for (int j = 0; j < C0; j++)
                s_row[j] = f_img && f_blk ? row[16 * j] : 0.0;
            if (f_img && !f_blk)
            {
                const double* xn = B.delta + ((size_t)fy * w0 + fx) * C0;
#pragma unroll
                for (int j = 0; j < C0; j++)
                    acc += row[16 * j] * xn[j];
            }
            if (slot == 0 || !in)
                continue;
            const int ax = px - dx, ay = py - dy;
            const int mx = ax - gx * 4, my = ay - gy * 4;
            if (ax < 0 || ax >= w0 || ay < 0 || ay >= h0 || (mx >= 0 && mx < 4 && my >= 0 && my < 4))
                continue;
            const size_t nt = (size_t)ay * w0 + ax;
            const size_t nb = (size_t)(ay >> 2) * B.bx + (size_t)(ax >> 2);
            const double* col = B.bsten + ((nb * SLOTS + slot) * CC + i) * 16 + (size_t)((ay & 3) * 4 + (ax & 3));
            const double* xn = B.delta + nt * C0;
#pragma unroll
            for (int j = 0; j < C0; j++)
                acc += col[(size_t)16 * C0 * j] * xn[j];   // coefficient (j, i) of the neighbour's block
        }
        a1[r] = acc;
        dv[r] = in ? (double)B.v0[ti * C0 + i] - (double)B.prev[ti * C0 + i] : 0.0;
    }
    if (lane < C0)
    {
        s_ep[2 * lane] = B.ep[(gi * C0 + lane) * 2];
        s_ep[2 * lane + 1] = B.ep[(gi * C0 + lane) * 2 + 1];
    }
    for (int i = lane; i < N; i += 32)
        s_sel[i] = B.sel[gi * C0 * 16 + i];
    if (lane < 8)
        w8[lane] = bc4_weight8(lane);
    __syncwarp();

    // u = A2 d, row by row in column order
    double uv[RR];
#pragma unroll
    for (int q = 0; q < RR; q++)
    {
        uv[q] = 0.0;
        const int r = lane + 32 * q;
        if (r >= N)
            continue;
        const int t = r / C0, i = r % C0;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 9; k++)
        {
            const int u = block_neighbour(t, k);
            if (u < 0)
                continue;
#pragma unroll
            for (int j = 0; j < C0; j++)
                s += a2_entry<C0>(S, t, i, u, j, k) * dv[u * C0 + j];
        }
        uv[q] = s;
    }

    double taken = 0.0;
    const int t16 = lane & 15;
    // ---- (i) the endpoints of each channel (src/cpu/cpu_refine_bc.cpp:222-312)
    for (int c = 0; c < C0; c++)
    {
        const double step = ((double)R.hi0[c] - (double)R.lo0[c]) / 255.0;
        const int idx = t16 * C0 + c;
        const double u_idx = row_of(uv, idx);
        double tbp = 0.0, tbq = 0.0, tpap = 0.0, tpaq = 0.0, tqaq = 0.0;
        if (lane < 16)
        {
            const double a = w8[s_sel[c * 16 + lane]];
            const double p = step * a;
            const double q = step * (1.0 - a);
            const double b = a1[idx] + u_idx;
            double ap = 0.0, aq = 0.0;
#pragma unroll
            for (int k = 0; k < 9; k++)
            {
                const int u = block_neighbour(lane, k);
                if (u < 0)
                    continue;
                const double e = a2_entry<C0>(S, lane, c, u, c, k);
                const double aj = w8[s_sel[c * 16 + u]];
                ap += e * step * aj;
                aq += e * step * (1.0 - aj);
            }
            tbp = b * p;
            tbq = b * q;
            tpap = p * ap;
            tpaq = p * aq;
            tqaq = q * aq;
        }
        const double bp = fold16(tbp), bq = fold16(tbq), pap = fold16(tpap), paq = fold16(tpaq),
                     qaq = fold16(tqaq);
        const int r0 = s_ep[2 * c], r1 = s_ep[2 * c + 1];
        const double det = pap * qaq - paq * paq;
        double d0 = 0.0, d1 = 0.0;
        if (det > 1e-12 * pap * qaq)
        {
            d0 = (paq * bq - qaq * bp) / det;
            d1 = (paq * bp - pap * bq) / det;
        }
        const double v0r = (double)r0 + d0, v1r = (double)r1 + d1;
        const int c0r = (int)floor(v0r + 0.5), c1r = (int)floor(v1r + 0.5);
        double best = 0.0;
        int best0 = r0, best1 = r1;
        for (int e0 = -1; e0 <= 1; e0++)
            for (int e1 = -1; e1 <= 1; e1++)
            {
                const int a0 = c0r + e0 < 0 ? 0 : (c0r + e0 > 255 ? 255 : c0r + e0);
                const int a1i = c1r + e1 < 0 ? 0 : (c1r + e1 > 255 ? 255 : c1r + e1);
                if (a0 <= a1i)
                    continue;
                const double f0 = (double)(a0 - r0), f1 = (double)(a1i - r1);
                const double de = 2.0 * (bp * f0 + bq * f1) + pap * f0 * f0 + 2.0 * paq * f0 * f1 + qaq * f1 * f1;
                if (de < best)
                {
                    best = de;
                    best0 = a0;
                    best1 = a1i;
                }
            }
        if (best0 == r0 && best1 == r1)
            continue;
        if (lane < 16)
        {
            const float now = bc0_value(R.lo0[c], R.hi0[c], bc4_entry(r0, r1, s_sel[c * 16 + lane]));
            const float next = bc0_value(R.lo0[c], R.hi0[c], bc4_entry(best0, best1, s_sel[c * 16 + lane]));
            dlt[lane] = (double)next - (double)now;
        }
        __syncwarp();
        double term = 0.0;
        if (lane < 16)
        {
            double quad = 0.0;
#pragma unroll
            for (int k = 0; k < 9; k++)
            {
                const int u = block_neighbour(lane, k);
                if (u >= 0)
                    quad += a2_entry<C0>(S, lane, c, u, c, k) * dlt[u];
            }
            term = dlt[lane] * (2.0 * (a1[idx] + u_idx) + quad);
        }
        const double exact = fold16(term);
        if (exact < 0.0)
        {
#pragma unroll
            for (int q = 0; q < RR; q++)
            {
                const int r = lane + 32 * q;
                if (r >= N)
                    continue;
                const int t = r / C0, i = r % C0;
                double add = 0.0;
#pragma unroll
                for (int k = 0; k < 9; k++)
                {
                    const int u = block_neighbour(t, k);
                    if (u >= 0)
                        add += a2_entry<C0>(S, t, i, u, c, k) * dlt[u];
                }
                uv[q] += add;
            }
            if (lane == 0)
            {
                s_ep[2 * c] = best0;
                s_ep[2 * c + 1] = best1;
            }
            taken += exact;
        }
        __syncwarp();
    }

    // ---- (ii) the selectors: two Gauss-Seidel passes of exact 8-way argmins (src/cpu/cpu_refine_bc.cpp:314-345).
    // Every group of eight lanes evaluates the eight candidates, one per lane, and takes the lowest change in three
    // butterfly rounds, ties to the lower candidate: the candidate the reference's in-order scan with a strict `<`
    // keeps, and no candidate when none lowers E.
    //
    // The four groups of eight lanes take four consecutive texels' steps at once, each against the current u. A step's
    // inputs are the sequential scan's as long as no earlier step of the four moved a selector; so the first step of
    // the four that lowers E is taken, the steps before it stand (none of them lowered E), and the scan resumes after
    // it. Steps that lower nothing, the common case once the selectors settle, cost a quarter of an iteration each.
    const int k8 = lane & 7, grp = lane >> 3;
    for (int pass = 0; pass < 2; pass++)
        for (int c = 0; c < C0; c++)
        {
            const int r0 = s_ep[2 * c], r1 = s_ep[2 * c + 1];
            const double cand = (double)bc0_value(R.lo0[c], R.hi0[c], bc4_entry(r0, r1, k8));
            int t0 = 0;
            while (t0 < 16)
            {
                const int t = t0 + grp < 16 ? t0 + grp : 15;   // past the last texel a group repeats it, unused
                const int i = t * C0 + c;
                const double b = a1[i] + row_of(uv, i);
                const double a = S[t * TS + c * C0 + c];
                const int cur = s_sel[c * 16 + t];
                const double now = __shfl_sync(0xffffffffu, cand, cur);
                const double d = cand - now;
                const double de = 2.0 * b * d + a * d * d;
                // the lowest change of the group's eight candidates (a candidate that does not lower E counts as 0),
                // then the first candidate that reaches it: the one the reference's in-order scan with a strict `<`
                // keeps
                const double mine = de < 0.0 ? de : 0.0;
                double v = mine;
#pragma unroll
                for (int o = 1; o < 8; o <<= 1)
                    v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
                const unsigned hits = __ballot_sync(0xffffffffu, mine == v);
                const int id = __ffs((hits >> (grp * 8)) & 0xffu) - 1;
                const unsigned lowers = __ballot_sync(0xffffffffu, k8 == 0 && t0 + grp < 16 && v < 0.0);
                if (lowers == 0u)
                {
                    t0 += 4;
                    continue;
                }
                // the first group whose step lowers E: its texel, change, candidate and new value on every lane
                const int g = (__ffs(lowers) - 1) >> 3;
                const int tf = t0 + g;
                const double vf = __shfl_sync(0xffffffffu, v, g * 8);
                const int idf = __shfl_sync(0xffffffffu, id, g * 8);
                const double mv = __shfl_sync(0xffffffffu, d, g * 8 + idf);
#pragma unroll
                for (int q = 0; q < RR; q++)
                {
                    const int r = lane + 32 * q;
                    if (r >= N)
                        continue;
                    const int rt = r / C0, ri = r % C0;
                    const int k = neighbour_index(rt, tf);
                    if (k >= 0)
                        uv[q] += a2_entry<C0>(S, rt, ri, tf, c, k) * mv;
                }
                if (lane == 0)
                    s_sel[c * 16 + tf] = (unsigned char)idf;
                taken += vf;
                __syncwarp();
                t0 = tf + 1;
            }
        }

    // ---- what the block leaves behind
    if (lane < C0)
    {
        B.ep[(gi * C0 + lane) * 2] = (uint8_t)s_ep[2 * lane];
        B.ep[(gi * C0 + lane) * 2 + 1] = (uint8_t)s_ep[2 * lane + 1];
    }
    for (int i = lane; i < N; i += 32)
        B.sel[gi * C0 * 16 + i] = s_sel[i];
    if (lane < 16)
    {
        const int px = gx * 4 + (lane & 3), py = gy * 4 + (lane >> 2);
        if (px < w0 && py < h0)
        {
            const size_t ti = (size_t)py * w0 + px;
            for (int c = 0; c < C0; c++)
            {
                const float byte = bc4_entry(s_ep[2 * c], s_ep[2 * c + 1], s_sel[c * 16 + lane]);
                const float value = bc0_value(R.lo0[c], R.hi0[c], byte);
                const size_t idx = ti * C0 + c;
                B.v0[idx] = value;
                B.k0[idx] = bc0_index(byte);
                B.delta[idx] = (double)value - (double)B.prev[idx];
            }
        }
    }
    if (lane == 0 && taken < 0.0)
    {
        atomicAdd(R.stats + 2 * pl, taken);
        atomicAdd(R.stats + 2 * pl + 1, 1.0);
    }
}

template <class F>
static BcPlanes bc_planes(nntc_b200_device* d, F items)
{
    BcPlanes P{};
    P.n = (int)d->planes.size();
    P.c0 = d->c0;
    for (int c = 0; c < MAX_CH; c++)
        P.bits[c] = d->m.bits0[c];
    long long at = 0;
    for (int i = 0; i < P.n; i++)
    {
        DevPlane& s = d->planes[(size_t)i];
        BcPlane& b = P.p[i];
        b.w0 = s.w0;
        b.h0 = s.h0;
        b.bx = (s.w0 + 3) / 4;
        b.ep = s.bc_ep;
        b.sel = s.bc_sel;
        b.k0src = s.k0;
        b.v0 = s.v0;
        b.k0 = s.k0;
        b.delta = s.work[1].x;
        b.prev = s.work[1].prev;
        b.bsten = s.bc_sten;
        b.grad = s.work[1].grad;
        P.start[i] = at;
        at += (long long)items(i);
    }
    P.start[P.n] = at;
    return P;
}

int assemble_for_refine(nntc_b200_device* d, const nntc_b200_model* m, int k, double* ms);

int bc_decode_all(nntc_b200_device* d)
{
    BcPlanes P = bc_planes(d, [&](int i) { return (size_t)d->planes[(size_t)i].w0 * d->planes[(size_t)i].h0; });
    k_bc_decode<<<grid_for((size_t)P.start[P.n], 256), 256, 0, d->stream>>>(P, d->lo0, d->hi0);
    NB_LAUNCHED();
    return NNTC_B200_OK;
}

int bc_prepare(nntc_b200_device* d, const nntc_b200_model* m, int k, int seed, const uint8_t* const* k0_host,
               double* ms)
{
    if (!d->l0_bc8)
    {
        set_error(NNTC_B200_ERR_STATE, "the BC refinement runs only under --l0 bc8");
        return NNTC_B200_ERR_STATE;
    }
    double t0 = 0.0, t1 = 0.0;
    NB_TRY(assemble_for_refine(d, m, k, &t0));
    if (seed)
    {
        // The seed pack reads the model's index mirror when the caller has one, else the device's own indices.
        for (int i = 0; i < (int)d->planes.size(); i++)
        {
            DevPlane& p = d->planes[(size_t)i];
            BcPlanes P = bc_planes(d, [&](int j) { return j == i ? p.blocks() * d->c0 : (size_t)0; });
            if (k0_host && k0_host[i])
            {
                NB_TRY(upload(d, d->scratch8, k0_host[i], (size_t)p.w0 * p.h0 * d->c0));
                P.p[i].k0src = d->scratch8;
            }
            k_bc_seed<<<grid_for((size_t)P.start[P.n], 128), 128, 0, d->stream>>>(P);
            NB_LAUNCHED();
        }
    }
    NB_TRY(block_begin(d));
    NB_TRY(bc_decode_all(d));
    NB_TRY(block_end(d, &t1));
    if (ms)
        *ms = t0 + t1;
    return NNTC_B200_OK;
}

int bc_refine_passes(nntc_b200_device* d, const nntc_b200_model* m, int passes, nntc_b200_bc_report* rep, double* ms)
{
    (void)m;
    double total = 0.0;
    const int c0 = d->c0;
    if (c0 < 1 || c0 > MAX_CH)
    {
        set_error(NNTC_B200_ERR_STATE, "the BC refinement needs 1..4 level-0 channels");
        return NNTC_B200_ERR_STATE;
    }
    const int per_warp = c0 == 1 ? RefineShape<1>::PER_WARP
                                 : (c0 == 2 ? RefineShape<2>::PER_WARP
                                            : (c0 == 3 ? RefineShape<3>::PER_WARP : RefineShape<4>::PER_WARP));
    const size_t shared = (size_t)per_warp * REFINE_WARPS * sizeof(double);
    void (*kernel)(BcPlanes, RefineArgs) =
        c0 == 1 ? k_bc_refine<1> : (c0 == 2 ? k_bc_refine<2> : (c0 == 3 ? k_bc_refine<3> : k_bc_refine<4>));
    NB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shared));
    for (int pass = 0; pass < passes; pass++)
    {
        NB_CUDA(cudaMemsetAsync(d->bc_stats, 0, (size_t)MAX_PLANES * 2 * sizeof(double), d->stream));
        NB_TRY(block_begin(d));
        for (int colour = 0; colour < 4; colour++)
        {
            const int cx = colour & 1, cy = colour >> 1;
            BcPlanes P = bc_planes(d, [&](int i) {
                const DevPlane& p = d->planes[(size_t)i];
                const int bx = (p.w0 + 3) / 4, by = (p.h0 + 3) / 4;
                return (size_t)((bx - cx + 1) / 2) * (size_t)((by - cy + 1) / 2);
            });
            if (P.start[P.n] == 0)
                continue;
            RefineArgs R{ d->lo0, d->hi0, cx, cy, d->bc_stats };
            const int grid = grid_for((size_t)P.start[P.n], REFINE_WARPS);
            NB_TRY(ktimer_begin(d, NNTC_B200_K_REFINE));
            kernel<<<grid, 32 * REFINE_WARPS, shared, d->stream>>>(P, R);
            NB_TRY(ktimer_end(d));
            NB_LAUNCHED();
        }
        double t = 0.0;
        NB_TRY(block_end(d, &t));
        total += t;
        std::vector<double> stats((size_t)MAX_PLANES * 2);
        NB_TRY(download(d, stats.data(), d->bc_stats, stats.size() * sizeof(double)));
        nntc_b200_bc_report r{};
        r.pass = pass + 1;
        r.ms = t;
        for (int i = 0; i < (int)d->planes.size(); i++)
        {
            r.delta_e += stats[(size_t)2 * i];
            r.improved += (long long)stats[(size_t)2 * i + 1];
            r.blocks += (long long)d->planes[(size_t)i].blocks();
        }
        if (rep)
            rep[pass] = r;
    }
    if (ms)
        *ms = total;
    return NNTC_B200_OK;
}

}   // namespace nb

using namespace nb;

extern "C"
{

int nntc_b200_bc_pack_prepare(nntc_b200_device* d, const nntc_b200_model* m, int k, int seed,
                              const uint8_t* const* k0_host, double* ms)
{
    return bc_prepare(d, m, k, seed, k0_host, ms);
}

int nntc_b200_bc_refine(nntc_b200_device* d, const nntc_b200_model* m, int passes, nntc_b200_bc_report* rep,
                        double* ms)
{
    if (!d->l0_bc8)
    {
        set_error(NNTC_B200_ERR_STATE, "the BC refinement runs only under --l0 bc8");
        return NNTC_B200_ERR_STATE;
    }
    return bc_refine_passes(d, m, passes, rep, ms);
}

int nntc_b200_bc_state_save(nntc_b200_device* d, const nntc_b200_model* m, uint8_t* const* ep, uint8_t* const* sel)
{
    (void)m;
    for (size_t i = 0; i < d->planes.size(); i++)
    {
        const DevPlane& p = d->planes[i];
        if (ep && ep[i])
            NB_TRY(download(d, ep[i], p.bc_ep, p.blocks() * d->c0 * 2));
        if (sel && sel[i])
            NB_TRY(download(d, sel[i], p.bc_sel, p.blocks() * d->c0 * 16));
    }
    return NNTC_B200_OK;
}

int nntc_b200_bc_state_restore(nntc_b200_device* d, const nntc_b200_model* m, const uint8_t* const* ep,
                               const uint8_t* const* sel)
{
    (void)m;
    for (size_t i = 0; i < d->planes.size(); i++)
    {
        const DevPlane& p = d->planes[i];
        if (ep && ep[i])
            NB_TRY(upload(d, p.bc_ep, ep[i], p.blocks() * d->c0 * 2));
        if (sel && sel[i])
            NB_TRY(upload(d, p.bc_sel, sel[i], p.blocks() * d->c0 * 16));
    }
    return NNTC_B200_OK;
}

// The .dds bytes of one plane from endpoints and selectors, and the pack error against k0's exact index values
// (src/export.cpp:262-279, 333-370; shared/bc_pack.h:79-85, 169-176). Host code: a few bytes per block.
int nntc_b200_bc_pack_blocks(const nntc_b200_model* m, int plane, const uint8_t* ep, const uint8_t* sel,
                             const uint8_t* k0, uint8_t* const* files, double* se, size_t* n)
{
    if (plane < 0 || plane >= m->nplanes)
    {
        set_error(NNTC_B200_ERR_ARG, "plane outside the model");
        return NNTC_B200_ERR_ARG;
    }
    const int w0 = m->w0[plane], h0 = m->h0[plane], c0 = m->c0;
    const int bx = (w0 + 3) / 4, by = (h0 + 3) / 4;
    const int nfiles = c0 <= 2 ? 1 : 2;
    for (int f = 0; f < nfiles; f++)
    {
        const int nc = f == 0 ? (c0 == 1 ? 1 : 2) : c0 - 2, bpb = nc == 1 ? 8 : 16;
        for (int c = 0; c < nc; c++)
        {
            const int channel = 2 * f + c;
            for (size_t b = 0; b < (size_t)bx * by; b++)
            {
                uint8_t* blk = files[f] + b * bpb + (size_t)c * 8;
                const size_t slot = b * c0 + channel;
                blk[0] = ep[slot * 2];
                blk[1] = ep[slot * 2 + 1];
                uint64_t bits = 0;
                for (int t = 0; t < 16; t++)
                    bits |= (uint64_t)(sel[slot * 16 + t] & 7) << (3 * t);
                for (int i = 0; i < 6; i++)
                    blk[2 + i] = (uint8_t)(bits >> (8 * i));
            }
            if (!k0)
                continue;
            for (int y = 0; y < h0; y++)
                for (int x = 0; x < w0; x++)
                {
                    const uint8_t* blk = files[f] + ((size_t)(y / 4) * bx + x / 4) * bpb + (size_t)c * 8;
                    float p[8];
                    bc4_palette(blk[0], blk[1], p);
                    uint64_t bits = 0;
                    for (int i = 0; i < 6; i++)
                        bits |= (uint64_t)blk[2 + i] << (8 * i);
                    const float decoded = p[(bits >> (3 * ((y % 4) * 4 + x % 4))) & 7];
                    const int b8 = m->l0_bc8 ? 8 : m->bits0[channel];
                    const int kk = k0[((size_t)y * w0 + x) * c0 + channel];
                    const double exact = b8 >= 8 ? (double)kk : (double)kk * 255.0 / (double)((1 << b8) - 1);
                    const double e = (double)decoded - exact;
                    *se += e * e;
                    (*n)++;
                }
        }
    }
    return NNTC_B200_OK;
}

}   // extern "C"
