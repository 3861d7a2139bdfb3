// assemble.cu: the stencil and gradient assembly of blocks (b) and (c'), restructured for B200 - and bit-identical
// to the reference's per-texel gather (src/solve_level1.cu:259-581).
//
// The reference gives each texel one thread that walks every site whose bilinear footprint can reach it and, for each
// site that does, recomputes the whole site: its G (or Q) matrix, its residual and G^T diag(cw) r - about a thousand
// operations - then adds the site's monomials into five slots of fifteen sums. Every site is recomputed by each of the
// (up to four) texels it touches, and the 75 double accumulators of a thread spill.
//
// Two observations make it cheap without changing a single rounding:
//
//   - the gradient term of a site, t_s = G^T diag(cw) r, does not depend on which texel gathers it. One thread per
//     SITE computes it once, with the reference's arithmetic (rows in order, each column's sum over the rows in order,
//     no contraction), into a per-site buffer of doubles; the gather then adds w_self * t_s exactly as the reference
//     adds w_self * acc.
//   - the stencil's monomial sums need only the site's sample of the OTHER latent (a bilinear blend of four texels,
//     which k_site_terms also stores per site) and the tap weights - a few dozen operations. They are gathered by one
//     thread per (texel, slot): a block holds one slot, so a warp shares one slot and its site range (the
//     intersection of the two texels' footprints). Each slot's sums
//     receive the same terms in the same site order as the reference's, so every sum, and the expansion against the
//     monomial matrices after it, is the same bits.
//
// Every plane of the chain is in each launch (nb::Planes); the per-site buffer holds every plane's sites.

#include <algorithm>
#include <cstring>
#include <vector>

#include "device.cuh"
#include "footprint.cuh"

namespace nb
{

constexpr int SITE_THREADS = 256;
constexpr int GATHER_THREADS = 128;
constexpr int GATHER_RING = 4;   // visits in flight per thread on the interior walk (cp.async into shared memory)

// One visit's operands, staged by cp.async: the site's sample of the other latent and (self slot) its gradient term.
struct __align__(16) VisitSlot
{
    float4 y;
    double t[MAX_CH];
};

__device__ __forceinline__ void cp_async16(void* dst, const void* src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}

__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;" ::: "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The ten products y_i y_k (i <= k < 4) of the monomial layout, row by row: (0,0) (0,1) (0,2) (0,3) (1,1) (1,2)
// (1,3) (2,2) (2,3) (3,3). Functions rather than tables, so an unrolled index folds to a register name.
__host__ __device__ constexpr int pair_i(int p)
{
    return p < 4 ? 0 : (p < 7 ? 1 : (p < 9 ? 2 : 3));
}
__host__ __device__ constexpr int pair_k(int p)
{
    return p < 4 ? p : (p < 7 ? p - 3 : (p < 9 ? p - 5 : 3));
}

// Whether slot L of the fixed monomial layout (the constant, four linear terms, ten products) is a monomial of a
// latent with ny channels: the used slots, in slot order, are the reference's monomials in its order.
__host__ __device__ constexpr bool mono_used(int L, int ny)
{
    return L == 0 || (L <= MAX_CH ? L - 1 < ny : pair_k(L - 5) < ny);
}

struct SiteArgs
{
    double* terms;                      // [site][c] over every plane
    float4* y;                          // [site]: the site's sample of the other latent
    const float* tgt;                   // [fractional site][NOUT]: the targets of the sites j > 0 (k_site_targets)
    long long site0[MAX_PLANES + 1];    // the first site of each plane in `terms`
    long long tsite0[MAX_PLANES + 1];   // the first fractional site of each plane in `tgt`
};

struct TargetOffsets
{
    long long site0[MAX_PLANES + 1];    // the first fractional site of each plane
};

// The float target of every fractional site (j > 0): the source blended at the site's four level-0 taps, in blend()'s
// order and arithmetic (src/solve_level1.cu:322-333). It depends on nothing but the source and K, neither of which an
// encode changes, so it is formed once per device model and K and then read by every k_site_terms launch.
template <int NOUT>
__global__ void __launch_bounds__(SITE_THREADS) k_site_targets(Planes P, float* tgt, const __grid_constant__ TargetOffsets O)
{
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long fi = base - P.start[pl] + threadIdx.x;
    const int kc = P.kc;
    if (fi >= (long long)V.w0 * V.h0 * kc)
        return;
    const long long pixel = fi / kc;
    const int j = 1 + (int)(fi % kc);
    const int px = (int)(pixel % V.w0), py = (int)(pixel / V.w0);
    float dx, dy;
    site_offset(kc, j, px, py, dx, dy);
    const Tap t0 = tap_at(px, py, dx, dy, V.w0, V.h0, V.w0, V.h0);
    float w0[4];
    tap_weights(t0, w0);
    float* out = tgt + (size_t)(O.site0[pl] + fi) * NOUT;
#pragma unroll
    for (int r = 0; r < NOUT; r++)
    {
        const float* s = V.src + r;
        out[r] = w0[0] * __ldg(s + ((size_t)t0.y0 * V.w0 + t0.x0) * NOUT) +
                 w0[1] * __ldg(s + ((size_t)t0.y0 * V.w0 + t0.x1) * NOUT) +
                 w0[2] * __ldg(s + ((size_t)t0.y1 * V.w0 + t0.x0) * NOUT) +
                 w0[3] * __ldg(s + ((size_t)t0.y1 * V.w0 + t0.x1) * NOUT);
    }
}

// One thread per site: t_s[a] = sum_r cw_r G[r][a] res_r (level 1, block b) or sum_r cw_r Q[r][a] res_r (level 0,
// block c'), in the reference's order of operations (src/solve_level1.cu:335-361, 518-544).
// The decoder as a launch parameter, each row at a fixed stride of 24 slots, [c_q (4)][s_i (4)][s_i c_q (4 x 4)]: with
// the row loop unrolled every weight is a constant-bank operand. Slots of channels the layout does not use are never
// read (the channel loops are guarded), so the arithmetic is the reference's operation for operation.
struct SiteDecoder
{
    float w[MAX_NOUT * 24];
    float b[MAX_NOUT];
    float cw[MAX_NOUT];
};

// MIXED (the adjoint form, whose stencil and sums are FP32): the same terms with fused multiply-adds and the gradient
// term summed in FP32 - half the instructions of the reference's unfused float arithmetic and no FP64 work per output.
template <bool LEVEL0, int NOUT, bool MIXED>
__global__ void __launch_bounds__(SITE_THREADS) k_site_terms(Planes P, const __grid_constant__ SiteArgs A, SiteDecoder W)
{
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long si = base - P.start[pl] + threadIdx.x;
    const int kc = P.kc, per = 1 + kc;
    if (si >= (long long)V.w0 * V.h0 * per)
        return;
    const int c0 = P.c0, c1 = P.c1;
    const long long pixel = si / per;
    const int j = (int)(si % per);
    const int px = (int)(pixel % V.w0), py = (int)(pixel / V.w0);
    float dx, dy;
    site_offset(kc, j, px, py, dx, dy);
    float sbar[MAX_CH], cbar[MAX_CH];
    const Tap tp = tap_at(px, py, dx, dy, V.w0, V.h0, V.w1, V.h1);
    blend_u<MAX_CH>(V.v1, V.w1, c1, tp, cbar);
    if (j == 0)
    {
#pragma unroll
        for (int i = 0; i < MAX_CH; i++)
            if (i < c0)
                sbar[i] = V.v0[pixel * c0 + i];
    }
    else
    {
        const Tap t0 = tap_at(px, py, dx, dy, V.w0, V.h0, V.w0, V.h0);
        blend_u<MAX_CH>(V.v0, V.w0, c0, t0, sbar);
    }
    // the targets: the pixel's own source at the centre site, else the fractional site's blend from k_site_targets
    const float* tgt = j > 0 ? A.tgt + (size_t)(A.tsite0[pl] + pixel * kc + (j - 1)) * NOUT : V.src + pixel * NOUT;
    double acc[MAX_CH];
    float accf[MAX_CH];
#pragma unroll
    for (int a = 0; a < MAX_CH; a++)
    {
        acc[a] = 0.0;
        accf[a] = 0.0f;
    }
    // a + b c, unfused (the reference's rounding) or fused (MIXED)
    auto madd = [](float a, float b, float c) { return MIXED ? __fmaf_rn(b, c, a) : a + b * c; };
#pragma unroll
    for (int r = 0; r < NOUT; r++)
    {
        const float target = __ldg(tgt + r);
        const float* row = W.w + r * 24;   // [c_q][s_i][s_i c_q]
        float out = W.b[r];
        float col[MAX_CH];
        if (!LEVEL0)
        {
#pragma unroll
            for (int i = 0; i < MAX_CH; i++)
                if (i < c0)
                    out = madd(out, row[4 + i], sbar[i]);
#pragma unroll
            for (int q = 0; q < MAX_CH; q++)
                if (q < c1)
                {
                    float gg = row[q];
#pragma unroll
                    for (int i = 0; i < MAX_CH; i++)
                        if (i < c0)
                            gg = madd(gg, sbar[i], row[8 + i * 4 + q]);
                    col[q] = gg;
                    out = madd(out, gg, cbar[q]);
                }
        }
        else
        {
#pragma unroll
            for (int q = 0; q < MAX_CH; q++)
                if (q < c1)
                    out = madd(out, row[q], cbar[q]);
#pragma unroll
            for (int i = 0; i < MAX_CH; i++)
                if (i < c0)
                {
                    float qq = row[4 + i];
#pragma unroll
                    for (int q = 0; q < MAX_CH; q++)
                        if (q < c1)
                            qq = madd(qq, cbar[q], row[8 + i * 4 + q]);
                    col[i] = qq;
                    out = madd(out, qq, sbar[i]);
                }
        }
        const float res = out - target;
        const int c = LEVEL0 ? c0 : c1;
#pragma unroll
        for (int a = 0; a < MAX_CH; a++)
            if (a < c)
            {
                if (MIXED)
                    accf[a] = __fmaf_rn(W.cw[r] * col[a], res, accf[a]);
                else
                    acc[a] += (double)W.cw[r] * (double)col[a] * (double)res;
            }
    }
    if (MIXED)
    {
#pragma unroll
        for (int a = 0; a < MAX_CH; a++)
            acc[a] = (double)accf[a];
    }
    const int c = LEVEL0 ? c0 : c1;
    double* out_t = A.terms + (size_t)(A.site0[pl] + si) * c;
#pragma unroll
    for (int a = 0; a < MAX_CH; a++)
        if (a < c)
            out_t[a] = acc[a];
    // the other latent's sample, which every (texel, slot) of the gather that meets this site needs again
    float y[MAX_CH];
    const int ny = LEVEL0 ? c1 : c0;
#pragma unroll
    for (int i = 0; i < MAX_CH; i++)
        y[i] = i < ny ? (LEVEL0 ? cbar[i] : sbar[i]) : 0.0f;
    A.y[A.site0[pl] + si] = make_float4(y[0], y[1], y[2], y[3]);
}

// ---- the gather's visit tables
//
// Away from the borders the sites that touch a texel and one of its neighbours, and their two weights, depend only on
// where the texel sits relative to the pixel grid: for level 0 (the unknown at the pixels' own resolution, site
// positions px + dx exact in float) on the texel's parity, which decides the subtexel rotation of its pixels; for
// level 1 at exactly a quarter of a power-of-two plane (site positions ((px + 0.5 + dx) w) / w0 - 0.5 exact in
// float) on nothing at all. So the visits are listed once, in the reference's site order, by running site_touches
// on a texel in the middle of a plane of that shape, and every interior texel walks its list instead of testing
// every site of its footprint; texels near a border, and planes of any other shape, take the full walk.

constexpr int GATHER_CLASSES = 4;
constexpr int GATHER_MARGIN = 3;   // texels this far from every border walk the table

struct GatherTable
{
    int off[GATHER_CLASSES][SLOTS + 1];
};

// entry: x = (dpx + 64) | (dpy + 64) << 8 | j << 16, y = w_self bits, z = w_other bits; (dpx, dpy) relative to the
// texel's first pixel (the texel itself at level 0, 4 tx / 4 ty at level 1)
template <bool LEVEL0>
static void build_gather_table(int kc, std::vector<int4>& tab, GatherTable& gt)
{
    tab.clear();
    const int w = 64, h = 64, w0 = LEVEL0 ? 64 : 256, h0 = LEVEL0 ? 64 : 256, scale = LEVEL0 ? 1 : 4;
    for (int cls = 0; cls < GATHER_CLASSES; cls++)
    {
        if (!LEVEL0 && cls > 0)
        {
            // level 1 has one class
            for (int slot = 0; slot <= SLOTS; slot++)
                gt.off[cls][slot] = gt.off[0][slot];
            continue;
        }
        const int tx = 32 + (LEVEL0 ? (cls & 1) : 0), ty = 32 + (LEVEL0 ? (cls >> 1) : 0);
        const int bx = tx * scale, by = ty * scale;
        for (int slot = 0; slot < SLOTS; slot++)
        {
            gt.off[cls][slot] = (int)tab.size();
            int ox, oy;
            slot_offset(slot, ox, oy);
            const int nbx = tx + ox, nby = ty + oy;
            int px_lo, px_hi, py_lo, py_hi, qx_lo, qx_hi, qy_lo, qy_hi;
            reach(tx, w0, w, px_lo, px_hi);
            reach(ty, h0, h, py_lo, py_hi);
            reach(nbx, w0, w, qx_lo, qx_hi);
            reach(nby, h0, h, qy_lo, qy_hi);
            px_lo = std::max(px_lo, qx_lo);
            px_hi = std::min(px_hi, qx_hi);
            py_lo = std::max(py_lo, qy_lo);
            py_hi = std::min(py_hi, qy_hi);
            for (int py = py_lo; py <= py_hi; py++)
                for (int px = px_lo; px <= px_hi; px++)
                    for (int j = 0; j <= kc; j++)
                    {
                        float ws, wo;
                        if (!site_touches<LEVEL0>(px, py, j, kc, tx, ty, nbx, nby, w0, h0, w, h, ws, wo))
                            continue;
                        int4 e;
                        e.x = (px - bx + 64) | (py - by + 64) << 8 | j << 16;
                        std::memcpy(&e.y, &ws, sizeof(float));
                        std::memcpy(&e.z, &wo, sizeof(float));
                        e.w = 0;
                        tab.push_back(e);
                    }
        }
        gt.off[cls][SLOTS] = (int)tab.size();
    }
}

struct GatherArgs
{
    const double* terms;
    const float4* y;      // [site]: the site's sample of the other latent, from k_site_terms
    // the monomial matrices (c x c, row-major) at their monomial's slot of the fixed layout, unused slots left out:
    // with the expansion unrolled every entry is a constant-bank operand, no loads
    double mono[MAX_MONO][MAX_CH * MAX_CH];
    float monof[MAX_MONO][MAX_CH * MAX_CH];   // the same in FP32, for the FP32 stencil of the adjoint form
    const int4* tab;      // the visit tables of this level and K
    GatherTable gt;
    unsigned tabled;      // bit i: plane i's interior texels may use the tables
    long long site0[MAX_PLANES + 1];
    long long bstart[MAX_PLANES + 1];   // each plane's first block
    int slots;            // slots gathered: SLOTS, or 1 for the diagonal blocks and the gradient alone
    int bc_copy;          // level 0, FP64, for the BC refinement: each block also into the block-major copy
};

// Where coefficient e of slot `slot` of texel (x, y) sits in the block-major copy: block (y / 4, x / 4) of a plane
// bx blocks wide, then slot, coefficient and the texel's place in its 4x4 block.
__device__ __forceinline__ size_t bc_sten_pos(int x, int y, int bx, int slot, int cc, int e)
{
    const size_t blk = (size_t)(y >> 2) * bx + (x >> 2);
    return ((blk * SLOTS + slot) * cc + e) * 16 + (size_t)((y & 3) * 4 + (x & 3));
}

// The texel at position `pos` of the stencil's colour-major order (the inverse of stencil_pos).
__device__ __forceinline__ void stencil_texel(long long pos, int w, int h, int& x, int& y)
{
    const long long w0c = (w + 1) >> 1, w1c = w >> 1, h0c = (h + 1) >> 1, h1c = h >> 1;
    const long long n0 = w0c * h0c, n1 = w1c * h0c, n2 = w0c * h1c;
    int cx = 0, cy = 0;
    long long r = pos, rw = w0c;
    if (r >= n0 + n1 + n2)
    {
        r -= n0 + n1 + n2;
        cx = 1;
        cy = 1;
        rw = w1c;
    }
    else if (r >= n0 + n1)
    {
        r -= n0 + n1;
        cy = 1;
    }
    else if (r >= n0)
    {
        r -= n0;
        cx = 1;
        rw = w1c;
    }
    x = 2 * (int)(r % rw) + cx;
    y = 2 * (int)(r / rw) + cy;
}

// One thread per (texel, slot): the slot's monomial sums over every site that touches both the texel and the slot's
// neighbour, in site order, expanded into the slot's block; the self-slot thread also gathers the gradient. Threads
// take the texels in the stencil's colour-major order, so a warp's texels share a parity class (one visit table) and
// its stores are contiguous.
template <typename TS>
__device__ __forceinline__ TS mono_entry(const GatherArgs& A, int L, int e);
template <>
__device__ __forceinline__ double mono_entry<double>(const GatherArgs& A, int L, int e)
{
    return A.mono[L][e];
}
template <>
__device__ __forceinline__ float mono_entry<float>(const GatherArgs& A, int L, int e)
{
    return A.monof[L][e];
}

// TS: the stencil's stored type and the sums' type - double for the plain form (the reference's bits), float for the
// adjoint form (the sweeps then read half the bytes; the gradient stays in double either way).
template <bool LEVEL0, typename TS>
__device__ __forceinline__ void gather_body(const Planes& P, const GatherArgs& A)
{
    // Block order: (region, colour, slot) with the slot fastest. The five slots of one run of texels, and the four
    // colours of one region of the plane, are consecutive blocks, so they run side by side and share the region's sites
    // in L2: every slot of every texel that a site touches reads it, and the texels of one colour alone already touch
    // every site of their region.
    int pl = 0;
    while (pl + 1 < P.n && A.bstart[pl + 1] <= (long long)blockIdx.x)
        pl++;
    const long long lb = (long long)blockIdx.x - A.bstart[pl];
    const int slot = (int)(lb % A.slots);
    const int colour = (int)((lb / A.slots) % 4);
    const long long region = lb / A.slots / 4;
    const PlaneView& V = P.p[pl];
    const int tw_ = V.w, th_ = V.h;
    const long long w0c = (tw_ + 1) >> 1, w1c = tw_ >> 1, h0c = (th_ + 1) >> 1, h1c = th_ >> 1;
    const long long n0 = w0c * h0c, n1 = w1c * h0c, n2 = w0c * h1c, n3 = w1c * h1c;
    const long long ncol = colour == 0 ? n0 : (colour == 1 ? n1 : (colour == 2 ? n2 : n3));
    const long long within = region * GATHER_THREADS + threadIdx.x;
    if (within >= ncol)
        return;
    // the texel's place in the stencil's colour-major order
    const long long sp = within + (colour == 0 ? 0 : (colour == 1 ? n0 : (colour == 2 ? n0 + n1 : n0 + n1 + n2)));
    const int c0 = P.c0, c1 = P.c1, kc = P.kc, per = 1 + kc;
    const int c = LEVEL0 ? c0 : c1;
    int tx, ty;
    stencil_texel(sp, tw_, th_, tx, ty);
    const size_t ti = (size_t)ty * tw_ + tx;
    int ox, oy;
    slot_offset(slot, ox, oy);
    const int nbx = tx + ox, nby = ty + oy;
    const size_t T = (size_t)tw_ * th_;
    const int cc = c * c;
    const bool bc_copy = LEVEL0 && sizeof(TS) == sizeof(double) && A.bc_copy;
    if (nbx < 0 || nbx >= tw_ || nby >= th_)
    {
        // no neighbour in this direction: the reference's block is zero (no site touches both)
        for (int e = 0; e < cc; e++)
        {
            reinterpret_cast<TS*>(V.stencil)[sten_index<TS>(slot, e, cc, T, sp)] = (TS)0;
            if (bc_copy)
                V.bc_sten[bc_sten_pos(tx, ty, (tw_ + 3) >> 2, slot, cc, e)] = 0.0;
        }
        return;
    }

    TS sums[MAX_MONO];
#pragma unroll
    for (int i = 0; i < MAX_MONO; i++)
        sums[i] = (TS)0;
    double g[MAX_CH];
#pragma unroll
    for (int a = 0; a < MAX_CH; a++)
        g[a] = 0.0;
    const double* terms = A.terms + (size_t)A.site0[pl] * c;
    const float4* ys = A.y + A.site0[pl];
    const int ny_ = LEVEL0 ? c1 : c0;

    // one visit: the site's sample of the other latent (k_site_terms sampled it with the same taps and blend: the
    // same floats) and its monomials in a fixed layout: the constant, the four linear terms, then the ten products
    // (i <= k) row by row; a narrower latent uses the entries whose indices are all below its channel count, which is
    // the reference's order
    // the sums' part of a visit (every slot)
    auto visit_sums = [&](float4 y4, float w_self, float w_other) {
        const float y[MAX_CH] = { y4.x, y4.y, y4.z, y4.w };
        const TS scale = (TS)w_self * (TS)w_other;
        sums[0] += scale * (TS)1;
#pragma unroll
        for (int i = 0; i < MAX_CH; i++)
            if (i < ny_)
                sums[1 + i] += scale * (TS)y[i];
#pragma unroll
        for (int p = 0; p < 10; p++)
        {
            const int i = pair_i(p), k2 = pair_k(p);
            if (k2 < ny_)
                sums[5 + p] += scale * ((TS)y[i] * (TS)y[k2]);
        }
    };
    auto visit_y = [&](size_t site, float4 y4, float w_self, float w_other) {
        if (slot == 0)
        {
            const double* ts = terms + site * c;
#pragma unroll
            for (int a = 0; a < MAX_CH; a++)
                if (a < c)
                    g[a] += (double)w_self * ts[a];
        }
        visit_sums(y4, w_self, w_other);
    };
    auto visit = [&](int px, int py, int j, float w_self, float w_other) {
        const size_t site = (size_t)(py * V.w0 + px) * per + j;
        visit_y(site, __ldg(ys + site), w_self, w_other);
    };

    const bool interior = ((A.tabled >> pl) & 1u) && tx >= GATHER_MARGIN && tx < tw_ - GATHER_MARGIN &&
                          ty >= GATHER_MARGIN && ty < th_ - GATHER_MARGIN;
    if (interior)
    {
        const int cls = LEVEL0 ? (tx & 1) + 2 * (ty & 1) : 0;
        const int bx = LEVEL0 ? tx : 4 * tx, by = LEVEL0 ? ty : 4 * ty;
        const int e0 = A.gt.off[cls][slot], e1 = A.gt.off[cls][slot + 1];
        auto site_of = [&](const int4& en) {
            return (size_t)((by + ((en.x >> 8) & 0xff) - 64) * V.w0 + (bx + (en.x & 0xff) - 64)) * per + (en.x >> 16);
        };
        if constexpr (LEVEL0)
        {
            // a level-0 texel meets a dozen or so sites per slot: one visit ahead (the next entry and its sample are
            // loaded while this one is added), at the occupancy of a kernel without the ring's shared memory
            if (e0 < e1)
            {
                int4 en = __ldg(A.tab + e0);
                size_t site = site_of(en);
                float4 y4 = __ldg(ys + site);
                for (int e = e0; e < e1; e++)
                {
                    int4 nen = en;
                    size_t nsite = site;
                    float4 ny4 = y4;
                    if (e + 1 < e1)
                    {
                        nen = __ldg(A.tab + e + 1);
                        nsite = site_of(nen);
                        ny4 = __ldg(ys + nsite);
                    }
                    visit_y(site, y4, __int_as_float(en.y), __int_as_float(en.z));
                    en = nen;
                    site = nsite;
                    y4 = ny4;
                }
            }
        }
        else
        {
            // Level 1's walk (a few hundred visits per texel) keeps GATHER_RING visits in flight: visit e's sample
            // (and gradient term) is copied into this thread's ring slot e % GATHER_RING by cp.async GATHER_RING
            // visits before it is added, so that many L2 reads per thread overlap without holding registers; the
            // sums still take the visits in table order. A slot is refilled only after its visit's values are used.
            __shared__ VisitSlot ring[GATHER_RING][GATHER_THREADS];
            float wsq[GATHER_RING], woq[GATHER_RING];
            const bool grad = slot == 0;
            auto issue = [&](int i, int e) {
                const int4 en = __ldg(A.tab + e);
                wsq[i] = __int_as_float(en.y);
                woq[i] = __int_as_float(en.z);
                const size_t site = site_of(en);
                VisitSlot& rs = ring[i][threadIdx.x];
                cp_async16(&rs.y, ys + site);
                if (grad)
                {
                    if (c == MAX_CH)
                    {
                        cp_async16(&rs.t[0], terms + site * MAX_CH);
                        cp_async16(&rs.t[2], terms + site * MAX_CH + 2);
                    }
                    else
                    {
                        for (int a = 0; a < c; a++)
                            rs.t[a] = __ldg(terms + site * c + a);
                    }
                }
            };
    #pragma unroll
            for (int i = 0; i < GATHER_RING; i++)
            {
                if (e0 + i < e1)
                    issue(i, e0 + i);
                cp_async_commit();
            }
            for (int e = e0; e < e1; e += GATHER_RING)
            {
    #pragma unroll
                for (int i = 0; i < GATHER_RING; i++)
                {
                    if (e + i < e1)
                    {
                        // every group but the newest GATHER_RING - 1 has landed: visit e + i's among them
                        cp_async_wait<GATHER_RING - 1>();
                        const VisitSlot& rs = ring[i][threadIdx.x];
                        if (grad)
                        {
    #pragma unroll
                            for (int a = 0; a < MAX_CH; a++)
                                if (a < c)
                                    g[a] += (double)wsq[i] * rs.t[a];
                        }
                        visit_sums(rs.y, wsq[i], woq[i]);
                        if (e + i + GATHER_RING < e1)
                            issue(i, e + i + GATHER_RING);
                    }
                    cp_async_commit();
                }
            }
        }
    }
    else
    {
        // the pixel range of sites that can touch both texels: the intersection of their footprints
        int px_lo, px_hi, py_lo, py_hi, qx_lo, qx_hi, qy_lo, qy_hi;
        const int n1x = LEVEL0 ? V.w0 : V.w1, n1y = LEVEL0 ? V.h0 : V.h1;
        reach(tx, V.w0, n1x, px_lo, px_hi);
        reach(ty, V.h0, n1y, py_lo, py_hi);
        reach(nbx, V.w0, n1x, qx_lo, qx_hi);
        reach(nby, V.h0, n1y, qy_lo, qy_hi);
        px_lo = max(px_lo, qx_lo);
        px_hi = min(px_hi, qx_hi);
        py_lo = max(py_lo, qy_lo);
        py_hi = min(py_hi, qy_hi);
        for (int py = py_lo; py <= py_hi; py++)
            for (int px = px_lo; px <= px_hi; px++)
                for (int j = 0; j <= kc; j++)
                {
                    float ws, wo;
                    if (site_touches<LEVEL0>(px, py, j, kc, tx, ty, nbx, nby, V.w0, V.h0, LEVEL0 ? V.w0 : V.w1,
                                             LEVEL0 ? V.h0 : V.h1, ws, wo))
                        visit(px, py, j, ws, wo);
                }
    }

    // the slot's block, expanded once against the monomial matrices in the reference's order (src/solve_level1.cu:382-399);
    // level 1 expands it in two halves of eight entries (each entry's own sum still in monomial order) so that fewer
    // doubles are live at once and six blocks (FP64) or eight (FP32) fit an SM
    // (where the gradient's store goes changes only which registers are live when: each level's place is the one that
    // spills least at its occupancy)
    auto store_grad = [&]() {
        if (slot == 0)
        {
#pragma unroll
            for (int a = 0; a < MAX_CH; a++)
                if (a < c)
                    V.grad[ti * c + a] = g[a];
        }
    };
    if (!LEVEL0)
        store_grad();
    constexpr int PART = LEVEL0 ? MAX_CH * MAX_CH : 8;
#pragma unroll
    for (int part = 0; part < MAX_CH * MAX_CH / PART; part++)
    {
        TS blk[PART];
#pragma unroll
        for (int e = 0; e < PART; e++)
            blk[e] = (TS)0;
#pragma unroll
        for (int L = 0; L < MAX_MONO; L++)
        {
            if (!mono_used(L, ny_))
                continue;
            const TS s = sums[L];
            if (s == (TS)0)
                continue;
#pragma unroll
            for (int e = 0; e < PART; e++)
                if (part * PART + e < cc)
                    blk[e] += s * mono_entry<TS>(A, L, part * PART + e);
        }
        if constexpr (sizeof(TS) == sizeof(float))
        {
            // the FP32 stencil keeps a texel's block contiguous: whole 16-byte stores when the block is 16 floats
            if (cc == MAX_CH * MAX_CH)
            {
                float4* out = reinterpret_cast<float4*>(reinterpret_cast<float*>(V.stencil) +
                                                        sten_index<float>(slot, part * PART, cc, T, sp));
#pragma unroll
                for (int v = 0; v < PART / 4; v++)
                    out[v] = make_float4(blk[4 * v], blk[4 * v + 1], blk[4 * v + 2], blk[4 * v + 3]);
                continue;
            }
        }
#pragma unroll
        for (int e = 0; e < PART; e++)
            if (part * PART + e < cc)
            {
                reinterpret_cast<TS*>(V.stencil)[sten_index<TS>(slot, part * PART + e, cc, T, sp)] = blk[e];
                if (bc_copy)
                    V.bc_sten[bc_sten_pos(tx, ty, (tw_ + 3) >> 2, slot, cc, part * PART + e)] = (double)blk[e];
            }
    }
    if (LEVEL0)
        store_grad();
}

// The two levels' kernels: level 1's FP64 gather capped at six blocks per SM (its expansion is split for that), its
// FP32 gather at eight (64 registers; the visit rings' shared memory allows nine); level 0's FP64 gather left at the register count it takes (a cap made it spill and run
// slower), its FP32 gather at eight blocks per SM (64 registers, no spills: 18.4 -> 17.7 ms per assembly).
template <typename TS>
__global__ void __launch_bounds__(GATHER_THREADS, (sizeof(TS) == sizeof(float) ? 8 : 1)) k_gather_level0(Planes P, const __grid_constant__ GatherArgs A)
{
    gather_body<true, TS>(P, A);
}

template <typename TS>
__global__ void __launch_bounds__(GATHER_THREADS, (sizeof(TS) == sizeof(float) ? 8 : 6)) k_gather_level1(Planes P, const __grid_constant__ GatherArgs A)
{
    gather_body<false, TS>(P, A);
}

// Launch both passes for every plane: the per-site terms, then the per-(texel, slot) gather.
// The fractional sites' float targets at K in d->site_tgt ([fractional site][nout], planes in order), formed when the
// device does not hold them for this K yet: read by the assembly's site pass and the mixed-precision objective.
int ensure_site_targets(nntc_b200_device* d, int k, int level0)
{
    if (d->site_tgt_kc == k || k == 0)
        return NNTC_B200_OK;
    TargetOffsets O{};
    long long ft = 0;
    for (int i = 0; i < (int)d->planes.size(); i++)
    {
        O.site0[i] = ft;
        ft += (long long)d->planes[(size_t)i].w0 * d->planes[(size_t)i].h0 * k;
    }
    O.site0[d->planes.size()] = ft;
    Planes T = planes_for(d, level0, [&](int i) {
        const DevPlane& p = d->planes[(size_t)i];
        return (size_t)p.w0 * p.h0 * (size_t)k;
    });
    T.kc = k;
    const int tblocks = (int)(T.start[T.n] / SITE_THREADS);
#define NB_TARGETS(NO)                                                                                                \
    case NO:                                                                                                          \
        k_site_targets<NO><<<tblocks, SITE_THREADS, 0, d->stream>>>(T, d->site_tgt, O);                               \
        break;
    switch (d->nout)
    {
        NB_TARGETS(3)
        NB_TARGETS(6)
        NB_TARGETS(9)
        NB_TARGETS(12)
        NB_TARGETS(15)
        NB_TARGETS(18)
    default:
        set_error(NNTC_B200_ERR_STATE, "a material holds 1..6 RGB textures");
        return NNTC_B200_ERR_STATE;
    }
#undef NB_TARGETS
    NB_LAUNCHED();
    d->site_tgt_kc = k;
    return NNTC_B200_OK;
}

int assemble_split(nntc_b200_device* d, int k, int level0, const Planes& P_texels, int nmono, const double* mono,
                   int slots, bool f32)
{
    Planes S = planes_for(d, level0, [&](int i) {
        const DevPlane& p = d->planes[(size_t)i];
        return (size_t)p.w0 * p.h0 * (size_t)(1 + k);
    });
    S.kc = k;
    SiteArgs A{ d->site_terms, (float4*)d->site_y, {} };
    GatherArgs G{};
    G.slots = slots;
    G.terms = d->site_terms;
    G.y = (const float4*)d->site_y;
    {
        const int ny = level0 ? d->c1 : d->c0, c = level0 ? d->c0 : d->c1;
        int q = 0;
        for (int L = 0; L < MAX_MONO; L++)
            if (mono_used(L, ny))
            {
                std::memcpy(G.mono[L], mono + (size_t)q * c * c, (size_t)c * c * sizeof(double));
                for (int e = 0; e < c * c; e++)
                    G.monof[L][e] = (float)G.mono[L][e];
                q++;
            }
        if (q != nmono)
        {
            set_error(NNTC_B200_ERR_STATE, "monomial layout and count disagree");
            return NNTC_B200_ERR_STATE;
        }
    }
    if (d->gtab_kc[level0] != k)
    {
        std::vector<int4> tab;
        GatherTable gt{};
        if (level0)
            build_gather_table<true>(k, tab, gt);
        else
            build_gather_table<false>(k, tab, gt);
        if (tab.size() > (size_t)GATHER_TABLE_MAX)
        {
            set_error(NNTC_B200_ERR_STATE, "the gather's visit table outgrew its buffer");
            return NNTC_B200_ERR_STATE;
        }
        NB_TRY(upload(d, d->gtab[level0], tab.data(), tab.size() * sizeof(int4)));
        static_assert(sizeof(d->gtab_off[0]) == sizeof(GatherTable), "visit table offsets");
        std::memcpy(d->gtab_off[level0], &gt, sizeof(gt));
        d->gtab_kc[level0] = k;
    }
    G.bc_copy = level0 && !f32 && d->bc_copy ? 1 : 0;
    d->bc_copied = G.bc_copy && slots == SLOTS;
    G.tab = (const int4*)d->gtab[level0];
    std::memcpy(&G.gt, d->gtab_off[level0], sizeof(G.gt));
    auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
    for (int i = 0; i < (int)d->planes.size(); i++)
    {
        const DevPlane& p = d->planes[(size_t)i];
        const bool ok = level0 || (p.w0 == 4 * p.w1 && p.h0 == 4 * p.h1 && pow2(p.w1) && pow2(p.h1));
        if (ok)
            G.tabled |= 1u << i;
    }
    long long at = 0;
    for (int i = 0; i < S.n; i++)
    {
        A.site0[i] = G.site0[i] = at;
        at += (long long)d->planes[(size_t)i].w0 * d->planes[(size_t)i].h0 * (1 + k);
    }
    A.site0[S.n] = G.site0[S.n] = at;
    // the fractional sites' targets, formed on the first assembly at this K
    A.tgt = d->site_tgt;
    {
        long long ft = 0;
        for (int i = 0; i < S.n; i++)
        {
            A.tsite0[i] = ft;
            ft += (long long)d->planes[(size_t)i].w0 * d->planes[(size_t)i].h0 * k;
        }
        A.tsite0[S.n] = ft;
    }
    NB_TRY(ensure_site_targets(d, k, level0));
    const int sblocks = (int)(S.start[S.n] / SITE_THREADS);
    SiteDecoder W{};
    const int nin = d->nin, c0 = d->c0, c1 = d->c1;
    for (int r = 0; r < d->nout; r++)
    {
        for (int q = 0; q < c1; q++)
            W.w[r * 24 + q] = d->host_weights[(size_t)r * nin + q];
        for (int i = 0; i < c0; i++)
            W.w[r * 24 + 4 + i] = d->host_weights[(size_t)r * nin + c1 + i];
        for (int i = 0; i < c0; i++)
            for (int q = 0; q < c1; q++)
                W.w[r * 24 + 8 + i * 4 + q] = d->host_weights[(size_t)r * nin + c1 + c0 + i * c1 + q];
        W.b[r] = d->host_bias[r];
        W.cw[r] = d->m.cw[r];
    }
#define NB_SITES(NO)                                                                                                  \
    case NO:                                                                                                          \
        if (level0)                                                                                                   \
        {                                                                                                             \
            if (f32)                                                                                                  \
                k_site_terms<true, NO, true><<<sblocks, SITE_THREADS, 0, d->stream>>>(S, A, W);                       \
            else                                                                                                      \
                k_site_terms<true, NO, false><<<sblocks, SITE_THREADS, 0, d->stream>>>(S, A, W);                      \
        }                                                                                                             \
        else if (f32)                                                                                                 \
            k_site_terms<false, NO, true><<<sblocks, SITE_THREADS, 0, d->stream>>>(S, A, W);                          \
        else                                                                                                          \
            k_site_terms<false, NO, false><<<sblocks, SITE_THREADS, 0, d->stream>>>(S, A, W);                         \
        break;
    switch (d->nout)
    {
        NB_SITES(3)
        NB_SITES(6)
        NB_SITES(9)
        NB_SITES(12)
        NB_SITES(15)
        NB_SITES(18)
    default:
        set_error(NNTC_B200_ERR_STATE, "a material holds 1..6 RGB textures");
        return NNTC_B200_ERR_STATE;
    }
#undef NB_SITES
    NB_LAUNCHED();
    long long blocks = 0;
    for (int i = 0; i < P_texels.n; i++)
    {
        G.bstart[i] = blocks;
        const PlaneView& v = P_texels.p[i];
        const long long largest = (long long)((v.w + 1) / 2) * ((v.h + 1) / 2);   // colour 0
        blocks += (largest + GATHER_THREADS - 1) / GATHER_THREADS * 4 * slots;
    }
    G.bstart[P_texels.n] = blocks;
    const unsigned grid = (unsigned)blocks;
    if (level0 && f32)
        k_gather_level0<float><<<grid, GATHER_THREADS, 0, d->stream>>>(P_texels, G);
    else if (level0)
        k_gather_level0<double><<<grid, GATHER_THREADS, 0, d->stream>>>(P_texels, G);
    else if (f32)
        k_gather_level1<float><<<grid, GATHER_THREADS, 0, d->stream>>>(P_texels, G);
    else
        k_gather_level1<double><<<grid, GATHER_THREADS, 0, d->stream>>>(P_texels, G);
    NB_LAUNCHED();
    return NNTC_B200_OK;
}

}   // namespace nb
