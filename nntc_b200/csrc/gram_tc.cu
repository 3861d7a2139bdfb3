// gram_tc.cu: block (a)'s normal equations on the fifth-generation tensor cores (tcgen05), BF16 operands split hi + lo,
// FP32 accumulators in tensor memory, FP64 across batches: the mixed-precision form of the accumulation that
// decoder.cu's k_ls_accumulate_mma does in FP64 (the sums of src/solve_decoder.cu:87-161).
//
// Every entry the decoder's system needs is an entry of the Gram Z^T Z of the site rows Z = [phi | 1 | t] (at most 43
// columns, padded to 48). A float x is split x = hi + lo with hi = bf16(x) and lo = bf16(x - hi) (x - hi is exact in
// float), which holds x to about 2^-17 of itself. One CTA stages 128 sites' rows; the rows [Z_hi ; Z_lo] become one
// K-major operand tile of 128 rows (48 hi, 48 lo, 32 zero) by 16 sites per MMA step, and one MMA of M = 128, N = 96,
// K = 16 with that tile as both A and B produces the four products of the split at once:
//
//   D = [Z_hi ; Z_lo ; 0] [Z_hi ; Z_lo]^T  =  [[hi hi, hi lo], [lo hi, lo lo], 0]     (128 x 96, FP32, in TMEM)
//
// so Z^T Z = hi hi + hi lo + lo hi + lo lo: the compensated three-product form plus the lo lo term, which costs
// nothing more here. After every batch of 256 sites the accumulator is read back (row r of D is TMEM lane r) and
// added into FP64 registers, the hi and lo halves of each column in a fixed order; a CTA writes one partial per
// entry, which k_ls_reduce folds in block order as it does for the FP64 form. Deterministic: the tensor core's sums of
// a batch are a fixed function of the tile, the rest is fixed-order FP64.
//
// The tensor-core plumbing, all by inline PTX: tcgen05.alloc / dealloc of 128 TMEM columns per CTA (three CTAs per SM
// by registers and shared memory, 384 of the 512 columns, so an allocation never waits on another CTA), shared-memory matrix descriptors of the
// no-swizzle K-major canonical layout (8-row x 16-byte core matrices, LBO = the K-neighbour's offset, SBO = the next
// eight rows'), tcgen05.mma.cta_group::1.kind::f16 issued by one thread, tcgen05.commit to an mbarrier, tcgen05.ld of
// 32 lanes x 32 columns per warp. No TMA, no multicast, no cluster: the operands are built in shared memory by the
// threads from the planes (the rows are computed, not copied). Every wait on the mbarrier is bounded; a wait that
// gives up raises the device status word, waits (bounded) once more, frees the tensor memory and leaves.

#include <cstdint>

#include <cuda_bf16.h>

#include "device.cuh"

namespace nb
{

constexpr int TG_THREADS = 128;           // four warps: one TMEM lane quadrant each
constexpr int TG_SITES = 128;             // sites per stage (one per thread)
constexpr int TG_KSTEPS = TG_SITES / 16;  // MMAs per stage
constexpr int TG_STAGES_PER_BATCH = 2;    // FP32 accumulation spans 256 sites
constexpr int TG_ROW = 57;                // floats per staged site row (odd: conflict-free column reads)
constexpr int TG_TILE_BYTES = 128 * 16 * 2;   // one K-step operand tile: 128 rows x 16 bf16
constexpr int TG_TMEM_COLS = 128;         // allocation (power of two >= 96)
constexpr int TG_BUFFERS = 1;             // operand buffers: one stage's MMAs run while the next stage's site rows
                                          // are formed; a second buffer (the tile build overlapping too) measured no
                                          // faster and costs the third CTA per SM
constexpr uint32_t TG_WAIT_LIMIT = 1u << 26;

struct TcArgs
{
    double* partial;        // [plane][entry][LS_GRID]
    int entries;
    unsigned int* status;   // raised on a wait that gave up
};

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// The shared-memory matrix descriptor (tcgen05): start address, leading and stride byte offsets (all >> 4), the
// descriptor version 1 at bit 46, base offset 0, no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = (uint64_t)((addr & 0x3FFFFu) >> 4);
    d |= (uint64_t)((lbo & 0x3FFFFu) >> 4) << 16;
    d |= (uint64_t)((sbo & 0x3FFFFu) >> 4) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// The instruction descriptor of kind::f16: FP32 accumulator (bit 4), A and B BF16 (bits 7 and 10), both K-major,
// N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    const uint32_t a = smem_addr(bar);
    for (uint32_t it = 0; it < TG_WAIT_LIMIT; it++)
    {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (done)
            return true;
    }
    return false;
}

// Staged site row of Z (phi | 1 | t | zeros) for site `si` of plane V, with the arithmetic of the FP64 form.
__device__ __forceinline__ void site_row(const Planes& P, const PlaneView& V, size_t si, size_t sites, float* row)
{
    const int c0 = P.c0, c1 = P.c1, nout = P.nout, kc = P.kc, per_pixel = 1 + kc;
    int q = 0;
    if (si < sites)
    {
        const size_t pixel = si / (size_t)per_pixel;
        const int j = (int)(si % (size_t)per_pixel);
        const int px = (int)(pixel % (size_t)V.w0), py = (int)(pixel / (size_t)V.w0);
        float dx, dy;
        site_offset(kc, j, px, py, dx, dy);
        float s[MAX_CH], c[MAX_CH], w4[4];
        blend_u<MAX_CH>(V.v1, V.w1, c1, tap_at(px, py, dx, dy, V.w0, V.h0, V.w1, V.h1), c);
        Tap t0{};
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
        for (int b = 0; b < MAX_CH; b++)
            if (b < c1)
                row[q++] = c[b];
#pragma unroll
        for (int i = 0; i < MAX_CH; i++)
            if (i < c0)
                row[q++] = s[i];
#pragma unroll
        for (int i = 0; i < MAX_CH; i++)
#pragma unroll
            for (int b = 0; b < MAX_CH; b++)
                if (i < c0 && b < c1)
                    row[q++] = s[i] * c[b];
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
}

// Byte offset of (row r, site k) of K-step tile `step` in the canonical no-swizzle K-major layout: core matrix
// (r / 8, k / 8) of 128 bytes, K-neighbours 128 bytes apart (LBO), row groups 256 bytes apart (SBO).
__host__ __device__ constexpr uint32_t tile_offset(int step, int r, int k)
{
    return (uint32_t)step * TG_TILE_BYTES + (uint32_t)(((r >> 3) * 2 + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint32_t pack_bf16x2(__nv_bfloat16 a, __nv_bfloat16 b)
{
    return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

// 32 columns of this warp's TMEM lane quadrant into registers.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* v)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                 "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                   "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                   "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                   "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                   "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                 : "r"(taddr));
}

__global__ void __launch_bounds__(TG_THREADS, 3) k_ls_accumulate_tc(Planes P, TcArgs A)
{
    extern __shared__ __align__(128) unsigned char tg_sh[];
    // the operand buffers (TG_BUFFERS x TG_KSTEPS tiles of 4 KB), then the staged site rows [site][TG_ROW]
    unsigned char* tiles = tg_sh;
    float* rows = reinterpret_cast<float*>(tg_sh + TG_BUFFERS * TG_KSTEPS * TG_TILE_BYTES);
    __shared__ uint64_t mbar[2];
    __shared__ uint32_t tmem_base;
    __shared__ int failed;

    const int pl = blockIdx.y;
    const PlaneView& V = P.p[pl];
    const int mm = P.nin + 1, nout = P.nout, kc = P.kc;
    const size_t sites = (size_t)V.w0 * V.h0 * (1 + kc);
    const size_t chunks = (sites + TG_SITES - 1) / TG_SITES;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int row_id = tid;   // this thread's TMEM lane (row of D)

    double acc[48];
#pragma unroll
    for (int j = 0; j < 48; j++)
        acc[j] = 0.0;

    const bool work = (size_t)blockIdx.x < chunks;
    if (work)
    {
        // the zero rows 96..127 of every tile, once; the other rows are rewritten every stage
        for (int i = tid; i < TG_BUFFERS * TG_KSTEPS * TG_TILE_BYTES / 16; i += TG_THREADS)
            reinterpret_cast<uint4*>(tiles)[i] = make_uint4(0u, 0u, 0u, 0u);
        if (warp == 0)
        {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                             smem_addr(&tmem_base)),
                         "r"((uint32_t)TG_TMEM_COLS)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
        if (tid == 0)
        {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar[0])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar[1])) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            failed = 0;
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tmem = tmem_base;
        const uint32_t tiles_addr = smem_addr(tiles);
        constexpr uint32_t idesc = umma_idesc_bf16(128, 96);
        // per buffer: the parity of its next completion, and whether a commit on it is still unwaited (every thread
        // keeps the same copy: all take the same branches)
        uint32_t ph[2] = { 0u, 0u };
        bool pending[2] = { false, false };
        auto settle = [&](int x) {
            if (!pending[x])
                return;
            if (!mbar_wait(&mbar[x], ph[x]))
                failed = 1;
            ph[x] ^= 1u;
            pending[x] = false;
        };
        int in_batch = 0, stage = 0;

        for (size_t chunk = blockIdx.x; chunk < chunks; chunk += gridDim.x, stage++)
        {
            const int bsel = stage % TG_BUFFERS;
            unsigned char* tb = tiles + (size_t)bsel * TG_KSTEPS * TG_TILE_BYTES;
            // 1. this thread's site row, in float (the MMAs of the previous stage run meanwhile)
            site_row(P, V, chunk * TG_SITES + tid, sites, rows + tid * TG_ROW);
            // 2. the buffer's previous MMAs are done before it is overwritten
            settle(bsel);
            __syncthreads();
            if (failed)
                break;
            // 3. the operand tiles: item (column f, 8-site group g) packs 8 sites of column f into 16 bytes, hi into
            //    row f and lo into row 48 + f
            for (int it = tid; it < 48 * (TG_SITES / 8); it += TG_THREADS)
            {
                const int f = it % 48, g = it / 48;
                uint32_t hi[4], lo[4];
#pragma unroll
                for (int q = 0; q < 8; q += 2)
                {
                    const float x0 = rows[(g * 8 + q) * TG_ROW + f], x1 = rows[(g * 8 + q + 1) * TG_ROW + f];
                    const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
                    const __nv_bfloat16 l0 = __float2bfloat16_rn(x0 - __bfloat162float(h0));
                    const __nv_bfloat16 l1 = __float2bfloat16_rn(x1 - __bfloat162float(h1));
                    hi[q / 2] = pack_bf16x2(h0, h1);
                    lo[q / 2] = pack_bf16x2(l0, l1);
                }
                const int step = g / 2, k = (g & 1) * 8;
                *reinterpret_cast<uint4*>(tb + tile_offset(step, f, k)) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
                *reinterpret_cast<uint4*>(tb + tile_offset(step, 48 + f, k)) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
            }
            // generic-proxy stores become visible to the tensor core's async proxy; the rows are free again
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncthreads();
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // 4. one thread issues the stage's MMAs and commits them to the buffer's barrier; nobody waits here
            if (tid == 0)
            {
                const uint32_t base = tiles_addr + (uint32_t)bsel * TG_KSTEPS * TG_TILE_BYTES;
                for (int s = 0; s < TG_KSTEPS; s++)
                {
                    const uint64_t desc = umma_desc(base + (uint32_t)s * TG_TILE_BYTES, 128, 256);
                    const uint32_t accumulate = (in_batch > 0 || s > 0) ? 1u : 0u;
                    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                                 "l"(desc), "l"(desc), "r"(idesc), "r"(accumulate)
                                 : "memory");
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_addr(&mbar[bsel]))
                             : "memory");
            }
            pending[bsel] = true;
            const bool last = chunk + gridDim.x >= chunks;
            if (++in_batch == TG_STAGES_PER_BATCH || last)
            {
                // 5. the batch's MMAs done, its FP32 sums into FP64: row r of D, columns j (hi) and 48 + j (lo)
                settle(0);
                settle(1);
                __syncthreads();
                if (failed)
                    break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                if (warp < 3)
                {
                    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
                    uint32_t v[32];
                    tmem_ld32(lane_base + 0, v);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int j = 0; j < 32; j++)
                        acc[j] += (double)__uint_as_float(v[j]);
                    tmem_ld32(lane_base + 32, v);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int j = 0; j < 16; j++)
                        acc[32 + j] += (double)__uint_as_float(v[j]);
#pragma unroll
                    for (int j = 0; j < 16; j++)
                        acc[j] += (double)__uint_as_float(v[16 + j]);
                    tmem_ld32(lane_base + 64, v);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int j = 0; j < 32; j++)
                        acc[16 + j] += (double)__uint_as_float(v[j]);
                }
                in_batch = 0;
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncthreads();
            }
        }
        if (failed)
        {
            if (tid == 0)
                atomicOr(A.status, 1u);
            // bounded: whatever the tensor core still holds of this CTA's work
            for (int x = 0; x < 2; x++)
                if (pending[x])
                    mbar_wait(&mbar[x], ph[x]);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (warp == 0)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                         "r"((uint32_t)TG_TMEM_COLS)
                         : "memory");
    }

    // the hi and lo rows of each Gram row added, then the entries the system needs, one partial per block
    __syncthreads();
    double* red = reinterpret_cast<double*>(tg_sh);   // [96][49] doubles: every row's sums
    if (row_id < 96)
    {
#pragma unroll
        for (int j = 0; j < 48; j++)
            red[row_id * 49 + j] = acc[j];
    }
    __syncthreads();
    if (row_id < mm)
    {
        const int a = row_id;
        for (int b = a; b < mm + nout; b++)
        {
            const double g = red[a * 49 + b] + red[(48 + a) * 49 + b];
            const int e = b < mm ? tri_index(a, b, mm) : mm * (mm + 1) / 2 + (b - mm) * mm + a;
            A.partial[((size_t)pl * A.entries + e) * LS_GRID + blockIdx.x] = g;
        }
    }
}

size_t ls_tc_shared_bytes()
{
    const size_t stage = (size_t)TG_BUFFERS * TG_KSTEPS * TG_TILE_BYTES + (size_t)TG_SITES * TG_ROW * sizeof(float);
    const size_t sums = (size_t)96 * 49 * sizeof(double);
    return stage > sums ? stage : sums;
}

int launch_ls_accumulate_tc(nntc_b200_device* d, const Planes& P, double* partial, int entries, cudaStream_t stream)
{
    const size_t shared = ls_tc_shared_bytes();
    NB_CUDA(cudaFuncSetAttribute(k_ls_accumulate_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shared));
    dim3 grid(LS_GRID, (unsigned)P.n);
    k_ls_accumulate_tc<<<grid, TG_THREADS, shared, stream>>>(P, TcArgs{ partial, entries, d->counters + CNT_STATUS });
    NB_LAUNCHED();
    return NNTC_B200_OK;
}

}   // namespace nb
