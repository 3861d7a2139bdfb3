// gram_tc.cu: block (a)'s normal equations on the fifth-generation tensor cores (tcgen05), BF16 operands split hi + lo,
// FP32 accumulators in tensor memory, FP64 across batches: the mixed-precision form of the accumulation that
// decoder.cu's k_ls_accumulate_mma does in FP64 (the sums of src/solve_decoder.cu:87-161).
//
// Every entry the decoder's system needs is an entry of the Gram Z^T Z of the site rows Z = [phi | 1 | t] (site_z()'s
// fixed 48-slot layout). A float x is split x = hi + lo with hi = bf16(x) and lo = bf16(x - hi) (x - hi is exact in
// float), which holds x to about 2^-17 of itself. A stage is 128 sites (site j of the 128 texels of a chunk, one per
// thread); their rows [Z_hi ; Z_lo] form one operand of 96 rows (48 hi, 48 lo) by 128 sites, and eight MMAs of
// M = 128, N = 96, K = 16 with that operand as both A and B produce the four products of the split at once:
//
//   D = [Z_hi ; Z_lo ; *] [Z_hi ; Z_lo]^T  =  [[hi hi, hi lo], [lo hi, lo lo], *]     (128 x 96, FP32, in TMEM)
//
// so Z^T Z = hi hi + hi lo + lo hi + lo lo: the compensated three-product form plus the lo lo term, which costs
// nothing more here. The rows are shifted before the split, z' = z - mu with mu the mean of the CTA's first 128
// centre sites (the constant's slot not shifted), and the shift is undone on the sums in FP64 at the end: the FP32
// accumulators then hold sums of small centred products instead of the large mean-dominated ones, whose rounding the
// decoder's system (nearly collinear with its constant column) would amplify (unshifted, the decoder of a converged
// state differed from the FP64 form's by 2.4e-4 of its largest coefficient). A's rows 96..127 are whatever follows
// in shared memory; the rows of D they produce are never read. After every batch of 256 sites the rows of D the
// system reads (phi and 1: 25 hi rows, 25 lo rows; row r of D is TMEM lane r) are read back, the hi and lo halves of
// each column added in FP32 and the sums added into FP64 rows in shared memory; a CTA writes one partial per entry,
// which k_ls_reduce folds in block order as it does for the FP64 form. Deterministic: the tensor core's sums of a
// batch are a fixed function of the operand, the rest is fixed-order.
//
// The operand is stored MN-major (no swizzle): a core matrix is 8 sites x 8 consecutive rows (16 bytes per site), so
// each thread writes its site's 96 values as twelve 16-byte stores straight from registers, rows 8g..8g+7 at
// g x TG_MN, the next eight sites at TG_KG. In the descriptor of this layout (MN-major, no swizzle) the leading byte
// offset is the K direction's stride and the stride byte offset the MN direction's. The offsets are chosen so that
// every byte the MMAs can address under either reading of the two strides lies inside the CTA's shared memory
// (checked at compile time below).
//
// The tensor-core plumbing, all by inline PTX: tcgen05.alloc / dealloc of 128 TMEM columns per CTA (at most four CTAs
// per SM by shared memory and registers, 512 of the 512 columns, so an allocation never waits on another CTA),
// shared-memory matrix
// descriptors, tcgen05.mma.cta_group::1.kind::f16 issued by one thread, tcgen05.commit to an mbarrier per operand
// buffer (one buffer: the next stage's rows are formed in registers while the stage's MMAs run, and stored once they
// are done; a second buffer measured slower, costing the fourth CTA per SM), tcgen05.ld of 32 lanes x 32
// columns per warp. No TMA, no multicast, no cluster: the operands are computed by the threads, not copied. Every wait
// on an mbarrier is bounded; a wait that gives up raises the device status word, waits (bounded) once more, frees the
// tensor memory and leaves.

#include <cstdint>

#include <cuda_bf16.h>

#include "device.cuh"
#include "site_rows.cuh"

namespace nb
{

constexpr int TG_THREADS = 128;                    // four warps; a thread's texel, and TMEM lane = row of D
constexpr int TG_SITES = 128;                      // sites per stage
constexpr int TG_KSTEPS = TG_SITES / 16;           // MMAs per stage
constexpr int TG_BUFFERS = 1;                      // operand buffers
constexpr int TG_STAGES_PER_BATCH = 2;             // FP32 accumulation spans 256 sites (512 measured
                                                   // 5x the decoder error at a converged state)
constexpr uint32_t TG_CORE = 128;                  // one core matrix: 8 sites x 8 rows of bf16
constexpr uint32_t TG_MN = TG_CORE;                // MN direction: the next eight rows
constexpr uint32_t TG_KG = 12 * TG_CORE;           // K direction: the next eight sites, after the 12 row groups
constexpr uint32_t TG_STEP = 2 * TG_KG;            // one K-step of 16 sites
constexpr uint32_t TG_BUF = TG_KSTEPS * TG_STEP;   // one stage's operand, 24 KB
constexpr int TG_ROWS = 25;                        // Gram rows the system reads (site_z slots 0..24)
constexpr int TG_ACC_STRIDE = 49;                  // doubles per FP64 row in shared memory
constexpr uint32_t TG_ACC_OFFSET = TG_BUFFERS * TG_BUF + 4 * TG_CORE;   // past A's rows 96..127 of the last step
constexpr uint32_t TG_ACC_BYTES = 2 * TG_ROWS * TG_ACC_STRIDE * sizeof(double);
constexpr int TG_TMEM_COLS = 128;                  // allocation (power of two >= 96)
constexpr uint32_t TG_WAIT_LIMIT = 1u << 26;

// The farthest byte an MMA of the last step of the last buffer can address, under either reading of LBO and SBO
// (16 row groups of A at the larger stride, the second K group at the larger stride, a 16-byte row): the dynamic
// shared memory is at least this long.
constexpr uint32_t TG_MAX_STRIDE = TG_MN > TG_KG ? TG_MN : TG_KG;
constexpr uint32_t TG_REACH = (TG_BUFFERS - 1) * TG_BUF + (TG_KSTEPS - 1) * TG_STEP + 16 * TG_MAX_STRIDE + 16;
constexpr uint32_t TG_SHARED = TG_ACC_OFFSET + TG_ACC_BYTES > TG_REACH ? TG_ACC_OFFSET + TG_ACC_BYTES : TG_REACH;
static_assert(TG_SHARED <= 56 * 1024, "four CTAs per SM");
static_assert(TG_ACC_OFFSET % 16 == 0 && TG_BUF % 16 == 0, "16-byte aligned operand and accumulator regions");

// The decoder for the objective the accumulation can form on the way (its own rows of Z are the sites' features and
// targets): each output row at a fixed stride of 24, [c (4)][s (4)][s c (4 x 4)], as the FP32 objective lays it out.
struct TcObjective
{
    float w[MAX_NOUT * 24];
    float b[MAX_NOUT];
    float cw[MAX_NOUT];
    double* partial;        // [plane][3][LS_GRID]: sum cw e^2, the centre sites' sum e^2, the fractional sites'
};

struct TcArgs
{
    double* partial;        // [plane][entry][LS_GRID]
    int entries;
    unsigned int* status;   // raised on a wait that gave up
    SiteTargetView tgt;
    TcObjective obj;        // read only by the OBJ instantiation
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

// The instruction descriptor of kind::f16: FP32 accumulator (bit 4), A and B BF16 (bits 7 and 10), A and B both
// MN-major (bits 15 and 16), N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t umma_idesc_bf16_mn(int m, int n)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(n >> 3) << 17) |
           ((uint32_t)(m >> 4) << 24);
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

// The batch's FP32 sums into the FP64 rows: warp w holds TMEM lanes 32w..32w+31; row r < 25 (hi) goes to FP64 row r,
// row 48 + r (lo) to FP64 row 25 + r; columns j (hi) and 48 + j (lo) of D are added first.
__device__ __forceinline__ void tc_readback(uint32_t tmem, int warp, int lane, double* acc)
{
    if (warp >= 3)
        return;
    const int r = warp * 32 + lane;
    const int row = r < TG_ROWS ? r : (r >= 48 && r < 48 + TG_ROWS ? TG_ROWS + r - 48 : -1);
    const uint32_t base = tmem + ((uint32_t)(warp * 32) << 16);
    float g[48];
    uint32_t v[32];
    tmem_ld32(base + 0, v);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; j++)
        g[j] = __uint_as_float(v[j]);
    tmem_ld32(base + 32, v);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; j++)
        g[32 + j] = __uint_as_float(v[j]);
#pragma unroll
    for (int j = 0; j < 16; j++)
        g[j] += __uint_as_float(v[16 + j]);
    tmem_ld32(base + 64, v);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; j++)
        g[16 + j] += __uint_as_float(v[j]);
    if (row >= 0)
    {
        double* a = acc + row * TG_ACC_STRIDE;
#pragma unroll
        for (int j = 0; j < 48; j++)
            a[j] += (double)g[j];
    }
}

// OBJ: also E of the decoder in A.obj at the same sites - the FP32 objective's decode and sums (k_objective_f32's
// arithmetic, its fused multiply-adds in its order), each site's squared residuals summed in FP32, the sites' sums per
// thread in FP64, one partial per CTA - so that the round's closing objective pass and the next round's normal
// equations, which read the same sites at the same latents, are one pass.
template <int NOUT, bool OBJ>
__global__ void __launch_bounds__(TG_THREADS, 4) k_ls_accumulate_tc(Planes P, const __grid_constant__ TcArgs A)
{
    extern __shared__ __align__(1024) unsigned char tg_sh[];
    unsigned char* tiles = tg_sh;
    double* acc = reinterpret_cast<double*>(tg_sh + TG_ACC_OFFSET);
    __shared__ uint64_t mbar[TG_BUFFERS];
    __shared__ uint32_t tmem_base;
    __shared__ __align__(16) float mu[ZS_WIDTH];   // the CTA's shift (zero in the constant's slot)

    const int pl = blockIdx.y;
    const PlaneView& V = P.p[pl];
    const int mm = P.nin + 1, kc = P.kc;
    const long long texels = (long long)V.w0 * V.h0;
    const long long chunks = (texels + TG_THREADS - 1) / TG_THREADS;
    const float* tgt = A.tgt.t + (size_t)A.tgt.site0[pl] * NOUT;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    double e_weighted = 0.0, e_centre = 0.0, e_fractional = 0.0;   // OBJ: this thread's sites' sums

    for (int i = tid; i < 2 * TG_ROWS * TG_ACC_STRIDE; i += TG_THREADS)
        acc[i] = 0.0;

    if ((long long)blockIdx.x < chunks)
    {
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
            for (int x = 0; x < TG_BUFFERS; x++)
                asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mbar[x])) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const uint32_t tmem = tmem_base;
        const uint32_t tiles_addr = smem_addr(tiles);
        constexpr uint32_t idesc = umma_idesc_bf16_mn(128, 96);
        // per buffer: the parity of its next completion, and whether a commit on it is still unwaited (every thread
        // keeps the same copy: all take the same branches); gave_up: one of this thread's waits ran out, which the
        // next barrier (__syncthreads_or) makes every thread's decision at once
        // (bit x of each mask for buffer x, so that nothing is indexed at run time)
        uint32_t ph = 0u, pending = 0u;
        bool gave_up = false;
        auto settle = [&](int x) {
            const uint32_t bit = 1u << x;
            if (!(pending & bit))
                return;
            if (!mbar_wait(&mbar[x], (ph >> x) & 1u))
                gave_up = true;
            ph ^= bit;
            pending &= ~bit;
        };
        // the shift: the mean of the centre sites of the CTA's first chunk, in a fixed order (rows staged in the first
        // operand buffer as floats, then one column per thread)
        {
            const long long pixel = (long long)blockIdx.x * TG_THREADS + tid;
            const bool valid = pixel < texels;
            float z[ZS_WIDTH];
            if (valid)
                site_z<NOUT>(P, V, tgt, pixel, (int)(pixel % V.w0), (int)(pixel / V.w0), 0, z);
            float* rows = reinterpret_cast<float*>(tiles);   // [TG_THREADS][ZS_WIDTH + 1]
#pragma unroll
            for (int q = 0; q < ZS_WIDTH; q++)
                rows[tid * (ZS_WIDTH + 1) + q] = valid ? z[q] : 0.0f;
            __syncthreads();
            if (tid < ZS_WIDTH)
            {
                const int n = (int)min((long long)TG_THREADS, texels - (long long)blockIdx.x * TG_THREADS);
                float sum = 0.0f;
                for (int t = 0; t < n; t++)
                    sum += rows[t * (ZS_WIDTH + 1) + tid];
                mu[tid] = tid == ZS_ONE ? 0.0f : sum / (float)n;
            }
            __syncthreads();
        }
        // this thread's site within a stage: K-step tid / 16, K group (tid / 8) % 2, row tid % 8 of its core matrices
        const uint32_t my_site = (uint32_t)(tid >> 4) * TG_STEP + (uint32_t)((tid >> 3) & 1) * TG_KG +
                                 (uint32_t)(tid & 7) * 16;
        int in_batch = 0, stage = 0;
        bool stop = false;

        for (long long chunk = blockIdx.x; chunk < chunks && !stop; chunk += gridDim.x)
        {
            const long long pixel = chunk * TG_THREADS + tid;
            const bool valid = pixel < texels;
            const int px = valid ? (int)(pixel % V.w0) : 0, py = valid ? (int)(pixel / V.w0) : 0;
            for (int j = 0; j <= kc; j++, stage++)
            {
                const int bsel = stage % TG_BUFFERS;
                // 1. this thread's site row, split hi + lo in registers (the previous stage's MMAs run meanwhile)
                float z[ZS_WIDTH];
                if (valid)
                {
                    site_z<NOUT>(P, V, tgt, pixel, px, py, j, z);
                    if constexpr (OBJ)
                    {
                        float sw = 0.0f, ss = 0.0f;
#pragma unroll
                        for (int r = 0; r < NOUT; r++)
                        {
                            float acc = A.obj.b[r];
#pragma unroll
                            for (int h = 0; h < 4; h++)
                                acc = __fmaf_rn(A.obj.w[r * 24 + h], z[ZS_C + h], acc);
#pragma unroll
                            for (int h = 0; h < 4; h++)
                                acc = __fmaf_rn(A.obj.w[r * 24 + 4 + h], z[ZS_S + h], acc);
#pragma unroll
                            for (int h = 0; h < 16; h++)
                                acc = __fmaf_rn(A.obj.w[r * 24 + 8 + h], z[ZS_SC + h], acc);
                            const float e = acc - z[ZS_T + r];
                            sw = __fmaf_rn(A.obj.cw[r] * e, e, sw);
                            ss = __fmaf_rn(e, e, ss);
                        }
                        e_weighted += (double)sw;
                        if (j == 0)
                            e_centre += (double)ss;
                        else
                            e_fractional += (double)ss;
                    }
#pragma unroll
                    for (int q = 0; q < ZS_WIDTH; q += 4)
                    {
                        const float4 m4 = *reinterpret_cast<const float4*>(mu + q);
                        z[q] -= m4.x;
                        z[q + 1] -= m4.y;
                        z[q + 2] -= m4.z;
                        z[q + 3] -= m4.w;
                    }
                }
                else
                {
#pragma unroll
                    for (int q = 0; q < ZS_WIDTH; q++)
                        z[q] = 0.0f;
                }
                uint32_t hi[ZS_WIDTH / 2], lo[ZS_WIDTH / 2];
#pragma unroll
                for (int q = 0; q < ZS_WIDTH / 2; q++)
                {
                    const __nv_bfloat162 h = __floats2bfloat162_rn(z[2 * q], z[2 * q + 1]);
                    const float2 hf = __bfloat1622float2(h);
                    const __nv_bfloat162 l = __floats2bfloat162_rn(z[2 * q] - hf.x, z[2 * q + 1] - hf.y);
                    hi[q] = *reinterpret_cast<const uint32_t*>(&h);
                    lo[q] = *reinterpret_cast<const uint32_t*>(&l);
                }
                // 2. the buffer's previous MMAs are done before it is overwritten
                settle(bsel);
                unsigned char* at = tiles + (size_t)bsel * TG_BUF + my_site;
#pragma unroll
                for (int g = 0; g < 6; g++)
                {
                    *reinterpret_cast<uint4*>(at + g * TG_MN) =
                        make_uint4(hi[4 * g], hi[4 * g + 1], hi[4 * g + 2], hi[4 * g + 3]);
                    *reinterpret_cast<uint4*>(at + (6 + g) * TG_MN) =
                        make_uint4(lo[4 * g], lo[4 * g + 1], lo[4 * g + 2], lo[4 * g + 3]);
                }
                // generic-proxy stores become visible to the tensor core's async proxy
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                if (__syncthreads_or(gave_up))
                {
                    stop = true;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                // 3. one thread issues the stage's MMAs and commits them to the buffer's barrier; nobody waits here
                if (tid == 0)
                {
                    const uint32_t base = tiles_addr + (uint32_t)bsel * TG_BUF;
                    for (int s = 0; s < TG_KSTEPS; s++)
                    {
                        const uint64_t desc = umma_desc(base + (uint32_t)s * TG_STEP, TG_KG, TG_MN);
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
                pending |= 1u << bsel;
                if (++in_batch == TG_STAGES_PER_BATCH)
                {
                    // 4. the batch's MMAs done, its FP32 sums into the FP64 rows
                    for (int x = 0; x < TG_BUFFERS; x++)
                        settle(x);
                    if (__syncthreads_or(gave_up))
                    {
                        stop = true;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    tc_readback(tmem, warp, lane, acc);
                    in_batch = 0;
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    __syncthreads();
                }
            }
        }
        if (!stop && in_batch > 0)
        {
            for (int x = 0; x < TG_BUFFERS; x++)
                settle(x);
            if (!__syncthreads_or(gave_up))
            {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                tc_readback(tmem, warp, lane, acc);
            }
        }
        if (__syncthreads_or(gave_up))
        {
            if (tid == 0)
                atomicOr(A.status, 1u);
            // bounded: whatever the tensor core still holds of this CTA's work
            for (int x = 0; x < TG_BUFFERS; x++)
                if (pending & (1u << x))
                    mbar_wait(&mbar[x], (ph >> x) & 1u);
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (warp == 0)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                         "r"((uint32_t)TG_TMEM_COLS)
                         : "memory");
    }

    // entry (a, b) of the compact system from the shifted sums c (FP64 rows z_slot(a) (hi) plus 25 + z_slot(a) (lo),
    // column z_slot(b)): with z = z' + mu and the constant's slot unshifted, sum z_a z_b = c_ab + mu_a c_1b + mu_b c_1a
    // + mu_a mu_b c_11, in FP64
    __syncthreads();
    const bool shifted = (long long)blockIdx.x < chunks;
    auto cs = [&](int r, int col) {
        return acc[r * TG_ACC_STRIDE + col] + acc[(TG_ROWS + r) * TG_ACC_STRIDE + col];
    };
    const int tri = mm * (mm + 1) / 2;
    for (int e = tid; e < A.entries; e += TG_THREADS)
    {
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
        double g = cs(sa, sb);
        if (shifted)
        {
            const double ma = (double)mu[sa], mb = (double)mu[sb];
            g += ma * cs(ZS_ONE, sb) + mb * cs(ZS_ONE, sa) + ma * mb * cs(ZS_ONE, ZS_ONE);
        }
        A.partial[((size_t)pl * A.entries + e) * LS_GRID + blockIdx.x] = g;
    }
    if constexpr (OBJ)
    {
        // the CTA's three objective sums: each warp's in lane order, then the four warps' in warp order
        __shared__ double ored[3][TG_THREADS / 32];
        double v[3] = { e_weighted, e_centre, e_fractional };
#pragma unroll
        for (int q = 0; q < 3; q++)
        {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
            if (lane == 0)
                ored[q][warp] = v[q];
        }
        __syncthreads();
        if (tid < 3)
        {
            double t = 0.0;
            for (int w = 0; w < TG_THREADS / 32; w++)
                t += ored[tid][w];
            A.obj.partial[((size_t)pl * 3 + tid) * LS_GRID + blockIdx.x] = t;
        }
    }
}

int launch_ls_accumulate_tc(nntc_b200_device* d, const Planes& P, double* partial, int entries,
                            const SiteTargetView& tgt, cudaStream_t stream, double* obj_partial)
{
    dim3 grid(LS_GRID, (unsigned)P.n);
    TcArgs args{ partial, entries, d->counters + CNT_STATUS, tgt, {} };
    if (obj_partial)
    {
        // the decoder as uploaded, in the objective's row layout
        const int nin = d->nin, c0 = d->c0, c1 = d->c1;
        for (int r = 0; r < d->nout; r++)
        {
            for (int q = 0; q < c1; q++)
                args.obj.w[r * 24 + q] = d->host_weights[(size_t)r * nin + q];
            for (int i = 0; i < c0; i++)
                args.obj.w[r * 24 + 4 + i] = d->host_weights[(size_t)r * nin + c1 + i];
            for (int i = 0; i < c0; i++)
                for (int q = 0; q < c1; q++)
                    args.obj.w[r * 24 + 8 + i * 4 + q] = d->host_weights[(size_t)r * nin + c1 + c0 + i * c1 + q];
            args.obj.b[r] = d->host_bias[r];
            args.obj.cw[r] = d->m.cw[r];
        }
        args.obj.partial = obj_partial;
    }
#define NB_TC(NO)                                                                                                     \
    case NO:                                                                                                          \
        if (obj_partial)                                                                                              \
        {                                                                                                             \
            NB_CUDA(cudaFuncSetAttribute(k_ls_accumulate_tc<NO, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,  \
                                         (int)TG_SHARED));                                                            \
            k_ls_accumulate_tc<NO, true><<<grid, TG_THREADS, TG_SHARED, stream>>>(P, args);                           \
        }                                                                                                             \
        else                                                                                                          \
        {                                                                                                             \
            NB_CUDA(cudaFuncSetAttribute(k_ls_accumulate_tc<NO, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                         (int)TG_SHARED));                                                            \
            k_ls_accumulate_tc<NO, false><<<grid, TG_THREADS, TG_SHARED, stream>>>(P, args);                          \
        }                                                                                                             \
        break;
    switch (d->nout)
    {
        NB_TC(3)
        NB_TC(6)
        NB_TC(9)
        NB_TC(12)
        NB_TC(15)
        NB_TC(18)
    default:
        set_error(NNTC_B200_ERR_STATE, "a material holds 1..6 RGB textures");
        return NNTC_B200_ERR_STATE;
    }
#undef NB_TC
    NB_LAUNCHED();
    return NNTC_B200_OK;
}

}   // namespace nb
