// device.cuh: the device-resident model of one encode (the reference's DeviceModel, src/device.cuh:193-375).
//
// Differences from the reference's layout, all B200-first:
//
// - ONE stream. Every kernel covers every plane of the chain in one launch through nb::Planes, so there is no
//   per-plane stream fan-out / fan-in (src/device.cuh:378-434) and no per-plane launch cost.
// - The stencil is stored structure-of-arrays, [slot][i][j][texel], so that a warp reading one coefficient of 32
//   consecutive texels reads 256 contiguous bytes; the reference's [texel][slot][i][j] puts 640 bytes between two
//   lanes at C = 4. The probe transposes it back into the reference's order on download.
// - Reductions are per (plane, block) partials on a fixed grid, added in a fixed order by a second kernel: the same
//   determinism rule as the reference (src/device.cuh:88-90), with one launch for every plane.
#pragma once

#include <vector>

#include "common.cuh"

namespace nb
{

// Scalars one plane's block (b)/(c') solve keeps on the device (src/device.cuh:145-165).
enum Scalar
{
    S_DIAG_SUM = 0,
    S_DIAG_MIN,
    S_DIAG_MAX,
    S_LAMBDA,
    S_RHS2,
    S_RZ,
    S_RZ_NEW,
    S_PAP,
    S_RR,
    S_RESID,
    S_ALPHA,
    S_BETA,
    S_MOVED,
    S_DELTA2,
    S_PLANE2,
    S_ACTIVE,
    S_ITER,
    S_LO,
    S_HI = S_LO + MAX_CH,
    S_COUNT = S_HI + MAX_CH
};

// The fixed reduction grid: partials are [row][plane][RGRID].
constexpr int RGRID = 148 * 4;
constexpr int RROWS = 3 + 2 * MAX_CH;
constexpr int THREADS = 256;
constexpr int GATHER_TABLE_MAX = 8192;   // int4 entries of one visit table
constexpr int LS_GRID = 148 * 4;         // normal equations: blocks per plane (four per SM at the base plane)
constexpr int COV_GRID = 512;            // init covariance: partials per entry
constexpr int HIST_BINS = 4096;          // init0: the percentile histogram
// The counter words: the quantised sweeps' moved count per plane, block (c)'s four colour passes per plane, and the
// conjugate gradients' active-plane counts of the last CG_PROBE iterations.
constexpr int CNT_SWEEP = 0;
constexpr int CNT_SEARCH = 16;
constexpr int CNT_ACTIVE = CNT_SEARCH + 4 * 16;
constexpr int CNT_STATUS = CNT_ACTIVE + 16;   // the device status word: raised by a bounded wait that gave up
constexpr int COUNTERS = CNT_STATUS + 1;

// Entry (i, j), i <= j, of an m x m symmetric matrix's upper triangle stored row by row.
__host__ __device__ inline int tri_index(int i, int j, int mm)
{
    return i * mm - i * (i - 1) / 2 + (j - i);
}

struct Work
{
    int w = 0, h = 0, c = 0;
    double* stencil = nullptr;
    double* grad = nullptr;
    float* precond = nullptr;
    double* x = nullptr;
    double* r = nullptr;
    double* z = nullptr;
    double* p = nullptr;
    double* ap = nullptr;
    float* prev = nullptr;
    size_t texels() const { return (size_t)w * h; }
    size_t values() const { return texels() * (size_t)c; }
};

struct DevPlane
{
    int w0 = 0, h0 = 0, w1 = 0, h1 = 0;
    float* src = nullptr;
    float* v0 = nullptr;
    float* v1 = nullptr;
    uint8_t* k0 = nullptr;
    uint8_t* k1 = nullptr;
    Work work[2];             // [0] level 1 (block b), [1] level 0 (block c', bc8 only)
    uint8_t* bc_ep = nullptr; // blocks * c0 * 2
    uint8_t* bc_sel = nullptr;// blocks * c0 * 16
    // level 0's FP64 stencil again, block-major for the BC refinement: [block][slot][i][j][texel of the 4x4 block],
    // written by the assembly the refinement runs on (a block's whole stencil is one contiguous run)
    double* bc_sten = nullptr;
    size_t blocks() const { return (size_t)((w0 + 3) / 4) * (size_t)((h0 + 3) / 4); }
};

}   // namespace nb

struct nntc_b200_device
{
    nntc_b200_model m{};                 // the layout and the last decoder / grids uploaded
    std::vector<nb::DevPlane> planes;
    float* weights = nullptr;            // nout * nin
    float* bias = nullptr;               // nout
    // Host copies of exactly what `weights` and `bias` hold (zero until a decoder is uploaded), for kernels that take
    // the decoder as a launch parameter.
    float host_weights[NNTC_B200_MAX_NOUT * NNTC_B200_MAX_NIN] = {};
    float host_bias[NNTC_B200_MAX_NOUT] = {};
    float* palette = nullptr;            // MAX_CH * 16
    float* lo1 = nullptr;
    float* hi1 = nullptr;
    float* lo0 = nullptr;
    float* hi0 = nullptr;
    float* cw = nullptr;
    double* mono[2] = { nullptr, nullptr };   // monomial matrices of block (b) and block (c')
    double* partial = nullptr;           // RROWS * (the chain's 256-texel blocks)
    double* scalars = nullptr;           // MAX_PLANES * S_COUNT
    unsigned int* counters = nullptr;    // COUNTERS words
    double* reduction = nullptr;         // the normal equations of the last block (a)
    void* dec_solve = nullptr;           // the device decoder solve's answer: the rung and the decoder (2 KB)
    double* ls_partial = nullptr;        // planes * entries * LS_GRID, then one weight per plane
    double* obj_partial = nullptr;       // 3 * MAX_PLANES * OBJ_GRID
    double* ls_obj = nullptr;            // planes * 3 * LS_GRID: the objective sums the normal equations' pass forms
    double* bc_stats = nullptr;          // MAX_PLANES * 2
    unsigned int* radix = nullptr;       // 2 * MAX_CH * 2048 words: the grid fit's histograms and flags
    double* site_terms = nullptr;        // every site's gradient term of the assembly, max(C0, C1) per site at K = 4
    size_t site_terms_count = 0;         // doubles in site_terms
    float* site_y = nullptr;             // every site's sample of the OTHER latent, 4 floats per site (assembly)
    float* site_tgt = nullptr;           // the fractional sites' float targets at K, nout per site (assembly)
    int site_tgt_kc = -1;                // the K site_tgt holds (-1: none yet; the source never changes)
    double* obj_tgt = nullptr;           // the fractional sites' double targets at K, nout per site (objective)
    int obj_tgt_kc = -1;                 // the K obj_tgt holds (-1: none yet)
    void* gtab[2] = { nullptr, nullptr };// the gather's visit tables of level 1 / level 0 (GATHER_TABLE_MAX int4 each)
    int gtab_kc[2] = { -1, -1 };         // the K each table was built for (-1: none yet)
    int gtab_off[2][4][6] = {};          // each table's entry ranges per parity class and slot
    int reference_shaped_assembly = 0;   // 1: the per-texel gather of the reference's shape (same bits, slower)
    int mixed_gram = 0;                  // 1: block (a)'s sums on the tensor cores, BF16 hi + lo (gram_tc.cu)
    int bc_copy = 0;                     // 1 while the assembly for the BC refinement runs: also write bc_sten
    int bc_copied = 0;                   // the last such assembly wrote bc_sten itself
    int adjoint_cg = 0;                  // 1: blocks (b) and (c')'s conjugate gradients matrix-free (adjoint_cg.cu)
    int mixed_objective = 0;             // 1: the objective's decode in FP32, its squares summed in FP64
    int mixed_stencil = 0;               // 1: blocks (b) and (c') assemble an FP32 stencil (gathers in FP32)
    bool sten_f32[2] = { false, false }; // what the last assembly of level 1 / level 0 stored: FP32 or FP64
    double* cov = nullptr;               // the init's moment partials, [entry][COV_GRID]
    void* basis = nullptr;               // the init's principal directions, peaks and divisor (1 KB)
    unsigned long long* hist = nullptr;  // the percentile histogram (init0, palette mode)
    float* scratch = nullptr;            // the largest plane's worth of floats (level 0 or level 1)
    uint8_t* scratch8 = nullptr;         // the largest plane's worth of bytes
    uint8_t* rgb8 = nullptr;             // the largest level's decoded bytes
    size_t scratch_floats = 0, scratch_bytes = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[4] = {};
    double* host_scalars = nullptr;      // pinned, MAX_PLANES * S_COUNT
    unsigned int* host_counters = nullptr;
    void* arena = nullptr;               // the one device allocation every buffer above is a slice of
    void* keep = nullptr;                // bc8: the outer repack loop's copy of both latents and the BC state
    size_t bytes = 0;                    // the arena's size
    int nout = 0, nin = 0, c0 = 0, c1 = 0;
    bool l0_bc8 = false;

    // Per-kernel event timing (nntc_b200_kernel_timing): pairs recorded around each launch of a hot kernel, read back
    // after the block that launched them has been waited for.
    struct Pending
    {
        int kind;
        cudaEvent_t a, b;
    };
    bool ktiming = false;
    std::vector<cudaEvent_t> kpool;
    std::vector<Pending> kpending;
    long long klaunches[NNTC_B200_K_COUNT] = {};
    double kms[NNTC_B200_K_COUNT] = {};
};

namespace nb
{

// What the outer repack loop keeps of a rejected pass (bc8): both latents' values and indices and the BC state of
// every plane, each part at a 256-byte boundary of the device's `keep` buffer.
template <typename F>
void for_each_kept(nntc_b200_device* d, F f)
{
    for (DevPlane& p : d->planes)
    {
        const size_t n0 = (size_t)p.w0 * p.h0 * d->c0, n1 = (size_t)p.w1 * p.h1 * d->c1;
        f((void*)p.v0, n0 * sizeof(float));
        f((void*)p.k0, n0);
        f((void*)p.v1, n1 * sizeof(float));
        f((void*)p.k1, n1);
        if (d->l0_bc8)
        {
            f((void*)p.bc_ep, p.blocks() * d->c0 * 2);
            f((void*)p.bc_sel, p.blocks() * d->c0 * 16);
        }
    }
}

// The Planes descriptor of a call, with the per-plane item ranges padded to whole THREADS-sized chunks so that no
// chunk of a launch straddles two planes. `items(i)` is the plane's work-item count.
template <class F>
inline Planes planes_for(const nntc_b200_device* d, int level0, F items)
{
    Planes P{};
    P.n = (int)d->planes.size();
    P.c0 = d->c0;
    P.c1 = d->c1;
    P.nin = d->nin;
    P.nout = d->nout;
    P.c = level0 ? d->c0 : d->c1;
    long long at = 0;
    for (int i = 0; i < P.n; i++)
    {
        const DevPlane& s = d->planes[(size_t)i];
        PlaneView& v = P.p[i];
        v.w0 = s.w0;
        v.h0 = s.h0;
        v.w1 = s.w1;
        v.h1 = s.h1;
        v.src = s.src;
        v.v0 = s.v0;
        v.v1 = s.v1;
        v.k0 = s.k0;
        v.k1 = s.k1;
        const Work& w = s.work[level0 ? 1 : 0];
        v.w = level0 ? s.w0 : s.w1;
        v.h = level0 ? s.h0 : s.h1;
        v.v = level0 ? s.v0 : s.v1;
        v.k = level0 ? s.k0 : s.k1;
        v.stencil = w.stencil;
        v.grad = w.grad;
        v.precond = w.precond;
        v.x = w.x;
        v.r = w.r;
        v.z = w.z;
        v.p = w.p;
        v.ap = w.ap;
        v.prev = w.prev;
        v.bc_sten = level0 ? s.bc_sten : nullptr;
        P.start[i] = at;
        const long long n = (long long)items(i);
        at += (n + THREADS - 1) / THREADS * THREADS;
    }
    P.start[P.n] = at;
    return P;
}

// Record the span of a block of work on the model's stream and return it in ms after synchronising.
int block_begin(nntc_b200_device* d);
int block_end(nntc_b200_device* d, double* ms);

// Brackets of one launch of a hot kernel (no-ops unless kernel timing is on); harvested at every block_end.
int ktimer_begin(nntc_b200_device* d, int kind);
int ktimer_end(nntc_b200_device* d);
int ktimer_harvest(nntc_b200_device* d);

// Planes 1.. of the source chain from plane 0, on the device: each level the 2x2 box of the one above.
int build_source_chain(nntc_b200_device* d);

// Upload on the model's stream and wait (the staging buffer is the caller's).
int upload(nntc_b200_device* d, void* dst, const void* src, size_t bytes);
int download(nntc_b200_device* d, void* dst, const void* src, size_t bytes);

// Host-side ownership checks shared by the entry points.
int check_plane(const nntc_b200_device* d, int plane);

// The decoder and the grids as the model carries them, uploaded (src/device.cuh:436-478).
int upload_decoder(nntc_b200_device* d, const nntc_b200_model* m);
int upload_grids(nntc_b200_device* d, const nntc_b200_model* m);

// The monomial matrices of block (b) (level0 = 0) or block (c') (level0 = 1), built on the host from the decoder
// (src/solve_level1.cu:164-244).
void build_monomials(const nntc_b200_model& m, int level0, std::vector<double>& p);
// The layout checks device_create applies to a model (counts, caps, plane sizes); NNTC_B200_OK or ERR_ARG with a message.
int validate_model(const nntc_b200_model* m);

}   // namespace nb
