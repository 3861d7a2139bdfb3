/* nntc_b200.h: the C ABI of the B200-native encoder hot path.
 *
 * Every entry point here stands in for one function of the reference's device seam. The reference declares those as
 * 46 C++ functions over `DeviceModel*` (src/cuda_backend.h:20-80, which is src/backend.h:86-150 with DeviceModel* in
 * place of be::Device*); their C++ signatures carry std::vector, std::string and Model&, which no FFI can bind. This
 * header restates each one over plain pointers and sizes:
 *
 *   - the reference's `Model` (src/model.h:56-114) becomes `nntc_b200_model`, a fixed-size POD carrying the layout,
 *     the decoder, the per-output weights and the grids. The per-plane arrays Model owns (k0, k1, the BC blocks) are
 *     passed as caller-owned per-plane buffers, one pointer per stored plane, sized by the layout;
 *   - the report structs (Level1Report, Level0Report, Objective, BcRefineReport, Level1InitReport,
 *     Init0ChannelReport, src/model.h:281-519) become fixed-size PODs with the same fields;
 *   - every call returns an int status (NNTC_B200_OK on success) instead of printing and exiting; the message of the
 *     last failure is nntc_b200_last_error(). The C++ adapter in nntc_b200/seam turns a failure back into the
 *     reference's one ERROR line and exit status 1 (src/device.cuh:45-76).
 *
 * Threading: one host thread per device handle. Every call returns with its results visible to the host, as the
 * reference's calls do (each block ends with one synchronisation of the master stream, src/device.cuh:403-411).
 */
#ifndef NNTC_B200_H
#define NNTC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NNTC_B200_MAX_PLANES 13    /* the base and MAX_MIP_LEVELS = 12 more (src/model.h:32) */
#define NNTC_B200_MAX_CHANNELS 4   /* per-level channel cap (src/device.cuh:80) */
#define NNTC_B200_MAX_NIN 24       /* |phi| cap (src/device.cuh:81) */
#define NNTC_B200_MAX_NOUT 18      /* 3 channels x MAX_TEXTURES 6 (src/model.h:39, src/device.cuh:82) */

enum nntc_b200_status
{
    NNTC_B200_OK = 0,
    NNTC_B200_ERR_ARG = 1,     /* an argument the call cannot take (a size, a plane index, a null pointer) */
    NNTC_B200_ERR_CUDA = 2,    /* a CUDA call failed; the message names it */
    NNTC_B200_ERR_OOM = 3,     /* device memory ran out (src/init.cu:135-149 says it in the user's terms) */
    NNTC_B200_ERR_NODEV = 4,   /* no usable device */
    NNTC_B200_ERR_STATE = 5,   /* the call needs state the handle does not have (e.g. level 0's grid outside bc8) */
    NNTC_B200_ERR_TIMEOUT = 6, /* a bounded device-side wait gave up; the device status word says where */
    NNTC_B200_ERR_IO = 7       /* a file could not be written (the asset writer) */
};

/* The model: src/model.h:56-114 as a fixed-size POD. Fields that are std::vector in the reference carry a count. */
typedef struct nntc_b200_model
{
    int textures;                 /* T */
    int nout;                     /* 3 T */
    int width, height;            /* level 0's base extent */
    int c0, c1;                   /* level-0 and level-1 channels */
    int bits0[NNTC_B200_MAX_CHANNELS];
    int bits1;
    int bc0;                      /* the shipped level-0 format is BC4/BC5 (decides the palette) */
    int l0_bc8;                   /* --l0 bc8: level 0 is a continuous 8-bit plane on lo0/hi0 */
    int init0_residual, init0_texture, init0_chain;
    int nin;                      /* C1 + C0 + C0 C1 */
    int nplanes;                  /* the base first */
    int w0[NNTC_B200_MAX_PLANES], h0[NNTC_B200_MAX_PLANES];
    int w1[NNTC_B200_MAX_PLANES], h1[NNTC_B200_MAX_PLANES];
    float cw[NNTC_B200_MAX_NOUT]; /* per-output weight of the objective */
    int has_decoder;              /* 0: m.dec.w / m.dec.b are empty (no decoder yet) */
    float dec_w[NNTC_B200_MAX_NOUT * NNTC_B200_MAX_NIN];   /* nout x nin, row-major */
    float dec_b[NNTC_B200_MAX_NOUT];
    int palette0_len[NNTC_B200_MAX_CHANNELS];              /* 0 under --l0 bc8 */
    float palette0[NNTC_B200_MAX_CHANNELS][16];
    int has_lo0, has_lo1;         /* lo0/hi0 and lo1/hi1 present (non-empty vectors in the reference) */
    float lo0[NNTC_B200_MAX_CHANNELS], hi0[NNTC_B200_MAX_CHANNELS];
    float lo1[NNTC_B200_MAX_CHANNELS], hi1[NNTC_B200_MAX_CHANNELS];
} nntc_b200_model;

typedef struct nntc_b200_device_info
{
    char name[256];
    int major, minor;
    char error[512];
} nntc_b200_device_info;

/* Level1Report, src/model.h:374-398. */
typedef struct nntc_b200_plane_report
{
    int iterations;
    double residual, lambda, min_diag, max_diag;
    double ms_assemble, ms_precond, ms_cg;
    long long moved_values;
    double delta2, plane2;
    float lo[NNTC_B200_MAX_CHANNELS], hi[NNTC_B200_MAX_CHANNELS];
    int quantised, sweeps;
    long long moved;
    double ms_sweeps;
} nntc_b200_plane_report;

/* Level0Report, src/model.h:440-447. */
typedef struct nntc_b200_level0_report
{
    long long moved[4];
    long long moved_total;
    double ms;
    int joint;
    long long states;
} nntc_b200_level0_report;

/* Objective, src/model.h:467-478, with the per-plane vectors as fixed arrays of nplanes entries. */
typedef struct nntc_b200_objective
{
    double e;
    double e_plane[NNTC_B200_MAX_PLANES];
    double centre_mse, sampled_mse;
    double centre_plane[NNTC_B200_MAX_PLANES];
    double ms;
} nntc_b200_objective;

/* Level1InitReport, src/model.h:281-289. */
typedef struct nntc_b200_init1_report
{
    int pca, components;
    double eigenvalue[4], peak[4];
    double total_variance;
} nntc_b200_init1_report;

/* Init0ChannelReport, src/model.h:314-326. */
typedef struct nntc_b200_init0_report
{
    double eigenvalue, total_variance, share, peak, divisor;
    double dir[NNTC_B200_MAX_NOUT];
    int nout, texture;
} nntc_b200_init0_report;

/* BcRefineReport, src/model.h:512-519. */
typedef struct nntc_b200_bc_report
{
    int pass;
    long long blocks, improved;
    double delta_e, ms;
} nntc_b200_bc_report;

typedef struct nntc_b200_device nntc_b200_device;

/* The message of the last failed call on this thread; "" when none failed. */
const char* nntc_b200_last_error(void);
/* The ABI version of this header (1). */
int nntc_b200_version(void);
/* sizeof of the ABI's structs, in declaration order (model, device_info, plane_report, level0_report, objective,
 * init1_report, init0_report, bc_report, encode_args, encode_result), so a foreign binding can check its mirror.
 * Touches no device. Returns the count written (at most n). */
int nntc_b200_abi_sizes(size_t* out, int n);

/* ---- lifecycle: src/init.cu:76-382 (device_select, device_create, device_destroy, device_memory) ---- */
int nntc_b200_device_select(int index, nntc_b200_device_info* info);           /* returns 1 if usable */
int nntc_b200_device_create(const nntc_b200_model* m, const float* const* source_chain, nntc_b200_device** out);
/* The same device model from the base plane alone (w0[0] x h0[0] x nout floats): the other levels of the default
 * source chain - each the 2x2 box of the one above, src/mips.cpp:80-84 over src/image.h:343-364 - are built on the
 * device, bit for bit the reference's. The model's planes must be that chain's sizes (each the floor halving of the
 * one above, never below one texel). */
int nntc_b200_device_create_from_base(const nntc_b200_model* m, const float* base, nntc_b200_device** out);
void nntc_b200_device_destroy(nntc_b200_device* d);                             /* NULL is a no-op */
size_t nntc_b200_device_memory(const nntc_b200_device* d);

/* ---- initialisation and grids: src/init.cu:446-1400 ---- */
int nntc_b200_init_level0(nntc_b200_device* d, const nntc_b200_model* m, const float luma[3], int luma_channel0,
                          uint8_t* const* k0_out);
int nntc_b200_init_level1(nntc_b200_device* d, nntc_b200_model* m, int pca, nntc_b200_init1_report* rep,
                          uint8_t* const* k1_out);
int nntc_b200_init0_residual_channel(nntc_b200_device* d, const nntc_b200_model* m, int channel,
                                     const double* plane_weight, nntc_b200_init0_report* rep, uint8_t* const* k0_io);
/* range_pct: 1 for --q1-range pct, 0 for minmax. lo/hi written into m, indices into k_out. */
int nntc_b200_quantise_level1(nntc_b200_device* d, nntc_b200_model* m, int range_pct, uint8_t* const* k1_out);
int nntc_b200_freeze_level1_grid(nntc_b200_device* d, nntc_b200_model* m, int range_pct, uint8_t* const* k1_out);
int nntc_b200_quantise_level0(nntc_b200_device* d, nntc_b200_model* m, int range_pct, uint8_t* const* k0_out);
int nntc_b200_freeze_level0_grid(nntc_b200_device* d, nntc_b200_model* m, int range_pct, uint8_t* const* k0_out);
int nntc_b200_snap_level0_on_grid(nntc_b200_device* d, const nntc_b200_model* m, uint8_t* const* k0_out);
int nntc_b200_stencil_monomials(int c0);

/* ---- block (a): src/solve_decoder.cu:267-458. m->dec_w / dec_b / has_decoder are read and written. ---- */
int nntc_b200_solve_decoder(nntc_b200_device* d, nntc_b200_model* m, int k, const double* per_site, double* ms);
void nntc_b200_decoder_ridge_tally(long long out[4]);

/* ---- blocks (b) and (c'): src/solve_level1.cu:1222-1449. rep holds m->nplanes entries. ---- */
int nntc_b200_solve_level1_all(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge,
                               nntc_b200_plane_report* rep, double* ms);
int nntc_b200_sweep_level1_all(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge, int sweeps,
                               nntc_b200_plane_report* rep, double* ms);
int nntc_b200_solve_level0_cont_all(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge,
                                    nntc_b200_plane_report* rep, double* ms);
int nntc_b200_sweep_level0_cont_all(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge, int sweeps,
                                    nntc_b200_plane_report* rep, double* ms);
int nntc_b200_assemble_level0_for_refine(nntc_b200_device* d, const nntc_b200_model* m, int k, double* ms);

/* ---- transfers: src/solve_level1.cu:1098-1500, src/solve_level0.cu:329-369. A size that does not match the plane
 * is silently ignored on upload, as the reference's uploads do (src/solve_level1.cu:1478-1479). ---- */
int nntc_b200_level1_download_indices(nntc_b200_device* d, int plane, uint8_t* k1, size_t n);
int nntc_b200_level1_upload(nntc_b200_device* d, int plane, const float* v1, size_t n);
int nntc_b200_level1_upload_indices(nntc_b200_device* d, int plane, const uint8_t* k1, size_t n);
int nntc_b200_level0_upload_indices(nntc_b200_device* d, int plane, const uint8_t* k0, size_t n);
int nntc_b200_upload_decoder(nntc_b200_device* d, const nntc_b200_model* m);
int nntc_b200_upload_grids(nntc_b200_device* d, const nntc_b200_model* m);
int nntc_b200_level1_download(nntc_b200_device* d, int plane, float* v1, size_t n);
int nntc_b200_level1_delta(nntc_b200_device* d, int plane, double* delta, size_t n);
int nntc_b200_level1_poke(nntc_b200_device* d, int plane, size_t index, float value);
int nntc_b200_level1_range(nntc_b200_device* d, int plane, float* lo, float* hi);
int nntc_b200_solve_level1_dense_host(nntc_b200_device* d, const nntc_b200_model* m, int k, int plane, double lambda,
                                      const float* c_prev, size_t n_prev, double* delta, int max_unknowns);
int nntc_b200_level0_download(nntc_b200_device* d, int plane, uint8_t* k0, size_t n);
int nntc_b200_level0_upload(nntc_b200_device* d, int plane, const float* v0, size_t n);
int nntc_b200_level0_download_values(nntc_b200_device* d, int plane, float* v0, size_t n);

/* ---- block (c), palette mode: src/solve_level0.cu:275-327. k0 host mirror written per plane. ---- */
int nntc_b200_solve_level0_all(nntc_b200_device* d, const nntc_b200_model* m, int k, int sweeps,
                               nntc_b200_level0_report* rep, double* ms);

/* ---- the objective and the decode: src/objective.cu:53-380 ---- */
int nntc_b200_decode_plane(nntc_b200_device* d, const nntc_b200_model* m, int plane, uint8_t* rgb8, size_t n);
int nntc_b200_objective_eval(nntc_b200_device* d, const nntc_b200_model* m, int k, const double* per_site,
                             nntc_b200_objective* r);
double nntc_b200_objective_total_ms(void);
long long nntc_b200_objective_passes(void);
int nntc_b200_objective_check_host(nntc_b200_device* d, const nntc_b200_model* m, int k, const double* per_site,
                                   nntc_b200_objective* r);

/* The objective of ONE plane held in the caller's own device memory, with no device allocation. This entry point has
 * no counterpart in the reference: it serves a host that manages its plane buffers itself (a device model of its own,
 * or memory committed to its own arena) and cannot afford nntc_b200_device_create's encode workspace or a cudaMalloc.
 * Every pointer is device memory of the current device (or managed memory): v0 (w0 h0 c0), v1 (w1 h1 c1), src
 * (w0 h0 nout), weights (nout x nin, row-major), bias (nout), cw (nout), and sums (3 doubles, written, need not start
 * at zero): the cw-weighted sum over the 1 + k sites of every pixel, the unweighted centre-site sum and the unweighted
 * sum over the k fractional sites - the three raw sums nntc_b200_objective_eval keeps per plane before it normalises
 * them (e_plane = sums[0] / (sum cw (1 + k) w0 h0)). Both kernels are queued on `stream` (a cudaStream_t; 0 is the
 * legacy default stream) and the call returns without waiting. The only scratch is a fixed static device array of
 * 1.5 MiB, hence the limit of NNTC_B200_NOALLOC_MAX_PIXELS pixels per call; a larger plane is rejected with
 * NNTC_B200_ERR_ARG and a message naming the limit. Every call looks up the scratch's address on the current device
 * (cudaGetSymbolAddress, which allocates nothing); the first call on a device also loads the library's device code
 * there, so it should come before any stream capture.
 * Calls in flight at the same time on one device (different streams, or host threads without ordering) share that
 * scratch and race: order them, e.g. on one stream. */
#define NNTC_B200_NOALLOC_MAX_PIXELS (4096LL * 4096LL)
int nntc_b200_objective_plane_noalloc(const float* v0, int w0, int h0, int c0, const float* v1, int w1, int h1,
                                      int c1, const float* src, int nout, const float* weights, const float* bias,
                                      const float* cw, int nin, int k, double* sums, void* stream);

/* ---- the BC refinement: src/refine_bc.cu:504-644. ep / sel are per-plane buffers of blocks*C0*2 and blocks*C0*16
 * bytes (block-major, then channel), exactly as the reference holds them. k0_host is the model's k0 mirror (what
 * the seed pack reads, src/export.cpp:294-328). ---- */
int nntc_b200_bc_pack_prepare(nntc_b200_device* d, const nntc_b200_model* m, int k, int seed,
                              const uint8_t* const* k0_host, double* ms);
int nntc_b200_bc_refine(nntc_b200_device* d, const nntc_b200_model* m, int passes, nntc_b200_bc_report* rep,
                        double* ms);
int nntc_b200_bc_state_save(nntc_b200_device* d, const nntc_b200_model* m, uint8_t* const* ep, uint8_t* const* sel);
int nntc_b200_bc_state_restore(nntc_b200_device* d, const nntc_b200_model* m, const uint8_t* const* ep,
                               const uint8_t* const* sel);
/* The .dds block bytes of one plane from ep/sel (src/export.cpp:333-370, shared/bc_pack.h:74-85), and the pack's
 * squared error in byte units against k0's exact index values, ADDED to *se and *n. files[f] holds
 * blocks * (nc == 1 ? 8 : 16) bytes for file f (one file for 1-2 channels, two for 3-4). */
int nntc_b200_bc_pack_blocks(const nntc_b200_model* m, int plane, const uint8_t* ep, const uint8_t* sel,
                             const uint8_t* k0, uint8_t* const* files, double* se, size_t* n);

/* ---- the whole encode: the caller of the hot path (src/main.cpp:1930-2743, the round loop and the post-fit BC path,
 * with the reference's defaults, src/options.h:82-163) ---- */
typedef struct nntc_b200_encode_args
{
    int k;                 /* subtexel sites per texel (--k 4) */
    int rounds;            /* --rounds 20 */
    double tol;            /* --tol 1e-4 */
    int q1_start;          /* --q1-start 3 */
    int q1_sweeps;         /* --q1-sweeps 4 */
    int range_pct;         /* --q1-range pct (1) or minmax (0) */
    double ridge;          /* --ridge 1e-4 */
    int sweeps;            /* --sweeps 2 (palette mode) */
    int init_pca;          /* --init pca (1) or box (0) */
    int bc_refine;         /* --bc-refine 4 */
    int bc_refine_after;   /* --bc-refine-after 0 */
    int bc_outer;          /* --bc-outer 2 */
    float luma[3];         /* 0.299, 0.587, 0.114 */
    /* 0: the plain form, the reference's arithmetic (FP64 stencils and sums). 1: the adjoint + mixed-precision form:
     * block (a)'s sums on the tensor cores (NNTC_B200_OPT_MIXED_PRECISION_GRAM), the objective's decode in FP32
     * (NNTC_B200_OPT_MIXED_OBJECTIVE), the stencils of blocks (b) and (c') assembled and applied in FP32
     * (NNTC_B200_OPT_FP32_STENCIL; the conjugate gradients then stop at 1e-6 of the right-hand side), and after the
     * repack passes one joint latent / decoder pass (bc8) along the objective's gradient from the decode's adjoint: a
     * step of both latents along their preconditioned gradients with the decoder re-solved, the best of three step
     * lengths, re-packed and refined, kept only when the shipped E falls. The matrix-free products of the conjugate
     * gradients (NNTC_B200_OPT_ADJOINT_CG) are not part of it: on the B200 they cost several times an FP32 stencil
     * product. Has no counterpart in the reference. */
    int form;
} nntc_b200_encode_args;

typedef struct nntc_b200_encode_result
{
    int rounds_used;
    int stop;              /* 0 budget, 1 no-move, 2 tol */
    int outer_taken;
    double e_init, e_after_rounds, e_ship;         /* the objective before block (a), after the loop, shipped */
    double centre_mse, sampled_mse;
    double psnr[6];        /* per texture: 8-bit decode at the base plane's texel centres vs the source bytes */
    double ms_a, ms_b, ms_c, ms_e, ms_pack, ms_refine, ms_total;   /* CUDA-event spans of each kind of block */
    long long objective_passes;
    int joint_taken;       /* form 1: 1 the joint pass was kept (the shipped E fell, no texture's base PSNR fell by
                              more than 0.01 dB), 0 refused (E did not fall), -1 refused by the PSNR guard */
    double e_before_joint; /* form 1: the shipped E the joint pass started from (0 when it did not run) */
    double e_joint;        /* form 1: the shipped E the joint pass reached, kept or not (0 when it did not run) */
    double ms_joint;       /* form 1: the joint pass's span */
} nntc_b200_encode_result;

void nntc_b200_encode_defaults(nntc_b200_encode_args* a);
/* The encode on a device model whose source chain is already resident (device_create). m carries the layout and is
 * reset to the start state; on return it holds the fitted decoder and grids. k0 / k1 (per plane, optional) receive the
 * final indices; ep / sel (per plane, optional, bc8) the final endpoints and selectors. */
int nntc_b200_encode_on_device(nntc_b200_device* d, nntc_b200_model* m, const nntc_b200_encode_args* a,
                               const double* per_site, nntc_b200_encode_result* r, uint8_t* const* k0,
                               uint8_t* const* k1, uint8_t* const* ep, uint8_t* const* sel);

/* The gradient of the objective E (the normalised E of nntc_b200_objective_eval) at the current state, with respect to
 * every level-1 value (g_v1[i]: w1 h1 c1 doubles per plane), every level-0 value (g_v0[i]: w0 h0 c0 doubles per
 * plane; bc8 only, else pass null) and the decoder (g_dec: nout rows of [dE/dW_c (nin) | dE/db_c]), from one pass of
 * the decode's adjoint: the latents' parts are the assembly's J^T diag(cw) r gathered per texel, the decoder's part
 * 2 cw_c (A x_c - rhs_c) from the normal equations at the current latents. No counterpart in the reference (its
 * gradients live inside its stencil assembly and are not exposed). */
int nntc_b200_objective_gradient(nntc_b200_device* d, const nntc_b200_model* m, int k, const double* per_site,
                                 double* const* g_v0, double* const* g_v1, double* g_dec);

/* ---- kernel-shape options: the results are the same bits either way ---- */
enum nntc_b200_option
{
    /* 1: assemble the stencils with one thread per texel recomputing every site it touches, the reference's shape
     * (src/solve_level1.cu:259-581); 0 (default): one pass per site for the gradient terms, then one thread per
     * (texel, slot) for the monomial sums. */
    NNTC_B200_OPT_REFERENCE_SHAPED_ASSEMBLY = 0,
    /* 1: block (a)'s normal equations on the tcgen05 tensor cores with the site rows split into BF16 hi + lo parts
     * and FP32 accumulators, added in FP64 per 256 sites (the mixed-precision form; NOT the same bits: the sums hold
     * to about 1e-6 relative); 0 (default): exact products summed in FP64 (src/solve_decoder.cu:87-161). */
    NNTC_B200_OPT_MIXED_PRECISION_GRAM = 1,
    /* 1: the conjugate gradients of blocks (b) and (c') apply (H + lambda I) matrix-free from the decode's forward pass
     * and its adjoint in FP32, with FP64 inner products and recurrences, and stop at 1e-6 of the right-hand side; only
     * the gradient and the diagonal blocks are assembled (the adjoint form; NOT the same bits). 0 (default): the
     * assembled FP64 stencil (src/solve_level1.cu:781-828, 1222-1338). The quantised sweeps assemble in full either way. */
    NNTC_B200_OPT_ADJOINT_CG = 2,
    /* 1: the objective's per-site decode in FP32 (the assembly's float tap rule and float targets) with every
     * residual's square summed in FP64 (the adjoint form; E to about 1e-7 relative). 0 (default): the decode in FP64 on
     * the double u-space sampling rule (src/objective.cu:97-211). */
    NNTC_B200_OPT_MIXED_OBJECTIVE = 3,
    /* 1: blocks (b) and (c') assemble their stencils in FP32 (the gathers' sums and the stored blocks), which the
     * quantised sweeps then read at half the bytes; the BC refinement's assembly stays FP64 (the adjoint form). 0
     * (default): FP64, the reference's bits (src/solve_level1.cu:259-581). */
    NNTC_B200_OPT_FP32_STENCIL = 4
};
int nntc_b200_set_option(nntc_b200_device* d, int option, int value);

/* ---- measurement ---- */
/* Kernels this library has launched since the process started (every launch, every device). */
long long nntc_b200_launch_count(void);
/* The hot kernels whose launches can be timed individually with CUDA events on the library's own stream. */
enum nntc_b200_kernel
{
    NNTC_B200_K_OBJECTIVE = 0,   /* the objective over every site of every plane */
    NNTC_B200_K_NORMAL_EQ,       /* block (a)'s normal equations */
    NNTC_B200_K_ASSEMBLE1,       /* block (b)'s stencil and gradient gather */
    NNTC_B200_K_ASSEMBLE0,       /* block (c')'s stencil and gradient gather */
    NNTC_B200_K_MATVEC,          /* one conjugate-gradient product over every plane, block (b) (level 1) */
    NNTC_B200_K_SWEEP,           /* one colour of the quantised sweeps */
    NNTC_B200_K_REFINE,          /* one colour of the BC refinement */
    NNTC_B200_K_MATVEC0,         /* one conjugate-gradient product over every plane, block (c') (level 0) */
    NNTC_B200_K_COUNT
};
/* The measured fused-multiply-add peaks of the current device's FP64 and FP32 vector pipes, in TFLOP/s (2 flops per
 * FMA): eight independent chains per thread, four blocks per SM, timed with CUDA events. No counterpart in the
 * reference; the denominators of the compute fractions the benchmark reports for pipe-bound kernels. */
int nntc_b200_measure_fma_peaks(double* fp64_tflops, double* fp32_tflops);
/* on != 0 brackets every launch of the kernels above with a pair of CUDA events; stats accumulate until reset. */
int nntc_b200_kernel_timing(nntc_b200_device* d, int on);
/* The launches of `kernel` since the last reset and their summed event time; reset != 0 clears every kernel's. */
int nntc_b200_kernel_stats(nntc_b200_device* d, int kernel, long long* launches, double* ms, int reset);

/* ---- the asset on disk (src/export.cpp:89-146 dds_write, 470-812 write_asset; the layout of docs/FORMAT.md) ----
 * Writes PREFIX_lat0.dds (PREFIX_lat0a.dds and PREFIX_lat0b.dds for a block-compressed level 0 of three or four
 * channels), PREFIX_lat1.dds and the JSON descriptor at json_path (PREFIX_nntc.json when null), all from host memory.
 * Per plane i of the chain, the base first: k1[i] holds level 1's indices (w1 h1 c1 bytes); for a block-compressed level
 * 0 (m->bc0) ep[i] and sel[i] hold the blocks the refinement chose (blocks c0 2 and blocks c0 16 bytes, the layout
 * nntc_b200_bc_state_save returns) and are written as they stand, or, when null, k0[i] (w0 h0 c0 bytes) is packed by the
 * seed pack; an uncompressed level 0 writes k0[i] (under bc8 that is the reference's uncompressed twin, --bc0 both). m supplies the extents, bits, grids and decoder. source_width and
 * source_height are the extent before any padding. sizes (three entries, or null) receives the bytes written for level
 * 0's file(s), level 1's file and the descriptor. Refuses (NNTC_B200_ERR_ARG, nothing written) a non-finite decoder or
 * grid and a level-1 index that does not read back as itself on its published grid; NNTC_B200_ERR_IO on a failed write. */
int nntc_b200_write_asset(const nntc_b200_model* m, const uint8_t* const* k0, const uint8_t* const* k1,
                          const uint8_t* const* ep, const uint8_t* const* sel, int source_width, int source_height,
                          const char* prefix, const char* json_path, size_t* sizes);

/* ---- probes: what the reference's per-kernel harness reads (src/backend_check_probe.h:20-37) ---- */
int nntc_b200_probe_normal_equations(nntc_b200_device* d, double* out, size_t n);
int nntc_b200_probe_workspace(nntc_b200_device* d, int plane, int level0, double* stencil, double* grad,
                              float* precond, double* cg_x, float* prev);
int nntc_b200_probe_monomials(nntc_b200_device* d, int level0, double* out, size_t n);
int nntc_b200_probe_source(nntc_b200_device* d, int plane, float* out, size_t n);   /* plane's source, HWC */
/* y = H x for block (b)'s Gauss-Newton operator on one plane, applied matrix-free from the decode and its adjoint (the
 * product the assembled stencil of src/solve_level1.cu:259-438 gives, to rounding). x and y: w1 h1 c1 doubles. Uses the
 * plane's CG vectors as scratch. */
int nntc_b200_probe_jtj_level1(nntc_b200_device* d, int k, int plane, const double* x, double* y, size_t n);
/* The same for block (c')'s operator over level 0 (src/solve_level1.cu:440-581): x and y w0 h0 c0 doubles; bc8 only. */
int nntc_b200_probe_jtj_level0(nntc_b200_device* d, int k, int plane, const double* x, double* y, size_t n);
/* The adjoint form's round-closing pass (no counterpart in the reference, whose objective and normal equations are
 * separate passes): block (a)'s normal equations on the tensor cores (left where nntc_b200_probe_normal_equations reads
 * them) and E of the uploaded decoder at the same sites, in one pass. Needs NNTC_B200_OPT_MIXED_PRECISION_GRAM on. */
int nntc_b200_probe_objective_with_normal_equations(nntc_b200_device* d, const nntc_b200_model* m, int k,
                                                    const double* per_site, nntc_b200_objective* r);

#ifdef __cplusplus
}
#endif

#endif /* NNTC_B200_H */
