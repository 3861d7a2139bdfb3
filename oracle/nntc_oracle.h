/* nntc_oracle.h: a plain-C restatement of the NNTC encoder's hot path, for checking the CUDA path.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product links, loads or calls this; the parity tests, smoke() and the
 * benchmark's CPU-baseline leg do. Every function is serial, single-threaded C over plain arrays, in the order of
 * operations of the reference file and line it cites. It is pinned against the reference itself: the golden vectors
 * under tests/golden/ were produced by the reference's own CPU arm (oracle/ref_shim.cpp over src/cpu/*.cpp) and
 * tests/test_oracle_golden.py checks this restatement against every one of them.
 *
 * Layouts are the reference's: planes interleaved [texel][channel]; the stencil [texel][slot][i][j] with the slots
 * self, right, down-left, down, down-right; the decoder row-major nout x nin.
 */
#ifndef NNTC_ORACLE_H
#define NNTC_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One stored level of the chain. */
typedef struct orc_plane
{
    int w0, h0, w1, h1;
    const float* src; /* w0 h0 nout */
    float* v0;        /* w0 h0 c0 */
    float* v1;        /* w1 h1 c1 */
} orc_plane;

typedef struct orc_decoder
{
    int c0, c1, nin, nout, k;
    const float* w;   /* nout x nin */
    const float* b;   /* nout */
    const float* cw;  /* nout */
} orc_decoder;

/* src/model.h:141-199 */
int orc_rep_index(int k, int bits);
float orc_grid_value(float lo, float hi, int bits, int k);
int orc_grid_index(float lo, float hi, int bits, float value);

/* src/objective.cu:317-380: the three raw sums of one plane (weighted, centre, fractional), site by site. */
void orc_objective_plane(const orc_plane* p, const orc_decoder* d, double out[3]);
/* src/objective.cu:53-75 */
void orc_decode_plane(const orc_plane* p, const orc_decoder* d, uint8_t* rgb8);

/* src/solve_decoder.cu:87-161: one plane's unweighted normal equations (upper triangle of A, then nout rhs rows). */
void orc_normal_equations_plane(const orc_plane* p, const orc_decoder* d, double* entries);
/* src/solve_decoder.cu:184-458: the ridge ladder on the weighted sums. w / b in-out; returns the rung (3 = refused). */
int orc_decoder_solve(const double* acc, int nin, int nout, const float* cw, double inv_norm, int norm_ok,
                      int had_previous, float* w, float* b);

/* src/solve_level1.cu:164-244: the monomial matrices of block (b) (level0 = 0) or block (c') (level0 = 1). */
int orc_monomials(const orc_decoder* d, int level0, double* out);
/* src/solve_level1.cu:259-581: the stencil [texel][5][c][c] and gradient [texel][c] of the unknown latent. */
void orc_assemble(const orc_plane* p, const orc_decoder* d, int level0, const double* mono, double* stencil,
                  double* grad);
/* src/solve_level1.cu:625-687: sum, min, max of diag(H) and lambda = ridge mean(diag). out[4]. */
void orc_diag(const double* stencil, size_t texels, int c, double ridge, double out[4]);
/* src/solve_level1.cu:689-878, 1222-1338: block-Jacobi PCG on (H + lambda I) x = -grad from x = 0, with the probe
 * rule (stop at a multiple of 4 iterations once |r|/|rhs| < 1e-10, at most 200). Returns the iterations. */
int orc_pcg(const double* stencil, const double* grad, int w, int h, int c, double lambda, double* x,
            double* resid);
/* src/solve_level1.cu:1023-1098, 1343-1403: `sweeps` four-colour quantised Gauss-Seidel sweeps from x = 0 at prev.
 * v, k, x updated in place; returns the index changes. */
long long orc_quant_sweeps(const double* stencil, const double* grad, const float* prev, int w, int h, int c,
                           double lambda, const float* lo, const float* hi, int bits, int sweeps, double* x, float* v,
                           uint8_t* k);

/* shared/bc_pack.h:95-166 over src/export.cpp:294-328: the seed endpoints and selectors of one plane. */
void orc_bc_seed(const uint8_t* k0, int w0, int h0, int c0, const int* bits, uint8_t* ep, uint8_t* sel);
/* src/refine_bc.cu:155-174 */
void orc_bc_decode(const uint8_t* ep, const uint8_t* sel, const float* lo0, const float* hi0, int w0, int h0, int c0,
                   const float* prev, float* v0, uint8_t* k0, double* delta);
/* src/cpu/cpu_refine_bc.cpp:134-400: one colour pass of the refinement over one plane. Returns the accepted
 * decrease; *improved counts the blocks that took one. */
double orc_bc_refine_colour(const double* stencil, const double* grad, const float* prev, const float* lo0,
                            const float* hi0, int w0, int h0, int c0, int colour, uint8_t* ep, uint8_t* sel,
                            double* delta, float* v0, uint8_t* k0, long long* improved);

/* src/init.cu:484-517, 838-872 */
void orc_init_level1_box(const float* src, int w0, int h0, int nout, int w1, int h1, int c1, float* out);
/* src/init.cu:1034-1055 */
void orc_residual(const orc_plane* p, const orc_decoder* d, float* resid);

#ifdef __cplusplus
}
#endif

#endif
