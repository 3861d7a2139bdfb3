// common.cuh: what every kernel file of the B200 encoder shares.
//
// - the status plumbing of the C ABI (a thread-local message, CUDA calls checked into an int status);
// - the sampling rule and the site set (the reference's src/sample.cuh:43-178), the grid arithmetic
//   (src/model.h:141-199) and the stencil's slot table (src/device.cuh:99-126), restated for this library;
// - the multi-plane descriptor: every mip plane of the chain is described in one struct passed BY VALUE as a kernel
//   parameter, so one launch covers every plane (the reference issues one launch per plane on its own stream,
//   src/device.cuh:378-411; with 148 SMs the deep planes are a few blocks each and cost only their launches).
//
// Arithmetic that the reference evaluates without FMA contraction (its CUDA build uses -fmad=false,
// CMakeLists.txt:183-186, and its CPU twin -ffp-contract=off) is compiled here with -fmad=false too, so a per-texel
// or per-site value is the same bits as the reference's given the same inputs. Kernels that WANT fused
// multiply-adds (the mixed-precision paths) spell them with __fmaf_rn / __fma_rn explicitly.
#pragma once

#include <cstdint>
#include <cstdio>
#include <string>

#include <cuda_runtime.h>

#include "nntc_b200.h"

namespace nb
{

constexpr int MAX_PLANES = NNTC_B200_MAX_PLANES;
constexpr int MAX_CH = NNTC_B200_MAX_CHANNELS;
constexpr int MAX_NIN = NNTC_B200_MAX_NIN;
constexpr int MAX_NOUT = NNTC_B200_MAX_NOUT;
constexpr int SLOTS = 5;          // owned stencil blocks per texel: self, right, down-left, down, down-right
constexpr int MAX_MONO = 15;      // 1 + C + C (C + 1) / 2 at C = 4
constexpr int CG_PROBE = 4;       // the host looks at the residual every 4th iteration (src/solve_level1.cu:99)
// The stop of conjugate gradients whose products are FP32 (the matrix-free operator, or an FP32 stencil: about 1e-7
// relative): the recursive residual is taken down to 1e-7 of the right-hand side, where the FP64 stencil form goes
// on to 1e-10 (at 1e-6 the correction of a converged level-0 state differed from the FP64 form's by 1.3e-4 of its
// largest entry, above the 1e-4 the form is held to).
constexpr double CG_TOL_FP32 = 1e-7;
constexpr int CG_MAX_IT = 200;    // src/solve_level1.cu:1261
constexpr double CG_TOL = 1e-10;  // src/solve_level1.cu:1257

// ---- status ------------------------------------------------------------------------------------------------------

void set_error(int status, const std::string& msg);
int cuda_status(cudaError_t err, const char* call, const char* file, int line);

#define NB_CUDA(call)                                                                                                 \
    do                                                                                                                \
    {                                                                                                                 \
        const cudaError_t nb_err_ = (call);                                                                           \
        if (nb_err_ != cudaSuccess)                                                                                   \
            return ::nb::cuda_status(nb_err_, #call, __FILE__, __LINE__);                                            \
    } while (0)

#define NB_TRY(expr)                                                                                                  \
    do                                                                                                                \
    {                                                                                                                 \
        const int nb_st_ = (expr);                                                                                    \
        if (nb_st_ != NNTC_B200_OK)                                                                                   \
            return nb_st_;                                                                                            \
    } while (0)

// Every kernel launch is followed by this: it counts the launch (nntc_b200_launch_count) and checks it.
void count_launch();
#define NB_LAUNCHED()                                                                                                 \
    do                                                                                                                \
    {                                                                                                                 \
        ::nb::count_launch();                                                                                         \
        NB_CUDA(cudaGetLastError());                                                                                  \
    } while (0)

inline int grid_for(size_t n, int threads)
{
    return (int)((n + (size_t)threads - 1) / (size_t)threads);
}

// ---- the sampling rule (src/sample.cuh:43-71) ----------------------------------------------------------------------

struct Tap
{
    int x0, x1, y0, y1;
    float fx, fy;
};

__host__ __device__ __forceinline__ int clampi(int i, int n)
{
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

// A site is pixel (px, py) of a w0 x h0 plane plus an offset (dx, dy) in that plane's pixels; its position in a w x h
// plane is the exact pixel coordinate scaled by w / w0 (exactly the pixel itself when w == w0), and the two taps per
// axis are floor and floor + 1, clamped.
__host__ __device__ __forceinline__ Tap tap_at(int px, int py, float dx, float dy, int w0, int h0, int w, int h)
{
    const float x = w == w0 ? (float)px + dx : (((float)px + 0.5f + dx) * (float)w) / (float)w0 - 0.5f;
    const float y = h == h0 ? (float)py + dy : (((float)py + 0.5f + dy) * (float)h) / (float)h0 - 0.5f;
    const int xf = (int)floorf(x), yf = (int)floorf(y);
    Tap t;
    t.fx = x - (float)xf;
    t.fy = y - (float)yf;
    t.x0 = clampi(xf, w);
    t.x1 = clampi(xf + 1, w);
    t.y0 = clampi(yf, h);
    t.y1 = clampi(yf + 1, h);
    return t;
}

// The four corner weights in the order (x0,y0), (x1,y0), (x0,y1), (x1,y1).
__host__ __device__ __forceinline__ void tap_weights(const Tap& t, float w[4])
{
    w[0] = (1.0f - t.fx) * (1.0f - t.fy);
    w[1] = t.fx * (1.0f - t.fy);
    w[2] = (1.0f - t.fx) * t.fy;
    w[3] = t.fx * t.fy;
}

template <int MAXC>
__host__ __device__ __forceinline__ void blend(const float* plane, int w, int c, const Tap& t, float* out)
{
    const float* a = plane + ((size_t)t.y0 * w + t.x0) * c;
    const float* b = plane + ((size_t)t.y0 * w + t.x1) * c;
    const float* e = plane + ((size_t)t.y1 * w + t.x0) * c;
    const float* f = plane + ((size_t)t.y1 * w + t.x1) * c;
    float wt[4];
    tap_weights(t, wt);
    for (int k = 0; k < c; k++)
        out[k] = wt[0] * a[k] + wt[1] * b[k] + wt[2] * e[k] + wt[3] * f[k];
}

// blend() with the channel loop unrolled to MAXC and guarded, so `out` stays in registers; the same arithmetic.
template <int MAXC>
__device__ __forceinline__ void blend_u(const float* plane, int w, int c, const Tap& t, float* out)
{
    const float* a = plane + ((size_t)t.y0 * w + t.x0) * c;
    const float* b = plane + ((size_t)t.y0 * w + t.x1) * c;
    const float* e = plane + ((size_t)t.y1 * w + t.x0) * c;
    const float* f = plane + ((size_t)t.y1 * w + t.x1) * c;
    float wt[4];
    tap_weights(t, wt);
#pragma unroll
    for (int k = 0; k < MAXC; k++)
        if (k < c)
            out[k] = wt[0] * __ldg(a + k) + wt[1] * __ldg(b + k) + wt[2] * __ldg(e + k) + wt[3] * __ldg(f + k);
}

// phi in the shader's order: [c_j] [s_i] [s_i c_j], i outer (src/sample.cuh:74-85).
template <typename T>
__host__ __device__ __forceinline__ int features(const T* s, int c0, const T* c, int c1, T* phi)
{
    int k = 0;
    for (int j = 0; j < c1; j++)
        phi[k++] = c[j];
    for (int i = 0; i < c0; i++)
        phi[k++] = s[i];
    for (int i = 0; i < c0; i++)
        for (int j = 0; j < c1; j++)
            phi[k++] = s[i] * c[j];
    return k;
}

// The fixed subtexel offsets (src/sample.cuh:112-137): the rotated grid of four at K = 4, turned a quarter turn per
// texel parity class; the diagonal pair at K = 2; (1/4, 1/4) turned per texel at K = 1.
__host__ __device__ __forceinline__ void subtexel(int kc, int j, int tx, int ty, float& dx, float& dy)
{
    if (kc == 2)
    {
        dx = j == 0 ? -0.25f : 0.25f;
        dy = j == 0 ? 0.25f : -0.25f;
        return;
    }
    float ox = 0.25f, oy = 0.25f;
    if (kc == 4)
    {
        // the four offsets {(-3/8, -1/8), (-1/8, 3/8), (1/8, -3/8), (3/8, 1/8)}, selected rather than indexed so that
        // a runtime j stays in registers
        ox = j == 0 ? -0.375f : (j == 1 ? -0.125f : (j == 2 ? 0.125f : 0.375f));
        oy = j == 0 ? -0.125f : (j == 1 ? 0.375f : (j == 2 ? -0.375f : 0.125f));
    }
    const int turns = (ty & 1) * 2 + (tx & 1);
    for (int r = 0; r < turns; r++)
    {
        const float t = ox;
        ox = -oy;
        oy = t;
    }
    dx = ox;
    dy = oy;
}

// Site j of a pixel: 0 the centre, 1..K the fractional sites.
__host__ __device__ __forceinline__ void site_offset(int kc, int j, int px, int py, float& dx, float& dy)
{
    dx = 0.0f;
    dy = 0.0f;
    if (j > 0)
        subtexel(kc, j - 1, px, py, dx, dy);
}

// ---- grid arithmetic (src/model.h:141-199) ------------------------------------------------------------------------

__host__ __device__ __forceinline__ int rep_index(int k, int bits)
{
    unsigned b8 = 0;
    for (int sh = 8 - bits; sh > -bits; sh -= bits)
        b8 |= sh >= 0 ? ((unsigned)k << sh) : ((unsigned)k >> -sh);
    return (int)(b8 & 0xFFu);
}

// value = lo + rep(k) / 255 * (hi - lo), in double, the multiply and the add rounded separately, then to float.
__host__ __device__ __forceinline__ float grid_value(float lo, float hi, int bits, int k)
{
    const double span = (double)hi - (double)lo;
    const double frac = (double)rep_index(k, bits) / 255.0;
#ifdef __CUDA_ARCH__
    return (float)__dadd_rn((double)lo, __dmul_rn(frac, span));
#else
    return (float)((double)lo + frac * span);
#endif
}

// The index whose grid VALUE is nearest; a tie keeps the lower index.
__host__ __device__ __forceinline__ int grid_index(float lo, float hi, int bits, float value)
{
    const double span = (double)hi - (double)lo;
    const int levels = (1 << bits) - 1;
    if (!(span > 0.0))
        return 0;
    double x = ((double)value - (double)lo) / span * (double)levels;
    x = x < 0.0 ? 0.0 : (x > (double)levels ? (double)levels : x);
    int k = (int)(x + 0.5);
    k = k < 0 ? 0 : (k > levels ? levels : k);
    int best = k;
    double best_d = fabs((double)value - (double)grid_value(lo, hi, bits, k));
    for (int d = -1; d <= 1; d += 2)
    {
        const int n = k + d;
        if (n < 0 || n > levels)
            continue;
        const double dist = fabs((double)value - (double)grid_value(lo, hi, bits, n));
        if (dist < best_d || (dist == best_d && n < best))
        {
            best_d = dist;
            best = n;
        }
    }
    return best;
}

// ---- the 9-point stencil's owned slots (src/device.cuh:99-126) -----------------------------------------------------

__host__ __device__ __forceinline__ void slot_offset(int slot, int& dx, int& dy)
{
    // self, right, down-left, down, down-right
    dx = slot == 0 ? 0 : (slot == 1 ? 1 : (slot == 2 ? -1 : (slot == 3 ? 0 : 1)));
    dy = slot <= 1 ? 0 : 1;
}

// Where texel (x, y) of a w x h plane sits in the stencil's texel order. The order is colour-major: the four colours of
// the quantised sweeps, (x & 1) + 2 (y & 1) in sweep order, one after another, each row-major. A sweep over one colour
// then reads each of its stencil planes as one contiguous run instead of every other double, which halves the DRAM
// sectors it touches; a row-major walk over all texels still reads two contiguous runs per warp.
__host__ __device__ __forceinline__ size_t stencil_pos(int x, int y, int w, int h)
{
    const size_t w0c = (size_t)(w + 1) >> 1, w1c = (size_t)w >> 1;   // texels per row of x parity 0 / 1
    const size_t h0c = (size_t)(h + 1) >> 1, h1c = (size_t)h >> 1;   // rows of y parity 0 / 1
    const int cx = x & 1, cy = y & 1;
    size_t base = cy ? (w0c + w1c) * h0c : 0;
    if (cx)
        base += cy ? w0c * h1c : w0c * h0c;
    return base + (size_t)(y >> 1) * (cx ? w1c : w0c) + (size_t)(x >> 1);
}

// Where coefficient e (= i C + j) of owned slot `slot` of the texel at stencil position sp sits in a stored stencil of
// T texels. FP64 (the plain form): structure of arrays, [slot][e][texel], one plane per coefficient. FP32 (the adjoint
// form): [slot][texel][e], a texel's C x C block of one slot contiguous, so a thread reads a block as whole 16-byte
// vectors and a warp's 32 blocks as one contiguous run.
template <typename TS>
__host__ __device__ __forceinline__ size_t sten_index(int slot, int e, int cc, size_t T, size_t sp)
{
    return sizeof(TS) == sizeof(double) ? (size_t)(slot * cc + e) * T + sp : ((size_t)slot * T + sp) * cc + (size_t)e;
}

// The floor halving of a mip chain, never below one texel (src/image.h:335-338).
__host__ __device__ __forceinline__ int mip_dim(int n)
{
    return n / 2 > 0 ? n / 2 : 1;
}

__host__ __device__ __forceinline__ int slot_of(int dx, int dy)
{
    for (int s = 0; s < SLOTS; s++)
    {
        int ox, oy;
        slot_offset(s, ox, oy);
        if (ox == dx && oy == dy)
            return s;
    }
    return -1;
}

__host__ __device__ __forceinline__ int monomial_count(int c)
{
    return 1 + c + c * (c + 1) / 2;
}

// ---- the multi-plane descriptor ----------------------------------------------------------------------------------

// One stored level as a kernel sees it.
struct PlaneView
{
    int w0, h0, w1, h1;
    const float* src;   // w0 h0 nout
    float* v0;          // w0 h0 c0
    float* v1;          // w1 h1 c1
    uint8_t* k0;
    uint8_t* k1;
    // the unknown of a block (b) / (c') call: level 1 or level 0 of this plane
    int w, h;
    float* v;
    uint8_t* k;
    double* stencil;    // SoA: [slot][c][c][texel]
    double* grad;       // [texel][c]
    float* precond;     // [texel][c][c]
    double* x;          // the correction, [texel][c]
    double* r;
    double* z;
    double* p;
    double* ap;
    float* prev;        // the plane the stencil was assembled at
    double* bc_sten;    // level 0 under bc8: the BC refinement's block-major copy of the FP64 stencil
};

struct Planes
{
    int n;
    int c0, c1, nin, nout, kc;
    int c;              // the unknown's channel count in a block (b)/(c') call
    long long start[MAX_PLANES + 1];   // prefix of the per-plane work items of the launch
    PlaneView p[MAX_PLANES];
};

// The plane that work item i of a launch belongs to (start[] ascending, start[n] the total).
__device__ __forceinline__ int plane_of(const Planes& P, long long i)
{
    int lo = 0;
    while (lo + 1 < P.n && P.start[lo + 1] <= i)
        lo++;
    return lo;
}

}   // namespace nb
