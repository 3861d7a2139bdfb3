// device.cu: the C ABI's status plumbing, the device model's lifecycle and every plain transfer.
//
// Follows src/init.cu:76-382 (device_select, device_create, device_destroy, device_memory) and the transfers of
// src/solve_level1.cu:1098-1500 / src/solve_level0.cu:329-369, over this library's own single-stream model.

#include <algorithm>
#include <atomic>
#include <cstring>
#include <string>
#include <vector>

#include "device.cuh"

namespace nb
{

static thread_local std::string g_error;

void set_error(int status, const std::string& msg)
{
    (void)status;
    g_error = msg;
}

int cuda_status(cudaError_t err, const char* call, const char* file, int line)
{
    const char* base = file;
    for (const char* s = file; *s; s++)
        if (*s == '/' || *s == '\\')
            base = s + 1;
    char buf[1024];
    if (err == cudaErrorMemoryAllocation)
    {
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        snprintf(buf, sizeof(buf),
                 "out of GPU memory in CUDA call %s at %s:%d (%zu/%zu MB free): the material is too large for this "
                 "GPU; try fewer or smaller textures, or fewer latent channels",
                 call, base, line, free_b >> 20, total_b >> 20);
        set_error(NNTC_B200_ERR_OOM, buf);
        return NNTC_B200_ERR_OOM;
    }
    const bool fault = err == cudaErrorIllegalAddress || err == cudaErrorLaunchFailure ||
                       err == cudaErrorIllegalInstruction || err == cudaErrorMisalignedAddress ||
                       err == cudaErrorAssert;
    snprintf(buf, sizeof(buf), "CUDA call %s failed at %s:%d: %s (%s)%s", call, base, line, cudaGetErrorString(err),
             cudaGetErrorName(err),
             fault ? "; a kernel's fault is reported by the first CUDA call that waits for it, so it may have come "
                     "from an earlier launch"
                   : "");
    set_error(NNTC_B200_ERR_CUDA, buf);
    return NNTC_B200_ERR_CUDA;
}

static std::atomic<long long> g_launches{ 0 };

void count_launch()
{
    g_launches.fetch_add(1, std::memory_order_relaxed);
}

int ktimer_begin(nntc_b200_device* d, int kind)
{
    if (!d->ktiming)
        return NNTC_B200_OK;
    cudaEvent_t e[2];
    for (cudaEvent_t& x : e)
    {
        if (d->kpool.empty())
            NB_CUDA(cudaEventCreate(&x));
        else
        {
            x = d->kpool.back();
            d->kpool.pop_back();
        }
    }
    d->kpending.push_back({ kind, e[0], e[1] });
    NB_CUDA(cudaEventRecord(e[0], d->stream));
    return NNTC_B200_OK;
}

int ktimer_end(nntc_b200_device* d)
{
    if (!d->ktiming || d->kpending.empty())
        return NNTC_B200_OK;
    NB_CUDA(cudaEventRecord(d->kpending.back().b, d->stream));
    return NNTC_B200_OK;
}

int ktimer_harvest(nntc_b200_device* d)
{
    for (const nntc_b200_device::Pending& p : d->kpending)
    {
        float t = 0.0f;
        NB_CUDA(cudaEventElapsedTime(&t, p.a, p.b));
        d->klaunches[p.kind]++;
        d->kms[p.kind] += (double)t;
        d->kpool.push_back(p.a);
        d->kpool.push_back(p.b);
    }
    d->kpending.clear();
    return NNTC_B200_OK;
}

int block_begin(nntc_b200_device* d)
{
    NB_CUDA(cudaEventRecord(d->ev[0], d->stream));
    return NNTC_B200_OK;
}

int block_end(nntc_b200_device* d, double* ms)
{
    NB_CUDA(cudaEventRecord(d->ev[1], d->stream));
    NB_CUDA(cudaStreamSynchronize(d->stream));
    float t = 0.0f;
    NB_CUDA(cudaEventElapsedTime(&t, d->ev[0], d->ev[1]));
    if (ms)
        *ms = (double)t;
    return ktimer_harvest(d);
}

int upload(nntc_b200_device* d, void* dst, const void* src, size_t bytes)
{
    if (bytes == 0)
        return NNTC_B200_OK;
    NB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, d->stream));
    NB_CUDA(cudaStreamSynchronize(d->stream));
    return NNTC_B200_OK;
}

int download(nntc_b200_device* d, void* dst, const void* src, size_t bytes)
{
    if (bytes == 0)
        return NNTC_B200_OK;
    NB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, d->stream));
    NB_CUDA(cudaStreamSynchronize(d->stream));
    return NNTC_B200_OK;
}

int check_plane(const nntc_b200_device* d, int plane)
{
    if (!d || plane < 0 || plane >= (int)d->planes.size())
    {
        set_error(NNTC_B200_ERR_ARG, "plane index " + std::to_string(plane) + " is outside the model");
        return NNTC_B200_ERR_ARG;
    }
    return NNTC_B200_OK;
}

int upload_decoder(nntc_b200_device* d, const nntc_b200_model* m)
{
    d->m.has_decoder = m->has_decoder;
    std::memcpy(d->m.dec_w, m->dec_w, sizeof(m->dec_w));
    std::memcpy(d->m.dec_b, m->dec_b, sizeof(m->dec_b));
    // The reference uploads the model's vectors as they are; an empty decoder uploads nothing and the device keeps
    // what it had (src/device.cuh:472-478 with zero bytes).
    if (!m->has_decoder)
        return NNTC_B200_OK;
    NB_TRY(upload(d, d->weights, m->dec_w, (size_t)d->nout * d->nin * sizeof(float)));
    NB_TRY(upload(d, d->bias, m->dec_b, (size_t)d->nout * sizeof(float)));
    std::memcpy(d->host_weights, m->dec_w, (size_t)d->nout * d->nin * sizeof(float));
    std::memcpy(d->host_bias, m->dec_b, (size_t)d->nout * sizeof(float));
    return NNTC_B200_OK;
}

int upload_grids(nntc_b200_device* d, const nntc_b200_model* m)
{
    std::vector<float> pal((size_t)MAX_CH * 16, 0.0f);
    for (int c = 0; c < d->c0; c++)
        for (int k = 0; k < m->palette0_len[c] && k < 16; k++)
            pal[(size_t)c * 16 + k] = m->palette0[c][k];
    NB_TRY(upload(d, d->palette, pal.data(), pal.size() * sizeof(float)));
    float lo[MAX_CH] = {}, hi[MAX_CH] = {};
    if (m->has_lo1)
        for (int c = 0; c < d->c1; c++)
        {
            lo[c] = m->lo1[c];
            hi[c] = m->hi1[c];
        }
    NB_TRY(upload(d, d->lo1, lo, sizeof(lo)));
    NB_TRY(upload(d, d->hi1, hi, sizeof(hi)));
    if (d->lo0)
    {
        float l0[MAX_CH] = {}, h0[MAX_CH] = {};
        if (m->has_lo0)
            for (int c = 0; c < d->c0; c++)
            {
                l0[c] = m->lo0[c];
                h0[c] = m->hi0[c];
            }
        NB_TRY(upload(d, d->lo0, l0, sizeof(l0)));
        NB_TRY(upload(d, d->hi0, h0, sizeof(h0)));
    }
    d->m.has_lo0 = m->has_lo0;
    d->m.has_lo1 = m->has_lo1;
    std::memcpy(d->m.lo0, m->lo0, sizeof(m->lo0));
    std::memcpy(d->m.hi0, m->hi0, sizeof(m->hi0));
    std::memcpy(d->m.lo1, m->lo1, sizeof(m->lo1));
    std::memcpy(d->m.hi1, m->hi1, sizeof(m->hi1));
    std::memcpy(d->m.palette0, m->palette0, sizeof(m->palette0));
    std::memcpy(d->m.palette0_len, m->palette0_len, sizeof(m->palette0_len));
    return NNTC_B200_OK;
}

// X^T C Y products of a form X(y) = X0 + sum_i y_i Y_i, in the monomial order constant, y_i, y_i y_j (i <= j)
// (src/solve_level1.cu:164-204).
static void form_matrices(const nntc_b200_model& m, const std::vector<double>& x0, const std::vector<double>& y,
                          int terms, int dim, std::vector<double>& p)
{
    const int nout = m.nout;
    const int nmono = monomial_count(terms);
    p.assign((size_t)nmono * dim * dim, 0.0);
    auto product = [&](const double* x, const double* z, double* out) {
        for (int u = 0; u < dim; u++)
            for (int v = 0; v < dim; v++)
            {
                double s = 0.0;
                for (int r = 0; r < nout; r++)
                    s += (double)m.cw[r] * x[(size_t)r * dim + u] * z[(size_t)r * dim + v];
                out[u * dim + v] += s;
            }
    };
    int slot = 0;
    product(x0.data(), x0.data(), p.data());
    slot++;
    for (int i = 0; i < terms; i++, slot++)
    {
        const double* yi = y.data() + (size_t)i * nout * dim;
        product(yi, x0.data(), p.data() + (size_t)slot * dim * dim);
        product(x0.data(), yi, p.data() + (size_t)slot * dim * dim);
    }
    for (int i = 0; i < terms; i++)
        for (int j = i; j < terms; j++, slot++)
        {
            const double* yi = y.data() + (size_t)i * nout * dim;
            const double* yj = y.data() + (size_t)j * nout * dim;
            product(yi, yj, p.data() + (size_t)slot * dim * dim);
            if (i != j)
                product(yj, yi, p.data() + (size_t)slot * dim * dim);
        }
}

void build_monomials(const nntc_b200_model& m, int level0, std::vector<double>& p)
{
    const int c0 = m.c0, c1 = m.c1, nout = m.nout, nin = m.nin;
    if (!level0)
    {
        // G(s) = A + sum_i s_i M_i: A the a-block (columns 0..C1-1), M_i the sc-block of channel i.
        std::vector<double> a((size_t)nout * c1), mi((size_t)MAX_CH * nout * c1, 0.0);
        for (int r = 0; r < nout; r++)
        {
            const float* row = m.dec_w + (size_t)r * nin;
            for (int q = 0; q < c1; q++)
                a[(size_t)r * c1 + q] = (double)row[q];
            for (int i = 0; i < c0; i++)
                for (int q = 0; q < c1; q++)
                    mi[((size_t)i * nout + r) * c1 + q] = (double)row[c1 + c0 + i * c1 + q];
        }
        form_matrices(m, a, mi, c0, c1, p);
    }
    else
    {
        // Q(c) = B + sum_q c_q N_q: B the b-block (columns C1..C1+C0-1), column i of N_q is W[:, C1 + C0 + i C1 + q].
        std::vector<double> b((size_t)nout * c0), nq((size_t)MAX_CH * nout * c0, 0.0);
        for (int r = 0; r < nout; r++)
        {
            const float* row = m.dec_w + (size_t)r * nin;
            for (int i = 0; i < c0; i++)
                b[(size_t)r * c0 + i] = (double)row[c1 + i];
            for (int q = 0; q < c1; q++)
                for (int i = 0; i < c0; i++)
                    nq[((size_t)q * nout + r) * c0 + i] = (double)row[c1 + c0 + i * c1 + q];
        }
        form_matrices(m, b, nq, c1, c0, p);
    }
}

}   // namespace nb

using namespace nb;

namespace
{

// Every buffer of the device model is a 256-byte-aligned slice of one device allocation, the arena: a create costs
// one cudaMalloc and a destroy one cudaFree, and nothing is allocated while an encode runs. The layout below runs
// twice, once to measure (no base) and once to carve.
struct Carver
{
    char* base = nullptr;
    size_t at = 0;
    template <typename T>
    void operator()(T*& p, size_t bytes)
    {
        at = (at + 255) / 256 * 256;
        p = base && bytes ? reinterpret_cast<T*>(base + at) : nullptr;
        at += bytes;
    }
};

void layout(nntc_b200_device* d, const nntc_b200_model* m, Carver& take)
{
    size_t max0 = 0, max1 = 0, blocks = 0, sites = 0;
    for (DevPlane& p : d->planes)
    {
        const size_t n0 = (size_t)p.w0 * p.h0, n1 = (size_t)p.w1 * p.h1;
        max0 = std::max(max0, n0);
        max1 = std::max(max1, n1);
        blocks += (n0 + THREADS - 1) / THREADS;
        sites += n0 * 5;
        take(p.src, n0 * m->nout * sizeof(float));
        take(p.v0, n0 * m->c0 * sizeof(float));
        take(p.v1, n1 * m->c1 * sizeof(float));
        take(p.k0, n0 * m->c0);
        take(p.k1, n1 * m->c1);
        for (int lv = 0; lv < (m->l0_bc8 ? 2 : 1); lv++)
        {
            Work& w = p.work[lv];
            const size_t t = w.texels(), c = (size_t)w.c;
            take(w.stencil, t * SLOTS * c * c * sizeof(double));
            take(w.grad, t * c * sizeof(double));
            take(w.precond, t * c * c * sizeof(float));
            take(w.x, t * c * sizeof(double));
            take(w.r, t * c * sizeof(double));
            take(w.z, t * c * sizeof(double));
            take(w.p, t * c * sizeof(double));
            take(w.ap, t * c * sizeof(double));
            take(w.prev, t * c * sizeof(float));
        }
        if (m->l0_bc8)
        {
            take(p.bc_ep, p.blocks() * m->c0 * 2);
            take(p.bc_sel, p.blocks() * m->c0 * 16);
            take(p.bc_sten, p.blocks() * SLOTS * m->c0 * m->c0 * 16 * sizeof(double));
        }
    }
    take(d->weights, (size_t)m->nout * m->nin * sizeof(float));
    take(d->bias, (size_t)m->nout * sizeof(float));
    take(d->palette, (size_t)MAX_CH * 16 * sizeof(float));
    take(d->lo1, MAX_CH * sizeof(float));
    take(d->hi1, MAX_CH * sizeof(float));
    if (m->l0_bc8)
    {
        take(d->lo0, MAX_CH * sizeof(float));
        take(d->hi0, MAX_CH * sizeof(float));
        take(d->mono[1], (size_t)monomial_count(m->c1) * m->c0 * m->c0 * sizeof(double));
    }
    take(d->mono[0], (size_t)monomial_count(m->c0) * m->c1 * m->c1 * sizeof(double));
    take(d->cw, (size_t)m->nout * sizeof(float));
    // one partial per 256-item block of every plane's padded range and per reduction row (level 0 is the wider
    // unknown, so its texels bound every launch's block count)
    take(d->partial, (size_t)RROWS * blocks * sizeof(double));
    take(d->scalars, (size_t)MAX_PLANES * S_COUNT * sizeof(double));
    take(d->counters, (size_t)COUNTERS * sizeof(unsigned int));
    const int mm = m->nin + 1;
    const size_t entries = (size_t)(mm * (mm + 1) / 2 + m->nout * mm);
    take(d->reduction, entries * sizeof(double));
    take(d->dec_solve, 2048);
    // the normal equations' per-block partials of every plane, then one per-site weight per plane
    take(d->ls_partial, (d->planes.size() * entries * LS_GRID + MAX_PLANES) * sizeof(double));
    take(d->bc_stats, (size_t)MAX_PLANES * 2 * sizeof(double));
    take(d->radix, (size_t)std::max(2 * MAX_CH * 2048, MAX_NOUT * MAX_NOUT) * sizeof(unsigned int));
    // the assembly's per-site gradient terms: every site of every plane at the largest K (4), one double per channel
    // of the wider unknown; and every site's sample of the other latent
    d->site_terms_count = sites * (size_t)std::max(m->c0, m->c1);
    take(d->site_terms, d->site_terms_count * sizeof(double));
    take(d->site_y, sites * 4 * sizeof(float));
    take(d->site_tgt, sites / 5 * 4 * m->nout * sizeof(float));   // four fractional sites per pixel at K = 4
    take(d->obj_tgt, sites / 5 * 4 * m->nout * sizeof(double));
    take(d->gtab[0], (size_t)GATHER_TABLE_MAX * 16);
    take(d->gtab[1], (size_t)GATHER_TABLE_MAX * 16);
    // the objective's partials: two triples per 256-pixel block (its blocks are 128 threads), then three sums per plane
    take(d->obj_partial, (2 * blocks * 3 + 3 * MAX_PLANES) * sizeof(double));
    take(d->ls_obj, (d->planes.size() * 3 * LS_GRID + 3 * MAX_PLANES) * sizeof(double));
    d->scratch_floats = std::max(max0 * (size_t)m->c0, max1 * (size_t)m->c1);
    d->scratch_bytes = d->scratch_floats;
    take(d->scratch, d->scratch_floats * sizeof(float));
    take(d->scratch8, d->scratch_bytes);
    take(d->rgb8, max0 * m->nout);
    take(d->cov, (size_t)(MAX_NOUT + MAX_NOUT * MAX_NOUT) * COV_GRID * sizeof(double));
    take(d->basis, 1024);
    take(d->hist, (size_t)HIST_BINS * sizeof(unsigned long long));
    if (m->l0_bc8)
    {
        size_t kept = 0;
        for_each_kept(d, [&](void*, size_t b) { kept += (b + 255) / 256 * 256; });
        take(d->keep, kept);
    }
}

int arena_alloc(nntc_b200_device* d, size_t bytes)
{
    const cudaError_t err = cudaMalloc(&d->arena, bytes);
    if (err == cudaErrorMemoryAllocation)
    {
        d->arena = nullptr;
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        char buf[512];
        snprintf(buf, sizeof(buf),
                 "out of GPU memory allocating %.1f MB for the encode's device model (%zu/%zu MB free): the material "
                 "is too large for this GPU; try fewer or smaller textures, or fewer latent channels",
                 bytes / 1048576.0, free_b >> 20, total_b >> 20);
        set_error(NNTC_B200_ERR_OOM, buf);
        return NNTC_B200_ERR_OOM;
    }
    NB_CUDA(err);
    d->bytes = bytes;
    return NNTC_B200_OK;
}

int validate(const nntc_b200_model* m)
{
    auto bad = [](const std::string& s) {
        set_error(NNTC_B200_ERR_ARG, s);
        return NNTC_B200_ERR_ARG;
    };
    if (!m)
        return bad("model is null");
    if (m->c0 < 1 || m->c0 > MAX_CH || m->c1 < 1 || m->c1 > MAX_CH)
        return bad("latent channel counts must be 1..4");
    if (m->textures < 1 || m->textures > 6 || m->nout != 3 * m->textures)
        return bad("a material holds 1..6 RGB textures");
    if (m->nin != m->c1 + m->c0 + m->c0 * m->c1)
        return bad("nin must be C1 + C0 + C0 C1");
    if (m->nplanes < 1 || m->nplanes > MAX_PLANES)
        return bad("the chain holds 1..13 planes");
    for (int i = 0; i < m->nplanes; i++)
        if (m->w0[i] < 1 || m->h0[i] < 1 || m->w1[i] < 1 || m->h1[i] < 1)
            return bad("plane " + std::to_string(i) + " has an empty extent");
    if (m->bits1 < 1 || m->bits1 > 8)
        return bad("bits1 must be 1..8");
    return NNTC_B200_OK;
}

}   // namespace

// The model's layout checks, for host code outside this file (the asset writer).
int nb::validate_model(const nntc_b200_model* m)
{
    return validate(m);
}

extern "C"
{

const char* nntc_b200_last_error(void)
{
    return g_error.c_str();
}

int nntc_b200_version(void)
{
    return 1;
}

long long nntc_b200_launch_count(void)
{
    return g_launches.load();
}

int nntc_b200_kernel_timing(nntc_b200_device* d, int on)
{
    NB_CUDA(cudaStreamSynchronize(d->stream));
    NB_TRY(ktimer_harvest(d));
    d->ktiming = on != 0;
    return NNTC_B200_OK;
}

int nntc_b200_kernel_stats(nntc_b200_device* d, int kernel, long long* launches, double* ms, int reset)
{
    if (kernel < 0 || kernel >= NNTC_B200_K_COUNT)
    {
        set_error(NNTC_B200_ERR_ARG, "no such kernel");
        return NNTC_B200_ERR_ARG;
    }
    NB_CUDA(cudaStreamSynchronize(d->stream));
    NB_TRY(ktimer_harvest(d));
    if (launches)
        *launches = d->klaunches[kernel];
    if (ms)
        *ms = d->kms[kernel];
    if (reset)
        for (int k = 0; k < NNTC_B200_K_COUNT; k++)
        {
            d->klaunches[k] = 0;
            d->kms[k] = 0.0;
        }
    return NNTC_B200_OK;
}

int nntc_b200_abi_sizes(size_t* out, int n)
{
    const size_t sizes[] = { sizeof(nntc_b200_model),         sizeof(nntc_b200_device_info),
                             sizeof(nntc_b200_plane_report),  sizeof(nntc_b200_level0_report),
                             sizeof(nntc_b200_objective),     sizeof(nntc_b200_init1_report),
                             sizeof(nntc_b200_init0_report),  sizeof(nntc_b200_bc_report),
                             sizeof(nntc_b200_encode_args),   sizeof(nntc_b200_encode_result) };
    const int count = (int)(sizeof(sizes) / sizeof(sizes[0]));
    for (int i = 0; i < count && i < n; i++)
        out[i] = sizes[i];
    return count < n ? count : n;
}

int nntc_b200_device_select(int index, nntc_b200_device_info* info)
{
    std::memset(info, 0, sizeof(*info));
    auto refuse = [&](const std::string& s) {
        snprintf(info->error, sizeof(info->error), "%s", s.c_str());
        return 0;
    };
    int count = 0;
    cudaError_t err = cudaGetDeviceCount(&count);
    if (err == cudaErrorNoDevice || (err == cudaSuccess && count <= 0))
        return refuse("no NVIDIA GPU was found");
    if (err == cudaErrorInsufficientDriver)
        return refuse("there is no NVIDIA driver, or it is older than this build's CUDA runtime");
    if (err != cudaSuccess)
        return refuse(std::string("the CUDA runtime could not start (cudaGetDeviceCount: ") +
                      cudaGetErrorString(err) + ")");
    if (index < 0 || index >= count)
        return refuse("there is no CUDA device " + std::to_string(index) + " (the machine has " +
                      std::to_string(count) + " CUDA device" + (count == 1 ? "" : "s") + ")");
    err = cudaSetDevice(index);
    if (err != cudaSuccess)
        return refuse(std::string("CUDA device ") + std::to_string(index) + " could not be used (cudaSetDevice: " +
                      cudaGetErrorString(err) + ")");
    cudaDeviceProp prop;
    err = cudaGetDeviceProperties(&prop, index);
    if (err != cudaSuccess)
        return refuse(std::string("cudaGetDeviceProperties: ") + cudaGetErrorString(err));
    snprintf(info->name, sizeof(info->name), "%s", prop.name);
    info->major = prop.major;
    info->minor = prop.minor;
    // This library carries sm_100a code only: a device of any other capability has no kernel image to run.
    if (prop.major != 10 || prop.minor != 0)
        return refuse(std::string("this build carries sm_100a kernels only; device '") + prop.name +
                      "' is compute capability " + std::to_string(prop.major) + "." + std::to_string(prop.minor));
    return 1;
}

static int refuse_arg(const std::string& why)
{
    nb::set_error(NNTC_B200_ERR_ARG, why);
    return NNTC_B200_ERR_ARG;
}

// The device model; a null chain[i] leaves plane i's source to the caller (the from-base path fills it on the device).
static int device_create_impl(const nntc_b200_model* m, const float* const* chain, nntc_b200_device** out)
{
    *out = nullptr;
    NB_TRY(validate(m));
    nntc_b200_device* d = new nntc_b200_device();
    d->m = *m;
    d->nout = m->nout;
    d->nin = m->nin;
    d->c0 = m->c0;
    d->c1 = m->c1;
    d->l0_bc8 = m->l0_bc8 != 0;
    auto fail = [&](int st) {
        nntc_b200_device_destroy(d);
        return st;
    };
#define NB_CK(call)                                                                                                   \
    do                                                                                                                \
    {                                                                                                                 \
        const cudaError_t e_ = (call);                                                                                \
        if (e_ != cudaSuccess)                                                                                        \
            return fail(cuda_status(e_, #call, __FILE__, __LINE__));                                                 \
    } while (0)

    NB_CK(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking));
    for (int e = 0; e < 4; e++)
        NB_CK(cudaEventCreate(&d->ev[e]));

    d->planes.resize((size_t)m->nplanes);
    for (int i = 0; i < m->nplanes; i++)
    {
        DevPlane& p = d->planes[(size_t)i];
        p.w0 = m->w0[i];
        p.h0 = m->h0[i];
        p.w1 = m->w1[i];
        p.h1 = m->h1[i];
        for (int lv = 0; lv < (m->l0_bc8 ? 2 : 1); lv++)
        {
            Work& w = p.work[lv];
            w.w = lv ? p.w0 : p.w1;
            w.h = lv ? p.h0 : p.h1;
            w.c = lv ? m->c0 : m->c1;
        }
    }
    {
        Carver measure;
        layout(d, m, measure);
        const int st = arena_alloc(d, measure.at);
        if (st)
            return fail(st);
        Carver carve;
        carve.base = (char*)d->arena;
        layout(d, m, carve);
    }
    for (int i = 0; i < m->nplanes; i++)
    {
        DevPlane& p = d->planes[(size_t)i];
        const size_t n0 = (size_t)p.w0 * p.h0, n1 = (size_t)p.w1 * p.h1;
        if (chain[i])
            NB_CK(cudaMemcpy(p.src, chain[i], n0 * m->nout * sizeof(float), cudaMemcpyHostToDevice));
        NB_CK(cudaMemset(p.v0, 0, n0 * m->c0 * sizeof(float)));
        NB_CK(cudaMemset(p.v1, 0, n1 * m->c1 * sizeof(float)));
        NB_CK(cudaMemset(p.k0, 0, n0 * m->c0));
        NB_CK(cudaMemset(p.k1, 0, n1 * m->c1));
        for (int lv = 0; lv < (m->l0_bc8 ? 2 : 1); lv++)
        {
            Work& w = p.work[lv];
            const size_t t = w.texels(), c = (size_t)w.c;
            NB_CK(cudaMemset(w.x, 0, t * c * sizeof(double)));
            NB_CK(cudaMemset(w.prev, 0, t * c * sizeof(float)));
        }
        if (m->l0_bc8)
        {
            NB_CK(cudaMemset(p.bc_ep, 0, p.blocks() * m->c0 * 2));
            NB_CK(cudaMemset(p.bc_sel, 0, p.blocks() * m->c0 * 16));
        }
    }
    // The decoder starts at zero: the first objective pass measures the zero decoder (src/init.cu:262-267).
    NB_CK(cudaMemset(d->weights, 0, (size_t)m->nout * m->nin * sizeof(float)));
    NB_CK(cudaMemset(d->bias, 0, (size_t)m->nout * sizeof(float)));
    NB_CK(cudaMemset(d->palette, 0, (size_t)MAX_CH * 16 * sizeof(float)));
    NB_CK(cudaMemset(d->lo1, 0, MAX_CH * sizeof(float)));
    NB_CK(cudaMemset(d->hi1, 0, MAX_CH * sizeof(float)));
    if (m->l0_bc8)
    {
        NB_CK(cudaMemset(d->lo0, 0, MAX_CH * sizeof(float)));
        NB_CK(cudaMemset(d->hi0, 0, MAX_CH * sizeof(float)));
    }
    NB_CK(cudaMemcpy(d->cw, m->cw, (size_t)m->nout * sizeof(float), cudaMemcpyHostToDevice));
    NB_CK(cudaMemset(d->scalars, 0, (size_t)MAX_PLANES * S_COUNT * sizeof(double)));
    {
        const int mm = m->nin + 1;
        NB_CK(cudaMemset(d->reduction, 0, (size_t)(mm * (mm + 1) / 2 + m->nout * mm) * sizeof(double)));
    }
    NB_CK(cudaMallocHost(&d->host_scalars, (size_t)MAX_PLANES * S_COUNT * sizeof(double)));
    NB_CK(cudaMallocHost(&d->host_counters, (size_t)COUNTERS * sizeof(unsigned int)));
    // the set-up's copies and clears went to the legacy stream; the model's own stream does not wait for it
    NB_CK(cudaDeviceSynchronize());
    d->m.has_decoder = 0;
#undef NB_CK
    *out = d;
    return NNTC_B200_OK;
}

int nntc_b200_device_create(const nntc_b200_model* m, const float* const* chain, nntc_b200_device** out)
{
    *out = nullptr;
    NB_TRY(validate(m));
    if (!chain)
        return refuse_arg("the source chain is null");
    for (int i = 0; i < m->nplanes; i++)
        if (!chain[i])
            return refuse_arg("plane " + std::to_string(i) + " of the source chain is null");
    return device_create_impl(m, chain, out);
}

int nntc_b200_device_create_from_base(const nntc_b200_model* m, const float* base, nntc_b200_device** out)
{
    *out = nullptr;
    NB_TRY(validate(m));
    if (!base)
        return refuse_arg("the base plane is null");
    // the chain must be the default one: every level the floor halving of the one above, never below one texel
    for (int i = 1; i < m->nplanes; i++)
        if (m->w0[i] != nb::mip_dim(m->w0[i - 1]) || m->h0[i] != nb::mip_dim(m->h0[i - 1]))
            return refuse_arg("plane " + std::to_string(i) + " is not the box halving of plane " + std::to_string(i - 1));
    std::vector<const float*> chain((size_t)m->nplanes, nullptr);
    chain[0] = base;
    NB_TRY(device_create_impl(m, chain.data(), out));
    const int st = nb::build_source_chain(*out);
    if (st != NNTC_B200_OK)
    {
        nntc_b200_device_destroy(*out);
        *out = nullptr;
    }
    return st;
}

void nntc_b200_device_destroy(nntc_b200_device* d)
{
    if (!d)
        return;
    if (d->stream)
        cudaStreamSynchronize(d->stream);
    cudaFree(d->arena);
    cudaFreeHost(d->host_scalars);
    cudaFreeHost(d->host_counters);
    for (const nntc_b200_device::Pending& p : d->kpending)
    {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    for (cudaEvent_t e : d->kpool)
        cudaEventDestroy(e);
    for (cudaEvent_t e : d->ev)
        if (e)
            cudaEventDestroy(e);
    if (d->stream)
        cudaStreamDestroy(d->stream);
    delete d;
}

size_t nntc_b200_device_memory(const nntc_b200_device* d)
{
    return d ? d->bytes : 0;
}

int nntc_b200_stencil_monomials(int c0)
{
    return monomial_count(c0);
}

// ---- transfers ----------------------------------------------------------------------------------------------------

int nntc_b200_level1_download_indices(nntc_b200_device* d, int plane, uint8_t* k1, size_t n)
{
    NB_TRY(check_plane(d, plane));
    const DevPlane& p = d->planes[(size_t)plane];
    const size_t want = (size_t)p.w1 * p.h1 * d->c1;
    if (n < want)
    {
        set_error(NNTC_B200_ERR_ARG, "level-1 index buffer too small");
        return NNTC_B200_ERR_ARG;
    }
    return download(d, k1, p.k1, want);
}

int nntc_b200_level1_upload(nntc_b200_device* d, int plane, const float* v1, size_t n)
{
    NB_TRY(check_plane(d, plane));
    const DevPlane& p = d->planes[(size_t)plane];
    if (n != (size_t)p.w1 * p.h1 * d->c1)
        return NNTC_B200_OK;   // a size that does not match is ignored, as the reference's upload does
    return upload(d, p.v1, v1, n * sizeof(float));
}

int nntc_b200_level1_upload_indices(nntc_b200_device* d, int plane, const uint8_t* k1, size_t n)
{
    NB_TRY(check_plane(d, plane));
    const DevPlane& p = d->planes[(size_t)plane];
    if (n != (size_t)p.w1 * p.h1 * d->c1)
        return NNTC_B200_OK;
    return upload(d, p.k1, k1, n);
}

int nntc_b200_level0_upload_indices(nntc_b200_device* d, int plane, const uint8_t* k0, size_t n)
{
    NB_TRY(check_plane(d, plane));
    const DevPlane& p = d->planes[(size_t)plane];
    if (n != (size_t)p.w0 * p.h0 * d->c0)
        return NNTC_B200_OK;
    return upload(d, p.k0, k0, n);
}

int nntc_b200_upload_decoder(nntc_b200_device* d, const nntc_b200_model* m)
{
    return upload_decoder(d, m);
}

int nntc_b200_upload_grids(nntc_b200_device* d, const nntc_b200_model* m)
{
    return upload_grids(d, m);
}

int nntc_b200_level1_download(nntc_b200_device* d, int plane, float* v1, size_t n)
{
    NB_TRY(check_plane(d, plane));
    const DevPlane& p = d->planes[(size_t)plane];
    const size_t want = (size_t)p.w1 * p.h1 * d->c1;
    if (n < want)
    {
        set_error(NNTC_B200_ERR_ARG, "level-1 value buffer too small");
        return NNTC_B200_ERR_ARG;
    }
    return download(d, v1, p.v1, want * sizeof(float));
}

int nntc_b200_level1_delta(nntc_b200_device* d, int plane, double* delta, size_t n)
{
    NB_TRY(check_plane(d, plane));
    const Work& w = d->planes[(size_t)plane].work[0];
    if (n < w.values())
    {
        set_error(NNTC_B200_ERR_ARG, "level-1 delta buffer too small");
        return NNTC_B200_ERR_ARG;
    }
    return download(d, delta, w.x, w.values() * sizeof(double));
}

int nntc_b200_level1_poke(nntc_b200_device* d, int plane, size_t index, float value)
{
    NB_TRY(check_plane(d, plane));
    const DevPlane& p = d->planes[(size_t)plane];
    if (index >= (size_t)p.w1 * p.h1 * d->c1)
    {
        set_error(NNTC_B200_ERR_ARG, "level-1 poke outside the plane");
        return NNTC_B200_ERR_ARG;
    }
    return upload(d, p.v1 + index, &value, sizeof(float));
}

int nntc_b200_level1_range(nntc_b200_device* d, int plane, float* lo, float* hi)
{
    NB_TRY(check_plane(d, plane));
    const DevPlane& p = d->planes[(size_t)plane];
    std::vector<float> v((size_t)p.w1 * p.h1 * d->c1);
    NB_TRY(download(d, v.data(), p.v1, v.size() * sizeof(float)));
    for (int c = 0; c < d->c1; c++)
    {
        lo[c] = 1e30f;
        hi[c] = -1e30f;
    }
    for (size_t i = 0; i < v.size(); i++)
    {
        const int c = (int)(i % (size_t)d->c1);
        lo[c] = v[i] < lo[c] ? v[i] : lo[c];
        hi[c] = v[i] > hi[c] ? v[i] : hi[c];
    }
    return NNTC_B200_OK;
}

int nntc_b200_level0_download(nntc_b200_device* d, int plane, uint8_t* k0, size_t n)
{
    NB_TRY(check_plane(d, plane));
    const DevPlane& p = d->planes[(size_t)plane];
    const size_t want = (size_t)p.w0 * p.h0 * d->c0;
    if (n < want)
    {
        set_error(NNTC_B200_ERR_ARG, "level-0 index buffer too small");
        return NNTC_B200_ERR_ARG;
    }
    return download(d, k0, p.k0, want);
}

int nntc_b200_level0_upload(nntc_b200_device* d, int plane, const float* v0, size_t n)
{
    NB_TRY(check_plane(d, plane));
    const DevPlane& p = d->planes[(size_t)plane];
    if (n != (size_t)p.w0 * p.h0 * d->c0)
        return NNTC_B200_OK;
    return upload(d, p.v0, v0, n * sizeof(float));
}

int nntc_b200_level0_download_values(nntc_b200_device* d, int plane, float* v0, size_t n)
{
    NB_TRY(check_plane(d, plane));
    const DevPlane& p = d->planes[(size_t)plane];
    const size_t want = (size_t)p.w0 * p.h0 * d->c0;
    if (n < want)
    {
        set_error(NNTC_B200_ERR_ARG, "level-0 value buffer too small");
        return NNTC_B200_ERR_ARG;
    }
    return download(d, v0, p.v0, want * sizeof(float));
}

// ---- probes (src/backend_check_probe.h:20-37) ---------------------------------------------------------------------

int nntc_b200_probe_normal_equations(nntc_b200_device* d, double* out, size_t n)
{
    const int mm = d->nin + 1;
    const size_t entries = (size_t)(mm * (mm + 1) / 2 + d->nout * mm);
    if (n < entries)
    {
        set_error(NNTC_B200_ERR_ARG, "normal-equation buffer too small");
        return NNTC_B200_ERR_ARG;
    }
    return download(d, out, d->reduction, entries * sizeof(double));
}

// The workspace in the reference's layout: the SoA stencil transposed back to [texel][slot][i][j].
int nntc_b200_probe_workspace(nntc_b200_device* d, int plane, int level0, double* stencil, double* grad,
                              float* precond, double* cg_x, float* prev)
{
    NB_TRY(check_plane(d, plane));
    if (level0 && !d->l0_bc8)
    {
        set_error(NNTC_B200_ERR_STATE, "level 0 has no workspace outside --l0 bc8");
        return NNTC_B200_ERR_STATE;
    }
    const Work& w = d->planes[(size_t)plane].work[level0 ? 1 : 0];
    const size_t t = w.texels(), c = (size_t)w.c, per = SLOTS * c * c;
    if (stencil)
    {
        std::vector<double> soa(t * per);
        if (d->sten_f32[level0 ? 1 : 0])
        {
            // an FP32 stencil (the adjoint form's, [slot][texel][e]), widened into the SoA order
            std::vector<float> f(t * per);
            NB_TRY(download(d, f.data(), w.stencil, f.size() * sizeof(float)));
            const int cc = (int)(c * c);
            for (int slot = 0; slot < SLOTS; slot++)
                for (size_t at = 0; at < t; at++)
                    for (int e = 0; e < cc; e++)
                        soa[(size_t)(slot * cc + e) * t + at] = (double)f[sten_index<float>(slot, e, cc, t, at)];
        }
        else
            NB_TRY(download(d, soa.data(), w.stencil, soa.size() * sizeof(double)));
        // back from the colour-major SoA order to the reference's [texel][slot][i][j]
        for (size_t i = 0; i < t; i++)
        {
            const size_t at = stencil_pos((int)(i % (size_t)w.w), (int)(i / (size_t)w.w), w.w, w.h);
            for (size_t e = 0; e < per; e++)
                stencil[i * per + e] = soa[e * t + at];
        }
    }
    if (grad)
        NB_TRY(download(d, grad, w.grad, t * c * sizeof(double)));
    if (precond)
        NB_TRY(download(d, precond, w.precond, t * c * c * sizeof(float)));
    if (cg_x)
        NB_TRY(download(d, cg_x, w.x, t * c * sizeof(double)));
    if (prev)
        NB_TRY(download(d, prev, w.prev, t * c * sizeof(float)));
    return NNTC_B200_OK;
}

int nntc_b200_probe_source(nntc_b200_device* d, int plane, float* out, size_t n)
{
    NB_TRY(check_plane(d, plane));
    const DevPlane& p = d->planes[(size_t)plane];
    const size_t want = (size_t)p.w0 * p.h0 * d->nout;
    if (n < want)
    {
        set_error(NNTC_B200_ERR_ARG, "source buffer too small");
        return NNTC_B200_ERR_ARG;
    }
    return download(d, out, p.src, want * sizeof(float));
}

int nntc_b200_probe_monomials(nntc_b200_device* d, int level0, double* out, size_t n)
{
    if (level0 && !d->l0_bc8)
    {
        set_error(NNTC_B200_ERR_STATE, "level 0 has no monomials outside --l0 bc8");
        return NNTC_B200_ERR_STATE;
    }
    const int dim = level0 ? d->c0 : d->c1;
    const size_t want = (size_t)monomial_count(level0 ? d->c1 : d->c0) * dim * dim;
    if (n < want)
    {
        set_error(NNTC_B200_ERR_ARG, "monomial buffer too small");
        return NNTC_B200_ERR_ARG;
    }
    return download(d, out, d->mono[level0 ? 1 : 0], want * sizeof(double));
}

}   // extern "C"
