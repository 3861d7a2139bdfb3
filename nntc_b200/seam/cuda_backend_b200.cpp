// cuda_backend_b200.cpp: the reference's CUDA arm, replaced.
//
// This is the drop-in for src/cuda_backend.cpp and the six .cu files behind it. It defines the 46 functions of
// src/cuda_backend.h:20-80 (namespace nntc_cuda, DeviceModel*) with exactly those C++ signatures, and the three reads
// of src/backend_check_probe.h:20-37 (namespace nntc_probe) the per-kernel harness makes, each as a thin translation
// onto the C ABI of include/nntc_b200.h:
//
//   - DeviceModel, opaque to the reference's host (src/model.h:253), is defined here as the library's handle plus the
//     POD mirror of the model it was created from;
//   - the reference's Model& is copied into that POD before each call, and what the call mutates (the decoder, the
//     grids, the index mirrors k0 / k1, the BC blocks) is copied back after it;
//   - a failed call prints the reference's one ERROR line and exits with status 1, as its CUDA_CHECK does
//     (src/device.cuh:45-76), so the host's behaviour on failure is unchanged.
//
// It is compiled against the reference's own headers (model.h, image.h, options.h, cuda_backend.h,
// backend_check_probe.h) by oracle/Makefile's `dropin` target, which links the reference's host sources with
// libnntc_b200.so; nothing here is built into the library itself.

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "backend_check_probe.h"
#include "cuda_backend.h"
#include "model.h"
#include "nntc_b200.h"

struct DeviceModel
{
    nntc_b200_device* dev = nullptr;
    nntc_b200_model pod{};
};

namespace
{

[[noreturn]] void fail(const char* call)
{
    fprintf(stderr, "ERROR: %s: %s\n", call, nntc_b200_last_error());
    exit(EXIT_FAILURE);
}

#define NB_CALL(expr)                                                                                                 \
    do                                                                                                                \
    {                                                                                                                 \
        if ((expr) != NNTC_B200_OK)                                                                                   \
            fail(#expr);                                                                                              \
    } while (0)

void to_pod(const Model& m, nntc_b200_model& p)
{
    std::memset(&p, 0, sizeof(p));
    p.textures = m.textures;
    p.nout = m.nout;
    p.width = m.width;
    p.height = m.height;
    p.c0 = m.c0;
    p.c1 = m.c1;
    for (int c = 0; c < m.c0 && c < (int)m.bits0.size(); c++)
        p.bits0[c] = m.bits0[(size_t)c];
    p.bits1 = m.bits1;
    p.bc0 = m.bc0;
    p.l0_bc8 = m.l0_bc8;
    p.init0_residual = m.init0_residual;
    p.init0_texture = m.init0_texture;
    p.init0_chain = m.init0_chain;
    p.nin = m.dec.nin;
    p.nplanes = (int)m.planes.size();
    for (size_t i = 0; i < m.planes.size() && i < NNTC_B200_MAX_PLANES; i++)
    {
        p.w0[i] = m.planes[i].w0;
        p.h0[i] = m.planes[i].h0;
        p.w1[i] = m.planes[i].w1;
        p.h1[i] = m.planes[i].h1;
    }
    for (int c = 0; c < m.nout && c < (int)m.cw.size(); c++)
        p.cw[c] = m.cw[(size_t)c];
    p.has_decoder = !m.dec.w.empty() && !m.dec.b.empty();
    if (p.has_decoder)
    {
        std::memcpy(p.dec_w, m.dec.w.data(), m.dec.w.size() * sizeof(float));
        std::memcpy(p.dec_b, m.dec.b.data(), m.dec.b.size() * sizeof(float));
    }
    for (size_t c = 0; c < m.palette0.size() && c < NNTC_B200_MAX_CHANNELS; c++)
    {
        p.palette0_len[c] = (int)std::min<size_t>(m.palette0[c].size(), 16);
        for (int k = 0; k < p.palette0_len[c]; k++)
            p.palette0[c][k] = m.palette0[c][(size_t)k];
    }
    p.has_lo0 = !m.lo0.empty();
    for (size_t c = 0; c < m.lo0.size() && c < NNTC_B200_MAX_CHANNELS; c++)
    {
        p.lo0[c] = m.lo0[c];
        p.hi0[c] = m.hi0[c];
    }
    p.has_lo1 = !m.lo1.empty();
    for (size_t c = 0; c < m.lo1.size() && c < NNTC_B200_MAX_CHANNELS; c++)
    {
        p.lo1[c] = m.lo1[c];
        p.hi1[c] = m.hi1[c];
    }
}

void decoder_back(const nntc_b200_model& p, Model& m)
{
    if (!p.has_decoder)
        return;
    m.dec.w.assign(p.dec_w, p.dec_w + (size_t)p.nout * p.nin);
    m.dec.b.assign(p.dec_b, p.dec_b + p.nout);
}

void grid1_back(const nntc_b200_model& p, Model& m)
{
    m.lo1.assign(p.lo1, p.lo1 + p.c1);
    m.hi1.assign(p.hi1, p.hi1 + p.c1);
}

void grid0_back(const nntc_b200_model& p, Model& m)
{
    m.lo0.assign(p.lo0, p.lo0 + p.c0);
    m.hi0.assign(p.hi0, p.hi0 + p.c0);
}

// Per-plane index mirrors, sized for the layout, and the pointer table the C ABI takes.
struct Mirror
{
    std::vector<uint8_t*> ptr;
    Mirror(std::vector<std::vector<uint8_t>>& k, const Model& m, bool level0)
    {
        k.resize(m.planes.size());
        for (size_t i = 0; i < m.planes.size(); i++)
        {
            const PlaneSize& p = m.planes[i];
            const size_t n = level0 ? (size_t)p.w0 * p.h0 * m.c0 : (size_t)p.w1 * p.h1 * m.c1;
            k[i].resize(n);
            ptr.push_back(k[i].data());
        }
    }
};

void level1_report(const nntc_b200_plane_report& r, Level1Report& o)
{
    o = Level1Report();
    o.iterations = r.iterations;
    o.residual = r.residual;
    o.lambda = r.lambda;
    o.min_diag = r.min_diag;
    o.max_diag = r.max_diag;
    o.ms_assemble = r.ms_assemble;
    o.ms_precond = r.ms_precond;
    o.ms_cg = r.ms_cg;
    o.moved_values = r.moved_values;
    o.delta2 = r.delta2;
    o.plane2 = r.plane2;
    for (int c = 0; c < 4; c++)
    {
        o.lo[c] = r.lo[c];
        o.hi[c] = r.hi[c];
    }
    o.quantised = r.quantised != 0;
    o.sweeps = r.sweeps;
    o.moved = r.moved;
    o.ms_sweeps = r.ms_sweeps;
}

size_t plane_blocks(const Model& m, size_t i)
{
    return (size_t)((m.planes[i].w0 + 3) / 4) * (size_t)((m.planes[i].h0 + 3) / 4);
}

// The endpoints and selectors the device holds into the model's .dds blocks, with the pack's error against m.k0's
// exact index values (src/refine_bc.cu:589-608; src/export.cpp:333-370).
void blocks_from_device(DeviceModel* d, Model& m, double& pack_psnr, size_t& pack_texels)
{
    const size_t np = m.planes.size();
    std::vector<std::vector<uint8_t>> ep(np), sel(np);
    std::vector<uint8_t*> pe, ps;
    for (size_t i = 0; i < np; i++)
    {
        ep[i].resize(plane_blocks(m, i) * m.c0 * 2);
        sel[i].resize(plane_blocks(m, i) * m.c0 * 16);
        pe.push_back(ep[i].data());
        ps.push_back(sel[i].data());
    }
    NB_CALL(nntc_b200_bc_state_save(d->dev, &d->pod, pe.data(), ps.data()));
    m.bc0_blocks.assign(np, std::vector<std::vector<uint8_t>>());
    double se = 0.0;
    size_t n = 0;
    for (size_t i = 0; i < np; i++)
        level0_pack_blocks(m, (int)i, ep[i], sel[i], m.bc0_blocks[i], se, n);
    pack_texels = n;
    pack_psnr = n > 0 && se > 0.0 ? 10.0 * std::log10(255.0 * 255.0 / (se / (double)n)) : 100.0;
}

}   // namespace

namespace nntc_cuda
{

bool device_select(int index, DeviceInfo& info)
{
    nntc_b200_device_info i{};
    const int ok = nntc_b200_device_select(index, &i);
    info.name = i.name;
    info.major = i.major;
    info.minor = i.minor;
    info.error = i.error;
    return ok == 1;
}

DeviceModel* device_create(const Model& m, const std::vector<Image>& source_chain)
{
    DeviceModel* d = new DeviceModel();
    to_pod(m, d->pod);
    std::vector<const float*> chain;
    for (const Image& im : source_chain)
        chain.push_back(im.v.data());
    NB_CALL(nntc_b200_device_create(&d->pod, chain.data(), &d->dev));
    return d;
}

void device_destroy(DeviceModel* d)
{
    if (!d)
        return;
    nntc_b200_device_destroy(d->dev);
    delete d;
}

size_t device_memory(const DeviceModel* d)
{
    return d ? nntc_b200_device_memory(d->dev) : 0;
}

void init_level0(DeviceModel* d, Model& m, const float* luma_weights, bool luma_channel0)
{
    to_pod(m, d->pod);
    std::vector<std::vector<uint8_t>> k0;
    Mirror mk(k0, m, true);
    NB_CALL(nntc_b200_init_level0(d->dev, &d->pod, luma_weights, luma_channel0 ? 1 : 0, mk.ptr.data()));
    m.k0 = k0;
}

void init_level1(DeviceModel* d, Model& m, bool pca, Level1InitReport& rep)
{
    to_pod(m, d->pod);
    std::vector<std::vector<uint8_t>> k1;
    Mirror mk(k1, m, false);
    nntc_b200_init1_report r{};
    NB_CALL(nntc_b200_init_level1(d->dev, &d->pod, pca ? 1 : 0, &r, mk.ptr.data()));
    grid1_back(d->pod, m);
    m.k1 = k1;
    rep = Level1InitReport();
    rep.pca = r.pca != 0;
    rep.components = r.components;
    for (int i = 0; i < 4; i++)
    {
        rep.eigenvalue[i] = r.eigenvalue[i];
        rep.peak[i] = r.peak[i];
    }
    rep.total_variance = r.total_variance;
}

void init0_residual_channel(DeviceModel* d, Model& m, int channel, const std::vector<double>& plane_weight,
                            Init0ChannelReport& rep)
{
    to_pod(m, d->pod);
    if (m.k0.size() != m.planes.size())
        m.k0.assign(m.planes.size(), std::vector<uint8_t>());
    std::vector<uint8_t*> ptr;
    for (size_t i = 0; i < m.planes.size(); i++)
    {
        m.k0[i].resize((size_t)m.planes[i].w0 * m.planes[i].h0 * m.c0);
        ptr.push_back(m.k0[i].data());
    }
    nntc_b200_init0_report r{};
    NB_CALL(nntc_b200_init0_residual_channel(d->dev, &d->pod, channel, plane_weight.data(), &r, ptr.data()));
    rep = Init0ChannelReport();
    rep.eigenvalue = r.eigenvalue;
    rep.total_variance = r.total_variance;
    rep.share = r.share;
    rep.peak = r.peak;
    rep.divisor = r.divisor;
    for (int i = 0; i < 3 * MAX_TEXTURES; i++)
        rep.dir[i] = r.dir[i];
    rep.nout = r.nout;
    rep.texture = r.texture;
}

void quantise_level1(DeviceModel* d, Model& m, const std::string& range_policy)
{
    to_pod(m, d->pod);
    std::vector<std::vector<uint8_t>> k1;
    Mirror mk(k1, m, false);
    NB_CALL(nntc_b200_quantise_level1(d->dev, &d->pod, range_policy == "pct" ? 1 : 0, mk.ptr.data()));
    grid1_back(d->pod, m);
    m.k1 = k1;
}

void freeze_level1_grid(DeviceModel* d, Model& m, const std::string& range_policy)
{
    to_pod(m, d->pod);
    std::vector<std::vector<uint8_t>> k1;
    Mirror mk(k1, m, false);
    NB_CALL(nntc_b200_freeze_level1_grid(d->dev, &d->pod, range_policy == "pct" ? 1 : 0, mk.ptr.data()));
    grid1_back(d->pod, m);
    m.k1 = k1;
}

void quantise_level0(DeviceModel* d, Model& m, const std::string& range_policy)
{
    to_pod(m, d->pod);
    std::vector<std::vector<uint8_t>> k0;
    Mirror mk(k0, m, true);
    NB_CALL(nntc_b200_quantise_level0(d->dev, &d->pod, range_policy == "pct" ? 1 : 0, mk.ptr.data()));
    grid0_back(d->pod, m);
    m.k0 = k0;
}

void freeze_level0_grid(DeviceModel* d, Model& m, const std::string& range_policy)
{
    to_pod(m, d->pod);
    std::vector<std::vector<uint8_t>> k0;
    Mirror mk(k0, m, true);
    NB_CALL(nntc_b200_freeze_level0_grid(d->dev, &d->pod, range_policy == "pct" ? 1 : 0, mk.ptr.data()));
    grid0_back(d->pod, m);
    m.k0 = k0;
}

void snap_level0_on_grid(DeviceModel* d, Model& m)
{
    to_pod(m, d->pod);
    std::vector<std::vector<uint8_t>> k0;
    Mirror mk(k0, m, true);
    NB_CALL(nntc_b200_snap_level0_on_grid(d->dev, &d->pod, mk.ptr.data()));
    m.k0 = k0;
}

int stencil_monomials(int c0)
{
    return nntc_b200_stencil_monomials(c0);
}

double solve_decoder(DeviceModel* d, Model& m, int k, const std::vector<double>& per_site)
{
    to_pod(m, d->pod);
    double ms = 0.0;
    NB_CALL(nntc_b200_solve_decoder(d->dev, &d->pod, k, per_site.data(), &ms));
    decoder_back(d->pod, m);
    return ms;
}

void decoder_ridge_tally(long long out[4])
{
    nntc_b200_decoder_ridge_tally(out);
}

static double block_call(int (*fn)(nntc_b200_device*, const nntc_b200_model*, int, double, nntc_b200_plane_report*,
                                   double*),
                         DeviceModel* d, const Model& m, int k, double ridge, std::vector<Level1Report>& rep,
                         const char* name)
{
    to_pod(m, d->pod);
    std::vector<nntc_b200_plane_report> r(m.planes.size());
    double ms = 0.0;
    if (fn(d->dev, &d->pod, k, ridge, r.data(), &ms) != NNTC_B200_OK)
        fail(name);
    rep.assign(m.planes.size(), Level1Report());
    for (size_t i = 0; i < r.size(); i++)
        level1_report(r[i], rep[i]);
    return ms;
}

static double sweep_call(int (*fn)(nntc_b200_device*, const nntc_b200_model*, int, double, int,
                                   nntc_b200_plane_report*, double*),
                         DeviceModel* d, const Model& m, int k, double ridge, int sweeps,
                         std::vector<Level1Report>& rep, const char* name)
{
    to_pod(m, d->pod);
    std::vector<nntc_b200_plane_report> r(m.planes.size());
    double ms = 0.0;
    if (fn(d->dev, &d->pod, k, ridge, sweeps, r.data(), &ms) != NNTC_B200_OK)
        fail(name);
    rep.assign(m.planes.size(), Level1Report());
    for (size_t i = 0; i < r.size(); i++)
        level1_report(r[i], rep[i]);
    return ms;
}

double solve_level1_all(DeviceModel* d, const Model& m, int k, double ridge, std::vector<Level1Report>& rep)
{
    return block_call(nntc_b200_solve_level1_all, d, m, k, ridge, rep, "solve_level1_all");
}

double sweep_level1_all(DeviceModel* d, const Model& m, int k, double ridge, int sweeps,
                        std::vector<Level1Report>& rep)
{
    return sweep_call(nntc_b200_sweep_level1_all, d, m, k, ridge, sweeps, rep, "sweep_level1_all");
}

double solve_level0_cont_all(DeviceModel* d, const Model& m, int k, double ridge, std::vector<Level1Report>& rep)
{
    return block_call(nntc_b200_solve_level0_cont_all, d, m, k, ridge, rep, "solve_level0_cont_all");
}

double sweep_level0_cont_all(DeviceModel* d, const Model& m, int k, double ridge, int sweeps,
                             std::vector<Level1Report>& rep)
{
    return sweep_call(nntc_b200_sweep_level0_cont_all, d, m, k, ridge, sweeps, rep, "sweep_level0_cont_all");
}

double assemble_level0_for_refine(DeviceModel* d, const Model& m, int k)
{
    to_pod(m, d->pod);
    double ms = 0.0;
    NB_CALL(nntc_b200_assemble_level0_for_refine(d->dev, &d->pod, k, &ms));
    return ms;
}

void level1_download_indices(DeviceModel* d, const Model& m, int plane, std::vector<uint8_t>& k1)
{
    const PlaneSize& p = m.planes[(size_t)plane];
    k1.resize((size_t)p.w1 * p.h1 * m.c1);
    NB_CALL(nntc_b200_level1_download_indices(d->dev, plane, k1.data(), k1.size()));
}

void level1_upload(DeviceModel* d, const Model& m, int plane, const std::vector<float>& v1)
{
    (void)m;
    NB_CALL(nntc_b200_level1_upload(d->dev, plane, v1.data(), v1.size()));
}

void level1_upload_indices(DeviceModel* d, const Model& m, int plane, const std::vector<uint8_t>& k1)
{
    (void)m;
    NB_CALL(nntc_b200_level1_upload_indices(d->dev, plane, k1.data(), k1.size()));
}

void level0_upload_indices(DeviceModel* d, const Model& m, int plane, const std::vector<uint8_t>& k0)
{
    (void)m;
    NB_CALL(nntc_b200_level0_upload_indices(d->dev, plane, k0.data(), k0.size()));
}

void upload_decoder_to_device(DeviceModel* d, const Model& m)
{
    to_pod(m, d->pod);
    NB_CALL(nntc_b200_upload_decoder(d->dev, &d->pod));
}

void upload_grids_to_device(DeviceModel* d, const Model& m)
{
    to_pod(m, d->pod);
    NB_CALL(nntc_b200_upload_grids(d->dev, &d->pod));
}

void level1_download(DeviceModel* d, const Model& m, int plane, std::vector<float>& v)
{
    const PlaneSize& p = m.planes[(size_t)plane];
    v.resize((size_t)p.w1 * p.h1 * m.c1);
    NB_CALL(nntc_b200_level1_download(d->dev, plane, v.data(), v.size()));
}

void level1_delta(DeviceModel* d, const Model& m, int plane, std::vector<double>& delta)
{
    const PlaneSize& p = m.planes[(size_t)plane];
    delta.resize((size_t)p.w1 * p.h1 * m.c1);
    NB_CALL(nntc_b200_level1_delta(d->dev, plane, delta.data(), delta.size()));
}

void level1_poke(DeviceModel* d, int plane, size_t index, float value)
{
    NB_CALL(nntc_b200_level1_poke(d->dev, plane, index, value));
}

void level1_range(DeviceModel* d, const Model& m, int plane, std::vector<float>& lo, std::vector<float>& hi)
{
    float l[4], h[4];
    NB_CALL(nntc_b200_level1_range(d->dev, plane, l, h));
    lo.assign(l, l + m.c1);
    hi.assign(h, h + m.c1);
}

bool solve_level1_dense_host(DeviceModel* d, const Model& m, int k, int plane, double lambda,
                             const std::vector<float>& c_prev, std::vector<double>& delta, int max_unknowns)
{
    to_pod(m, d->pod);
    const PlaneSize& p = m.planes[(size_t)plane];
    const int nunk = p.w1 * p.h1 * m.c1;
    if (nunk > max_unknowns)
        return false;
    delta.assign((size_t)nunk, 0.0);
    const int st = nntc_b200_solve_level1_dense_host(d->dev, &d->pod, k, plane, lambda, c_prev.data(), c_prev.size(),
                                                     delta.data(), max_unknowns);
    if (st == NNTC_B200_ERR_STATE)
        return false;
    if (st != NNTC_B200_OK)
        fail("solve_level1_dense_host");
    return true;
}

double solve_level0_all(DeviceModel* d, const Model& m, int k, int sweeps, std::vector<Level0Report>& rep)
{
    to_pod(m, d->pod);
    std::vector<nntc_b200_level0_report> r(m.planes.size());
    double ms = 0.0;
    NB_CALL(nntc_b200_solve_level0_all(d->dev, &d->pod, k, sweeps, r.data(), &ms));
    rep.assign(m.planes.size(), Level0Report());
    for (size_t i = 0; i < r.size(); i++)
    {
        for (int c = 0; c < 4; c++)
            rep[i].moved[c] = r[i].moved[c];
        rep[i].moved_total = r[i].moved_total;
        rep[i].ms = r[i].ms;
        rep[i].joint = r[i].joint != 0;
        rep[i].states = r[i].states;
    }
    return ms;
}

void level0_download(DeviceModel* d, const Model& m, int plane, std::vector<uint8_t>& k0)
{
    const PlaneSize& p = m.planes[(size_t)plane];
    k0.resize((size_t)p.w0 * p.h0 * m.c0);
    NB_CALL(nntc_b200_level0_download(d->dev, plane, k0.data(), k0.size()));
}

void level0_upload(DeviceModel* d, const Model& m, int plane, const std::vector<float>& v0)
{
    (void)m;
    NB_CALL(nntc_b200_level0_upload(d->dev, plane, v0.data(), v0.size()));
}

void level0_download_values(DeviceModel* d, const Model& m, int plane, std::vector<float>& v0)
{
    const PlaneSize& p = m.planes[(size_t)plane];
    v0.resize((size_t)p.w0 * p.h0 * m.c0);
    NB_CALL(nntc_b200_level0_download_values(d->dev, plane, v0.data(), v0.size()));
}

void decode_plane(DeviceModel* d, const Model& m, int plane, std::vector<uint8_t>& rgb8)
{
    to_pod(m, d->pod);
    const PlaneSize& p = m.planes[(size_t)plane];
    rgb8.resize((size_t)p.w0 * p.h0 * m.nout);
    NB_CALL(nntc_b200_decode_plane(d->dev, &d->pod, plane, rgb8.data(), rgb8.size()));
}

static void objective_out(const nntc_b200_objective& o, const Model& m, Objective& r)
{
    r = Objective();
    r.e = o.e;
    r.centre_mse = o.centre_mse;
    r.sampled_mse = o.sampled_mse;
    r.e_plane.assign(o.e_plane, o.e_plane + m.planes.size());
    r.centre_plane.assign(o.centre_plane, o.centre_plane + m.planes.size());
    r.ms = o.ms;
}

void objective_eval(DeviceModel* d, const Model& m, int k, const std::vector<double>& per_site, Objective& r)
{
    to_pod(m, d->pod);
    nntc_b200_objective o{};
    NB_CALL(nntc_b200_objective_eval(d->dev, &d->pod, k, per_site.data(), &o));
    objective_out(o, m, r);
}

double objective_total_ms()
{
    return nntc_b200_objective_total_ms();
}

long long objective_passes()
{
    return nntc_b200_objective_passes();
}

void objective_check_host(DeviceModel* d, const Model& m, int k, const std::vector<double>& per_site, Objective& r)
{
    to_pod(m, d->pod);
    nntc_b200_objective o{};
    NB_CALL(nntc_b200_objective_check_host(d->dev, &d->pod, k, per_site.data(), &o));
    objective_out(o, m, r);
}

double bc_pack_prepare(DeviceModel* d, Model& m, int k, bool seed, double& pack_psnr, size_t& pack_texels)
{
    to_pod(m, d->pod);
    std::vector<const uint8_t*> k0;
    for (size_t i = 0; i < m.planes.size(); i++)
        k0.push_back(i < m.k0.size() && !m.k0[i].empty() ? m.k0[i].data() : nullptr);
    double ms = 0.0;
    NB_CALL(nntc_b200_bc_pack_prepare(d->dev, &d->pod, k, seed ? 1 : 0, k0.data(), &ms));
    blocks_from_device(d, m, pack_psnr, pack_texels);
    return ms;
}

double bc_refine(DeviceModel* d, Model& m, int passes, std::vector<BcRefineReport>& rep, double& pack_psnr,
                 size_t& pack_texels)
{
    rep.clear();
    if (passes <= 0)
        return 0.0;
    to_pod(m, d->pod);
    std::vector<nntc_b200_bc_report> r((size_t)passes);
    double ms = 0.0;
    NB_CALL(nntc_b200_bc_refine(d->dev, &d->pod, passes, r.data(), &ms));
    for (const nntc_b200_bc_report& x : r)
    {
        BcRefineReport o;
        o.pass = x.pass;
        o.blocks = x.blocks;
        o.improved = x.improved;
        o.delta_e = x.delta_e;
        o.ms = x.ms;
        rep.push_back(o);
    }
    blocks_from_device(d, m, pack_psnr, pack_texels);
    return ms;
}

void bc_blocks_from_device(DeviceModel* d, Model& m, double& pack_psnr, size_t& pack_texels)
{
    blocks_from_device(d, m, pack_psnr, pack_texels);
}

void bc_state_save(const DeviceModel* d, const Model& m, std::vector<std::vector<uint8_t>>& ep,
                   std::vector<std::vector<uint8_t>>& sel)
{
    const size_t np = m.planes.size();
    ep.assign(np, std::vector<uint8_t>());
    sel.assign(np, std::vector<uint8_t>());
    std::vector<uint8_t*> pe, ps;
    for (size_t i = 0; i < np; i++)
    {
        ep[i].assign(plane_blocks(m, i) * m.c0 * 2, 0);
        sel[i].assign(plane_blocks(m, i) * m.c0 * 16, 0);
        pe.push_back(ep[i].data());
        ps.push_back(sel[i].data());
    }
    NB_CALL(nntc_b200_bc_state_save(d->dev, &d->pod, pe.data(), ps.data()));
}

void bc_state_restore(DeviceModel* d, const Model& m, const std::vector<std::vector<uint8_t>>& ep,
                      const std::vector<std::vector<uint8_t>>& sel)
{
    const size_t np = m.planes.size();
    if (ep.size() != np || sel.size() != np)
        return;
    std::vector<const uint8_t*> pe, ps;
    for (size_t i = 0; i < np; i++)
    {
        pe.push_back(ep[i].data());
        ps.push_back(sel[i].data());
    }
    NB_CALL(nntc_b200_bc_state_restore(d->dev, &d->pod, pe.data(), ps.data()));
}

}   // namespace nntc_cuda

// The per-kernel harness's reads (src/backend_check_probe.h:20-37).
namespace nntc_probe
{

void normal_equations(DeviceModel* d, const Model& m, std::vector<double>& out)
{
    const int mm = m.dec.nin + 1;
    out.assign((size_t)(mm * (mm + 1) / 2 + m.nout * mm), 0.0);
    NB_CALL(nntc_b200_probe_normal_equations(d->dev, out.data(), out.size()));
}

void workspace(DeviceModel* d, const Model& m, int plane, bool level0, Workspace& w)
{
    w = Workspace();
    if (level0 && !m.l0_bc8)
        return;
    const PlaneSize& p = m.planes[(size_t)plane];
    const size_t t = level0 ? (size_t)p.w0 * p.h0 : (size_t)p.w1 * p.h1;
    const size_t c = (size_t)(level0 ? m.c0 : m.c1);
    w.stencil.resize(t * 5 * c * c);
    w.grad.resize(t * c);
    w.precond.resize(t * c * c);
    w.cg_x.resize(t * c);
    w.prev.resize(t * c);
    NB_CALL(nntc_b200_probe_workspace(d->dev, plane, level0 ? 1 : 0, w.stencil.data(), w.grad.data(),
                                      w.precond.data(), w.cg_x.data(), w.prev.data()));
}

void monomials(DeviceModel* d, const Model& m, bool level0, std::vector<double>& out)
{
    if (level0 && !m.l0_bc8)
    {
        out.clear();
        return;
    }
    const int dim = level0 ? m.c0 : m.c1;
    out.assign((size_t)nntc_b200_stencil_monomials(level0 ? m.c1 : m.c0) * dim * dim, 0.0);
    NB_CALL(nntc_b200_probe_monomials(d->dev, level0 ? 1 : 0, out.data(), out.size()));
}

}   // namespace nntc_probe
