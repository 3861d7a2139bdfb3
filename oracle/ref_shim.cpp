// ref_shim.cpp: single seam calls of the REFERENCE's CPU arm (src/cpu/*.cpp, namespace nntc_cpu) on POD inputs.
//
// Test infrastructure only. It is compiled by oracle/Makefile together with the reference's own sources where they
// lie, into oracle/_ref/libnntc_ref.so, and the golden-vector script (tests/golden/make_golden.py) and the parity
// tests call it through ctypes to learn what the reference itself computes for a given input. It shares no code with
// the product: it translates the POD model of include/nntc_b200.h into the reference's Model (src/model.h:56-114) and
// calls nntc_cpu::* (src/cpu/cpu_backend.h:39-90), then reads results back out of the reference's own CpuModel
// (src/cpu/cpu_model.h), the same buffers its per-kernel harness reads (src/backend_check_probe.h:20-37).

// export.cpp writes PNGs and mips.cpp resizes through the reference's vendored single-header libraries, whose
// implementations the reference compiles into main.cpp (src/main.cpp:15-23); this library has no main.cpp.
#define STB_IMAGE_WRITE_IMPLEMENTATION
#define STB_IMAGE_RESIZE_IMPLEMENTATION
#include "stb_image_write.h"
#include "stb_image_resize2.h"
#undef STB_IMAGE_WRITE_IMPLEMENTATION
#undef STB_IMAGE_RESIZE_IMPLEMENTATION

#include <cstring>
#include <string>
#include <vector>

#include "cpu/cpu_backend.h"
#include "cpu/cpu_model.h"
#include "model.h"
#include "nntc_b200.h"

namespace
{

struct Session
{
    Model m;
    std::vector<Image> chain;
    nntc_cpu::CpuModel* d = nullptr;
};

void model_in(const nntc_b200_model& p, Model& m)
{
    m.textures = p.textures;
    m.nout = p.nout;
    m.width = p.width;
    m.height = p.height;
    m.source_width = p.width;
    m.source_height = p.height;
    m.c0 = p.c0;
    m.c1 = p.c1;
    m.bits0.assign(p.bits0, p.bits0 + p.c0);
    m.bits1 = p.bits1;
    m.bc0 = p.bc0 != 0;
    m.l0_bc8 = p.l0_bc8 != 0;
    m.init0_residual = p.init0_residual != 0;
    m.init0_texture = p.init0_texture != 0;
    m.init0_chain = p.init0_chain != 0;
    m.planes.assign((size_t)p.nplanes, PlaneSize());
    for (int i = 0; i < p.nplanes; i++)
    {
        m.planes[(size_t)i].w0 = p.w0[i];
        m.planes[(size_t)i].h0 = p.h0[i];
        m.planes[(size_t)i].w1 = p.w1[i];
        m.planes[(size_t)i].h1 = p.h1[i];
    }
    m.cw.assign(p.cw, p.cw + p.nout);
    m.dec.nin = p.nin;
    m.dec.nout = p.nout;
    if (p.has_decoder)
    {
        m.dec.w.assign(p.dec_w, p.dec_w + (size_t)p.nout * p.nin);
        m.dec.b.assign(p.dec_b, p.dec_b + p.nout);
    }
    else
    {
        m.dec.w.clear();
        m.dec.b.clear();
    }
    m.palette0.assign((size_t)p.c0, std::vector<float>());
    bool any_palette = false;
    for (int c = 0; c < p.c0; c++)
    {
        m.palette0[(size_t)c].assign(p.palette0[c], p.palette0[c] + p.palette0_len[c]);
        any_palette = any_palette || p.palette0_len[c] > 0;
    }
    if (!any_palette)
        m.palette0.clear();
    if (p.has_lo0)
    {
        m.lo0.assign(p.lo0, p.lo0 + p.c0);
        m.hi0.assign(p.hi0, p.hi0 + p.c0);
    }
    else
    {
        m.lo0.clear();
        m.hi0.clear();
    }
    if (p.has_lo1)
    {
        m.lo1.assign(p.lo1, p.lo1 + p.c1);
        m.hi1.assign(p.hi1, p.hi1 + p.c1);
    }
    else
    {
        m.lo1.clear();
        m.hi1.clear();
    }
    if (m.k0.size() != m.planes.size())
        m.k0.assign(m.planes.size(), std::vector<uint8_t>());
    if (m.k1.size() != m.planes.size())
        m.k1.assign(m.planes.size(), std::vector<uint8_t>());
}

void model_out(const Model& m, nntc_b200_model& p)
{
    p.has_decoder = !m.dec.w.empty() && !m.dec.b.empty();
    if (p.has_decoder)
    {
        std::memcpy(p.dec_w, m.dec.w.data(), m.dec.w.size() * sizeof(float));
        std::memcpy(p.dec_b, m.dec.b.data(), m.dec.b.size() * sizeof(float));
    }
    p.has_lo0 = !m.lo0.empty();
    for (size_t c = 0; c < m.lo0.size(); c++)
    {
        p.lo0[c] = m.lo0[c];
        p.hi0[c] = m.hi0[c];
    }
    p.has_lo1 = !m.lo1.empty();
    for (size_t c = 0; c < m.lo1.size(); c++)
    {
        p.lo1[c] = m.lo1[c];
        p.hi1[c] = m.hi1[c];
    }
}

void report_out(const Level1Report& r, nntc_b200_plane_report& o)
{
    std::memset(&o, 0, sizeof(o));
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
    o.quantised = r.quantised;
    o.sweeps = r.sweeps;
    o.moved = r.moved;
    o.ms_sweeps = r.ms_sweeps;
}

}   // namespace

extern "C"
{

// The reference's layout and mip weights (src/mips.cpp:25-40, 141-169), for the generator's own restatement to be
// checked against. sizes is 4 ints per plane; returns the plane count.
int ref_layout(int width, int height, int mip_min, int want_mips, int k, const char* kind, double mix, int* sizes,
               double* per_site)
{
    Model m;
    m.width = width;
    m.height = height;
    build_plane_sizes(m, mip_min, want_mips != 0);
    std::vector<double> share, site;
    build_mip_weights(m.planes, kind, mix, k, share, site);
    for (size_t i = 0; i < m.planes.size(); i++)
    {
        sizes[4 * i + 0] = m.planes[i].w0;
        sizes[4 * i + 1] = m.planes[i].h0;
        sizes[4 * i + 2] = m.planes[i].w1;
        sizes[4 * i + 3] = m.planes[i].h1;
        per_site[i] = site[i];
    }
    return (int)m.planes.size();
}

// The reference's default source chain (src/image.h:343-366, src/mips.cpp:53-70): each level the 2x2 box of the last.
void ref_source_chain(const float* base, int w, int h, int nc, int levels, float* const* out)
{
    Image cur;
    cur.w = w;
    cur.h = h;
    cur.nc = nc;
    cur.v.assign(base, base + (size_t)w * h * nc);
    for (int i = 0; i < levels; i++)
    {
        Image next;
        image_box(cur, next);
        std::memcpy(out[i], next.v.data(), next.v.size() * sizeof(float));
        cur = next;
    }
}

void* ref_open(const nntc_b200_model* pm, const float* const* chain, int threads)
{
    Session* s = new Session();
    model_in(*pm, s->m);
    s->chain.resize((size_t)pm->nplanes);
    for (int i = 0; i < pm->nplanes; i++)
    {
        Image& im = s->chain[(size_t)i];
        im.w = pm->w0[i];
        im.h = pm->h0[i];
        im.nc = pm->nout;
        im.v.assign(chain[i], chain[i] + (size_t)im.w * im.h * im.nc);
    }
    s->d = nntc_cpu::device_create(s->m, s->chain, threads);
    return s;
}

void ref_close(void* h)
{
    Session* s = (Session*)h;
    nntc_cpu::device_destroy(s->d);
    delete s;
}

// The decoder and the grids as the POD gives them, uploaded as the reference's restore path does.
void ref_sync_in(void* h, const nntc_b200_model* pm)
{
    Session* s = (Session*)h;
    model_in(*pm, s->m);
    if (!s->m.dec.w.empty())
        nntc_cpu::upload_decoder_to_device(s->d, s->m);
    nntc_cpu::upload_grids_to_device(s->d, s->m);
}

void ref_sync_out(void* h, nntc_b200_model* pm)
{
    model_out(((Session*)h)->m, *pm);
}

void ref_set_planes(void* h, int plane, const float* v0, const float* v1)
{
    Session* s = (Session*)h;
    const PlaneSize& p = s->m.planes[(size_t)plane];
    if (v0)
        nntc_cpu::level0_upload(s->d, s->m, plane,
                                std::vector<float>(v0, v0 + (size_t)p.w0 * p.h0 * s->m.c0));
    if (v1)
        nntc_cpu::level1_upload(s->d, s->m, plane,
                                std::vector<float>(v1, v1 + (size_t)p.w1 * p.h1 * s->m.c1));
}

void ref_set_indices(void* h, int plane, const uint8_t* k0, const uint8_t* k1)
{
    Session* s = (Session*)h;
    const PlaneSize& p = s->m.planes[(size_t)plane];
    if (k0)
    {
        std::vector<uint8_t> v(k0, k0 + (size_t)p.w0 * p.h0 * s->m.c0);
        nntc_cpu::level0_upload_indices(s->d, s->m, plane, v);
        s->m.k0[(size_t)plane] = v;
    }
    if (k1)
    {
        std::vector<uint8_t> v(k1, k1 + (size_t)p.w1 * p.h1 * s->m.c1);
        nntc_cpu::level1_upload_indices(s->d, s->m, plane, v);
        s->m.k1[(size_t)plane] = v;
    }
}

void ref_get_planes(void* h, int plane, float* v0, float* v1, uint8_t* k0, uint8_t* k1)
{
    Session* s = (Session*)h;
    const nntc_cpu::CpuPlane& p = s->d->planes[(size_t)plane];
    if (v0)
        std::memcpy(v0, p.v0.data(), p.v0.size() * sizeof(float));
    if (v1)
        std::memcpy(v1, p.v1.data(), p.v1.size() * sizeof(float));
    if (k0)
        std::memcpy(k0, p.k0.data(), p.k0.size());
    if (k1)
        std::memcpy(k1, p.k1.data(), p.k1.size());
}

// The host mirror m.k0 / m.k1, which the seam functions that write indices fill.
void ref_get_host_indices(void* h, int plane, uint8_t* k0, uint8_t* k1)
{
    Session* s = (Session*)h;
    if (k0 && plane < (int)s->m.k0.size())
        std::memcpy(k0, s->m.k0[(size_t)plane].data(), s->m.k0[(size_t)plane].size());
    if (k1 && plane < (int)s->m.k1.size())
        std::memcpy(k1, s->m.k1[(size_t)plane].data(), s->m.k1[(size_t)plane].size());
}

void ref_objective(void* h, int k, const double* per_site, nntc_b200_objective* out)
{
    Session* s = (Session*)h;
    Objective r;
    nntc_cpu::objective_eval(s->d, s->m, k, std::vector<double>(per_site, per_site + s->m.planes.size()), r);
    std::memset(out, 0, sizeof(*out));
    out->e = r.e;
    out->centre_mse = r.centre_mse;
    out->sampled_mse = r.sampled_mse;
    for (size_t i = 0; i < r.e_plane.size(); i++)
    {
        out->e_plane[i] = r.e_plane[i];
        out->centre_plane[i] = r.centre_plane[i];
    }
}

void ref_decode(void* h, int plane, uint8_t* rgb8)
{
    Session* s = (Session*)h;
    std::vector<uint8_t> out;
    nntc_cpu::decode_plane(s->d, s->m, plane, out);
    std::memcpy(rgb8, out.data(), out.size());
}

void ref_solve_decoder(void* h, int k, const double* per_site)
{
    Session* s = (Session*)h;
    nntc_cpu::solve_decoder(s->d, s->m, k, std::vector<double>(per_site, per_site + s->m.planes.size()));
}

void ref_ridge_tally(long long out[4])
{
    nntc_cpu::decoder_ridge_tally(out);
}

// The normal equations the last solve_decoder reduced (upper triangle of A, then the nout right-hand sides).
int ref_normal_equations(void* h, double* out)
{
    Session* s = (Session*)h;
    std::memcpy(out, s->d->reduction.data(), s->d->reduction.size() * sizeof(double));
    return (int)s->d->reduction.size();
}

// One block (b) / (c'): level0 picks the latent, sweeps > 0 takes the quantised path.
void ref_solve_block(void* h, int level0, int k, double ridge, int sweeps, nntc_b200_plane_report* rep)
{
    Session* s = (Session*)h;
    std::vector<Level1Report> r;
    if (level0)
    {
        if (sweeps > 0)
            nntc_cpu::sweep_level0_cont_all(s->d, s->m, k, ridge, sweeps, r);
        else
            nntc_cpu::solve_level0_cont_all(s->d, s->m, k, ridge, r);
    }
    else
    {
        if (sweeps > 0)
            nntc_cpu::sweep_level1_all(s->d, s->m, k, ridge, sweeps, r);
        else
            nntc_cpu::solve_level1_all(s->d, s->m, k, ridge, r);
    }
    for (size_t i = 0; i < r.size(); i++)
        report_out(r[i], rep[i]);
}

void ref_assemble_for_refine(void* h, int k)
{
    Session* s = (Session*)h;
    nntc_cpu::assemble_level0_for_refine(s->d, s->m, k);
}

void ref_monomials(void* h, int level0, double* out)
{
    Session* s = (Session*)h;
    const std::vector<double>& v = level0 ? s->d->mono0 : s->d->mono;
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}

void ref_workspace(void* h, int plane, int level0, double* stencil, double* grad, float* precond, double* cg_x,
                   float* prev)
{
    Session* s = (Session*)h;
    const nntc_cpu::CpuPlane& p = s->d->planes[(size_t)plane];
    auto put = [](auto* dst, const auto& src) {
        if (dst)
            std::memcpy(dst, src.data(), src.size() * sizeof(src[0]));
    };
    if (level0)
    {
        put(stencil, p.stencil0);
        put(grad, p.grad0);
        put(precond, p.precond0);
        put(cg_x, p.cg0_x);
        put(prev, p.q0_prev);
    }
    else
    {
        put(stencil, p.stencil);
        put(grad, p.grad);
        put(precond, p.precond);
        put(cg_x, p.cg_x);
        put(prev, p.q1_prev);
    }
}

// Writes stencil / grad / cg_x / prev of one plane's level-0 workspace, so a refinement can be replayed from a state
// the caller chose.
void ref_set_workspace0(void* h, int plane, const double* stencil, const double* grad, const double* cg_x,
                        const float* prev)
{
    Session* s = (Session*)h;
    nntc_cpu::CpuPlane& p = s->d->planes[(size_t)plane];
    if (stencil)
        std::memcpy(p.stencil0.data(), stencil, p.stencil0.size() * sizeof(double));
    if (grad)
        std::memcpy(p.grad0.data(), grad, p.grad0.size() * sizeof(double));
    if (cg_x)
        std::memcpy(p.cg0_x.data(), cg_x, p.cg0_x.size() * sizeof(double));
    if (prev)
        std::memcpy(p.q0_prev.data(), prev, p.q0_prev.size() * sizeof(float));
}

void ref_bc_prepare(void* h, int k, int seed)
{
    Session* s = (Session*)h;
    double psnr = 0.0;
    size_t texels = 0;
    nntc_cpu::bc_pack_prepare(s->d, s->m, k, seed != 0, psnr, texels);
}

void ref_bc_refine(void* h, int passes, nntc_b200_bc_report* rep)
{
    Session* s = (Session*)h;
    double psnr = 0.0;
    size_t texels = 0;
    std::vector<BcRefineReport> r;
    nntc_cpu::bc_refine(s->d, s->m, passes, r, psnr, texels);
    for (size_t i = 0; i < r.size(); i++)
    {
        rep[i].pass = r[i].pass;
        rep[i].blocks = r[i].blocks;
        rep[i].improved = r[i].improved;
        rep[i].delta_e = r[i].delta_e;
        rep[i].ms = r[i].ms;
    }
}

void ref_bc_state(void* h, int plane, uint8_t* ep, uint8_t* sel)
{
    Session* s = (Session*)h;
    const nntc_cpu::CpuPlane& p = s->d->planes[(size_t)plane];
    if (ep)
        std::memcpy(ep, p.bc_ep.data(), p.bc_ep.size());
    if (sel)
        std::memcpy(sel, p.bc_sel.data(), p.bc_sel.size());
}

void ref_bc_set_state(void* h, int plane, const uint8_t* ep, const uint8_t* sel)
{
    Session* s = (Session*)h;
    nntc_cpu::CpuPlane& p = s->d->planes[(size_t)plane];
    std::memcpy(p.bc_ep.data(), ep, p.bc_ep.size());
    std::memcpy(p.bc_sel.data(), sel, p.bc_sel.size());
}

// The .dds blocks of one plane as bc_blocks_from_device left them in the model (file-major).
int ref_bc_blocks(void* h, int plane, int file, uint8_t* out)
{
    Session* s = (Session*)h;
    if (plane >= (int)s->m.bc0_blocks.size() || file >= (int)s->m.bc0_blocks[(size_t)plane].size())
        return 0;
    const std::vector<uint8_t>& b = s->m.bc0_blocks[(size_t)plane][(size_t)file];
    if (out)
        std::memcpy(out, b.data(), b.size());
    return (int)b.size();
}

// The seed pack alone (src/export.cpp:294-328) over the model's k0 mirror.
void ref_pack_seed(void* h, int plane, uint8_t* ep, uint8_t* sel)
{
    Session* s = (Session*)h;
    std::vector<uint8_t> e, q;
    level0_pack_seed(s->m, plane, e, q);
    std::memcpy(ep, e.data(), e.size());
    std::memcpy(sel, q.data(), q.size());
}

void ref_init_level0(void* h, const float luma[3], int luma_channel0)
{
    Session* s = (Session*)h;
    nntc_cpu::init_level0(s->d, s->m, luma, luma_channel0 != 0);
}

void ref_init_level1(void* h, int pca, nntc_b200_init1_report* rep)
{
    Session* s = (Session*)h;
    Level1InitReport r;
    nntc_cpu::init_level1(s->d, s->m, pca != 0, r);
    rep->pca = r.pca;
    rep->components = r.components;
    for (int i = 0; i < 4; i++)
    {
        rep->eigenvalue[i] = r.eigenvalue[i];
        rep->peak[i] = r.peak[i];
    }
    rep->total_variance = r.total_variance;
}

void ref_init0_residual_channel(void* h, int channel, const double* plane_weight, nntc_b200_init0_report* rep)
{
    Session* s = (Session*)h;
    Init0ChannelReport r;
    nntc_cpu::init0_residual_channel(s->d, s->m, channel,
                                     std::vector<double>(plane_weight, plane_weight + s->m.planes.size()), r);
    rep->eigenvalue = r.eigenvalue;
    rep->total_variance = r.total_variance;
    rep->share = r.share;
    rep->peak = r.peak;
    rep->divisor = r.divisor;
    for (int i = 0; i < 18; i++)
        rep->dir[i] = r.dir[i];
    rep->nout = r.nout;
    rep->texture = r.texture;
}

// which: 0 quantise_level1, 1 freeze_level1_grid, 2 quantise_level0, 3 freeze_level0_grid, 4 snap_level0_on_grid
void ref_grid(void* h, int which, int range_pct)
{
    Session* s = (Session*)h;
    const std::string policy = range_pct ? "pct" : "minmax";
    switch (which)
    {
    case 0:
        nntc_cpu::quantise_level1(s->d, s->m, policy);
        break;
    case 1:
        nntc_cpu::freeze_level1_grid(s->d, s->m, policy);
        break;
    case 2:
        nntc_cpu::quantise_level0(s->d, s->m, policy);
        break;
    case 3:
        nntc_cpu::freeze_level0_grid(s->d, s->m, policy);
        break;
    default:
        nntc_cpu::snap_level0_on_grid(s->d, s->m);
        break;
    }
}

void ref_solve_level0_palette(void* h, int k, int sweeps, nntc_b200_level0_report* rep)
{
    Session* s = (Session*)h;
    std::vector<Level0Report> r;
    nntc_cpu::solve_level0_all(s->d, s->m, k, sweeps, r);
    for (size_t i = 0; i < r.size(); i++)
    {
        for (int c = 0; c < 4; c++)
            rep[i].moved[c] = r[i].moved[c];
        rep[i].moved_total = r[i].moved_total;
        rep[i].ms = r[i].ms;
        rep[i].joint = r[i].joint;
        rep[i].states = r[i].states;
    }
}

}   // extern "C"
