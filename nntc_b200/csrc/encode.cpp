// encode.cpp: the whole encode over the C ABI, the caller of the hot path.
//
// The round loop and the post-fit BC path of the reference's encoder (src/main.cpp:1930-2743), with its semantics:
// initialise both latents (level 1 by the box or pca rule, level 0 from the residual one channel at a time, each seed
// followed by a refit of the decoder); then rounds of (a) decoder, (b) level 1, (c') / (c) level 0, each followed by
// the objective, freezing both grids at --q1-start and switching to the quantised sweeps; the no-move and the
// two-consecutive-tol stops; the final sweeps or snaps; then under --l0 bc8 the seed pack, its refinement, the level-1
// and decoder refit, and up to --bc-outer repack passes accepted only when the shipped E falls (a rejected pass is
// restored exactly, src/main.cpp:2557-2668). The reporting, the asset writer and the option parsing stay with the
// host that calls this; what is returned is the model and the per-phase times.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "device.cuh"

namespace
{

constexpr double E_REL = 1e-6, E_NOISE = 1e-8;   // src/main.cpp:371-372 (the rise warning, not a decision)

// Both latents' planes, indices and BC state of every plane, copied device to device into the device's `keep`
// slice: what the outer repack loop restores when a pass does not lower the shipped E.
int snapshot(nntc_b200_device* d, bool save)
{
    if (!d->keep)
    {
        nb::set_error(NNTC_B200_ERR_STATE, "the outer repack loop runs only under --l0 bc8");
        return NNTC_B200_ERR_STATE;
    }
    size_t at = 0;
    int st = NNTC_B200_OK;
    nb::for_each_kept(d, [&](void* part, size_t bytes) {
        char* slot = (char*)d->keep + at;
        at += (bytes + 255) / 256 * 256;
        if (st != NNTC_B200_OK || bytes == 0)
            return;
        const cudaError_t e = save ? cudaMemcpyAsync(slot, part, bytes, cudaMemcpyDeviceToDevice, d->stream)
                                   : cudaMemcpyAsync(part, slot, bytes, cudaMemcpyDeviceToDevice, d->stream);
        if (e != cudaSuccess)
            st = nb::cuda_status(e, "cudaMemcpyAsync", __FILE__, __LINE__);
    });
    NB_TRY(st);
    NB_CUDA(cudaStreamSynchronize(d->stream));
    return NNTC_B200_OK;
}

}   // namespace

namespace nb
{
int descent_direction(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge, int level0);
int joint_apply(nntc_b200_device* d, const nntc_b200_model* m, int k, int level0, float alpha);
int psnr_base(nntc_b200_device* d, const nntc_b200_model* m, double* psnr);
int normal_equations_and_objective(nntc_b200_device* d, const nntc_b200_model* m, int k, const double* per_site,
                                   nntc_b200_objective* e, double* ms);
int solve_decoder_prepared(nntc_b200_device* d, nntc_b200_model* m, int k, const double* per_site);
}

namespace
{

constexpr double JOINT_PSNR_SLACK = 0.01;   // dB a texture's base-level PSNR may lose to the joint pass

// The adjoint form's joint pass (bc8, after the repack passes; the method is described in joint.cu): both latents step
// along their preconditioned objective gradients by the best of alpha in {1, 1/2, 1/4} (snapped onto their grids, the
// decoder held), the decoder is re-solved at the step taken, the step is re-packed into BC blocks and refined, and the
// whole pass is kept only when the shipped E falls below e_ship AND no texture's 8-bit PSNR at the base level falls
// by more than JOINT_PSNR_SLACK dB (checked first on the step before the re-pack, which then refuses it without the
// pack and the refinement); otherwise every part of the state is restored exactly. The guard exists because E
// is one sum over every texture: a step that lowers it can move error from the textures with the most of it onto
// the nearly exact ones (a binary metalness map loses decibels to a handful of texels that cross an 8-bit rounding
// boundary while E barely moves).
template <class Obj, class BlockA>
int joint_pass(nntc_b200_device* d, nntc_b200_model* m, const nntc_b200_encode_args* a, int k,
               const double* per_site, Obj objective, BlockA block_a, double& e_ship, nntc_b200_encode_result* r)
{
    (void)per_site;
    cudaEvent_t j0, j1;
    NB_CUDA(cudaEventCreate(&j0));
    NB_CUDA(cudaEventCreate(&j1));
    NB_CUDA(cudaEventRecord(j0, d->stream));
    // the pass's span, recorded on every way out
    auto finish = [&](int status) -> int {
        NB_CUDA(cudaEventRecord(j1, d->stream));
        NB_CUDA(cudaEventSynchronize(j1));
        float jm = 0.0f;
        NB_CUDA(cudaEventElapsedTime(&jm, j0, j1));
        r->ms_joint = jm;
        cudaEventDestroy(j0);
        cudaEventDestroy(j1);
        return status;
    };
    r->e_before_joint = e_ship;
    double psnr_before[6] = {};
    NB_TRY(nb::psnr_base(d, m, psnr_before));
    NB_TRY(snapshot(d, true));
    const nntc_b200_model keep_m = *m;
    auto restore = [&]() -> int {
        NB_TRY(snapshot(d, false));
        *m = keep_m;
        NB_TRY(nntc_b200_upload_decoder(d, m));
        return nntc_b200_upload_grids(d, m);
    };
    NB_TRY(nb::descent_direction(d, m, k, a->ridge, 0));
    NB_TRY(nb::descent_direction(d, m, k, a->ridge, 1));
    // the pass starts from the shipped state, whose E the caller measured (e_ship)
    nntc_b200_objective e{};
    double best_e = e_ship;
    float best = 0.0f;
    // the step lengths tried with the decoder held (E alone decides among them); the decoder is re-solved once, at
    // the step taken
    for (float alpha = 1.0f; alpha >= 0.25f; alpha *= 0.5f)
    {
        NB_TRY(nb::joint_apply(d, m, k, 0, alpha));
        NB_TRY(nb::joint_apply(d, m, k, 1, alpha));
        NB_TRY(objective(e));
        if (e.e < best_e)
        {
            best_e = e.e;
            best = alpha;
        }
    }
    int st = NNTC_B200_OK;
    if (best == 0.0f)
        st = restore();
    else
    {
        *m = keep_m;
        NB_TRY(nntc_b200_upload_decoder(d, m));
        NB_TRY(nb::joint_apply(d, m, k, 0, best));
        NB_TRY(nb::joint_apply(d, m, k, 1, best));
        NB_TRY(block_a());
        // the guard first on the step itself (its latents on their grids, before the BC re-pack, which only loses
        // quality): a texture already below the guard here is refused without the pack and the refinement
        double psnr_step[6] = {};
        NB_TRY(nb::psnr_base(d, m, psnr_step));
        bool early = true;
        for (int t = 0; t < m->textures && t < 6; t++)
            early = early && psnr_step[t] >= psnr_before[t] - JOINT_PSNR_SLACK;
        if (!early)
        {
            r->joint_taken = -1;
            NB_TRY(restore());
            return finish(NNTC_B200_OK);
        }
        double ms = 0.0;
        NB_TRY(nntc_b200_bc_pack_prepare(d, m, k, 1, nullptr, &ms));
        r->ms_pack += ms;
        std::vector<nntc_b200_bc_report> rp((size_t)(a->bc_refine > 0 ? a->bc_refine : 1));
        NB_TRY(nntc_b200_bc_refine(d, m, a->bc_refine, rp.data(), &ms));
        r->ms_refine += ms;
        NB_TRY(objective(e));
        r->e_joint = e.e;
        double psnr_after[6] = {};
        NB_TRY(nb::psnr_base(d, m, psnr_after));
        bool guard = true;
        for (int t = 0; t < m->textures && t < 6; t++)
            guard = guard && psnr_after[t] >= psnr_before[t] - JOINT_PSNR_SLACK;
        if (e.e < e_ship && guard)
        {
            e_ship = e.e;
            r->joint_taken = 1;
        }
        else
        {
            r->joint_taken = e.e < e_ship ? -1 : 0;
            st = restore();
        }
    }
    return finish(st);
}

}   // namespace

namespace nb
{
int channel_copies(nntc_b200_device* d, std::vector<unsigned char>& same);
}

using namespace nb;

extern "C"
{

void nntc_b200_encode_defaults(nntc_b200_encode_args* a)
{
    std::memset(a, 0, sizeof(*a));
    a->k = 4;
    a->rounds = 20;
    a->tol = 1e-4;
    a->q1_start = 3;
    a->q1_sweeps = 4;
    a->range_pct = 1;
    a->ridge = 1e-4;
    a->sweeps = 2;
    a->init_pca = 0;
    a->bc_refine = 4;
    a->bc_refine_after = 0;
    a->bc_outer = 2;
    a->luma[0] = 0.299f;
    a->luma[1] = 0.587f;
    a->luma[2] = 0.114f;
}

int nntc_b200_encode_on_device(nntc_b200_device* d, nntc_b200_model* m, const nntc_b200_encode_args* a,
                               const double* per_site, nntc_b200_encode_result* r, uint8_t* const* k0_out,
                               uint8_t* const* k1_out, uint8_t* const* ep_out, uint8_t* const* sel_out)
{
    *r = nntc_b200_encode_result{};
    const int np = m->nplanes, k = a->k;
    const bool bc8 = m->l0_bc8 != 0;
    // The adjoint + mixed-precision form: the tensor-core normal equations and the matrix-free conjugate gradients for
    // this encode, the device's own settings put back on every way out.
    struct FormScope
    {
        nntc_b200_device* d;
        int gram, cg, obj, sten;
        ~FormScope()
        {
            d->mixed_gram = gram;
            d->adjoint_cg = cg;
            d->mixed_objective = obj;
            d->mixed_stencil = sten;
        }
    } form_scope{ d, d->mixed_gram, d->adjoint_cg, d->mixed_objective, d->mixed_stencil };
    if (a->form == 1)
    {
        // the conjugate gradients run on the FP32 stencil: their matrix-free products (NNTC_B200_OPT_ADJOINT_CG)
        // measured several times slower per product on the B200 than reading the assembled FP32 stencil
        d->mixed_gram = 1;
        d->adjoint_cg = 0;
        d->mixed_objective = 1;
        d->mixed_stencil = 1;
    }
    else if (a->form != 0)
    {
        set_error(NNTC_B200_ERR_ARG, "form must be 0 (plain) or 1 (adjoint + mixed precision)");
        return NNTC_B200_ERR_ARG;
    }
    cudaEvent_t t0, t1;
    NB_CUDA(cudaEventCreate(&t0));
    NB_CUDA(cudaEventCreate(&t1));
    NB_CUDA(cudaEventRecord(t0, d->stream));
    const long long passes0 = nntc_b200_objective_passes();
    // The fractional sites' targets (a pure function of the source chain and K) are formed inside every encode, so an
    // encode's time does not depend on what an earlier encode on the same device model left behind.
    d->site_tgt_kc = -1;
    d->obj_tgt_kc = -1;

    // The start state (src/main.cpp:1838-1915): no decoder (the device's is zero), level 0's grid [-1, 1] under bc8,
    // no level-1 grid yet.
    std::memset(m->dec_w, 0, sizeof(m->dec_w));
    std::memset(m->dec_b, 0, sizeof(m->dec_b));
    m->has_decoder = 1;
    NB_TRY(nntc_b200_upload_decoder(d, m));
    m->has_decoder = 0;
    if (bc8)
    {
        m->has_lo0 = 1;
        for (int c = 0; c < m->c0; c++)
        {
            m->lo0[c] = -1.0f;
            m->hi0[c] = 1.0f;
        }
    }
    m->has_lo1 = 0;

    nntc_b200_objective e{};
    double ms = 0.0;
    auto objective = [&](nntc_b200_objective& out) {
        const int st = nntc_b200_objective_eval(d, m, k, per_site, &out);
        r->ms_e += out.ms;
        return st;
    };
    auto block_a = [&]() {
        double t = 0.0;
        const int st = nntc_b200_solve_decoder(d, m, k, per_site, &t);
        r->ms_a += t;
        return st;
    };

    // ---- initialisation (src/main.cpp:1930-2122)
    NB_TRY(nntc_b200_init_level0(d, m, a->luma, m->init0_residual ? 0 : 1, nullptr));
    nntc_b200_init1_report irep{};
    NB_TRY(nntc_b200_init_level1(d, m, a->init_pca, &irep, nullptr));
    if (!a->init_pca)
    {
        // The box init takes the source channels in order with every exact copy of an earlier channel moved to the
        // back (src/main.cpp:1938-2012); where that changes which channels are taken, level 1 is re-formed from them.
        const int nout = m->nout, taken = m->c1 < nout ? m->c1 : nout;
        std::vector<unsigned char> same;
        NB_TRY(channel_copies(d, same));
        std::vector<int> order, copies;
        for (int s2 = 0; s2 < nout; s2++)
        {
            bool copy = false;
            for (int e2 = 0; e2 < s2 && !copy; e2++)
                copy = same[(size_t)s2 * nout + e2] != 0;
            (copy ? copies : order).push_back(s2);
        }
        order.insert(order.end(), copies.begin(), copies.end());
        std::vector<int> chosen((size_t)taken);
        for (int c = 0; c < taken; c++)
            chosen[(size_t)c] = order[(size_t)c];
        std::sort(chosen.begin(), chosen.end());
        bool plain = true;
        for (int c = 0; c < taken; c++)
            plain = plain && chosen[(size_t)c] == c;
        if (!plain)
        {
            std::vector<std::vector<float>> src((size_t)np);
            for (int i = 0; i < np; i++)
            {
                src[(size_t)i].resize((size_t)m->w0[i] * m->h0[i] * nout);
                NB_TRY(download(d, src[(size_t)i].data(), d->planes[(size_t)i].src,
                                src[(size_t)i].size() * sizeof(float)));
            }
            for (int i = 0; i < np; i++)
            {
                const int w0 = m->w0[i], h0 = m->h0[i], w1 = m->w1[i], h1 = m->h1[i];
                std::vector<float> v1((size_t)w1 * h1 * m->c1);
                for (int y = 0; y < h1; y++)
                    for (int x = 0; x < w1; x++)
                    {
                        int xa = (int)((long long)x * w0 / w1), xb = (int)((long long)(x + 1) * w0 / w1);
                        int ya = (int)((long long)y * h0 / h1), yb = (int)((long long)(y + 1) * h0 / h1);
                        xb = std::min(w0, xb <= xa ? xa + 1 : xb);
                        yb = std::min(h0, yb <= ya ? ya + 1 : yb);
                        for (int c = 0; c < m->c1; c++)
                        {
                            const size_t t1 = (size_t)y * w1 + x;
                            if (c >= nout)
                            {
                                v1[t1 * m->c1 + c] = 0.0f;
                                continue;
                            }
                            const int sc = order[(size_t)c];
                            float acc = 0.0f;
                            int n = 0;
                            for (int sy = ya; sy < yb; sy++)
                                for (int sx = xa; sx < xb; sx++)
                                {
                                    acc += src[(size_t)i][((size_t)sy * w0 + sx) * nout + sc];
                                    n++;
                                }
                            const float inv = n > 0 ? 1.0f / (float)n : 0.0f;
                            v1[t1 * m->c1 + c] = 2.0f * acc * inv - 1.0f;
                        }
                    }
                NB_TRY(nntc_b200_level1_upload(d, i, v1.data(), v1.size()));
            }
            NB_TRY(nntc_b200_quantise_level1(d, m, 0, nullptr));
        }
    }
    NB_TRY(objective(e));
    r->e_init = e.e;
    NB_TRY(block_a());
    // E between the init's steps is the reference's report and decides nothing until the last one, which the first
    // round's stop test compares against; the adjoint form leaves the others out, the plain form keeps them
    const bool seeding = m->init0_residual && m->c0 > 0;
    if (a->form == 0 || !seeding)
        NB_TRY(objective(e));
    if (m->init0_residual)
        for (int c = 0; c < m->c0; c++)
        {
            nntc_b200_init0_report crep{};
            NB_TRY(nntc_b200_init0_residual_channel(d, m, c, per_site, &crep, nullptr));
            if (a->form == 0)
                NB_TRY(objective(e));
            NB_TRY(block_a());
            if (a->form == 0 || c == m->c0 - 1 || !bc8)
                NB_TRY(objective(e));
            if (!bc8)
            {
                std::vector<nntc_b200_level0_report> l0((size_t)np);
                NB_TRY(nntc_b200_solve_level0_all(d, m, k, a->sweeps, l0.data(), &ms));
                r->ms_c += ms;
                NB_TRY(block_a());
                NB_TRY(objective(e));
            }
        }

    // ---- the round loop (src/main.cpp:2165-2390)
    std::vector<nntc_b200_plane_report> lr((size_t)np), lr0((size_t)np);
    bool frozen = false;
    int tol_hits = 0;
    double e_prev = e.e;
    // the adjoint form closes a round with one pass that forms E and the next round's normal equations together (same
    // sites, same latents): `prepared` says the device holds those normal equations for the next block (a)
    bool prepared = false;
    for (int round = 1; round <= a->rounds; round++)
    {
        nntc_b200_objective ea{}, eb{}, ec{};
        if (prepared)
        {
            NB_TRY(nb::solve_decoder_prepared(d, m, k, per_site));
            prepared = false;
        }
        else
            NB_TRY(block_a());
        // E after blocks (a) and (b) is the reference's report (src/main.cpp's per-block lines) and decides nothing;
        // the adjoint form leaves it out, the plain form keeps the reference's passes
        if (a->form == 0)
            NB_TRY(objective(ea));
        if (a->q1_start > 0 && round >= a->q1_start && !frozen)
        {
            NB_TRY(nntc_b200_freeze_level1_grid(d, m, a->range_pct, nullptr));
            if (bc8)
                NB_TRY(nntc_b200_freeze_level0_grid(d, m, a->range_pct, nullptr));
            frozen = true;
        }
        if (frozen)
            NB_TRY(nntc_b200_sweep_level1_all(d, m, k, a->ridge, a->q1_sweeps, lr.data(), &ms));
        else
            NB_TRY(nntc_b200_solve_level1_all(d, m, k, a->ridge, lr.data(), &ms));
        r->ms_b += ms;
        long long moved1 = 0;
        double delta2 = 0.0, plane2 = 0.0;
        for (int p = 0; p < np; p++)
        {
            moved1 += lr[(size_t)p].quantised ? lr[(size_t)p].moved : lr[(size_t)p].moved_values;
            delta2 += lr[(size_t)p].delta2;
            plane2 += lr[(size_t)p].plane2;
        }
        if (a->form == 0)
            NB_TRY(objective(eb));
        long long moved0 = 0;
        if (bc8)
        {
            if (frozen)
                NB_TRY(nntc_b200_sweep_level0_cont_all(d, m, k, a->ridge, a->q1_sweeps, lr0.data(), &ms));
            else
                NB_TRY(nntc_b200_solve_level0_cont_all(d, m, k, a->ridge, lr0.data(), &ms));
            for (int p = 0; p < np; p++)
                moved0 += lr0[(size_t)p].quantised ? lr0[(size_t)p].moved : lr0[(size_t)p].moved_values;
        }
        else
        {
            std::vector<nntc_b200_level0_report> l0((size_t)np);
            NB_TRY(nntc_b200_solve_level0_all(d, m, k, a->sweeps, l0.data(), &ms));
            for (int p = 0; p < np; p++)
                moved0 += l0[(size_t)p].moved_total;
        }
        r->ms_c += ms;
        if (a->form == 1 && d->mixed_gram)
        {
            double t = 0.0;
            NB_TRY(nb::normal_equations_and_objective(d, m, k, per_site, &ec, &t));
            r->ms_a += t;
            prepared = true;
        }
        else
            NB_TRY(objective(ec));
        (void)E_REL;
        (void)E_NOISE;
        r->rounds_used = round;
        const double drop = ec.e > 0.0 ? (e_prev - ec.e) / ec.e : 0.0;
        e_prev = ec.e;
        const double dn = std::sqrt(delta2), pn = std::sqrt(plane2);
        const bool level1_still = frozen ? moved1 == 0 : dn <= 1e-7 * (pn > 0.0 ? pn : 1.0);
        if (moved0 == 0 && level1_still)
        {
            r->stop = 1;
            break;
        }
        tol_hits = drop < a->tol ? tol_hits + 1 : 0;
        if (tol_hits >= 2)
        {
            r->stop = 2;
            break;
        }
    }
    if (frozen)
        NB_TRY(nntc_b200_sweep_level1_all(d, m, k, a->ridge, a->q1_sweeps, lr.data(), &ms));
    else
        NB_TRY(nntc_b200_quantise_level1(d, m, a->range_pct, nullptr));
    r->ms_b += frozen ? ms : 0.0;
    if (bc8)
    {
        if (frozen)
        {
            NB_TRY(nntc_b200_sweep_level0_cont_all(d, m, k, a->ridge, a->q1_sweeps, lr0.data(), &ms));
            r->ms_c += ms;
        }
        else
            NB_TRY(nntc_b200_quantise_level0(d, m, a->range_pct, nullptr));
    }
    else
    {
        std::vector<nntc_b200_level0_report> l0((size_t)np);
        NB_TRY(nntc_b200_solve_level0_all(d, m, k, a->sweeps, l0.data(), &ms));
        r->ms_c += ms;
    }
    NB_TRY(block_a());
    NB_TRY(objective(e));
    r->e_after_rounds = e.e;

    // ---- the post-fit BC path (src/main.cpp:2485-2694)
    if (bc8)
    {
        auto refit_level1 = [&]() {
            const int st = nntc_b200_sweep_level1_all(d, m, k, a->ridge, a->q1_sweeps, lr.data(), &ms);
            r->ms_b += ms;
            return st;
        };
        nntc_b200_objective probe{};
        NB_TRY(nntc_b200_bc_pack_prepare(d, m, k, 1, nullptr, &ms));
        r->ms_pack += ms;
        std::vector<nntc_b200_bc_report> rp((size_t)(a->bc_refine > 0 ? a->bc_refine : 1));
        NB_TRY(nntc_b200_bc_refine(d, m, a->bc_refine, rp.data(), &ms));
        r->ms_refine += ms;
        NB_TRY(refit_level1());
        NB_TRY(block_a());
        NB_TRY(objective(probe));
        if (a->bc_refine_after > 0)
        {
            NB_TRY(nntc_b200_bc_pack_prepare(d, m, k, 0, nullptr, &ms));
            r->ms_pack += ms;
            std::vector<nntc_b200_bc_report> ra((size_t)a->bc_refine_after);
            NB_TRY(nntc_b200_bc_refine(d, m, a->bc_refine_after, ra.data(), &ms));
            r->ms_refine += ms;
            NB_TRY(objective(probe));
        }
        double e_ship = probe.e;
        for (int pass = 1; pass <= a->bc_outer; pass++)
        {
            // Everything a rejected pass would leave behind, kept on the device (src/main.cpp:2561-2590).
            NB_TRY(snapshot(d, true));
            const nntc_b200_model keep_m = *m;
            NB_TRY(refit_level1());
            NB_TRY(block_a());
            if (frozen)
                NB_TRY(nntc_b200_sweep_level0_cont_all(d, m, k, a->ridge, a->q1_sweeps, lr0.data(), &ms));
            else
            {
                NB_TRY(nntc_b200_solve_level0_cont_all(d, m, k, a->ridge, lr0.data(), &ms));
                NB_TRY(nntc_b200_snap_level0_on_grid(d, m, nullptr));
            }
            r->ms_c += ms;
            NB_TRY(nntc_b200_bc_pack_prepare(d, m, k, 1, nullptr, &ms));
            r->ms_pack += ms;
            NB_TRY(nntc_b200_bc_refine(d, m, a->bc_refine, rp.data(), &ms));
            r->ms_refine += ms;
            NB_TRY(objective(probe));
            if (probe.e < e_ship)
            {
                e_ship = probe.e;
                r->outer_taken++;
                continue;
            }
            NB_TRY(snapshot(d, false));
            *m = keep_m;
            NB_TRY(nntc_b200_upload_decoder(d, m));
            NB_TRY(nntc_b200_upload_grids(d, m));
            break;
        }
        if (a->form == 1)
            NB_TRY(joint_pass(d, m, a, k, per_site, objective, block_a, e_ship, r));
        NB_TRY(refit_level1());
        NB_TRY(block_a());
    }

    nntc_b200_objective shipped{};
    NB_TRY(objective(shipped));
    r->e_ship = shipped.e;
    r->centre_mse = shipped.centre_mse;
    r->sampled_mse = shipped.sampled_mse;
    NB_CUDA(cudaEventRecord(t1, d->stream));
    NB_CUDA(cudaEventSynchronize(t1));
    float total = 0.0f;
    NB_CUDA(cudaEventElapsedTime(&total, t0, t1));
    r->ms_total = total;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    r->objective_passes = nntc_b200_objective_passes() - passes0;

    // The per-texture 8-bit PSNR of the base level against the source bytes (src/main.cpp:2743, 3000-3060), summed
    // on the device.
    NB_TRY(psnr_base(d, m, r->psnr));
    for (int i = 0; i < np; i++)
    {
        if (k0_out && k0_out[i])
            NB_TRY(nntc_b200_level0_download(d, i, k0_out[i], (size_t)m->w0[i] * m->h0[i] * m->c0));
        if (k1_out && k1_out[i])
            NB_TRY(nntc_b200_level1_download_indices(d, i, k1_out[i], (size_t)m->w1[i] * m->h1[i] * m->c1));
    }
    if (bc8 && ((ep_out && ep_out[0]) || (sel_out && sel_out[0])))
        NB_TRY(nntc_b200_bc_state_save(d, m, ep_out, sel_out));
    return NNTC_B200_OK;
}

}   // extern "C"
