// joint.cu: the objective's gradient with respect to both latents and the decoder, and the adjoint form's joint pass.
//
// E = sum_planes omega_p sum_sites sum_r cw_r (decode_r - target_r)^2 / (sum(cw) sum_planes omega_p w0 h0 (1 + K)).
// The decode is affine in the decoder and, site by site, in each latent's bilinear sample, so
//
//   dE/dv_t = 2 omega_p / norm  sum_{sites s reaching t} w_st J_s^T diag(cw) r_s     (J_s: G_s for level 1, Q_s for 0)
//   dE/dx_c = 2 cw_c / norm  (A x_c - rhs_c)                                            (x_c = [W_c | b_c])
//
// with A, rhs the omega-weighted normal equations of block (a) at the current latents. The latents' sums are the
// assembly's gradient (J^T diag(cw) r gathered per texel, the adjoint of the site's forward pass), the decoder's the
// normal equations' - one pass of the decode's adjoint over every site for each.
//
// The joint pass (the adjoint form's last step, under --l0 bc8): from the shipped state, both latents move along their
// preconditioned descent directions z = -(H_tt + lambda I)^-1 dE/dv (block Jacobi, the diagonal blocks the CG uses)
// by a step alpha in {1, 1/2, 1/4}, each snapped onto its grid; the alpha with the lowest E, if it lowers E, is taken
// with the decoder re-solved exactly at it (block (a) is the decoder's exact step given the latents), re-packed into BC
// blocks, refined, and kept only when the shipped E falls below the shipped E it started from and no texture's
// base-level 8-bit PSNR falls by more than 0.01 dB; otherwise everything (both latents, their indices, the BC state,
// the decoder and the grids) is restored exactly. The shipped E therefore never rises across the pass, and no texture
// pays for another's gain.

#include <cmath>
#include <cstring>
#include <vector>

#include "device.cuh"

namespace nb
{

int assemble(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge, int level0, bool diag_only);
int descent_direction(nntc_b200_device* d, const nntc_b200_model* m, int k, double ridge, int level0);
int normal_equations(nntc_b200_device* d, int k, const double* per_site, double* ms, std::vector<double>* obj_sums);

// v = prev + alpha z, then onto the grid (bits, lo, hi) with its index when `snap`.
__global__ void k_joint_apply(Planes P, float alpha, int snap, int bits, const float* lo, const float* hi)
{
    const long long base = (long long)blockIdx.x * blockDim.x;
    const int pl = plane_of(P, base);
    const PlaneView& V = P.p[pl];
    const long long t = base - P.start[pl] + threadIdx.x;
    if (t >= (long long)V.w * V.h)
        return;
    for (int a = 0; a < P.c; a++)
    {
        const size_t q = (size_t)t * P.c + a;
        const float x = (float)((double)V.prev[q] + (double)alpha * V.z[q]);
        if (snap)
        {
            const int kk = grid_index(lo[a], hi[a], bits, x);
            V.v[q] = grid_value(lo[a], hi[a], bits, kk);
            V.k[q] = (uint8_t)kk;
        }
        else
            V.v[q] = x;
    }
}

int joint_apply(nntc_b200_device* d, const nntc_b200_model* m, int k, int level0, float alpha)
{
    Planes P = planes_for(d, level0, [&](int i) { return d->planes[(size_t)i].work[level0 ? 1 : 0].texels(); });
    P.kc = k;
    const bool snap = level0 ? m->has_lo0 != 0 : m->has_lo1 != 0;
    k_joint_apply<<<(unsigned)(P.start[P.n] / THREADS), THREADS, 0, d->stream>>>(
        P, alpha, snap ? 1 : 0, level0 ? 8 : m->bits1, level0 ? d->lo0 : d->lo1, level0 ? d->hi0 : d->hi1);
    NB_LAUNCHED();
    return NNTC_B200_OK;
}

static double normaliser(const nntc_b200_model* m, int k, const double* per_site)
{
    double sum_cw = 0.0, den = 0.0;
    for (int c = 0; c < m->nout; c++)
        sum_cw += (double)m->cw[c];
    for (int i = 0; i < m->nplanes; i++)
        den += per_site[i] * (double)m->w0[i] * (double)m->h0[i] * (double)(1 + k);
    return sum_cw * den;
}

}   // namespace nb

using namespace nb;

extern "C" int nntc_b200_objective_gradient(nntc_b200_device* d, const nntc_b200_model* m, int k,
                                            const double* per_site, double* const* g_v0, double* const* g_v1,
                                            double* g_dec)
{
    if (k < 0 || k > 4 || k == 3)
    {
        set_error(NNTC_B200_ERR_ARG, "k must be 0, 1, 2 or 4");
        return NNTC_B200_ERR_ARG;
    }
    if (g_v0 && !d->l0_bc8)
    {
        set_error(NNTC_B200_ERR_STATE, "level 0's gradient is assembled only under --l0 bc8");
        return NNTC_B200_ERR_STATE;
    }
    const double norm = normaliser(m, k, per_site);
    if (!(norm > 0.0))
    {
        set_error(NNTC_B200_ERR_ARG, "the objective's normaliser is not positive");
        return NNTC_B200_ERR_ARG;
    }
    NB_TRY(upload_decoder(d, m));
    for (int level0 = 0; level0 < 2; level0++)
    {
        double* const* out = level0 ? g_v0 : g_v1;
        if (!out)
            continue;
        NB_TRY(assemble(d, m, k, 0.0, level0, true));
        for (size_t i = 0; i < d->planes.size(); i++)
        {
            if (!out[i])
                continue;
            const Work& w = d->planes[i].work[level0];
            NB_TRY(download(d, out[i], w.grad, w.values() * sizeof(double)));
            const double s = 2.0 * per_site[i] / norm;
            for (size_t q = 0; q < w.values(); q++)
                out[i][q] *= s;
        }
    }
    if (g_dec)
    {
        double t = 0.0;
        NB_TRY(normal_equations(d, k, per_site, &t, nullptr));
        const int nin = m->nin, nout = m->nout, mm = nin + 1, tri = mm * (mm + 1) / 2;
        std::vector<double> ne((size_t)(tri + nout * mm));
        NB_TRY(download(d, ne.data(), d->reduction, ne.size() * sizeof(double)));
        for (int c = 0; c < nout; c++)
            for (int i = 0; i < mm; i++)
            {
                double ax = 0.0;
                for (int j = 0; j < mm; j++)
                {
                    const double xj = j < nin ? (double)m->dec_w[c * nin + j] : (double)m->dec_b[c];
                    ax += ne[(size_t)tri_index(i < j ? i : j, i < j ? j : i, mm)] * xj;
                }
                g_dec[c * mm + i] = 2.0 * (double)m->cw[c] * (ax - ne[(size_t)tri + (size_t)c * mm + i]) / norm;
            }
    }
    return NNTC_B200_OK;
}

