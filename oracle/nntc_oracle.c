/* nntc_oracle.c: the plain-C restatement of the encoder's hot path (see nntc_oracle.h). TEST INFRASTRUCTURE ONLY.
 *
 * Built by oracle/Makefile with -ffp-contract=off, as the reference's CPU arm is (CMakeLists.txt:196-199), so float
 * and double expressions round exactly as they are written. */
#include "nntc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXC 4
#define MAXNIN 24
#define MAXNOUT 18
#define SLOTS 5

/* ---- the sampling rule, src/sample.cuh:43-178 ---- */

typedef struct
{
    int x0, x1, y0, y1;
    float fx, fy;
} tap;

static int clampi(int i, int n)
{
    return i < 0 ? 0 : (i >= n ? n - 1 : i);
}

static tap tap_at(int px, int py, float dx, float dy, int w0, int h0, int w, int h)
{
    const float x = w == w0 ? (float)px + dx : (((float)px + 0.5f + dx) * (float)w) / (float)w0 - 0.5f;
    const float y = h == h0 ? (float)py + dy : (((float)py + 0.5f + dy) * (float)h) / (float)h0 - 0.5f;
    const int xf = (int)floorf(x), yf = (int)floorf(y);
    tap t;
    t.fx = x - (float)xf;
    t.fy = y - (float)yf;
    t.x0 = clampi(xf, w);
    t.x1 = clampi(xf + 1, w);
    t.y0 = clampi(yf, h);
    t.y1 = clampi(yf + 1, h);
    return t;
}

static void corner_weights(const tap* t, float w[4])
{
    w[0] = (1.0f - t->fx) * (1.0f - t->fy);
    w[1] = t->fx * (1.0f - t->fy);
    w[2] = (1.0f - t->fx) * t->fy;
    w[3] = t->fx * t->fy;
}

static void blend(const float* plane, int w, int c, const tap* t, float* out)
{
    const float* a = plane + ((size_t)t->y0 * w + t->x0) * c;
    const float* b = plane + ((size_t)t->y0 * w + t->x1) * c;
    const float* e = plane + ((size_t)t->y1 * w + t->x0) * c;
    const float* f = plane + ((size_t)t->y1 * w + t->x1) * c;
    float wt[4];
    corner_weights(t, wt);
    for (int k = 0; k < c; k++)
        out[k] = wt[0] * a[k] + wt[1] * b[k] + wt[2] * e[k] + wt[3] * f[k];
}

static void subtexel(int kc, int j, int tx, int ty, float* dx, float* dy)
{
    if (kc == 2)
    {
        *dx = j == 0 ? -0.25f : 0.25f;
        *dy = j == 0 ? 0.25f : -0.25f;
        return;
    }
    float ox = 0.25f, oy = 0.25f;
    if (kc == 4)
    {
        static const float ax[4] = { -0.375f, -0.125f, 0.125f, 0.375f };
        static const float ay[4] = { -0.125f, 0.375f, -0.375f, 0.125f };
        ox = ax[j];
        oy = ay[j];
    }
    const int turns = (ty & 1) * 2 + (tx & 1);
    for (int r = 0; r < turns; r++)
    {
        const float t = ox;
        ox = -oy;
        oy = t;
    }
    *dx = ox;
    *dy = oy;
}

static void site_offset(int kc, int j, int px, int py, float* dx, float* dy)
{
    *dx = 0.0f;
    *dy = 0.0f;
    if (j > 0)
        subtexel(kc, j - 1, px, py, dx, dy);
}

/* ---- grids, src/model.h:141-199 ---- */

int orc_rep_index(int k, int bits)
{
    unsigned b8 = 0;
    for (int sh = 8 - bits; sh > -bits; sh -= bits)
        b8 |= sh >= 0 ? ((unsigned)k << sh) : ((unsigned)k >> -sh);
    return (int)(b8 & 0xFFu);
}

float orc_grid_value(float lo, float hi, int bits, int k)
{
    const double span = (double)hi - (double)lo;
    const double frac = (double)orc_rep_index(k, bits) / 255.0;
    return (float)((double)lo + frac * span);
}

int orc_grid_index(float lo, float hi, int bits, float value)
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
    double best_d = fabs((double)value - (double)orc_grid_value(lo, hi, bits, k));
    for (int dd = -1; dd <= 1; dd += 2)
    {
        const int n = k + dd;
        if (n < 0 || n > levels)
            continue;
        const double dist = fabs((double)value - (double)orc_grid_value(lo, hi, bits, n));
        if (dist < best_d || (dist == best_d && n < best))
        {
            best_d = dist;
            best = n;
        }
    }
    return best;
}

/* ---- the objective, src/objective.cu:317-380 ---- */

static void sample_d(const float* plane, int w, int h, int c, double u, double v, double* out)
{
    const double x = u * (double)w - 0.5, y = v * (double)h - 0.5;
    const double xf = floor(x), yf = floor(y);
    const double fx = x - xf, fy = y - yf;
    const int x0 = clampi((int)xf, w), x1 = clampi((int)xf + 1, w);
    const int y0 = clampi((int)yf, h), y1 = clampi((int)yf + 1, h);
    for (int q = 0; q < c; q++)
    {
        const double a = plane[((size_t)y0 * w + x0) * c + q], b = plane[((size_t)y0 * w + x1) * c + q];
        const double e = plane[((size_t)y1 * w + x0) * c + q], f = plane[((size_t)y1 * w + x1) * c + q];
        out[q] = (1.0 - fx) * (1.0 - fy) * a + fx * (1.0 - fy) * b + (1.0 - fx) * fy * e + fx * fy * f;
    }
}

void orc_objective_plane(const orc_plane* p, const orc_decoder* d, double out[3])
{
    const int c0 = d->c0, c1 = d->c1, nin = d->nin, nout = d->nout, k = d->k;
    out[0] = out[1] = out[2] = 0.0;
    for (int py = 0; py < p->h0; py++)
        for (int px = 0; px < p->w0; px++)
            for (int j = 0; j <= k; j++)
            {
                float dx = 0.0f, dy = 0.0f;
                if (j > 0)
                    subtexel(k, j - 1, px, py, &dx, &dy);
                const double u = ((double)px + 0.5 + (double)dx) / (double)p->w0;
                const double v = ((double)py + 0.5 + (double)dy) / (double)p->h0;
                double s[MAXC], c[MAXC], t[MAXNOUT], phi[MAXNIN];
                sample_d(p->v1, p->w1, p->h1, c1, u, v, c);
                if (j == 0)
                {
                    const size_t idx = (size_t)py * p->w0 + px;
                    for (int i = 0; i < c0; i++)
                        s[i] = p->v0[idx * c0 + i];
                    for (int i = 0; i < nout; i++)
                        t[i] = p->src[idx * nout + i];
                }
                else
                {
                    sample_d(p->v0, p->w0, p->h0, c0, u, v, s);
                    sample_d(p->src, p->w0, p->h0, nout, u, v, t);
                }
                int n = 0;
                for (int q = 0; q < c1; q++)
                    phi[n++] = c[q];
                for (int i = 0; i < c0; i++)
                    phi[n++] = s[i];
                for (int i = 0; i < c0; i++)
                    for (int q = 0; q < c1; q++)
                        phi[n++] = s[i] * c[q];
                for (int row = 0; row < nout; row++)
                {
                    double y = (double)d->b[row];
                    for (int i = 0; i < nin; i++)
                        y += (double)d->w[(size_t)row * nin + i] * phi[i];
                    const double e = y - t[row];
                    out[0] += (double)d->cw[row] * e * e;
                    out[j == 0 ? 1 : 2] += e * e;
                }
            }
}

static int features(const float* s, int c0, const float* c, int c1, float* phi)
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

void orc_decode_plane(const orc_plane* p, const orc_decoder* d, uint8_t* rgb8)
{
    for (int py = 0; py < p->h0; py++)
        for (int px = 0; px < p->w0; px++)
        {
            const size_t idx = (size_t)py * p->w0 + px;
            float s[MAXC], c[MAXC], phi[MAXNIN];
            for (int i = 0; i < d->c0; i++)
                s[i] = p->v0[idx * d->c0 + i];
            const tap t = tap_at(px, py, 0.0f, 0.0f, p->w0, p->h0, p->w1, p->h1);
            blend(p->v1, p->w1, d->c1, &t, c);
            features(s, d->c0, c, d->c1, phi);
            for (int r = 0; r < d->nout; r++)
            {
                float acc = d->b[r];
                for (int i = 0; i < d->nin; i++)
                    acc += d->w[(size_t)r * d->nin + i] * phi[i];
                acc = acc < 0.0f ? 0.0f : (acc > 1.0f ? 1.0f : acc);
                rgb8[idx * d->nout + r] = (uint8_t)lroundf(acc * 255.0f);
            }
        }
}

/* The site's phi and target in float, the solver's arithmetic (src/sample.cuh:154-178). */
static void site_row(const orc_plane* p, const orc_decoder* d, int j, int px, int py, float* phi, float* target)
{
    float dx, dy, s[MAXC], c[MAXC];
    site_offset(d->k, j, px, py, &dx, &dy);
    const tap t1 = tap_at(px, py, dx, dy, p->w0, p->h0, p->w1, p->h1);
    blend(p->v1, p->w1, d->c1, &t1, c);
    if (j == 0)
    {
        const size_t idx = (size_t)py * p->w0 + px;
        for (int i = 0; i < d->c0; i++)
            s[i] = p->v0[idx * d->c0 + i];
        for (int i = 0; i < d->nout; i++)
            target[i] = p->src[idx * d->nout + i];
    }
    else
    {
        const tap t0 = tap_at(px, py, dx, dy, p->w0, p->h0, p->w0, p->h0);
        blend(p->v0, p->w0, d->c0, &t0, s);
        blend(p->src, p->w0, d->nout, &t0, target);
    }
    features(s, d->c0, c, d->c1, phi);
}

static int tri_index(int i, int j, int mm)
{
    return i * mm - i * (i - 1) / 2 + (j - i);
}

void orc_normal_equations_plane(const orc_plane* p, const orc_decoder* d, double* entries)
{
    const int mm = d->nin + 1, tri = mm * (mm + 1) / 2, nout = d->nout;
    memset(entries, 0, (size_t)(tri + nout * mm) * sizeof(double));
    for (int py = 0; py < p->h0; py++)
        for (int px = 0; px < p->w0; px++)
            for (int j = 0; j <= d->k; j++)
            {
                float v[MAXNIN + 1], t[MAXNOUT];
                site_row(p, d, j, px, py, v, t);
                v[d->nin] = 1.0f;
                for (int a = 0; a < mm; a++)
                    for (int b = a; b < mm; b++)
                        entries[tri_index(a, b, mm)] += (double)v[a] * (double)v[b];
                for (int c = 0; c < nout; c++)
                    for (int a = 0; a < mm; a++)
                        entries[tri + c * mm + a] += (double)t[c] * (double)v[a];
            }
}

static int gauss_jordan(double* g, int m, int nrhs)
{
    const int cols = m + nrhs;
    for (int k = 0; k < m; k++)
    {
        int pivot = k;
        double best = fabs(g[(size_t)k * cols + k]);
        for (int i = k + 1; i < m; i++)
        {
            const double a = fabs(g[(size_t)i * cols + k]);
            if (a > best)
            {
                best = a;
                pivot = i;
            }
        }
        if (best == 0.0)
            return 0;
        if (pivot != k)
            for (int j = 0; j < cols; j++)
            {
                const double t = g[(size_t)k * cols + j];
                g[(size_t)k * cols + j] = g[(size_t)pivot * cols + j];
                g[(size_t)pivot * cols + j] = t;
            }
        const double inv = 1.0 / g[(size_t)k * cols + k];
        for (int j = 0; j < cols; j++)
            g[(size_t)k * cols + j] *= inv;
        for (int i = 0; i < m; i++)
        {
            if (i == k)
                continue;
            const double f = g[(size_t)i * cols + k];
            if (f == 0.0)
                continue;
            for (int j = 0; j < cols; j++)
                g[(size_t)i * cols + j] -= f * g[(size_t)k * cols + j];
        }
    }
    return 1;
}

static double qform(const double* acc, const double* x, int mm, int nout, const float* cw, double inv_norm,
                    double* err)
{
    const int tri = mm * (mm + 1) / 2;
    double q = 0.0, e = 0.0;
    for (int c = 0; c < nout; c++)
    {
        double qc = 0.0, ec = 0.0;
        for (int i = 0; i < mm; i++)
        {
            for (int j = 0; j < mm; j++)
            {
                const double a = i <= j ? acc[tri_index(i, j, mm)] : acc[tri_index(j, i, mm)];
                qc += x[(size_t)c * mm + i] * a * x[(size_t)c * mm + j];
                ec += fabs(x[(size_t)c * mm + i]) * fabs(a) * fabs(x[(size_t)c * mm + j]);
            }
            qc -= 2.0 * x[(size_t)c * mm + i] * acc[tri + c * mm + i];
            ec += 2.0 * fabs(x[(size_t)c * mm + i]) * fabs(acc[tri + c * mm + i]);
        }
        q += (double)cw[c] * qc;
        e += (double)cw[c] * ec;
    }
    *err = 2.220446049250313e-16 * (double)mm * e * inv_norm;
    return q;
}

int orc_decoder_solve(const double* acc, int nin, int nout, const float* cw, double inv_norm, int norm_ok,
                      int had_previous, float* w, float* b)
{
    static const double ladder[3] = { 1e-9, 1e-12, 0.0 };
    const int mm = nin + 1, tri = mm * (mm + 1) / 2, cols = mm + nout;
    double trace = 0.0;
    for (int i = 0; i < mm; i++)
        trace += acc[tri_index(i, i, mm)];
    const double mean_diag = trace > 0.0 ? trace / mm : 1.0;
    double* x_prev = calloc((size_t)nout * mm, sizeof(double));
    double* x_new = calloc((size_t)nout * mm, sizeof(double));
    double* g = calloc((size_t)mm * cols, sizeof(double));
    if (had_previous)
        for (int c = 0; c < nout; c++)
        {
            for (int i = 0; i < nin; i++)
                x_prev[(size_t)c * mm + i] = w[(size_t)c * nin + i];
            x_prev[(size_t)c * mm + nin] = b[c];
        }
    double err_prev = 0.0;
    const double q_prev = had_previous ? qform(acc, x_prev, mm, nout, cw, inv_norm, &err_prev) : 0.0;
    int accepted = 0, taken = 0;
    for (int step = 0; step < 3 && !accepted; step++)
    {
        const double ridge = ladder[step] * mean_diag;
        memset(g, 0, (size_t)mm * cols * sizeof(double));
        for (int i = 0; i < mm; i++)
        {
            for (int j = i; j < mm; j++)
            {
                const double a = acc[tri_index(i, j, mm)];
                g[(size_t)i * cols + j] = a;
                g[(size_t)j * cols + i] = a;
            }
            g[(size_t)i * cols + i] += ridge;
            for (int c = 0; c < nout; c++)
                g[(size_t)i * cols + mm + c] = acc[tri + c * mm + i];
        }
        if (!gauss_jordan(g, mm, nout))
            continue;
        int finite = 1;
        for (int c = 0; c < nout; c++)
            for (int i = 0; i < mm; i++)
            {
                const double v = (double)(float)g[(size_t)i * cols + mm + c];
                x_new[(size_t)c * mm + i] = v;
                finite = finite && isfinite(v);
            }
        if (!finite)
            continue;
        double err_cand = 0.0;
        const double q_cand = qform(acc, x_new, mm, nout, cw, inv_norm, &err_cand);
        if (!had_previous || (norm_ok && (q_cand - q_prev) * inv_norm + err_prev + err_cand <= 1e-12))
        {
            accepted = 1;
            taken = step;
        }
    }
    if (accepted)
        for (int c = 0; c < nout; c++)
        {
            for (int i = 0; i < nin; i++)
                w[(size_t)c * nin + i] = (float)x_new[(size_t)c * mm + i];
            b[c] = (float)x_new[(size_t)c * mm + nin];
        }
    else if (!had_previous)
    {
        const double count = acc[tri_index(nin, nin, mm)];
        for (int i = 0; i < nout * nin; i++)
            w[i] = 0.0f;
        for (int c = 0; c < nout; c++)
            b[c] = count > 0.0 ? (float)(acc[tri + c * mm + nin] / count) : 0.0f;
    }
    free(x_prev);
    free(x_new);
    free(g);
    return accepted ? taken : 3;
}

/* ---- the stencil, src/solve_level1.cu:142-581 ---- */

static int monomial_count(int c)
{
    return 1 + c + c * (c + 1) / 2;
}

static void form_product(const double* x, const double* z, int dim, int nout, const float* cw, double* out)
{
    for (int u = 0; u < dim; u++)
        for (int v = 0; v < dim; v++)
        {
            double s = 0.0;
            for (int r = 0; r < nout; r++)
                s += (double)cw[r] * x[(size_t)r * dim + u] * z[(size_t)r * dim + v];
            out[u * dim + v] += s;
        }
}

int orc_monomials(const orc_decoder* d, int level0, double* out)
{
    const int c0 = d->c0, c1 = d->c1, nout = d->nout, nin = d->nin;
    const int dim = level0 ? c0 : c1, terms = level0 ? c1 : c0;
    const int nmono = monomial_count(terms);
    double x0[MAXNOUT * MAXC], y[MAXC * MAXNOUT * MAXC];
    memset(out, 0, (size_t)nmono * dim * dim * sizeof(double));
    for (int r = 0; r < nout; r++)
    {
        const float* row = d->w + (size_t)r * nin;
        if (!level0)
        {
            for (int q = 0; q < c1; q++)
                x0[r * c1 + q] = row[q];
            for (int i = 0; i < c0; i++)
                for (int q = 0; q < c1; q++)
                    y[((size_t)i * nout + r) * c1 + q] = row[c1 + c0 + i * c1 + q];
        }
        else
        {
            for (int i = 0; i < c0; i++)
                x0[r * c0 + i] = row[c1 + i];
            for (int q = 0; q < c1; q++)
                for (int i = 0; i < c0; i++)
                    y[((size_t)q * nout + r) * c0 + i] = row[c1 + c0 + i * c1 + q];
        }
    }
    int slot = 0;
    form_product(x0, x0, dim, nout, d->cw, out);
    slot++;
    for (int i = 0; i < terms; i++, slot++)
    {
        const double* yi = y + (size_t)i * nout * dim;
        form_product(yi, x0, dim, nout, d->cw, out + (size_t)slot * dim * dim);
        form_product(x0, yi, dim, nout, d->cw, out + (size_t)slot * dim * dim);
    }
    for (int i = 0; i < terms; i++)
        for (int j = i; j < terms; j++, slot++)
        {
            const double* yi = y + (size_t)i * nout * dim;
            const double* yj = y + (size_t)j * nout * dim;
            form_product(yi, yj, dim, nout, d->cw, out + (size_t)slot * dim * dim);
            if (i != j)
                form_product(yj, yi, dim, nout, d->cw, out + (size_t)slot * dim * dim);
        }
    return nmono;
}

static void slot_offset(int slot, int* dx, int* dy)
{
    static const int ox[SLOTS] = { 0, 1, -1, 0, 1 };
    static const int oy[SLOTS] = { 0, 0, 1, 1, 1 };
    *dx = ox[slot];
    *dy = oy[slot];
}

static int slot_of(int dx, int dy)
{
    for (int s = 0; s < SLOTS; s++)
    {
        int ox, oy;
        slot_offset(s, &ox, &oy);
        if (ox == dx && oy == dy)
            return s;
    }
    return -1;
}

static void footprint(int ti, int n0, int n1, int* lo, int* hi)
{
    const double r = (double)n0 / (double)n1;
    *lo = (int)ceil(((double)ti - 0.5) * r - 1.0);
    *hi = (int)ceil(((double)ti + 1.5) * r) - 1;
    *lo = *lo < 0 ? 0 : *lo;
    *hi = *hi > n0 - 1 ? n0 - 1 : *hi;
}

static int merge_taps(const tap* t, int* nx, int* ny, float* tw)
{
    const int cx[4] = { t->x0, t->x1, t->x0, t->x1 };
    const int cy[4] = { t->y0, t->y0, t->y1, t->y1 };
    float cwt[4];
    corner_weights(t, cwt);
    int taps = 0;
    for (int q = 0; q < 4; q++)
    {
        int found = -1;
        for (int e = 0; e < taps; e++)
            if (nx[e] == cx[q] && ny[e] == cy[q])
                found = e;
        if (found >= 0)
            tw[found] += cwt[q];
        else
        {
            nx[taps] = cx[q];
            ny[taps] = cy[q];
            tw[taps] = cwt[q];
            taps++;
        }
    }
    return taps;
}

static void mono_values(const float* y, int n, double* out)
{
    int k = 0;
    out[k++] = 1.0;
    for (int i = 0; i < n; i++)
        out[k++] = (double)y[i];
    for (int i = 0; i < n; i++)
        for (int j = i; j < n; j++)
            out[k++] = (double)y[i] * (double)y[j];
}

void orc_assemble(const orc_plane* p, const orc_decoder* d, int level0, const double* mono, double* stencil,
                  double* grad)
{
    const int c0 = d->c0, c1 = d->c1, nin = d->nin, nout = d->nout, kc = d->k;
    const int c = level0 ? c0 : c1, nmono = monomial_count(level0 ? c1 : c0);
    const int tw_ = level0 ? p->w0 : p->w1, th_ = level0 ? p->h0 : p->h1;
    double sums[SLOTS * 15];
    for (int ty = 0; ty < th_; ty++)
        for (int tx = 0; tx < tw_; tx++)
        {
            const size_t ti = (size_t)ty * tw_ + tx;
            double g[MAXC] = { 0, 0, 0, 0 };
            for (int i = 0; i < SLOTS * nmono; i++)
                sums[i] = 0.0;
            int px_lo, px_hi, py_lo, py_hi;
            footprint(tx, p->w0, level0 ? p->w0 : p->w1, &px_lo, &px_hi);
            footprint(ty, p->h0, level0 ? p->h0 : p->h1, &py_lo, &py_hi);
            for (int py = py_lo; py <= py_hi; py++)
                for (int px = px_lo; px <= px_hi; px++)
                    for (int j = 0; j <= kc; j++)
                    {
                        float dx, dy, sbar[MAXC], cbar[MAXC], target[MAXNOUT], tw[4];
                        int nx[4], ny[4], taps = 0;
                        site_offset(kc, j, px, py, &dx, &dy);
                        const tap tp = tap_at(px, py, dx, dy, p->w0, p->h0, p->w1, p->h1);
                        if (!level0)
                            taps = merge_taps(&tp, nx, ny, tw);
                        blend(p->v1, p->w1, c1, &tp, cbar);
                        if (j == 0)
                        {
                            const size_t pi = (size_t)py * p->w0 + px;
                            for (int i = 0; i < c0; i++)
                                sbar[i] = p->v0[pi * c0 + i];
                            for (int r = 0; r < nout; r++)
                                target[r] = p->src[pi * nout + r];
                            if (level0)
                            {
                                nx[0] = px;
                                ny[0] = py;
                                tw[0] = 1.0f;
                                taps = 1;
                            }
                        }
                        else
                        {
                            const tap t0 = tap_at(px, py, dx, dy, p->w0, p->h0, p->w0, p->h0);
                            blend(p->v0, p->w0, c0, &t0, sbar);
                            blend(p->src, p->w0, nout, &t0, target);
                            if (level0)
                                taps = merge_taps(&t0, nx, ny, tw);
                        }
                        int self = -1;
                        for (int e = 0; e < taps; e++)
                            if (nx[e] == tx && ny[e] == ty)
                                self = e;
                        if (self < 0)
                            continue;
                        float mat[MAXNOUT * MAXC], res[MAXNOUT];
                        for (int r = 0; r < nout; r++)
                        {
                            const float* row = d->w + (size_t)r * nin;
                            float out = d->b[r];
                            if (!level0)
                            {
                                for (int i = 0; i < c0; i++)
                                    out += row[c1 + i] * sbar[i];
                                for (int q = 0; q < c1; q++)
                                {
                                    float gg = row[q];
                                    for (int i = 0; i < c0; i++)
                                        gg += sbar[i] * row[c1 + c0 + i * c1 + q];
                                    mat[r * c1 + q] = gg;
                                    out += gg * cbar[q];
                                }
                            }
                            else
                            {
                                for (int q = 0; q < c1; q++)
                                    out += row[q] * cbar[q];
                                for (int i = 0; i < c0; i++)
                                {
                                    float qq = row[c1 + i];
                                    for (int q = 0; q < c1; q++)
                                        qq += cbar[q] * row[c1 + c0 + i * c1 + q];
                                    mat[r * c0 + i] = qq;
                                    out += qq * sbar[i];
                                }
                            }
                            res[r] = out - target[r];
                        }
                        double mv[15];
                        mono_values(level0 ? cbar : sbar, level0 ? c1 : c0, mv);
                        const float w_self = tw[self];
                        for (int a = 0; a < c; a++)
                        {
                            double acc = 0.0;
                            for (int r = 0; r < nout; r++)
                                acc += (double)d->cw[r] * (double)mat[r * c + a] * (double)res[r];
                            g[a] += (double)w_self * acc;
                        }
                        for (int e = 0; e < taps; e++)
                        {
                            const int slot = slot_of(nx[e] - tx, ny[e] - ty);
                            if (slot < 0)
                                continue;
                            const double scale = (double)w_self * (double)tw[e];
                            for (int i = 0; i < nmono; i++)
                                sums[slot * nmono + i] += scale * mv[i];
                        }
                    }
            double* out_h = stencil + ti * (size_t)(SLOTS * c * c);
            for (int slot = 0; slot < SLOTS; slot++)
            {
                double* blk = out_h + (size_t)slot * c * c;
                for (int i = 0; i < c * c; i++)
                    blk[i] = 0.0;
                for (int i = 0; i < nmono; i++)
                {
                    const double s = sums[slot * nmono + i];
                    if (s == 0.0)
                        continue;
                    for (int e = 0; e < c * c; e++)
                        blk[e] += s * mono[(size_t)i * c * c + e];
                }
            }
            for (int i = 0; i < c; i++)
                grad[ti * c + i] = g[i];
        }
}

void orc_diag(const double* stencil, size_t texels, int c, double ridge, double out[4])
{
    double sum = 0.0, lo = 1e300, hi = -1e300;
    for (size_t t = 0; t < texels; t++)
        for (int a = 0; a < c; a++)
        {
            const double x = stencil[t * (size_t)(SLOTS * c * c) + (size_t)(a * c + a)];
            sum += x;
            lo = x < lo ? x : lo;
            hi = x > hi ? x : hi;
        }
    out[0] = sum;
    out[1] = lo;
    out[2] = hi;
    out[3] = texels > 0 ? ridge * sum / (double)(texels * (size_t)c) : 0.0;
}

static int invert(double* a, int n, double* inv)
{
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            inv[i * n + j] = i == j ? 1.0 : 0.0;
    for (int k = 0; k < n; k++)
    {
        int pivot = k;
        double best = fabs(a[k * n + k]);
        for (int i = k + 1; i < n; i++)
            if (fabs(a[i * n + k]) > best)
            {
                best = fabs(a[i * n + k]);
                pivot = i;
            }
        if (!(best > 0.0))
            return 0;
        if (pivot != k)
            for (int j = 0; j < n; j++)
            {
                double t = a[k * n + j];
                a[k * n + j] = a[pivot * n + j];
                a[pivot * n + j] = t;
                t = inv[k * n + j];
                inv[k * n + j] = inv[pivot * n + j];
                inv[pivot * n + j] = t;
            }
        const double s = 1.0 / a[k * n + k];
        for (int j = 0; j < n; j++)
        {
            a[k * n + j] *= s;
            inv[k * n + j] *= s;
        }
        for (int i = 0; i < n; i++)
        {
            if (i == k)
                continue;
            const double f = a[i * n + k];
            if (f == 0.0)
                continue;
            for (int j = 0; j < n; j++)
            {
                a[i * n + j] -= f * a[k * n + j];
                inv[i * n + j] -= f * inv[k * n + j];
            }
        }
    }
    return 1;
}

static void matvec(const double* st, int w, int h, int c, double lambda, const double* x, double* y)
{
    const size_t bs = (size_t)(SLOTS * c * c);
    for (int ty = 0; ty < h; ty++)
        for (int tx = 0; tx < w; tx++)
        {
            const size_t t = (size_t)ty * w + tx;
            const double* own = st + t * bs;
            double acc[MAXC];
            for (int i = 0; i < c; i++)
            {
                double s = lambda * x[t * c + i];
                for (int j = 0; j < c; j++)
                    s += own[i * c + j] * x[t * c + j];
                acc[i] = s;
            }
            for (int slot = 1; slot < SLOTS; slot++)
            {
                int dx, dy;
                slot_offset(slot, &dx, &dy);
                const int fx = tx + dx, fy = ty + dy;
                if (fx >= 0 && fx < w && fy >= 0 && fy < h)
                {
                    const double* blk = own + (size_t)slot * c * c;
                    const double* xn = x + ((size_t)fy * w + fx) * c;
                    for (int i = 0; i < c; i++)
                        for (int j = 0; j < c; j++)
                            acc[i] += blk[i * c + j] * xn[j];
                }
                const int bx = tx - dx, by = ty - dy;
                if (bx >= 0 && bx < w && by >= 0 && by < h)
                {
                    const size_t nt = (size_t)by * w + bx;
                    const double* blk = st + nt * bs + (size_t)slot * c * c;
                    const double* xn = x + nt * c;
                    for (int i = 0; i < c; i++)
                        for (int j = 0; j < c; j++)
                            acc[i] += blk[j * c + i] * xn[j];
                }
            }
            for (int i = 0; i < c; i++)
                y[t * c + i] = acc[i];
        }
}

static double dot(const double* a, const double* b, size_t n)
{
    double s = 0.0;
    for (size_t i = 0; i < n; i++)
        s += a[i] * b[i];
    return s;
}

static void precond_apply(const float* pc, const double* r, size_t texels, int c, double* z)
{
    for (size_t t = 0; t < texels; t++)
        for (int i = 0; i < c; i++)
        {
            double acc = 0.0;
            for (int j = 0; j < c; j++)
                acc += (double)pc[t * c * c + i * c + j] * r[t * c + j];
            z[t * c + i] = acc;
        }
}

int orc_pcg(const double* stencil, const double* grad, int w, int h, int c, double lambda, double* x,
            double* resid)
{
    const size_t texels = (size_t)w * h, n = texels * c;
    float* pc = malloc(texels * c * c * sizeof(float));
    double *r = malloc(n * sizeof(double)), *z = malloc(n * sizeof(double)), *p = malloc(n * sizeof(double)),
           *ap = malloc(n * sizeof(double));
    for (size_t t = 0; t < texels; t++)
    {
        double a[16], inv[16];
        for (int i = 0; i < c; i++)
            for (int j = 0; j < c; j++)
                a[i * c + j] = stencil[t * SLOTS * c * c + i * c + j] + (i == j ? lambda : 0.0);
        if (!invert(a, c, inv))
            for (int i = 0; i < c * c; i++)
                inv[i] = (i / c) == (i % c) ? 1.0 : 0.0;
        for (int i = 0; i < c * c; i++)
            pc[t * c * c + i] = (float)inv[i];
    }
    for (size_t i = 0; i < n; i++)
    {
        x[i] = 0.0;
        r[i] = -grad[i];
    }
    precond_apply(pc, r, texels, c, z);
    memcpy(p, z, n * sizeof(double));
    const double rhs2 = dot(r, r, n);
    double rz = dot(r, z, n), res = 0.0;
    int it = 0;
    for (; it < 200;)
    {
        matvec(stencil, w, h, c, lambda, p, ap);
        const double pap = dot(p, ap, n);
        const double alpha = pap > 0.0 ? rz / pap : 0.0;
        for (size_t i = 0; i < n; i++)
        {
            x[i] += 1.0 * alpha * p[i];
            r[i] += -1.0 * alpha * ap[i];
        }
        const double rr = dot(r, r, n);
        precond_apply(pc, r, texels, c, z);
        const double rz_new = dot(r, z, n);
        const double beta = rz != 0.0 ? rz_new / rz : 0.0;
        rz = rz_new;
        res = rhs2 > 0.0 ? sqrt((rr > 0.0 ? rr : 0.0) / rhs2) : 0.0;
        for (size_t i = 0; i < n; i++)
            p[i] = z[i] + beta * p[i];
        it++;
        if (it % 4 == 0 && !(res >= 1e-10))
            break;
    }
    *resid = res;
    free(pc);
    free(r);
    free(z);
    free(p);
    free(ap);
    return it;
}

long long orc_quant_sweeps(const double* stencil, const double* grad, const float* prev, int w, int h, int c,
                           double lambda, const float* lo, const float* hi, int bits, int sweeps, double* x, float* v,
                           uint8_t* k)
{
    const size_t bs = (size_t)(SLOTS * c * c);
    long long moved = 0;
    for (size_t i = 0; i < (size_t)w * h * c; i++)
        x[i] = 0.0;
    for (int s = 0; s < sweeps; s++)
        for (int colour = 0; colour < 4; colour++)
        {
            const int cx = colour & 1, cy = colour >> 1;
            for (int ty = cy; ty < h; ty += 2)
                for (int tx = cx; tx < w; tx += 2)
                {
                    const size_t t = (size_t)ty * w + tx;
                    const double* own = stencil + t * bs;
                    double nb[MAXC] = { 0, 0, 0, 0 };
                    for (int slot = 1; slot < SLOTS; slot++)
                    {
                        int dx, dy;
                        slot_offset(slot, &dx, &dy);
                        const int fx = tx + dx, fy = ty + dy;
                        if (fx >= 0 && fx < w && fy >= 0 && fy < h)
                        {
                            const double* blk = own + (size_t)slot * c * c;
                            const double* xn = x + ((size_t)fy * w + fx) * c;
                            for (int i = 0; i < c; i++)
                                for (int j = 0; j < c; j++)
                                    nb[i] += blk[i * c + j] * xn[j];
                        }
                        const int bx = tx - dx, by = ty - dy;
                        if (bx >= 0 && bx < w && by >= 0 && by < h)
                        {
                            const size_t nt = (size_t)by * w + bx;
                            const double* blk = stencil + nt * bs + (size_t)slot * c * c;
                            const double* xn = x + nt * c;
                            for (int i = 0; i < c; i++)
                                for (int j = 0; j < c; j++)
                                    nb[i] += blk[j * c + i] * xn[j];
                        }
                    }
                    for (int q = 0; q < c; q++)
                    {
                        const size_t idx = t * c + q;
                        const float l = lo[q], span = hi[q] - lo[q];
                        const double a = own[q * c + q] + lambda;
                        if (!(a > 0.0) || !(span > 0.0f))
                            continue;
                        double rest = nb[q];
                        for (int j = 0; j < c; j++)
                            if (j != q)
                                rest += own[q * c + j] * x[t * c + j];
                        const double b = grad[idx] + rest;
                        const double want = (double)prev[idx] - b / a;
                        const int kk = orc_grid_index(l, hi[q], bits, (float)want);
                        const float value = orc_grid_value(l, hi[q], bits, kk);
                        if ((int)k[idx] != kk)
                        {
                            k[idx] = (uint8_t)kk;
                            moved++;
                        }
                        v[idx] = value;
                        x[idx] = (double)value - (double)prev[idx];
                    }
                }
        }
    return moved;
}

/* ---- BC4 / BC5, shared/bc_pack.h:62-188, src/refine_bc.cu, src/cpu/cpu_refine_bc.cpp ---- */

static void bc4_palette(int r0, int r1, float p[8])
{
    p[0] = (float)r0;
    p[1] = (float)r1;
    if (r0 > r1)
        for (int i = 2; i < 8; i++)
            p[i] = (float)((8 - i) * r0 + (i - 1) * r1) / 7.0f;
    else
    {
        for (int i = 2; i < 6; i++)
            p[i] = (float)((6 - i) * r0 + (i - 1) * r1) / 5.0f;
        p[6] = 0.0f;
        p[7] = 255.0f;
    }
}

void orc_bc_seed(const uint8_t* k0, int w0, int h0, int c0, const int* bits, uint8_t* ep, uint8_t* sel)
{
    const int bx = (w0 + 3) / 4, by = (h0 + 3) / 4;
    for (int gy = 0; gy < by; gy++)
        for (int gx = 0; gx < bx; gx++)
            for (int c = 0; c < c0; c++)
            {
                int v[16], s[16], r0 = 0, r1 = 0;
                for (int t = 0; t < 16; t++)
                {
                    const int px = gx * 4 + t % 4 < w0 - 1 ? gx * 4 + t % 4 : w0 - 1;
                    const int py = gy * 4 + t / 4 < h0 - 1 ? gy * 4 + t / 4 : h0 - 1;
                    v[t] = orc_rep_index(k0[((size_t)py * w0 + px) * c0 + c], bits[c]);
                }
                const int b = bits[c];
                if (b == 3)
                {
                    r0 = 255;
                    r1 = 0;
                    for (int t = 0; t < 16; t++)
                    {
                        const int k = v[t] >> 5;
                        s[t] = k == 7 ? 0 : (k == 0 ? 1 : 8 - k);
                    }
                }
                else if (b == 2)
                {
                    r0 = 85;
                    r1 = 170;
                    for (int t = 0; t < 16; t++)
                    {
                        const int k = v[t] >> 6;
                        s[t] = k == 0 ? 6 : (k == 1 ? 0 : (k == 2 ? 1 : 7));
                    }
                }
                else if (b == 1)
                {
                    r0 = 0;
                    r1 = 255;
                    for (int t = 0; t < 16; t++)
                        s[t] = (v[t] >> 7) ? 7 : 6;
                }
                else
                {
                    const int levels = (1 << b) - 1;
                    int kmin = levels, kmax = 0;
                    for (int t = 0; t < 16; t++)
                    {
                        const int k = v[t] >> (8 - b);
                        kmin = k < kmin ? k : kmin;
                        kmax = k > kmax ? k : kmax;
                    }
                    r0 = (int)lround(kmax * 255.0 / levels);
                    r1 = (int)lround(kmin * 255.0 / levels);
                    if (r0 == r1)
                        for (int t = 0; t < 16; t++)
                            s[t] = 0;
                    else
                    {
                        float p[8];
                        bc4_palette(r0, r1, p);
                        for (int t = 0; t < 16; t++)
                        {
                            const float target = (float)(v[t] >> (8 - b)) * 255.0f / (float)levels;
                            int best = 0;
                            float best_d = 1e30f;
                            for (int i = 0; i < 8; i++)
                            {
                                const float dd = fabsf(p[i] - target);
                                if (dd < best_d)
                                {
                                    best_d = dd;
                                    best = i;
                                }
                            }
                            s[t] = best;
                        }
                    }
                }
                const size_t slot = ((size_t)gy * bx + gx) * c0 + c;
                ep[slot * 2] = (uint8_t)r0;
                ep[slot * 2 + 1] = (uint8_t)r1;
                for (int t = 0; t < 16; t++)
                    sel[slot * 16 + t] = (uint8_t)s[t];
            }
}

static double w8(int sel)
{
    return sel == 0 ? 1.0 : (sel == 1 ? 0.0 : (double)(8 - sel) / 7.0);
}

static float entry(int r0, int r1, int sel)
{
    if (sel == 0)
        return (float)r0;
    if (sel == 1)
        return (float)r1;
    return (float)((8 - sel) * r0 + (sel - 1) * r1) / 7.0f;
}

static float bc0_value(float lo, float hi, float byte)
{
    const double frac = (double)byte / 255.0;
    const double span = (double)hi - (double)lo;
    return (float)((double)lo + frac * span);
}

static uint8_t bc0_index(float byte)
{
    return (uint8_t)(byte < 0.0f ? 0 : (byte > 255.0f ? 255 : (int)(byte + 0.5f)));
}

void orc_bc_decode(const uint8_t* ep, const uint8_t* sel, const float* lo0, const float* hi0, int w0, int h0, int c0,
                   const float* prev, float* v0, uint8_t* k0, double* delta)
{
    const int bx = (w0 + 3) / 4;
    for (int py = 0; py < h0; py++)
        for (int px = 0; px < w0; px++)
        {
            const size_t ti = (size_t)py * w0 + px;
            const size_t gi = (size_t)(py / 4) * bx + (px / 4);
            const int t = (py % 4) * 4 + (px % 4);
            for (int c = 0; c < c0; c++)
            {
                const size_t b = gi * c0 + c;
                const float byte = entry(ep[b * 2], ep[b * 2 + 1], sel[b * 16 + t]);
                const float value = bc0_value(lo0[c], hi0[c], byte);
                v0[ti * c0 + c] = value;
                k0[ti * c0 + c] = bc0_index(byte);
                delta[ti * c0 + c] = (double)value - (double)prev[ti * c0 + c];
            }
        }
}

static double refine_block(const double* stencil, const double* grad, const float* prev, const float* lo0,
                           const float* hi0, int w0, int h0, int c0, int gx, int gy, uint8_t* ep, uint8_t* sel,
                           double* delta, float* v0, uint8_t* k0)
{
    const int n = 16 * c0, bx = (w0 + 3) / 4;
    double a2[64 * 64], a1[64], dv[64], uv[64], dlt[16];
    int s_ep[8];
    unsigned char s_sel[64];
    memset(a2, 0, sizeof(a2));
    memset(a1, 0, sizeof(a1));
    memset(dv, 0, sizeof(dv));
    memset(uv, 0, sizeof(uv));
    const size_t bs = (size_t)(SLOTS * c0 * c0);
    for (int tid = 0; tid < 16; tid++)
    {
        const int px = gx * 4 + (tid & 3), py = gy * 4 + (tid >> 2);
        if (!(px < w0 && py < h0))
            continue;
        const size_t ti = (size_t)py * w0 + px;
        const double* own = stencil + ti * bs;
        double acc[MAXC];
        for (int i = 0; i < c0; i++)
            acc[i] = grad[ti * c0 + i];
        for (int slot = 0; slot < SLOTS; slot++)
        {
            int dx, dy;
            slot_offset(slot, &dx, &dy);
            const int fx = px + dx, fy = py + dy;
            if (fx >= 0 && fx < w0 && fy >= 0 && fy < h0)
            {
                const double* blk = own + (size_t)slot * c0 * c0;
                const int lx = fx - gx * 4, ly = fy - gy * 4;
                if (lx >= 0 && lx < 4 && ly >= 0 && ly < 4)
                {
                    const int ft = ly * 4 + lx;
                    for (int i = 0; i < c0; i++)
                        for (int j = 0; j < c0; j++)
                        {
                            a2[(tid * c0 + i) * n + (ft * c0 + j)] += blk[i * c0 + j];
                            if (slot != 0)
                                a2[(ft * c0 + j) * n + (tid * c0 + i)] += blk[i * c0 + j];
                        }
                }
                else
                {
                    const double* xn = delta + ((size_t)fy * w0 + fx) * c0;
                    for (int i = 0; i < c0; i++)
                        for (int j = 0; j < c0; j++)
                            acc[i] += blk[i * c0 + j] * xn[j];
                }
            }
            if (slot == 0)
                continue;
            const int ax = px - dx, ay = py - dy;
            const int lx = ax - gx * 4, ly = ay - gy * 4;
            if (ax < 0 || ax >= w0 || ay < 0 || ay >= h0 || (lx >= 0 && lx < 4 && ly >= 0 && ly < 4))
                continue;
            const size_t nt = (size_t)ay * w0 + ax;
            const double* blk = stencil + nt * bs + (size_t)slot * c0 * c0;
            const double* xn = delta + nt * c0;
            for (int i = 0; i < c0; i++)
                for (int j = 0; j < c0; j++)
                    acc[i] += blk[j * c0 + i] * xn[j];
        }
        for (int i = 0; i < c0; i++)
        {
            a1[tid * c0 + i] = acc[i];
            dv[tid * c0 + i] = (double)v0[ti * c0 + i] - (double)prev[ti * c0 + i];
        }
    }
    for (int r = 0; r < n; r++)
    {
        double s = 0.0;
        for (int j = 0; j < n; j++)
            s += a2[r * n + j] * dv[j];
        uv[r] = s;
    }
    const size_t gi = (size_t)gy * bx + gx;
    for (int c = 0; c < c0; c++)
    {
        s_ep[2 * c] = ep[(gi * c0 + c) * 2];
        s_ep[2 * c + 1] = ep[(gi * c0 + c) * 2 + 1];
    }
    for (int i = 0; i < n; i++)
        s_sel[i] = sel[gi * c0 * 16 + i];
    double taken = 0.0;
    for (int c = 0; c < c0; c++)
    {
        const double step = ((double)hi0[c] - (double)lo0[c]) / 255.0;
        double bp = 0.0, bq = 0.0, pap = 0.0, paq = 0.0, qaq = 0.0;
        for (int tid = 0; tid < 16; tid++)
        {
            const int idx = tid * c0 + c;
            const double a = w8(s_sel[c * 16 + tid]);
            const double p = step * a;
            const double q = step * (1.0 - a);
            const double b = a1[idx] + uv[idx];
            double ap = 0.0, aq = 0.0;
            for (int j = 0; j < 16; j++)
            {
                const double e = a2[idx * n + (j * c0 + c)];
                const double aj = w8(s_sel[c * 16 + j]);
                ap += e * step * aj;
                aq += e * step * (1.0 - aj);
            }
            bp += b * p;
            bq += b * q;
            pap += p * ap;
            paq += p * aq;
            qaq += q * aq;
        }
        const int r0 = s_ep[2 * c], r1 = s_ep[2 * c + 1];
        const double det = pap * qaq - paq * paq;
        double d0 = 0.0, d1 = 0.0;
        if (det > 1e-12 * pap * qaq)
        {
            d0 = (paq * bq - qaq * bp) / det;
            d1 = (paq * bp - pap * bq) / det;
        }
        const int c0r = (int)floor((double)r0 + d0 + 0.5), c1r = (int)floor((double)r1 + d1 + 0.5);
        double best = 0.0;
        int best0 = r0, best1 = r1;
        for (int e0 = -1; e0 <= 1; e0++)
            for (int e1 = -1; e1 <= 1; e1++)
            {
                const int a0 = c0r + e0 < 0 ? 0 : (c0r + e0 > 255 ? 255 : c0r + e0);
                const int a1i = c1r + e1 < 0 ? 0 : (c1r + e1 > 255 ? 255 : c1r + e1);
                if (a0 <= a1i)
                    continue;
                const double f0 = (double)(a0 - r0), f1 = (double)(a1i - r1);
                const double de = 2.0 * (bp * f0 + bq * f1) + pap * f0 * f0 + 2.0 * paq * f0 * f1 + qaq * f1 * f1;
                if (de < best)
                {
                    best = de;
                    best0 = a0;
                    best1 = a1i;
                }
            }
        if (best0 == r0 && best1 == r1)
            continue;
        for (int tid = 0; tid < 16; tid++)
        {
            const float now = bc0_value(lo0[c], hi0[c], entry(r0, r1, s_sel[c * 16 + tid]));
            const float next = bc0_value(lo0[c], hi0[c], entry(best0, best1, s_sel[c * 16 + tid]));
            dlt[tid] = (double)next - (double)now;
        }
        double exact = 0.0;
        for (int tid = 0; tid < 16; tid++)
        {
            const int idx = tid * c0 + c;
            double quad = 0.0;
            for (int j = 0; j < 16; j++)
                quad += a2[idx * n + (j * c0 + c)] * dlt[j];
            exact += dlt[tid] * (2.0 * (a1[idx] + uv[idx]) + quad);
        }
        if (exact < 0.0)
        {
            for (int r = 0; r < n; r++)
            {
                double add = 0.0;
                for (int j = 0; j < 16; j++)
                    add += a2[r * n + (j * c0 + c)] * dlt[j];
                uv[r] += add;
            }
            s_ep[2 * c] = best0;
            s_ep[2 * c + 1] = best1;
            for (int j = 0; j < 16; j++)
                dv[j * c0 + c] += dlt[j];
            taken += exact;
        }
    }
    for (int pass = 0; pass < 2; pass++)
        for (int c = 0; c < c0; c++)
            for (int t = 0; t < 16; t++)
            {
                const int i = t * c0 + c;
                const double b = a1[i] + uv[i], a = a2[i * n + i];
                const int r0 = s_ep[2 * c], r1 = s_ep[2 * c + 1];
                const double now = (double)bc0_value(lo0[c], hi0[c], entry(r0, r1, s_sel[c * 16 + t]));
                double best = 0.0, move = 0.0;
                int which = s_sel[c * 16 + t];
                for (int kk = 0; kk < 8; kk++)
                {
                    const double dd = (double)bc0_value(lo0[c], hi0[c], entry(r0, r1, kk)) - now;
                    const double de = 2.0 * b * dd + a * dd * dd;
                    if (de < best)
                    {
                        best = de;
                        move = dd;
                        which = kk;
                    }
                }
                if (best < 0.0)
                {
                    for (int r = 0; r < n; r++)
                        uv[r] += a2[r * n + i] * move;
                    s_sel[c * 16 + t] = (unsigned char)which;
                    dv[i] += move;
                    taken += best;
                }
            }
    for (int c = 0; c < c0; c++)
    {
        ep[(gi * c0 + c) * 2] = (uint8_t)s_ep[2 * c];
        ep[(gi * c0 + c) * 2 + 1] = (uint8_t)s_ep[2 * c + 1];
    }
    for (int i = 0; i < n; i++)
        sel[gi * c0 * 16 + i] = s_sel[i];
    for (int tid = 0; tid < 16; tid++)
    {
        const int px = gx * 4 + (tid & 3), py = gy * 4 + (tid >> 2);
        if (!(px < w0 && py < h0))
            continue;
        const size_t ti = (size_t)py * w0 + px;
        for (int c = 0; c < c0; c++)
        {
            const float byte = entry(s_ep[2 * c], s_ep[2 * c + 1], s_sel[c * 16 + tid]);
            const float value = bc0_value(lo0[c], hi0[c], byte);
            v0[ti * c0 + c] = value;
            k0[ti * c0 + c] = bc0_index(byte);
            delta[ti * c0 + c] = (double)value - (double)prev[ti * c0 + c];
        }
    }
    return taken;
}

double orc_bc_refine_colour(const double* stencil, const double* grad, const float* prev, const float* lo0,
                            const float* hi0, int w0, int h0, int c0, int colour, uint8_t* ep, uint8_t* sel,
                            double* delta, float* v0, uint8_t* k0, long long* improved)
{
    const int bx = (w0 + 3) / 4, by = (h0 + 3) / 4, cx = colour & 1, cy = colour >> 1;
    double total = 0.0;
    for (int gy = cy; gy < by; gy += 2)
        for (int gx = cx; gx < bx; gx += 2)
        {
            const double t = refine_block(stencil, grad, prev, lo0, hi0, w0, h0, c0, gx, gy, ep, sel, delta, v0, k0);
            if (t < 0.0)
            {
                total += t;
                (*improved)++;
            }
        }
    return total;
}

/* ---- initialisation, src/init.cu ---- */

void orc_init_level1_box(const float* src, int w0, int h0, int nout, int w1, int h1, int c1, float* out)
{
    for (int y = 0; y < h1; y++)
        for (int x = 0; x < w1; x++)
        {
            int xa = (int)((long long)x * w0 / w1), xb = (int)((long long)(x + 1) * w0 / w1);
            int ya = (int)((long long)y * h0 / h1), yb = (int)((long long)(y + 1) * h0 / h1);
            if (xb <= xa)
                xb = xa + 1;
            if (yb <= ya)
                yb = ya + 1;
            xb = xb > w0 ? w0 : xb;
            yb = yb > h0 ? h0 : yb;
            float acc[MAXC] = { 0, 0, 0, 0 };
            int n = 0;
            for (int sy = ya; sy < yb; sy++)
                for (int sx = xa; sx < xb; sx++)
                {
                    const float* s = src + ((size_t)sy * w0 + sx) * nout;
                    for (int c = 0; c < c1; c++)
                        acc[c] += c < nout ? s[c] : 0.0f;
                    n++;
                }
            const float inv = n > 0 ? 1.0f / (float)n : 0.0f;
            for (int c = 0; c < c1; c++)
                out[((size_t)y * w1 + x) * c1 + c] = c < nout ? 2.0f * acc[c] * inv - 1.0f : 0.0f;
        }
}

void orc_residual(const orc_plane* p, const orc_decoder* d, float* resid)
{
    for (int py = 0; py < p->h0; py++)
        for (int px = 0; px < p->w0; px++)
        {
            const size_t idx = (size_t)py * p->w0 + px;
            float s[MAXC], c[MAXC], phi[MAXNIN];
            for (int i = 0; i < d->c0; i++)
                s[i] = p->v0[idx * d->c0 + i];
            const tap t = tap_at(px, py, 0.0f, 0.0f, p->w0, p->h0, p->w1, p->h1);
            blend(p->v1, p->w1, d->c1, &t, c);
            features(s, d->c0, c, d->c1, phi);
            for (int r = 0; r < d->nout; r++)
            {
                float acc = d->b[r];
                for (int i = 0; i < d->nin; i++)
                    acc += d->w[(size_t)r * d->nin + i] * phi[i];
                resid[idx * d->nout + r] = acc - p->src[idx * d->nout + r];
            }
        }
}
