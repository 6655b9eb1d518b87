/*
 * fdo_driver.c -- oracle time loops and the generated point kernels.
 *
 * TEST INFRASTRUCTURE ONLY (the checker of the CUDA path; see fdo.h).
 *
 * forward:  src/time_stepping.c:747-860 (one shot, one device)
 * adjoint:  src/time_stepping.c:862-940
 * sources:  src/automatic_kernels.c:394-629
 * varsout:  src/automatic_kernels.c:22-219
 * residuals src/automatic_kernels.c:631-836
 * gradient transform: src/calc_grad.c:975-1107
 * DFT gradient (BACK_PROP_TYPE=2): the same loops with the transforms of
 *   fdo_dft.c, src/time_stepping.c:766-781 (forward), :862-972 (adjoint)
 */

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "fdo.h"   /* after the system headers: FDO_FP64 retypes float */

typedef int64_t i64;

/* Which wave fields a source of `type` feeds, given the set of types used
 * anywhere in the acquisition (bit t for t = 0..3, bit 4 for type 100).
 * Restates the generated "sources" kernel: with a single target variable the
 * type is not checked; with several, a variable field is fed when the type
 * equals the variable's position in the model's variable list (the
 * reference's test at automatic_kernels.c:565-567), and the pressure
 * components when the type is 100 (:589-591).  div is the pressure split
 * (n2ave = ND), 0 for a direct field.  Returns the number of targets. */
int fdo_source_targets(int nd, int mask, int type, int *fields, float *div)
{
    /* model variable list order, src/assign_modeling_case.c:1049-1076 */
    static const int vl2[] = {W_VX, W_VZ, W_SXX, W_SZZ, W_SXZ};
    static const int vl3[] = {W_VX, W_VY, W_VZ, W_SXX, W_SZZ, W_SXZ, W_SXY, W_SYZ, W_SYY};
    static const int vl21[] = {W_VY, W_SXY, W_SYZ};
    static const int vl22[] = {W_VX, W_VZ, W_SXX}; /* vx, vz, p */
    /* the acoustic model has a variable named p; the others average p */
    int name_of_type[4] = {W_VX, W_VY, W_VZ, nd == 22 ? W_SXX : -1};
    const int *vl = nd == 3 ? vl3 : (nd == 21 ? vl21 : (nd == 22 ? vl22 : vl2));
    int nvl = nd == 3 ? 9 : (nd == 21 || nd == 22 ? 3 : 5);
    int has_p_average = nd == 2 || nd == 3;
    int tos[9] = {0};
    int tos_p = 0;
    for (int t = 0; t < 4; t++) {
        if (!(mask & (1 << t))) continue;
        if (name_of_type[t] >= 0)
            for (int j = 0; j < nvl; j++)
                if (vl[j] == name_of_type[t]) tos[j] = 1;
        if (t == 3 && has_p_average) tos_p = 1;
    }
    if ((mask & (1 << 4)) && has_p_average) tos_p = 1;
    int ntypes = tos_p;
    for (int j = 0; j < nvl; j++) ntypes += tos[j];
    int n = 0;
    for (int j = 0; j < nvl; j++)
        if (tos[j] && (ntypes == 1 || type == j)) { fields[n] = vl[j]; div[n] = 0; n++; }
    if (tos_p && (ntypes == 1 || type == 100)) {
        fields[n] = W_SXX; div[n] = (float)nd; n++;
        fields[n] = W_SZZ; div[n] = (float)nd; n++;
        if (nd == 3) { fields[n] = W_SYY; div[n] = (float)nd; n++; }
    }
    return n;
}

static void cell_of(const fdo_state *s, const float *pos, int *i, int *j, int *k)
{
    int F = s->c.fdoh;
    *i = (int)(pos[0] / s->DH) + F;
    *j = (int)(pos[1] / s->DH) + F;
    *k = (int)(pos[2] / s->DH) + F;
}

static i64 pos_index(const fdo_state *s, int i, int j, int k)
{
    if (s->c.nd == 3) return ((i64)i * s->NYp + j) * s->NZp + k;
    return (i64)i * s->NZp + k;
}

static void inject_sources(fdo_state *s, const fdo_shot *sh, int mask, int t, int pdir)
{
    int F = s->c.fdoh, NT = s->c.nt;
    for (int g = 0; g < sh->nsrc; g++) {
        int i, j, k;
        cell_of(s, sh->src_pos + 5 * g, &i, &j, &k);
        if (i < F || i > s->NXp - F - 1) continue;
        if (s->c.freesurf && pdir == -1 && k < 2 * F) continue;
        int type = (int)sh->src_pos[4 + 5 * g];
        float amp = (float)pdir * (s->DT * sh->src[(i64)g * NT + t]);
        int fields[9];
        float div[9];
        int n = fdo_source_targets(s->c.nd, mask, type, fields, div);
        i64 ix = pos_index(s, i, j, k);
        for (int q = 0; q < n; q++) {
            float *f = s->w[fields[q]];
            if (div[q] == 0) f[ix] += amp;
            else f[ix] += amp / (double)div[q];
        }
    }
}

static const int out_field[O_N] = {W_VX, W_VY, W_VZ, W_SXX, W_SYY, W_SZZ, W_SXY, W_SYZ, W_SXZ, -1};

static void record(fdo_state *s, const fdo_shot *sh, const int outsel[O_N], float *const seis[O_N], int t)
{
    int F = s->c.fdoh, NT = s->c.nt;
    for (int g = 0; g < sh->nrec; g++) {
        int i, j, k;
        cell_of(s, sh->rec_pos + 8 * g, &i, &j, &k);
        if (i < F || i > s->NXp - F - 1) continue;
        i64 ix = pos_index(s, i, j, k);
        for (int o = 0; o < O_N; o++) {
            if (!outsel[o]) continue;
            float v;
            if (o == O_P) {
                if (s->c.nd == 3) v = (s->w[W_SXX][ix] + s->w[W_SZZ][ix] + s->w[W_SYY][ix]) / 3.0;
                else if (s->c.nd == 22) v = s->w[W_SXX][ix];
                else v = (s->w[W_SXX][ix] + s->w[W_SZZ][ix]) / 2.0;
            } else v = s->w[out_field[o]][ix];
            seis[o][(i64)NT * g + t] = v;
        }
    }
}

static void inject_residuals(fdo_state *s, const fdo_shot *sh, const int outsel[O_N], float *const res[O_N], int t)
{
    int F = s->c.fdoh, NT = s->c.nt;
    for (int g = 0; g < sh->nrec; g++) {
        int i, j, k;
        cell_of(s, sh->rec_pos + 8 * g, &i, &j, &k);
        if (i < F || i > s->NXp - F - 1) continue;
        i64 ix = pos_index(s, i, j, k);
        for (int o = 0; o < O_N; o++) {
            if (!outsel[o]) continue;
            float r = res[o][(i64)NT * g + t];
            if (o == O_P) {
                int n2 = s->c.nd == 3 ? 3 : 2;
                s->wr[W_SXX][ix] += r / n2;
                s->wr[W_SZZ][ix] += r / n2;
                if (s->c.nd == 3) s->wr[W_SYY][ix] += r / n2;
            } else s->wr[out_field[o]][ix] += r;
        }
    }
}

static void zero_fields(fdo_state *s, float **w, float **r)
{
    for (int q = 0; q < s->nwave; q++) memset(w[s->wave_ids[q]], 0, sizeof(float) * s->nvol);
    if (s->c.L > 0)
        for (int q = 0; q < s->nmem; q++) memset(r[s->mem_ids[q]], 0, sizeof(float) * s->nvol * s->c.L);
}

void fdo_zero_gradients(fdo_state *s)
{
    for (int i = 0; i < G_N; i++) {
        memset(s->grad[i], 0, sizeof(float) * s->npar);
        if (s->hess[i]) memset(s->hess[i], 0, sizeof(float) * s->npar);
    }
}

static void zero_psi(fdo_state *s)
{
    int nab = s->c.nab;
    i64 sx = 2 * (i64)nab * s->c.ny * s->c.nz, sy = (i64)s->c.nx * 2 * nab * s->c.nz,
        sz = (i64)s->c.nx * s->c.ny * 2 * nab;
    i64 psz[PS_N] = {sx, sx, sx, sy, sy, sy, sz, sz, sz, sx, sx, sx, sy, sy, sy, sz, sz, sz};
    for (int i = 0; i < PS_N; i++)
        if (s->psi[i]) memset(s->psi[i], 0, sizeof(float) * psz[i]);
}

int fdo_forward(fdo_state *s, const fdo_kernels *k, const fdo_shot *sh, const int outsel[O_N], int mask,
                float *const seis[O_N], int save_boundaries)
{
    /* initialize_forward: zero wave fields, memory variables and CPML memory */
    zero_fields(s, s->w, s->r);
    zero_psi(s);
    for (int o = 0; o < O_N; o++)
        if (outsel[o]) memset(seis[o], 0, sizeof(float) * (i64)s->c.nt * sh->nrec);
    /* a gradient run keeps the boundary shells (BACK_PROP_TYPE 1) or the
     * forward transforms (2) */
    int dft = save_boundaries && s->c.back_prop_type == 2;
    int bnd = save_boundaries && !dft;
    if (bnd) {
        for (int q = 0; q < s->nwave; q++) {
            int w = s->wave_ids[q];
            if (!s->bnd[w]) s->bnd[w] = calloc((size_t)s->c.nt * s->nbnd + 1, sizeof(float));
        }
    }
    if (dft) fdo_zero_dft(s, 0);
    for (int t = 0; t < s->c.tmax; t++) {
        /* the state after t steps, before the sources of step t */
        if (dft && t >= s->c.tmin && (t - s->c.tmin) % s->dtnyq == 0) fdo_savefreqs(s, 0, (t - s->c.tmin) / s->dtnyq);
        inject_sources(s, sh, mask, t, 1);
        k->update_v(s);
        k->update_s(s);
        if (bnd) k->savebnd(s, t);
        if (s->c.freesurf) k->surface(s, 1);
        record(s, sh, outsel, seis, t);
    }
    return 0;
}

/* DFT adjoint (src/time_stepping.c:621-680 and :862-972 with
 * BACK_PROP_TYPE=2): the adjoint kernels' "r" arguments are bound to the
 * forward buffers (src/clprogram.c:869-880), which start from zero together
 * with the CPML memory; no boundary injection, no source removal; the
 * adjoint fields are transformed at the forward's sampling times and the
 * gradient is assembled from both transforms at the end. */
static int adjoint_dft(fdo_state *s, const fdo_kernels *k, const fdo_shot *sh, const int outsel[O_N],
                       float *const res[O_N])
{
    float *wr_keep[W_N], *rr_keep[R_N];
    memcpy(wr_keep, s->wr, sizeof wr_keep);
    memcpy(rr_keep, s->rr, sizeof rr_keep);
    memcpy(s->wr, s->w, sizeof wr_keep);
    memcpy(s->rr, s->r, sizeof rr_keep);
    zero_fields(s, s->w, s->r);
    zero_psi(s);
    fdo_zero_dft(s, 1);
    for (int t = s->c.tmax - 1; t > s->c.tmin; t--) {
        if (s->c.freesurf) k->surface_adj(s);
        inject_residuals(s, sh, outsel, res, t);
        k->update_adjs(s);
        k->update_adjv(s);
        if ((t - s->c.tmin) % s->dtnyq == 0) fdo_savefreqs(s, 1, (t - s->c.tmin) / s->dtnyq);
    }
    fdo_calc_grad(s);
    memcpy(s->wr, wr_keep, sizeof wr_keep);
    memcpy(s->rr, rr_keep, sizeof rr_keep);
    return 0;
}

int fdo_adjoint(fdo_state *s, const fdo_kernels *k, const fdo_shot *sh, const int outsel[O_N], int mask,
                float *const res[O_N])
{
    if (s->c.back_prop_type == 2) return adjoint_dft(s, k, sh, outsel, res);
    /* initialize_adj: adjoint fields and memory variables start at zero; the
     * CPML memory keeps the forward run's final values (the adjoint kernels
     * bind the forward psi buffers by name, src/clprogram.c:806-811). */
    zero_fields(s, s->wr, s->rr);
    for (int t = s->c.tmax - 1; t > s->c.tmin; t--) {
        for (int q = 0; q < s->nwave; q++) {
            int w = s->wave_ids[q];
            s->bnd_cur[w] = s->bnd[w] + (i64)(t - 1) * s->nbnd;
        }
        if (s->c.freesurf) k->surface_adj(s);
        inject_residuals(s, sh, outsel, res, t);
        k->update_adjs(s);
        k->update_adjv(s);
        inject_sources(s, sh, mask, t, -1);
    }
    return 0;
}

/* src/calc_grad.c:975-1107 for param_type 0 (vp, vs, rho): grad of the
 * stored (M, mu, rho) divided by dt and chain-ruled.  Inputs are the raw
 * accumulators; out receives gradvp, gradvs, gradrho. */
void fdo_transf_grad(const fdo_state *s, float *gvp, float *gvs, float *grho)
{
    i64 n = s->npar;
    float dt = s->c.dt, dh = s->c.dh;
    for (i64 i = 0; i < n; i++) {
        float rho = 1.0 / s->p[P_RHO][i] * dt / dh * powf(2, -0);
        float M = s->p[P_M][i];
        float mu = s->p[P_MU][i];
        float gr = s->grad[G_RHO][i];
        float gM = s->grad[G_M][i];
        float gmu = s->grad[G_MU][i];
        gr /= dt;
        M *= dh / dt * powf(2, -0);
        gM /= dt;
        mu *= dh / dt * powf(2, -0);
        gmu /= dt;
        gr = gr + M / rho * gM;
        if (mu > 0) gr = gr + mu / rho * gmu;
        gM = 2.0 * sqrt((double)rho * (double)M) * gM;
        gmu = 2.0 * sqrt((double)rho * (double)mu) * gmu;
        gvp[i] = gM;
        gvs[i] = gmu;
        grho[i] = gr;
    }
}

/* The approximate Hessian through transf_grad's chain rule
 * (src/calc_grad.c:1004-1090): the parameters are rescaled as for the
 * gradient, the Hessian is not divided by dt.  out (rho, M, mu, taup, taus
 * order) receives Hrho, HM, Hmu and the raw taup/taus Hessians. */
static void transf_hess(const fdo_state *s, float **out)
{
    i64 n = s->npar;
    float dt = s->c.dt, dh = s->c.dh;
    int pt = s->c.param_type;
    for (i64 i = 0; i < n; i++) {
        float rho = 1.0 / s->p[P_RHO][i] * dt / dh * powf(2, -0);
        float M = s->p[P_M][i] * (dh / dt * powf(2, -0));
        float mu = s->p[P_MU][i] * (dh / dt * powf(2, -0));
        float hr = s->hess[G_RHO][i], hM = s->hess[G_M][i], hmu = s->hess[G_MU][i];
        if (pt == 0 || pt == 2) {
            hr = hr + M / rho * hM;
            if (mu > 0) hr = hr + mu / rho * hmu;
        }
        if (pt == 0) {
            hM = 2.0 * sqrt((double)rho * (double)M) * hM;
            hmu = 2.0 * sqrt((double)rho * (double)mu) * hmu;
        } else if (pt == 2) {
            hM = 2.0 * sqrt((double)M / (double)rho) * hM;
            hmu = 2.0 * sqrt((double)mu / (double)rho) * hmu;
        }
        if (out[G_RHO]) out[G_RHO][i] = hr;
        if (out[G_M]) out[G_M][i] = hM;
        if (out[G_MU]) out[G_MU][i] = hmu;
        if (out[G_TAUP]) out[G_TAUP][i] = s->hess[G_TAUP][i];
        if (out[G_TAUS]) out[G_TAUS][i] = s->hess[G_TAUS][i];
    }
}

/* ---- flat entry points for ctypes ---- */
typedef struct fdo_handle {
    fdo_state s;
    const fdo_kernels *k;
} fdo_handle;

const fdo_kernels *fdo_ref_kernels_or_null(void) __attribute__((weak));

void *fdo_create(const fdo_cfg *c, int use_ref, int *err)
{
    fdo_handle *h = calloc(1, sizeof *h);
    *err = fdo_state_init(&h->s, c);
    h->k = &fdo_port_kernels;
    if (use_ref) {
        if (fdo_ref_kernels_or_null) h->k = fdo_ref_kernels_or_null();
        else *err = 10;
    }
    return h;
}
void fdo_destroy(void *hp)
{
    fdo_handle *h = hp;
    fdo_state_free(&h->s);
    free(h);
}
int fdo_model(void *hp, const float *a, const float *b, const float *rho, const float *taup, const float *taus)
{
    fdo_handle *h = hp;
    return fdo_set_model(&h->s, a, b, rho, taup, taus);
}
int fdo_run_forward(void *hp, int nsrc, const float *src_pos, const float *src, int nrec, const float *rec_pos,
                    const int *outsel, int mask, float **seis, int save_bnd)
{
    fdo_handle *h = hp;
    fdo_shot sh = {nsrc, nrec, src_pos, src, rec_pos};
    return fdo_forward(&h->s, h->k, &sh, outsel, mask, seis, save_bnd);
}
int fdo_run_adjoint(void *hp, int nsrc, const float *src_pos, const float *src, int nrec, const float *rec_pos,
                    const int *outsel, int mask, float **res)
{
    fdo_handle *h = hp;
    fdo_shot sh = {nsrc, nrec, src_pos, src, rec_pos};
    return fdo_adjoint(&h->s, h->k, &sh, outsel, mask, res);
}
void fdo_get_grad(void *hp, float *gvp, float *gvs, float *grho, float *rawM, float *rawmu, float *rawrho)
{
    fdo_handle *h = hp;
    fdo_transf_grad(&h->s, gvp, gvs, grho);
    i64 n = h->s.npar;
    if (rawM) memcpy(rawM, h->s.grad[G_M], n * sizeof(float));
    if (rawmu) memcpy(rawmu, h->s.grad[G_MU], n * sizeof(float));
    if (rawrho) memcpy(rawrho, h->s.grad[G_RHO], n * sizeof(float));
}
void fdo_clear_grad(void *hp) { fdo_zero_gradients(&((fdo_handle *)hp)->s); }
/* the accumulators as they are: rho, M, mu, taup, taus (G_* order) */
void fdo_get_grad_raw(void *hp, float **out)
{
    fdo_handle *h = hp;
    for (int i = 0; i < G_N; i++)
        if (out[i]) memcpy(out[i], h->s.grad[i], h->s.npar * sizeof(float));
}
/* the Hessian accumulators (transform 0) or their transf_grad form
 * (transform 1; not for the DFT gradient, which the reference leaves as is) */
void fdo_get_hess(void *hp, int transform, float **out)
{
    fdo_handle *h = hp;
    if (!h->s.hess[0]) return;
    if (transform) { transf_hess(&h->s, out); return; }
    for (int i = 0; i < G_N; i++)
        if (out[i]) memcpy(out[i], h->s.hess[i], h->s.npar * sizeof(float));
}
/* DFT of slot (0 forward, 1 adjoint): kind 0 wave field, 1 memory variable */
float *fdo_dft_array(void *hp, int slot, int kind, int id)
{
    fdo_state *s = &((fdo_handle *)hp)->s;
    return kind == 0 ? s->fw[slot][id] : s->fr[slot][id];
}
/* dtnyq, ntnyq and df of a DFT-gradient state; gradfreqsn into fn */
void fdo_dft_info(void *hp, int *ni, float *df, float *fn)
{
    fdo_state *s = &((fdo_handle *)hp)->s;
    ni[0] = s->dtnyq; ni[1] = s->ntnyq; *df = s->df;
    for (int j = 0; j < s->c.nfreqs; j++) fn[j] = s->gradfreqsn[j];
}
/* assemble the gradient from the transforms now held (for the pin) */
void fdo_run_calc_grad(void *hp) { fdo_calc_grad(&((fdo_handle *)hp)->s); }

/* Access to internal arrays for field-level comparisons.  kind: 0 wave,
 * 1 adjoint wave, 2 memory, 3 adjoint memory, 4 psi, 5 param, 6 cpml x,
 * 7 cpml y, 8 cpml z, 9 taper, 10 eta, 11 boundary store. */
float *fdo_array(void *hp, int kind, int id)
{
    fdo_state *s = &((fdo_handle *)hp)->s;
    switch (kind) {
    case 0: return s->w[id];
    case 1: return s->wr[id];
    case 2: return s->r[id];
    case 3: return s->rr[id];
    case 4: return s->psi[id];
    case 5: return s->p[id];
    case 6: return s->cx[id];
    case 7: return s->cy[id];
    case 8: return s->cz[id];
    case 9: return s->taper;
    case 10: return s->eta;
    case 11: return s->bnd[id];
    default: return 0;
    }
}
void fdo_info(void *hp, int64_t *out)
{
    fdo_state *s = &((fdo_handle *)hp)->s;
    out[0] = s->NZp; out[1] = s->NYp; out[2] = s->NXp; out[3] = s->nvol; out[4] = s->npar; out[5] = s->nbnd;
}
/* steps of the forward loop, for the bounded CPU-baseline sample */
int fdo_run_steps(void *hp, int nsteps)
{
    fdo_handle *h = hp;
    for (int t = 0; t < nsteps; t++) {
        h->k->update_v(&h->s);
        h->k->update_s(&h->s);
        if (h->s.c.freesurf) h->k->surface(&h->s, 1);
    }
    return 0;
}
