/*
 * fdo_setup.c -- oracle set-up: FD coefficients, CPML profiles, parameter
 * transforms, stability check, boundary-shell size.
 *
 * TEST INFRASTRUCTURE ONLY (the checker of the CUDA path; see fdo.h).
 *
 * Every routine keeps the float/double mix of the reference host code so the
 * results are bit-identical to the reference compiled as C.
 */

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fdo.h"   /* after the system headers: FDO_FP64 retypes float */

#define FDO_PI (3.141592653589793238462643383279502884197169)

/* Holberg (1987) optimal staggered-grid coefficients and the Taylor ones.
 * Rows: MAXRELERROR 0 (Taylor), 1 (0.1 %), 2 (0.5 %), 3 (1 %), 4 (3 %).
 * Columns: points per wavelength, then c1..c6.  The numbers are the published
 * table that src/third_party/SOFI3D/holbergcoeff.c:41-83 also carries; they
 * must be the same values for the stencils to agree.  The reference stores the
 * table as float and widens to double (holbergcoeff.c:41, 96-98). */
static const float holberg_tab[5][6][7] = {
    {{23.0f, 1.0f, 0, 0, 0, 0, 0},
     {8.0f, 9.0f / 8.0f, -1.0f / 24.0f, 0, 0, 0, 0},
     {6.0f, 75.0f / 64.0f, -25.0f / 384.0f, 3.0f / 640.0f, 0, 0, 0},
     {5.0f, 1225.0f / 1024.0f, -245.0f / 3072.0f, 49.0f / 5120.0f, -5.0f / 7168.0f, 0, 0},
     {5.0f, 19845.0f / 16384.0f, -735.0f / 8192.0f, 567.0f / 40960.0f, -405.0f / 229376.0f,
      35.0f / 294912.0f, 0},
     {4.0f, 160083.0f / 131072.0f, -12705.0f / 131072.0f, 22869.0f / 1310720.0f,
      -5445.0f / 1835008.0f, 847.0f / 2359296.0f, -63.0f / 2883584.0f}},
    {{49.7f, 1.0010f, 0, 0, 0, 0, 0},
     {8.32f, 1.1382f, -0.046414f, 0, 0, 0, 0},
     {4.77f, 1.1965f, -0.078804f, 0.0081781f, 0, 0, 0},
     {3.69f, 1.2257f, -0.099537f, 0.018063f, -0.0026274f, 0, 0},
     {3.19f, 1.2415f, -0.11231f, 0.026191f, -0.0064682f, 0.001191f, 0},
     {2.91f, 1.2508f, -0.12034f, 0.032131f, -0.010142f, 0.0029857f, -0.00066667f}},
    {{22.2f, 1.0050f, 0, 0, 0, 0, 0},
     {5.65f, 1.1534f, -0.052806f, 0, 0, 0, 0},
     {3.74f, 1.2111f, -0.088313f, 0.011768f, 0, 0, 0},
     {3.11f, 1.2367f, -0.10815f, 0.023113f, -0.0046905f, 0, 0},
     {2.80f, 1.2496f, -0.11921f, 0.031130f, -0.0093272f, 0.0025161f, 0},
     {2.62f, 1.2568f, -0.12573f, 0.036423f, -0.013132f, 0.0047484f, -0.0015979f}},
    {{15.8f, 1.0100f, 0, 0, 0, 0, 0},
     {4.80f, 1.1640f, -0.057991f, 0, 0, 0, 0},
     {3.39f, 1.2192f, -0.094070f, 0.014608f, 0, 0, 0},
     {2.90f, 1.2422f, -0.11269f, 0.026140f, -0.0064054f, 0, 0},
     {2.65f, 1.2534f, -0.12257f, 0.033755f, -0.011081f, 0.0036784f, 0},
     {2.51f, 1.2596f, -0.12825f, 0.038550f, -0.014763f, 0.0058619f, -0.0024538f}},
    {{9.16f, 1.0300f, 0, 0, 0, 0, 0},
     {3.47f, 1.1876f, -0.072518f, 0, 0, 0, 0},
     {2.91f, 1.2341f, -0.10569f, 0.022589f, 0, 0, 0},
     {2.61f, 1.2516f, -0.12085f, 0.032236f, -0.011459f, 0, 0},
     {2.45f, 1.2596f, -0.12829f, 0.038533f, -0.014681f, 0.0072580f, 0},
     {2.36f, 1.2640f, -0.13239f, 0.042217f, -0.017803f, 0.0081959f, -0.0051848f}},
};

int fdo_holberg(int fdorder, int maxrelerror, double hc[7])
{
    if (fdorder < 2 || fdorder > 12 || (fdorder % 2) != 0) return 1;
    if (maxrelerror < 0 || maxrelerror > 4) return 1;
    for (int i = 0; i < 7; i++) hc[i] = (double)holberg_tab[maxrelerror][fdorder / 2 - 1][i];
    return 0;
}

/* The reference passes host floats/doubles to the kernels as "%9.9f"
 * literals (src/clprogram.c:493-520).  This is the value such a literal
 * parses to. */
void fdo_literal(double *out, float v)
{
    char buf[64];
    snprintf(buf, sizeof buf, "%9.9f", (double)v);
    *out = strtod(buf, NULL);
}
static double literal_d(double v)
{
    char buf[64];
    snprintf(buf, sizeof buf, "%9.9f", v);
    return strtod(buf, NULL);
}

/* Komatitsch & Martin (2007) convolutional PML profiles, d0 from the INRIA
 * report formula, at full and half nodes, mirrored for the far side.  Same
 * operation order and precision as src/third_party/SOFI3D/CPML_COEFF.c:26-189.
 * Arrays hold 2*nab values and must be zeroed by the caller. */
int fdo_cpml_coeff(float npower_in, float k_max, float fpml, float vppml, float dh,
                   float dt, int nab, float *K, float *b, float *a,
                   float *K_half, float *b_half, float *a_half)
{
    int err = 0;
    const float npower = npower_in;
    const float alpha_max = 2.0 * FDO_PI * (fpml / 2.0);
    const float rcoef = 0.0008;
    const float ca = 0.25, cb = 0.75, cc = 0.0;
    float *d = calloc((size_t)2 * nab + 2, sizeof(float));
    float *dh_ = calloc((size_t)2 * nab + 2, sizeof(float));
    float *al = calloc((size_t)2 * nab + 2, sizeof(float));
    float *alh = calloc((size_t)2 * nab + 2, sizeof(float));
    float d0 = -(npower + 1) * vppml * log(rcoef) / (2.0 * nab * dh);

    for (int i = 0; i <= nab; i++) {
        float pos = (nab - i) * dh;
        float pn = pos / (nab * dh);
        d[i] = d0 * (ca * pn + cb * pow(pn, npower) + cc * pow(pn, (4)));
        K[i] = 1.0 + (k_max - 1.0) * pow(pn, npower);
        al[i] = alpha_max * (1.0 - pn);
        if (al[i] < 0.0) err = 1;
        b[i] = exp(-(d[i] / K[i] + al[i]) * dt);
        if (fabsf(d[i]) > 1.0e-6)
            a[i] = d[i] * (b[i] - 1.0) / (K[i] * (d[i] + K[i] * al[i]));
        else
            a[i] = 0.0;
        if (i <= nab - 1) {
            pos = (nab - i + 0.5 - 1.0) * dh;
            pn = pos / (nab * dh);
            dh_[i] = d0 * (ca * pn + cb * pow(pn, npower) + cc * pow(pn, (4)));
            if (pos < 0.0) err = 1;
            K_half[i] = 1.0 + (k_max - 1.0) * pow(pn, npower);
            alh[i] = alpha_max * (1.0 - pn);
            if (alh[i] < 0.0) err = 1;
            b_half[i] = exp(-(dh_[i] / K_half[i] + alh[i]) * dt);
            if (fabs(dh_[i]) > 1.0e-6)
                a_half[i] = dh_[i] * (b_half[i] - 1.0) / (K_half[i] * (dh_[i] + K_half[i] * alh[i]));
            /* far side mirrors the near side */
            int l = 2 * nab - i - 1;
            if (i > 0) {
                K[l + 1] = K[i];
                b[l + 1] = b[i];
                if (fabs(d[i]) > 1.0e-6) a[l + 1] = a[i];
            }
            K_half[l] = K_half[i];
            b_half[l] = b_half[i];
            if (fabs(d[i]) > 1.0e-6) a_half[l] = a_half[i];
        }
    }
    free(d); free(dh_); free(al); free(alh);
    return err;
}

/* Saved-boundary cell count per field (src/Init_OpenCL.c:988-1021, single
 * device). */
static int nbnd_count(const fdo_cfg *c)
{
    int F = c->fdoh, nab = c->nab;
    int lenz = c->freesurf ? c->nz - nab - F : c->nz - 2 * nab - 2 * F;
    if (c->nd == 3)
        return (c->nx - 2 * nab) * (c->ny - 2 * nab) * 2 * F + (c->nx - 2 * nab) * lenz * 2 * F +
               (c->ny - 2 * nab - 2 * F) * lenz * 2 * F;
    return (c->nx - 2 * nab) * 2 * F + lenz * 2 * F;
}

static float *zalloc(int64_t n) { return (float *)calloc((size_t)(n > 0 ? n : 1), sizeof(float)); }

int fdo_state_init(fdo_state *s, const fdo_cfg *c)
{
    memset(s, 0, sizeof *s);
    s->c = *c;
    int F = c->fdoh;
    if (c->tmax <= 0) s->c.tmax = c->nt;
    s->NZp = c->nz + 2 * F;
    s->NXp = c->nx + 2 * F;
    s->NYp = c->nd == 3 ? c->ny + 2 * F : 1;
    if (c->nd != 3) s->c.ny = 1;
    s->nvol = (int64_t)s->NZp * s->NYp * s->NXp;
    s->npar = (int64_t)c->nz * s->c.ny * c->nx;
    if (fdo_holberg(c->fdorder, c->maxrelerror, s->hc)) return 2;
    for (int i = 1; i <= 6; i++) s->hc[i] = literal_d(s->hc[i]);
    fdo_literal(&s->DT, c->dt);
    s->DT2 = literal_d((double)c->dt / 2.0);
    fdo_literal(&s->DH, c->dh);

    int ids3[] = {W_VX, W_VY, W_VZ, W_SXX, W_SYY, W_SZZ, W_SXY, W_SYZ, W_SXZ};
    int ids2[] = {W_VX, W_VZ, W_SXX, W_SZZ, W_SXZ};
    int rid3[] = {R_XX, R_YY, R_ZZ, R_XY, R_YZ, R_XZ};
    int rid2[] = {R_XX, R_ZZ, R_XZ};
    int ids22[] = {W_VX, W_VZ, W_SXX}, rid22[] = {R_XX};     /* acoustic: p, rp */
    int ids21[] = {W_VY, W_SXY, W_SYZ}, rid21[] = {R_XY, R_YZ}; /* SH */
    if (c->nd == 3) {
        s->nwave = 9; memcpy(s->wave_ids, ids3, sizeof ids3);
        s->nmem = 6; memcpy(s->mem_ids, rid3, sizeof rid3);
    } else if (c->nd == 22) {
        s->nwave = 3; memcpy(s->wave_ids, ids22, sizeof ids22);
        s->nmem = 1; memcpy(s->mem_ids, rid22, sizeof rid22);
    } else if (c->nd == 21) {
        s->nwave = 3; memcpy(s->wave_ids, ids21, sizeof ids21);
        s->nmem = 2; memcpy(s->mem_ids, rid21, sizeof rid21);
    } else {
        s->nwave = 5; memcpy(s->wave_ids, ids2, sizeof ids2);
        s->nmem = 3; memcpy(s->mem_ids, rid2, sizeof rid2);
    }
    for (int i = 0; i < s->nwave; i++) {
        int w = s->wave_ids[i];
        s->w[w] = zalloc(s->nvol);
        s->wr[w] = zalloc(s->nvol);
    }
    if (c->L > 0)
        for (int i = 0; i < s->nmem; i++) {
            int r = s->mem_ids[i];
            s->r[r] = zalloc(s->nvol * c->L);
            s->rr[r] = zalloc(s->nvol * c->L);
        }
    int nab = c->nab;
    int64_t nx_ = c->nx, ny_ = s->c.ny, nz_ = c->nz;
    int64_t sx = 2 * nab * ny_ * nz_, sy = nx_ * 2 * nab * nz_, sz = nx_ * ny_ * 2 * nab;
    int64_t psz[PS_N] = {sx, sx, sx, sy, sy, sy, sz, sz, sz, sx, sx, sx, sy, sy, sy, sz, sz, sz};
    if (c->abs_type == 1 && nab > 0)
        for (int i = 0; i < PS_N; i++) s->psi[i] = zalloc(psz[i]);
    for (int i = 0; i < P_N; i++) s->p[i] = zalloc(s->npar);
    for (int i = 0; i < C_N; i++) {
        s->cx[i] = zalloc(2 * nab + 2);
        s->cy[i] = zalloc(2 * nab + 2);
        s->cz[i] = zalloc(2 * nab + 2);
    }
    s->taper = zalloc(nab + 1);
    s->eta = zalloc(c->L + 1);
    for (int i = 0; i < G_N; i++) s->grad[i] = zalloc(s->npar);
    /* the reference's 3D Hessian kernel does not compile (update_adjv3D.cl:486) */
    if (c->hout && c->nd == 3 && c->back_prop_type != 2) return 5;
    if (c->hout)
        for (int i = 0; i < G_N; i++) s->hess[i] = zalloc(s->npar);

    if (c->abs_type == 1 && nab > 0) {
        if (fdo_cpml_coeff(c->npower, c->k_max_cpml, c->fpml, c->vppml, c->dh, c->dt, nab,
                           s->cz[C_K], s->cz[C_B], s->cz[C_A], s->cz[C_KH], s->cz[C_BH], s->cz[C_AH]))
            return 3;
        fdo_cpml_coeff(c->npower, c->k_max_cpml, c->fpml, c->vppml, c->dh, c->dt, nab,
                       s->cx[C_K], s->cx[C_B], s->cx[C_A], s->cx[C_KH], s->cx[C_BH], s->cx[C_AH]);
        fdo_cpml_coeff(c->npower, c->k_max_cpml, c->fpml, c->vppml, c->dh, c->dt, nab,
                       s->cy[C_K], s->cy[C_B], s->cy[C_A], s->cy[C_KH], s->cy[C_BH], s->cy[C_AH]);
    }
    if (c->abs_type == 2 && nab > 0) {
        /* Cerjan taper, src/assign_modeling_case.c:571-584 */
        float amp = 1 - c->abpc / 100;
        float aa = sqrt(-log(amp) / ((nab - 1) * (nab - 1)));
        for (int i = 1; i <= nab; i++) s->taper[i - 1] = exp(-(aa * aa * (nab - i) * (nab - i)));
    }
    for (int l = 0; l < c->L; l++) s->eta[l] = (2.0 * FDO_PI * c->fl[l]) * c->dt; /* :536-548 */

    s->nbnd = nbnd_count(&s->c);

    if (c->back_prop_type == 2) {
        /* DFT gradient frequencies, src/assign_modeling_case.c:549-570 */
        if (c->nfreqs < 1 || c->nfreqs > FDO_MAXFREQ) return 4;
        float fmaxout = 0;
        for (int j = 0; j < c->nfreqs; j++)
            if (c->gradfreqs[j] > fmaxout) fmaxout = c->gradfreqs[j];
        if (!(fmaxout > 0)) return 4;
        s->dtnyq = (int)ceil(0.0156 / fmaxout / c->dt);
        s->ntnyq = (s->c.tmax - s->c.tmin) / s->dtnyq + 1;
        s->df = 1.0 / s->ntnyq / c->dt / s->dtnyq;
        for (int j = 0; j < c->nfreqs; j++) s->gradfreqsn[j] = floor(c->gradfreqs[j] / s->df);
        for (int slot = 0; slot < 2; slot++) {
            for (int i = 0; i < s->nwave; i++) s->fw[slot][s->wave_ids[i]] = zalloc(2 * c->nfreqs * s->nvol);
            if (c->L > 0)
                for (int i = 0; i < s->nmem; i++)
                    s->fr[slot][s->mem_ids[i]] = zalloc(2 * c->nfreqs * s->nvol * c->L);
        }
    }
    return 0;
}

void fdo_state_free(fdo_state *s)
{
    for (int i = 0; i < W_N; i++) { free(s->w[i]); free(s->wr[i]); free(s->bnd[i]); }
    for (int i = 0; i < R_N; i++) { free(s->r[i]); free(s->rr[i]); }
    for (int i = 0; i < PS_N; i++) free(s->psi[i]);
    for (int i = 0; i < P_N; i++) free(s->p[i]);
    for (int i = 0; i < C_N; i++) { free(s->cx[i]); free(s->cy[i]); free(s->cz[i]); }
    for (int i = 0; i < G_N; i++) { free(s->grad[i]); free(s->hess[i]); }
    for (int slot = 0; slot < 2; slot++) {
        for (int i = 0; i < W_N; i++) free(s->fw[slot][i]);
        for (int i = 0; i < R_N; i++) free(s->fr[slot][i]);
    }
    free(s->taper);
    free(s->eta);
    memset(s, 0, sizeof *s);
}

/* ---- parameter averaging, src/assign_modeling_case.c:50-301 ---- */
/* dims: NZ (fast), NY, NX (slow); 2D has NY = 1 */
static void ave_arith1(const float *pin, float *pout, int NZ, int NY, int NX, const int dir[3])
{
    for (int k = 0; k < NZ - dir[0]; k++)
        for (int j = 0; j < NY - dir[1]; j++)
            for (int i = 0; i < NX - dir[2]; i++) {
                int64_t i1 = ((int64_t)i * NY + j) * NZ + k;
                int64_t i2 = ((int64_t)(i + dir[2]) * NY + (j + dir[1])) * NZ + (k + dir[0]);
                pout[i1] = 0.5 * (pin[i1] + pin[i2]);
            }
    int NX0 = 0, NY0 = 0, NZ0 = 0;
    if (dir[2] == 1) NX0 = NX - 1;
    else if (dir[1] == 1) NY0 = NY - 1;
    if (dir[0] == 1) NZ0 = NZ - 1;
    for (int k = NZ0; k < NZ; k++)
        for (int j = NY0; j < NY; j++)
            for (int i = NX0; i < NX; i++) {
                int64_t i1 = ((int64_t)i * NY + j) * NZ + k;
                pout[i1] = pin[i1];
            }
}

/* Two-direction averages.  harmonic=1: 4/sum(1/p) (ave_harmonic), else
 * 0.25*sum(p) (ave_arithmetic2).  The edge copy keeps the reference's carried
 * NX0/NY0 (assign_modeling_case.c:134-170, 262-298): only the first direction's
 * last slab and a corner line are copied; the rest of the second direction's
 * last slab stays zero. */
static void ave_two(const float *pin, float *pout, int NZ, int NY, int NX, const int dir[2][3],
                    int harmonic)
{
    for (int k = 0; k < NZ - dir[0][0] - dir[1][0]; k++)
        for (int j = 0; j < NY - dir[0][1] - dir[1][1]; j++)
            for (int i = 0; i < NX - dir[0][2] - dir[1][2]; i++) {
                int64_t i1 = ((int64_t)i * NY + j) * NZ + k;
                int64_t i2 = ((int64_t)(i + dir[0][2]) * NY + (j + dir[0][1])) * NZ + (k + dir[0][0]);
                int64_t i3 = ((int64_t)(i + dir[1][2]) * NY + (j + dir[1][1])) * NZ + (k + dir[1][0]);
                int64_t i4 = ((int64_t)(i + dir[0][2] + dir[1][2]) * NY + (j + dir[0][1] + dir[1][1])) * NZ +
                             (k + dir[0][0] + dir[1][0]);
                if (harmonic)
                    pout[i1] = 4.0 / (1.0 / pin[i1] + 1.0 / pin[i2] + 1.0 / pin[i3] + 1.0 / pin[i4]);
                else
                    pout[i1] = 0.25 * (pin[i1] + pin[i2] + pin[i3] + pin[i4]);
            }
    int NX0 = 0, NY0 = 0, NZ0 = 0;
    for (int d = 0; d < 2; d++) {
        if (dir[d][2] == 1) NX0 = NX - 1;
        else if (dir[d][1] == 1) NY0 = NY - 1;
        if (dir[d][0] == 1) NZ0 = NZ - 1;
        for (int k = NZ0; k < NZ; k++)
            for (int j = NY0; j < NY; j++)
                for (int i = NX0; i < NX; i++) {
                    int64_t i1 = ((int64_t)i * NY + j) * NZ + k;
                    pout[i1] = pin[i1];
                }
    }
}

/* src/assign_modeling_case.c:305-487 (transforms), 730-827 (stability) */
int fdo_set_model(fdo_state *s, const float *a, const float *b, const float *rho_in,
                  const float *taup_in, const float *taus_in)
{
    const fdo_cfg *c = &s->c;
    int64_t n = s->npar;
    float *M = s->p[P_M], *mu = s->p[P_MU], *rho = s->p[P_RHO];
    float *taup = s->p[P_TAUP], *taus = s->p[P_TAUS];
    memcpy(rho, rho_in, n * sizeof(float));
    if (a) memcpy(M, a, n * sizeof(float));
    if (b) memcpy(mu, b, n * sizeof(float));
    if (c->L > 0) {
        memcpy(taup, taup_in, n * sizeof(float));
        memcpy(taus, taus_in, n * sizeof(float));
    }
    float dt = c->dt, dh = c->dh;
    /* M (:380-449) */
    for (int64_t i = 0; i < n; i++) {
        if (c->param_type == 0) M[i] = powf(M[i], 2) * rho[i] * dt / dh;
        else if (c->param_type == 1) M[i] = M[i] * dt / dh;
        else if (c->param_type == 2) M[i] = powf(M[i] / rho[i], 2) * rho[i] * dt / dh;
    }
    if (c->L > 0) {
        float pts[8];
        for (int l = 0; l < c->L; l++) pts[l] = dt / s->eta[l];
        float ws = 2.0 * FDO_PI * c->f0;
        for (int64_t i = 0; i < n; i++) {
            float sumpi = 0.0;
            for (int l = 0; l < c->L; l++)
                sumpi += ((ws * ws * pts[l] * pts[l] * taup[i]) / (1.0 + ws * ws * pts[l] * pts[l]));
            M[i] = M[i] / (1.0 + sumpi);
        }
    }
    /* mu (:305-379) */
    for (int64_t i = 0; i < n; i++) {
        if (c->param_type == 0) mu[i] = powf(mu[i], 2) * rho[i] * dt / dh;
        else if (c->param_type == 1) mu[i] = mu[i] * dt / dh;
        else if (c->param_type == 2) mu[i] = powf(mu[i] / rho[i], 2) * rho[i] * dt / dh;
    }
    if (c->L > 0) {
        float pts[8];
        for (int l = 0; l < c->L; l++) pts[l] = dt / s->eta[l];
        float ws = 2.0 * FDO_PI * c->f0;
        float sumu = 0.0;
        for (int l = 0; l < c->L; l++) sumu += ((ws * ws * pts[l] * pts[l]) / (1.0 + ws * ws * pts[l] * pts[l]));
        for (int64_t i = 0; i < n; i++) mu[i] = mu[i] / (1.0 + sumu * taus[i]);
    }
    /* rho (:451-462), par_scale = 0 in FP32 */
    for (int64_t i = 0; i < n; i++) rho[i] = 1.0 / rho[i] * dt / dh * powf(2, -0);

    int NZ = c->nz, NY = c->ny, NX = c->nx;
    int dx[3] = {0, 0, 1}, dy[3] = {0, 1, 0}, dz[3] = {1, 0, 0};
    ave_arith1(rho, s->p[P_RIP], NZ, NY, NX, dx);
    if (c->nd == 3) ave_arith1(rho, s->p[P_RJP], NZ, NY, NX, dy);
    ave_arith1(rho, s->p[P_RKP], NZ, NY, NX, dz);
    int dxz[2][3] = {{0, 0, 1}, {1, 0, 0}};
    int dxy[2][3] = {{0, 0, 1}, {0, 1, 0}};
    int dyz[2][3] = {{0, 1, 0}, {1, 0, 0}};
    ave_two(mu, s->p[P_MUIPKP], NZ, NY, NX, dxz, 1);
    if (c->nd == 3) {
        ave_two(mu, s->p[P_MUIPJP], NZ, NY, NX, dxy, 1);
        ave_two(mu, s->p[P_MUJPKP], NZ, NY, NX, dyz, 1);
    }
    if (c->L > 0) {
        ave_two(taus, s->p[P_TAUSIPKP], NZ, NY, NX, dxz, 0);
        if (c->nd == 3) {
            ave_two(taus, s->p[P_TAUSIPJP], NZ, NY, NX, dxy, 0);
            ave_two(taus, s->p[P_TAUSJPKP], NZ, NY, NX, dyz, 0);
        }
    }

    /* stability (:730-827) */
    float vpmax = 0, vsmax = 0, vpmin = 99999, vsmin = 99999;
    for (int64_t i = 0; i < n; i++) {
        float v = sqrt(mu[i] * rho[i]) / dt * dh;
        if (vsmax < v) vsmax = v;
        if (vsmin > v && v > 0.1) vsmin = v;
        v = sqrt(M[i] * rho[i]) / dt * dh;
        if (vpmax < v) vpmax = v;
        if (vpmin > v && v > 0.1) vpmin = v;
    }
    float vmax = vpmax == 0 ? vsmax : vpmax;
    float gamma;
    switch (c->fdorder) {
    case 2: gamma = 1.0; break;
    case 4: gamma = 1.184614; break;
    case 6: gamma = 1.283482; break;
    case 8: gamma = 1.345927; break;
    case 10: gamma = 1.38766; break;
    case 12: gamma = 1.417065; break;
    default: gamma = 1.0;
    }
    float dtstable = c->nd == 3 ? dh / (gamma * sqrt(3.0) * vmax) : dh / (gamma * sqrt(2.0) * vmax);
    if (dt > dtstable) return 1;
    return 0;
}
