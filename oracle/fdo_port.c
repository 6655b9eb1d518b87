/*
 * fdo_port.c -- oracle stencil kernels (CPU restatement, runtime sizes).
 *
 * TEST INFRASTRUCTURE ONLY (the checker of the CUDA path; see fdo.h).
 *
 * Each function restates one reference kernel, looping over the cells the
 * kernel's work-items cover.  Derivatives are accumulated in double with the
 * reference's "%9.9f" coefficient literals and rounded to float on assignment,
 * as the reference kernels do when HC1..HC6 are double literals
 * (src/header_FD.cl:87-265, src/clprogram.c:493-496).
 */

#include <math.h>
#include <stdint.h>
#include <string.h>

#include "fdo.h"   /* after the system headers: FDO_FP64 retypes float */

typedef int64_t i64;

/* forward difference: c1 (v[i+1]-v[i]) + c2 (v[i+2]-v[i-1]) + ...   (Dxp/Dyp/Dzp) */
static inline float dfw(const float *v, i64 i, i64 st, const double *hc, int F)
{
    double acc = hc[1] * (v[i + st] - v[i]);
    for (int m = 2; m <= F; m++) acc = acc + hc[m] * (v[i + m * st] - v[i - (m - 1) * st]);
    return (float)acc;
}
/* backward difference: c1 (v[i]-v[i-1]) + c2 (v[i+1]-v[i-2]) + ...   (Dxm/Dym/Dzm) */
static inline float dbw(const float *v, i64 i, i64 st, const double *hc, int F)
{
    double acc = hc[1] * (v[i] - v[i - st]);
    for (int m = 2; m <= F; m++) acc = acc + hc[m] * (v[i + (m - 1) * st] - v[i - m * st]);
    return (float)acc;
}

/* CPML correction of one derivative: psi = b psi + a d ; d = d/K + psi */
#define CPML(psi_, idx, K_, a_, b_, ci, d)                                  \
    do {                                                                   \
        psi_[idx] = (b_)[ci] * psi_[idx] + (a_)[ci] * (d);                  \
        d = d / (K_)[ci] + psi_[idx];                                      \
    } while (0)

/* ======================================================================
 * 2D P-SV
 * ====================================================================== */

/* src/update_v2D.cl:32-246 (also the adjoint CPML part of update_adjv2D.cl) */
static void cpml_v2d(fdo_state *s, int gz, int gx, float *sxx_x, float *szz_z, float *sxz_x,
                     float *sxz_z)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NAB = c->nab, NZ = s->NZp, NX = s->NXp, nz = c->nz;
    float **ps = s->psi;
    if (gz > NZ - NAB - F - 1) {
        int i = gx - F, k = gz - NZ + NAB + F + NAB, ind = 2 * NAB - 1 - k;
        i64 q = (i64)i * (2 * NAB) + k;
        CPML(ps[PS_SXZ_Z], q, s->cz[C_K], s->cz[C_A], s->cz[C_B], ind + 1, *sxz_z);
        CPML(ps[PS_SZZ_Z], q, s->cz[C_KH], s->cz[C_AH], s->cz[C_BH], ind, *szz_z);
    } else if (!c->freesurf && gz - F < NAB) {
        int i = gx - F, k = gz - F;
        i64 q = (i64)i * (2 * NAB) + k;
        CPML(ps[PS_SXZ_Z], q, s->cz[C_K], s->cz[C_A], s->cz[C_B], k, *sxz_z);
        CPML(ps[PS_SZZ_Z], q, s->cz[C_KH], s->cz[C_AH], s->cz[C_BH], k, *szz_z);
    }
    if (gx - F < NAB) {
        int i = gx - F, k = gz - F;
        i64 q = (i64)i * nz + k;
        CPML(ps[PS_SXX_X], q, s->cx[C_KH], s->cx[C_AH], s->cx[C_BH], i, *sxx_x);
        CPML(ps[PS_SXZ_X], q, s->cx[C_K], s->cx[C_A], s->cx[C_B], i, *sxz_x);
    }
    if (gx > NX - NAB - F - 1) {
        int i = gx - NX + NAB + F + NAB, k = gz - F, ind = 2 * NAB - 1 - i;
        i64 q = (i64)i * nz + k;
        CPML(ps[PS_SXX_X], q, s->cx[C_KH], s->cx[C_AH], s->cx[C_BH], ind, *sxx_x);
        CPML(ps[PS_SXZ_X], q, s->cx[C_K], s->cx[C_A], s->cx[C_B], ind + 1, *sxz_x);
    }
}

/* taper of the Cerjan layer, src/update_v2D.cl:216-243 */
static void taper2d(fdo_state *s, int gz, int gx, float **f, int nf, i64 iv)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NAB = c->nab, NZ = s->NZp, NX = s->NXp;
    if (!c->freesurf && gz - F < NAB)
        for (int q = 0; q < nf; q++) f[q][iv] *= s->taper[gz - F];
    if (gz > NZ - NAB - F - 1)
        for (int q = 0; q < nf; q++) f[q][iv] *= s->taper[NZ - F - gz - 1];
    if (gx - F < NAB)
        for (int q = 0; q < nf; q++) f[q][iv] *= s->taper[gx - F];
    if (gx > NX - NAB - F - 1)
        for (int q = 0; q < nf; q++) f[q][iv] *= s->taper[NX - F - gx - 1];
}

static void port_update_v2d(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NZ = s->NZp, NX = s->NXp, nz = c->nz;
    const double *hc = s->hc;
    float *vx = s->w[W_VX], *vz = s->w[W_VZ];
    const float *sxx = s->w[W_SXX], *szz = s->w[W_SZZ], *sxz = s->w[W_SXZ];
    const float *rip = s->p[P_RIP], *rkp = s->p[P_RKP];
#pragma omp parallel for schedule(static)
    for (int gx = F; gx < NX - F; gx++)
        for (int gz = F; gz < NZ - F; gz++) {
            i64 ip = (i64)(gx - F) * nz + (gz - F), iv = (i64)gx * NZ + gz;
            float sxx_x = dfw(sxx, iv, NZ, hc, F);
            float szz_z = dfw(szz, iv, 1, hc, F);
            float sxz_z = dbw(sxz, iv, 1, hc, F);
            float sxz_x = dbw(sxz, iv, NZ, hc, F);
            if (c->abs_type == 1) cpml_v2d(s, gz, gx, &sxx_x, &szz_z, &sxz_x, &sxz_z);
            vx[iv] += ((sxx_x + sxz_z) * rip[ip]);
            vz[iv] += ((szz_z + sxz_x) * rkp[ip]);
            if (c->abs_type == 2) {
                float *f[2] = {vx, vz};
                taper2d(s, gz, gx, f, 2, iv);
            }
        }
}

/* CPML for the stress update, src/update_s2D.cl:145-208 */
static void cpml_s2d(fdo_state *s, int gz, int gx, float *vxx, float *vxz, float *vzx, float *vzz)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NAB = c->nab, NZ = s->NZp, NX = s->NXp, nz = c->nz;
    float **ps = s->psi;
    if (gz > NZ - NAB - F - 1) {
        int i = gx - F, k = gz - NZ + NAB + F + NAB, ind = 2 * NAB - 1 - k;
        i64 q = (i64)i * (2 * NAB) + k;
        CPML(ps[PS_VX_Z], q, s->cz[C_KH], s->cz[C_AH], s->cz[C_BH], ind, *vxz);
        CPML(ps[PS_VZ_Z], q, s->cz[C_K], s->cz[C_A], s->cz[C_B], ind + 1, *vzz);
    } else if (!c->freesurf && gz - F < NAB) {
        int i = gx - F, k = gz - F;
        i64 q = (i64)i * (2 * NAB) + k;
        CPML(ps[PS_VX_Z], q, s->cz[C_KH], s->cz[C_AH], s->cz[C_BH], k, *vxz);
        CPML(ps[PS_VZ_Z], q, s->cz[C_K], s->cz[C_A], s->cz[C_B], k, *vzz);
    }
    if (gx - F < NAB) {
        int i = gx - F, k = gz - F;
        i64 q = (i64)i * nz + k;
        CPML(ps[PS_VX_X], q, s->cx[C_K], s->cx[C_A], s->cx[C_B], i, *vxx);
        CPML(ps[PS_VZ_X], q, s->cx[C_KH], s->cx[C_AH], s->cx[C_BH], i, *vzx);
    }
    if (gx > NX - NAB - F - 1) {
        int i = gx - NX + NAB + F + NAB, k = gz - F, ind = 2 * NAB - 1 - i;
        i64 q = (i64)i * nz + k;
        CPML(ps[PS_VX_X], q, s->cx[C_K], s->cx[C_A], s->cx[C_B], ind + 1, *vxx);
        CPML(ps[PS_VZ_X], q, s->cx[C_KH], s->cx[C_AH], s->cx[C_BH], ind, *vzx);
    }
}

/* src/update_s2D.cl:30-327 */
static void port_update_s2d(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NZ = s->NZp, NX = s->NXp, nz = c->nz, L = c->L;
    const double *hc = s->hc;
    const double DT = s->DT, DT2 = s->DT2;
    const float *vx = s->w[W_VX], *vz = s->w[W_VZ];
    float *sxx = s->w[W_SXX], *szz = s->w[W_SZZ], *sxz = s->w[W_SXZ];
    float *rxx = s->r[R_XX], *rzz = s->r[R_ZZ], *rxz = s->r[R_XZ];
    const float *M = s->p[P_M], *mu = s->p[P_MU], *muipkp = s->p[P_MUIPKP];
    const float *taup = s->p[P_TAUP], *taus = s->p[P_TAUS], *tausipkp = s->p[P_TAUSIPKP];
    const i64 NXNZ = (i64)NX * NZ;
#pragma omp parallel for schedule(static)
    for (int gx = F; gx < NX - F; gx++)
        for (int gz = F; gz < NZ - F; gz++) {
            i64 ip = (i64)(gx - F) * nz + (gz - F), iv = (i64)gx * NZ + gz;
            float vxx = dbw(vx, iv, NZ, hc, F);
            float vxz = dfw(vx, iv, 1, hc, F);
            float vzz = dbw(vz, iv, 1, hc, F);
            float vzx = dfw(vz, iv, NZ, hc, F);
            if (c->abs_type == 1) cpml_s2d(s, gz, gx, &vxx, &vxz, &vzx, &vzz);
            if (L == 0) {
                float fipkp = muipkp[ip];
                float f = 2.0 * mu[ip];
                float g = M[ip];
                sxz[iv] += (fipkp * (vxz + vzx));
                sxx[iv] += (g * (vxx + vzz)) - (f * vzz);
                szz[iv] += (g * (vxx + vzz)) - (f * vxx);
            } else {
                float lM = M[ip], lmu = mu[ip], lmuipkp = muipkp[ip];
                float ltaup = taup[ip], ltaus = taus[ip], ltausipkp = tausipkp[ip];
                float fipkp = lmuipkp * (1.0 + (float)L * ltausipkp);
                float g = lM * (1.0 + (float)L * ltaup);
                float f = 2.0 * lmu * (1.0 + (float)L * ltaus);
                float dipkp = lmuipkp * ltausipkp / DT;
                float d = 2.0 * lmu * ltaus / DT;
                float e = lM * ltaup / DT;
                float sumrxz = 0, sumrxx = 0, sumrzz = 0;
                for (int l = 0; l < L; l++) {
                    i64 ir = l * NXNZ + iv;
                    sumrxz += rxz[ir];
                    sumrxx += rxx[ir];
                    sumrzz += rzz[ir];
                }
                float lsxz = (fipkp * (vxz + vzx)) + (DT2 * sumrxz);
                float lsxx = ((g * (vxx + vzz)) - (f * vzz)) + (DT2 * sumrxx);
                float lszz = ((g * (vxx + vzz)) - (f * vxx)) + (DT2 * sumrzz);
                sumrxz = sumrxx = sumrzz = 0;
                for (int l = 0; l < L; l++) {
                    float b = 1.0 / (1.0 + (s->eta[l] * 0.5));
                    float cc = 1.0 - (s->eta[l] * 0.5);
                    float el = s->eta[l];
                    i64 ir = l * NXNZ + iv;
                    rxz[ir] = b * (rxz[ir] * cc - el * (dipkp * (vxz + vzx)));
                    rxx[ir] = b * (rxx[ir] * cc - el * ((e * (vxx + vzz)) - (d * vzz)));
                    rzz[ir] = b * (rzz[ir] * cc - el * ((e * (vxx + vzz)) - (d * vxx)));
                    sumrxz += rxz[ir];
                    sumrxx += rxx[ir];
                    sumrzz += rzz[ir];
                }
                sxz[iv] += lsxz + (DT2 * sumrxz);
                sxx[iv] += lsxx + (DT2 * sumrxx);
                szz[iv] += lszz + (DT2 * sumrzz);
            }
            if (c->abs_type == 2) {
                float *f[3] = {sxx, szz, sxz};
                taper2d(s, gz, gx, f, 3, iv);
            }
        }
}

/* src/surface2D.cl:30-193 */
static void port_surface2d(fdo_state *s, int pdir)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NZ = s->NZp, NX = s->NXp, nz = c->nz, L = c->L, NAB = c->nab;
    const double *hc = s->hc;
    const double DT = s->DT, DT2 = s->DT2;
    float *vx = s->w[W_VX], *vz = s->w[W_VZ];
    float *sxx = s->w[W_SXX], *szz = s->w[W_SZZ], *sxz = s->w[W_SXZ];
    float *rxx = s->r[R_XX], *rzz = s->r[R_ZZ];
    const float *M = s->p[P_M], *mu = s->p[P_MU], *taup = s->p[P_TAUP], *taus = s->p[P_TAUS];
    const i64 NXNZ = (i64)NX * NZ;
    int gz = F;
    for (int gx = F; gx <= NX - F - 1; gx++) {
        i64 ip = (i64)(gx - F) * nz + (gz - F);
        szz[(i64)gx * NZ + gz] = 0.0;
        for (int l = 0; l < L; l++) rzz[l * NXNZ + (i64)gx * NZ + gz] = 0.0;
        for (int m = 1; m <= F; m++) {
            szz[(i64)gx * NZ + gz - m] = -szz[(i64)gx * NZ + gz + m];
            sxz[(i64)gx * NZ + gz - m] = -sxz[(i64)gx * NZ + gz + m - 1];
        }
        i64 iv = (i64)gx * NZ + gz;
        float vxx = dbw(vx, iv, NZ, hc, F);
        float vzz = dbw(vz, iv, 1, hc, F);
        if (c->abs_type == 1) {
            if (gx - F < NAB) {
                int i = gx - F, k = gz - F;
                vxx = vxx / s->cx[C_K][i] + s->psi[PS_VX_X][(i64)i * nz + k];
            }
            if (gx > NX - NAB - F - 1) {
                int i = gx - NX + NAB + F + NAB, k = gz - F, ind = 2 * NAB - 1 - i;
                vxx = vxx / s->cx[C_K][ind + 1] + s->psi[PS_VX_X][(i64)i * nz + k];
            }
        }
        if (L == 0) {
            float f = mu[ip] * 2.0;
            float g = M[ip];
            float h = -((g - f) * (g - f) * (vxx) / g) - ((g - f) * vzz);
            sxx[iv] += pdir * h;
        } else {
            float f = mu[ip] * 2.0 * (1.0 + L * taus[ip]);
            float g = M[ip] * (1.0 + L * taup[ip]);
            float h = -((g - f) * (g - f) * (vxx) / g) - ((g - f) * vzz);
            float sump = 0;
            for (int l = 0; l < L; l++) sump += rxx[l * NXNZ + iv];
            h += -DT2 * sump;
            sxx[iv] += pdir * h;
            float d = 2.0 * mu[ip] * taus[ip] / DT;
            float e = M[ip] * taup[ip] / DT;
            sump = 0;
            for (int l = 0; l < L; l++) {
                float b = s->eta[l] / (1.0 + (s->eta[l] * 0.5));
                h = b * (((d - e) * ((f / g) - 1.0) * vxx) - ((d - e) * vzz));
                rxx[l * NXNZ + iv] += pdir * h;
                sump += rxx[l * NXNZ + iv];
            }
            sxx[iv] += pdir * (DT2 * sump);
        }
    }
}

/* ---- boundary shells (single device), src/savebnd2D.cl:43-93 and
 * src/header_injectbnd.cl:238-283 ---- */
static void bnd_dims(const fdo_state *s, int *NXbnd, int *NYbnd, int *NZbnd, int *lbnd, int *lbnds)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NAB = c->nab;
    *NXbnd = s->NXp - 2 * F - 2 * NAB;
    *NYbnd = c->nd == 3 ? s->NYp - 2 * F - 2 * NAB : 1;
    if (!c->freesurf) {
        *NZbnd = s->NZp - 2 * F - 2 * NAB;
        *lbnd = F + NAB;
        *lbnds = F + NAB;
    } else {
        *NZbnd = s->NZp - 2 * F - NAB;
        *lbnd = F + NAB;
        *lbnds = F;
    }
}

static int inject_ind2d(const fdo_state *s, int k, int i)
{
    int F = s->c.fdoh, NXbnd, NYbnd, NZbnd, lbnd, lbnds;
    bnd_dims(s, &NXbnd, &NYbnd, &NZbnd, &lbnd, &lbnds);
    int m = -1;
    i -= lbnd;
    k -= lbnds;
    if ((k > F - 1 && k < NZbnd - F) && (i > F - 1 && i < NXbnd - F)) m = -1;
    else if (k < 0 || k > NZbnd - 1 || i < 0 || i > NXbnd - 1) m = -1;
    else if (i < F) m = i * NZbnd + k;
    else if (i > NXbnd - 1 - F) { i = i - NXbnd + F; m = NZbnd * F + i * NZbnd + k; }
    else if (k < F) { i = i - F; m = NZbnd * F * 2 + (NXbnd - 2 * F) * F + i + k * (NXbnd - 2.0 * F); }
    else { i = i - F; k = k - NZbnd + F; m = NZbnd * F * 2 + i + k * (NXbnd - 2.0 * F); }
    return m;
}

static int savebnd_cell2d(const fdo_state *s, int gid, int *pi, int *pk)
{
    int F = s->c.fdoh, NAB = s->c.nab, NXbnd, NYbnd, NZbnd, lbnd, lbnds, i, k, gidf;
    bnd_dims(s, &NXbnd, &NYbnd, &NZbnd, &lbnd, &lbnds);
    if (gid < NZbnd * F) { gidf = gid; i = gidf / NZbnd + lbnd; k = gidf % NZbnd + lbnds; }
    else if (gid < NZbnd * F * 2) { gidf = gid - NZbnd * F; i = gidf / NZbnd + NXbnd + NAB; k = gidf % NZbnd + lbnds; }
    else if (gid < NZbnd * F * 2 + (NXbnd - 2 * F) * F) {
        gidf = gid - NZbnd * F * 2;
        i = gidf % (NXbnd - 2 * F) + lbnd + F;
        k = gidf / (NXbnd - 2 * F) + NZbnd + lbnds - F;
    } else if (gid < NZbnd * F * 2 + (NXbnd - 2 * F) * 2 * F) {
        gidf = gid - NZbnd * F * 2 - (NXbnd - 2 * F) * F;
        i = gidf % (NXbnd - 2 * F) + lbnd + F;
        k = gidf / (NXbnd - 2 * F) + lbnds;
    } else return 0;
    *pi = i; *pk = k;
    return 1;
}

/* ======================================================================
 * 3D
 * ====================================================================== */
#define IV3(z, y, x) (((i64)(x) * NY + (y)) * NZ + (z))

/* src/update_v3D.cl:209-314 */
static void cpml_v3d(fdo_state *s, int gz, int gy, int gx, float *sxx_x, float *syy_y, float *szz_z,
                     float *sxy_y, float *sxy_x, float *syz_y, float *syz_z, float *sxz_x, float *sxz_z)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NAB = c->nab, NZ = s->NZp, NY = s->NYp, NX = s->NXp;
    i64 nz = c->nz, ny = c->ny;
    float **ps = s->psi;
    if (gz > NZ - NAB - F - 1) {
        i64 i = gx - F, j = gy - F, k = gz - NZ + NAB + F + NAB;
        int ind = 2 * NAB - 1 - (int)k;
        i64 q = (i * ny + j) * (2 * NAB) + k;
        CPML(ps[PS_SXZ_Z], q, s->cz[C_K], s->cz[C_A], s->cz[C_B], ind + 1, *sxz_z);
        CPML(ps[PS_SYZ_Z], q, s->cz[C_K], s->cz[C_A], s->cz[C_B], ind + 1, *syz_z);
        CPML(ps[PS_SZZ_Z], q, s->cz[C_KH], s->cz[C_AH], s->cz[C_BH], ind, *szz_z);
    } else if (!c->freesurf && gz - F < NAB) {
        i64 i = gx - F, j = gy - F, k = gz - F;
        i64 q = (i * ny + j) * (2 * NAB) + k;
        CPML(ps[PS_SXZ_Z], q, s->cz[C_K], s->cz[C_A], s->cz[C_B], k, *sxz_z);
        CPML(ps[PS_SYZ_Z], q, s->cz[C_K], s->cz[C_A], s->cz[C_B], k, *syz_z);
        CPML(ps[PS_SZZ_Z], q, s->cz[C_KH], s->cz[C_AH], s->cz[C_BH], k, *szz_z);
    }
    if (gy - F < NAB) {
        i64 i = gx - F, j = gy - F, k = gz - F;
        i64 q = (i * (2 * NAB) + j) * nz + k;
        CPML(ps[PS_SXY_Y], q, s->cy[C_K], s->cy[C_A], s->cy[C_B], j, *sxy_y);
        CPML(ps[PS_SYY_Y], q, s->cy[C_KH], s->cy[C_AH], s->cy[C_BH], j, *syy_y);
        CPML(ps[PS_SYZ_Y], q, s->cy[C_K], s->cy[C_A], s->cy[C_B], j, *syz_y);
    } else if (gy > NY - NAB - F - 1) {
        i64 i = gx - F, j = gy - NY + NAB + F + NAB, k = gz - F;
        int ind = 2 * NAB - 1 - (int)j;
        i64 q = (i * (2 * NAB) + j) * nz + k;
        CPML(ps[PS_SXY_Y], q, s->cy[C_K], s->cy[C_A], s->cy[C_B], ind + 1, *sxy_y);
        CPML(ps[PS_SYY_Y], q, s->cy[C_KH], s->cy[C_AH], s->cy[C_BH], ind, *syy_y);
        CPML(ps[PS_SYZ_Y], q, s->cy[C_K], s->cy[C_A], s->cy[C_B], ind + 1, *syz_y);
    }
    if (gx - F < NAB) {
        i64 i = gx - F, j = gy - F, k = gz - F;
        i64 q = (i * ny + j) * nz + k;
        CPML(ps[PS_SXX_X], q, s->cx[C_KH], s->cx[C_AH], s->cx[C_BH], i, *sxx_x);
        CPML(ps[PS_SXY_X], q, s->cx[C_K], s->cx[C_A], s->cx[C_B], i, *sxy_x);
        CPML(ps[PS_SXZ_X], q, s->cx[C_K], s->cx[C_A], s->cx[C_B], i, *sxz_x);
    }
    if (gx > NX - NAB - F - 1) {
        i64 i = gx - NX + NAB + F + NAB, j = gy - F, k = gz - F;
        int ind = 2 * NAB - 1 - (int)i;
        i64 q = (i * ny + j) * nz + k;
        CPML(ps[PS_SXX_X], q, s->cx[C_KH], s->cx[C_AH], s->cx[C_BH], ind, *sxx_x);
        CPML(ps[PS_SXY_X], q, s->cx[C_K], s->cx[C_A], s->cx[C_B], ind + 1, *sxy_x);
        CPML(ps[PS_SXZ_X], q, s->cx[C_K], s->cx[C_A], s->cx[C_B], ind + 1, *sxz_x);
    }
}

static void taper3d(fdo_state *s, int gz, int gy, int gx, float **f, int nf, i64 iv)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NAB = c->nab, NZ = s->NZp, NY = s->NYp, NX = s->NXp;
    if (!c->freesurf && gz - F < NAB)
        for (int q = 0; q < nf; q++) f[q][iv] *= s->taper[gz - F];
    if (gz > NZ - NAB - F - 1)
        for (int q = 0; q < nf; q++) f[q][iv] *= s->taper[NZ - F - gz - 1];
    if (gy - F < NAB)
        for (int q = 0; q < nf; q++) f[q][iv] *= s->taper[gy - F];
    if (gy > NY - NAB - F - 1)
        for (int q = 0; q < nf; q++) f[q][iv] *= s->taper[NY - F - gy - 1];
    if (gx - F < NAB)
        for (int q = 0; q < nf; q++) f[q][iv] *= s->taper[gx - F];
    if (gx > NX - NAB - F - 1)
        for (int q = 0; q < nf; q++) f[q][iv] *= s->taper[NX - F - gx - 1];
}

/* src/update_v3D.cl:34-369 */
static void port_update_v3d(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NZ = s->NZp, NY = s->NYp, NX = s->NXp;
    i64 nz = c->nz, ny = c->ny;
    const double *hc = s->hc;
    float *vx = s->w[W_VX], *vy = s->w[W_VY], *vz = s->w[W_VZ];
    const float *sxx = s->w[W_SXX], *syy = s->w[W_SYY], *szz = s->w[W_SZZ];
    const float *sxy = s->w[W_SXY], *syz = s->w[W_SYZ], *sxz = s->w[W_SXZ];
    const float *rip = s->p[P_RIP], *rjp = s->p[P_RJP], *rkp = s->p[P_RKP];
    const i64 sx = (i64)NY * NZ, sy = NZ;
#pragma omp parallel for collapse(2) schedule(static)
    for (int gx = F; gx < NX - F; gx++)
        for (int gy = F; gy < NY - F; gy++)
            for (int gz = F; gz < NZ - F; gz++) {
                i64 ip = ((i64)(gx - F) * ny + (gy - F)) * nz + (gz - F), iv = IV3(gz, gy, gx);
                float szz_z = dfw(szz, iv, 1, hc, F);
                float sxx_x = dfw(sxx, iv, sx, hc, F);
                float sxz_x = dbw(sxz, iv, sx, hc, F);
                float sxz_z = dbw(sxz, iv, 1, hc, F);
                float syz_y = dbw(syz, iv, sy, hc, F);
                float syz_z = dbw(syz, iv, 1, hc, F);
                float syy_y = dfw(syy, iv, sy, hc, F);
                float sxy_x = dbw(sxy, iv, sx, hc, F);
                float sxy_y = dbw(sxy, iv, sy, hc, F);
                if (c->abs_type == 1)
                    cpml_v3d(s, gz, gy, gx, &sxx_x, &syy_y, &szz_z, &sxy_y, &sxy_x, &syz_y, &syz_z, &sxz_x,
                             &sxz_z);
                vx[iv] += ((sxx_x + sxy_y + sxz_z) * rip[ip]);
                vy[iv] += ((syy_y + sxy_x + syz_z) * rjp[ip]);
                vz[iv] += ((szz_z + sxz_x + syz_y) * rkp[ip]);
                if (c->abs_type == 2) {
                    float *f[3] = {vx, vy, vz};
                    taper3d(s, gz, gy, gx, f, 3, iv);
                }
            }
}

/* src/update_s3D.cl:190-298.  Note the z-top and y-far branches are separate
 * "if"s here, unlike update_v3D. */
static void cpml_s3d(fdo_state *s, int gz, int gy, int gx, float *vxx, float *vxy, float *vxz, float *vyx,
                     float *vyy, float *vyz, float *vzx, float *vzy, float *vzz, int adjoint_form)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NAB = c->nab, NZ = s->NZp, NY = s->NYp, NX = s->NXp;
    i64 nz = c->nz, ny = c->ny;
    float **ps = s->psi;
    int zb = gz > NZ - NAB - F - 1;
    if (zb) {
        i64 i = gx - F, j = gy - F, k = gz - NZ + NAB + F + NAB;
        int ind = 2 * NAB - 1 - (int)k;
        i64 q = (i * ny + j) * (2 * NAB) + k;
        CPML(ps[PS_VX_Z], q, s->cz[C_KH], s->cz[C_AH], s->cz[C_BH], ind, *vxz);
        CPML(ps[PS_VY_Z], q, s->cz[C_KH], s->cz[C_AH], s->cz[C_BH], ind, *vyz);
        CPML(ps[PS_VZ_Z], q, s->cz[C_K], s->cz[C_A], s->cz[C_B], ind + 1, *vzz);
    }
    /* update_s3D.cl:211 is a plain "if"; update_adjs3D.cl uses "else if" */
    if (!c->freesurf && gz - F < NAB && !(adjoint_form && zb)) {
        i64 i = gx - F, j = gy - F, k = gz - F;
        i64 q = (i * ny + j) * (2 * NAB) + k;
        CPML(ps[PS_VX_Z], q, s->cz[C_KH], s->cz[C_AH], s->cz[C_BH], k, *vxz);
        CPML(ps[PS_VY_Z], q, s->cz[C_KH], s->cz[C_AH], s->cz[C_BH], k, *vyz);
        CPML(ps[PS_VZ_Z], q, s->cz[C_K], s->cz[C_A], s->cz[C_B], k, *vzz);
    }
    int yb = gy - F < NAB;
    if (yb) {
        i64 i = gx - F, j = gy - F, k = gz - F;
        i64 q = (i * (2 * NAB) + j) * nz + k;
        CPML(ps[PS_VX_Y], q, s->cy[C_KH], s->cy[C_AH], s->cy[C_BH], j, *vxy);
        CPML(ps[PS_VY_Y], q, s->cy[C_K], s->cy[C_A], s->cy[C_B], j, *vyy);
        CPML(ps[PS_VZ_Y], q, s->cy[C_KH], s->cy[C_AH], s->cy[C_BH], j, *vzy);
    }
    if (gy > NY - NAB - F - 1 && !(adjoint_form && yb)) {
        i64 i = gx - F, j = gy - NY + NAB + F + NAB, k = gz - F;
        int ind = 2 * NAB - 1 - (int)j;
        i64 q = (i * (2 * NAB) + j) * nz + k;
        CPML(ps[PS_VX_Y], q, s->cy[C_KH], s->cy[C_AH], s->cy[C_BH], ind, *vxy);
        CPML(ps[PS_VY_Y], q, s->cy[C_K], s->cy[C_A], s->cy[C_B], ind + 1, *vyy);
        CPML(ps[PS_VZ_Y], q, s->cy[C_KH], s->cy[C_AH], s->cy[C_BH], ind, *vzy);
    }
    if (gx - F < NAB) {
        i64 i = gx - F, j = gy - F, k = gz - F;
        i64 q = (i * ny + j) * nz + k;
        CPML(ps[PS_VX_X], q, s->cx[C_K], s->cx[C_A], s->cx[C_B], i, *vxx);
        CPML(ps[PS_VY_X], q, s->cx[C_KH], s->cx[C_AH], s->cx[C_BH], i, *vyx);
        CPML(ps[PS_VZ_X], q, s->cx[C_KH], s->cx[C_AH], s->cx[C_BH], i, *vzx);
    }
    if (gx > NX - NAB - F - 1) {
        i64 i = gx - NX + NAB + F + NAB, j = gy - F, k = gz - F;
        int ind = 2 * NAB - 1 - (int)i;
        i64 q = (i * ny + j) * nz + k;
        CPML(ps[PS_VX_X], q, s->cx[C_K], s->cx[C_A], s->cx[C_B], ind + 1, *vxx);
        CPML(ps[PS_VY_X], q, s->cx[C_KH], s->cx[C_AH], s->cx[C_BH], ind, *vyx);
        CPML(ps[PS_VZ_X], q, s->cx[C_KH], s->cx[C_AH], s->cx[C_BH], ind, *vzx);
    }
}

/* src/update_s3D.cl:35-489 */
static void port_update_s3d(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NZ = s->NZp, NY = s->NYp, NX = s->NXp, L = c->L;
    i64 nz = c->nz, ny = c->ny;
    const double *hc = s->hc;
    const double DT = s->DT, DT2 = s->DT2;
    const float *vx = s->w[W_VX], *vy = s->w[W_VY], *vz = s->w[W_VZ];
    float *sxx = s->w[W_SXX], *syy = s->w[W_SYY], *szz = s->w[W_SZZ];
    float *sxy = s->w[W_SXY], *syz = s->w[W_SYZ], *sxz = s->w[W_SXZ];
    float *rxx = s->r[R_XX], *ryy = s->r[R_YY], *rzz = s->r[R_ZZ];
    float *rxy = s->r[R_XY], *ryz = s->r[R_YZ], *rxz = s->r[R_XZ];
    const float *M = s->p[P_M], *mu = s->p[P_MU];
    const float *muipjp = s->p[P_MUIPJP], *mujpkp = s->p[P_MUJPKP], *muipkp = s->p[P_MUIPKP];
    const float *taup = s->p[P_TAUP], *taus = s->p[P_TAUS];
    const float *tausipjp = s->p[P_TAUSIPJP], *tausjpkp = s->p[P_TAUSJPKP], *tausipkp = s->p[P_TAUSIPKP];
    const i64 sx = (i64)NY * NZ, sy = NZ, NV = (i64)NX * NY * NZ;
#pragma omp parallel for collapse(2) schedule(static)
    for (int gx = F; gx < NX - F; gx++)
        for (int gy = F; gy < NY - F; gy++)
            for (int gz = F; gz < NZ - F; gz++) {
                i64 ip = ((i64)(gx - F) * ny + (gy - F)) * nz + (gz - F), iv = IV3(gz, gy, gx);
                float vzx = dfw(vz, iv, sx, hc, F);
                float vzy = dfw(vz, iv, sy, hc, F);
                float vzz = dbw(vz, iv, 1, hc, F);
                float vyx = dfw(vy, iv, sx, hc, F);
                float vyy = dbw(vy, iv, sy, hc, F);
                float vyz = dfw(vy, iv, 1, hc, F);
                float vxx = dbw(vx, iv, sx, hc, F);
                float vxy = dfw(vx, iv, sy, hc, F);
                float vxz = dfw(vx, iv, 1, hc, F);
                if (c->abs_type == 1) cpml_s3d(s, gz, gy, gx, &vxx, &vxy, &vxz, &vyx, &vyy, &vyz, &vzx, &vzy, &vzz, 0);
                float vxyyx = vxy + vyx, vyzzy = vyz + vzy, vxzzx = vxz + vzx;
                float vxxyyzz = vxx + vyy + vzz, vyyzz = vyy + vzz, vxxzz = vxx + vzz, vxxyy = vxx + vyy;
                if (L == 0) {
                    float fipjp = muipjp[ip], fjpkp = mujpkp[ip], fipkp = muipkp[ip];
                    float g = M[ip];
                    float f = 2.0 * mu[ip];
                    sxy[iv] += (fipjp * vxyyx);
                    syz[iv] += (fjpkp * vyzzy);
                    sxz[iv] += (fipkp * vxzzx);
                    sxx[iv] += ((g * vxxyyzz) - (f * vyyzz));
                    syy[iv] += ((g * vxxyyzz) - (f * vxxzz));
                    szz[iv] += ((g * vxxyyzz) - (f * vxxyy));
                } else {
                    float lM = M[ip], lmu = mu[ip];
                    float lmuipkp = muipkp[ip], lmuipjp = muipjp[ip], lmujpkp = mujpkp[ip];
                    float ltaup = taup[ip], ltaus = taus[ip];
                    float ltausipkp = tausipkp[ip], ltausipjp = tausipjp[ip], ltausjpkp = tausjpkp[ip];
                    float fipjp = lmuipjp * (1.0 + (float)L * ltausipjp);
                    float fjpkp = lmujpkp * (1.0 + (float)L * ltausjpkp);
                    float fipkp = lmuipkp * (1.0 + (float)L * ltausipkp);
                    float g = lM * (1.0 + (float)L * ltaup);
                    float f = 2.0 * lmu * (1.0 + (float)L * ltaus);
                    float dipjp = lmuipjp * ltausipjp / DT;
                    float djpkp = lmujpkp * ltausjpkp / DT;
                    float dipkp = lmuipkp * ltausipkp / DT;
                    float d = 2.0 * lmu * ltaus / DT;
                    float e = lM * ltaup / DT;
                    float sxy_ = 0, syz_ = 0, sxz_ = 0, sxx_ = 0, syy_ = 0, szz_ = 0;
                    for (int l = 0; l < L; l++) {
                        i64 ir = l * NV + iv;
                        sxy_ += rxy[ir]; syz_ += ryz[ir]; sxz_ += rxz[ir];
                        sxx_ += rxx[ir]; syy_ += ryy[ir]; szz_ += rzz[ir];
                    }
                    float lsxy = (fipjp * vxyyx) + (DT2 * sxy_);
                    float lsyz = (fjpkp * vyzzy) + (DT2 * syz_);
                    float lsxz = (fipkp * vxzzx) + (DT2 * sxz_);
                    float lsxx = ((g * vxxyyzz) - (f * vyyzz)) + (DT2 * sxx_);
                    float lsyy = ((g * vxxyyzz) - (f * vxxzz)) + (DT2 * syy_);
                    float lszz = ((g * vxxyyzz) - (f * vxxyy)) + (DT2 * szz_);
                    sxy_ = syz_ = sxz_ = sxx_ = syy_ = szz_ = 0;
                    for (int l = 0; l < L; l++) {
                        float el = s->eta[l];
                        float b = 1.0 / (1.0 + (el * 0.5));
                        float cc = 1.0 - (el * 0.5);
                        i64 ir = l * NV + iv;
                        rxy[ir] = b * (rxy[ir] * cc - el * (dipjp * vxyyx));
                        ryz[ir] = b * (ryz[ir] * cc - el * (djpkp * vyzzy));
                        rxz[ir] = b * (rxz[ir] * cc - el * (dipkp * vxzzx));
                        rxx[ir] = b * (rxx[ir] * cc - el * ((e * vxxyyzz) - (d * vyyzz)));
                        ryy[ir] = b * (ryy[ir] * cc - el * ((e * vxxyyzz) - (d * vxxzz)));
                        rzz[ir] = b * (rzz[ir] * cc - el * ((e * vxxyyzz) - (d * vxxyy)));
                        sxy_ += rxy[ir]; syz_ += ryz[ir]; sxz_ += rxz[ir];
                        sxx_ += rxx[ir]; syy_ += ryy[ir]; szz_ += rzz[ir];
                    }
                    sxy[iv] += lsxy + (DT2 * sxy_);
                    syz[iv] += lsyz + (DT2 * syz_);
                    sxz[iv] += lsxz + (DT2 * sxz_);
                    sxx[iv] += lsxx + (DT2 * sxx_);
                    syy[iv] += lsyy + (DT2 * syy_);
                    szz[iv] += lszz + (DT2 * szz_);
                }
                if (c->abs_type == 2) {
                    float *f[6] = {sxy, syz, sxz, sxx, syy, szz};
                    taper3d(s, gz, gy, gx, f, 6, iv);
                }
            }
}

/* src/surface3D.cl:39-271.  The elastic branch adds h without pdir
 * (:172-173), as does the viscoelastic rxx/ryy update (:233-234). */
static void port_surface3d(fdo_state *s, int pdir)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NZ = s->NZp, NY = s->NYp, NX = s->NXp, L = c->L, NAB = c->nab;
    i64 nz = c->nz, ny = c->ny;
    const double *hc = s->hc;
    const double DT = s->DT, DT2 = s->DT2;
    float *vx = s->w[W_VX], *vy = s->w[W_VY], *vz = s->w[W_VZ];
    float *sxx = s->w[W_SXX], *syy = s->w[W_SYY], *szz = s->w[W_SZZ];
    float *syz = s->w[W_SYZ], *sxz = s->w[W_SXZ];
    float *rxx = s->r[R_XX], *ryy = s->r[R_YY], *rzz = s->r[R_ZZ];
    const float *M = s->p[P_M], *mu = s->p[P_MU], *taup = s->p[P_TAUP], *taus = s->p[P_TAUS];
    const i64 sx = (i64)NY * NZ, sy = NZ, NV = (i64)NX * NY * NZ;
    int gz = F;
#pragma omp parallel for collapse(2) schedule(static)
    for (int gx = F; gx <= NX - F - 1; gx++)
        for (int gy = F; gy <= NY - F - 1; gy++) {
            i64 ip = ((i64)(gx - F) * ny + (gy - F)) * nz + (gz - F);
            i64 iv = IV3(gz, gy, gx);
            szz[iv] = 0.0;
            for (int l = 0; l < L; l++) rzz[l * NV + iv] = 0.0;
            for (int m = 1; m <= F; m++) {
                szz[iv - m] = -szz[iv + m];
                sxz[iv - m] = -sxz[iv + m - 1];
                syz[iv - m] = -syz[iv + m - 1];
            }
            float vxx = dbw(vx, iv, sx, hc, F);
            float vyy = dbw(vy, iv, sy, hc, F);
            float vzz = dbw(vz, iv, 1, hc, F);
            if (c->abs_type == 1) {
                if (gy - F < NAB) {
                    i64 i = gx - F, j = gy - F, k = gz - F;
                    vyy = vyy / s->cy[C_K][j] + s->psi[PS_VY_Y][(i * (2 * NAB) + j) * nz + k];
                } else if (gy > NY - NAB - F - 1) {
                    i64 i = gx - F, j = gy - NY + NAB + F + NAB, k = gz - F;
                    int ind = 2 * NAB - 1 - (int)j;
                    vyy = vyy / s->cy[C_K][ind + 1] + s->psi[PS_VY_Y][(i * (2 * NAB) + j) * nz + k];
                }
                /* the reference guards these with the undefined macro DEV (== 0),
                 * which is true on a single device */
                if (gx - F < NAB) {
                    i64 i = gx - F, j = gy - F, k = gz - F;
                    vxx = vxx / s->cx[C_K][i] + s->psi[PS_VX_X][(i * ny + j) * nz + k];
                }
                if (gx > NX - NAB - F - 1) {
                    i64 i = gx - NX + NAB + F + NAB, j = gy - F, k = gz - F;
                    int ind = 2 * NAB - 1 - (int)i;
                    vxx = vxx / s->cx[C_K][ind + 1] + s->psi[PS_VX_X][(i * ny + j) * nz + k];
                }
            }
            if (L == 0) {
                float f = mu[ip] * 2.0f;
                float g = M[ip];
                float h = -((g - f) * (g - f) * (vxx + vyy) / g) - ((g - f) * vzz);
                sxx[iv] += h;
                syy[iv] += h;
            } else {
                float f = mu[ip] * 2.0 * (1.0 + L * taus[ip]);
                float g = M[ip] * (1.0 + L * taup[ip]);
                float h = -((g - f) * (g - f) * (vxx + vyy) / g) - ((g - f) * vzz);
                float sumx = 0, sumy = 0;
                for (int l = 0; l < L; l++) {
                    sumx += rxx[l * NV + iv];
                    sumy += ryy[l * NV + iv];
                }
                sxx[iv] += pdir * (h - DT2 * sumx);
                syy[iv] += pdir * (h - DT2 * sumy);
                float d = 2.0 * mu[ip] * taus[ip] / DT;
                float e = M[ip] * taup[ip] / DT;
                sumx = 0; sumy = 0;
                for (int l = 0; l < L; l++) {
                    float b = s->eta[l] / (1.0 + (s->eta[l] * 0.5));
                    h = b * (((d - e) * ((f / g) - 1.0) * (vxx + vyy)) - ((d - e) * vzz));
                    rxx[l * NV + iv] += h;
                    ryy[l * NV + iv] += h;
                    sumx += rxx[l * NV + iv];
                    sumy += ryy[l * NV + iv];
                }
                sxx[iv] += (DT2 * sumx);
                syy[iv] += (DT2 * sumy);
            }
        }
}

/* src/header_injectbnd.cl:25-84 */
static int inject_ind3d(const fdo_state *s, int k, int j, int i)
{
    int F = s->c.fdoh, NXbnd, NYbnd, NZbnd, lbnd, lbnds;
    bnd_dims(s, &NXbnd, &NYbnd, &NZbnd, &lbnd, &lbnds);
    int m = -1;
    i -= lbnd; j -= lbnd; k -= lbnds;
    if ((k > F - 1 && k < NZbnd - F) && (j > F - 1 && j < NYbnd - F) && (i > F - 1 && i < NXbnd - F)) m = -1;
    else if (k < 0 || k > NZbnd - 1 || j < 0 || j > NYbnd - 1 || i < 0 || i > NXbnd - 1) m = -1;
    else if (i < F) m = i * NYbnd * NZbnd + j * NZbnd + k;
    else if (i > NXbnd - 1 - F) { i = i - NXbnd + F; m = NYbnd * NZbnd * F + i * NYbnd * NZbnd + j * NZbnd + k; }
    else if (j < F) { i = i - F; m = NYbnd * NZbnd * F * 2 + i * F * NZbnd + j * NZbnd + k; }
    else if (j > NYbnd - 1 - F) {
        i = i - F; j = j - NYbnd + F;
        m = NYbnd * NZbnd * F * 2 + (NXbnd - 2 * F) * NZbnd * F + i * F * NZbnd + j * NZbnd + k;
    } else if (k < F) {
        i = i - F; j = j - F;
        m = NYbnd * NZbnd * F * 2 + (NXbnd - 2 * F) * NZbnd * F * 2 + (NXbnd - 2 * F) * (NYbnd - 2 * F) * F +
            i * (NYbnd - 2 * F) * F + j * F + k;
    } else {
        i = i - F; j = j - F; k = k - NZbnd + F;
        m = NYbnd * NZbnd * F * 2 + (NXbnd - 2 * F) * NZbnd * F * 2 + i * (NYbnd - 2 * F) * F + j * F + k;
    }
    return m;
}

/* src/savebnd3D.cl:38-103 */
static int savebnd_cell3d(const fdo_state *s, int gid, int *pi, int *pj, int *pk)
{
    int F = s->c.fdoh, NAB = s->c.nab, NXbnd, NYbnd, NZbnd, lbnd, lbnds, i, j, k, gidf;
    bnd_dims(s, &NXbnd, &NYbnd, &NZbnd, &lbnd, &lbnds);
    int a0 = NYbnd * NZbnd * F, a1 = NZbnd * (NXbnd - 2 * F) * F, a2 = (NYbnd - 2 * F) * (NXbnd - 2 * F) * F;
    if (gid < a0) { gidf = gid; i = gidf / (NYbnd * NZbnd) + lbnd; j = (gidf / NZbnd) % NYbnd + lbnd; k = gidf % NZbnd + lbnds; }
    else if (gid < 2 * a0) { gidf = gid - a0; i = gidf / (NYbnd * NZbnd) + NXbnd + NAB; j = (gidf / NZbnd) % NYbnd + lbnd; k = gidf % NZbnd + lbnds; }
    else if (gid < 2 * a0 + a1) { gidf = gid - 2 * a0; i = gidf / (NZbnd * F) + lbnd + F; j = (gidf / NZbnd) % F + lbnd; k = gidf % NZbnd + lbnds; }
    else if (gid < 2 * a0 + 2 * a1) { gidf = gid - 2 * a0 - a1; i = gidf / (NZbnd * F) + lbnd + F; j = (gidf / NZbnd) % F + NYbnd + NAB; k = gidf % NZbnd + lbnds; }
    else if (gid < 2 * a0 + 2 * a1 + a2) {
        gidf = gid - 2 * a0 - 2 * a1;
        i = gidf / (F * (NYbnd - 2 * F)) + lbnd + F;
        j = (gidf / F) % (NYbnd - 2 * F) + lbnd + F;
        k = gidf % F + NZbnd + lbnds - F;
    } else if (gid < 2 * a0 + 2 * a1 + 2 * a2) {
        gidf = gid - 2 * a0 - 2 * a1 - a2;
        i = gidf / (F * (NYbnd - 2 * F)) + lbnd + F;
        j = (gidf / F) % (NYbnd - 2 * F) + lbnd + F;
        k = gidf % F + lbnds;
    } else return 0;
    *pi = i; *pj = j; *pk = k;
    return 1;
}

static void port_savebnd(fdo_state *s, int t)
{
    int NZ = s->NZp, NY = s->NYp;
    for (int gid = 0; gid < s->nbnd; gid++) {
        int i, j = 0, k;
        int ok = s->c.nd == 3 ? savebnd_cell3d(s, gid, &i, &j, &k) : savebnd_cell2d(s, gid, &i, &k);
        if (!ok) continue;
        i64 iv = IV3(k, j, i);
        for (int q = 0; q < s->nwave; q++) {
            int w = s->wave_ids[q];
            s->bnd[w][(i64)t * s->nbnd + gid] = s->w[w][iv];
        }
    }
}

/* ======================================================================
 * adjoint, 2D (src/update_adjv2D.cl, src/update_adjs2D.cl, surface2D_adj.cl)
 * ====================================================================== */
static void port_update_adjv2d(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    /* BACK_PROP_TYPE 2 compiles out the forward reconstruction, the
     * boundary injection and the gradient (#if BACK_PROP_TYPE==1 blocks) */
    const int bp1 = c->back_prop_type != 2;
    int F = c->fdoh, NZ = s->NZp, NX = s->NXp, nz = c->nz;
    const double *hc = s->hc;
    float *vx = s->w[W_VX], *vz = s->w[W_VZ];
    const float *sxx = s->w[W_SXX], *szz = s->w[W_SZZ], *sxz = s->w[W_SXZ];
    float *vxr = s->wr[W_VX], *vzr = s->wr[W_VZ];
    const float *sxxr = s->wr[W_SXX], *szzr = s->wr[W_SZZ], *sxzr = s->wr[W_SXZ];
    const float *rip = s->p[P_RIP], *rkp = s->p[P_RKP];
    float *gradrho = s->grad[G_RHO];
#pragma omp parallel for schedule(static)
    for (int gx = F; gx < NX - F; gx++)
        for (int gz = F; gz < NZ - F; gz++) {
            i64 ip = (i64)(gx - F) * nz + (gz - F), iv = (i64)gx * NZ + gz;
            float sxx_x = dfw(sxx, iv, NZ, hc, F);
            float szz_z = dfw(szz, iv, 1, hc, F);
            float sxz_z = dbw(sxz, iv, 1, hc, F);
            float sxz_x = dbw(sxz, iv, NZ, hc, F);
            float sxx_xr = dfw(sxxr, iv, NZ, hc, F);
            float szz_zr = dfw(szzr, iv, 1, hc, F);
            float sxz_zr = dbw(sxzr, iv, 1, hc, F);
            float sxz_xr = dbw(sxzr, iv, NZ, hc, F);
            float lvx = ((sxx_x + sxz_z) * rip[ip]);
            float lvz = ((szz_z + sxz_x) * rkp[ip]);
            if (bp1) {
                vx[iv] -= lvx;
                vz[iv] -= lvz;
                int m = inject_ind2d(s, gz, gx);
                if (m != -1) {
                    vx[iv] = s->bnd_cur[W_VX][m];
                    vz[iv] = s->bnd_cur[W_VZ][m];
                }
            }
            if (c->abs_type == 1) cpml_v2d(s, gz, gx, &sxx_xr, &szz_zr, &sxz_xr, &sxz_zr);
            lvx = ((sxx_xr + sxz_zr) * rip[ip]);
            lvz = ((szz_zr + sxz_xr) * rkp[ip]);
            vxr[iv] += lvx;
            vzr[iv] += lvz;
            if (c->abs_type == 2) {
                float *f[2] = {vxr, vzr};
                taper2d(s, gz, gx, f, 2, iv);
            }
            if (bp1) gradrho[ip] += -vx[iv] * lvx - vz[iv] * lvz;
        }
}

static void port_update_adjs2d(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    /* BACK_PROP_TYPE 2 compiles out the forward reconstruction, the
     * boundary injection and the gradient (#if BACK_PROP_TYPE==1 blocks) */
    const int bp1 = c->back_prop_type != 2;
    int F = c->fdoh, NZ = s->NZp, NX = s->NXp, nz = c->nz, L = c->L;
    const double *hc = s->hc;
    const double DT = s->DT, DT2 = s->DT2;
    const float *vx = s->w[W_VX], *vz = s->w[W_VZ];
    float *sxx = s->w[W_SXX], *szz = s->w[W_SZZ], *sxz = s->w[W_SXZ];
    const float *vxr = s->wr[W_VX], *vzr = s->wr[W_VZ];
    float *sxxr = s->wr[W_SXX], *szzr = s->wr[W_SZZ], *sxzr = s->wr[W_SXZ];
    float *rxx = s->r[R_XX], *rzz = s->r[R_ZZ], *rxz = s->r[R_XZ];
    float *rxxr = s->rr[R_XX], *rzzr = s->rr[R_ZZ], *rxzr = s->rr[R_XZ];
    const float *M = s->p[P_M], *mu = s->p[P_MU], *muipkp = s->p[P_MUIPKP];
    const float *taup = s->p[P_TAUP], *taus = s->p[P_TAUS], *tausipkp = s->p[P_TAUSIPKP];
    float *gradM = s->grad[G_M], *gradmu = s->grad[G_MU];
    const i64 NXNZ = (i64)NX * NZ;
#pragma omp parallel for schedule(static)
    for (int gx = F; gx < NX - F; gx++)
        for (int gz = F; gz < NZ - F; gz++) {
            i64 ip = (i64)(gx - F) * nz + (gz - F), iv = (i64)gx * NZ + gz;
            float vxx = dbw(vx, iv, NZ, hc, F);
            float vxz = dfw(vx, iv, 1, hc, F);
            float vzz = dbw(vz, iv, 1, hc, F);
            float vzx = dfw(vz, iv, NZ, hc, F);
            float vxxr = dbw(vxr, iv, NZ, hc, F);
            float vxzr = dfw(vxr, iv, 1, hc, F);
            float vzzr = dbw(vzr, iv, 1, hc, F);
            float vzxr = dfw(vzr, iv, NZ, hc, F);
            float fipkp, f, g, lM, lmu, dipkp = 0, d = 0, e = 0;
            if (L == 0) {
                fipkp = muipkp[ip]; lmu = mu[ip]; lM = M[ip];
                f = 2.0 * lmu; g = lM;
            } else {
                lM = M[ip]; lmu = mu[ip];
                float lmuipkp = muipkp[ip], ltaup = taup[ip], ltaus = taus[ip], ltausipkp = tausipkp[ip];
                fipkp = lmuipkp * (1.0 + (float)L * ltausipkp);
                g = lM * (1.0 + (float)L * ltaup);
                f = 2.0 * lmu * (1.0 + (float)L * ltaus);
                dipkp = lmuipkp * ltausipkp / DT;
                d = 2.0 * lmu * ltaus / DT;
                e = lM * ltaup / DT;
            }
            /* reconstruct the forward stresses (BACK_PROP_TYPE 1 only) */
            if (!bp1) {
            } else if (L == 0) {
                sxz[iv] -= (fipkp * (vxz + vzx));
                sxx[iv] -= (g * (vxx + vzz)) - (f * vzz);
                szz[iv] -= (g * (vxx + vzz)) - (f * vxx);
            } else {
                float sumrxz = 0, sumrxx = 0, sumrzz = 0;
                for (int l = 0; l < L; l++) {
                    i64 ir = l * NXNZ + iv;
                    sumrxz += rxz[ir]; sumrxx += rxx[ir]; sumrzz += rzz[ir];
                }
                float lsxz = (fipkp * (vxz + vzx)) + (DT2 * sumrxz);
                float lsxx = ((g * (vxx + vzz)) - (f * vzz)) + (DT2 * sumrxx);
                float lszz = ((g * (vxx + vzz)) - (f * vxx)) + (DT2 * sumrzz);
                sumrxz = sumrxx = sumrzz = 0;
                for (int l = 0; l < L; l++) {
                    float el = s->eta[l];
                    float b = 1.0 / (1.0 - (el * 0.5));
                    float cc = 1.0 + (el * 0.5);
                    i64 ir = l * NXNZ + iv;
                    rxz[ir] = b * (rxz[ir] * cc - el * (dipkp * (vxz + vzx)));
                    rxx[ir] = b * (rxx[ir] * cc - el * ((e * (vxx + vzz)) - (d * vzz)));
                    rzz[ir] = b * (rzz[ir] * cc - el * ((e * (vxx + vzz)) - (d * vxx)));
                    sumrxz += rxz[ir]; sumrxx += rxx[ir]; sumrzz += rzz[ir];
                }
                sxz[iv] -= lsxz + (DT2 * sumrxz);
                sxx[iv] -= lsxx + (DT2 * sumrxx);
                szz[iv] -= lszz + (DT2 * sumrzz);
            }
            int m = bp1 ? inject_ind2d(s, gz, gx) : -1;
            if (m != -1) {
                sxx[iv] = s->bnd_cur[W_SXX][m];
                szz[iv] = s->bnd_cur[W_SZZ][m];
                sxz[iv] = s->bnd_cur[W_SXZ][m];
            }
            if (c->abs_type == 1) cpml_s2d(s, gz, gx, &vxxr, &vxzr, &vzxr, &vzzr);
            float lsxz, lsxx, lszz;
            if (L == 0) {
                lsxz = (fipkp * (vxzr + vzxr));
                lsxx = ((g * (vxxr + vzzr)) - (f * vzzr));
                lszz = ((g * (vxxr + vzzr)) - (f * vxxr));
                sxzr[iv] += lsxz;
                sxxr[iv] += lsxx;
                szzr[iv] += lszz;
            } else {
                float sumrxz = 0, sumrxx = 0, sumrzz = 0;
                i64 ir = 0;
                for (int l = 0; l < L; l++) {
                    ir = l * NXNZ + iv;
                    sumrxz += rxzr[ir]; sumrxx += rxxr[ir]; sumrzz += rzzr[ir];
                }
                lsxz = (fipkp * (vxzr + vzxr)) + (DT2 * sumrxz);
                lsxx = ((g * (vxxr + vzzr)) - (f * vzzr)) + (DT2 * sumrxx);
                lszz = ((g * (vxxr + vzzr)) - (f * vxxr)) + (DT2 * sumrzz);
                sumrxz = sumrxx = sumrzz = 0;
                /* the reference reuses the last mechanism's index in this
                 * loop (update_adjs2D.cl:379-391) */
                for (int l = 0; l < L; l++) {
                    float el = s->eta[l];
                    float b = 1.0 / (1.0 + (el * 0.5));
                    float cc = 1.0 - (el * 0.5);
                    rxzr[ir] = b * (rxzr[ir] * cc - el * (dipkp * (vxzr + vzxr)));
                    rxxr[ir] = b * (rxxr[ir] * cc - el * ((e * (vxxr + vzzr)) - (d * vzzr)));
                    rzzr[ir] = b * (rzzr[ir] * cc - el * ((e * (vxxr + vzzr)) - (d * vxxr)));
                    sumrxz += rxzr[ir]; sumrxx += rxxr[ir]; sumrzz += rzzr[ir];
                }
                sxzr[iv] += lsxz + (DT2 * sumrxz);
                sxxr[iv] += lsxx + (DT2 * sumrxx);
                szzr[iv] += lszz + (DT2 * sumrzz);
            }
            if (c->abs_type == 2) {
                float *fl[3] = {sxzr, sxxr, szzr};
                taper2d(s, gz, gx, fl, 3, iv);
            }
            if (!bp1) {
            } else if (c->restype == 0) {
                float c1 = 1.0 / ((2.0 * lM - 2.0 * lmu) * (2.0 * lM - 2.0 * lmu));
                float c3 = 1.0 / (lmu * lmu);
                float c5 = 0.25 * c3;
                float dM = c1 * (sxx[iv] + szz[iv]) * (lsxx + lszz);
                gradM[ip] += -dM;
                gradmu[ip] += -c3 * (sxz[iv] * lsxz) + dM - c5 * ((sxx[iv] - szz[iv]) * (lsxx - lszz));
                if (c->hout) {
                    /* update_adjs2D.cl:453-457: the mu term subtracts the
                     * gradient's dM, not dMH */
                    float dMH = c1 * (sxx[iv] + szz[iv]) * (sxx[iv] + szz[iv]);
                    s->hess[G_M][ip] += dMH;
                    s->hess[G_MU][ip] += c3 * sxz[iv] * sxz[iv] - dM + c5 * (sxx[iv] - szz[iv]) * (sxx[iv] - szz[iv]);
                }
            } else {
                float dM = (sxx[iv] + szz[iv]) * (lsxx + lszz);
                gradM[ip] += -dM;
                if (c->hout) {
                    float dMH = (sxx[iv] + szz[iv]) * (sxx[iv] + szz[iv]);
                    s->hess[G_M][ip] += dMH;
                }
            }
        }
}

/* src/surface2D_adj.cl:35-148, run in ascending x as a sequential loop */
static void port_surface_adj2d(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NZ = s->NZp, NX = s->NXp, nz = c->nz;
    float *vxr = s->wr[W_VX], *vzr = s->wr[W_VZ], *sxxr = s->wr[W_SXX], *szzr = s->wr[W_SZZ];
    const float *M = s->p[P_M], *mu = s->p[P_MU], *rip = s->p[P_RIP], *rkp = s->p[P_RKP];
    float hc[6];
    for (int i = 0; i < 6; i++) hc[i] = (float)s->hc[i + 1];
    int gz = F;
#define INDV2(z, x) ((i64)(x) * NZ + (z))
#define INDP2(z, x) ((i64)((x) - F) * nz + ((z) - F))
    for (int gx = F; gx <= NX - F - 1; gx++) {
        float lszz = szzr[INDV2(gz, gx)];
        float lsxx = sxxr[INDV2(gz, gx)];
        float lmu = mu[INDP2(gz, gx)];
        float lM = M[INDP2(gz, gx)];
        {
            float t1 = lsxx, t2 = lszz;
            float a = (float)1.0 / ((float)4.0 * lM * lmu - (float)4.0 * lmu * lmu);
            lsxx = -a * (lM * t1 + (-lM + (float)2.0 * lmu) * t2);
            lszz = -a * (lM * t2 + (-lM + (float)2.0 * lmu) * t1);
        }
        lszz = 0.0;
        float hx = -((lM - lmu * (float)2.0) * (lM - lmu * (float)2.0) / lM);
        float hz = -(lM - lmu * (float)2.0);
        for (int m = 0; m < F; m++) {
            if ((gx - F + m) < (NX - 2 * F))
                vxr[INDV2(gz, gx + m)] += (hc[m] * hx * lsxx * rip[INDP2(gz, gx + m)]);
            if ((gx - (m + 1)) > (F - 1))
                vxr[INDV2(gz, gx - (m + 1))] += (-hc[m] * hx * lsxx * rip[INDP2(gz, gx - (m + 1))]);
            vzr[INDV2(gz + m, gx)] += (hc[m] * hz * lsxx * rkp[INDP2(gz + m, gx)]);
        }
        szzr[INDV2(gz, gx)] = -(lM * lszz + (lM - (float)2.0 * lmu) * lsxx);
        sxxr[INDV2(gz, gx)] = -(lM * lsxx + (lM - (float)2.0 * lmu) * lszz);
    }
#undef INDV2
#undef INDP2
}

/* ======================================================================
 * adjoint, 3D (src/update_adjv3D.cl, src/update_adjs3D.cl, surface3D_adj.cl)
 * ====================================================================== */
static void port_update_adjv3d(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    /* BACK_PROP_TYPE 2 compiles out the forward reconstruction, the
     * boundary injection and the gradient (#if BACK_PROP_TYPE==1 blocks) */
    const int bp1 = c->back_prop_type != 2;
    int F = c->fdoh, NZ = s->NZp, NY = s->NYp, NX = s->NXp;
    i64 nz = c->nz, ny = c->ny;
    const double *hc = s->hc;
    float *vx = s->w[W_VX], *vy = s->w[W_VY], *vz = s->w[W_VZ];
    const float *sxx = s->w[W_SXX], *syy = s->w[W_SYY], *szz = s->w[W_SZZ];
    const float *sxy = s->w[W_SXY], *syz = s->w[W_SYZ], *sxz = s->w[W_SXZ];
    float *vxr = s->wr[W_VX], *vyr = s->wr[W_VY], *vzr = s->wr[W_VZ];
    const float *sxxr = s->wr[W_SXX], *syyr = s->wr[W_SYY], *szzr = s->wr[W_SZZ];
    const float *sxyr = s->wr[W_SXY], *syzr = s->wr[W_SYZ], *sxzr = s->wr[W_SXZ];
    const float *rip = s->p[P_RIP], *rjp = s->p[P_RJP], *rkp = s->p[P_RKP];
    float *gradrho = s->grad[G_RHO];
    const i64 sx = (i64)NY * NZ, sy = NZ;
#pragma omp parallel for collapse(2) schedule(static)
    for (int gx = F; gx < NX - F; gx++)
        for (int gy = F; gy < NY - F; gy++)
            for (int gz = F; gz < NZ - F; gz++) {
                i64 ip = ((i64)(gx - F) * ny + (gy - F)) * nz + (gz - F), iv = IV3(gz, gy, gx);
                float szz_z = dfw(szz, iv, 1, hc, F);
                float sxx_x = dfw(sxx, iv, sx, hc, F);
                float sxz_x = dbw(sxz, iv, sx, hc, F);
                float sxz_z = dbw(sxz, iv, 1, hc, F);
                float syz_y = dbw(syz, iv, sy, hc, F);
                float syz_z = dbw(syz, iv, 1, hc, F);
                float syy_y = dfw(syy, iv, sy, hc, F);
                float sxy_x = dbw(sxy, iv, sx, hc, F);
                float sxy_y = dbw(sxy, iv, sy, hc, F);
                float szz_zr = dfw(szzr, iv, 1, hc, F);
                float sxx_xr = dfw(sxxr, iv, sx, hc, F);
                float sxz_xr = dbw(sxzr, iv, sx, hc, F);
                float sxz_zr = dbw(sxzr, iv, 1, hc, F);
                float syz_yr = dbw(syzr, iv, sy, hc, F);
                float syz_zr = dbw(syzr, iv, 1, hc, F);
                float syy_yr = dfw(syyr, iv, sy, hc, F);
                float sxy_xr = dbw(sxyr, iv, sx, hc, F);
                float sxy_yr = dbw(sxyr, iv, sy, hc, F);
                float lvx = ((sxx_x + sxy_y + sxz_z) * rip[ip]);
                float lvy = ((syy_y + sxy_x + syz_z) * rjp[ip]);
                float lvz = ((szz_z + sxz_x + syz_y) * rkp[ip]);
                if (bp1) {
                    vx[iv] -= lvx;
                    vy[iv] -= lvy;
                    vz[iv] -= lvz;
                }
                int m = bp1 ? inject_ind3d(s, gz, gy, gx) : -1;
                if (m != -1) {
                    vx[iv] = s->bnd_cur[W_VX][m];
                    vy[iv] = s->bnd_cur[W_VY][m];
                    vz[iv] = s->bnd_cur[W_VZ][m];
                }
                if (c->abs_type == 1)
                    cpml_v3d(s, gz, gy, gx, &sxx_xr, &syy_yr, &szz_zr, &sxy_yr, &sxy_xr, &syz_yr, &syz_zr,
                             &sxz_xr, &sxz_zr);
                lvx = ((sxx_xr + sxy_yr + sxz_zr) * rip[ip]);
                lvy = ((syy_yr + sxy_xr + syz_zr) * rjp[ip]);
                lvz = ((szz_zr + sxz_xr + syz_yr) * rkp[ip]);
                vxr[iv] += lvx;
                vyr[iv] += lvy;
                vzr[iv] += lvz;
                if (c->abs_type == 2) {
                    float *f[3] = {vxr, vyr, vzr};
                    taper3d(s, gz, gy, gx, f, 3, iv);
                }
                if (bp1) gradrho[ip] += -vx[iv] * lvx - vy[iv] * lvy - vz[iv] * lvz;
            }
}

static void port_update_adjs3d(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    /* BACK_PROP_TYPE 2 compiles out the forward reconstruction, the
     * boundary injection and the gradient (#if BACK_PROP_TYPE==1 blocks) */
    const int bp1 = c->back_prop_type != 2;
    int F = c->fdoh, NZ = s->NZp, NY = s->NYp, NX = s->NXp, L = c->L;
    i64 nz = c->nz, ny = c->ny;
    const double *hc = s->hc;
    const double DT = s->DT, DT2 = s->DT2;
    const float *vx = s->w[W_VX], *vy = s->w[W_VY], *vz = s->w[W_VZ];
    float *sxx = s->w[W_SXX], *syy = s->w[W_SYY], *szz = s->w[W_SZZ];
    float *sxy = s->w[W_SXY], *syz = s->w[W_SYZ], *sxz = s->w[W_SXZ];
    const float *vxr = s->wr[W_VX], *vyr = s->wr[W_VY], *vzr = s->wr[W_VZ];
    float *sxxr = s->wr[W_SXX], *syyr = s->wr[W_SYY], *szzr = s->wr[W_SZZ];
    float *sxyr = s->wr[W_SXY], *syzr = s->wr[W_SYZ], *sxzr = s->wr[W_SXZ];
    float *rxx = s->r[R_XX], *ryy = s->r[R_YY], *rzz = s->r[R_ZZ];
    float *rxy = s->r[R_XY], *ryz = s->r[R_YZ], *rxz = s->r[R_XZ];
    float *rxxr = s->rr[R_XX], *ryyr = s->rr[R_YY], *rzzr = s->rr[R_ZZ];
    float *rxyr = s->rr[R_XY], *ryzr = s->rr[R_YZ], *rxzr = s->rr[R_XZ];
    const float *M = s->p[P_M], *mu = s->p[P_MU];
    const float *muipjp = s->p[P_MUIPJP], *mujpkp = s->p[P_MUJPKP], *muipkp = s->p[P_MUIPKP];
    const float *taup = s->p[P_TAUP], *taus = s->p[P_TAUS];
    const float *tausipjp = s->p[P_TAUSIPJP], *tausjpkp = s->p[P_TAUSJPKP], *tausipkp = s->p[P_TAUSIPKP];
    float *gradM = s->grad[G_M], *gradmu = s->grad[G_MU];
    const i64 sx = (i64)NY * NZ, sy = NZ, NV = (i64)NX * NY * NZ;
#pragma omp parallel for collapse(2) schedule(static)
    for (int gx = F; gx < NX - F; gx++)
        for (int gy = F; gy < NY - F; gy++)
            for (int gz = F; gz < NZ - F; gz++) {
                i64 ip = ((i64)(gx - F) * ny + (gy - F)) * nz + (gz - F), iv = IV3(gz, gy, gx);
                float vzx = dfw(vz, iv, sx, hc, F), vzy = dfw(vz, iv, sy, hc, F), vzz = dbw(vz, iv, 1, hc, F);
                float vyx = dfw(vy, iv, sx, hc, F), vyy = dbw(vy, iv, sy, hc, F), vyz = dfw(vy, iv, 1, hc, F);
                float vxx = dbw(vx, iv, sx, hc, F), vxy = dfw(vx, iv, sy, hc, F), vxz = dfw(vx, iv, 1, hc, F);
                float vzxr = dfw(vzr, iv, sx, hc, F), vzyr = dfw(vzr, iv, sy, hc, F), vzzr = dbw(vzr, iv, 1, hc, F);
                float vyxr = dfw(vyr, iv, sx, hc, F), vyyr = dbw(vyr, iv, sy, hc, F), vyzr = dfw(vyr, iv, 1, hc, F);
                float vxxr = dbw(vxr, iv, sx, hc, F), vxyr = dfw(vxr, iv, sy, hc, F), vxzr = dfw(vxr, iv, 1, hc, F);
                float fipjp, fjpkp, fipkp, g, f, lM, lmu, dipjp = 0, djpkp = 0, dipkp = 0, d = 0, e = 0;
                if (L == 0) {
                    lM = M[ip]; lmu = mu[ip];
                    fipjp = muipjp[ip]; fjpkp = mujpkp[ip]; fipkp = muipkp[ip];
                    g = lM; f = 2.0 * lmu;
                } else {
                    lM = M[ip]; lmu = mu[ip];
                    float lmuipkp = muipkp[ip], lmuipjp = muipjp[ip], lmujpkp = mujpkp[ip];
                    float ltaup = taup[ip], ltaus = taus[ip];
                    float ltausipkp = tausipkp[ip], ltausipjp = tausipjp[ip], ltausjpkp = tausjpkp[ip];
                    fipjp = lmuipjp * (1.0 + (float)L * ltausipjp);
                    fjpkp = lmujpkp * (1.0 + (float)L * ltausjpkp);
                    fipkp = lmuipkp * (1.0 + (float)L * ltausipkp);
                    g = lM * (1.0 + (float)L * ltaup);
                    f = 2.0 * lmu * (1.0 + (float)L * ltaus);
                    dipjp = lmuipjp * ltausipjp / DT;
                    djpkp = lmujpkp * ltausjpkp / DT;
                    dipkp = lmuipkp * ltausipkp / DT;
                    d = 2.0 * lmu * ltaus / DT;
                    e = lM * ltaup / DT;
                }
                float vxyyx = vxy + vyx, vyzzy = vyz + vzy, vxzzx = vxz + vzx;
                float vxxyyzz = vxx + vyy + vzz, vyyzz = vyy + vzz, vxxzz = vxx + vzz, vxxyy = vxx + vyy;
                if (!bp1) {
                } else if (L == 0) {
                    sxy[iv] -= (fipjp * vxyyx);
                    syz[iv] -= (fjpkp * vyzzy);
                    sxz[iv] -= (fipkp * vxzzx);
                    sxx[iv] -= ((g * vxxyyzz) - (f * vyyzz));
                    syy[iv] -= ((g * vxxyyzz) - (f * vxxzz));
                    szz[iv] -= ((g * vxxyyzz) - (f * vxxyy));
                } else {
                    float a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
                    for (int l = 0; l < L; l++) {
                        i64 ir = l * NV + iv;
                        a1 += rxy[ir]; a2 += ryz[ir]; a3 += rxz[ir]; a4 += rxx[ir]; a5 += ryy[ir]; a6 += rzz[ir];
                    }
                    float lsxy = (fipjp * vxyyx) + (DT2 * a1);
                    float lsyz = (fjpkp * vyzzy) + (DT2 * a2);
                    float lsxz = (fipkp * vxzzx) + (DT2 * a3);
                    float lsxx = ((g * vxxyyzz) - (f * vyyzz)) + (DT2 * a4);
                    float lsyy = ((g * vxxyyzz) - (f * vxxzz)) + (DT2 * a5);
                    float lszz = ((g * vxxyyzz) - (f * vxxyy)) + (DT2 * a6);
                    a1 = a2 = a3 = a4 = a5 = a6 = 0;
                    /* 3D reconstruction keeps the forward-time coefficients
                     * (update_adjs3D.cl:357-359) */
                    for (int l = 0; l < L; l++) {
                        float el = s->eta[l];
                        float b = 1.0 / (1.0 + (el * 0.5));
                        float cc = 1.0 - (el * 0.5);
                        i64 ir = l * NV + iv;
                        rxy[ir] = b * (rxy[ir] * cc - el * (dipjp * vxyyx));
                        ryz[ir] = b * (ryz[ir] * cc - el * (djpkp * vyzzy));
                        rxz[ir] = b * (rxz[ir] * cc - el * (dipkp * vxzzx));
                        rxx[ir] = b * (rxx[ir] * cc - el * ((e * vxxyyzz) - (d * vyyzz)));
                        ryy[ir] = b * (ryy[ir] * cc - el * ((e * vxxyyzz) - (d * vxxzz)));
                        rzz[ir] = b * (rzz[ir] * cc - el * ((e * vxxyyzz) - (d * vxxyy)));
                        a1 += rxy[ir]; a2 += ryz[ir]; a3 += rxz[ir]; a4 += rxx[ir]; a5 += ryy[ir]; a6 += rzz[ir];
                    }
                    sxy[iv] -= lsxy + (DT2 * a1);
                    syz[iv] -= lsyz + (DT2 * a2);
                    sxz[iv] -= lsxz + (DT2 * a3);
                    sxx[iv] -= lsxx + (DT2 * a4);
                    syy[iv] -= lsyy + (DT2 * a5);
                    szz[iv] -= lszz + (DT2 * a6);
                }
                int m = bp1 ? inject_ind3d(s, gz, gy, gx) : -1;
                if (m != -1) {
                    sxx[iv] = s->bnd_cur[W_SXX][m];
                    syy[iv] = s->bnd_cur[W_SYY][m];
                    szz[iv] = s->bnd_cur[W_SZZ][m];
                    sxy[iv] = s->bnd_cur[W_SXY][m];
                    syz[iv] = s->bnd_cur[W_SYZ][m];
                    sxz[iv] = s->bnd_cur[W_SXZ][m];
                }
                if (c->abs_type == 1)
                    cpml_s3d(s, gz, gy, gx, &vxxr, &vxyr, &vxzr, &vyxr, &vyyr, &vyzr, &vzxr, &vzyr, &vzzr, 1);
                float vxyyxr = vxyr + vyxr, vyzzyr = vyzr + vzyr, vxzzxr = vxzr + vzxr;
                float vxxyyzzr = vxxr + vyyr + vzzr, vyyzzr = vyyr + vzzr, vxxzzr = vxxr + vzzr, vxxyyr = vxxr + vyyr;
                float lsxy, lsyz, lsxz, lsxx, lsyy, lszz;
                if (L == 0) {
                    lsxy = (fipjp * vxyyxr);
                    lsyz = (fjpkp * vyzzyr);
                    lsxz = (fipkp * vxzzxr);
                    lsxx = ((g * vxxyyzzr) - (f * vyyzzr));
                    lsyy = ((g * vxxyyzzr) - (f * vxxzzr));
                    lszz = ((g * vxxyyzzr) - (f * vxxyyr));
                    sxyr[iv] += lsxy; syzr[iv] += lsyz; sxzr[iv] += lsxz;
                    sxxr[iv] += lsxx; syyr[iv] += lsyy; szzr[iv] += lszz;
                } else {
                    float a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0;
                    for (int l = 0; l < L; l++) {
                        i64 ir = l * NV + iv;
                        a1 += rxyr[ir]; a2 += ryzr[ir]; a3 += rxzr[ir]; a4 += rxxr[ir]; a5 += ryyr[ir]; a6 += rzzr[ir];
                    }
                    lsxy = (fipjp * vxyyxr) + (DT2 * a1);
                    lsyz = (fjpkp * vyzzyr) + (DT2 * a2);
                    lsxz = (fipkp * vxzzxr) + (DT2 * a3);
                    lsxx = ((g * vxxyyzzr) - (f * vyyzzr)) + (DT2 * a4);
                    lsyy = ((g * vxxyyzzr) - (f * vxxzzr)) + (DT2 * a5);
                    lszz = ((g * vxxyyzzr) - (f * vxxyyr)) + (DT2 * a6);
                    a1 = a2 = a3 = a4 = a5 = a6 = 0;
                    /* the reference writes the result into the forward memory
                     * variables and keeps only the last value of each sum
                     * (update_adjs3D.cl:566-583) */
                    for (int l = 0; l < L; l++) {
                        float el = s->eta[l];
                        float b = 1.0 / (1.0 + (el * 0.5));
                        float cc = 1.0 - (el * 0.5);
                        i64 ir = l * NV + iv;
                        rxy[ir] = b * (rxyr[ir] * cc - el * (dipjp * vxyyxr));
                        ryz[ir] = b * (ryzr[ir] * cc - el * (djpkp * vyzzyr));
                        rxz[ir] = b * (rxzr[ir] * cc - el * (dipkp * vxzzxr));
                        rxx[ir] = b * (rxxr[ir] * cc - el * ((e * vxxyyzzr) - (d * vyyzzr)));
                        ryy[ir] = b * (ryyr[ir] * cc - el * ((e * vxxyyzzr) - (d * vxxzzr)));
                        rzz[ir] = b * (rzzr[ir] * cc - el * ((e * vxxyyzzr) - (d * vxxyyr)));
                        a1 = rxyr[ir]; a2 = ryzr[ir]; a3 = rxzr[ir]; a4 = rxxr[ir]; a5 = ryyr[ir]; a6 = rzzr[ir];
                    }
                    sxyr[iv] += lsxy + (DT2 * a1);
                    syzr[iv] += lsyz + (DT2 * a2);
                    sxzr[iv] += lsxz + (DT2 * a3);
                    sxxr[iv] += lsxx + (DT2 * a4);
                    syyr[iv] += lsyy + (DT2 * a5);
                    szzr[iv] += lszz + (DT2 * a6);
                }
                if (c->abs_type == 2) {
                    float *fl[6] = {sxyr, syzr, sxzr, sxxr, syyr, szzr};
                    taper3d(s, gz, gy, gx, fl, 6, iv);
                }
                if (!bp1) {
                } else if (c->restype == 0) {
                    float c1 = 1.0 / (3.0 * lM - 4.0 * lmu) / (3.0 * lM - 4.0 * lmu);
                    float c3 = 1.0 / lmu / lmu;
                    float c5 = 1.0 / 6.0 * c3;
                    float dM = c1 * (sxx[iv] + syy[iv] + szz[iv]) * (lsxx + lsyy + lszz);
                    gradM[ip] += -dM;
                    gradmu[ip] += -c3 * (sxz[iv] * lsxz + sxy[iv] * lsxy + syz[iv] * lsyz) + 4.0 / 3 * dM -
                                  c5 * (lsxx * (2.0 * sxx[iv] - syy[iv] - szz[iv]) +
                                        lsyy * (2.0 * syy[iv] - sxx[iv] - szz[iv]) +
                                        lszz * (2.0 * szz[iv] - sxx[iv] - syy[iv]));
                } else {
                    float dM = (sxx[iv] + syy[iv] + szz[iv]) * (lsxx + lsyy + lszz);
                    gradM[ip] += -dM;
                }
            }
}

/* src/surface3D_adj.cl:29-116, sequential in x then y.  Reads syyr from
 * sxxr as the reference does (:62). */
static void port_surface_adj3d(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NZ = s->NZp, NY = s->NYp, NX = s->NXp;
    i64 nz = c->nz, ny = c->ny;
    float *vxr = s->wr[W_VX], *vyr = s->wr[W_VY], *vzr = s->wr[W_VZ];
    float *sxxr = s->wr[W_SXX], *syyr = s->wr[W_SYY], *szzr = s->wr[W_SZZ];
    const float *M = s->p[P_M], *mu = s->p[P_MU], *rip = s->p[P_RIP], *rjp = s->p[P_RJP], *rkp = s->p[P_RKP];
    float hc[6];
    for (int i = 0; i < 6; i++) hc[i] = (float)s->hc[i + 1];
    int gz = F;
#define INDP3(z, y, x) (((i64)((x) - F) * ny + ((y) - F)) * nz + ((z) - F))
    for (int gx = F; gx <= NX - F - 1; gx++)
        for (int gy = F; gy <= NY - F - 1; gy++) {
            float lszz = -szzr[IV3(gz, gy, gx)];
            float lsxx = -sxxr[IV3(gz, gy, gx)];
            float lsyy = -sxxr[IV3(gz, gy, gx)];
            float lmu = mu[INDP3(gz, gy, gx)];
            float lM = M[INDP3(gz, gy, gx)];
            {
                float t1 = lsxx, t2 = lsyy, t3 = lszz;
                float a = (float)1.0 / ((float)6.0 * lM * lmu - (float)8.0 * lmu * lmu);
                lsxx = a * ((float)2.0 * (lM - lmu) * t1 + (-lM + (float)2.0 * lmu) * (t2 + t3));
                lsyy = a * ((float)2.0 * (lM - lmu) * t2 + (-lM + (float)2.0 * lmu) * (t1 + t3));
                lszz = a * ((float)2.0 * (lM - lmu) * t3 + (-lM + (float)2.0 * lmu) * (t1 + t2));
            }
            lszz = 0.0;
            float h = -((lM - lmu * (float)2.0) * (lM - lmu * (float)2.0) / lM);
            float hz = -(lM - lmu * (float)2.0);
            for (int m = 0; m < F; m++) {
                if ((gx - F + m) < (NX - 2 * F))
                    vxr[IV3(gz, gy, gx + m)] += (hc[m] * h * (lsxx + lsyy) * rip[INDP3(gz, gy, gx + m)]);
                if ((gx - (m + 1)) > (F - 1))
                    vxr[IV3(gz, gy, gx - (m + 1))] += (-hc[m] * h * (lsxx + lsyy) * rip[INDP3(gz, gy, gx - (m + 1))]);
                if ((gy - F + m) < (NY - 2 * F))
                    vyr[IV3(gz, gy + m, gx)] += (hc[m] * h * (lsxx + lsyy) * rjp[INDP3(gz, gy + m, gx)]);
                if ((gy - (m + 1)) > (F - 1))
                    vyr[IV3(gz, gy - (m + 1), gx)] += (-hc[m] * h * (lsxx + lsyy) * rjp[INDP3(gz, gy - (m + 1), gx)]);
                vzr[IV3(gz + m, gy, gx)] += (hc[m] * hz * (lsxx + lsyy) * rkp[INDP3(gz + m, gy, gx)]);
            }
            sxxr[IV3(gz, gy, gx)] = -(lM * lsxx + (lM - (float)2.0 * lmu) * (lsyy + lszz));
            syyr[IV3(gz, gy, gx)] = -(lM * lsyy + (lM - (float)2.0 * lmu) * (lsxx + lszz));
            szzr[IV3(gz, gy, gx)] = -(lM * lszz + (lM - (float)2.0 * lmu) * (lsxx + lsyy));
        }
#undef INDP3
}


/* ======================================================================
 * 2D acoustic (ND=22): src/update_v2D_acc.cl:80-324, update_s2D_acc.cl:79-402.
 * The pressure lives in the W_SXX slot, its memory variable in R_XX, and
 * psi_p_x / psi_p_z in the PS_SXX_X / PS_SZZ_Z slots.
 * ====================================================================== */
static void port_update_v_acc(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NZ = s->NZp, NX = s->NXp, nz = c->nz, NAB = c->nab;
    const double *hc = s->hc;
    float *vx = s->w[W_VX], *vz = s->w[W_VZ];
    const float *p = s->w[W_SXX], *rip = s->p[P_RIP], *rkp = s->p[P_RKP];
    float **ps = s->psi;
#pragma omp parallel for schedule(static)
    for (int gx = F; gx < NX - F; gx++)
        for (int gz = F; gz < NZ - F; gz++) {
            i64 ip = (i64)(gx - F) * nz + (gz - F), iv = (i64)gx * NZ + gz;
            float p_x = dfw(p, iv, NZ, hc, F);
            float p_z = dfw(p, iv, 1, hc, F);
            if (c->abs_type == 1) {
                if (gz > NZ - NAB - F - 1) {
                    int i = gx - F, k = gz - NZ + NAB + F + NAB, ind = 2 * NAB - 1 - k;
                    CPML(ps[PS_SZZ_Z], (i64)i * (2 * NAB) + k, s->cz[C_KH], s->cz[C_AH], s->cz[C_BH], ind, p_z);
                } else if (!c->freesurf && gz - F < NAB) {
                    int i = gx - F, k = gz - F;
                    CPML(ps[PS_SZZ_Z], (i64)i * (2 * NAB) + k, s->cz[C_KH], s->cz[C_AH], s->cz[C_BH], k, p_z);
                }
                if (gx - F < NAB) {
                    int i = gx - F, k = gz - F;
                    CPML(ps[PS_SXX_X], (i64)i * nz + k, s->cx[C_KH], s->cx[C_AH], s->cx[C_BH], i, p_x);
                }
                if (gx > NX - NAB - F - 1) {
                    int i = gx - NX + NAB + F + NAB, k = gz - F, ind = 2 * NAB - 1 - i;
                    CPML(ps[PS_SXX_X], (i64)i * nz + k, s->cx[C_KH], s->cx[C_AH], s->cx[C_BH], ind, p_x);
                }
            }
            vx[iv] += (p_x * rip[ip]);
            vz[iv] += (p_z * rkp[ip]);
            if (c->abs_type == 2) {
                /* the acoustic kernels taper the top even with a free surface */
                float *f[2] = {vx, vz};
                if (gz - F < NAB) for (int q = 0; q < 2; q++) f[q][iv] *= s->taper[gz - F];
                if (gz > NZ - NAB - F - 1) for (int q = 0; q < 2; q++) f[q][iv] *= s->taper[NZ - F - gz - 1];
                if (gx - F < NAB) for (int q = 0; q < 2; q++) f[q][iv] *= s->taper[gx - F];
                if (gx > NX - NAB - F - 1) for (int q = 0; q < 2; q++) f[q][iv] *= s->taper[NX - F - gx - 1];
            }
        }
}

static void port_update_s_acc(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NZ = s->NZp, NX = s->NXp, nz = c->nz, NAB = c->nab, L = c->L;
    const double *hc = s->hc;
    const double DT2 = s->DT2;
    const float *vx = s->w[W_VX], *vz = s->w[W_VZ];
    float *p = s->w[W_SXX], *rp = s->r[R_XX];
    const float *M = s->p[P_M], *taup = s->p[P_TAUP];
    float **ps = s->psi;
    const i64 NXNZ = (i64)NX * NZ;
#pragma omp parallel for schedule(static)
    for (int gx = F; gx < NX - F; gx++)
        for (int gz = F; gz < NZ - F; gz++) {
            i64 ip = (i64)(gx - F) * nz + (gz - F), iv = (i64)gx * NZ + gz;
            float vxx = dbw(vx, iv, NZ, hc, F);
            float vzz = dbw(vz, iv, 1, hc, F);
            if (c->abs_type == 1) {
                if (gz > NZ - NAB - F - 1) {
                    int i = gx - F, k = gz - NZ + NAB + F + NAB, ind = 2 * NAB - 1 - k;
                    CPML(ps[PS_VZ_Z], (i64)i * (2 * NAB) + k, s->cz[C_K], s->cz[C_A], s->cz[C_B], ind + 1, vzz);
                } else if (!c->freesurf && gz - F < NAB) {
                    int i = gx - F, k = gz - F;
                    CPML(ps[PS_VZ_Z], (i64)i * (2 * NAB) + k, s->cz[C_K], s->cz[C_A], s->cz[C_B], k, vzz);
                }
                if (gx - F < NAB) {
                    int i = gx - F, k = gz - F;
                    CPML(ps[PS_VX_X], (i64)i * nz + k, s->cx[C_K], s->cx[C_A], s->cx[C_B], i, vxx);
                }
                if (gx > NX - NAB - F - 1) {
                    int i = gx - NX + NAB + F + NAB, k = gz - F, ind = 2 * NAB - 1 - i;
                    CPML(ps[PS_VX_X], (i64)i * nz + k, s->cx[C_K], s->cx[C_A], s->cx[C_B], ind + 1, vxx);
                }
            }
            if (L == 0) {
                float g = M[ip];
                p[iv] += (g * (vxx + vzz));
            } else {
                float lM = M[ip], ltaup = taup[ip];
                float g = lM * (1.0 + (float)L * ltaup);
                /* no 1/DT here, unlike the elastic kernels (update_s2D_acc.cl:333) */
                float e = lM * ltaup;
                float sumrp = 0;
                for (int l = 0; l < L; l++) sumrp += rp[l * NXNZ + iv];
                float lp = (g * (vxx + vzz)) + (DT2 * sumrp);
                sumrp = 0;
                for (int l = 0; l < L; l++) {
                    float el = s->eta[l];
                    float b = 1.0 / (1.0 + (el * 0.5));
                    float cc = 1.0 - (el * 0.5);
                    i64 ir = l * NXNZ + iv;
                    rp[ir] = b * (rp[ir] * cc - el * e * (vxx + vzz));
                    sumrp += rp[ir];
                }
                p[iv] += lp + (DT2 * sumrp);
            }
            if (c->abs_type == 2) {
                if (gz - F < NAB) p[iv] *= s->taper[gz - F];
                if (gz > NZ - NAB - F - 1) p[iv] *= s->taper[NZ - F - gz - 1];
                if (gx - F < NAB) p[iv] *= s->taper[gx - F];
                if (gx > NX - NAB - F - 1) p[iv] *= s->taper[NX - F - gx - 1];
            }
        }
}

/* ======================================================================
 * 2D SH (ND=21): src/update_v2D_SH.cl:106-356, update_s2D_SH.cl:109-421.
 * Buoyancy and shear modulus are used at the cell, unaveraged, as the
 * reference does; at FDOH=1 the stress kernel's differences carry no
 * coefficient (update_s2D_SH.cl:204-205); stresses are not tapered (the
 * reference tests the lower-case macro abstype).  The reference binds the
 * stress kernel's CPML arrays under names no buffer has (psi_vyx, psi_vyz);
 * here they are psi_vy_x / psi_vy_z.
 * ====================================================================== */
static void port_update_v_sh(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NZ = s->NZp, NX = s->NXp, nz = c->nz, NAB = c->nab;
    const double *hc = s->hc;
    float *vy = s->w[W_VY];
    const float *sxy = s->w[W_SXY], *syz = s->w[W_SYZ], *rho = s->p[P_RHO];
    float **ps = s->psi;
#pragma omp parallel for schedule(static)
    for (int gx = F; gx < NX - F; gx++)
        for (int gz = F; gz < NZ - F; gz++) {
            i64 ip = (i64)(gx - F) * nz + (gz - F), iv = (i64)gx * NZ + gz;
            float sxy_x = dbw(sxy, iv, NZ, hc, F);
            float syz_z = dbw(syz, iv, 1, hc, F);
            if (c->abs_type == 1) {
                if (gz > NZ - NAB - F - 1) {
                    int i = gx - F, k = gz - NZ + NAB + F + NAB, ind = 2 * NAB - 1 - k;
                    CPML(ps[PS_SYZ_Z], (i64)i * (2 * NAB) + k, s->cz[C_K], s->cz[C_A], s->cz[C_B], ind + 1, syz_z);
                } else if (!c->freesurf && gz - F < NAB) {
                    int i = gx - F, k = gz - F;
                    CPML(ps[PS_SYZ_Z], (i64)i * (2 * NAB) + k, s->cz[C_K], s->cz[C_A], s->cz[C_B], k, syz_z);
                }
                if (gx - F < NAB) {
                    int i = gx - F, k = gz - F;
                    CPML(ps[PS_SXY_X], (i64)i * nz + k, s->cx[C_K], s->cx[C_A], s->cx[C_B], i, sxy_x);
                }
                if (gx > NX - NAB - F - 1) {
                    /* full-node coefficients at ind, not ind+1 (update_v2D_SH.cl:309-310) */
                    int i = gx - NX + NAB + F + NAB, k = gz - F, ind = 2 * NAB - 1 - i;
                    CPML(ps[PS_SXY_X], (i64)i * nz + k, s->cx[C_K], s->cx[C_A], s->cx[C_B], ind, sxy_x);
                }
            }
            vy[iv] += ((sxy_x + syz_z) * rho[ip]);
            if (c->abs_type == 2) {
                if (!c->freesurf && gz - F < NAB) vy[iv] *= s->taper[gz - F];
                if (gz > NZ - NAB - F - 1) vy[iv] *= s->taper[NZ - F - gz - 1];
                if (gx - F < NAB) vy[iv] *= s->taper[gx - F];
                if (gx > NX - NAB - F - 1) vy[iv] *= s->taper[NX - F - gx - 1];
            }
        }
}

static void port_update_s_sh(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    int F = c->fdoh, NZ = s->NZp, NX = s->NXp, nz = c->nz, NAB = c->nab;
    const double *hc = s->hc;
    const float *vy = s->w[W_VY];
    float *sxy = s->w[W_SXY], *syz = s->w[W_SYZ];
    const float *mu = s->p[P_MU];
    float **ps = s->psi;
    double one[7] = {0, 1, 0, 0, 0, 0, 0};
    const double *h = F == 1 ? one : hc;
#pragma omp parallel for schedule(static)
    for (int gx = F; gx < NX - F; gx++)
        for (int gz = F; gz < NZ - F; gz++) {
            i64 ip = (i64)(gx - F) * nz + (gz - F), iv = (i64)gx * NZ + gz;
            float vyx = dfw(vy, iv, NZ, h, F);
            float vyz = dfw(vy, iv, 1, h, F);
            if (c->abs_type == 1) {
                if (gz > NZ - NAB - F - 1) {
                    int i = gx - F, k = gz - NZ + NAB + F + NAB, ind = 2 * NAB - 1 - k;
                    CPML(ps[PS_VY_Z], (i64)i * (2 * NAB) + k, s->cz[C_KH], s->cz[C_AH], s->cz[C_BH], ind, vyz);
                } else if (!c->freesurf && gz - F < NAB) {
                    int i = gx - F, k = gz - F;
                    CPML(ps[PS_VY_Z], (i64)i * (2 * NAB) + k, s->cz[C_KH], s->cz[C_AH], s->cz[C_BH], k, vyz);
                }
                if (gx - F < NAB) {
                    int i = gx - F, k = gz - F;
                    CPML(ps[PS_VY_X], (i64)i * nz + k, s->cx[C_KH], s->cx[C_AH], s->cx[C_BH], i, vyx);
                }
                if (gx > NX - NAB - F - 1) {
                    int i = gx - NX + NAB + F + NAB, k = gz - F, ind = 2 * NAB - 1 - i;
                    CPML(ps[PS_VY_X], (i64)i * nz + k, s->cx[C_KH], s->cx[C_AH], s->cx[C_BH], ind, vyx);
                }
            }
            float f = mu[ip];
            sxy[iv] += (f * vyx);
            syz[iv] += (f * vyz);
        }
}

/* free surface for SH: image syz above the surface.  The reference's SH
 * kernel is named "surface" while the loader asks for "freesurface"
 * (src/surface2D_SH.cl:23, assign_modeling_case.c:989); this is its body. */
static void port_surface_sh(fdo_state *s, int pdir)
{
    (void)pdir;
    int F = s->c.fdoh, NZ = s->NZp, NX = s->NXp;
    float *syz = s->w[W_SYZ];
    for (int gx = F; gx <= NX - F - 1; gx++)
        for (int m = 1; m <= F; m++) syz[(i64)gx * NZ + F - m] = -syz[(i64)gx * NZ + F + m - 1];
}

static void port_update_v(fdo_state *s)
{
    if (s->c.nd == 3) port_update_v3d(s);
    else if (s->c.nd == 22) port_update_v_acc(s);
    else if (s->c.nd == 21) port_update_v_sh(s);
    else port_update_v2d(s);
}
static void port_update_s(fdo_state *s)
{
    if (s->c.nd == 3) port_update_s3d(s);
    else if (s->c.nd == 22) port_update_s_acc(s);
    else if (s->c.nd == 21) port_update_s_sh(s);
    else port_update_s2d(s);
}
static void port_surface(fdo_state *s, int pdir)
{
    if (s->c.nd == 3) port_surface3d(s, pdir);
    else if (s->c.nd == 21) port_surface_sh(s, pdir);
    else if (s->c.nd == 2) port_surface2d(s, pdir);
}
static void port_update_adjv(fdo_state *s) { if (s->c.nd == 3) port_update_adjv3d(s); else port_update_adjv2d(s); }
static void port_update_adjs(fdo_state *s) { if (s->c.nd == 3) port_update_adjs3d(s); else port_update_adjs2d(s); }
static void port_surface_adj(fdo_state *s) { if (s->c.nd == 3) port_surface_adj3d(s); else port_surface_adj2d(s); }

const fdo_kernels fdo_port_kernels = {
    port_update_v, port_update_s, port_surface, port_update_adjv,
    port_update_adjs, port_surface_adj, port_savebnd, "port",
};

/* exported for tests: boundary-shell index maps */
int fdo_inject_ind(const fdo_state *s, int k, int j, int i)
{
    return s->c.nd == 3 ? inject_ind3d(s, k, j, i) : inject_ind2d(s, k, i);
}
int fdo_savebnd_cell(const fdo_state *s, int gid, int *i, int *j, int *k)
{
    *j = 0;
    return s->c.nd == 3 ? savebnd_cell3d(s, gid, i, j, k) : savebnd_cell2d(s, gid, i, k);
}
