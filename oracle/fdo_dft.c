/*
 * fdo_dft.c -- oracle of the frequency-domain (DFT) gradient,
 * SeisCL's BACK_PROP_TYPE=2.
 *
 * TEST INFRASTRUCTURE ONLY (the checker of the CUDA path; see fdo.h).
 *
 * The forward and the adjoint run accumulate a discrete Fourier transform of
 * every wave field and memory variable at a few frequencies; the gradient is
 * then assembled cell by cell from products of the two transforms.
 *
 *   frequency set-up  src/assign_modeling_case.c:549-570 (DTNYQ, NTNYQ, df,
 *                     gradfreqsn), restated in fdo_setup.c
 *   accumulation      the generated "savefreqs" kernel,
 *                     src/automatic_kernels.c:1024-1150
 *   assembly          calc_grad, src/calc_grad.c:111-260 (coefficients) and
 *                     :376-960 (per-cell products), ND = 2 and 3
 *
 * Coverage: here the transforms cover every cell of each variable.  The
 * reference launches savefreqs/initsavefreqs with prod(N) work-items over
 * padded buffers of prod(N+FDORDER) (times L) elements
 * (src/automatic_kernels.c:1150-1160), so cells whose flat padded index is
 * >= prod(N) -- the last columns of the grid and every memory-variable slab
 * but the first -- are never accumulated and read back unset.  That launch
 * size is not reproduced.
 *
 * calc_grad keeps the reference's formulas, including three of its
 * peculiarities that change results: (1) in 3D the three "normal minus the
 * other two" memory-variable combinations are all frxx - fryy - frzz
 * (calc_grad.c:671-673); (2) in 3D the adjoint syz transform is corrected
 * with the forward ryz memory variable (:664); (3) for param_type 2 without
 * attenuation the rho coefficient of the M product is -M/rho, without the
 * squared-modulus denominator the other terms carry (:267).  tests/
 * test_oracle_pin.py checks this file against the reference's calc_grad
 * compiled in place.
 */

#include <math.h>
#include <stdint.h>
#include <string.h>

#include "fdo.h"   /* after the system headers: FDO_FP64 retypes float */

#define FDO_PI 3.141592653589793238462643383279502884197169

typedef int64_t i64;

/* cos(pi x) and sin(pi x) for the DFT phase 2 k n / NTNYQ: the argument is
 * reduced modulo 2 exactly before it is scaled by pi. */
static double cos_pi(double x) { return cos(FDO_PI * fmod(x, 2.0)); }
static double sin_pi(double x) { return sin(FDO_PI * fmod(x, 2.0)); }

/* Factors of sample `thist` (the generated kernel's fact[freq],
 * automatic_kernels.c:1106-1110): DTNYQ*DT*exp(-i pi 2 k n / NTNYQ), formed
 * in double and stored as float. */
void fdo_dft_factors(const fdo_state *s, int thist, float *re, float *im)
{
    for (int f = 0; f < s->c.nfreqs; f++) {
        double ph = 2.0 * s->gradfreqsn[f] * thist / s->ntnyq;
        re[f] = (float)(s->dtnyq * s->DT * cos_pi(ph));
        im[f] = (float)(-s->dtnyq * s->DT * sin_pi(ph));
    }
}

static void accumulate(float *dst, const float *v, i64 n, int nf, const float *re, const float *im)
{
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < n; i++) {
        float x = v[i];
        for (int f = 0; f < nf; f++) {
            float *d = dst + 2 * ((i64)f * n + i);
            d[0] += re[f] * x;
            d[1] += im[f] * x;
        }
    }
}

/* Add sample `thist` of the current wave fields and memory variables to the
 * transforms of `slot` (0 forward, 1 adjoint).  In the DFT adjoint the
 * adjoint fields live in the forward buffers (src/clprogram.c:869-880), so
 * both slots read s->w and s->r. */
void fdo_savefreqs(fdo_state *s, int slot, int thist)
{
    float re[FDO_MAXFREQ], im[FDO_MAXFREQ];
    fdo_dft_factors(s, thist, re, im);
    int nf = s->c.nfreqs;
    for (int q = 0; q < s->nwave; q++) {
        int w = s->wave_ids[q];
        accumulate(s->fw[slot][w], s->w[w], s->nvol, nf, re, im);
    }
    if (s->c.L > 0)
        for (int q = 0; q < s->nmem; q++) {
            int r = s->mem_ids[q];
            accumulate(s->fr[slot][r], s->r[r], s->nvol * s->c.L, nf, re, im);
        }
}

void fdo_zero_dft(fdo_state *s, int slot)
{
    i64 nf = s->c.nfreqs;
    for (int q = 0; q < s->nwave; q++) memset(s->fw[slot][s->wave_ids[q]], 0, sizeof(float) * 2 * nf * s->nvol);
    if (s->c.L > 0)
        for (int q = 0; q < s->nmem; q++)
            memset(s->fr[slot][s->mem_ids[q]], 0, sizeof(float) * 2 * nf * s->nvol * s->c.L);
}

/* ---------------------------------------------------------------------
 * gradient coefficients (calc_grad.c:111-260)
 *
 * For one cell: c[0..7] weight the products of the M and mu gradients,
 * c[8..15] those of taup and taus, c[16..23] the chain-rule terms of rho.
 * With attenuation the moduli are relaxed by A = 1 + L tau and
 * B = 1 + al tau (al = sum over mechanisms of (w0 tau_l)^2/(1+(w0 tau_l)^2));
 * without it, only the entries below are non-zero.
 * --------------------------------------------------------------------- */
typedef struct { double c[24]; } coefs;

static coefs cell_coefs(int par_type, int visc, float M, float mu, float taup, float taus, float rho, float ND,
                        float L, float al)
{
    coefs k;
    memset(&k, 0, sizeof k);
    double *c = k.c;
    /* scale of the modulus products and of the rho chain term per
     * parametrisation: 0 (vp, vs, rho), 1 (M, mu, rho), 2 (Ip, Is, rho) */
    double sM, smu, rM, rmu;
    if (par_type == 0) {
        sM = 2.0 * sqrtf(rho * M); smu = 2.0 * sqrtf(rho * mu);
        rM = M / rho; rmu = mu / rho;
    } else if (par_type == 1) {
        sM = smu = 1.0;
        rM = rmu = 0.0;
    } else {
        sM = 2.0 * sqrtf(M / rho); smu = 2.0 * sqrtf(mu / rho);
        rM = -M / rho; rmu = -mu / rho;
    }
    double nd3 = (ND + 1.0) / 3.0;
    if (!visc) {
        double den = ND * M - 2.0 * (ND - 1.0) * mu;
        den *= den;
        c[0] = sM / den;
        c[2] = smu / ((double)mu * mu);
        c[3] = smu * nd3 / den;
        c[4] = smu / (2.0 * ND * mu * mu);
        c[16] = par_type == 2 ? rM : rM / den;
        c[18] = rmu / ((double)mu * mu);
        c[19] = rmu * nd3 / den;
        c[20] = rmu / (2.0 * ND * mu * mu);
        return k;
    }
    double Ap = 1.0 + L * taup, As = 1.0 + L * taus;
    double Bp = 1.0 + al * taup, Bs = 1.0 + al * taus;
    double f1 = ND * M * Ap * Bs - 2.0 * (ND - 1.0) * mu * As * Bp;
    double f2 = ND * M * taup * Bs - 2.0 * (ND - 1.0) * mu * taus * Bp;
    f1 *= f1;
    f2 *= f2;
    double mu2 = (double)mu * mu, Lal = L - al;
    /* unit-scale terms, multiplied below by sM/smu (gradients) and rM/rmu (rho) */
    double u[8];
    u[0] = Ap * Bp * Bs * Bs / f1;
    u[1] = taup * Bp * Bs * Bs / f2;
    u[2] = Bs / (mu2 * As);
    u[3] = nd3 * As * Bs * Bp * Bp / f1;
    u[4] = Bs / (2.0 * ND * mu2 * As);
    u[5] = Bs / (mu2 * taus);
    u[6] = nd3 * taus * Bs * Bp * Bp / f2;
    u[7] = Bs / (2.0 * ND * mu2 * taus);
    for (int i = 0; i < 8; i++) {
        double sc = i < 2 ? sM : smu, rc = i < 2 ? rM : rmu;
        c[i] = sc * u[i];
        c[16 + i] = rc * u[i];
    }
    c[8] = M * Lal * Bs * Bs / f1;
    c[9] = M * Bs * Bs / f2;
    c[10] = Lal / (mu * As * As);
    c[11] = nd3 * mu * Lal * Bp * Bp / f1;
    c[12] = Lal / (2.0 * ND * mu * As * As);
    c[13] = 1.0 / (mu * (double)taus * taus);
    c[14] = nd3 * mu * Bp * Bp / f2;
    c[15] = 1.0 / (2.0 * ND * mu * (double)taus * taus);
    return k;
}

/* ---- complex helpers on interleaved (re, im) floats ---- */
typedef struct { float x, y; } cpx;

static inline cpx ld(const float *b, i64 i) { cpx r = {b[2 * i], b[2 * i + 1]}; return r; }
static inline cpx add(cpx a, cpx b) { cpx r = {a.x + b.x, a.y + b.y}; return r; }
static inline cpx sub(cpx a, cpx b) { cpx r = {a.x - b.x, a.y - b.y}; return r; }
/* time integral at angular frequency w: X / (i w) */
static inline cpx integ(cpx a, float w) { cpx r = {a.y / w, -a.x / w}; return r; }
/* Im(b conj(a))-type product of the stress/velocity terms */
static inline float itreal(cpx a, cpx b) { return a.y * b.x - a.x * b.y; }
/* memory-variable product with relaxation time ts */
static inline float rmprod(cpx a, cpx b, float ts, float w) { return ts * (a.x * b.x + a.y * b.y) + (a.x * b.y - a.y * b.x) / w; }
/* time derivative at angular frequency w: i w X */
static inline cpx deriv(cpx a, float w) { cpx r = {-a.y * w, a.x * w}; return r; }
/* squared modulus, formed in double and rounded once */
static inline float norm2(cpx a) { return (float)(pow(a.x, 2) + pow(a.y, 2)); }

/* Add this shot's DFT gradient to s->grad (float accumulators, as the
 * reference's host arrays).  The forward transforms are slot 0, the adjoint
 * ones slot 1; neither is modified. */
void fdo_calc_grad(fdo_state *s)
{
    const fdo_cfg *c = &s->c;
    const int L = c->L, nf = c->nfreqs, nd = c->nd;
    const float ND = (float)nd;
    const int F = c->fdoh;
    float df = 1.0 / s->ntnyq / c->dt / s->dtnyq;
    float w0 = 2.0 * FDO_PI * c->f0;
    float al = 0;
    float tausig[8];
    for (int l = 0; l < L; l++) {
        tausig[l] = 1.0 / (2.0 * FDO_PI * c->fl[l]);
        double q = pow(w0 / (2.0 * FDO_PI * c->fl[l]), 2);
        al += q / (1.0 + q);
    }
    const float NTN = (float)s->ntnyq;
    const int nx = c->nx, ny = nd == 3 ? c->ny : 1, nz = c->nz;
    const i64 nvol = s->nvol;
    float *const *P = s->p;
    /* pointers of the transforms; absent components stay NULL */
    const float *W0[W_N], *W1[W_N], *R0[R_N], *R1[R_N];
    for (int w = 0; w < W_N; w++) { W0[w] = s->fw[0][w]; W1[w] = s->fw[1][w]; }
    for (int r = 0; r < R_N; r++) { R0[r] = L ? s->fr[0][r] : 0; R1[r] = L ? s->fr[1][r] : 0; }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++)
            for (int k = 0; k < nz; k++) {
                i64 im = ((i64)i * ny + j) * nz + k;
                i64 iv = nd == 3 ? ((i64)(i + F) * s->NYp + (j + F)) * s->NZp + (k + F)
                                 : (i64)(i + F) * s->NZp + (k + F);
                float lmu = P[P_MU][im];
                coefs K = cell_coefs(c->param_type, L > 0, P[P_M][im], lmu, L ? P[P_TAUP][im] : 0.0f,
                                     L ? P[P_TAUS][im] : 0.0f, P[P_RHO][im], ND, (float)L, al);
                double *cc = K.c;
                if (lmu < 1) {
                    for (int n = 2; n < 8; n++) cc[n] = 0;
                    for (int n = 10; n < 16; n++) cc[n] = 0;
                    for (int n = 18; n < 24; n++) cc[n] = 0;
                }
                for (int f = 0; f < nf; f++) {
                    float w = 2.0 * FDO_PI * df * s->gradfreqsn[f];
                    i64 ic = (i64)f * nvol + iv;
                    double d[9] = {0}, hd[9] = {0};
                    if (nd == 3) {
                        cpx sf[6], sa[6];  /* xx yy zz xy yz xz */
                        static const int sid[6] = {W_SXX, W_SYY, W_SZZ, W_SXY, W_SYZ, W_SXZ};
                        for (int q = 0; q < 6; q++) { sf[q] = ld(W0[sid[q]], ic); sa[q] = ld(W1[sid[q]], ic); }
                        for (int l = 0; l < L; l++) {
                            i64 il = ((i64)f * L + l) * nvol + iv;
                            cpx rxx = ld(R0[R_XX], il), ryy = ld(R0[R_YY], il), rzz = ld(R0[R_ZZ], il);
                            cpx rxy = ld(R0[R_XY], il), ryz = ld(R0[R_YZ], il), rxz = ld(R0[R_XZ], il);
                            cpx axx = ld(R1[R_XX], il), ayy = ld(R1[R_YY], il), azz = ld(R1[R_ZZ], il);
                            cpx axy = ld(R1[R_XY], il), ayz = ld(R1[R_YZ], il), axz = ld(R1[R_XZ], il);
                            cpx fr[6] = {rxx, ryy, rzz, rxy, ryz, rxz};
                            cpx ar[6] = {axx, ayy, azz, axy, ryz, axz};  /* (2): forward ryz */
                            for (int q = 0; q < 6; q++) {
                                sf[q] = sub(sf[q], integ(fr[q], w));
                                sa[q] = sub(sa[q], integ(ar[q], w));
                            }
                            cpx tr = add(add(rxx, ryy), rzz), tra = add(add(axx, ayy), azz);
                            cpx dev = sub(sub(rxx, ryy), rzz);  /* (1): used for all three */
                            d[1] += rmprod(tra, tr, tausig[l], w) / NTN;
                            d[5] += (rmprod(axy, rxy, tausig[l], w) + rmprod(axz, rxz, tausig[l], w) +
                                     rmprod(ayz, ryz, tausig[l], w)) / NTN;
                            d[6] = d[1];
                            d[7] += (rmprod(axx, dev, tausig[l], w) + rmprod(ayy, dev, tausig[l], w) +
                                     rmprod(azz, dev, tausig[l], w)) / NTN;
                        }
                        cpx tr = add(add(sf[0], sf[1]), sf[2]), tra = add(add(sa[0], sa[1]), sa[2]);
                        cpx dxx = sub(sub(sf[0], sf[1]), sf[2]);
                        cpx dyy = sub(sub(sf[1], sf[0]), sf[2]);
                        cpx dzz = sub(sub(sf[2], sf[0]), sf[1]);
                        d[0] = w * itreal(tra, tr) / NTN;
                        d[2] = w * (itreal(sa[3], sf[3]) + itreal(sa[5], sf[5]) + itreal(sa[4], sf[4])) / NTN;
                        d[3] = d[0];
                        d[4] = w * (itreal(sa[0], dxx) + itreal(sa[1], dyy) + itreal(sa[2], dzz)) / NTN;
                        d[8] = w * (itreal(ld(W1[W_VX], ic), ld(W0[W_VX], ic)) + itreal(ld(W1[W_VY], ic), ld(W0[W_VY], ic)) +
                                    itreal(ld(W1[W_VZ], ic), ld(W0[W_VZ], ic))) / NTN;
                    } else {
                        cpx fxx = ld(W0[W_SXX], ic), fzz = ld(W0[W_SZZ], ic), fxz = ld(W0[W_SXZ], ic);
                        cpx axx = ld(W1[W_SXX], ic), azz = ld(W1[W_SZZ], ic), axz = ld(W1[W_SXZ], ic);
                        for (int l = 0; l < L; l++) {
                            i64 il = ((i64)f * L + l) * nvol + iv;
                            cpx rxx = ld(R0[R_XX], il), rzz = ld(R0[R_ZZ], il), rxz = ld(R0[R_XZ], il);
                            cpx qxx = ld(R1[R_XX], il), qzz = ld(R1[R_ZZ], il), qxz = ld(R1[R_XZ], il);
                            fxx = sub(fxx, integ(rxx, w)); fzz = sub(fzz, integ(rzz, w)); fxz = sub(fxz, integ(rxz, w));
                            axx = sub(axx, integ(qxx, w)); azz = sub(azz, integ(qzz, w)); axz = sub(axz, integ(qxz, w));
                            d[1] += rmprod(add(qxx, qzz), add(rxx, rzz), tausig[l], w) / NTN;
                            d[5] += (rmprod(qxz, rxz, tausig[l], w)) / NTN;
                            d[6] = d[1];
                            d[7] += (rmprod(qxx, sub(rxx, rzz), tausig[l], w) + rmprod(qzz, sub(rzz, rxx), tausig[l], w)) / NTN;
                        }
                        d[0] = w * itreal(add(axx, azz), add(fxx, fzz)) / NTN;
                        d[2] = w * (itreal(axz, fxz)) / NTN;
                        d[3] = d[0];
                        d[4] = w * (itreal(axx, sub(fxx, fzz)) + itreal(azz, sub(fzz, fxx))) / NTN;
                        d[8] = w * (itreal(ld(W1[W_VX], ic), ld(W0[W_VX], ic)) + itreal(ld(W1[W_VZ], ic), ld(W0[W_VZ], ic))) / NTN;
                        if (c->hout) {
                            /* approximate Hessian (calc_grad.c:838-905, ND = 2 only): squared
                             * moduli of the forward transforms, with the stresses as
                             * corrected above */
                            for (int l = 0; l < L; l++) {
                                i64 il = ((i64)f * L + l) * nvol + iv;
                                cpx rxx = ld(R0[R_XX], il), rzz = ld(R0[R_ZZ], il), rxz = ld(R0[R_XZ], il);
                                cpx sum = add(rxx, rzz), dxx = sub(rxx, rzz), dzz = sub(rzz, rxx);
                                float wt = w * tausig[l];
                                hd[1] += norm2(add(sum, deriv(sum, wt))) / NTN;
                                hd[5] += norm2(add(rxz, deriv(rxz, wt))) / NTN;
                                hd[6] = hd[1];
                                hd[7] += (norm2(add(dxx, deriv(dxx, wt))) + norm2(add(dzz, deriv(dzz, wt)))) / NTN;
                            }
                            hd[0] = norm2(deriv(add(fxx, fzz), w)) / NTN;
                            hd[2] = norm2(deriv(fxz, w)) / NTN;
                            hd[3] = hd[0];
                            hd[4] = (norm2(deriv(sub(fxx, fzz), w)) + norm2(deriv(sub(fzz, fxx), w))) / NTN;
                            hd[8] = (norm2(deriv(ld(W0[W_VX], ic), w)) + norm2(deriv(ld(W0[W_VZ], ic), w))) / NTN;
                        }
                    }
                    /* signs: products of the moduli enter with -, +, -, +, -, + */
                    double sM = -cc[0] * d[0] + cc[1] * d[1];
                    double smu = -cc[2] * d[2] + cc[3] * d[3] - cc[4] * d[4] + cc[5] * d[5] - cc[6] * d[6] + cc[7] * d[7];
                    double stp = -cc[8] * d[0] + cc[9] * d[1];
                    double sts = -cc[10] * d[2] + cc[11] * d[3] - cc[12] * d[4] + cc[13] * d[5] - cc[14] * d[6] +
                                 cc[15] * d[7];
                    double srho = -d[8] + cc[16] * d[0] - cc[17] * d[1] + cc[18] * d[2] - cc[19] * d[3] + cc[20] * d[4] -
                                  cc[21] * d[5] + cc[22] * d[6] - cc[23] * d[7];
                    /* float accumulators, one rounding per frequency as the reference */
                    s->grad[G_M][im] += sM;
                    s->grad[G_MU][im] += smu;
                    if (L > 0) {
                        s->grad[G_TAUP][im] += stp;
                        s->grad[G_TAUS][im] += sts;
                    }
                    s->grad[G_RHO][im] += srho;
                    if (c->hout && nd != 3) {
                        /* the Hessian enters with the gradient's signs reversed */
                        s->hess[G_M][im] += cc[0] * hd[0] - cc[1] * hd[1];
                        s->hess[G_MU][im] += cc[2] * hd[2] - cc[3] * hd[3] + cc[4] * hd[4] - cc[5] * hd[5] +
                                             cc[6] * hd[6] - cc[7] * hd[7];
                        if (L > 0) {
                            s->hess[G_TAUP][im] += cc[8] * hd[0] - cc[9] * hd[1];
                            s->hess[G_TAUS][im] += cc[10] * hd[2] - cc[11] * hd[3] + cc[12] * hd[4] -
                                                   cc[13] * hd[5] + cc[14] * hd[6] - cc[15] * hd[7];
                        }
                        s->hess[G_RHO][im] += hd[8] - cc[16] * hd[0] + cc[17] * hd[1] - cc[18] * hd[2] +
                                              cc[19] * hd[3] - cc[20] * hd[4] + cc[21] * hd[5] - cc[22] * hd[6] +
                                              cc[23] * hd[7];
                    }
                }
            }
}
