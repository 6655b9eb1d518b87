// sfd_dft.cu -- the frequency-domain (DFT) gradient of SeisCL's
// BACK_PROP_TYPE=2 on the device.
//
// * k_savefreqs adds one time sample of every wave field and memory variable
//   to its running DFT at up to MAXFREQ frequencies (the generated
//   "savefreqs" kernel, src/automatic_kernels.c:1024-1150).  All variables of
//   a step go in one launch (blockIdx.y = variable); the per-sample factors
//   DTNYQ*DT*exp(-i 2 pi k n / NTNYQ) are formed on the host in FP64 and
//   passed by value.  The reference covers only the first prod(N) elements
//   of each padded buffer; here every element is transformed.
// * k_calc_grad assembles the gradient cell by cell from the forward and
//   adjoint transforms (calc_grad, src/calc_grad.c:111-260 and 376-960, which
//   the reference runs on the host after copying the transforms back).  The
//   coefficient algebra is FP64 as in the reference; the per-frequency
//   products are FP32 as there; the sums accumulate in FP64 (the reference
//   rounds them to FP32 after every frequency and shot).
//
// Memory-bound: savefreqs reads 4 bytes and updates 8 per element and
// frequency; calc_grad reads each transform once.
#include <cuda_runtime.h>

#include "sfd_internal.h"
#include "sfd_kernels.h"

namespace sfd {

typedef int64_t i64;

__global__ void __launch_bounds__(256) k_savefreqs(DftSet d)
{
    const int q = blockIdx.y;
    const float *__restrict__ v = d.v[q];
    float2 *__restrict__ f = d.f[q];
    const i64 n = d.n[q];
    const int nf = d.nf;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        const float x = v[i];
        for (int k = 0; k < nf; k++) {
            float2 a = f[k * n + i];
            a.x += d.re[k] * x;
            a.y += d.im[k] * x;
            f[k * n + i] = a;
        }
    }
}

void launch_savefreqs(const DftSet &d, cudaStream_t st)
{
    if (d.nvar <= 0) return;
    i64 nmax = 0;
    for (int q = 0; q < d.nvar; q++) nmax = d.n[q] > nmax ? d.n[q] : nmax;
    i64 blocks = (nmax + 255) / 256;
    // a few waves of CTAs per SM; the loop strides over the rest
    if (blocks > 148 * 8) blocks = 148 * 8;
    dim3 gr((unsigned)blocks, (unsigned)d.nvar);
    k_savefreqs<<<gr, 256, 0, st>>>(d);
}

// ---------------------------------------------------------------- assembly
namespace {

// Per-cell coefficients of calc_grad.c:111-260 (param_type 0, 1, 2; with and
// without attenuation).  c[0..7] weight the M and mu products, c[8..15] the
// taup and taus ones, c[16..23] the chain-rule terms of rho.  The relaxation
// factors are A = 1 + L tau and B = 1 + al tau.  As in the reference, for
// param_type 2 without attenuation c[16] carries no squared-modulus
// denominator.
__device__ void cell_coefs(double *c, int par_type, bool visc, float M, float mu, float taup, float taus, float rho,
                           float ND, float L, float al)
{
    for (int i = 0; i < 24; i++) c[i] = 0.0;
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
    const double nd3 = (ND + 1.0) / 3.0;
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
        return;
    }
    const double Ap = 1.0 + L * taup, As = 1.0 + L * taus;
    const double Bp = 1.0 + al * taup, Bs = 1.0 + al * taus;
    double f1 = ND * M * Ap * Bs - 2.0 * (ND - 1.0) * mu * As * Bp;
    double f2 = ND * M * taup * Bs - 2.0 * (ND - 1.0) * mu * taus * Bp;
    f1 *= f1;
    f2 *= f2;
    const double mu2 = (double)mu * mu, Lal = L - al;
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
        c[i] = (i < 2 ? sM : smu) * u[i];
        c[16 + i] = (i < 2 ? rM : rmu) * u[i];
    }
    c[8] = M * Lal * Bs * Bs / f1;
    c[9] = M * Bs * Bs / f2;
    c[10] = Lal / (mu * As * As);
    c[11] = nd3 * mu * Lal * Bp * Bp / f1;
    c[12] = Lal / (2.0 * ND * mu * As * As);
    c[13] = 1.0 / (mu * (double)taus * taus);
    c[14] = nd3 * mu * Bp * Bp / f2;
    c[15] = 1.0 / (2.0 * ND * mu * (double)taus * taus);
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// time integral at angular frequency w: X / (i w)
__device__ __forceinline__ float2 cinteg(float2 a, float w) { return make_float2(a.y / w, -a.x / w); }
__device__ __forceinline__ float itreal(float2 a, float2 b) { return a.y * b.x - a.x * b.y; }
__device__ __forceinline__ float rmprod(float2 a, float2 b, float ts, float w)
{
    return ts * (a.x * b.x + a.y * b.y) + (a.x * b.y - a.y * b.x) / w;
}
// time derivative at angular frequency w: i w X
__device__ __forceinline__ float2 cderiv(float2 a, float w) { return make_float2(-a.y * w, a.x * w); }
// squared modulus, formed in FP64 and rounded once
__device__ __forceinline__ float cnorm2(float2 a) { return (float)((double)a.x * a.x + (double)a.y * a.y); }

}  // namespace

__global__ void __launch_bounds__(128) k_calc_grad(Grid g, Fields f, AdjFields a, GradDft d)
{
    const i64 npar = (i64)g.nz * g.ny * g.nx;
    const i64 im = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (im >= npar) return;
    const int k = (int)(im % g.nz), j = (int)((im / g.nz) % g.ny), i = (int)(im / ((i64)g.nz * g.ny));
    const int F = g.F, L = g.L;
    const i64 iv = g.nd == 3 ? ((i64)(i + F) * g.NY + (j + F)) * g.NZ + (k + F) : (i64)(i + F) * g.NZ + (k + F);
    const float lmu = f.p[PMU][im];
    double c[24];
    cell_coefs(c, d.par_type, L > 0, f.p[PM][im], lmu, L ? f.p[PTAUP][im] : 0.0f, L ? f.p[PTAUS][im] : 0.0f,
               f.p[PRHO][im], g.nd == 3 ? 3.0f : 2.0f, (float)L, d.al);
    if (lmu < 1.0f) {
        for (int n = 2; n < 8; n++) c[n] = 0;
        for (int n = 10; n < 16; n++) c[n] = 0;
        for (int n = 18; n < 24; n++) c[n] = 0;
    }
    const float N = d.ntnyq;
    double gM = 0, gmu = 0, gtp = 0, gts = 0, grho = 0;
    double hM = 0, hmu = 0, htp = 0, hts = 0, hrho = 0;
    for (int fq = 0; fq < d.nf; fq++) {
        const float w = d.w[fq];
        const i64 ic = (i64)fq * g.nvol + iv;
        float dd[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (g.nd == 3) {
            const int sid[6] = {SXX, SYY, SZZ, SXY, SYZ, SXZ};
            float2 sf[6], sa[6];
            for (int q = 0; q < 6; q++) { sf[q] = d.fw[0][sid[q]][ic]; sa[q] = d.fw[1][sid[q]][ic]; }
            for (int l = 0; l < L; l++) {
                const i64 il = ((i64)fq * L + l) * g.nvol + iv;
                const float2 rxx = d.fr[0][RXX][il], ryy = d.fr[0][RYY][il], rzz = d.fr[0][RZZ][il];
                const float2 rxy = d.fr[0][RXY][il], ryz = d.fr[0][RYZ][il], rxz = d.fr[0][RXZ][il];
                const float2 axx = d.fr[1][RXX][il], ayy = d.fr[1][RYY][il], azz = d.fr[1][RZZ][il];
                const float2 axy = d.fr[1][RXY][il], ayz = d.fr[1][RYZ][il], axz = d.fr[1][RXZ][il];
                const float2 fr[6] = {rxx, ryy, rzz, rxy, ryz, rxz};
                // the adjoint syz is corrected with the forward ryz (calc_grad.c:664)
                const float2 ar[6] = {axx, ayy, azz, axy, ryz, axz};
                for (int q = 0; q < 6; q++) {
                    sf[q] = csub(sf[q], cinteg(fr[q], w));
                    sa[q] = csub(sa[q], cinteg(ar[q], w));
                }
                const float2 tr = cadd(cadd(rxx, ryy), rzz), tra = cadd(cadd(axx, ayy), azz);
                // one deviatoric combination for all three terms (calc_grad.c:671-673)
                const float2 dev = csub(csub(rxx, ryy), rzz);
                const float ts = d.tausig[l];
                dd[1] += rmprod(tra, tr, ts, w) / N;
                dd[5] += (rmprod(axy, rxy, ts, w) + rmprod(axz, rxz, ts, w) + rmprod(ayz, ryz, ts, w)) / N;
                dd[6] = dd[1];
                dd[7] += (rmprod(axx, dev, ts, w) + rmprod(ayy, dev, ts, w) + rmprod(azz, dev, ts, w)) / N;
            }
            const float2 tr = cadd(cadd(sf[0], sf[1]), sf[2]), tra = cadd(cadd(sa[0], sa[1]), sa[2]);
            const float2 dxx = csub(csub(sf[0], sf[1]), sf[2]);
            const float2 dyy = csub(csub(sf[1], sf[0]), sf[2]);
            const float2 dzz = csub(csub(sf[2], sf[0]), sf[1]);
            dd[0] = w * itreal(tra, tr) / N;
            dd[2] = w * (itreal(sa[3], sf[3]) + itreal(sa[5], sf[5]) + itreal(sa[4], sf[4])) / N;
            dd[3] = dd[0];
            dd[4] = w * (itreal(sa[0], dxx) + itreal(sa[1], dyy) + itreal(sa[2], dzz)) / N;
            dd[8] = w * (itreal(d.fw[1][VX][ic], d.fw[0][VX][ic]) + itreal(d.fw[1][VY][ic], d.fw[0][VY][ic]) +
                         itreal(d.fw[1][VZ][ic], d.fw[0][VZ][ic])) / N;
        } else {
            float2 fxx = d.fw[0][SXX][ic], fzz = d.fw[0][SZZ][ic], fxz = d.fw[0][SXZ][ic];
            float2 axx = d.fw[1][SXX][ic], azz = d.fw[1][SZZ][ic], axz = d.fw[1][SXZ][ic];
            for (int l = 0; l < L; l++) {
                const i64 il = ((i64)fq * L + l) * g.nvol + iv;
                const float2 rxx = d.fr[0][RXX][il], rzz = d.fr[0][RZZ][il], rxz = d.fr[0][RXZ][il];
                const float2 qxx = d.fr[1][RXX][il], qzz = d.fr[1][RZZ][il], qxz = d.fr[1][RXZ][il];
                fxx = csub(fxx, cinteg(rxx, w)); fzz = csub(fzz, cinteg(rzz, w)); fxz = csub(fxz, cinteg(rxz, w));
                axx = csub(axx, cinteg(qxx, w)); azz = csub(azz, cinteg(qzz, w)); axz = csub(axz, cinteg(qxz, w));
                const float ts = d.tausig[l];
                dd[1] += rmprod(cadd(qxx, qzz), cadd(rxx, rzz), ts, w) / N;
                dd[5] += rmprod(qxz, rxz, ts, w) / N;
                dd[6] = dd[1];
                dd[7] += (rmprod(qxx, csub(rxx, rzz), ts, w) + rmprod(qzz, csub(rzz, rxx), ts, w)) / N;
            }
            dd[0] = w * itreal(cadd(axx, azz), cadd(fxx, fzz)) / N;
            dd[2] = w * itreal(axz, fxz) / N;
            dd[3] = dd[0];
            dd[4] = w * (itreal(axx, csub(fxx, fzz)) + itreal(azz, csub(fzz, fxx))) / N;
            dd[8] = w * (itreal(d.fw[1][VX][ic], d.fw[0][VX][ic]) + itreal(d.fw[1][VZ][ic], d.fw[0][VZ][ic])) / N;
            if (g.hout) {
                // approximate Hessian (calc_grad.c:838-905, 2D only): squared moduli of
                // the forward transforms, with the stresses as corrected above
                float hd[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                for (int l = 0; l < L; l++) {
                    const i64 il = ((i64)fq * L + l) * g.nvol + iv;
                    const float2 rxx = d.fr[0][RXX][il], rzz = d.fr[0][RZZ][il], rxz = d.fr[0][RXZ][il];
                    const float2 sum = cadd(rxx, rzz), dxx = csub(rxx, rzz), dzz = csub(rzz, rxx);
                    const float wt = w * d.tausig[l];
                    hd[1] += cnorm2(cadd(sum, cderiv(sum, wt))) / N;
                    hd[5] += cnorm2(cadd(rxz, cderiv(rxz, wt))) / N;
                    hd[6] = hd[1];
                    hd[7] += (cnorm2(cadd(dxx, cderiv(dxx, wt))) + cnorm2(cadd(dzz, cderiv(dzz, wt)))) / N;
                }
                hd[0] = cnorm2(cderiv(cadd(fxx, fzz), w)) / N;
                hd[2] = cnorm2(cderiv(fxz, w)) / N;
                hd[3] = hd[0];
                hd[4] = (cnorm2(cderiv(csub(fxx, fzz), w)) + cnorm2(cderiv(csub(fzz, fxx), w))) / N;
                hd[8] = (cnorm2(cderiv(d.fw[0][VX][ic], w)) + cnorm2(cderiv(d.fw[0][VZ][ic], w))) / N;
                double h[9];
                for (int q = 0; q < 9; q++) h[q] = hd[q];
                // the gradient's signs reversed
                hM += c[0] * h[0] - c[1] * h[1];
                hmu += c[2] * h[2] - c[3] * h[3] + c[4] * h[4] - c[5] * h[5] + c[6] * h[6] - c[7] * h[7];
                htp += c[8] * h[0] - c[9] * h[1];
                hts += c[10] * h[2] - c[11] * h[3] + c[12] * h[4] - c[13] * h[5] + c[14] * h[6] - c[15] * h[7];
                hrho += h[8] - c[16] * h[0] + c[17] * h[1] - c[18] * h[2] + c[19] * h[3] - c[20] * h[4] +
                        c[21] * h[5] - c[22] * h[6] + c[23] * h[7];
            }
        }
        double e[9];
        for (int q = 0; q < 9; q++) e[q] = dd[q];
        gM += -c[0] * e[0] + c[1] * e[1];
        gmu += -c[2] * e[2] + c[3] * e[3] - c[4] * e[4] + c[5] * e[5] - c[6] * e[6] + c[7] * e[7];
        gtp += -c[8] * e[0] + c[9] * e[1];
        gts += -c[10] * e[2] + c[11] * e[3] - c[12] * e[4] + c[13] * e[5] - c[14] * e[6] + c[15] * e[7];
        grho += -e[8] + c[16] * e[0] - c[17] * e[1] + c[18] * e[2] - c[19] * e[3] + c[20] * e[4] - c[21] * e[5] +
                c[22] * e[6] - c[23] * e[7];
    }
    a.grad[GM][im] += gM;
    a.grad[GMU][im] += gmu;
    a.grad[GRHO][im] += grho;
    if (L > 0) {
        a.grad[GTAUP][im] += gtp;
        a.grad[GTAUS][im] += gts;
    }
    if (g.hout && g.nd != 3) {
        a.hess[GM][im] += hM;
        a.hess[GMU][im] += hmu;
        a.hess[GRHO][im] += hrho;
        if (L > 0) {
            a.hess[GTAUP][im] += htp;
            a.hess[GTAUS][im] += hts;
        }
    }
}

void launch_calc_grad(const Grid &g, const Fields &f, const AdjFields &a, const GradDft &d, cudaStream_t st)
{
    const i64 npar = (i64)g.nz * g.ny * g.nx;
    k_calc_grad<<<(unsigned)((npar + 127) / 128), 128, 0, st>>>(g, f, a, d);
}

}  // namespace sfd
