// sfd_setup.cpp -- host-side model set-up of the FDTD engine, in FP64.
//
// Restates the single-device set-up of SeisCL:
//   Holberg / Taylor coefficients  src/third_party/SOFI3D/holbergcoeff.c:22-102
//   CPML profiles (Komatitsch & Martin 2007)  src/third_party/SOFI3D/CPML_COEFF.c:26-200
//   Cerjan taper, eta                        src/assign_modeling_case.c:536-584
//   parameter transforms and averages        src/assign_modeling_case.c:50-535
//   stability check                          src/assign_modeling_case.c:730-827
//   saved-boundary size                      src/Init_OpenCL.c:988-1021
//   source / receiver cells                  src/automatic_kernels.c:95-105, 501-511
// Coefficients and transforms are computed in double and rounded once to
// float; the reference computes them in float, so values agree to a few ulp.
// Cell indices use the reference's "%9.9f" dh literal so they agree exactly.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "sfd_setup.h"

namespace sfd {

static const double kPi = 3.141592653589793238462643383279502884197169;

// Holberg (1987) / Taylor staggered-grid coefficients: rows MAXRELERROR 0..4,
// columns FDORDER/2 = 1..6; entries c1..c6.  Published values; the reference
// keeps them as float (holbergcoeff.c:41), so they are widened from float
// here to give the same numbers.
static const float kHolberg[5][6][6] = {
    {{1.0f, 0, 0, 0, 0, 0},
     {9.0f / 8.0f, -1.0f / 24.0f, 0, 0, 0, 0},
     {75.0f / 64.0f, -25.0f / 384.0f, 3.0f / 640.0f, 0, 0, 0},
     {1225.0f / 1024.0f, -245.0f / 3072.0f, 49.0f / 5120.0f, -5.0f / 7168.0f, 0, 0},
     {19845.0f / 16384.0f, -735.0f / 8192.0f, 567.0f / 40960.0f, -405.0f / 229376.0f, 35.0f / 294912.0f, 0},
     {160083.0f / 131072.0f, -12705.0f / 131072.0f, 22869.0f / 1310720.0f, -5445.0f / 1835008.0f,
      847.0f / 2359296.0f, -63.0f / 2883584.0f}},
    {{1.0010f, 0, 0, 0, 0, 0},
     {1.1382f, -0.046414f, 0, 0, 0, 0},
     {1.1965f, -0.078804f, 0.0081781f, 0, 0, 0},
     {1.2257f, -0.099537f, 0.018063f, -0.0026274f, 0, 0},
     {1.2415f, -0.11231f, 0.026191f, -0.0064682f, 0.001191f, 0},
     {1.2508f, -0.12034f, 0.032131f, -0.010142f, 0.0029857f, -0.00066667f}},
    {{1.0050f, 0, 0, 0, 0, 0},
     {1.1534f, -0.052806f, 0, 0, 0, 0},
     {1.2111f, -0.088313f, 0.011768f, 0, 0, 0},
     {1.2367f, -0.10815f, 0.023113f, -0.0046905f, 0, 0},
     {1.2496f, -0.11921f, 0.031130f, -0.0093272f, 0.0025161f, 0},
     {1.2568f, -0.12573f, 0.036423f, -0.013132f, 0.0047484f, -0.0015979f}},
    {{1.0100f, 0, 0, 0, 0, 0},
     {1.1640f, -0.057991f, 0, 0, 0, 0},
     {1.2192f, -0.094070f, 0.014608f, 0, 0, 0},
     {1.2422f, -0.11269f, 0.026140f, -0.0064054f, 0, 0},
     {1.2534f, -0.12257f, 0.033755f, -0.011081f, 0.0036784f, 0},
     {1.2596f, -0.12825f, 0.038550f, -0.014763f, 0.0058619f, -0.0024538f}},
    {{1.0300f, 0, 0, 0, 0, 0},
     {1.1876f, -0.072518f, 0, 0, 0, 0},
     {1.2341f, -0.10569f, 0.022589f, 0, 0, 0},
     {1.2516f, -0.12085f, 0.032236f, -0.011459f, 0, 0},
     {1.2596f, -0.12829f, 0.038533f, -0.014681f, 0.0072580f, 0},
     {1.2640f, -0.13239f, 0.042217f, -0.017803f, 0.0081959f, -0.0051848f}},
};

bool holberg(int fdorder, int maxrelerror, double hc[6])
{
    if (fdorder < 2 || fdorder > 12 || fdorder % 2) return false;
    if (maxrelerror < 0 || maxrelerror > 4) return false;
    for (int i = 0; i < 6; i++) hc[i] = (double)kHolberg[maxrelerror][fdorder / 2 - 1][i];
    return true;
}

double literal9(double v)
{
    char buf[64];
    snprintf(buf, sizeof buf, "%9.9f", v);
    return strtod(buf, nullptr);
}

// Full- and half-node CPML profiles over 2*nab entries (the far half mirrors
// the near half).  K, a, b at full nodes; *_h at half nodes.
bool cpml_profiles(double npower, double kmax, double fpml, double vppml, double dh, double dt, int nab, float *K,
                   float *a, float *b, float *Kh, float *ah, float *bh)
{
    if (nab <= 0) return true;
    const double alpha_max = 2.0 * kPi * (fpml / 2.0);
    const double rcoef = 0.0008;
    const double d0 = -(npower + 1) * vppml * std::log(rcoef) / (2.0 * nab * dh);
    for (int i = 0; i < 2 * nab; i++) K[i] = a[i] = b[i] = Kh[i] = ah[i] = bh[i] = 0.0f;
    for (int i = 0; i <= nab; i++) {
        double pn = ((nab - i) * dh) / (nab * dh);
        double d = d0 * (0.25 * pn + 0.75 * std::pow(pn, npower));
        double Kv = 1.0 + (kmax - 1.0) * std::pow(pn, npower);
        double al = alpha_max * (1.0 - pn);
        if (al < 0) return false;
        double bv = std::exp(-(d / Kv + al) * dt);
        double av = std::fabs(d) > 1.0e-6 ? d * (bv - 1.0) / (Kv * (d + Kv * al)) : 0.0;
        if (i < 2 * nab) { K[i] = (float)Kv; b[i] = (float)bv; a[i] = (float)av; }
        if (i <= nab - 1) {
            double pnh = ((nab - i + 0.5 - 1.0) * dh) / (nab * dh);
            double dhh = d0 * (0.25 * pnh + 0.75 * std::pow(pnh, npower));
            double Khv = 1.0 + (kmax - 1.0) * std::pow(pnh, npower);
            double alh = alpha_max * (1.0 - pnh);
            if (alh < 0) return false;
            double bhv = std::exp(-(dhh / Khv + alh) * dt);
            double ahv = std::fabs(dhh) > 1.0e-6 ? dhh * (bhv - 1.0) / (Khv * (dhh + Khv * alh)) : 0.0;
            Kh[i] = (float)Khv; bh[i] = (float)bhv; ah[i] = (float)ahv;
            int l = 2 * nab - i - 1;
            if (i > 0) {
                K[l + 1] = K[i];
                b[l + 1] = b[i];
                if (std::fabs(d) > 1.0e-6) a[l + 1] = a[i];
            }
            Kh[l] = Kh[i];
            bh[l] = bh[i];
            if (std::fabs(d) > 1.0e-6) ah[l] = ah[i];
        }
    }
    return true;
}

void cerjan_taper(double abpc, int nab, float *taper)
{
    if (nab <= 0) return;
    double amp = 1.0 - abpc / 100.0;
    double aa = std::sqrt(-std::log(amp) / ((double)(nab - 1) * (nab - 1)));
    for (int i = 1; i <= nab; i++) taper[i - 1] = (float)std::exp(-(aa * aa * (double)(nab - i) * (nab - i)));
}

int nbnd_cells(int nd, int nz, int ny, int nx, int F, int nab, int freesurf)
{
    int lenz = freesurf ? nz - nab - F : nz - 2 * nab - 2 * F;
    if (nd == 3)
        return (nx - 2 * nab) * (ny - 2 * nab) * 2 * F + (nx - 2 * nab) * lenz * 2 * F + (ny - 2 * nab - 2 * F) * lenz * 2 * F;
    return (nx - 2 * nab) * 2 * F + lenz * 2 * F;
}

// [nx][ny][nz] indexing
static inline int64_t at(int NZ, int NY, int i, int j, int k) { return ((int64_t)i * NY + j) * NZ + k; }

// arithmetic mean along one axis, last slab copied (assign_modeling_case.c:50-99)
static void ave1(const std::vector<double> &in, std::vector<double> &out, int NZ, int NY, int NX, const int dir[3])
{
    for (int i = 0; i < NX; i++)
        for (int j = 0; j < NY; j++)
            for (int k = 0; k < NZ; k++) {
                int64_t a = at(NZ, NY, i, j, k);
                if (i < NX - dir[2] && j < NY - dir[1] && k < NZ - dir[0])
                    out[a] = 0.5 * (in[a] + in[at(NZ, NY, i + dir[2], j + dir[1], k + dir[0])]);
                else
                    out[a] = in[a];
            }
}

// two-direction mean (harmonic or arithmetic) with the reference's edge
// handling: the first direction's last slab is copied, the second
// direction's only where it meets the first (assign_modeling_case.c:100-301);
// the remaining edge cells keep zero.
static void ave2(const std::vector<double> &in, std::vector<double> &out, int NZ, int NY, int NX,
                 const int dir[2][3], bool harmonic)
{
    std::fill(out.begin(), out.end(), 0.0);
    int ex = dir[0][2] + dir[1][2], ey = dir[0][1] + dir[1][1], ez = dir[0][0] + dir[1][0];
    for (int i = 0; i < NX - ex; i++)
        for (int j = 0; j < NY - ey; j++)
            for (int k = 0; k < NZ - ez; k++) {
                int64_t a1 = at(NZ, NY, i, j, k);
                int64_t a2 = at(NZ, NY, i + dir[0][2], j + dir[0][1], k + dir[0][0]);
                int64_t a3 = at(NZ, NY, i + dir[1][2], j + dir[1][1], k + dir[1][0]);
                int64_t a4 = at(NZ, NY, i + ex, j + ey, k + ez);
                if (harmonic)
                    out[a1] = 4.0 / (1.0 / in[a1] + 1.0 / in[a2] + 1.0 / in[a3] + 1.0 / in[a4]);
                else
                    out[a1] = 0.25 * (in[a1] + in[a2] + in[a3] + in[a4]);
            }
    int X0 = 0, Y0 = 0, Z0 = 0;
    for (int d = 0; d < 2; d++) {
        if (dir[d][2] == 1) X0 = NX - 1;
        else if (dir[d][1] == 1) Y0 = NY - 1;
        if (dir[d][0] == 1) Z0 = NZ - 1;
        for (int i = X0; i < NX; i++)
            for (int j = Y0; j < NY; j++)
                for (int k = Z0; k < NZ; k++) out[at(NZ, NY, i, j, k)] = in[at(NZ, NY, i, j, k)];
    }
}

int transform_model(const sfd_config &c, int nz, int ny, int nx, const float *const *params,
                    std::vector<float> out[NPAR], std::string &err)
{
    const int64_t n = (int64_t)nz * ny * nx;
    const int L = c.L;
    const double dt = c.dt, dh = c.dh;
    std::vector<double> M(n), mu(n), rho(n), taup(n, 0.0), taus(n, 0.0);
    const float *pa = params[0], *pb = params[1], *prho = params[2];
    // SH reads only vs and rho, acoustic only vp and rho (assign_modeling_case.c:1004-1016)
    if (c.nd == 21) pa = nullptr;
    if (c.nd == 22) pb = nullptr;
    if ((c.nd != 21 && !pa) || (c.nd == 21 && !pb) || !prho) {
        err = c.nd == 21 ? "vs (or mu / Is) and rho are required" : "vp (or M / Ip) and rho are required";
        return SFD_ERR_ARG;
    }
    for (int64_t i = 0; i < n; i++) {
        double r = prho[i];
        if (!(r > 0)) { err = "rho must be positive everywhere"; return SFD_ERR_ARG; }
        double a = pa ? pa[i] : 0.0, b = pb ? pb[i] : 0.0;
        if (c.param_type == 0) { M[i] = a * a * r * dt / dh; mu[i] = b * b * r * dt / dh; }
        else if (c.param_type == 1) { M[i] = a * dt / dh; mu[i] = b * dt / dh; }
        else if (c.param_type == 2) { M[i] = (a / r) * (a / r) * r * dt / dh; mu[i] = (b / r) * (b / r) * r * dt / dh; }
        else { err = "param_type must be 0, 1 or 2"; return SFD_ERR_UNSUPPORTED; }
        rho[i] = r;
        if (L > 0) {
            if (!params[3] || !params[4]) { err = "taup and taus are required when L > 0"; return SFD_ERR_ARG; }
            taup[i] = params[3][i];
            taus[i] = params[4][i];
        }
    }
    if (L > 0) {
        // phase-velocity correction at f0 (assign_modeling_case.c:345-365, 414-437)
        double ws = 2.0 * kPi * c.f0, sumu = 0.0;
        std::vector<double> wl(L);
        for (int l = 0; l < L; l++) {
            double eta = 2.0 * kPi * c.fl[l] * dt;
            double pts = dt / eta;
            wl[l] = ws * ws * pts * pts / (1.0 + ws * ws * pts * pts);
            sumu += wl[l];
        }
        for (int64_t i = 0; i < n; i++) {
            double sumpi = 0.0;
            for (int l = 0; l < L; l++) sumpi += wl[l] * taup[i];
            M[i] /= (1.0 + sumpi);
            mu[i] /= (1.0 + sumu * taus[i]);
        }
    }
    std::vector<double> brho(n);
    for (int64_t i = 0; i < n; i++) brho[i] = dt / (dh * rho[i]);  // assign_modeling_case.c:460
    for (int k = 0; k < NPAR; k++) out[k].assign(n, 0.0f);
    auto store = [&](int id, const std::vector<double> &v) {
        for (int64_t i = 0; i < n; i++) out[id][i] = (float)v[i];
    };
    store(PM, M);
    store(PMU, mu);
    store(PRHO, brho);
    if (L > 0) { store(PTAUP, taup); store(PTAUS, taus); }
    std::vector<double> tmp(n);
    int dx[3] = {0, 0, 1}, dy[3] = {0, 1, 0}, dz[3] = {1, 0, 0};
    ave1(brho, tmp, nz, ny, nx, dx); store(PRIP, tmp);
    if (c.nd == 3) { ave1(brho, tmp, nz, ny, nx, dy); store(PRJP, tmp); }
    ave1(brho, tmp, nz, ny, nx, dz); store(PRKP, tmp);
    int dxz[2][3] = {{0, 0, 1}, {1, 0, 0}}, dxy[2][3] = {{0, 0, 1}, {0, 1, 0}}, dyz[2][3] = {{0, 1, 0}, {1, 0, 0}};
    ave2(mu, tmp, nz, ny, nx, dxz, true); store(PMUIPKP, tmp);
    if (c.nd == 3) {
        ave2(mu, tmp, nz, ny, nx, dxy, true); store(PMUIPJP, tmp);
        ave2(mu, tmp, nz, ny, nx, dyz, true); store(PMUJPKP, tmp);
    }
    if (L > 0) {
        ave2(taus, tmp, nz, ny, nx, dxz, false); store(PTAUSIPKP, tmp);
        if (c.nd == 3) {
            ave2(taus, tmp, nz, ny, nx, dxy, false); store(PTAUSIPJP, tmp);
            ave2(taus, tmp, nz, ny, nx, dyz, false); store(PTAUSJPKP, tmp);
        }
    }
    // stability: v = sqrt(M rho_b) dh / dt over the transformed model
    double vmax = 0.0, vsmax = 0.0;
    for (int64_t i = 0; i < n; i++) {
        vmax = std::max(vmax, std::sqrt(M[i] * brho[i]) / dt * dh);
        vsmax = std::max(vsmax, std::sqrt(mu[i] * brho[i]) / dt * dh);
    }
    if (vmax == 0.0) vmax = vsmax;
    double gamma;
    switch (c.fdorder) {
    case 2: gamma = 1.0; break;
    case 4: gamma = 1.184614; break;
    case 6: gamma = 1.283482; break;
    case 8: gamma = 1.345927; break;
    case 10: gamma = 1.38766; break;
    case 12: gamma = 1.417065; break;
    default: gamma = 1.0;
    }
    double dtstable = dh / (gamma * std::sqrt(c.nd == 3 ? 3.0 : 2.0) * vmax);
    // SEISCL_B200_UNCHECKED_CFL=1 skips the check: a test hook that lets a
    // test drive an unstable run into the instability detection
    const char *skip = std::getenv("SEISCL_B200_UNCHECKED_CFL");
    if ((double)(float)c.dt > dtstable && !(skip && skip[0] == '1')) {
        char buf[160];
        snprintf(buf, sizeof buf, "Time step too large, to be stable, set dt<%f", dtstable);
        err = buf;
        return SFD_ERR_CFL;
    }
    return SFD_OK;
}

// Which wave fields a source of `type` feeds, given the source types present
// anywhere in the acquisition (bit t for types 0..3, bit 4 for type 100).
// Follows the generated "sources" kernel: with a single fed variable the type
// is not checked; with several, a variable is fed when the type equals the
// variable's position in the model's variable list
// (automatic_kernels.c:565-567) and the normal stresses when the type is 100
// (:589-591), each receiving amp/ND.
int source_targets(int nd, int mask, int type, int fields[3], float div[3])
{
    static const int vl2[] = {VX, VZ, SXX, SZZ, SXZ};
    static const int vl3[] = {VX, VY, VZ, SXX, SZZ, SXZ, SXY, SYZ, SYY};
    static const int vl21[] = {VY, SXY, SYZ};
    static const int vl22[] = {VX, VZ, SXX};  // vx, vz, p (acoustic pressure in the SXX slot)
    // type 3 is a variable named p in the acoustic model, the average of the
    // normal stresses in P-SV and 3D; SH and acoustic have no averaged p
    const int by_type[4] = {VX, VY, VZ, nd == 22 ? SXX : -1};
    const int *vl = nd == 3 ? vl3 : (nd == 21 ? vl21 : (nd == 22 ? vl22 : vl2));
    int nvl = nd == 3 ? 9 : (nd == 21 || nd == 22 ? 3 : 5);
    bool has_avg = nd == 2 || nd == 3;
    bool fed[9] = {false};
    bool fed_p = has_avg && (mask & (1 << 4)) != 0;
    for (int t = 0; t < 4; t++) {
        if (!(mask & (1 << t))) continue;
        if (by_type[t] >= 0)
            for (int j = 0; j < nvl; j++)
                if (vl[j] == by_type[t]) fed[j] = true;
        if (t == 3 && has_avg) fed_p = true;
    }
    int ntypes = fed_p ? 1 : 0;
    for (int j = 0; j < nvl; j++) ntypes += fed[j];
    int n = 0;
    for (int j = 0; j < nvl && n < 3; j++)
        if (fed[j] && (ntypes == 1 || type == j)) { fields[n] = vl[j]; div[n] = 0.0f; n++; }
    if (fed_p && (ntypes == 1 || type == 100) && n == 0) {
        fields[n] = SXX; div[n] = (float)nd; n++;
        fields[n] = SZZ; div[n] = (float)nd; n++;
        if (nd == 3) { fields[n] = SYY; div[n] = (float)nd; n++; }
    }
    return n;
}

// cell of a source/receiver row: (int)(pos/DH) + F per axis, the DH literal
// of the reference (automatic_kernels.c:501-503)
void point_cell(const float *pos, double DH, int F, int &i, int &j, int &k)
{
    i = (int)((double)pos[0] / DH) + F;
    j = (int)((double)pos[1] / DH) + F;
    k = (int)((double)pos[2] / DH) + F;
}

}  // namespace sfd
