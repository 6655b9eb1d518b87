// sfd_kernels3d_tma.cu -- TMA-pipelined 3D velocity and stress updates
// (sm_100a, 8th-order stencils).
//
// A CTA owns a TZ x TY tile of the (z, y) plane and marches along x (the
// slowest axis).  Every operand arrives in shared memory through TMA tile
// copies (cp.async.bulk.tensor) completing on one mbarrier per stage, DPF
// planes ahead of the plane being updated:
//   ring   fields with an x derivative: haloed tiles (TZ+2F) x (TY+2F) of
//          planes x-F .. x+F, kept in a ring of 2F+1+DPF planes;
//   plane  fields with y/z derivatives only: the haloed tile of plane x;
//   centre per-cell streams (the updated fields, memory variables, material
//          parameters): the TZ x TY tile of plane x.
// One warp issues the copies; all warps compute from shared memory and store
// the updated cells straight to global memory (coalesced along z).  With a
// stage in flight per CTA of ~36 KB, the SM keeps the bytes in flight that
// HBM3e needs without relying on warp count.
//
// Same physics, CPML branch structure and operation order as the general
// kernels in sfd_kernels.cu (update_v3D.cl / update_s3D.cl).
//
// Eligibility (checked on the host, general kernels otherwise): 3D, F = 4,
// nz a multiple of 4 (so every TMA x coordinate and row pitch is a multiple
// of 16 bytes), L <= 3.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "sfd_cache.h"
#include "sfd_internal.h"
#include "sfd_kernels.h"

namespace sfd {
namespace {

typedef int64_t i64;

constexpr int TF = 4;                    // stencil half width
constexpr int TZ = 32, TY = 8;           // CTA tile (z fastest)
constexpr int HZ = TZ + 2 * TF;          // haloed tile row length
constexpr int HY = TY + 2 * TF;
constexpr int HALO = HZ * HY;            // floats per haloed tile
constexpr int CT = TZ * TY;              // floats per centre tile
// DPF (planes in flight through shared memory) is a template parameter of the
// kernels: the ring then holds 2F+1+DPF planes and the centre/plane slots
// DPF+1; the host picks the deepest pipeline that fits in shared memory.
constexpr int MAXDPF = 4;
constexpr int NTHR = TZ * TY;
constexpr int MAXC = 6 + 6 * 3 + 10;     // centre streams of the stress kernel at L = 3
constexpr unsigned long long WAIT_NS = 2000000000ull;  // bound on any wait: 2 s

struct TmaMaps {
    CUtensorMap ring[3];
    CUtensorMap plane[3];
    CUtensorMap ctr[MAXC];
};

__device__ int g_tma_status;             // 0 ok, 1 a stage never arrived

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long globaltimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// 3D tile copy global -> shared, completing on `bar` (no multicast)
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

// 3D tile prefetch global -> L2 (no shared memory, no completion tracking)
__device__ __forceinline__ void tma_prefetch_3d(const CUtensorMap *map, int c0, int c1, int c2)
{
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(c0), "r"(c1), "r"(c2)
                 : "memory");
}

// ---------------------------------------------------------- stencil helpers
// P points at the centre cell of a haloed tile
__device__ __forceinline__ float dzf(const float *P, const float *hc)
{
    float a = hc[0] * (P[1] - P[0]);
#pragma unroll
    for (int m = 2; m <= TF; m++) a = fmaf(hc[m - 1], P[m] - P[-(m - 1)], a);
    return a;
}
__device__ __forceinline__ float dzb(const float *P, const float *hc)
{
    float a = hc[0] * (P[0] - P[-1]);
#pragma unroll
    for (int m = 2; m <= TF; m++) a = fmaf(hc[m - 1], P[m - 1] - P[-m], a);
    return a;
}
__device__ __forceinline__ float dyf(const float *P, const float *hc)
{
    float a = hc[0] * (P[HZ] - P[0]);
#pragma unroll
    for (int m = 2; m <= TF; m++) a = fmaf(hc[m - 1], P[m * HZ] - P[-(m - 1) * HZ], a);
    return a;
}
__device__ __forceinline__ float dyb(const float *P, const float *hc)
{
    float a = hc[0] * (P[0] - P[-HZ]);
#pragma unroll
    for (int m = 2; m <= TF; m++) a = fmaf(hc[m - 1], P[(m - 1) * HZ] - P[-m * HZ], a);
    return a;
}
// q[0..2F] = values at x-F .. x+F
__device__ __forceinline__ float dxf(const float *q, const float *hc)
{
    float a = hc[0] * (q[TF + 1] - q[TF]);
#pragma unroll
    for (int m = 2; m <= TF; m++) a = fmaf(hc[m - 1], q[TF + m] - q[TF - (m - 1)], a);
    return a;
}
__device__ __forceinline__ float dxb(const float *q, const float *hc)
{
    float a = hc[0] * (q[TF] - q[TF - 1]);
#pragma unroll
    for (int m = 2; m <= TF; m++) a = fmaf(hc[m - 1], q[TF + (m - 1)] - q[TF - m], a);
    return a;
}

__device__ __forceinline__ void cpml(float *psi, i64 q, const float *K, const float *a, const float *b, int ci,
                                     float &d)
{
    float ps = __ldg(b + ci) * psi[q] + __ldg(a + ci) * d;
    psi[q] = ps;
    d = d / __ldg(K + ci) + ps;
}

// ------------------------------------------------------- per-cell updates
// The update of a cell is split by output between consumer warps ("roles"),
// so a CTA runs two (stress) or three (velocity) warps per tile row without
// more shared memory.  Every output and every CPML memory array belongs to
// exactly one role, and each role evaluates its outputs with the operation
// order of the general kernels.
//
// rs[m] is the offset in shared memory of the ring slot of plane x-F+m; c is
// the thread's centre in a haloed tile; C points at the thread's cell in the
// centre tiles of plane x.

// One thread's cell on plane x.  The z and y slab memberships do not change
// along the thread's march in x and are computed once; the x memberships are
// uniform over the CTA and recomputed per plane.
struct Cell {
    int x, gz, gy;        // padded coordinates
    i64 iv;               // padded linear index
    unsigned zy;          // bit 0: z low slab, 1: z high, 2: y low, 3: y high
    unsigned xs;          // bit 0: x low slab, 1: x high
};

// slab tests of the reference kernels (update_v3D.cl / update_s3D.cl)
__device__ __forceinline__ unsigned zy_slabs(const Grid &g, int gz, int gy)
{
    return (unsigned)(!g.freesurf && gz - TF < g.nab) | (unsigned)(gz > g.NZ - g.nab - TF - 1) << 1 |
           (unsigned)(gy - TF < g.nab) << 2 | (unsigned)(gy > g.NY - g.nab - TF - 1) << 3;
}
__device__ __forceinline__ unsigned x_slabs(const Grid &g, int x)
{
    return (unsigned)(x - TF < g.nab) | (unsigned)(x > g.NX - g.nab - TF - 1) << 1;
}

// psi = b psi + a d;  d = d / K + psi, with 1/K precomputed
__device__ __forceinline__ void cpml_k(float *psi, i64 q, const float *Ki, const float *a, const float *b, int ci,
                                       float &d)
{
    float ps = __ldg(b + ci) * psi[q] + __ldg(a + ci) * d;
    psi[q] = ps;
    d = d * __ldg(Ki + ci) + ps;
}

// CPML update of derivative d in the z (or y) slabs; H selects the half-node
// profile, X that the two slabs are tested as if / else if (velocity kernel)
// rather than as two ifs (stress kernel), as in the reference.
template <bool H, bool X>
__device__ __forceinline__ void cpml_z(const Grid &g, const Fields &f, int psi, const Cell &e, float &d)
{
    const int NAB = g.nab;
    const float *Ki = f.kinv[2][H], *A = f.cz[H ? CAH : CA], *B = f.cz[H ? CBH : CB];
    if (e.zy & 2u) {
        i64 i = e.x - TF, j = e.gy - TF, kk = e.gz - g.NZ + NAB + TF + NAB;
        int ind = 2 * NAB - 1 - (int)kk;
        cpml_k(f.psi[psi], (i * g.ny + j) * (2 * NAB) + kk, Ki, A, B, H ? ind : ind + 1, d);
        if (X) return;
    }
    if (e.zy & 1u) {
        i64 i = e.x - TF, j = e.gy - TF, kk = e.gz - TF;
        cpml_k(f.psi[psi], (i * g.ny + j) * (2 * NAB) + kk, Ki, A, B, (int)kk, d);
    }
}
template <bool H, bool X>
__device__ __forceinline__ void cpml_y(const Grid &g, const Fields &f, int psi, const Cell &e, float &d)
{
    const int NAB = g.nab;
    const float *Ki = f.kinv[1][H], *A = f.cy[H ? CAH : CA], *B = f.cy[H ? CBH : CB];
    if (e.zy & 4u) {
        i64 i = e.x - TF, j = e.gy - TF, kk = e.gz - TF;
        cpml_k(f.psi[psi], (i * (2 * NAB) + j) * g.nz + kk, Ki, A, B, (int)j, d);
        if (X) return;
    }
    if (e.zy & 8u) {
        i64 i = e.x - TF, j = e.gy - g.NY + NAB + TF + NAB, kk = e.gz - TF;
        int ind = 2 * NAB - 1 - (int)j;
        cpml_k(f.psi[psi], (i * (2 * NAB) + j) * g.nz + kk, Ki, A, B, H ? ind : ind + 1, d);
    }
}
template <bool H>
__device__ __forceinline__ void cpml_x(const Grid &g, const Fields &f, int psi, const Cell &e, float &d)
{
    const int NAB = g.nab;
    const float *Ki = f.kinv[0][H], *A = f.cx[H ? CAH : CA], *B = f.cx[H ? CBH : CB];
    if (e.xs & 1u) {
        i64 i = e.x - TF, j = e.gy - TF, kk = e.gz - TF;
        cpml_k(f.psi[psi], (i * g.ny + j) * g.nz + kk, Ki, A, B, (int)i, d);
    }
    if (e.xs & 2u) {
        i64 i = e.x - g.NX + NAB + TF + NAB, j = e.gy - TF, kk = e.gz - TF;
        int ind = 2 * NAB - 1 - (int)i;
        cpml_k(f.psi[psi], (i * g.ny + j) * g.nz + kk, Ki, A, B, H ? ind : ind + 1, d);
    }
}

// Cerjan factors in the reference's order (update_v3D.cl / update_s3D.cl:426-488)
template <int N>
__device__ __forceinline__ void taper(const Grid &g, const Fields &f, const Cell &e, float (&v)[N])
{
    const float *tp = f.taper;
    auto mul = [&](float t) {
#pragma unroll
        for (int i = 0; i < N; i++) v[i] *= t;
    };
    if (e.zy & 1u) mul(tp[e.gz - TF]);
    if (e.zy & 2u) mul(tp[g.NZ - TF - e.gz - 1]);
    if (e.zy & 4u) mul(tp[e.gy - TF]);
    if (e.zy & 8u) mul(tp[g.NY - TF - e.gy - 1]);
    if (e.xs & 1u) mul(tp[e.x - TF]);
    if (e.xs & 2u) mul(tp[g.NX - TF - e.x - 1]);
}

// the 2F+1 ring values at tile offset `off`; rs[m] = slot offset of plane x-F+m
__device__ __forceinline__ void column(const float *sm, const int *rs, int off, float *q)
{
#pragma unroll
    for (int m = 0; m <= 2 * TF; m++) q[m] = sm[rs[m] + off];
}

// velocity: ring sxx, sxy, sxz; plane (P) syy, szz, syz; centre vx, vy, vz, rip, rjp, rkp
template <int ROLE>
__device__ __forceinline__ void cell_v(const Grid &g, const Fields &f, const float *sm, const int *rs, const float *P,
                                       const float *C, int c, const Cell &e, const float *hc)
{
    const float *Rx = sm + rs[TF];  // plane x of the ring fields
    const bool cp = g.abs_type == 1 && (e.zy | e.xs);
    float q[2 * TF + 1];
    float v;
    if (ROLE == 0) {           // vx = vx + (sxx_x + sxy_y + sxz_z) * rip
        column(sm, rs, c, q);
        float sxx_x = dxf(q, hc), sxy_y = dyb(Rx + HALO + c, hc), sxz_z = dzb(Rx + 2 * HALO + c, hc);
        if (cp) {
            cpml_z<false, true>(g, f, PSXZ_Z, e, sxz_z);
            cpml_y<false, true>(g, f, PSXY_Y, e, sxy_y);
            cpml_x<true>(g, f, PSXX_X, e, sxx_x);
        }
        v = C[0 * CT] + (sxx_x + sxy_y + sxz_z) * C[3 * CT];
    } else if (ROLE == 1) {    // vy = vy + (syy_y + sxy_x + syz_z) * rjp
        column(sm, rs, HALO + c, q);
        float syy_y = dyf(P + c, hc), sxy_x = dxb(q, hc), syz_z = dzb(P + 2 * HALO + c, hc);
        if (cp) {
            cpml_z<false, true>(g, f, PSYZ_Z, e, syz_z);
            cpml_y<true, true>(g, f, PSYY_Y, e, syy_y);
            cpml_x<false>(g, f, PSXY_X, e, sxy_x);
        }
        v = C[1 * CT] + (syy_y + sxy_x + syz_z) * C[4 * CT];
    } else {                   // vz = vz + (szz_z + sxz_x + syz_y) * rkp
        column(sm, rs, 2 * HALO + c, q);
        float szz_z = dzf(P + HALO + c, hc), sxz_x = dxb(q, hc), syz_y = dyb(P + 2 * HALO + c, hc);
        if (cp) {
            cpml_z<true, true>(g, f, PSZZ_Z, e, szz_z);
            cpml_y<false, true>(g, f, PSYZ_Y, e, syz_y);
            cpml_x<false>(g, f, PSXZ_X, e, sxz_x);
        }
        v = C[2 * CT] + (szz_z + sxz_x + syz_y) * C[5 * CT];
    }
    if (g.abs_type == 2 && (e.zy | e.xs)) {
        float t[1] = {v};
        taper<1>(g, f, e, t);
        v = t[0];
    }
    f.w[VX + ROLE][e.iv] = v;
}

// One shear stress Q (0: sxy, 1: syz, 2: sxz) and its memory variables, with
// the two cross derivatives it needs; the general kernels' expressions.
template <int L, int Q>
__device__ __forceinline__ void shear(const Grid &g, const Fields &f, const float *sm, const int *rs, const float *C,
                                      int c, const Cell &e, const float *hc)
{
    constexpr int CP = 6 + 6 * L;
    const float *R = sm + rs[TF];
    float q[2 * TF + 1];
    float d1, d2;  // the two derivatives, in the order of the general kernels' sums
    if (Q == 0) {         // vxy + vyx
        column(sm, rs, HALO + c, q);
        d1 = dyf(R + c, hc);
        d2 = dxf(q, hc);
        if (g.abs_type == 1 && (e.zy | e.xs)) {
            cpml_y<true, false>(g, f, PVX_Y, e, d1);
            cpml_x<true>(g, f, PVY_X, e, d2);
        }
    } else if (Q == 1) {  // vyz + vzy
        d1 = dzf(R + HALO + c, hc);
        d2 = dyf(R + 2 * HALO + c, hc);
        if (g.abs_type == 1 && (e.zy | e.xs)) {
            cpml_z<true, false>(g, f, PVY_Z, e, d1);
            cpml_y<true, false>(g, f, PVZ_Y, e, d2);
        }
    } else {              // vxz + vzx
        column(sm, rs, 2 * HALO + c, q);
        d1 = dzf(R + c, hc);
        d2 = dxf(q, hc);
        if (g.abs_type == 1 && (e.zy | e.xs)) {
            cpml_z<true, false>(g, f, PVX_Z, e, d1);
            cpml_x<true>(g, f, PVZ_X, e, d2);
        }
    }
    const float v = d1 + d2;
    float s = C[Q * CT];
    // elastic parameters: muipjp, mujpkp, muipkp; viscoelastic: mu?p at CP+{3,4,2}, taus?p at CP+{8,9,7}
    if (L == 0) {
        s += C[(CP + Q) * CT] * v;
    } else {
        constexpr int PM = Q == 0 ? 3 : (Q == 1 ? 4 : 2);
        constexpr int PT = Q == 0 ? 8 : (Q == 1 ? 9 : 7);
        const float lmu = C[(CP + PM) * CT], ltaus = C[(CP + PT) * CT];
        const float fm = lmu * (1.0f + (float)L * ltaus);
        const float dm = lmu * ltaus * g.inv_dt;
        float r[L > 0 ? L : 1];
        float a = 0;
#pragma unroll
        for (int l = 0; l < L; l++) {
            r[l] = C[(6 + 6 * l + Q) * CT];
            a += r[l];
        }
        const float ls = fm * v + g.dt2 * a;
        a = 0;
        constexpr int RQ = Q == 0 ? RXY : (Q == 1 ? RYZ : RXZ);
#pragma unroll
        for (int l = 0; l < L; l++) {
            r[l] = g.eta_b[l] * (r[l] * g.eta_c[l] - g.eta[l] * (dm * v));
            a += r[l];
            f.r[RQ][l * g.nvol + e.iv] = r[l];
        }
        s += ls + g.dt2 * a;
    }
    if (g.abs_type == 2 && (e.zy | e.xs)) {
        float t[1] = {s};
        taper<1>(g, f, e, t);
        s = t[0];
    }
    f.w[Q == 0 ? SXY : (Q == 1 ? SYZ : SXZ)][e.iv] = s;
}

// stress: ring vx, vy, vz; centre sxy, syz, sxz, sxx, syy, szz, r[l][xy, yz, xz, xx, yy, zz], parameters
// role 0: normal stresses and their memory variables; role 1: sxy and sxz;
// role 2: syz (the shear stresses through shear<>).
template <int L, int ROLE>
__device__ __forceinline__ void cell_s(const Grid &g, const Fields &f, const float *sm, const int *rs, const float *C, int c,
                                       const Cell &e, const float *hc)
{
    constexpr int CP = 6 + 6 * L;  // first parameter stream
    const float *R = sm + rs[TF];       // plane x of vx, vy, vz
    const float *Vx = R + c, *Vy = R + HALO + c, *Vz = R + 2 * HALO + c;
    const bool cp = g.abs_type == 1 && (e.zy | e.xs);
    float q[2 * TF + 1];
    float s[3];
    if (ROLE == 0) {
        column(sm, rs, c, q);
        float vxx = dxb(q, hc), vyy = dyb(Vy, hc), vzz = dzb(Vz, hc);
        if (cp) {
            cpml_z<false, false>(g, f, PVZ_Z, e, vzz);
            cpml_y<false, false>(g, f, PVY_Y, e, vyy);
            cpml_x<false>(g, f, PVX_X, e, vxx);
        }
        float vxxyyzz = vxx + vyy + vzz, vyyzz = vyy + vzz, vxxzz = vxx + vzz, vxxyy = vxx + vyy;
        s[0] = C[3 * CT]; s[1] = C[4 * CT]; s[2] = C[5 * CT];
        if (L == 0) {
            // parameters: muipjp, mujpkp, muipkp, M, mu
            float gm = C[(CP + 3) * CT], fm = 2.0f * C[(CP + 4) * CT];
            s[0] += gm * vxxyyzz - fm * vyyzz;
            s[1] += gm * vxxyyzz - fm * vxxzz;
            s[2] += gm * vxxyyzz - fm * vxxyy;
        } else {
            // parameters: M, mu, muipkp, muipjp, mujpkp, taup, taus, tausipkp, tausipjp, tausjpkp
            float lM = C[(CP + 0) * CT], lmu = C[(CP + 1) * CT];
            float ltaup = C[(CP + 5) * CT], ltaus = C[(CP + 6) * CT];
            float gm = lM * (1.0f + (float)L * ltaup);
            float fm = 2.0f * lmu * (1.0f + (float)L * ltaus);
            float d = 2.0f * lmu * ltaus * g.inv_dt, ee = lM * ltaup * g.inv_dt;
            float r[3][L > 0 ? L : 1];
#pragma unroll
            for (int l = 0; l < L; l++)
#pragma unroll
                for (int k = 0; k < 3; k++) r[k][l] = C[(6 + 6 * l + 3 + k) * CT];
            float a[3] = {0, 0, 0};
#pragma unroll
            for (int l = 0; l < L; l++)
#pragma unroll
                for (int k = 0; k < 3; k++) a[k] += r[k][l];
            float lsxx = (gm * vxxyyzz - fm * vyyzz) + g.dt2 * a[0];
            float lsyy = (gm * vxxyyzz - fm * vxxzz) + g.dt2 * a[1];
            float lszz = (gm * vxxyyzz - fm * vxxyy) + g.dt2 * a[2];
#pragma unroll
            for (int k = 0; k < 3; k++) a[k] = 0;
#pragma unroll
            for (int l = 0; l < L; l++) {
                float el = g.eta[l];
                float b = g.eta_b[l], cc = g.eta_c[l];
                r[0][l] = b * (r[0][l] * cc - el * (ee * vxxyyzz - d * vyyzz));
                r[1][l] = b * (r[1][l] * cc - el * (ee * vxxyyzz - d * vxxzz));
                r[2][l] = b * (r[2][l] * cc - el * (ee * vxxyyzz - d * vxxyy));
#pragma unroll
                for (int k = 0; k < 3; k++) a[k] += r[k][l];
                const i64 ir = l * g.nvol + e.iv;
                f.r[RXX][ir] = r[0][l]; f.r[RYY][ir] = r[1][l]; f.r[RZZ][ir] = r[2][l];
            }
            s[0] += lsxx + g.dt2 * a[0];
            s[1] += lsyy + g.dt2 * a[1];
            s[2] += lszz + g.dt2 * a[2];
        }
        if (g.abs_type == 2 && (e.zy | e.xs)) taper<3>(g, f, e, s);
        f.w[SXX][e.iv] = s[0]; f.w[SYY][e.iv] = s[1]; f.w[SZZ][e.iv] = s[2];
    } else if (ROLE == 1) {
        shear<L, 0>(g, f, sm, rs, C, c, e, hc);   // sxy
        shear<L, 2>(g, f, sm, rs, C, c, e, hc);   // sxz
    } else {
        shear<L, 1>(g, f, sm, rs, C, c, e, hc);   // syz
    }
}

// -------------------------------------------------------------- pipeline
// Warp-uniform bounded wait: lane 0 polls (at most WAIT_NS) and broadcasts
// the outcome; every lane then observes the completed phase itself (which
// succeeds at once) so the TMA writes are visible to it.
__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity)
{
    int ok = 0;
    if ((threadIdx.x & 31) == 0) {
        const unsigned long long t0 = globaltimer();
        for (uint32_t it = 0;; ++it) {
            if (mbar_try_wait(bar, parity)) { ok = 1; break; }
            if ((it & 63u) == 63u && globaltimer() - t0 > WAIT_NS) break;
        }
        if (!ok) atomicExch(&g_tma_status, 1);
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (ok)
        for (int it = 0; it < (1 << 20) && !mbar_try_wait(bar, parity); ++it) {}
    return ok != 0;
}

// consumer warps: one per tile row and role
template <int KIND>
constexpr int nwc() { return TY * 3; }

// Plane loop of one consumer warp: wait for stage k, update this thread's
// cell of plane xs+k, release the stage.  Per-thread quantities (tile
// offsets, slab memberships, linear index) are set up once and advanced per
// plane.
template <int KIND, int L, int DPF, int ROLE>
__device__ __forceinline__ void consume(const Grid &g, const Fields &f, const float *sm, int xs, int nst, int z0,
                                        int y0, int tz, int ty, uint64_t *full, uint64_t *empty)
{
    constexpr int NVR = 2 * TF + 1 + DPF, NCR = DPF + 1;
    constexpr int NCF = KIND == 0 ? 6 : 6 + 6 * L + (L > 0 ? 10 : 5);
    constexpr int NPL = KIND == 0 ? 3 : 0;
    constexpr int PRING = NVR * 3 * HALO;              // offsets (floats) of the slot arrays in sm
    constexpr int CRING = PRING + NCR * NPL * HALO;
    const int lane = tz;
    const int gz = z0 + tz, gy = y0 + ty;
    const bool active = gz <= g.NZ - TF - 1 && gy <= g.NY - TF - 1;
    const int c = (ty + TF) * HZ + tz + TF;           // this thread's centre in a haloed tile
    const int cc = ty * TZ + tz;                      // and in a centre tile
    const float *hc = g.hc;
    const i64 plane = (i64)g.NY * g.NZ;
    Cell e;
    e.gz = gz;
    e.gy = gy;
    e.zy = zy_slabs(g, gz, gy);
    e.iv = ((i64)xs * g.NY + gy) * g.NZ + gz;
    int s0 = (xs - TF) % NVR;                         // ring slot of plane x - F
    for (int k = 0; k < nst; k++) {
        const int sl = k % NCR;
        if (!warp_wait(&full[sl], (k / NCR) & 1)) return;
        e.x = xs + k;
        e.xs = x_slabs(g, e.x);
        if (active) {
            int rs[2 * TF + 1];
#pragma unroll
            for (int m = 0; m <= 2 * TF; m++) rs[m] = (s0 + m < NVR ? s0 + m : s0 + m - NVR) * 3 * HALO;
            const float *C = sm + CRING + sl * NCF * CT + cc;
            if (KIND == 0) cell_v<ROLE>(g, f, sm, rs, sm + PRING + sl * NPL * HALO, C, c, e, hc);
            else cell_s<L, ROLE>(g, f, sm, rs, C, c, e, hc);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[sl]);
        e.iv += plane;
        s0 = s0 + 1 == NVR ? 0 : s0 + 1;
    }
}

// KIND 0: velocity update, KIND 1: stress update with L mechanisms.
// Warp NWC is the producer: it issues the TMA copies of stage j once every
// consumer warp has released stage j - NCR (the `empty` barrier), and the
// stage completes on its `full` barrier.  Consumer warps wait on `full`,
// update their row of the tile and arrive on `empty`.  No CTA-wide barrier
// is used after set-up, so warps drift freely within the DPF-stage window.
template <int KIND, int L, int DPF>
__global__ void __launch_bounds__(32 * (nwc<KIND>() + 1), 1) k_tma(const __grid_constant__ TmaMaps tm, const Grid g, const Fields f,
                                                      int xchunk, int l2ahead)
{
    constexpr int NWC = nwc<KIND>();
    constexpr int NVR = 2 * TF + 1 + DPF;    // ring slots
    constexpr int NCR = DPF + 1;             // centre/plane slots
    constexpr int NCF = KIND == 0 ? 6 : 6 + 6 * L + (L > 0 ? 10 : 5);
    constexpr int NPL = KIND == 0 ? 3 : 0;           // haloed plane-x-only fields
    constexpr int CP = KIND == 0 ? 3 : 6 + 6 * L;    // first stream of the unpadded parameter maps
    extern __shared__ __align__(128) float sm[];
    float *vring = sm;                               // [NVR][3][HALO]
    float *pring = vring + NVR * 3 * HALO;           // [NCR][NPL][HALO]
    float *cring = pring + NCR * NPL * HALO;         // [NCR][NCF][CT]
    uint64_t *full = reinterpret_cast<uint64_t *>(cring + NCR * NCF * CT);
    uint64_t *empty = full + NCR;
    uint64_t *pro = empty + NCR;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int z0 = TF + blockIdx.x * TZ, y0 = TF + blockIdx.y * TY;
    const int xs = TF + blockIdx.z * xchunk, xe = min(xs + xchunk, g.NX - TF);
    const int nst = xe - xs;
    // after a failed stage anywhere on the device, later CTAs skip their work
    if (nst <= 0 || *(volatile int *)&g_tma_status) return;
    if (tid == 0) {
        for (int i = 0; i < NCR; i++) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], NWC);
        }
        mbar_init(pro, 1);
        fence_mbar_init();
    }
    __syncthreads();
    constexpr uint32_t RING_B = 3 * HALO * 4;
    constexpr uint32_t STAGE_B = RING_B + NPL * HALO * 4 + NCF * CT * 4;
    if (warp == NWC) {
        // prologue: ring planes xs-F .. xs+F-1
        if (lane == 0) mbar_expect_tx(pro, 2 * TF * RING_B);
        __syncwarp();
        for (int i = lane; i < 2 * TF * 3; i += 32) {
            const int p = xs - TF + i / 3, q = i % 3;
            tma_load_3d(vring + ((p % NVR) * 3 + q) * HALO, &tm.ring[q], z0 - TF, y0 - TF, p, pro);
        }
        int j = 0;
        for (; j < nst; j++) {
            const int sl = j % NCR;
            if (j >= NCR && !warp_wait(&empty[sl], ((j / NCR) - 1) & 1)) break;
            if (lane == 0) mbar_expect_tx(&full[sl], STAGE_B);
            __syncwarp();
            const int x = xs + j;
            float *rdst = vring + ((x + TF) % NVR) * 3 * HALO;
            float *pdst = pring + sl * NPL * HALO;
            float *cdst = cring + sl * NCF * CT;
            for (int i = lane; i < 3 + NPL + NCF; i += 32) {
                if (i < 3) {
                    tma_load_3d(rdst + i * HALO, &tm.ring[i], z0 - TF, y0 - TF, x + TF, &full[sl]);
                } else if (i < 3 + NPL) {
                    tma_load_3d(pdst + (i - 3) * HALO, &tm.plane[i - 3], z0 - TF, y0 - TF, x, &full[sl]);
                } else {
                    const int cc = i - 3 - NPL;
                    if (cc < CP) tma_load_3d(cdst + cc * CT, &tm.ctr[cc], z0, y0, x, &full[sl]);
                    else tma_load_3d(cdst + cc * CT, &tm.ctr[cc], z0 - TF, y0 - TF, x - TF, &full[sl]);
                }
            }
            // warm L2 with the tiles of stage j + l2ahead, beyond the shared-memory window
            const int jp = j + l2ahead;
            if (l2ahead > 0 && jp < nst) {
                const int xp = xs + jp;
                for (int i = lane; i < 3 + NPL + NCF; i += 32) {
                    if (i < 3) tma_prefetch_3d(&tm.ring[i], z0 - TF, y0 - TF, xp + TF);
                    else if (i < 3 + NPL) tma_prefetch_3d(&tm.plane[i - 3], z0 - TF, y0 - TF, xp);
                    else if (i - 3 - NPL < CP) tma_prefetch_3d(&tm.ctr[i - 3 - NPL], z0, y0, xp);
                    else tma_prefetch_3d(&tm.ctr[i - 3 - NPL], z0 - TF, y0 - TF, xp - TF);
                }
            }
        }
        // the copies of the last stages land before this warp retires
        for (int jj = j - NCR > 0 ? j - NCR : 0; jj < j; jj++) warp_wait(&full[jj % NCR], (jj / NCR) & 1);
        return;
    }
    const int tz = lane, ty = warp % TY, role = warp / TY;
    if (!warp_wait(pro, 0)) return;
    // one specialised plane loop per role (the role is uniform over a warp)
    if (KIND == 0) {
        if (role == 0) consume<KIND, L, DPF, 0>(g, f, sm, xs, nst, z0, y0, tz, ty, full, empty);
        else if (role == 1) consume<KIND, L, DPF, 1>(g, f, sm, xs, nst, z0, y0, tz, ty, full, empty);
        else consume<KIND, L, DPF, 2>(g, f, sm, xs, nst, z0, y0, tz, ty, full, empty);
    } else {
        if (role == 0) consume<KIND, L, DPF, 0>(g, f, sm, xs, nst, z0, y0, tz, ty, full, empty);
        else if (role == 1) consume<KIND, L, DPF, 1>(g, f, sm, xs, nst, z0, y0, tz, ty, full, empty);
        else consume<KIND, L, DPF, 2>(g, f, sm, xs, nst, z0, y0, tz, ty, full, empty);
    }
}

// ------------------------------------------------------------------ host
PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// A 3D FP32 map over an array [d2][d1][d0] (d0 fastest) with box {b0, b1, 1}.
bool make_map(CUtensorMap *m, const float *base, uint64_t d0, uint64_t d1, uint64_t d2, uint32_t b0, uint32_t b1)
{
    auto enc = encode_fn();
    if (!enc || !base || (reinterpret_cast<uintptr_t>(base) & 15u) || (d0 * 4) % 16) return false;
    cuuint64_t dims[3] = {d0, d1, d2};
    cuuint64_t strides[2] = {d0 * 4, d0 * d1 * 4};
    cuuint32_t box[3] = {b0, b1, 1};
    cuuint32_t es[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(base), dims, strides, box, es,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// What the maps depend on: sizes and base pointers.
struct MapKey {
    int nz, ny, nx, NZ, NY, NX, L;
    int64_t nvol;
    const void *ptr[NW + NR + NPAR];
    bool operator==(const MapKey &o) const
    {
        if (nz != o.nz || ny != o.ny || nx != o.nx || NZ != o.NZ || NY != o.NY || NX != o.NX || L != o.L ||
            nvol != o.nvol)
            return false;
        for (int i = 0; i < NW + NR + NPAR; i++)
            if (ptr[i] != o.ptr[i]) return false;
        return true;
    }
};

MapKey key_of(const Grid &g, const Fields &f)
{
    MapKey k;
    k.nz = g.nz; k.ny = g.ny; k.nx = g.nx; k.NZ = g.NZ; k.NY = g.NY; k.NX = g.NX; k.L = g.L; k.nvol = g.nvol;
    for (int i = 0; i < NW; i++) k.ptr[i] = f.w[i];
    for (int i = 0; i < NR; i++) k.ptr[NW + i] = f.r[i];
    for (int i = 0; i < NPAR; i++) k.ptr[NW + NR + i] = f.p[i];
    return k;
}

struct CacheEntry {
    TmaMaps v, s;
    bool ok_v, ok_s;
};
// encoded maps, 16 most recent grid/field sets; launches copy their maps
// out under the cache's lock (plans run on several threads at once)
KeyedCache<MapKey, CacheEntry, 16> g_cache;

bool eligible(const Grid &g)
{
    return g.nd == 3 && g.F == TF && g.kernels == 3 && g.nz % 4 == 0 && g.NZ % 4 == 0 &&
           g.L >= 0 && g.L <= 3;
}

bool build_maps(const Grid &g, const Fields &f, CacheEntry &e)
{
    std::memset(&e.v, 0, sizeof(TmaMaps));
    std::memset(&e.s, 0, sizeof(TmaMaps));
    const uint64_t NZ = g.NZ, NY = g.NY, NX = g.NX, nz = g.nz, ny = g.ny, nx = g.nx;
    auto padded_halo = [&](CUtensorMap *m, const float *p) { return make_map(m, p, NZ, NY, NX, HZ, HY); };
    auto padded_ctr = [&](CUtensorMap *m, const float *p) { return make_map(m, p, NZ, NY, NX, TZ, TY); };
    auto param_ctr = [&](CUtensorMap *m, const float *p) { return make_map(m, p, nz, ny, nx, TZ, TY); };
    bool ok = true;
    // velocity kernel
    ok &= padded_halo(&e.v.ring[0], f.w[SXX]) && padded_halo(&e.v.ring[1], f.w[SXY]) &&
          padded_halo(&e.v.ring[2], f.w[SXZ]);
    ok &= padded_halo(&e.v.plane[0], f.w[SYY]) && padded_halo(&e.v.plane[1], f.w[SZZ]) &&
          padded_halo(&e.v.plane[2], f.w[SYZ]);
    ok &= padded_ctr(&e.v.ctr[0], f.w[VX]) && padded_ctr(&e.v.ctr[1], f.w[VY]) && padded_ctr(&e.v.ctr[2], f.w[VZ]);
    ok &= param_ctr(&e.v.ctr[3], f.p[PRIP]) && param_ctr(&e.v.ctr[4], f.p[PRJP]) &&
          param_ctr(&e.v.ctr[5], f.p[PRKP]);
    e.ok_v = ok;
    // stress kernel
    bool oks = padded_halo(&e.s.ring[0], f.w[VX]) && padded_halo(&e.s.ring[1], f.w[VY]) &&
               padded_halo(&e.s.ring[2], f.w[VZ]);
    const int sidx[6] = {SXY, SYZ, SXZ, SXX, SYY, SZZ};
    const int ridx[6] = {RXY, RYZ, RXZ, RXX, RYY, RZZ};
    for (int q = 0; q < 6; q++) oks &= padded_ctr(&e.s.ctr[q], f.w[sidx[q]]);
    for (int l = 0; l < g.L; l++)
        for (int q = 0; q < 6; q++) oks &= padded_ctr(&e.s.ctr[6 + 6 * l + q], f.r[ridx[q]] ? f.r[ridx[q]] + l * g.nvol : nullptr);
    const int cp = 6 + 6 * g.L;
    if (g.L == 0) {
        const int pidx[5] = {PMUIPJP, PMUJPKP, PMUIPKP, PM, PMU};
        for (int q = 0; q < 5; q++) oks &= param_ctr(&e.s.ctr[cp + q], f.p[pidx[q]]);
    } else {
        const int pidx[10] = {PM, PMU, PMUIPKP, PMUIPJP, PMUJPKP, PTAUP, PTAUS, PTAUSIPKP, PTAUSIPJP, PTAUSJPKP};
        for (int q = 0; q < 10; q++) oks &= param_ctr(&e.s.ctr[cp + q], f.p[pidx[q]]);
    }
    e.ok_s = oks;
    return ok || oks;
}

// Maps of this grid and field set, encoded once and reused; entries are keyed
// by every pointer and size, so a reused allocation address with other sizes
// gets its own entry.  `which` 0 copies the velocity kernel's maps into *out,
// 1 the stress kernel's; returns whether they were encoded.
bool maps_for(const Grid &g, const Fields &f, int which, TmaMaps *out)
{
    return g_cache.with(
        key_of(g, f),
        [&](CacheEntry &e) {
            std::memset(&e, 0, sizeof(e));
            build_maps(g, f, e);
        },
        [&](const CacheEntry &e) {
            if (out) *out = which == 0 ? e.v : e.s;
            return which == 0 ? e.ok_v : e.ok_s;
        });
}

int sm_count()
{
    int dev = 0, n = 148;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    return n;
}

// x planes per CTA: minimise (waves of CTAs) x (planes per CTA + pipeline fill)
int tma_xchunk(const Grid &g, int ctas_per_sm, int dpf)
{
    const long tiles = (long)((g.nz + TZ - 1) / TZ) * ((g.ny + TY - 1) / TY);
    const long slots = (long)sm_count() * ctas_per_sm;
    const int nxi = g.NX - 2 * TF;
    int best = nxi;
    double best_t = 1e300;
    for (int c = 1; c <= 32; c++) {
        const int xc = (nxi + c - 1) / c;
        const long waves = (tiles * c + slots - 1) / slots;
        const double t = (double)waves * (xc + 2 * TF + dpf);
        if (t < best_t) { best_t = t; best = xc; }
    }
    return best;
}

// dynamic shared memory: ring, plane and centre slots plus 2 NCR + 1 barriers
size_t smem_bytes(int kind, int L, int dpf)
{
    const int ncf = kind == 0 ? 6 : 6 + 6 * L + (L > 0 ? 10 : 5);
    const int npl = kind == 0 ? 3 : 0;
    const size_t nvr = 2 * TF + 1 + dpf, ncr = dpf + 1;
    return sizeof(float) * (nvr * 3 * HALO + ncr * npl * HALO + ncr * ncf * CT) + 8 * (2 * ncr + 1);
}

constexpr size_t SMEM_LIMIT = 227 * 1024;   // opt-in dynamic shared memory per CTA on sm_100

// deepest pipeline (2..MAXDPF) that fits, unless SFD_TMA_STAGES caps it
int pick_dpf(int kind, int L)
{
    static const int cap = [] {
        const char *e = getenv("SFD_TMA_STAGES");
        int v = e ? atoi(e) : MAXDPF;
        return v < 2 ? 2 : (v > MAXDPF ? MAXDPF : v);
    }();
    int d = cap;
    while (d > 2 && smem_bytes(kind, L, d) > SMEM_LIMIT) d--;
    return d;
}

// planes between the shared-memory stages and the L2 prefetch (0 disables)
int l2_ahead()
{
    static const int v = [] {
        const char *e = getenv("SFD_TMA_L2_AHEAD");
        int a = e ? atoi(e) : 0;
        return a < 0 ? 0 : (a > 32 ? 32 : a);
    }();
    return v;
}

// Raise the dynamic shared-memory limit of `kernel` once per device.
template <typename K>
bool set_smem(K kernel, size_t bytes, std::atomic<uint64_t> &done)
{
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = 1ull << (dev & 63);
    if (done.load() & bit) return true;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
        return false;
    done.fetch_or(bit);
    return true;
}

}  // namespace

template <int KIND, int L, int DPF>
static bool launch_tma_d(const Grid &g, const TmaMaps &m, const Fields &f, cudaStream_t st)
{
    const size_t sb = smem_bytes(KIND, L, DPF);
    if (sb > SMEM_LIMIT) return false;
    static std::atomic<uint64_t> done{0};
    if (!set_smem(k_tma<KIND, L, DPF>, sb, done)) return false;
    const int xc = tma_xchunk(g, 1, DPF);
    dim3 b(32 * (nwc<KIND>() + 1)), gr((g.nz + TZ - 1) / TZ, (g.ny + TY - 1) / TY, (g.NX - 2 * TF + xc - 1) / xc);
    k_tma<KIND, L, DPF><<<gr, b, sb, st>>>(m, g, f, xc, l2_ahead());
    return true;
}

template <int KIND, int L>
static bool launch_tma(const Grid &g, const TmaMaps &m, const Fields &f, cudaStream_t st)
{
    switch (pick_dpf(KIND, L)) {
    case 4: return launch_tma_d<KIND, L, 4>(g, m, f, st);
    case 3: return launch_tma_d<KIND, L, 3>(g, m, f, st);
    default: return launch_tma_d<KIND, L, 2>(g, m, f, st);
    }
}

bool launch_update_v_tma(const Grid &g, const Fields &f, cudaStream_t st)
{
    if (!eligible(g)) return false;
    TmaMaps m;
    if (!maps_for(g, f, 0, &m)) return false;
    return launch_tma<0, 0>(g, m, f, st);
}

bool launch_update_s_tma(const Grid &g, const Fields &f, cudaStream_t st)
{
    if (!eligible(g)) return false;
    TmaMaps m;
    if (!maps_for(g, f, 1, &m)) return false;
    switch (g.L) {
    case 0: return launch_tma<1, 0>(g, m, f, st);
    case 1: return launch_tma<1, 1>(g, m, f, st);
    case 2: return launch_tma<1, 2>(g, m, f, st);
    case 3: return launch_tma<1, 3>(g, m, f, st);
    default: return false;
    }
}

bool tma_ready(const Grid &g, const Fields &f)
{
    if (!eligible(g) || !encode_fn()) return false;
    return maps_for(g, f, 0, nullptr) && maps_for(g, f, 1, nullptr);
}

int tma_take_status()
{
    int v = 0, zero = 0;
    if (cudaMemcpyFromSymbol(&v, g_tma_status, sizeof(int)) != cudaSuccess) return -1;
    if (v) cudaMemcpyToSymbol(g_tma_status, &zero, sizeof(int));
    return v;
}

}  // namespace sfd
