// sfd_kernels3d_fast.cu -- register-blocked 3D stencil kernels (sm_100a).
//
// 2.5D blocking: a CTA owns a TZ x TY tile of the (z, y) plane and marches
// along x (the slowest axis) over a chunk of planes.  Each thread keeps, per
// field that needs an x derivative, a register queue of the 2F+1 values
// x-F .. x+F of its own (z, y) column, so every value of those fields is
// read from memory once per chunk instead of once per stencil tap.  The
// y and z taps come from a shared-memory copy of the current plane, whose
// interior is written from the queues and whose F-wide halo is read from L2.
// Per-cell streams (parameters, memory variables, the updated field itself)
// are read and written once, coalesced along z.
//
// Same physics, same CPML branch structure and same operation order as the
// general kernels in sfd_kernels.cu (update_v3D.cl / update_s3D.cl).
#include <cuda_runtime.h>

#include "sfd_internal.h"
#include "sfd_kernels.h"

namespace sfd {

typedef int64_t i64;

constexpr int TZ = 32;
constexpr int TY = 16;

// CPML recursion (identical to the general kernels)
__device__ __forceinline__ void cpml_f(float *psi, i64 q, const float *K, const float *a, const float *b, int ci,
                                       float &d)
{
    float ps = __ldg(b + ci) * psi[q] + __ldg(a + ci) * d;
    psi[q] = ps;
    d = d / __ldg(K + ci) + ps;
}

// one plane of one field in shared memory, rows of y, z fastest
template <int F>
struct Plane {
    float v[TY + 2 * F][TZ + 2 * F];
};

// Fill the halo of a plane tile from global memory (interior is written by
// the owning threads).  Cells outside the padded grid are left untouched:
// they are only read by threads whose own cell lies outside the update range.
template <int F>
__device__ __forceinline__ void load_halo(Plane<F> &pl, const float *__restrict__ fld, i64 plane_base, int y0, int z0,
                                          int NY, int NZ, int tid, int nthreads)
{
    constexpr int W = TZ + 2 * F;
    constexpr int NROWS = 2 * F * W;     // y-halo rows (top F and bottom F, full width)
    constexpr int NCOLS = TY * 2 * F;    // z-halo columns of interior rows
    for (int idx = tid; idx < NROWS + NCOLS; idx += nthreads) {
        int yy, zz;
        if (idx < NROWS) {
            int r = idx / W;
            zz = idx % W;
            yy = r < F ? r : TY + r;     // rows 0..F-1 and TY+F..TY+2F-1
        } else {
            int c = idx - NROWS;
            yy = F + c / (2 * F);
            int k = c % (2 * F);
            zz = k < F ? k : TZ + k;
        }
        int gy = y0 - F + yy, gz = z0 - F + zz;
        if (gy >= 0 && gy < NY && gz >= 0 && gz < NZ) pl.v[yy][zz] = __ldg(fld + plane_base + (i64)gy * NZ + gz);
    }
}

template <int F>
__device__ __forceinline__ float dz_fw(const Plane<F> &p, int ty, int tz, const float *hc)
{
    float acc = hc[0] * (p.v[ty + F][tz + F + 1] - p.v[ty + F][tz + F]);
#pragma unroll
    for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], p.v[ty + F][tz + F + m] - p.v[ty + F][tz + F - (m - 1)], acc);
    return acc;
}
template <int F>
__device__ __forceinline__ float dz_bw(const Plane<F> &p, int ty, int tz, const float *hc)
{
    float acc = hc[0] * (p.v[ty + F][tz + F] - p.v[ty + F][tz + F - 1]);
#pragma unroll
    for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], p.v[ty + F][tz + F + (m - 1)] - p.v[ty + F][tz + F - m], acc);
    return acc;
}
template <int F>
__device__ __forceinline__ float dy_fw(const Plane<F> &p, int ty, int tz, const float *hc)
{
    float acc = hc[0] * (p.v[ty + F + 1][tz + F] - p.v[ty + F][tz + F]);
#pragma unroll
    for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], p.v[ty + F + m][tz + F] - p.v[ty + F - (m - 1)][tz + F], acc);
    return acc;
}
template <int F>
__device__ __forceinline__ float dy_bw(const Plane<F> &p, int ty, int tz, const float *hc)
{
    float acc = hc[0] * (p.v[ty + F][tz + F] - p.v[ty + F - 1][tz + F]);
#pragma unroll
    for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], p.v[ty + F + (m - 1)][tz + F] - p.v[ty + F - m][tz + F], acc);
    return acc;
}
// x differences from a queue q[0..2F] holding x-F .. x+F (centre q[F])
template <int F>
__device__ __forceinline__ float dx_fw(const float *q, const float *hc)
{
    float acc = hc[0] * (q[F + 1] - q[F]);
#pragma unroll
    for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], q[F + m] - q[F - (m - 1)], acc);
    return acc;
}
template <int F>
__device__ __forceinline__ float dx_bw(const float *q, const float *hc)
{
    float acc = hc[0] * (q[F] - q[F - 1]);
#pragma unroll
    for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], q[F + (m - 1)] - q[F - m], acc);
    return acc;
}

template <int F>
__device__ __forceinline__ void shift_in(float *q, float v)
{
#pragma unroll
    for (int k = 0; k < 2 * F; k++) q[k] = q[k + 1];
    q[2 * F] = v;
}

// ------------------------------------------------------------- velocity
template <int F>
__global__ void __launch_bounds__(TZ *TY) k_v3d_fast(Grid g, Fields f, int xchunk)
{
    __shared__ Plane<F> s_syy, s_szz, s_sxy, s_syz, s_sxz;
    const int tz = threadIdx.x, ty = threadIdx.y, tid = ty * TZ + tz;
    const int z0 = blockIdx.x * TZ + F, y0 = blockIdx.y * TY + F;
    const int gz = z0 + tz, gy = y0 + ty;
    const int NZ = g.NZ, NY = g.NY, NX = g.NX;
    // inner: the cell lies in the padded grid (its value is loaded and shared);
    // active: the cell is updated
    const bool inner = gz < NZ && gy < NY;
    const bool active = gz <= NZ - F - 1 && gy <= NY - F - 1;
    const i64 sx = (i64)NY * NZ;
    const i64 col = (i64)gy * NZ + gz;  // offset of this thread's column within a plane
    const int xs = F + blockIdx.z * xchunk;
    const int xe = min(xs + xchunk, NX - F);
    const float *hc = g.hc;
    const float *sxx = f.w[SXX], *syy = f.w[SYY], *szz = f.w[SZZ], *sxy = f.w[SXY], *syz = f.w[SYZ], *sxz = f.w[SXZ];
    float qxx[2 * F + 1], qxy[2 * F + 1], qxz[2 * F + 1];
    // preload x = xs-F .. xs+F-1
#pragma unroll
    for (int k = 0; k < 2 * F; k++) {
        i64 o = (i64)(xs - F + k) * sx + col;
        qxx[k + 1] = inner ? __ldg(sxx + o) : 0.0f;
        qxy[k + 1] = inner ? __ldg(sxy + o) : 0.0f;
        qxz[k + 1] = inner ? __ldg(sxz + o) : 0.0f;
    }
    for (int x = xs; x < xe; x++) {
        const i64 pb = (i64)x * sx;
        {
            i64 o = (i64)(x + F) * sx + col;
            shift_in<F>(qxx, inner ? __ldg(sxx + o) : 0.0f);
            shift_in<F>(qxy, inner ? __ldg(sxy + o) : 0.0f);
            shift_in<F>(qxz, inner ? __ldg(sxz + o) : 0.0f);
        }
        __syncthreads();  // previous iteration done with the tiles
        if (inner) {
            s_syy.v[ty + F][tz + F] = __ldg(syy + pb + col);
            s_szz.v[ty + F][tz + F] = __ldg(szz + pb + col);
            s_syz.v[ty + F][tz + F] = __ldg(syz + pb + col);
        }
        s_sxy.v[ty + F][tz + F] = qxy[F];
        s_sxz.v[ty + F][tz + F] = qxz[F];
        load_halo<F>(s_syy, syy, pb, y0, z0, NY, NZ, tid, TZ * TY);
        load_halo<F>(s_szz, szz, pb, y0, z0, NY, NZ, tid, TZ * TY);
        load_halo<F>(s_sxy, sxy, pb, y0, z0, NY, NZ, tid, TZ * TY);
        load_halo<F>(s_syz, syz, pb, y0, z0, NY, NZ, tid, TZ * TY);
        load_halo<F>(s_sxz, sxz, pb, y0, z0, NY, NZ, tid, TZ * TY);
        __syncthreads();
        if (!active) continue;
        float szz_z = dz_fw<F>(s_szz, ty, tz, hc);
        float sxx_x = dx_fw<F>(qxx, hc);
        float sxz_x = dx_bw<F>(qxz, hc);
        float sxz_z = dz_bw<F>(s_sxz, ty, tz, hc);
        float syz_y = dy_bw<F>(s_syz, ty, tz, hc);
        float syz_z = dz_bw<F>(s_syz, ty, tz, hc);
        float syy_y = dy_fw<F>(s_syy, ty, tz, hc);
        float sxy_x = dx_bw<F>(qxy, hc);
        float sxy_y = dy_bw<F>(s_sxy, ty, tz, hc);
        const i64 iv = pb + col;
        const i64 ip = ((i64)(x - F) * g.ny + (gy - F)) * g.nz + (gz - F);
        if (g.abs_type == 1) {
            const int NAB = g.nab;
            const i64 nz = g.nz, ny = g.ny;
            if (gz > NZ - NAB - F - 1) {
                i64 i = x - F, j = gy - F, k = gz - NZ + NAB + F + NAB;
                int ind = 2 * NAB - 1 - (int)k;
                i64 q = (i * ny + j) * (2 * NAB) + k;
                cpml_f(f.psi[PSXZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], ind + 1, sxz_z);
                cpml_f(f.psi[PSYZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], ind + 1, syz_z);
                cpml_f(f.psi[PSZZ_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, szz_z);
            } else if (!g.freesurf && gz - F < NAB) {
                i64 i = x - F, j = gy - F, k = gz - F;
                i64 q = (i * ny + j) * (2 * NAB) + k;
                cpml_f(f.psi[PSXZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], (int)k, sxz_z);
                cpml_f(f.psi[PSYZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], (int)k, syz_z);
                cpml_f(f.psi[PSZZ_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], (int)k, szz_z);
            }
            if (gy - F < NAB) {
                i64 i = x - F, j = gy - F, k = gz - F;
                i64 q = (i * (2 * NAB) + j) * nz + k;
                cpml_f(f.psi[PSXY_Y], q, f.cy[CK], f.cy[CA], f.cy[CB], (int)j, sxy_y);
                cpml_f(f.psi[PSYY_Y], q, f.cy[CKH], f.cy[CAH], f.cy[CBH], (int)j, syy_y);
                cpml_f(f.psi[PSYZ_Y], q, f.cy[CK], f.cy[CA], f.cy[CB], (int)j, syz_y);
            } else if (gy > NY - NAB - F - 1) {
                i64 i = x - F, j = gy - NY + NAB + F + NAB, k = gz - F;
                int ind = 2 * NAB - 1 - (int)j;
                i64 q = (i * (2 * NAB) + j) * nz + k;
                cpml_f(f.psi[PSXY_Y], q, f.cy[CK], f.cy[CA], f.cy[CB], ind + 1, sxy_y);
                cpml_f(f.psi[PSYY_Y], q, f.cy[CKH], f.cy[CAH], f.cy[CBH], ind, syy_y);
                cpml_f(f.psi[PSYZ_Y], q, f.cy[CK], f.cy[CA], f.cy[CB], ind + 1, syz_y);
            }
            if (x - F < NAB) {
                i64 i = x - F, j = gy - F, k = gz - F;
                i64 q = (i * ny + j) * nz + k;
                cpml_f(f.psi[PSXX_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], (int)i, sxx_x);
                cpml_f(f.psi[PSXY_X], q, f.cx[CK], f.cx[CA], f.cx[CB], (int)i, sxy_x);
                cpml_f(f.psi[PSXZ_X], q, f.cx[CK], f.cx[CA], f.cx[CB], (int)i, sxz_x);
            }
            if (x > NX - NAB - F - 1) {
                i64 i = x - NX + NAB + F + NAB, j = gy - F, k = gz - F;
                int ind = 2 * NAB - 1 - (int)i;
                i64 q = (i * ny + j) * nz + k;
                cpml_f(f.psi[PSXX_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], ind, sxx_x);
                cpml_f(f.psi[PSXY_X], q, f.cx[CK], f.cx[CA], f.cx[CB], ind + 1, sxy_x);
                cpml_f(f.psi[PSXZ_X], q, f.cx[CK], f.cx[CA], f.cx[CB], ind + 1, sxz_x);
            }
        }
        float vx = f.w[VX][iv] + (sxx_x + sxy_y + sxz_z) * __ldg(f.p[PRIP] + ip);
        float vy = f.w[VY][iv] + (syy_y + sxy_x + syz_z) * __ldg(f.p[PRJP] + ip);
        float vz = f.w[VZ][iv] + (szz_z + sxz_x + syz_y) * __ldg(f.p[PRKP] + ip);
        if (g.abs_type == 2) {
            const int NAB = g.nab;
            const float *tp = f.taper;
            if (!g.freesurf && gz - F < NAB) { float t = tp[gz - F]; vx *= t; vy *= t; vz *= t; }
            if (gz > NZ - NAB - F - 1) { float t = tp[NZ - F - gz - 1]; vx *= t; vy *= t; vz *= t; }
            if (gy - F < NAB) { float t = tp[gy - F]; vx *= t; vy *= t; vz *= t; }
            if (gy > NY - NAB - F - 1) { float t = tp[NY - F - gy - 1]; vx *= t; vy *= t; vz *= t; }
            if (x - F < NAB) { float t = tp[x - F]; vx *= t; vy *= t; vz *= t; }
            if (x > NX - NAB - F - 1) { float t = tp[NX - F - x - 1]; vx *= t; vy *= t; vz *= t; }
        }
        f.w[VX][iv] = vx;
        f.w[VY][iv] = vy;
        f.w[VZ][iv] = vz;
    }
}

// --------------------------------------------------------------- stress
template <int F, int L>
__global__ void __launch_bounds__(TZ *TY) k_s3d_fast(Grid g, Fields f, int xchunk)
{
    __shared__ Plane<F> s_vx, s_vy, s_vz;
    const int tz = threadIdx.x, ty = threadIdx.y, tid = ty * TZ + tz;
    const int z0 = blockIdx.x * TZ + F, y0 = blockIdx.y * TY + F;
    const int gz = z0 + tz, gy = y0 + ty;
    const int NZ = g.NZ, NY = g.NY, NX = g.NX;
    const bool inner = gz < NZ && gy < NY;
    const bool active = gz <= NZ - F - 1 && gy <= NY - F - 1;
    const i64 sx = (i64)NY * NZ;
    const i64 col = (i64)gy * NZ + gz;
    const int xs = F + blockIdx.z * xchunk;
    const int xe = min(xs + xchunk, NX - F);
    const float *hc = g.hc;
    const float *vxp = f.w[VX], *vyp = f.w[VY], *vzp = f.w[VZ];
    float qx[2 * F + 1], qy[2 * F + 1], qz[2 * F + 1];
#pragma unroll
    for (int k = 0; k < 2 * F; k++) {
        i64 o = (i64)(xs - F + k) * sx + col;
        qx[k + 1] = inner ? __ldg(vxp + o) : 0.0f;
        qy[k + 1] = inner ? __ldg(vyp + o) : 0.0f;
        qz[k + 1] = inner ? __ldg(vzp + o) : 0.0f;
    }
    for (int x = xs; x < xe; x++) {
        const i64 pb = (i64)x * sx;
        {
            i64 o = (i64)(x + F) * sx + col;
            shift_in<F>(qx, inner ? __ldg(vxp + o) : 0.0f);
            shift_in<F>(qy, inner ? __ldg(vyp + o) : 0.0f);
            shift_in<F>(qz, inner ? __ldg(vzp + o) : 0.0f);
        }
        __syncthreads();
        s_vx.v[ty + F][tz + F] = qx[F];
        s_vy.v[ty + F][tz + F] = qy[F];
        s_vz.v[ty + F][tz + F] = qz[F];
        load_halo<F>(s_vx, vxp, pb, y0, z0, NY, NZ, tid, TZ * TY);
        load_halo<F>(s_vy, vyp, pb, y0, z0, NY, NZ, tid, TZ * TY);
        load_halo<F>(s_vz, vzp, pb, y0, z0, NY, NZ, tid, TZ * TY);
        __syncthreads();
        if (!active) continue;
        const i64 iv = pb + col;
        const i64 ip = ((i64)(x - F) * g.ny + (gy - F)) * g.nz + (gz - F);
        float vzx = dx_fw<F>(qz, hc), vzy = dy_fw<F>(s_vz, ty, tz, hc), vzz = dz_bw<F>(s_vz, ty, tz, hc);
        float vyx = dx_fw<F>(qy, hc), vyy = dy_bw<F>(s_vy, ty, tz, hc), vyz = dz_fw<F>(s_vy, ty, tz, hc);
        float vxx = dx_bw<F>(qx, hc), vxy = dy_fw<F>(s_vx, ty, tz, hc), vxz = dz_fw<F>(s_vx, ty, tz, hc);
        if (g.abs_type == 1) {
            const int NAB = g.nab;
            const i64 nz = g.nz, ny = g.ny;
            if (gz > NZ - NAB - F - 1) {
                i64 i = x - F, j = gy - F, k = gz - NZ + NAB + F + NAB;
                int ind = 2 * NAB - 1 - (int)k;
                i64 q = (i * ny + j) * (2 * NAB) + k;
                cpml_f(f.psi[PVX_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, vxz);
                cpml_f(f.psi[PVY_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, vyz);
                cpml_f(f.psi[PVZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], ind + 1, vzz);
            }
            if (!g.freesurf && gz - F < NAB) {
                i64 i = x - F, j = gy - F, k = gz - F;
                i64 q = (i * ny + j) * (2 * NAB) + k;
                cpml_f(f.psi[PVX_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], (int)k, vxz);
                cpml_f(f.psi[PVY_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], (int)k, vyz);
                cpml_f(f.psi[PVZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], (int)k, vzz);
            }
            if (gy - F < NAB) {
                i64 i = x - F, j = gy - F, k = gz - F;
                i64 q = (i * (2 * NAB) + j) * nz + k;
                cpml_f(f.psi[PVX_Y], q, f.cy[CKH], f.cy[CAH], f.cy[CBH], (int)j, vxy);
                cpml_f(f.psi[PVY_Y], q, f.cy[CK], f.cy[CA], f.cy[CB], (int)j, vyy);
                cpml_f(f.psi[PVZ_Y], q, f.cy[CKH], f.cy[CAH], f.cy[CBH], (int)j, vzy);
            }
            if (gy > NY - NAB - F - 1) {
                i64 i = x - F, j = gy - NY + NAB + F + NAB, k = gz - F;
                int ind = 2 * NAB - 1 - (int)j;
                i64 q = (i * (2 * NAB) + j) * nz + k;
                cpml_f(f.psi[PVX_Y], q, f.cy[CKH], f.cy[CAH], f.cy[CBH], ind, vxy);
                cpml_f(f.psi[PVY_Y], q, f.cy[CK], f.cy[CA], f.cy[CB], ind + 1, vyy);
                cpml_f(f.psi[PVZ_Y], q, f.cy[CKH], f.cy[CAH], f.cy[CBH], ind, vzy);
            }
            if (x - F < NAB) {
                i64 i = x - F, j = gy - F, k = gz - F;
                i64 q = (i * ny + j) * nz + k;
                cpml_f(f.psi[PVX_X], q, f.cx[CK], f.cx[CA], f.cx[CB], (int)i, vxx);
                cpml_f(f.psi[PVY_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], (int)i, vyx);
                cpml_f(f.psi[PVZ_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], (int)i, vzx);
            }
            if (x > NX - NAB - F - 1) {
                i64 i = x - NX + NAB + F + NAB, j = gy - F, k = gz - F;
                int ind = 2 * NAB - 1 - (int)i;
                i64 q = (i * ny + j) * nz + k;
                cpml_f(f.psi[PVX_X], q, f.cx[CK], f.cx[CA], f.cx[CB], ind + 1, vxx);
                cpml_f(f.psi[PVY_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], ind, vyx);
                cpml_f(f.psi[PVZ_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], ind, vzx);
            }
        }
        float vxyyx = vxy + vyx, vyzzy = vyz + vzy, vxzzx = vxz + vzx;
        float vxxyyzz = vxx + vyy + vzz, vyyzz = vyy + vzz, vxxzz = vxx + vzz, vxxyy = vxx + vyy;
        float s0 = f.w[SXY][iv], s1 = f.w[SYZ][iv], s2 = f.w[SXZ][iv];
        float s3 = f.w[SXX][iv], s4 = f.w[SYY][iv], s5 = f.w[SZZ][iv];
        if (L == 0) {
            float fipjp = __ldg(f.p[PMUIPJP] + ip), fjpkp = __ldg(f.p[PMUJPKP] + ip), fipkp = __ldg(f.p[PMUIPKP] + ip);
            float gm = __ldg(f.p[PM] + ip), fm = 2.0f * __ldg(f.p[PMU] + ip);
            s0 += fipjp * vxyyx;
            s1 += fjpkp * vyzzy;
            s2 += fipkp * vxzzx;
            s3 += gm * vxxyyzz - fm * vyyzz;
            s4 += gm * vxxyyzz - fm * vxxzz;
            s5 += gm * vxxyyzz - fm * vxxyy;
        } else {
            float lM = __ldg(f.p[PM] + ip), lmu = __ldg(f.p[PMU] + ip);
            float lmuipkp = __ldg(f.p[PMUIPKP] + ip), lmuipjp = __ldg(f.p[PMUIPJP] + ip),
                  lmujpkp = __ldg(f.p[PMUJPKP] + ip);
            float ltaup = __ldg(f.p[PTAUP] + ip), ltaus = __ldg(f.p[PTAUS] + ip);
            float ltausipkp = __ldg(f.p[PTAUSIPKP] + ip), ltausipjp = __ldg(f.p[PTAUSIPJP] + ip),
                  ltausjpkp = __ldg(f.p[PTAUSJPKP] + ip);
            float fipjp = lmuipjp * (1.0f + (float)L * ltausipjp);
            float fjpkp = lmujpkp * (1.0f + (float)L * ltausjpkp);
            float fipkp = lmuipkp * (1.0f + (float)L * ltausipkp);
            float gm = lM * (1.0f + (float)L * ltaup);
            float fm = 2.0f * lmu * (1.0f + (float)L * ltaus);
            float dipjp = lmuipjp * ltausipjp / g.dt, djpkp = lmujpkp * ltausjpkp / g.dt,
                  dipkp = lmuipkp * ltausipkp / g.dt;
            float d = 2.0f * lmu * ltaus / g.dt, e = lM * ltaup / g.dt;
            float r[6][L > 0 ? L : 1];
#pragma unroll
            for (int l = 0; l < L; l++) {
                i64 ir = l * g.nvol + iv;
                r[0][l] = f.r[RXY][ir]; r[1][l] = f.r[RYZ][ir]; r[2][l] = f.r[RXZ][ir];
                r[3][l] = f.r[RXX][ir]; r[4][l] = f.r[RYY][ir]; r[5][l] = f.r[RZZ][ir];
            }
            float a[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int l = 0; l < L; l++)
#pragma unroll
                for (int q = 0; q < 6; q++) a[q] += r[q][l];
            float lsxy = fipjp * vxyyx + g.dt2 * a[0];
            float lsyz = fjpkp * vyzzy + g.dt2 * a[1];
            float lsxz = fipkp * vxzzx + g.dt2 * a[2];
            float lsxx = (gm * vxxyyzz - fm * vyyzz) + g.dt2 * a[3];
            float lsyy = (gm * vxxyyzz - fm * vxxzz) + g.dt2 * a[4];
            float lszz = (gm * vxxyyzz - fm * vxxyy) + g.dt2 * a[5];
#pragma unroll
            for (int q = 0; q < 6; q++) a[q] = 0;
#pragma unroll
            for (int l = 0; l < L; l++) {
                float el = g.eta[l];
                float b = 1.0f / (1.0f + el * 0.5f), c = 1.0f - el * 0.5f;
                r[0][l] = b * (r[0][l] * c - el * (dipjp * vxyyx));
                r[1][l] = b * (r[1][l] * c - el * (djpkp * vyzzy));
                r[2][l] = b * (r[2][l] * c - el * (dipkp * vxzzx));
                r[3][l] = b * (r[3][l] * c - el * (e * vxxyyzz - d * vyyzz));
                r[4][l] = b * (r[4][l] * c - el * (e * vxxyyzz - d * vxxzz));
                r[5][l] = b * (r[5][l] * c - el * (e * vxxyyzz - d * vxxyy));
#pragma unroll
                for (int q = 0; q < 6; q++) a[q] += r[q][l];
                i64 ir = l * g.nvol + iv;
                f.r[RXY][ir] = r[0][l]; f.r[RYZ][ir] = r[1][l]; f.r[RXZ][ir] = r[2][l];
                f.r[RXX][ir] = r[3][l]; f.r[RYY][ir] = r[4][l]; f.r[RZZ][ir] = r[5][l];
            }
            s0 += lsxy + g.dt2 * a[0];
            s1 += lsyz + g.dt2 * a[1];
            s2 += lsxz + g.dt2 * a[2];
            s3 += lsxx + g.dt2 * a[3];
            s4 += lsyy + g.dt2 * a[4];
            s5 += lszz + g.dt2 * a[5];
        }
        if (g.abs_type == 2) {
            // Cerjan factors in the reference's order (update_s3D.cl:426-488)
            const int NAB = g.nab;
            const float *tp = f.taper;
            float t;
#define SFD_TAPER6(cond, idx) \
    if (cond) { t = tp[idx]; s0 *= t; s1 *= t; s2 *= t; s3 *= t; s4 *= t; s5 *= t; }
            SFD_TAPER6(!g.freesurf && gz - F < NAB, gz - F)
            SFD_TAPER6(gz > NZ - NAB - F - 1, NZ - F - gz - 1)
            SFD_TAPER6(gy - F < NAB, gy - F)
            SFD_TAPER6(gy > NY - NAB - F - 1, NY - F - gy - 1)
            SFD_TAPER6(x - F < NAB, x - F)
            SFD_TAPER6(x > NX - NAB - F - 1, NX - F - x - 1)
#undef SFD_TAPER6
        }
        f.w[SXY][iv] = s0; f.w[SYZ][iv] = s1; f.w[SXZ][iv] = s2;
        f.w[SXX][iv] = s3; f.w[SYY][iv] = s4; f.w[SZZ][iv] = s5;
    }
}

// ------------------------------------------------------------- launchers
static inline unsigned cdiv(long a, long b) { return (unsigned)((a + b - 1) / b); }

int fast3d_xchunk(const Grid &g)
{
    // enough CTAs for every SM to hold two, each chunk long enough that the
    // 2F-plane preload stays a small overhead
    long tiles = (long)cdiv(g.nz, TZ) * cdiv(g.ny, TY);
    int xc = 64;
    while (xc > 8 && tiles * cdiv(g.nx, xc) < 4L * 148) xc /= 2;
    return xc;
}

bool launch_update_v_fast(const Grid &g, const Fields &f, cudaStream_t st)
{
    if (g.nd != 3) return false;
    int xc = fast3d_xchunk(g);
    dim3 b(TZ, TY), gr(cdiv(g.nz, TZ), cdiv(g.ny, TY), cdiv(g.nx, xc));
    switch (g.F) {
    case 1: k_v3d_fast<1><<<gr, b, 0, st>>>(g, f, xc); break;
    case 2: k_v3d_fast<2><<<gr, b, 0, st>>>(g, f, xc); break;
    case 3: k_v3d_fast<3><<<gr, b, 0, st>>>(g, f, xc); break;
    case 4: k_v3d_fast<4><<<gr, b, 0, st>>>(g, f, xc); break;
    case 5: k_v3d_fast<5><<<gr, b, 0, st>>>(g, f, xc); break;
    case 6: k_v3d_fast<6><<<gr, b, 0, st>>>(g, f, xc); break;
    default: return false;
    }
    return true;
}

template <int F>
static bool launch_s_fast_F(const Grid &g, const Fields &f, cudaStream_t st)
{
    int xc = fast3d_xchunk(g);
    dim3 b(TZ, TY), gr(cdiv(g.nz, TZ), cdiv(g.ny, TY), cdiv(g.nx, xc));
    switch (g.L) {
    case 0: k_s3d_fast<F, 0><<<gr, b, 0, st>>>(g, f, xc); return true;
    case 1: k_s3d_fast<F, 1><<<gr, b, 0, st>>>(g, f, xc); return true;
    case 2: k_s3d_fast<F, 2><<<gr, b, 0, st>>>(g, f, xc); return true;
    case 3: k_s3d_fast<F, 3><<<gr, b, 0, st>>>(g, f, xc); return true;
    default: return false;
    }
}

bool launch_update_s_fast(const Grid &g, const Fields &f, cudaStream_t st)
{
    if (g.nd != 3) return false;
    switch (g.F) {
    case 1: return launch_s_fast_F<1>(g, f, st);
    case 2: return launch_s_fast_F<2>(g, f, st);
    case 3: return launch_s_fast_F<3>(g, f, st);
    case 4: return launch_s_fast_F<4>(g, f, st);
    case 5: return launch_s_fast_F<5>(g, f, st);
    case 6: return launch_s_fast_F<6>(g, f, st);
    default: return false;
    }
}

}  // namespace sfd
