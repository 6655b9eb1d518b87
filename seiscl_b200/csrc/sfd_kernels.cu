// sfd_kernels.cu -- general sm_100a kernels of the staggered-grid FDTD engine.
//
// One thread per grid cell; z (fastest) runs along the warp so every stencil
// tap is a coalesced row load served from L1/L2.  These kernels cover every
// configuration the engine accepts (2D P-SV and 3D, FDORDER 2..12, elastic
// and viscoelastic, CPML or Cerjan taper, free surface) and are the
// reference implementation inside the product; sfd_kernels3d_fast.cu holds
// the register-blocked 3D kernels used on the hot configurations.
//
// Semantics follow the reference kernels cell for cell:
//   update_v  src/update_v2D.cl:32-246,  src/update_v3D.cl:34-369
//   update_s  src/update_s2D.cl:30-327,  src/update_s3D.cl:35-489
//   surface   src/surface2D.cl:30-193,   src/surface3D.cl:39-271
//   adjoint   src/update_adj{v,s}{2D,3D}.cl, src/surface{2D,3D}_adj.cl
//   boundary  src/savebnd{2D,3D}.cl, src/header_injectbnd.cl
// Arithmetic is FP32 with FMA; gradients accumulate in FP64.
#include <algorithm>
#include <cstdlib>
#include <utility>
#include <type_traits>

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "sfd_internal.h"
#include "sfd_kernels.h"

namespace sfd {

typedef int64_t i64;

// ---------------------------------------------------------------- helpers
// forward difference c1 (v[i+1]-v[i]) + c2 (v[i+2]-v[i-1]) + ...  (Dxp)
template <int F>
__device__ __forceinline__ float dfw(const float *__restrict__ v, i64 i, i64 st, const float *hc)
{
    float acc = hc[0] * (__ldg(v + i + st) - __ldg(v + i));
#pragma unroll
    for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], __ldg(v + i + m * st) - __ldg(v + i - (m - 1) * st), acc);
    return acc;
}
// backward difference c1 (v[i]-v[i-1]) + c2 (v[i+1]-v[i-2]) + ...  (Dxm)
template <int F>
__device__ __forceinline__ float dbw(const float *__restrict__ v, i64 i, i64 st, const float *hc)
{
    float acc = hc[0] * (__ldg(v + i) - __ldg(v + i - st));
#pragma unroll
    for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], __ldg(v + i + (m - 1) * st) - __ldg(v + i - m * st), acc);
    return acc;
}
// non-cached variants for arrays written by the same kernel
template <int F>
__device__ __forceinline__ float dfw_rw(const float *v, i64 i, i64 st, const float *hc)
{
    float acc = hc[0] * (v[i + st] - v[i]);
#pragma unroll
    for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], v[i + m * st] - v[i - (m - 1) * st], acc);
    return acc;
}
template <int F>
__device__ __forceinline__ float dbw_rw(const float *v, i64 i, i64 st, const float *hc)
{
    float acc = hc[0] * (v[i] - v[i - st]);
#pragma unroll
    for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], v[i + (m - 1) * st] - v[i - m * st], acc);
    return acc;
}

// Wave-field storage access: FP32, or FP16 holding the field times a power
// of two (the kernels compute in FP32 either way).
template <class T> __device__ __forceinline__ float ldv(const T *p);
template <> __device__ __forceinline__ float ldv<float>(const float *p) { return *p; }
template <> __device__ __forceinline__ float ldv<__half>(const __half *p) { return __half2float(*p); }
template <class T> __device__ __forceinline__ float ldgv(const T *p);
template <> __device__ __forceinline__ float ldgv<float>(const float *p) { return __ldg(p); }
template <> __device__ __forceinline__ float ldgv<__half>(const __half *p) { return __half2float(__ldg(p)); }
template <class T> __device__ __forceinline__ void stv(T *p, float v);
template <> __device__ __forceinline__ void stv<float>(float *p, float v) { *p = v; }
template <> __device__ __forceinline__ void stv<__half>(__half *p, float v) { *p = __float2half_rn(v); }
template <class T> __device__ __forceinline__ T *fld(float *p) { return reinterpret_cast<T *>(p); }

template <int F, class T>
__device__ __forceinline__ float dfwT(const T *__restrict__ v, i64 i, i64 st, const float *hc)
{
    float acc = hc[0] * (ldgv(v + i + st) - ldgv(v + i));
#pragma unroll
    for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], ldgv(v + i + m * st) - ldgv(v + i - (m - 1) * st), acc);
    return acc;
}
template <int F, class T>
__device__ __forceinline__ float dbwT(const T *__restrict__ v, i64 i, i64 st, const float *hc)
{
    float acc = hc[0] * (ldgv(v + i) - ldgv(v + i - st));
#pragma unroll
    for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], ldgv(v + i + (m - 1) * st) - ldgv(v + i - m * st), acc);
    return acc;
}
template <int F, class T>
__device__ __forceinline__ float dbw_rwT(const T *v, i64 i, i64 st, const float *hc)
{
    float acc = hc[0] * (ldv(v + i) - ldv(v + i - st));
#pragma unroll
    for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], ldv(v + i + (m - 1) * st) - ldv(v + i - m * st), acc);
    return acc;
}

// psi = b psi + a d ; d = d/K + psi    (the CPML recursion of every kernel)
__device__ __forceinline__ void cpml(float *psi, i64 q, const float *K, const float *a, const float *b, int ci,
                                     float &d)
{
    float ps = __ldg(b + ci) * psi[q] + __ldg(a + ci) * d;
    psi[q] = ps;
    d = d / __ldg(K + ci) + ps;
}

template <typename T> __device__ __forceinline__ float to_f(T v);
template <> __device__ __forceinline__ float to_f<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }

// Programmatic dependent launch (the 3D modelling loop's kernels, see
// pdl_enabled): a kernel launched with programmatic stream serialization may
// be resident before the previous kernel of the stream has finished.
// pdl_wait returns once that kernel has completed and its stores are
// visible (at once for an ordinary launch); nothing it writes may be read,
// and nothing at all written, before it.  pdl_trigger lets the next
// kernel's CTAs launch once every CTA of this grid has passed it.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
template <typename T> __device__ __forceinline__ T from_f(float v);
template <> __device__ __forceinline__ float from_f<float>(float v) { return v; }
template <> __device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// batched shots: shot b of a launch (blockIdx.z) works on copy b of every
// per-shot array
__device__ __forceinline__ void shot_fields(const Grid &g, Fields &f, int b)
{
#pragma unroll
    for (int w = 0; w < NW; w++)
        if (f.w[w]) f.w[w] += b * g.sb_w;
#pragma unroll
    for (int r = 0; r < NR; r++)
        if (f.r[r]) f.r[r] += b * g.sb_r;
#pragma unroll
    for (int i = 0; i < NPSI; i++)
        if (f.psi[i]) f.psi[i] += b * g.sb_psi;
}
__device__ __forceinline__ void shot_adj(const Grid &g, AdjFields &a, int b)
{
#pragma unroll
    for (int w = 0; w < NW; w++) {
        if (a.wr[w]) a.wr[w] += b * g.sb_w;
        if (a.bnd[w]) a.bnd[w] = (const char *)a.bnd[w] + b * g.sb_bnd;
    }
#pragma unroll
    for (int r = 0; r < NR; r++)
        if (a.rr[r]) a.rr[r] += b * g.sb_r;
#pragma unroll
    for (int k = 0; k < NG; k++) {
        if (a.grad[k]) a.grad[k] += b * g.sb_g;
        if (a.hess[k]) a.hess[k] += b * g.sb_g;
    }
}
#define SHOT_F  if (g.nb > 1) shot_fields(g, f, blockIdx.z);
#define SHOT_FA if (g.nb > 1) { shot_fields(g, f, blockIdx.z); shot_adj(g, a, blockIdx.z); }

// a saved boundary value (slice t-1) back in field units: FP16 stores carry
// a power-of-two scale (exact; 1 for FP32 and BF16 stores)
template <class T>
__device__ __forceinline__ float bnd_at(const Grid &g, const AdjFields &a, int w, i64 m)
{
    return to_f<T>(((const T *)a.bnd[w])[m]) * g.bsci[w];
}

// checkpointed gradients (g.ckpt): the forward wave field of the adjoint
// step, stored when the forward run was recomputed from a snapshot (same
// storage type and scales as the saved boundaries)
template <class T>
__device__ __forceinline__ float fwd_at(const Grid &g, const AdjFields &a, int w, i64 iv)
{
    return to_f<T>(((const T *)a.fwd[w])[iv]) * g.bsci[w];
}

// ------------------------------------------------------- boundary shells
struct BndDims {
    int NXbnd, NYbnd, NZbnd, lbnd, lbnds;
};
__device__ __host__ inline BndDims bnd_dims(const Grid &g)
{
    BndDims b;
    b.NXbnd = g.NX - 2 * g.F - 2 * g.nab;
    b.NYbnd = g.nd == 3 ? g.NY - 2 * g.F - 2 * g.nab : 1;
    if (!g.freesurf) {
        b.NZbnd = g.NZ - 2 * g.F - 2 * g.nab;
        b.lbnd = g.F + g.nab;
        b.lbnds = g.F + g.nab;
    } else {
        b.NZbnd = g.NZ - 2 * g.F - g.nab;
        b.lbnd = g.F + g.nab;
        b.lbnds = g.F;
    }
    return b;
}

// index of cell (k, i) in the saved shell, -1 if not a shell cell
// (src/header_injectbnd.cl:238-283)
__device__ __forceinline__ int inject_ind2d(const Grid &g, int k, int i)
{
    BndDims b = bnd_dims(g);
    int F = g.F, m = -1;
    i -= b.lbnd;
    k -= b.lbnds;
    if ((k > F - 1 && k < b.NZbnd - F) && (i > F - 1 && i < b.NXbnd - F)) m = -1;
    else if (k < 0 || k > b.NZbnd - 1 || i < 0 || i > b.NXbnd - 1) m = -1;
    else if (i < F) m = i * b.NZbnd + k;
    else if (i > b.NXbnd - 1 - F) { i = i - b.NXbnd + F; m = b.NZbnd * F + i * b.NZbnd + k; }
    else if (k < F) { i = i - F; m = b.NZbnd * F * 2 + (b.NXbnd - 2 * F) * F + i + k * (b.NXbnd - 2 * F); }
    else { i = i - F; k = k - b.NZbnd + F; m = b.NZbnd * F * 2 + i + k * (b.NXbnd - 2 * F); }
    return m;
}
// (src/header_injectbnd.cl:25-84)
__device__ __forceinline__ int inject_ind3d(const Grid &g, int k, int j, int i)
{
    BndDims b = bnd_dims(g);
    int F = g.F, m = -1;
    i -= b.lbnd; j -= b.lbnd; k -= b.lbnds;
    int NX = b.NXbnd, NY = b.NYbnd, NZ = b.NZbnd;
    if ((k > F - 1 && k < NZ - F) && (j > F - 1 && j < NY - F) && (i > F - 1 && i < NX - F)) m = -1;
    else if (k < 0 || k > NZ - 1 || j < 0 || j > NY - 1 || i < 0 || i > NX - 1) m = -1;
    else if (i < F) m = i * NY * NZ + j * NZ + k;
    else if (i > NX - 1 - F) { i = i - NX + F; m = NY * NZ * F + i * NY * NZ + j * NZ + k; }
    else if (j < F) { i = i - F; m = NY * NZ * F * 2 + i * F * NZ + j * NZ + k; }
    else if (j > NY - 1 - F) { i = i - F; j = j - NY + F; m = NY * NZ * F * 2 + (NX - 2 * F) * NZ * F + i * F * NZ + j * NZ + k; }
    else if (k < F) {
        i = i - F; j = j - F;
        m = NY * NZ * F * 2 + (NX - 2 * F) * NZ * F * 2 + (NX - 2 * F) * (NY - 2 * F) * F + i * (NY - 2 * F) * F + j * F + k;
    } else {
        i = i - F; j = j - F; k = k - NZ + F;
        m = NY * NZ * F * 2 + (NX - 2 * F) * NZ * F * 2 + i * (NY - 2 * F) * F + j * F + k;
    }
    return m;
}

// shell cell of saved index gid (src/savebnd2D.cl:52-93, savebnd3D.cl:46-103)
__device__ __forceinline__ bool shell_cell(const Grid &g, int gid, int &i, int &j, int &k)
{
    BndDims b = bnd_dims(g);
    int F = g.F, NAB = g.nab, gidf;
    if (g.nd != 3) {
        j = 0;
        int NZ = b.NZbnd, NX = b.NXbnd;
        if (gid < NZ * F) { gidf = gid; i = gidf / NZ + b.lbnd; k = gidf % NZ + b.lbnds; }
        else if (gid < NZ * F * 2) { gidf = gid - NZ * F; i = gidf / NZ + NX + NAB; k = gidf % NZ + b.lbnds; }
        else if (gid < NZ * F * 2 + (NX - 2 * F) * F) {
            gidf = gid - NZ * F * 2; i = gidf % (NX - 2 * F) + b.lbnd + F; k = gidf / (NX - 2 * F) + NZ + b.lbnds - F;
        } else if (gid < NZ * F * 2 + (NX - 2 * F) * 2 * F) {
            gidf = gid - NZ * F * 2 - (NX - 2 * F) * F; i = gidf % (NX - 2 * F) + b.lbnd + F; k = gidf / (NX - 2 * F) + b.lbnds;
        } else return false;
        return true;
    }
    int NX = b.NXbnd, NY = b.NYbnd, NZ = b.NZbnd;
    int a0 = NY * NZ * F, a1 = NZ * (NX - 2 * F) * F, a2 = (NY - 2 * F) * (NX - 2 * F) * F;
    if (gid < a0) { gidf = gid; i = gidf / (NY * NZ) + b.lbnd; j = (gidf / NZ) % NY + b.lbnd; k = gidf % NZ + b.lbnds; }
    else if (gid < 2 * a0) { gidf = gid - a0; i = gidf / (NY * NZ) + NX + NAB; j = (gidf / NZ) % NY + b.lbnd; k = gidf % NZ + b.lbnds; }
    else if (gid < 2 * a0 + a1) { gidf = gid - 2 * a0; i = gidf / (NZ * F) + b.lbnd + F; j = (gidf / NZ) % F + b.lbnd; k = gidf % NZ + b.lbnds; }
    else if (gid < 2 * a0 + 2 * a1) { gidf = gid - 2 * a0 - a1; i = gidf / (NZ * F) + b.lbnd + F; j = (gidf / NZ) % F + NY + NAB; k = gidf % NZ + b.lbnds; }
    else if (gid < 2 * a0 + 2 * a1 + a2) {
        gidf = gid - 2 * a0 - 2 * a1;
        i = gidf / (F * (NY - 2 * F)) + b.lbnd + F; j = (gidf / F) % (NY - 2 * F) + b.lbnd + F; k = gidf % F + NZ + b.lbnds - F;
    } else if (gid < 2 * a0 + 2 * a1 + 2 * a2) {
        gidf = gid - 2 * a0 - 2 * a1 - a2;
        i = gidf / (F * (NY - 2 * F)) + b.lbnd + F; j = (gidf / F) % (NY - 2 * F) + b.lbnd + F; k = gidf % F + b.lbnds;
    } else return false;
    return true;
}

// ------------------------------------------------------------------ taper
template <int NF, class T = float>
__device__ __forceinline__ void apply_taper(const Grid &g, const float *taper, int gz, int gy, int gx,
                                            T *const *fs, i64 iv)
{
    int F = g.F, NAB = g.nab;
    auto mul = [&](float t) {
        for (int q = 0; q < NF; q++) stv(fs[q] + iv, ldv(fs[q] + iv) * t);
    };
    if (!g.freesurf && gz - F < NAB) mul(__ldg(taper + gz - F));
    if (gz > g.NZ - NAB - F - 1) mul(__ldg(taper + g.NZ - F - gz - 1));
    if (g.nd == 3) {
        if (gy - F < NAB) mul(__ldg(taper + gy - F));
        if (gy > g.NY - NAB - F - 1) mul(__ldg(taper + g.NY - F - gy - 1));
    }
    if (gx - F < NAB) mul(__ldg(taper + gx - F));
    if (gx > g.NX - NAB - F - 1) mul(__ldg(taper + g.NX - F - gx - 1));
}

// ===================================================================== 2D
// CPML on the stress derivatives (update_v2D.cl:146-207)
__device__ __forceinline__ void cpml_v2d(const Grid &g, const Fields &f, int gz, int gx, float &sxx_x,
                                         float &szz_z, float &sxz_x, float &sxz_z)
{
    int F = g.F, NAB = g.nab, NZ = g.NZ, NX = g.NX;
    if (gz > NZ - NAB - F - 1) {
        int i = gx - F, k = gz - NZ + NAB + F + NAB, ind = 2 * NAB - 1 - k;
        i64 q = (i64)i * (2 * NAB) + k;
        cpml(f.psi[PSXZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], ind + 1, sxz_z);
        cpml(f.psi[PSZZ_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, szz_z);
    } else if (!g.freesurf && gz - F < NAB) {
        int i = gx - F, k = gz - F;
        i64 q = (i64)i * (2 * NAB) + k;
        cpml(f.psi[PSXZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], k, sxz_z);
        cpml(f.psi[PSZZ_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], k, szz_z);
    }
    if (gx - F < NAB) {
        int i = gx - F, k = gz - F;
        i64 q = (i64)i * g.nz + k;
        cpml(f.psi[PSXX_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], i, sxx_x);
        cpml(f.psi[PSXZ_X], q, f.cx[CK], f.cx[CA], f.cx[CB], i, sxz_x);
    }
    if (gx > NX - NAB - F - 1) {
        int i = gx - NX + NAB + F + NAB, k = gz - F, ind = 2 * NAB - 1 - i;
        i64 q = (i64)i * g.nz + k;
        cpml(f.psi[PSXX_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], ind, sxx_x);
        cpml(f.psi[PSXZ_X], q, f.cx[CK], f.cx[CA], f.cx[CB], ind + 1, sxz_x);
    }
}

// CPML on the velocity derivatives (update_s2D.cl:145-208)
__device__ __forceinline__ void cpml_s2d(const Grid &g, const Fields &f, int gz, int gx, float &vxx, float &vxz,
                                         float &vzx, float &vzz)
{
    int F = g.F, NAB = g.nab, NZ = g.NZ, NX = g.NX;
    if (gz > NZ - NAB - F - 1) {
        int i = gx - F, k = gz - NZ + NAB + F + NAB, ind = 2 * NAB - 1 - k;
        i64 q = (i64)i * (2 * NAB) + k;
        cpml(f.psi[PVX_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, vxz);
        cpml(f.psi[PVZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], ind + 1, vzz);
    } else if (!g.freesurf && gz - F < NAB) {
        int i = gx - F, k = gz - F;
        i64 q = (i64)i * (2 * NAB) + k;
        cpml(f.psi[PVX_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], k, vxz);
        cpml(f.psi[PVZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], k, vzz);
    }
    if (gx - F < NAB) {
        int i = gx - F, k = gz - F;
        i64 q = (i64)i * g.nz + k;
        cpml(f.psi[PVX_X], q, f.cx[CK], f.cx[CA], f.cx[CB], i, vxx);
        cpml(f.psi[PVZ_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], i, vzx);
    }
    if (gx > NX - NAB - F - 1) {
        int i = gx - NX + NAB + F + NAB, k = gz - F, ind = 2 * NAB - 1 - i;
        i64 q = (i64)i * g.nz + k;
        cpml(f.psi[PVX_X], q, f.cx[CK], f.cx[CA], f.cx[CB], ind + 1, vxx);
        cpml(f.psi[PVZ_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], ind, vzx);
    }
}

// T: storage of the wave fields and memory variables (float, or __half
// holding them times power-of-two scales; the arithmetic is FP32)
template <int F, class T = float>
__global__ void __launch_bounds__(256) k_v2d(Grid g, Fields f)
{
    SHOT_F
    int gz = blockIdx.x * blockDim.x + threadIdx.x + F;
    int gx = blockIdx.y * blockDim.y + threadIdx.y + F;
    if (gz > g.NZ - F - 1 || gx > g.NX - F - 1) return;
    i64 ip = (i64)(gx - F) * g.nz + (gz - F), iv = (i64)gx * g.NZ + gz;
    const float *hc = g.hc;
    T *vx = fld<T>(f.w[VX]), *vz = fld<T>(f.w[VZ]);
    float sxx_x = dfwT<F>(fld<T>(f.w[SXX]), iv, g.NZ, hc);
    float szz_z = dfwT<F>(fld<T>(f.w[SZZ]), iv, 1, hc);
    float sxz_z = dbwT<F>(fld<T>(f.w[SXZ]), iv, 1, hc);
    float sxz_x = dbwT<F>(fld<T>(f.w[SXZ]), iv, g.NZ, hc);
    if (g.abs_type == 1) cpml_v2d(g, f, gz, gx, sxx_x, szz_z, sxz_x, sxz_z);
    stv(vx + iv, ldv(vx + iv) + (sxx_x + sxz_z) * __ldg(f.p[PRIP] + ip));
    stv(vz + iv, ldv(vz + iv) + (szz_z + sxz_x) * __ldg(f.p[PRKP] + ip));
    if (g.abs_type == 2) {
        T *fs[2] = {vx, vz};
        apply_taper<2>(g, f.taper, gz, 0, gx, fs, iv);
    }
}

// one cell of the P-SV stress update (update_s2D.cl:30-327)
template <int F, class T = float>
__device__ __forceinline__ void s2d_cell(const Grid &g, const Fields &f, int gz, int gx)
{
    i64 ip = (i64)(gx - F) * g.nz + (gz - F), iv = (i64)gx * g.NZ + gz;
    const float *hc = g.hc;
    T *wsxx = fld<T>(f.w[SXX]), *wszz = fld<T>(f.w[SZZ]), *wsxz = fld<T>(f.w[SXZ]);
    float vxx = dbwT<F>(fld<T>(f.w[VX]), iv, g.NZ, hc);
    float vxz = dfwT<F>(fld<T>(f.w[VX]), iv, 1, hc);
    float vzz = dbwT<F>(fld<T>(f.w[VZ]), iv, 1, hc);
    float vzx = dfwT<F>(fld<T>(f.w[VZ]), iv, g.NZ, hc);
    if (g.abs_type == 1) cpml_s2d(g, f, gz, gx, vxx, vxz, vzx, vzz);
    const int L = g.L;
    if (L == 0) {
        float fipkp = __ldg(f.p[PMUIPKP] + ip);
        float fm = 2.0f * __ldg(f.p[PMU] + ip);
        float gm = __ldg(f.p[PM] + ip);
        stv(wsxz + iv, ldv(wsxz + iv) + fipkp * (vxz + vzx));
        stv(wsxx + iv, ldv(wsxx + iv) + (gm * (vxx + vzz) - fm * vzz));
        stv(wszz + iv, ldv(wszz + iv) + (gm * (vxx + vzz) - fm * vxx));
    } else {
        float lM = __ldg(f.p[PM] + ip), lmu = __ldg(f.p[PMU] + ip), lmuipkp = __ldg(f.p[PMUIPKP] + ip);
        float ltaup = __ldg(f.p[PTAUP] + ip), ltaus = __ldg(f.p[PTAUS] + ip), ltausipkp = __ldg(f.p[PTAUSIPKP] + ip);
        float fipkp = lmuipkp * (1.0f + (float)L * ltausipkp);
        float gm = lM * (1.0f + (float)L * ltaup);
        float fm = 2.0f * lmu * (1.0f + (float)L * ltaus);
        float dipkp = lmuipkp * ltausipkp / g.dt;
        float d = 2.0f * lmu * ltaus / g.dt;
        float e = lM * ltaup / g.dt;
        T *rxx = fld<T>(f.r[RXX]), *rzz = fld<T>(f.r[RZZ]), *rxz = fld<T>(f.r[RXZ]);
        float sxz_ = 0, sxx_ = 0, szz_ = 0;
        for (int l = 0; l < L; l++) {
            i64 ir = l * g.nvol + iv;
            sxz_ += ldv(rxz + ir); sxx_ += ldv(rxx + ir); szz_ += ldv(rzz + ir);
        }
        float lsxz = fipkp * (vxz + vzx) + g.dt2 * sxz_;
        float lsxx = (gm * (vxx + vzz) - fm * vzz) + g.dt2 * sxx_;
        float lszz = (gm * (vxx + vzz) - fm * vxx) + g.dt2 * szz_;
        sxz_ = sxx_ = szz_ = 0;
        for (int l = 0; l < L; l++) {
            float el = g.eta[l];
            float b = 1.0f / (1.0f + el * 0.5f), c = 1.0f - el * 0.5f;
            i64 ir = l * g.nvol + iv;
            float a1 = b * (ldv(rxz + ir) * c - el * (dipkp * (vxz + vzx)));
            float a2 = b * (ldv(rxx + ir) * c - el * (e * (vxx + vzz) - d * vzz));
            float a3 = b * (ldv(rzz + ir) * c - el * (e * (vxx + vzz) - d * vxx));
            stv(rxz + ir, a1); stv(rxx + ir, a2); stv(rzz + ir, a3);
            // the stored values (rounded to T) are what the next step reads;
            // the sums use the FP32 ones, as the FP32 build does
            sxz_ += a1; sxx_ += a2; szz_ += a3;
        }
        stv(wsxz + iv, ldv(wsxz + iv) + (lsxz + g.dt2 * sxz_));
        stv(wsxx + iv, ldv(wsxx + iv) + (lsxx + g.dt2 * sxx_));
        stv(wszz + iv, ldv(wszz + iv) + (lszz + g.dt2 * szz_));
    }
    if (g.abs_type == 2) {
        T *fs[3] = {wsxx, wszz, wsxz};
        apply_taper<3>(g, f.taper, gz, 0, gx, fs, iv);
    }
}

// free surface of one column (surface2D.cl:30-193)
template <int F, class T = float>
__device__ __forceinline__ void surf2d_column(const Grid &g, const Fields &f, int gx, int pdir)
{
    int gz = F, NZ = g.NZ, L = g.L, NAB = g.nab;
    i64 ip = (i64)(gx - F) * g.nz + (gz - F), iv = (i64)gx * NZ + gz;
    T *vx = fld<T>(f.w[VX]), *vz = fld<T>(f.w[VZ]), *sxx = fld<T>(f.w[SXX]), *szz = fld<T>(f.w[SZZ]),
      *sxz = fld<T>(f.w[SXZ]);
    T *rxx = fld<T>(f.r[RXX]), *rzz = fld<T>(f.r[RZZ]);
    stv(szz + iv, 0.0f);
    for (int l = 0; l < L; l++) stv(rzz + l * g.nvol + iv, 0.0f);
#pragma unroll
    for (int m = 1; m <= F; m++) {
        stv(szz + iv - m, -ldv(szz + iv + m));
        stv(sxz + iv - m, -ldv(sxz + iv + m - 1));
    }
    float vxx = dbw_rwT<F>(vx, iv, NZ, g.hc);
    float vzz = dbw_rwT<F>(vz, iv, 1, g.hc);
    if (g.abs_type == 1) {
        if (gx - F < NAB) {
            int i = gx - F;
            vxx = vxx / f.cx[CK][i] + f.psi[PVX_X][(i64)i * g.nz + (gz - F)];
        }
        if (gx > g.NX - NAB - F - 1) {
            int i = gx - g.NX + NAB + F + NAB, ind = 2 * NAB - 1 - i;
            vxx = vxx / f.cx[CK][ind + 1] + f.psi[PVX_X][(i64)i * g.nz + (gz - F)];
        }
    }
    if (L == 0) {
        float fm = f.p[PMU][ip] * 2.0f, gm = f.p[PM][ip];
        float h = -((gm - fm) * (gm - fm) * vxx / gm) - ((gm - fm) * vzz);
        stv(sxx + iv, ldv(sxx + iv) + pdir * h);
    } else {
        float taus = f.p[PTAUS][ip], taup = f.p[PTAUP][ip], mu = f.p[PMU][ip], M = f.p[PM][ip];
        float fm = mu * 2.0f * (1.0f + L * taus);
        float gm = M * (1.0f + L * taup);
        float h = -((gm - fm) * (gm - fm) * vxx / gm) - ((gm - fm) * vzz);
        float sump = 0;
        for (int l = 0; l < L; l++) sump += ldv(rxx + l * g.nvol + iv);
        h += -g.dt2 * sump;
        stv(sxx + iv, ldv(sxx + iv) + pdir * h);
        float d = 2.0f * mu * taus / g.dt, e = M * taup / g.dt;
        sump = 0;
        for (int l = 0; l < L; l++) {
            float b = g.eta[l] / (1.0f + g.eta[l] * 0.5f);
            float hh = b * (((d - e) * ((fm / gm) - 1.0f) * vxx) - ((d - e) * vzz));
            float r = ldv(rxx + l * g.nvol + iv) + pdir * hh;
            stv(rxx + l * g.nvol + iv, r);
            sump += r;
        }
        stv(sxx + iv, ldv(sxx + iv) + pdir * (g.dt2 * sump));
    }
}

// free surface, one thread per surface column
template <int F, class T = float>
__global__ void k_surf2d(Grid g, Fields f, int pdir)
{
    SHOT_F
    int gx = blockIdx.x * blockDim.x + threadIdx.x + F;
    if (gx <= g.NX - F - 1) surf2d_column<F, T>(g, f, gx, pdir);
}

template <int F, class T = float>
__global__ void __launch_bounds__(256) k_s2d(Grid g, Fields f)
{
    SHOT_F
    int gz = blockIdx.x * blockDim.x + threadIdx.x + F;
    int gx = blockIdx.y * blockDim.y + threadIdx.y + F;
    if (gz <= g.NZ - F - 1 && gx <= g.NX - F - 1) s2d_cell<F, T>(g, f, gz, gx);
}

// ===================================================================== 3D
__device__ __forceinline__ void cpml_v3d(const Grid &g, const Fields &f, int gz, int gy, int gx, float &sxx_x,
                                         float &syy_y, float &szz_z, float &sxy_y, float &sxy_x, float &syz_y,
                                         float &syz_z, float &sxz_x, float &sxz_z)
{
    int F = g.F, NAB = g.nab, NZ = g.NZ, NY = g.NY, NX = g.NX;
    i64 nz = g.nz, ny = g.ny;
    if (gz > NZ - NAB - F - 1) {
        i64 i = gx - F, j = gy - F, k = gz - NZ + NAB + F + NAB;
        int ind = 2 * NAB - 1 - (int)k;
        i64 q = (i * ny + j) * (2 * NAB) + k;
        cpml(f.psi[PSXZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], ind + 1, sxz_z);
        cpml(f.psi[PSYZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], ind + 1, syz_z);
        cpml(f.psi[PSZZ_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, szz_z);
    } else if (!g.freesurf && gz - F < NAB) {
        i64 i = gx - F, j = gy - F, k = gz - F;
        i64 q = (i * ny + j) * (2 * NAB) + k;
        cpml(f.psi[PSXZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], (int)k, sxz_z);
        cpml(f.psi[PSYZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], (int)k, syz_z);
        cpml(f.psi[PSZZ_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], (int)k, szz_z);
    }
    if (gy - F < NAB) {
        i64 i = gx - F, j = gy - F, k = gz - F;
        i64 q = (i * (2 * NAB) + j) * nz + k;
        cpml(f.psi[PSXY_Y], q, f.cy[CK], f.cy[CA], f.cy[CB], (int)j, sxy_y);
        cpml(f.psi[PSYY_Y], q, f.cy[CKH], f.cy[CAH], f.cy[CBH], (int)j, syy_y);
        cpml(f.psi[PSYZ_Y], q, f.cy[CK], f.cy[CA], f.cy[CB], (int)j, syz_y);
    } else if (gy > NY - NAB - F - 1) {
        i64 i = gx - F, j = gy - NY + NAB + F + NAB, k = gz - F;
        int ind = 2 * NAB - 1 - (int)j;
        i64 q = (i * (2 * NAB) + j) * nz + k;
        cpml(f.psi[PSXY_Y], q, f.cy[CK], f.cy[CA], f.cy[CB], ind + 1, sxy_y);
        cpml(f.psi[PSYY_Y], q, f.cy[CKH], f.cy[CAH], f.cy[CBH], ind, syy_y);
        cpml(f.psi[PSYZ_Y], q, f.cy[CK], f.cy[CA], f.cy[CB], ind + 1, syz_y);
    }
    if (gx - F < NAB) {
        i64 i = gx - F, j = gy - F, k = gz - F;
        i64 q = (i * ny + j) * nz + k;
        cpml(f.psi[PSXX_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], (int)i, sxx_x);
        cpml(f.psi[PSXY_X], q, f.cx[CK], f.cx[CA], f.cx[CB], (int)i, sxy_x);
        cpml(f.psi[PSXZ_X], q, f.cx[CK], f.cx[CA], f.cx[CB], (int)i, sxz_x);
    }
    if (gx > NX - NAB - F - 1) {
        i64 i = gx - NX + NAB + F + NAB, j = gy - F, k = gz - F;
        int ind = 2 * NAB - 1 - (int)i;
        i64 q = (i * ny + j) * nz + k;
        cpml(f.psi[PSXX_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], ind, sxx_x);
        cpml(f.psi[PSXY_X], q, f.cx[CK], f.cx[CA], f.cx[CB], ind + 1, sxy_x);
        cpml(f.psi[PSXZ_X], q, f.cx[CK], f.cx[CA], f.cx[CB], ind + 1, sxz_x);
    }
}

// update_s3D.cl:190-298 (plain "if"s); the adjoint form uses "else if" for the
// z-top and y-far branches (update_adjs3D.cl)
__device__ __forceinline__ void cpml_s3d(const Grid &g, const Fields &f, int gz, int gy, int gx, float &vxx,
                                         float &vxy, float &vxz, float &vyx, float &vyy, float &vyz, float &vzx,
                                         float &vzy, float &vzz, bool adjoint_form)
{
    int F = g.F, NAB = g.nab, NZ = g.NZ, NY = g.NY, NX = g.NX;
    i64 nz = g.nz, ny = g.ny;
    bool zb = gz > NZ - NAB - F - 1;
    if (zb) {
        i64 i = gx - F, j = gy - F, k = gz - NZ + NAB + F + NAB;
        int ind = 2 * NAB - 1 - (int)k;
        i64 q = (i * ny + j) * (2 * NAB) + k;
        cpml(f.psi[PVX_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, vxz);
        cpml(f.psi[PVY_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, vyz);
        cpml(f.psi[PVZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], ind + 1, vzz);
    }
    if (!g.freesurf && gz - F < NAB && !(adjoint_form && zb)) {
        i64 i = gx - F, j = gy - F, k = gz - F;
        i64 q = (i * ny + j) * (2 * NAB) + k;
        cpml(f.psi[PVX_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], (int)k, vxz);
        cpml(f.psi[PVY_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], (int)k, vyz);
        cpml(f.psi[PVZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], (int)k, vzz);
    }
    bool yb = gy - F < NAB;
    if (yb) {
        i64 i = gx - F, j = gy - F, k = gz - F;
        i64 q = (i * (2 * NAB) + j) * nz + k;
        cpml(f.psi[PVX_Y], q, f.cy[CKH], f.cy[CAH], f.cy[CBH], (int)j, vxy);
        cpml(f.psi[PVY_Y], q, f.cy[CK], f.cy[CA], f.cy[CB], (int)j, vyy);
        cpml(f.psi[PVZ_Y], q, f.cy[CKH], f.cy[CAH], f.cy[CBH], (int)j, vzy);
    }
    if (gy > NY - NAB - F - 1 && !(adjoint_form && yb)) {
        i64 i = gx - F, j = gy - NY + NAB + F + NAB, k = gz - F;
        int ind = 2 * NAB - 1 - (int)j;
        i64 q = (i * (2 * NAB) + j) * nz + k;
        cpml(f.psi[PVX_Y], q, f.cy[CKH], f.cy[CAH], f.cy[CBH], ind, vxy);
        cpml(f.psi[PVY_Y], q, f.cy[CK], f.cy[CA], f.cy[CB], ind + 1, vyy);
        cpml(f.psi[PVZ_Y], q, f.cy[CKH], f.cy[CAH], f.cy[CBH], ind, vzy);
    }
    if (gx - F < NAB) {
        i64 i = gx - F, j = gy - F, k = gz - F;
        i64 q = (i * ny + j) * nz + k;
        cpml(f.psi[PVX_X], q, f.cx[CK], f.cx[CA], f.cx[CB], (int)i, vxx);
        cpml(f.psi[PVY_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], (int)i, vyx);
        cpml(f.psi[PVZ_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], (int)i, vzx);
    }
    if (gx > NX - NAB - F - 1) {
        i64 i = gx - NX + NAB + F + NAB, j = gy - F, k = gz - F;
        int ind = 2 * NAB - 1 - (int)i;
        i64 q = (i * ny + j) * nz + k;
        cpml(f.psi[PVX_X], q, f.cx[CK], f.cx[CA], f.cx[CB], ind + 1, vxx);
        cpml(f.psi[PVY_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], ind, vyx);
        cpml(f.psi[PVZ_X], q, f.cx[CKH], f.cx[CAH], f.cx[CBH], ind, vzx);
    }
}

// grid z: the x blocks of each shot of the launch, shot after shot
#define SHOT3D                                                                         \
    int shot = 0, xb_ = blockIdx.z;                                                    \
    if (MB) {                                                                          \
        const int nxb_ = gridDim.z / g.nb;                                             \
        shot = blockIdx.z / nxb_;                                                      \
        xb_ = blockIdx.z - shot * nxb_;                                                \
    }
#define CELL3D                                                                         \
    SHOT3D                                                                             \
    int gz = blockIdx.x * blockDim.x + threadIdx.x + F;                                \
    int gy = blockIdx.y * blockDim.y + threadIdx.y + F;                                \
    int gx = xb_ * blockDim.z + threadIdx.z + F;                                       \
    if (gz > g.NZ - F - 1 || gy > g.NY - F - 1 || gx > g.NX - F - 1) return;           \
    if (MB) shot_fields(g, f, shot);                                                   \
    const i64 sx = (i64)g.NY * g.NZ, sy = g.NZ;                                        \
    i64 iv = gx * sx + (i64)gy * sy + gz;                                              \
    i64 ip = ((i64)(gx - F) * g.ny + (gy - F)) * g.nz + (gz - F);

template <int F, bool MB = false>
__global__ void __launch_bounds__(256) k_v3d(Grid g, Fields f)
{
    CELL3D
    const float *hc = g.hc;
    float szz_z = dfw<F>(f.w[SZZ], iv, 1, hc);
    float sxx_x = dfw<F>(f.w[SXX], iv, sx, hc);
    float sxz_x = dbw<F>(f.w[SXZ], iv, sx, hc);
    float sxz_z = dbw<F>(f.w[SXZ], iv, 1, hc);
    float syz_y = dbw<F>(f.w[SYZ], iv, sy, hc);
    float syz_z = dbw<F>(f.w[SYZ], iv, 1, hc);
    float syy_y = dfw<F>(f.w[SYY], iv, sy, hc);
    float sxy_x = dbw<F>(f.w[SXY], iv, sx, hc);
    float sxy_y = dbw<F>(f.w[SXY], iv, sy, hc);
    if (g.abs_type == 1) cpml_v3d(g, f, gz, gy, gx, sxx_x, syy_y, szz_z, sxy_y, sxy_x, syz_y, syz_z, sxz_x, sxz_z);
    f.w[VX][iv] += (sxx_x + sxy_y + sxz_z) * __ldg(f.p[PRIP] + ip);
    f.w[VY][iv] += (syy_y + sxy_x + syz_z) * __ldg(f.p[PRJP] + ip);
    f.w[VZ][iv] += (szz_z + sxz_x + syz_y) * __ldg(f.p[PRKP] + ip);
    if (g.abs_type == 2) {
        float *fs[3] = {f.w[VX], f.w[VY], f.w[VZ]};
        apply_taper<3>(g, f.taper, gz, gy, gx, fs, iv);
    }
}

template <int F, bool MB = false>
__global__ void __launch_bounds__(256) k_s3d(Grid g, Fields f)
{
    CELL3D
    const float *hc = g.hc;
    float vzx = dfw<F>(f.w[VZ], iv, sx, hc), vzy = dfw<F>(f.w[VZ], iv, sy, hc), vzz = dbw<F>(f.w[VZ], iv, 1, hc);
    float vyx = dfw<F>(f.w[VY], iv, sx, hc), vyy = dbw<F>(f.w[VY], iv, sy, hc), vyz = dfw<F>(f.w[VY], iv, 1, hc);
    float vxx = dbw<F>(f.w[VX], iv, sx, hc), vxy = dfw<F>(f.w[VX], iv, sy, hc), vxz = dfw<F>(f.w[VX], iv, 1, hc);
    if (g.abs_type == 1) cpml_s3d(g, f, gz, gy, gx, vxx, vxy, vxz, vyx, vyy, vyz, vzx, vzy, vzz, false);
    float vxyyx = vxy + vyx, vyzzy = vyz + vzy, vxzzx = vxz + vzx;
    float vxxyyzz = vxx + vyy + vzz, vyyzz = vyy + vzz, vxxzz = vxx + vzz, vxxyy = vxx + vyy;
    const int L = g.L;
    if (L == 0) {
        float fipjp = __ldg(f.p[PMUIPJP] + ip), fjpkp = __ldg(f.p[PMUJPKP] + ip), fipkp = __ldg(f.p[PMUIPKP] + ip);
        float gm = __ldg(f.p[PM] + ip), fm = 2.0f * __ldg(f.p[PMU] + ip);
        f.w[SXY][iv] += fipjp * vxyyx;
        f.w[SYZ][iv] += fjpkp * vyzzy;
        f.w[SXZ][iv] += fipkp * vxzzx;
        f.w[SXX][iv] += gm * vxxyyzz - fm * vyyzz;
        f.w[SYY][iv] += gm * vxxyyzz - fm * vxxzz;
        f.w[SZZ][iv] += gm * vxxyyzz - fm * vxxyy;
    } else {
        float lM = __ldg(f.p[PM] + ip), lmu = __ldg(f.p[PMU] + ip);
        float lmuipkp = __ldg(f.p[PMUIPKP] + ip), lmuipjp = __ldg(f.p[PMUIPJP] + ip), lmujpkp = __ldg(f.p[PMUJPKP] + ip);
        float ltaup = __ldg(f.p[PTAUP] + ip), ltaus = __ldg(f.p[PTAUS] + ip);
        float ltausipkp = __ldg(f.p[PTAUSIPKP] + ip), ltausipjp = __ldg(f.p[PTAUSIPJP] + ip),
              ltausjpkp = __ldg(f.p[PTAUSJPKP] + ip);
        float fipjp = lmuipjp * (1.0f + (float)L * ltausipjp);
        float fjpkp = lmujpkp * (1.0f + (float)L * ltausjpkp);
        float fipkp = lmuipkp * (1.0f + (float)L * ltausipkp);
        float gm = lM * (1.0f + (float)L * ltaup);
        float fm = 2.0f * lmu * (1.0f + (float)L * ltaus);
        float dipjp = lmuipjp * ltausipjp / g.dt, djpkp = lmujpkp * ltausjpkp / g.dt, dipkp = lmuipkp * ltausipkp / g.dt;
        float d = 2.0f * lmu * ltaus / g.dt, e = lM * ltaup / g.dt;
        float a[6] = {0, 0, 0, 0, 0, 0};
        float *const *r = f.r;
        for (int l = 0; l < L; l++) {
            i64 ir = l * g.nvol + iv;
            a[0] += r[RXY][ir]; a[1] += r[RYZ][ir]; a[2] += r[RXZ][ir];
            a[3] += r[RXX][ir]; a[4] += r[RYY][ir]; a[5] += r[RZZ][ir];
        }
        float lsxy = fipjp * vxyyx + g.dt2 * a[0];
        float lsyz = fjpkp * vyzzy + g.dt2 * a[1];
        float lsxz = fipkp * vxzzx + g.dt2 * a[2];
        float lsxx = (gm * vxxyyzz - fm * vyyzz) + g.dt2 * a[3];
        float lsyy = (gm * vxxyyzz - fm * vxxzz) + g.dt2 * a[4];
        float lszz = (gm * vxxyyzz - fm * vxxyy) + g.dt2 * a[5];
        for (int q = 0; q < 6; q++) a[q] = 0;
        for (int l = 0; l < L; l++) {
            float el = g.eta[l];
            float b = 1.0f / (1.0f + el * 0.5f), c = 1.0f - el * 0.5f;
            i64 ir = l * g.nvol + iv;
            float n0 = b * (r[RXY][ir] * c - el * (dipjp * vxyyx));
            float n1 = b * (r[RYZ][ir] * c - el * (djpkp * vyzzy));
            float n2 = b * (r[RXZ][ir] * c - el * (dipkp * vxzzx));
            float n3 = b * (r[RXX][ir] * c - el * (e * vxxyyzz - d * vyyzz));
            float n4 = b * (r[RYY][ir] * c - el * (e * vxxyyzz - d * vxxzz));
            float n5 = b * (r[RZZ][ir] * c - el * (e * vxxyyzz - d * vxxyy));
            r[RXY][ir] = n0; r[RYZ][ir] = n1; r[RXZ][ir] = n2; r[RXX][ir] = n3; r[RYY][ir] = n4; r[RZZ][ir] = n5;
            a[0] += n0; a[1] += n1; a[2] += n2; a[3] += n3; a[4] += n4; a[5] += n5;
        }
        f.w[SXY][iv] += lsxy + g.dt2 * a[0];
        f.w[SYZ][iv] += lsyz + g.dt2 * a[1];
        f.w[SXZ][iv] += lsxz + g.dt2 * a[2];
        f.w[SXX][iv] += lsxx + g.dt2 * a[3];
        f.w[SYY][iv] += lsyy + g.dt2 * a[4];
        f.w[SZZ][iv] += lszz + g.dt2 * a[5];
    }
    if (g.abs_type == 2) {
        float *fs[6] = {f.w[SXY], f.w[SYZ], f.w[SXZ], f.w[SXX], f.w[SYY], f.w[SZZ]};
        apply_taper<6>(g, f.taper, gz, gy, gx, fs, iv);
    }
}

// ----------------------------------------------------- streaming 3D kernels
// Same arithmetic as k_v3d / k_s3d, one thread per cell, but every per-cell
// stream (the updated fields, memory variables and parameters) is loaded
// into registers before the stencil work starts, so each thread has all of
// its independent DRAM loads in flight at once; the updated values are
// stored once at the end (taper applied in registers, in the reference's
// factor order).  L is a template parameter so the memory variables stay in
// registers.  The stencil taps go through the read-only cache as in the
// general kernels.
template <int NF>
__device__ __forceinline__ void taper_regs(const Grid &g, const float *taper, int gz, int gy, int gx, float (&v)[NF])
{
    const int F = g.F, NAB = g.nab;
    auto mul = [&](float t) {
#pragma unroll
        for (int q = 0; q < NF; q++) v[q] *= t;
    };
    if (!g.freesurf && gz - F < NAB) mul(__ldg(taper + gz - F));
    if (gz > g.NZ - NAB - F - 1) mul(__ldg(taper + g.NZ - F - gz - 1));
    if (gy - F < NAB) mul(__ldg(taper + gy - F));
    if (gy > g.NY - NAB - F - 1) mul(__ldg(taper + g.NY - F - gy - 1));
    if (gx - F < NAB) mul(__ldg(taper + gx - F));
    if (gx > g.NX - NAB - F - 1) mul(__ldg(taper + g.NX - F - gx - 1));
}

template <int F, class T = float, bool MB = false>
__global__ void __launch_bounds__(256, 3) k_v3d_stream(Grid g, Fields f)
{
    CELL3D
    const float *hc = g.hc;
    T *wvx = fld<T>(f.w[VX]), *wvy = fld<T>(f.w[VY]), *wvz = fld<T>(f.w[VZ]);
    float v[3] = {ldgv(wvx + iv), ldgv(wvy + iv), ldgv(wvz + iv)};
    const float rip = __ldg(f.p[PRIP] + ip), rjp = __ldg(f.p[PRJP] + ip), rkp = __ldg(f.p[PRKP] + ip);
    const T *Sxx = fld<T>(f.w[SXX]), *Syy = fld<T>(f.w[SYY]), *Szz = fld<T>(f.w[SZZ]);
    const T *Sxy = fld<T>(f.w[SXY]), *Syz = fld<T>(f.w[SYZ]), *Sxz = fld<T>(f.w[SXZ]);
    float szz_z = dfwT<F>(Szz, iv, 1, hc);
    float sxx_x = dfwT<F>(Sxx, iv, sx, hc);
    float sxz_x = dbwT<F>(Sxz, iv, sx, hc);
    float sxz_z = dbwT<F>(Sxz, iv, 1, hc);
    float syz_y = dbwT<F>(Syz, iv, sy, hc);
    float syz_z = dbwT<F>(Syz, iv, 1, hc);
    float syy_y = dfwT<F>(Syy, iv, sy, hc);
    float sxy_x = dbwT<F>(Sxy, iv, sx, hc);
    float sxy_y = dbwT<F>(Sxy, iv, sy, hc);
    if (g.abs_type == 1) cpml_v3d(g, f, gz, gy, gx, sxx_x, syy_y, szz_z, sxy_y, sxy_x, syz_y, syz_z, sxz_x, sxz_z);
    v[0] += (sxx_x + sxy_y + sxz_z) * rip;
    v[1] += (syy_y + sxy_x + syz_z) * rjp;
    v[2] += (szz_z + sxz_x + syz_y) * rkp;
    if (g.abs_type == 2) taper_regs<3>(g, f.taper, gz, gy, gx, v);
    stv(wvx + iv, v[0]);
    stv(wvy + iv, v[1]);
    stv(wvz + iv, v[2]);
}

// ------------------------------------------------- 4-cell vectorised 3D kernels
// One thread updates four consecutive z cells with 128-bit loads and stores:
// the per-cell streams cost one load per four cells, a z derivative one
// 12-value window (three loads) for four cells, and an x or y derivative one
// load per tap for four cells -- about a fifth of the load instructions of
// the one-cell kernels, which are bound by load issue and latency, not by
// DRAM bytes.  Requires 8th order (F = 4, so the interior starts on a 16-byte
// boundary) and nz % 4 == 0 (so NZ = nz + 8 keeps every row aligned).  Same
// operation order per cell as k_v3d.
struct Q4 {
    float v[4];
};
__device__ __forceinline__ Q4 ldq(const float *p)
{
    float4 t = __ldg(reinterpret_cast<const float4 *>(p));
    return Q4{{t.x, t.y, t.z, t.w}};
}
__device__ __forceinline__ Q4 ldq_rw(const float *p)
{
    float4 t = *reinterpret_cast<const float4 *>(p);
    return Q4{{t.x, t.y, t.z, t.w}};
}
__device__ __forceinline__ void stq(float *p, const Q4 &q)
{
    *reinterpret_cast<float4 *>(p) = make_float4(q.v[0], q.v[1], q.v[2], q.v[3]);
}
// FP16 storage: four halves move as one 64-bit access
__device__ __forceinline__ Q4 q4_of(uint2 u)
{
    const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&u.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2 *>(&u.y));
    return Q4{{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ Q4 ldq(const __half *p) { return q4_of(__ldg(reinterpret_cast<const uint2 *>(p))); }
__device__ __forceinline__ Q4 ldq_rw(const __half *p) { return q4_of(*reinterpret_cast<const uint2 *>(p)); }
__device__ __forceinline__ void stq(__half *p, const Q4 &q)
{
    const __half2 a = __floats2half2_rn(q.v[0], q.v[1]), b = __floats2half2_rn(q.v[2], q.v[3]);
    uint2 u;
    u.x = *reinterpret_cast<const unsigned *>(&a);
    u.y = *reinterpret_cast<const unsigned *>(&b);
    *reinterpret_cast<uint2 *>(p) = u;
}
// Load policy of the stencil reads (template parameter LP): 0 the read-only
// path (__ldg; arrays no thread writes during the launch), 1 a plain global
// load (arrays that other CTAs write later in the same launch, read before
// they do), 2 L2 only (__ldcg: values other CTAs wrote earlier in the same
// launch, which a stale L1 line must not hide).
template <int LP>
__device__ __forceinline__ Q4 ldq_p(const float *p)
{
    float4 t;
    if constexpr (LP == 0) t = __ldg(reinterpret_cast<const float4 *>(p));
    else if constexpr (LP == 1) t = *reinterpret_cast<const float4 *>(p);
    else t = __ldcg(reinterpret_cast<const float4 *>(p));
    return Q4{{t.x, t.y, t.z, t.w}};
}
template <int LP>
__device__ __forceinline__ Q4 ldq_p(const __half *p)
{
    static_assert(LP == 0 || LP == 1, "FP16 fields are read through the read-only path or plainly");
    if constexpr (LP == 0) return ldq(p);
    else return ldq_rw(p);
}

// memory variables of four cells in storage type TR: with TR FP16 under
// FP32 wave fields (Grid::rhalf) they are stored times g.rsc
template <class T, class TR>
__device__ __forceinline__ Q4 ldr_q(const Grid &g, const TR *p)
{
    Q4 r = ldq_rw(p);
    if constexpr (!std::is_same<T, TR>::value) {
#pragma unroll
        for (int j = 0; j < 4; j++) r.v[j] *= g.rsci;
    }
    return r;
}
template <class T, class TR>
__device__ __forceinline__ void str_q(const Grid &g, TR *p, const Q4 &q)
{
    if constexpr (!std::is_same<T, TR>::value) {
        Q4 r;
#pragma unroll
        for (int j = 0; j < 4; j++) r.v[j] = q.v[j] * g.rsc;
        stq(p, r);
    } else {
        stq(p, q);
    }
}

// forward / backward differences of four cells along a stride (x or y)
template <int F, class T, int LP = 0>
__device__ __forceinline__ Q4 dfw_q(const T *__restrict__ v, i64 i, i64 st, const float *hc)
{
    Q4 a = ldq_p<LP>(v + i + st), b = ldq_p<LP>(v + i), r;
#pragma unroll
    for (int j = 0; j < 4; j++) r.v[j] = hc[0] * (a.v[j] - b.v[j]);
#pragma unroll
    for (int m = 2; m <= F; m++) {
        a = ldq_p<LP>(v + i + m * st);
        b = ldq_p<LP>(v + i - (m - 1) * st);
#pragma unroll
        for (int j = 0; j < 4; j++) r.v[j] = fmaf(hc[m - 1], a.v[j] - b.v[j], r.v[j]);
    }
    return r;
}
template <int F, class T, int LP = 0>
__device__ __forceinline__ Q4 dbw_q(const T *__restrict__ v, i64 i, i64 st, const float *hc)
{
    Q4 a = ldq_p<LP>(v + i), b = ldq_p<LP>(v + i - st), r;
#pragma unroll
    for (int j = 0; j < 4; j++) r.v[j] = hc[0] * (a.v[j] - b.v[j]);
#pragma unroll
    for (int m = 2; m <= F; m++) {
        a = ldq_p<LP>(v + i + (m - 1) * st);
        b = ldq_p<LP>(v + i - m * st);
#pragma unroll
        for (int j = 0; j < 4; j++) r.v[j] = fmaf(hc[m - 1], a.v[j] - b.v[j], r.v[j]);
    }
    return r;
}
// the 12 values z0-4 .. z0+7 around four cells starting at z0 (a multiple of 4)
struct W12 {
    float w[12];
};
template <class T, int LP = 0>
__device__ __forceinline__ W12 ldw(const T *__restrict__ v, i64 i)
{
    W12 r;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const Q4 t = ldq_p<LP>(v + i - 4 + 4 * k);
        r.w[4 * k] = t.v[0]; r.w[4 * k + 1] = t.v[1]; r.w[4 * k + 2] = t.v[2]; r.w[4 * k + 3] = t.v[3];
    }
    return r;
}
template <int F>
__device__ __forceinline__ Q4 dfw_z(const W12 &w, const float *hc)
{
    Q4 r;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        float acc = hc[0] * (w.w[5 + j] - w.w[4 + j]);
#pragma unroll
        for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], w.w[4 + j + m] - w.w[4 + j - (m - 1)], acc);
        r.v[j] = acc;
    }
    return r;
}
template <int F>
__device__ __forceinline__ Q4 dbw_z(const W12 &w, const float *hc)
{
    Q4 r;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        float acc = hc[0] * (w.w[4 + j] - w.w[3 + j]);
#pragma unroll
        for (int m = 2; m <= F; m++) acc = fmaf(hc[m - 1], w.w[4 + j + m - 1] - w.w[4 + j - m], acc);
        r.v[j] = acc;
    }
    return r;
}

// CPML recursion on four consecutive z cells sharing one profile index
// (y and x slabs: the psi arrays are z-fastest and 16-byte aligned there).
// cpml()'s recursion, with the division by K replaced by a multiplication by
// 1/K (Fields::kinv, rounded to FP32 on the host): within one rounding of
// the quotient per cell, and cheaper -- the FP32 divisions had cost the
// velocity update at 256^3 with 20-cell slabs 0.031 ms of its 0.306.
__device__ __forceinline__ void cpml_q(float *psi, i64 q, const float *Ki, const float *a, const float *b, int ci,
                                       Q4 &d)
{
    const float ki = __ldg(Ki + ci), aa = __ldg(a + ci), bb = __ldg(b + ci);
    Q4 p = ldq_rw(psi + q);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        float ps = bb * p.v[j] + aa * d.v[j];
        p.v[j] = ps;
        d.v[j] = d.v[j] * ki + ps;
    }
    stq(psi + q, p);
}

// z-slab CPML on a quad that lies entirely inside the slab: the psi cells
// are consecutive (z-type psi is [nx][ny][2 nab], k fastest), the profile
// index differs per cell (ci0 + step * j); multiplies by 1/K as cpml_q
__device__ __forceinline__ void cpml_zq(float *psi, i64 q, const float *Ki, const float *a, const float *b, int ci0,
                                        int step, Q4 &d)
{
    Q4 p = ldq_rw(psi + q);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int ci = ci0 + step * j;
        float ps = __ldg(b + ci) * p.v[j] + __ldg(a + ci) * d.v[j];
        p.v[j] = ps;
        d.v[j] = d.v[j] * __ldg(Ki + ci) + ps;
    }
    stq(psi + q, p);
}

// Grids whose absorbing slabs cannot overlap (every axis at least 2 nab
// cells, the z axis 2 nab + 4) with nab % 4 == 0: a cell lies in at most one
// slab per axis and a z quad lies wholly inside or outside a z slab, so each
// axis takes one path, its side picked by selects.  The general forms below
// follow the reference's branch structure, which small grids need.
__device__ __forceinline__ bool cpml_slabs_apart(const Grid &g)
{
    return g.nab % 4 == 0 && g.nz >= 2 * g.nab + 4 && g.ny >= 2 * g.nab && g.nx >= 2 * g.nab;
}

// The CPML corrections of cpml_v3d for a quad of z cells: z slabs per cell
// (a quad may straddle a z-slab edge), y and x slabs per quad.
__device__ __forceinline__ void cpml_v3d_q4(const Grid &g, const Fields &f, int gz0, int gy, int gx, Q4 &sxx_x,
                                            Q4 &syy_y, Q4 &szz_z, Q4 &sxy_y, Q4 &sxy_x, Q4 &syz_y, Q4 &syz_z,
                                            Q4 &sxz_x, Q4 &sxz_z)
{
    const int F = g.F, NAB = g.nab, NZ = g.NZ, NY = g.NY, NX = g.NX;
    const i64 nz = g.nz, ny = g.ny;
    if (cpml_slabs_apart(g)) {
        // side-merged form: far-side profile indices are 2 nab - k (integer
        // grid) and 2 nab - 1 - k (half grid) of the slab-local index k
        const i64 k0 = gz0 - F;
        const bool zhi = gz0 > NZ - NAB - F - 1, zlo = !g.freesurf && gz0 - F < NAB;
        if (zhi || zlo) {
            const int k = zhi ? gz0 - NZ + 2 * NAB + F : gz0 - F;
            const int st = zhi ? -1 : 1, cf = zhi ? 2 * NAB - k : k, ch = zhi ? 2 * NAB - 1 - k : k;
            const i64 q = ((i64)(gx - F) * ny + (gy - F)) * (2 * NAB) + k;
            cpml_zq(f.psi[PSXZ_Z], q, f.kinv[2][0], f.cz[CA], f.cz[CB], cf, st, sxz_z);
            cpml_zq(f.psi[PSYZ_Z], q, f.kinv[2][0], f.cz[CA], f.cz[CB], cf, st, syz_z);
            cpml_zq(f.psi[PSZZ_Z], q, f.kinv[2][1], f.cz[CAH], f.cz[CBH], ch, st, szz_z);
        }
        const bool ylo = gy - F < NAB, yhi = gy > NY - NAB - F - 1;
        if (ylo || yhi) {
            const int j = ylo ? gy - F : gy - NY + 2 * NAB + F;
            const int cf = ylo ? j : 2 * NAB - j, ch = ylo ? j : 2 * NAB - 1 - j;
            const i64 q = ((i64)(gx - F) * (2 * NAB) + j) * nz + k0;
            cpml_q(f.psi[PSXY_Y], q, f.kinv[1][0], f.cy[CA], f.cy[CB], cf, sxy_y);
            cpml_q(f.psi[PSYY_Y], q, f.kinv[1][1], f.cy[CAH], f.cy[CBH], ch, syy_y);
            cpml_q(f.psi[PSYZ_Y], q, f.kinv[1][0], f.cy[CA], f.cy[CB], cf, syz_y);
        }
        const bool xlo = gx - F < NAB, xhi = gx > NX - NAB - F - 1;
        if (xlo || xhi) {
            const int i = xlo ? gx - F : gx - NX + 2 * NAB + F;
            const int cf = xlo ? i : 2 * NAB - i, ch = xlo ? i : 2 * NAB - 1 - i;
            const i64 q = ((i64)i * ny + (gy - F)) * nz + k0;
            cpml_q(f.psi[PSXX_X], q, f.kinv[0][1], f.cx[CAH], f.cx[CBH], ch, sxx_x);
            cpml_q(f.psi[PSXY_X], q, f.kinv[0][0], f.cx[CA], f.cx[CB], cf, sxy_x);
            cpml_q(f.psi[PSXZ_X], q, f.kinv[0][0], f.cx[CA], f.cx[CB], cf, sxz_x);
        }
        return;
    }
    if (NAB % 4 == 0 && gz0 > NZ - NAB - F - 1) {
        i64 i = gx - F, jj = gy - F, k = gz0 - NZ + NAB + F + NAB;
        int ind = 2 * NAB - 1 - (int)k;
        i64 q = (i * ny + jj) * (2 * NAB) + k;
        cpml_zq(f.psi[PSXZ_Z], q, f.kinv[2][0], f.cz[CA], f.cz[CB], ind + 1, -1, sxz_z);
        cpml_zq(f.psi[PSYZ_Z], q, f.kinv[2][0], f.cz[CA], f.cz[CB], ind + 1, -1, syz_z);
        cpml_zq(f.psi[PSZZ_Z], q, f.kinv[2][1], f.cz[CAH], f.cz[CBH], ind, -1, szz_z);
    } else if (NAB % 4 == 0 && !g.freesurf && gz0 - F < NAB) {
        i64 i = gx - F, jj = gy - F, k = gz0 - F;
        i64 q = (i * ny + jj) * (2 * NAB) + k;
        cpml_zq(f.psi[PSXZ_Z], q, f.kinv[2][0], f.cz[CA], f.cz[CB], (int)k, 1, sxz_z);
        cpml_zq(f.psi[PSYZ_Z], q, f.kinv[2][0], f.cz[CA], f.cz[CB], (int)k, 1, syz_z);
        cpml_zq(f.psi[PSZZ_Z], q, f.kinv[2][1], f.cz[CAH], f.cz[CBH], (int)k, 1, szz_z);
    } else if (NAB % 4 != 0 && (gz0 + 3 > NZ - NAB - F - 1 || (!g.freesurf && gz0 - F < NAB))) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int gz = gz0 + j;
            if (gz > NZ - NAB - F - 1) {
                i64 i = gx - F, jj = gy - F, k = gz - NZ + NAB + F + NAB;
                int ind = 2 * NAB - 1 - (int)k;
                i64 q = (i * ny + jj) * (2 * NAB) + k;
                cpml(f.psi[PSXZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], ind + 1, sxz_z.v[j]);
                cpml(f.psi[PSYZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], ind + 1, syz_z.v[j]);
                cpml(f.psi[PSZZ_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, szz_z.v[j]);
            } else if (!g.freesurf && gz - F < NAB) {
                i64 i = gx - F, jj = gy - F, k = gz - F;
                i64 q = (i * ny + jj) * (2 * NAB) + k;
                cpml(f.psi[PSXZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], (int)k, sxz_z.v[j]);
                cpml(f.psi[PSYZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], (int)k, syz_z.v[j]);
                cpml(f.psi[PSZZ_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], (int)k, szz_z.v[j]);
            }
        }
    }
    const i64 k0 = gz0 - F;
    if (gy - F < NAB) {
        i64 i = gx - F, j = gy - F;
        i64 q = (i * (2 * NAB) + j) * nz + k0;
        cpml_q(f.psi[PSXY_Y], q, f.kinv[1][0], f.cy[CA], f.cy[CB], (int)j, sxy_y);
        cpml_q(f.psi[PSYY_Y], q, f.kinv[1][1], f.cy[CAH], f.cy[CBH], (int)j, syy_y);
        cpml_q(f.psi[PSYZ_Y], q, f.kinv[1][0], f.cy[CA], f.cy[CB], (int)j, syz_y);
    } else if (gy > NY - NAB - F - 1) {
        i64 i = gx - F, j = gy - NY + NAB + F + NAB;
        int ind = 2 * NAB - 1 - (int)j;
        i64 q = (i * (2 * NAB) + j) * nz + k0;
        cpml_q(f.psi[PSXY_Y], q, f.kinv[1][0], f.cy[CA], f.cy[CB], ind + 1, sxy_y);
        cpml_q(f.psi[PSYY_Y], q, f.kinv[1][1], f.cy[CAH], f.cy[CBH], ind, syy_y);
        cpml_q(f.psi[PSYZ_Y], q, f.kinv[1][0], f.cy[CA], f.cy[CB], ind + 1, syz_y);
    }
    if (gx - F < NAB) {
        i64 i = gx - F, j = gy - F;
        i64 q = (i * ny + j) * nz + k0;
        cpml_q(f.psi[PSXX_X], q, f.kinv[0][1], f.cx[CAH], f.cx[CBH], (int)i, sxx_x);
        cpml_q(f.psi[PSXY_X], q, f.kinv[0][0], f.cx[CA], f.cx[CB], (int)i, sxy_x);
        cpml_q(f.psi[PSXZ_X], q, f.kinv[0][0], f.cx[CA], f.cx[CB], (int)i, sxz_x);
    }
    if (gx > NX - NAB - F - 1) {
        i64 i = gx - NX + NAB + F + NAB, j = gy - F;
        int ind = 2 * NAB - 1 - (int)i;
        i64 q = (i * ny + j) * nz + k0;
        cpml_q(f.psi[PSXX_X], q, f.kinv[0][1], f.cx[CAH], f.cx[CBH], ind, sxx_x);
        cpml_q(f.psi[PSXY_X], q, f.kinv[0][0], f.cx[CA], f.cx[CB], ind + 1, sxy_x);
        cpml_q(f.psi[PSXZ_X], q, f.kinv[0][0], f.cx[CA], f.cx[CB], ind + 1, sxz_x);
    }
}

// MB (a template parameter of the kernel): the launch covers several shots
#define CELL3D_Q4                                                                      \
    constexpr int F = 4;                                                               \
    int shot = 0, xb_ = blockIdx.z;                                                    \
    if (MB) {                                                                          \
        const int nxb_ = gridDim.z / g.nb;                                             \
        shot = blockIdx.z / nxb_;                                                      \
        xb_ = blockIdx.z - shot * nxb_;                                                \
    }                                                                                  \
    const int gz0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4 + F;                   \
    const int gy = blockIdx.y * blockDim.y + threadIdx.y + F;                          \
    const int gx = xb_ * blockDim.z + threadIdx.z + F;                                 \
    if (gz0 > g.NZ - F - 1 || gy > g.NY - F - 1 || gx > g.NX - F - 1) return;          \
    if (MB) shot_fields(g, f, shot);                                                   \
    const i64 sx = (i64)g.NY * g.NZ, sy = g.NZ;                                        \
    const i64 iv = gx * sx + (i64)gy * sy + gz0;                                       \
    const i64 ip = ((i64)(gx - F) * g.ny + (gy - F)) * g.nz + (gz0 - F);

// velocity update of the quad (gz0..gz0+3, gy, gx); LP: load policy of the
// stress reads
template <class T, int LP = 0>
__device__ __forceinline__ void v3d_q4_at(const Grid &g, const Fields &f, int gz0, int gy, int gx, i64 iv, i64 ip)
{
    constexpr int F = 4;
    const i64 sx = (i64)g.NY * g.NZ, sy = g.NZ;
    const float *hc = g.hc;
    T *wvx = fld<T>(f.w[VX]), *wvy = fld<T>(f.w[VY]), *wvz = fld<T>(f.w[VZ]);
    const T *Sxx = fld<T>(f.w[SXX]), *Syy = fld<T>(f.w[SYY]), *Szz = fld<T>(f.w[SZZ]);
    const T *Sxy = fld<T>(f.w[SXY]), *Syz = fld<T>(f.w[SYZ]), *Sxz = fld<T>(f.w[SXZ]);
    Q4 vx = ldq_rw(wvx + iv), vy = ldq_rw(wvy + iv), vz = ldq_rw(wvz + iv);
    const Q4 rip = ldq(f.p[PRIP] + ip), rjp = ldq(f.p[PRJP] + ip), rkp = ldq(f.p[PRKP] + ip);
    const W12 wzz = ldw<T, LP>(Szz, iv), wxz = ldw<T, LP>(Sxz, iv), wyz = ldw<T, LP>(Syz, iv);
    Q4 szz_z = dfw_z<F>(wzz, hc);
    Q4 sxx_x = dfw_q<F, T, LP>(Sxx, iv, sx, hc);
    Q4 sxz_x = dbw_q<F, T, LP>(Sxz, iv, sx, hc);
    Q4 sxz_z = dbw_z<F>(wxz, hc);
    Q4 syz_y = dbw_q<F, T, LP>(Syz, iv, sy, hc);
    Q4 syz_z = dbw_z<F>(wyz, hc);
    Q4 syy_y = dfw_q<F, T, LP>(Syy, iv, sy, hc);
    Q4 sxy_x = dbw_q<F, T, LP>(Sxy, iv, sx, hc);
    Q4 sxy_y = dbw_q<F, T, LP>(Sxy, iv, sy, hc);
    if (g.abs_type == 1) cpml_v3d_q4(g, f, gz0, gy, gx, sxx_x, syy_y, szz_z, sxy_y, sxy_x, syz_y, syz_z, sxz_x, sxz_z);
#pragma unroll
    for (int j = 0; j < 4; j++) {
        float v3[3] = {vx.v[j] + (sxx_x.v[j] + sxy_y.v[j] + sxz_z.v[j]) * rip.v[j],
                       vy.v[j] + (syy_y.v[j] + sxy_x.v[j] + syz_z.v[j]) * rjp.v[j],
                       vz.v[j] + (szz_z.v[j] + sxz_x.v[j] + syz_y.v[j]) * rkp.v[j]};
        if (g.abs_type == 2) taper_regs<3>(g, f.taper, gz0 + j, gy, gx, v3);
        vx.v[j] = v3[0]; vy.v[j] = v3[1]; vz.v[j] = v3[2];
    }
    stq(wvx + iv, vx);
    stq(wvy + iv, vy);
    stq(wvz + iv, vz);
}

template <class T, bool MB>
__device__ __forceinline__ void v3d_q4(const Grid &g, Fields f)
{
    CELL3D_Q4
    v3d_q4_at<T, 0>(g, f, gz0, gy, gx, iv, ip);
}

template <class T, bool MB = false>
__global__ void __launch_bounds__(128) k_v3d_q4(Grid g, Fields f)
{
    v3d_q4<T, MB>(g, f);
}

// The single-shot FP32 launch asks for 4 resident CTAs per SM (at most 128
// registers, from 136, with a 36-byte spill): 0.333 ms against 0.345 at
// 256^3 L=2 on a B200.  5 CTAs (102 registers) is slower again, and a
// component-at-a-time update with 80 registers slower still (0.37 ms): the
// kernel is bound by the stencil loads each thread keeps in flight.
// TRIG: an ordinary launch that lets the next kernel (the stress update,
// launched with programmatic stream serialization) launch early.  Launched
// that way itself, the kernel would have to read the stresses with plain
// loads (see k_s3d_q4_pf), which cost it more than the overlap gives.
// Taking the x planes in the reverse of the stress kernel's order (each
// kernel starting on the planes the other has just written) was measured
// and is not faster: 16.96 against 17.00 Gcell/s at 256^3, L=2.
template <bool TRIG = false>
__global__ void __launch_bounds__(128, 4) k_v3d_q4_b4(Grid g, Fields f)
{
    if constexpr (TRIG) pdl_trigger();
    constexpr bool MB = false;
    CELL3D_Q4
    v3d_q4_at<float, 0>(g, f, gz0, gy, gx, iv, ip);
}

// ------------------------------------- velocity update staged by cp.async
// k_v3d_q4's arithmetic with its stress operands staged in shared memory by
// asynchronous copies (cp.async, 16 bytes each), so the bytes in flight do
// not hold registers.  A CTA owns a tile of AZ z cells x AY y rows and
// marches over AX x planes; one thread updates one quad (4 z cells) per
// plane.  Shared memory holds
//   ring   sxx, sxy, sxz (the x derivatives) over the tile's own columns, for
//          planes x-4 .. x+5 (10 slots; plane x+5 arrives while x is computed);
//   halo   syy, szz, syz, sxy, sxz over the tile plus a 4-cell y/z halo for
//          plane x (y and z derivatives), double-buffered.
// The copies of plane x+2 are issued after plane x is computed and committed
// as one group; cp.async.wait_group 1 then leaves only the newest group in
// flight.  The waits are on the thread's own copies: they always end.
constexpr int AZ = 32, AY = 16, AX = 16;
constexpr int AHZ = AZ + 8, AHY = AY + 8;
constexpr int ARING = 10;
struct VAsyncSmem {
    float ring[3][ARING][AY][AZ];
    float halo[2][5][AHY][AHZ];
};
constexpr size_t VASYNC_SMEM = sizeof(VAsyncSmem);

__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ Q4 lds4(const float *p)
{
    const float4 t = *reinterpret_cast<const float4 *>(p);
    return Q4{{t.x, t.y, t.z, t.w}};
}
// forward / backward differences of a quad over shared-memory rows `st`
// floats apart (the operation order of dfw_q / dbw_q)
__device__ __forceinline__ Q4 dfw_s(const float *p, int st, const float *hc)
{
    Q4 a = lds4(p + st), b = lds4(p), r;
#pragma unroll
    for (int j = 0; j < 4; j++) r.v[j] = hc[0] * (a.v[j] - b.v[j]);
#pragma unroll
    for (int m = 2; m <= 4; m++) {
        a = lds4(p + m * st);
        b = lds4(p - (m - 1) * st);
#pragma unroll
        for (int j = 0; j < 4; j++) r.v[j] = fmaf(hc[m - 1], a.v[j] - b.v[j], r.v[j]);
    }
    return r;
}
__device__ __forceinline__ Q4 dbw_s(const float *p, int st, const float *hc)
{
    Q4 a = lds4(p), b = lds4(p - st), r;
#pragma unroll
    for (int j = 0; j < 4; j++) r.v[j] = hc[0] * (a.v[j] - b.v[j]);
#pragma unroll
    for (int m = 2; m <= 4; m++) {
        a = lds4(p + (m - 1) * st);
        b = lds4(p - m * st);
#pragma unroll
        for (int j = 0; j < 4; j++) r.v[j] = fmaf(hc[m - 1], a.v[j] - b.v[j], r.v[j]);
    }
    return r;
}
// the 12 values z0-4 .. z0+7 of a quad from a halo row (p at z0 - 4)
__device__ __forceinline__ W12 ldw_s(const float *p)
{
    W12 r;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        const Q4 t = lds4(p + 4 * k);
        r.w[4 * k] = t.v[0]; r.w[4 * k + 1] = t.v[1]; r.w[4 * k + 2] = t.v[2]; r.w[4 * k + 3] = t.v[3];
    }
    return r;
}

// issue the copies of plane x: ring slot of plane x+5 (when inside the grid)
// and the haloed tiles of plane x into halo buffer hb
__device__ __forceinline__ void vasync_issue(const Grid &g, const Fields &f, VAsyncSmem &sm, int z0, int y0,
                                             int xr, int xh, int hb, int tid)
{
    const i64 sx = (i64)g.NY * g.NZ, sy = g.NZ;
    if (xr >= 0 && xr < g.NX) {
        const float *rf[3] = {f.w[SXX], f.w[SXY], f.w[SXZ]};
        const int slot = xr % ARING;
        for (int i = tid; i < 3 * AY * (AZ / 4); i += 128) {
            const int q = i / (AY * (AZ / 4)), r = (i / (AZ / 4)) % AY, c = i % (AZ / 4);
            const int gy = y0 + r, gz = z0 + 4 * c;
            if (gy < g.NY && gz + 3 < g.NZ)
                cp_async16(&sm.ring[q][slot][r][4 * c], rf[q] + xr * sx + (i64)gy * sy + gz);
        }
    }
    if (xh >= 0) {
        const float *hf[5] = {f.w[SYY], f.w[SZZ], f.w[SYZ], f.w[SXY], f.w[SXZ]};
        for (int i = tid; i < 5 * AHY * (AHZ / 4); i += 128) {
            const int q = i / (AHY * (AHZ / 4)), r = (i / (AHZ / 4)) % AHY, c = i % (AHZ / 4);
            const int gy = y0 - 4 + r, gz = z0 - 4 + 4 * c;
            if (gy >= 0 && gy < g.NY && gz >= 0 && gz + 3 < g.NZ)
                cp_async16(&sm.halo[hb][q][r][4 * c], hf[q] + xh * sx + (i64)gy * sy + gz);
        }
    }
}

__global__ void __launch_bounds__(128, 2) k_v3d_async(Grid g, Fields f)
{
    constexpr int F = 4;
    extern __shared__ __align__(16) unsigned char vasync_raw[];
    VAsyncSmem &sm = *reinterpret_cast<VAsyncSmem *>(vasync_raw);
    const int tid = threadIdx.x + 8 * threadIdx.y;
    const int z0 = F + blockIdx.x * AZ, y0 = F + blockIdx.y * AY;
    const int xb = F + blockIdx.z * AX, xe = min(xb + AX, g.NX - F);
    const int qz = threadIdx.x, yy = threadIdx.y;
    const int gz0 = z0 + 4 * qz, gy = y0 + yy;
    const bool ok = gz0 <= g.NZ - F - 1 && gy <= g.NY - F - 1;
    const float *hc = g.hc;
    const i64 sx = (i64)g.NY * g.NZ, sy = g.NZ;
    // prologue: ring planes xb-4 .. xb+4 and the halo of plane xb (group 0),
    // ring plane xb+5 and the halo of plane xb+1 (group 1)
    for (int xr = xb - 4; xr < xb + 4; xr++) vasync_issue(g, f, sm, z0, y0, xr, -1, 0, tid);
    vasync_issue(g, f, sm, z0, y0, xb + 4, xb, 0, tid);
    cp_async_commit();
    vasync_issue(g, f, sm, z0, y0, xb + 5, xb + 1 < xe ? xb + 1 : -1, 1, tid);
    cp_async_commit();
    for (int gx = xb; gx < xe; gx++) {
        const int hb = (gx - xb) & 1;
        Q4 vx, vy, vz, rip, rjp, rkp;
        const i64 iv = gx * sx + (i64)gy * sy + gz0;
        const i64 ip = ((i64)(gx - F) * g.ny + (gy - F)) * g.nz + (gz0 - F);
        if (ok) {
            vx = ldq_rw(f.w[VX] + iv); vy = ldq_rw(f.w[VY] + iv); vz = ldq_rw(f.w[VZ] + iv);
            rip = ldq(f.p[PRIP] + ip); rjp = ldq(f.p[PRJP] + ip); rkp = ldq(f.p[PRKP] + ip);
        }
        cp_async_wait<1>();
        __syncthreads();
        if (ok) {
            const float *H0 = &sm.halo[hb][0][0][0];
            const int HP = AHY * AHZ;                 // floats per haloed tile
            const int hrow = (yy + 4) * AHZ + 4 * qz;  // the quad's row, at z0 - 4 of its window
            const W12 wzz = ldw_s(H0 + 1 * HP + hrow), wxz = ldw_s(H0 + 4 * HP + hrow),
                      wyz = ldw_s(H0 + 2 * HP + hrow);
            const int RP = AY * AZ;                    // floats per ring slot
            const int rc = yy * AZ + 4 * qz;
            auto ring_at = [&](int q, int x) { return &sm.ring[q][x % ARING][0][0] + rc; };
            Q4 szz_z = dfw_z<F>(wzz, hc);
            Q4 sxx_x, sxz_x, sxy_x;
            {
                // x differences across ring slots (plane offsets wrap modulo ARING)
                const float *c0 = ring_at(0, gx);
                (void)RP;
                Q4 a = lds4(ring_at(0, gx + 1)), b = lds4(c0), r;
#pragma unroll
                for (int j = 0; j < 4; j++) r.v[j] = hc[0] * (a.v[j] - b.v[j]);
#pragma unroll
                for (int m = 2; m <= F; m++) {
                    a = lds4(ring_at(0, gx + m));
                    b = lds4(ring_at(0, gx - (m - 1)));
#pragma unroll
                    for (int j = 0; j < 4; j++) r.v[j] = fmaf(hc[m - 1], a.v[j] - b.v[j], r.v[j]);
                }
                sxx_x = r;
                for (int q = 1; q <= 2; q++) {
                    a = lds4(ring_at(q, gx));
                    b = lds4(ring_at(q, gx - 1));
#pragma unroll
                    for (int j = 0; j < 4; j++) r.v[j] = hc[0] * (a.v[j] - b.v[j]);
#pragma unroll
                    for (int m = 2; m <= F; m++) {
                        a = lds4(ring_at(q, gx + m - 1));
                        b = lds4(ring_at(q, gx - m));
#pragma unroll
                        for (int j = 0; j < 4; j++) r.v[j] = fmaf(hc[m - 1], a.v[j] - b.v[j], r.v[j]);
                    }
                    if (q == 1) sxy_x = r;
                    else sxz_x = r;
                }
            }
            Q4 sxz_z = dbw_z<F>(wxz, hc);
            Q4 syz_y = dbw_s(H0 + 2 * HP + hrow + 4, AHZ, hc);
            Q4 syz_z = dbw_z<F>(wyz, hc);
            Q4 syy_y = dfw_s(H0 + 0 * HP + hrow + 4, AHZ, hc);
            Q4 sxy_y = dbw_s(H0 + 3 * HP + hrow + 4, AHZ, hc);
            if (g.abs_type == 1)
                cpml_v3d_q4(g, f, gz0, gy, gx, sxx_x, syy_y, szz_z, sxy_y, sxy_x, syz_y, syz_z, sxz_x, sxz_z);
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float v3[3] = {vx.v[j] + (sxx_x.v[j] + sxy_y.v[j] + sxz_z.v[j]) * rip.v[j],
                               vy.v[j] + (syy_y.v[j] + sxy_x.v[j] + syz_z.v[j]) * rjp.v[j],
                               vz.v[j] + (szz_z.v[j] + sxz_x.v[j] + syz_y.v[j]) * rkp.v[j]};
                if (g.abs_type == 2) taper_regs<3>(g, f.taper, gz0 + j, gy, gx, v3);
                vx.v[j] = v3[0]; vy.v[j] = v3[1]; vz.v[j] = v3[2];
            }
            stq(f.w[VX] + iv, vx);
            stq(f.w[VY] + iv, vy);
            stq(f.w[VZ] + iv, vz);
        }
        __syncthreads();   // plane gx-4's ring slot and halo buffer hb are free
        vasync_issue(g, f, sm, z0, y0, gx + 6, gx + 2 < xe ? gx + 2 : -1, hb, tid);
        cp_async_commit();
    }
    cp_async_wait<0>();
}

bool launch_update_v_async(const Grid &g, const Fields &f, cudaStream_t st)
{
    if (g.nd != 3 || g.F != 4 || g.nz % 4 || g.fhalf || g.nb != 1) return false;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_v3d_async, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)VASYNC_SMEM) !=
            cudaSuccess)
            return false;
        attr = true;
    }
    const dim3 b(8, AY), gr((g.nz + AZ - 1) / AZ, (g.ny + AY - 1) / AY, (g.nx + AX - 1) / AX);
    k_v3d_async<<<gr, b, VASYNC_SMEM, st>>>(g, f);
    return true;
}

// CPML corrections of cpml_s3d (forward form) for a quad of z cells
__device__ __forceinline__ void cpml_s3d_q4(const Grid &g, const Fields &f, int gz0, int gy, int gx, Q4 &vxx,
                                            Q4 &vxy, Q4 &vxz, Q4 &vyx, Q4 &vyy, Q4 &vyz, Q4 &vzx, Q4 &vzy, Q4 &vzz)
{
    const int F = g.F, NAB = g.nab, NZ = g.NZ, NY = g.NY, NX = g.NX;
    const i64 nz = g.nz, ny = g.ny;
    if (cpml_slabs_apart(g)) {   // side-merged form, as in cpml_v3d_q4
        const i64 k0 = gz0 - F;
        const bool zhi = gz0 > NZ - NAB - F - 1, zlo = !g.freesurf && gz0 - F < NAB;
        if (zhi || zlo) {
            const int k = zhi ? gz0 - NZ + 2 * NAB + F : gz0 - F;
            const int st = zhi ? -1 : 1, cf = zhi ? 2 * NAB - k : k, ch = zhi ? 2 * NAB - 1 - k : k;
            const i64 q = ((i64)(gx - F) * ny + (gy - F)) * (2 * NAB) + k;
            cpml_zq(f.psi[PVX_Z], q, f.kinv[2][1], f.cz[CAH], f.cz[CBH], ch, st, vxz);
            cpml_zq(f.psi[PVY_Z], q, f.kinv[2][1], f.cz[CAH], f.cz[CBH], ch, st, vyz);
            cpml_zq(f.psi[PVZ_Z], q, f.kinv[2][0], f.cz[CA], f.cz[CB], cf, st, vzz);
        }
        const bool ylo = gy - F < NAB, yhi = gy > NY - NAB - F - 1;
        if (ylo || yhi) {
            const int j = ylo ? gy - F : gy - NY + 2 * NAB + F;
            const int cf = ylo ? j : 2 * NAB - j, ch = ylo ? j : 2 * NAB - 1 - j;
            const i64 q = ((i64)(gx - F) * (2 * NAB) + j) * nz + k0;
            cpml_q(f.psi[PVX_Y], q, f.kinv[1][1], f.cy[CAH], f.cy[CBH], ch, vxy);
            cpml_q(f.psi[PVY_Y], q, f.kinv[1][0], f.cy[CA], f.cy[CB], cf, vyy);
            cpml_q(f.psi[PVZ_Y], q, f.kinv[1][1], f.cy[CAH], f.cy[CBH], ch, vzy);
        }
        const bool xlo = gx - F < NAB, xhi = gx > NX - NAB - F - 1;
        if (xlo || xhi) {
            const int i = xlo ? gx - F : gx - NX + 2 * NAB + F;
            const int cf = xlo ? i : 2 * NAB - i, ch = xlo ? i : 2 * NAB - 1 - i;
            const i64 q = ((i64)i * ny + (gy - F)) * nz + k0;
            cpml_q(f.psi[PVX_X], q, f.kinv[0][0], f.cx[CA], f.cx[CB], cf, vxx);
            cpml_q(f.psi[PVY_X], q, f.kinv[0][1], f.cx[CAH], f.cx[CBH], ch, vyx);
            cpml_q(f.psi[PVZ_X], q, f.kinv[0][1], f.cx[CAH], f.cx[CBH], ch, vzx);
        }
        return;
    }
    // with NAB % 4 == 0 a quad lies in at most one z slab, entirely (the two
    // plain ifs of cpml_s3d can only both hold when the slabs overlap, which
    // needs nz < 2 NAB + 4 and takes the per-cell path)
    const bool zq = NAB % 4 == 0 && g.nz >= 2 * NAB + 4;
    if (zq && gz0 > NZ - NAB - F - 1) {
        i64 i = gx - F, jj = gy - F, k = gz0 - NZ + NAB + F + NAB;
        int ind = 2 * NAB - 1 - (int)k;
        i64 q = (i * ny + jj) * (2 * NAB) + k;
        cpml_zq(f.psi[PVX_Z], q, f.kinv[2][1], f.cz[CAH], f.cz[CBH], ind, -1, vxz);
        cpml_zq(f.psi[PVY_Z], q, f.kinv[2][1], f.cz[CAH], f.cz[CBH], ind, -1, vyz);
        cpml_zq(f.psi[PVZ_Z], q, f.kinv[2][0], f.cz[CA], f.cz[CB], ind + 1, -1, vzz);
    } else if (zq && !g.freesurf && gz0 - F < NAB) {
        i64 i = gx - F, jj = gy - F, k = gz0 - F;
        i64 q = (i * ny + jj) * (2 * NAB) + k;
        cpml_zq(f.psi[PVX_Z], q, f.kinv[2][1], f.cz[CAH], f.cz[CBH], (int)k, 1, vxz);
        cpml_zq(f.psi[PVY_Z], q, f.kinv[2][1], f.cz[CAH], f.cz[CBH], (int)k, 1, vyz);
        cpml_zq(f.psi[PVZ_Z], q, f.kinv[2][0], f.cz[CA], f.cz[CB], (int)k, 1, vzz);
    } else if (!zq && (gz0 + 3 > NZ - NAB - F - 1 || (!g.freesurf && gz0 - F < NAB))) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int gz = gz0 + j;
            if (gz > NZ - NAB - F - 1) {
                i64 i = gx - F, jj = gy - F, k = gz - NZ + NAB + F + NAB;
                int ind = 2 * NAB - 1 - (int)k;
                i64 q = (i * ny + jj) * (2 * NAB) + k;
                cpml(f.psi[PVX_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, vxz.v[j]);
                cpml(f.psi[PVY_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, vyz.v[j]);
                cpml(f.psi[PVZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], ind + 1, vzz.v[j]);
            }
            if (!g.freesurf && gz - F < NAB) {
                i64 i = gx - F, jj = gy - F, k = gz - F;
                i64 q = (i * ny + jj) * (2 * NAB) + k;
                cpml(f.psi[PVX_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], (int)k, vxz.v[j]);
                cpml(f.psi[PVY_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], (int)k, vyz.v[j]);
                cpml(f.psi[PVZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], (int)k, vzz.v[j]);
            }
        }
    }
    const i64 k0 = gz0 - F;
    if (gy - F < NAB) {
        i64 i = gx - F, j = gy - F;
        i64 q = (i * (2 * NAB) + j) * nz + k0;
        cpml_q(f.psi[PVX_Y], q, f.kinv[1][1], f.cy[CAH], f.cy[CBH], (int)j, vxy);
        cpml_q(f.psi[PVY_Y], q, f.kinv[1][0], f.cy[CA], f.cy[CB], (int)j, vyy);
        cpml_q(f.psi[PVZ_Y], q, f.kinv[1][1], f.cy[CAH], f.cy[CBH], (int)j, vzy);
    }
    if (gy > NY - NAB - F - 1) {
        i64 i = gx - F, j = gy - NY + NAB + F + NAB;
        int ind = 2 * NAB - 1 - (int)j;
        i64 q = (i * (2 * NAB) + j) * nz + k0;
        cpml_q(f.psi[PVX_Y], q, f.kinv[1][1], f.cy[CAH], f.cy[CBH], ind, vxy);
        cpml_q(f.psi[PVY_Y], q, f.kinv[1][0], f.cy[CA], f.cy[CB], ind + 1, vyy);
        cpml_q(f.psi[PVZ_Y], q, f.kinv[1][1], f.cy[CAH], f.cy[CBH], ind, vzy);
    }
    if (gx - F < NAB) {
        i64 i = gx - F, j = gy - F;
        i64 q = (i * ny + j) * nz + k0;
        cpml_q(f.psi[PVX_X], q, f.kinv[0][0], f.cx[CA], f.cx[CB], (int)i, vxx);
        cpml_q(f.psi[PVY_X], q, f.kinv[0][1], f.cx[CAH], f.cx[CBH], (int)i, vyx);
        cpml_q(f.psi[PVZ_X], q, f.kinv[0][1], f.cx[CAH], f.cx[CBH], (int)i, vzx);
    }
    if (gx > NX - NAB - F - 1) {
        i64 i = gx - NX + NAB + F + NAB, j = gy - F;
        int ind = 2 * NAB - 1 - (int)i;
        i64 q = (i * ny + j) * nz + k0;
        cpml_q(f.psi[PVX_X], q, f.kinv[0][0], f.cx[CA], f.cx[CB], ind + 1, vxx);
        cpml_q(f.psi[PVY_X], q, f.kinv[0][1], f.cx[CAH], f.cx[CBH], ind, vyx);
        cpml_q(f.psi[PVZ_X], q, f.kinv[0][1], f.cx[CAH], f.cx[CBH], ind, vzx);
    }
}

// Stress and memory-variable update of four z cells (the arithmetic of
// k_s3d_stream per cell).  The per-cell work runs in two phases -- normal
// stresses (sxx, syy, szz with rxx, ryy, rzz) then shear stresses (sxy, syz,
// sxz with rxy, ryz, rxz) -- each loading only its own memory variables and
// parameters, so the live state fits in registers; the components are
// independent, so the split changes no result.
//
// surf: the free surface of the same step follows the update in registers
// (the fused step kernel; k_surf3d's arithmetic at z = F, forward direction):
// the quad at gz0 = F zeroes szz and rzz there, corrects sxx, syy, rxx, ryy
// with the velocity derivatives of the update (CPML-corrected as k_surf3d
// forms them) and writes the images szz(F-m) = -szz(F+m) for m = 1..3 and
// sxz(F-m) = -sxz(F+m-1), syz(F-m) = -syz(F+m-1) for m = 1..4; the quad at
// gz0 = F+4 writes szz(F-4) = -szz(F+4).
template <int L, class T, class TR = T>
__device__ __forceinline__ void s_normal_q4(const Grid &g, const Fields &f, int gz0, int gy, int gx, i64 iv, i64 ip,
                                            const Q4 &vxx, const Q4 &vyy, const Q4 &vzz, bool surf = false)
{
    T *const ws[3] = {fld<T>(f.w[SXX]), fld<T>(f.w[SYY]), fld<T>(f.w[SZZ])};
    TR *const wr[3] = {fld<TR>(f.r[RXX]), fld<TR>(f.r[RYY]), fld<TR>(f.r[RZZ])};
    Q4 sq[3];
#pragma unroll
    for (int q = 0; q < 3; q++) sq[q] = ldq_rw(ws[q] + iv);
    const Q4 qM = ldq(f.p[PM] + ip), qmu = ldq(f.p[PMU] + ip);
    Q4 rq[3][L > 0 ? L : 1];
    Q4 qtaup, qtaus;
    if constexpr (L == 0) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float vxxyyzz = vxx.v[j] + vyy.v[j] + vzz.v[j], vyyzz = vyy.v[j] + vzz.v[j];
            float vxxzz = vxx.v[j] + vzz.v[j], vxxyy = vxx.v[j] + vyy.v[j];
            float gm = qM.v[j], fm = 2.0f * qmu.v[j];
            sq[0].v[j] += gm * vxxyyzz - fm * vyyzz;
            sq[1].v[j] += gm * vxxyyzz - fm * vxxzz;
            sq[2].v[j] += gm * vxxyyzz - fm * vxxyy;
        }
    } else {
        qtaup = ldq(f.p[PTAUP] + ip);
        qtaus = ldq(f.p[PTAUS] + ip);
#pragma unroll
        for (int l = 0; l < L; l++)
#pragma unroll
            for (int q = 0; q < 3; q++) rq[q][l] = ldr_q<T>(g, wr[q] + l * g.nvol + iv);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float vxxyyzz = vxx.v[j] + vyy.v[j] + vzz.v[j], vyyzz = vyy.v[j] + vzz.v[j];
            float vxxzz = vxx.v[j] + vzz.v[j], vxxyy = vxx.v[j] + vyy.v[j];
            const float lM = qM.v[j], lmu = qmu.v[j], ltaup = qtaup.v[j], ltaus = qtaus.v[j];
            float gm = lM * (1.0f + (float)L * ltaup);
            float fm = 2.0f * lmu * (1.0f + (float)L * ltaus);
            float d = 2.0f * lmu * ltaus / g.dt, e = lM * ltaup / g.dt;
            float a[3] = {0, 0, 0};
#pragma unroll
            for (int l = 0; l < L; l++)
#pragma unroll
                for (int q = 0; q < 3; q++) a[q] += rq[q][l].v[j];
            float ls[3] = {(gm * vxxyyzz - fm * vyyzz) + g.dt2 * a[0], (gm * vxxyyzz - fm * vxxzz) + g.dt2 * a[1],
                           (gm * vxxyyzz - fm * vxxyy) + g.dt2 * a[2]};
            a[0] = a[1] = a[2] = 0;
#pragma unroll
            for (int l = 0; l < L; l++) {
                float el = g.eta[l];
                float b = 1.0f / (1.0f + el * 0.5f), c = 1.0f - el * 0.5f;
                rq[0][l].v[j] = b * (rq[0][l].v[j] * c - el * (e * vxxyyzz - d * vyyzz));
                rq[1][l].v[j] = b * (rq[1][l].v[j] * c - el * (e * vxxyyzz - d * vxxzz));
                rq[2][l].v[j] = b * (rq[2][l].v[j] * c - el * (e * vxxyyzz - d * vxxyy));
#pragma unroll
                for (int q = 0; q < 3; q++) a[q] += rq[q][l].v[j];
            }
#pragma unroll
            for (int q = 0; q < 3; q++) sq[q].v[j] += ls[q] + g.dt2 * a[q];
        }
    }
    if (g.abs_type == 2) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float v3[3] = {sq[0].v[j], sq[1].v[j], sq[2].v[j]};
            taper_regs<3>(g, f.taper, gz0 + j, gy, gx, v3);
#pragma unroll
            for (int q = 0; q < 3; q++) sq[q].v[j] = v3[q];
        }
    }
    if (surf && gz0 == g.F + 4) stv(ws[2] + iv - 8, -sq[2].v[0]);
    if (surf && gz0 == g.F) {
        const float vx0 = vxx.v[0], vy0 = vyy.v[0], vz0 = vzz.v[0];
        sq[2].v[0] = 0.0f;
        if constexpr (L == 0) {
            float fm = qmu.v[0] * 2.0f, gm = qM.v[0];
            float h = -((gm - fm) * (gm - fm) * (vx0 + vy0) / gm) - ((gm - fm) * vz0);
            sq[0].v[0] += h;
            sq[1].v[0] += h;
        } else {
            const float taus = qtaus.v[0], taup = qtaup.v[0], mu = qmu.v[0], M = qM.v[0];
            float fm = mu * 2.0f * (1.0f + L * taus);
            float gm = M * (1.0f + L * taup);
            float h = -((gm - fm) * (gm - fm) * (vx0 + vy0) / gm) - ((gm - fm) * vz0);
            float sumx = 0, sumy = 0;
#pragma unroll
            for (int l = 0; l < L; l++) {
                rq[2][l].v[0] = 0.0f;
                sumx += rq[0][l].v[0];
                sumy += rq[1][l].v[0];
            }
            sq[0].v[0] = sq[0].v[0] + (h - g.dt2 * sumx);
            sq[1].v[0] = sq[1].v[0] + (h - g.dt2 * sumy);
            float d = 2.0f * mu * taus / g.dt, e = M * taup / g.dt;
            sumx = 0; sumy = 0;
#pragma unroll
            for (int l = 0; l < L; l++) {
                float b = g.eta[l] / (1.0f + g.eta[l] * 0.5f);
                float hh = b * (((d - e) * ((fm / gm) - 1.0f) * (vx0 + vy0)) - ((d - e) * vz0));
                rq[0][l].v[0] += hh;
                rq[1][l].v[0] += hh;
                sumx += rq[0][l].v[0];
                sumy += rq[1][l].v[0];
            }
            sq[0].v[0] += g.dt2 * sumx;
            sq[1].v[0] += g.dt2 * sumy;
        }
#pragma unroll
        for (int m = 1; m <= 3; m++) stv(ws[2] + iv - m, -sq[2].v[m]);
    }
    if constexpr (L > 0) {
#pragma unroll
        for (int l = 0; l < L; l++)
#pragma unroll
            for (int q = 0; q < 3; q++) str_q<T>(g, wr[q] + l * g.nvol + iv, rq[q][l]);
    }
#pragma unroll
    for (int q = 0; q < 3; q++) stq(ws[q] + iv, sq[q]);
}

template <int L, class T, class TR = T>
__device__ __forceinline__ void s_shear_q4(const Grid &g, const Fields &f, int gz0, int gy, int gx, i64 iv, i64 ip,
                                           const Q4 &vxyyx, const Q4 &vyzzy, const Q4 &vxzzx, bool surf = false)
{
    T *const ws[3] = {fld<T>(f.w[SXY]), fld<T>(f.w[SYZ]), fld<T>(f.w[SXZ])};
    TR *const wr[3] = {fld<TR>(f.r[RXY]), fld<TR>(f.r[RYZ]), fld<TR>(f.r[RXZ])};
    Q4 sq[3];
#pragma unroll
    for (int q = 0; q < 3; q++) sq[q] = ldq_rw(ws[q] + iv);
    const Q4 qmuipjp = ldq(f.p[PMUIPJP] + ip), qmujpkp = ldq(f.p[PMUJPKP] + ip), qmuipkp = ldq(f.p[PMUIPKP] + ip);
    if constexpr (L == 0) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            sq[0].v[j] += qmuipjp.v[j] * vxyyx.v[j];
            sq[1].v[j] += qmujpkp.v[j] * vyzzy.v[j];
            sq[2].v[j] += qmuipkp.v[j] * vxzzx.v[j];
        }
    } else {
        const Q4 qtausipjp = ldq(f.p[PTAUSIPJP] + ip), qtausjpkp = ldq(f.p[PTAUSJPKP] + ip),
                 qtausipkp = ldq(f.p[PTAUSIPKP] + ip);
        Q4 rq[3][L];
#pragma unroll
        for (int l = 0; l < L; l++)
#pragma unroll
            for (int q = 0; q < 3; q++) rq[q][l] = ldr_q<T>(g, wr[q] + l * g.nvol + iv);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float lmuipkp = qmuipkp.v[j], lmuipjp = qmuipjp.v[j], lmujpkp = qmujpkp.v[j];
            const float ltausipkp = qtausipkp.v[j], ltausipjp = qtausipjp.v[j], ltausjpkp = qtausjpkp.v[j];
            float fipjp = lmuipjp * (1.0f + (float)L * ltausipjp);
            float fjpkp = lmujpkp * (1.0f + (float)L * ltausjpkp);
            float fipkp = lmuipkp * (1.0f + (float)L * ltausipkp);
            float dipjp = lmuipjp * ltausipjp / g.dt, djpkp = lmujpkp * ltausjpkp / g.dt,
                  dipkp = lmuipkp * ltausipkp / g.dt;
            float a[3] = {0, 0, 0};
#pragma unroll
            for (int l = 0; l < L; l++)
#pragma unroll
                for (int q = 0; q < 3; q++) a[q] += rq[q][l].v[j];
            float ls[3] = {fipjp * vxyyx.v[j] + g.dt2 * a[0], fjpkp * vyzzy.v[j] + g.dt2 * a[1],
                           fipkp * vxzzx.v[j] + g.dt2 * a[2]};
            a[0] = a[1] = a[2] = 0;
#pragma unroll
            for (int l = 0; l < L; l++) {
                float el = g.eta[l];
                float b = 1.0f / (1.0f + el * 0.5f), c = 1.0f - el * 0.5f;
                rq[0][l].v[j] = b * (rq[0][l].v[j] * c - el * (dipjp * vxyyx.v[j]));
                rq[1][l].v[j] = b * (rq[1][l].v[j] * c - el * (djpkp * vyzzy.v[j]));
                rq[2][l].v[j] = b * (rq[2][l].v[j] * c - el * (dipkp * vxzzx.v[j]));
#pragma unroll
                for (int q = 0; q < 3; q++) a[q] += rq[q][l].v[j];
            }
#pragma unroll
            for (int q = 0; q < 3; q++) sq[q].v[j] += ls[q] + g.dt2 * a[q];
        }
#pragma unroll
        for (int l = 0; l < L; l++)
#pragma unroll
            for (int q = 0; q < 3; q++) str_q<T>(g, wr[q] + l * g.nvol + iv, rq[q][l]);
    }
    if (g.abs_type == 2) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            float v3[3] = {sq[0].v[j], sq[1].v[j], sq[2].v[j]};
            taper_regs<3>(g, f.taper, gz0 + j, gy, gx, v3);
#pragma unroll
            for (int q = 0; q < 3; q++) sq[q].v[j] = v3[q];
        }
    }
    if (surf && gz0 == g.F) {
#pragma unroll
        for (int m = 1; m <= 4; m++) {
            stv(ws[2] + iv - m, -sq[2].v[m - 1]);   // sxz
            stv(ws[1] + iv - m, -sq[1].v[m - 1]);   // syz
        }
    }
#pragma unroll
    for (int q = 0; q < 3; q++) stq(ws[q] + iv, sq[q]);
}

// stress update of the quad (gz0..gz0+3, gy, gx); LP: load policy of the
// velocity reads; surf: free surface folded in (see s_normal_q4); PF: first
// ask L2 for the quad's per-cell streams
template <int L, class T, int LP = 0, bool PF = false, bool PDL = false, class TR = T>
__device__ __forceinline__ void s3d_q4_at(const Grid &g, const Fields &f, int gz0, int gy, int gx, i64 iv, i64 ip,
                                          bool surf = false)
{
    constexpr int F = 4;
    const i64 sx = (i64)g.NY * g.NZ, sy = g.NZ;
    const float *hc = g.hc;
    if constexpr (PF) {
#pragma unroll
        for (int q = SXX; q <= SXZ; q++) asm volatile("prefetch.global.L2 [%0];" ::"l"(fld<T>(f.w[q]) + iv));
#pragma unroll
        for (int l = 0; l < L; l++)
#pragma unroll
            for (int q = 0; q < NR; q++)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(fld<TR>(f.r[q]) + l * g.nvol + iv));
        constexpr int np = L > 0 ? 10 : 5;
        constexpr int pid[10] = {PM, PMU, PMUIPJP, PMUJPKP, PMUIPKP, PTAUP, PTAUS, PTAUSIPJP, PTAUSJPKP, PTAUSIPKP};
#pragma unroll
        for (int k = 0; k < np; k++) asm volatile("prefetch.global.L2 [%0];" ::"l"(f.p[pid[k]] + ip));
    }
    // launched early (programmatic dependent launch): everything the
    // previous kernels write is read from here on
    if constexpr (PDL) pdl_wait();
    const T *Vx = fld<T>(f.w[VX]), *Vy = fld<T>(f.w[VY]), *Vz = fld<T>(f.w[VZ]);
    Q4 vzz = dbw_z<F>(ldw<T, LP>(Vz, iv), hc);
    Q4 vyz = dfw_z<F>(ldw<T, LP>(Vy, iv), hc);
    Q4 vxz = dfw_z<F>(ldw<T, LP>(Vx, iv), hc);
    Q4 vzx = dfw_q<F, T, LP>(Vz, iv, sx, hc), vzy = dfw_q<F, T, LP>(Vz, iv, sy, hc);
    Q4 vyx = dfw_q<F, T, LP>(Vy, iv, sx, hc), vyy = dbw_q<F, T, LP>(Vy, iv, sy, hc);
    Q4 vxx = dbw_q<F, T, LP>(Vx, iv, sx, hc), vxy = dfw_q<F, T, LP>(Vx, iv, sy, hc);
    if (g.abs_type == 1) cpml_s3d_q4(g, f, gz0, gy, gx, vxx, vxy, vxz, vyx, vyy, vyz, vzx, vzy, vzz);
    Q4 vxyyx, vyzzy, vxzzx;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        vxyyx.v[j] = vxy.v[j] + vyx.v[j];
        vyzzy.v[j] = vyz.v[j] + vzy.v[j];
        vxzzx.v[j] = vxz.v[j] + vzx.v[j];
    }
    s_normal_q4<L, T, TR>(g, f, gz0, gy, gx, iv, ip, vxx, vyy, vzz, surf);
    s_shear_q4<L, T, TR>(g, f, gz0, gy, gx, iv, ip, vxyyx, vyzzy, vxzzx, surf);
}

// surf: the free surface of the step applied in the same launch (single-shot
// modelling runs; see s_normal_q4)
template <int L, class T, bool MB = false>
__global__ void __launch_bounds__(128, 4) k_s3d_q4(Grid g, Fields f, bool surf)
{
    CELL3D_Q4
    s3d_q4_at<L, T, 0>(g, f, gz0, gy, gx, iv, ip, surf);
}

// Single-shot launches of the default selection: each thread first asks L2
// for its own per-cell streams (prefetch.global.L2 of its stresses, memory
// variables and parameters), so they are on their way while the velocity
// stencils load, and the launch takes 3 CTAs per SM (168 registers) so that
// more stencil loads stay in flight.  256^3, L=2, CPML 20, FP32 on a B200:
// 0.651 ms against 0.695 for k_s3d_q4 (0.571 against 0.601 without
// absorbing boundary); the prefetch at 4 CTAs per SM gave 0.674, 3 CTAs
// without it 0.713.
// PDL: launched with programmatic stream serialization (launch_pdl).  The
// velocities then come through plain loads: a read-only-path (ld.global.nc)
// load counts as invariant, and the compiler may move it above the wait.
// TR: storage type of the memory variables (FP16 under FP32 wave fields
// with Grid::rhalf)
template <int L, class T, bool PDL = false, class TR = T>
__global__ void __launch_bounds__(128, 3) k_s3d_q4_pf(Grid g, Fields f, bool surf)
{
    constexpr bool MB = false;
    if constexpr (PDL) pdl_trigger();
    CELL3D_Q4
    s3d_q4_at<L, T, PDL ? 1 : 0, true, PDL, TR>(g, f, gz0, gy, gx, iv, ip, surf);
}

// ------------------------------------------------- fused 3D forward step
// One launch advances the whole grid one time step: velocity update, stress
// and memory-variable update and (with a free surface) the free surface, so
// the stresses the velocity stencils read are read again by the stress
// updates of nearby work units, and the velocities written are read back,
// while both are still in L2.  Per cell the arithmetic is that of k_v3d_q4,
// k_s3d_q4 and k_surf3d, in that order.
//
// Work unit: a tile of FZ z cells x FY y rows in one x plane.  A CTA takes a
// ticket (atomicAdd) and works on unit number ticket - base; units are
// numbered plane by plane (x slowest).  Unit (c, t) first updates the
// velocities of plane F + c + 4 of tile t (unit 0 also planes F .. F + 3) and
// publishes its flag, then waits for the flags of the units whose velocities
// its stress stencils read -- planes F + c - 4 .. F + c + 4 of its own tile
// (units c - 8 .. c - 1) and plane F + c of the four y/z neighbour tiles
// (units c - 4) -- and updates the stresses of plane F + c.  Every wait is
// on a unit with a lower number, taken by a CTA that started earlier, so the
// waits always end however few CTAs are resident.  Everything is updated
// in place; the same waits order every stress overwrite after all velocity
// reads of the old value: the stresses of plane F + c in tile t are read by
// the velocity updates of planes F + c - 4 .. F + c + 4 in tile t (units
// c - 8 .. c) and of plane F + c in its neighbours (units c - 4), exactly
// the units (c, t) waits for.  Velocity reads of the stress phase go
// through L2 (__ldcg): other CTAs wrote them during the launch.  Waits are
// bounded (FUSED_WAIT_NS of %globaltimer); one that runs out sets
// g_fused_status, which makes every later CTA and launch skip its work and
// the host report an error.
constexpr int FZ = 32, FY = 16;
constexpr unsigned long long FUSED_WAIT_NS = 2000000000ull;
__device__ int g_fused_status;   // 0 ok, 1 a wait ran out

__device__ __forceinline__ int ld_acquire_gpu(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(int *p, int v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// wait until *flag >= want; false when the bound ran out or another CTA's did
__device__ bool fused_wait(const int *flag, int want)
{
    if (ld_acquire_gpu(flag) >= want) return true;
    const unsigned long long t0 = global_ns();
    unsigned ns = 32;
    for (;;) {
        __nanosleep(ns);
        if (ns < 512) ns *= 2;
        if (ld_acquire_gpu(flag) >= want) return true;
        if (*(volatile int *)&g_fused_status) return false;
        if (global_ns() - t0 > FUSED_WAIT_NS) return false;
    }
}

template <int L>
__global__ void __launch_bounds__(128, 4) k_fused3d_q4(Grid g, Fields f, FusedSync fs, int epoch)
{
    constexpr int F = 4;
    __shared__ int s_unit, s_go;
    const int tid = threadIdx.x + 8 * threadIdx.y;
    if (tid == 0) {
        s_unit = (int)(atomicAdd(fs.ticket, 1u) - fs.base);
        s_go = *(volatile int *)&g_fused_status == 0;
    }
    __syncthreads();
    if (!s_go) return;
    const int ntile = fs.ntz * fs.nty, unit = s_unit;
    if (unit < 0 || unit >= fs.units) {   // the counter was not reset: never index past the flags
        if (tid == 0) atomicExch(&g_fused_status, 1);
        return;
    }
    const int c = unit / ntile, tile = unit - c * ntile, ty = tile / fs.ntz, tz = tile - ty * fs.ntz;
    const int gz0 = F + tz * FZ + 4 * threadIdx.x, gy = F + ty * FY + threadIdx.y;
    const bool ok_cell = gz0 <= g.NZ - F - 1 && gy <= g.NY - F - 1;
    const int nxp = g.NX - 2 * F;   // x planes
    const i64 sx = (i64)g.NY * g.NZ, sy = g.NZ;
    // phase 1: velocities of plane F + c + 4 (unit 0: planes F .. F + 4).
    // The stress reads take the read-only path: no stress cell read here is
    // overwritten before this unit's flag is up, and nothing in this launch
    // reads a stress value written in it.
    if (ok_cell) {
        const int x0 = c == 0 ? F : F + c + 4, x1 = min(F + c + 5, g.NX - F);
        for (int gx = x0; gx < x1; gx++) {
            const i64 iv = gx * sx + (i64)gy * sy + gz0;
            const i64 ip = ((i64)(gx - F) * g.ny + (gy - F)) * g.nz + (gz0 - F);
            v3d_q4_at<float, 0>(g, f, gz0, gy, gx, iv, ip);
        }
    }
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        st_release_gpu(fs.flags + unit, epoch);
    }
    // the units this one reads velocities of: threads 0..7 the own tile's
    // planes (units c - 8 .. c - 1; unit 0 holds planes F .. F + 4), threads
    // 8..11 the neighbours' plane F + c (unit c - 4)
    bool ok = true;
    if (tid < 12) {
        int wu = -1;
        if (tid < 8) {
            const int uc = c - 8 + tid;
            if (uc >= 0 && uc <= nxp - 5) wu = uc * ntile + tile;
        } else {
            const int nt = tid == 8 ? (tz > 0 ? tile - 1 : -1)
                         : tid == 9 ? (tz < fs.ntz - 1 ? tile + 1 : -1)
                         : tid == 10 ? (ty > 0 ? tile - fs.ntz : -1)
                                     : (ty < fs.nty - 1 ? tile + fs.ntz : -1);
            if (nt >= 0) wu = max(c - 4, 0) * ntile + nt;
        }
        if (wu >= 0) ok = fused_wait(fs.flags + wu, epoch);
        __threadfence();
    }
    if (!__syncthreads_and(ok)) {
        if (tid == 0) atomicExch(&g_fused_status, 1);
        return;
    }
    if (!ok_cell) return;
    // phase 2: stresses, memory variables, free surface of plane F + c
    // (velocity reads through L2)
    const int gx = F + c;
    const i64 iv = gx * sx + (i64)gy * sy + gz0;
    const i64 ip = ((i64)(gx - F) * g.ny + (gy - F)) * g.nz + (gz0 - F);
    s3d_q4_at<L, float, 2>(g, f, gz0, gy, gx, iv, ip, g.freesurf != 0);
}

FusedShape fused_shape(const Grid &g)
{
    FusedShape s{0, 0, 0, 0};
    if (!g.fused || g.nd != 3 || g.F != 4 || g.nz % 4 || g.fhalf || g.L < 0 || g.L > 3 || g.kernels != 0) return s;
    const int ntz = (g.nz + FZ - 1) / FZ, nty = (g.ny + FY - 1) / FY, nch = g.nx;
    if (g.nx < 5 || (int64_t)ntz * nty * nch > (1 << 30)) return s;
    s.ntz = ntz;
    s.nty = nty;
    s.nchunk = nch;
    s.units = (int64_t)ntz * nty * nch;
    return s;
}

bool launch_fused_step(const Grid &g, const Fields &f, int *sync, int t, cudaStream_t st)
{
    const FusedShape sh = fused_shape(g);
    if (!sh.units || g.nb != 1 || !sync) return false;
    FusedSync fs{reinterpret_cast<unsigned *>(sync), sync + 1, (unsigned)((uint64_t)t * (uint64_t)sh.units),
                 sh.ntz, sh.nty, (int)sh.units};
    const dim3 b(8, FY, 1);
    const unsigned gr = (unsigned)sh.units;
    switch (g.L) {
    case 0: k_fused3d_q4<0><<<gr, b, 0, st>>>(g, f, fs, t + 1); break;
    case 1: k_fused3d_q4<1><<<gr, b, 0, st>>>(g, f, fs, t + 1); break;
    case 2: k_fused3d_q4<2><<<gr, b, 0, st>>>(g, f, fs, t + 1); break;
    default: k_fused3d_q4<3><<<gr, b, 0, st>>>(g, f, fs, t + 1); break;
    }
    return true;
}

int fused_take_status()
{
    int v = 0, zero = 0;
    if (cudaMemcpyFromSymbol(&v, g_fused_status, sizeof(int)) != cudaSuccess) return -1;
    if (v) cudaMemcpyToSymbol(g_fused_status, &zero, sizeof(int));
    return v;
}

// ------------------------------------------- 4-cell vectorised 3D adjoint
// The adjoint kernels of k_adjv3d / k_adjs3d on quads of z cells, with the
// same per-cell arithmetic: backpropagation of the forward field (not for
// the DFT gradient, g.bp2), saved-boundary injection per cell, the adjoint
// update with CPML, and the on-the-fly gradient accumulated in FP64.
__device__ __forceinline__ void grad_add4(double *g, i64 ip, const float (&d)[4])
{
    double2 *p = reinterpret_cast<double2 *>(g + ip);
    double2 a = p[0], b = p[1];
    a.x += (double)d[0]; a.y += (double)d[1]; b.x += (double)d[2]; b.y += (double)d[3];
    p[0] = a;
    p[1] = b;
}

// L2 prefetch of one quad's cell in a per-cell stream
__device__ __forceinline__ void pf_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// PF (single-shot launches of the default selection): the thread first asks
// L2 for its quad's per-cell streams -- the forward and adjoint velocities,
// the buoyancies and the density gradient sum -- and the launch takes 3 CTAs
// per SM, as k_s3d_q4_pf does for the forward stress update.
template <typename T, bool MB = false, bool PF = false>
__global__ void __launch_bounds__(128, PF ? 3 : 1) k_adjv3d_q4(Grid g, Fields f, AdjFields a)
{
    CELL3D_Q4
    if (MB) shot_adj(g, a, shot);
    if constexpr (PF) {
        const bool recon = !g.ckpt && !g.bp2;
#pragma unroll
        for (int q = VX; q <= VZ; q++) {
            pf_l2(a.wr[q] + iv);
            if (recon) pf_l2(f.w[q] + iv);
        }
        pf_l2(f.p[PRIP] + ip); pf_l2(f.p[PRJP] + ip); pf_l2(f.p[PRKP] + ip);
        if (!g.bp2) pf_l2(a.grad[GRHO] + ip);
    }
    const float *hc = g.hc;
    const Q4 rip = ldq(f.p[PRIP] + ip), rjp = ldq(f.p[PRJP] + ip), rkp = ldq(f.p[PRKP] + ip);
    Q4 vx = {{0, 0, 0, 0}}, vy = vx, vz = vx;
    if (g.ckpt) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            vx.v[j] = fwd_at<T>(g, a, VX, iv + j);
            vy.v[j] = fwd_at<T>(g, a, VY, iv + j);
            vz.v[j] = fwd_at<T>(g, a, VZ, iv + j);
        }
    } else if (!g.bp2) {  // backpropagate the forward velocities (update_adjv3D.cl:297-340)
        Q4 szz_z = dfw_z<F>(ldw(f.w[SZZ], iv), hc);
        Q4 sxx_x = dfw_q<F>(f.w[SXX], iv, sx, hc);
        Q4 sxz_x = dbw_q<F>(f.w[SXZ], iv, sx, hc);
        Q4 sxz_z = dbw_z<F>(ldw(f.w[SXZ], iv), hc);
        Q4 syz_y = dbw_q<F>(f.w[SYZ], iv, sy, hc);
        Q4 syz_z = dbw_z<F>(ldw(f.w[SYZ], iv), hc);
        Q4 syy_y = dfw_q<F>(f.w[SYY], iv, sy, hc);
        Q4 sxy_x = dbw_q<F>(f.w[SXY], iv, sx, hc);
        Q4 sxy_y = dbw_q<F>(f.w[SXY], iv, sy, hc);
        vx = ldq_rw(f.w[VX] + iv); vy = ldq_rw(f.w[VY] + iv); vz = ldq_rw(f.w[VZ] + iv);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            vx.v[j] = vx.v[j] - (sxx_x.v[j] + sxy_y.v[j] + sxz_z.v[j]) * rip.v[j];
            vy.v[j] = vy.v[j] - (syy_y.v[j] + sxy_x.v[j] + syz_z.v[j]) * rjp.v[j];
            vz.v[j] = vz.v[j] - (szz_z.v[j] + sxz_x.v[j] + syz_y.v[j]) * rkp.v[j];
            const int m = inject_ind3d(g, gz0 + j, gy, gx);
            if (m != -1) {
                vx.v[j] = bnd_at<T>(g, a, VX, m);
                vy.v[j] = bnd_at<T>(g, a, VY, m);
                vz.v[j] = bnd_at<T>(g, a, VZ, m);
            }
        }
        stq(f.w[VX] + iv, vx); stq(f.w[VY] + iv, vy); stq(f.w[VZ] + iv, vz);
    }
    Q4 szz_zr = dfw_z<F>(ldw(a.wr[SZZ], iv), hc);
    Q4 sxx_xr = dfw_q<F>(a.wr[SXX], iv, sx, hc);
    Q4 sxz_xr = dbw_q<F>(a.wr[SXZ], iv, sx, hc);
    Q4 sxz_zr = dbw_z<F>(ldw(a.wr[SXZ], iv), hc);
    Q4 syz_yr = dbw_q<F>(a.wr[SYZ], iv, sy, hc);
    Q4 syz_zr = dbw_z<F>(ldw(a.wr[SYZ], iv), hc);
    Q4 syy_yr = dfw_q<F>(a.wr[SYY], iv, sy, hc);
    Q4 sxy_xr = dbw_q<F>(a.wr[SXY], iv, sx, hc);
    Q4 sxy_yr = dbw_q<F>(a.wr[SXY], iv, sy, hc);
    if (g.abs_type == 1)
        cpml_v3d_q4(g, f, gz0, gy, gx, sxx_xr, syy_yr, szz_zr, sxy_yr, sxy_xr, syz_yr, syz_zr, sxz_xr, sxz_zr);
    Q4 wx = ldq_rw(a.wr[VX] + iv), wy = ldq_rw(a.wr[VY] + iv), wz = ldq_rw(a.wr[VZ] + iv);
    float gr[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const float lvx = (sxx_xr.v[j] + sxy_yr.v[j] + sxz_zr.v[j]) * rip.v[j];
        const float lvy = (syy_yr.v[j] + sxy_xr.v[j] + syz_zr.v[j]) * rjp.v[j];
        const float lvz = (szz_zr.v[j] + sxz_xr.v[j] + syz_yr.v[j]) * rkp.v[j];
        float w3[3] = {wx.v[j] + lvx, wy.v[j] + lvy, wz.v[j] + lvz};
        if (g.abs_type == 2) taper_regs<3>(g, f.taper, gz0 + j, gy, gx, w3);
        wx.v[j] = w3[0]; wy.v[j] = w3[1]; wz.v[j] = w3[2];
        gr[j] = -vx.v[j] * lvx - vy.v[j] * lvy - vz.v[j] * lvz;
    }
    stq(a.wr[VX] + iv, wx); stq(a.wr[VY] + iv, wy); stq(a.wr[VZ] + iv, wz);
    if (!g.bp2) grad_add4(a.grad[GRHO], ip, gr);
}

// CPML of the adjoint stress update (cpml_s3d with adjoint_form): as
// cpml_s3d_q4, except that a cell in both z slabs or both y slabs takes
// only the first (else-if), as update_adjs3D.cl does
__device__ __forceinline__ void cpml_s3d_adj_q4(const Grid &g, const Fields &f, int gz0, int gy, int gx, Q4 &vxx,
                                                Q4 &vxy, Q4 &vxz, Q4 &vyx, Q4 &vyy, Q4 &vyz, Q4 &vzx, Q4 &vzy,
                                                Q4 &vzz)
{
    const int F = g.F, NAB = g.nab, NZ = g.NZ, NY = g.NY, NX = g.NX;
    const i64 nz = g.nz, ny = g.ny;
    const bool zq = NAB % 4 == 0 && g.nz >= 2 * NAB + 4;
    if (zq && gz0 > NZ - NAB - F - 1) {
        i64 i = gx - F, jj = gy - F, k = gz0 - NZ + NAB + F + NAB;
        int ind = 2 * NAB - 1 - (int)k;
        i64 q = (i * ny + jj) * (2 * NAB) + k;
        cpml_zq(f.psi[PVX_Z], q, f.kinv[2][1], f.cz[CAH], f.cz[CBH], ind, -1, vxz);
        cpml_zq(f.psi[PVY_Z], q, f.kinv[2][1], f.cz[CAH], f.cz[CBH], ind, -1, vyz);
        cpml_zq(f.psi[PVZ_Z], q, f.kinv[2][0], f.cz[CA], f.cz[CB], ind + 1, -1, vzz);
    } else if (zq && !g.freesurf && gz0 - F < NAB) {
        i64 i = gx - F, jj = gy - F, k = gz0 - F;
        i64 q = (i * ny + jj) * (2 * NAB) + k;
        cpml_zq(f.psi[PVX_Z], q, f.kinv[2][1], f.cz[CAH], f.cz[CBH], (int)k, 1, vxz);
        cpml_zq(f.psi[PVY_Z], q, f.kinv[2][1], f.cz[CAH], f.cz[CBH], (int)k, 1, vyz);
        cpml_zq(f.psi[PVZ_Z], q, f.kinv[2][0], f.cz[CA], f.cz[CB], (int)k, 1, vzz);
    } else if (!zq && (gz0 + 3 > NZ - NAB - F - 1 || (!g.freesurf && gz0 - F < NAB))) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int gz = gz0 + j;
            const bool zb = gz > NZ - NAB - F - 1;
            if (zb) {
                i64 i = gx - F, jj = gy - F, k = gz - NZ + NAB + F + NAB;
                int ind = 2 * NAB - 1 - (int)k;
                i64 q = (i * ny + jj) * (2 * NAB) + k;
                cpml(f.psi[PVX_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, vxz.v[j]);
                cpml(f.psi[PVY_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, vyz.v[j]);
                cpml(f.psi[PVZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], ind + 1, vzz.v[j]);
            } else if (!g.freesurf && gz - F < NAB) {
                i64 i = gx - F, jj = gy - F, k = gz - F;
                i64 q = (i * ny + jj) * (2 * NAB) + k;
                cpml(f.psi[PVX_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], (int)k, vxz.v[j]);
                cpml(f.psi[PVY_Z], q, f.cz[CKH], f.cz[CAH], f.cz[CBH], (int)k, vyz.v[j]);
                cpml(f.psi[PVZ_Z], q, f.cz[CK], f.cz[CA], f.cz[CB], (int)k, vzz.v[j]);
            }
        }
    }
    const i64 k0 = gz0 - F;
    if (gy - F < NAB) {
        i64 i = gx - F, j = gy - F;
        i64 q = (i * (2 * NAB) + j) * nz + k0;
        cpml_q(f.psi[PVX_Y], q, f.kinv[1][1], f.cy[CAH], f.cy[CBH], (int)j, vxy);
        cpml_q(f.psi[PVY_Y], q, f.kinv[1][0], f.cy[CA], f.cy[CB], (int)j, vyy);
        cpml_q(f.psi[PVZ_Y], q, f.kinv[1][1], f.cy[CAH], f.cy[CBH], (int)j, vzy);
    } else if (gy > NY - NAB - F - 1) {
        i64 i = gx - F, j = gy - NY + NAB + F + NAB;
        int ind = 2 * NAB - 1 - (int)j;
        i64 q = (i * (2 * NAB) + j) * nz + k0;
        cpml_q(f.psi[PVX_Y], q, f.kinv[1][1], f.cy[CAH], f.cy[CBH], ind, vxy);
        cpml_q(f.psi[PVY_Y], q, f.kinv[1][0], f.cy[CA], f.cy[CB], ind + 1, vyy);
        cpml_q(f.psi[PVZ_Y], q, f.kinv[1][1], f.cy[CAH], f.cy[CBH], ind, vzy);
    }
    if (gx - F < NAB) {
        i64 i = gx - F, j = gy - F;
        i64 q = (i * ny + j) * nz + k0;
        cpml_q(f.psi[PVX_X], q, f.kinv[0][0], f.cx[CA], f.cx[CB], (int)i, vxx);
        cpml_q(f.psi[PVY_X], q, f.kinv[0][1], f.cx[CAH], f.cx[CBH], (int)i, vyx);
        cpml_q(f.psi[PVZ_X], q, f.kinv[0][1], f.cx[CAH], f.cx[CBH], (int)i, vzx);
    }
    if (gx > NX - NAB - F - 1) {
        i64 i = gx - NX + NAB + F + NAB, j = gy - F;
        int ind = 2 * NAB - 1 - (int)i;
        i64 q = (i * ny + j) * nz + k0;
        cpml_q(f.psi[PVX_X], q, f.kinv[0][0], f.cx[CA], f.cx[CB], ind + 1, vxx);
        cpml_q(f.psi[PVY_X], q, f.kinv[0][1], f.cx[CAH], f.cx[CBH], ind, vyx);
        cpml_q(f.psi[PVZ_X], q, f.kinv[0][1], f.cx[CAH], f.cx[CBH], ind, vzx);
    }
}

// PF: prefetch of the quad's per-cell streams (forward and adjoint stresses
// and memory variables, parameters, the M and mu gradient sums) and 3 CTAs
// per SM, as k_adjv3d_q4.  The saved-boundary index of each cell of the quad
// is found once and kept for the four phases.
template <int L, typename T, bool MB = false, bool PF = false>
__global__ void __launch_bounds__(128, PF ? 3 : 4) k_adjs3d_q4(Grid g, Fields f, AdjFields a)
{
    CELL3D_Q4
    if (MB) shot_adj(g, a, shot);
    const bool recon = !g.ckpt && !g.bp2;
    if constexpr (PF) {
#pragma unroll
        for (int q = SXX; q <= SXZ; q++) {
            pf_l2(a.wr[q] + iv);
            if (recon) pf_l2(f.w[q] + iv);
        }
#pragma unroll
        for (int l = 0; l < L; l++)
#pragma unroll
            for (int q = 0; q < NR; q++) {
                pf_l2(a.rr[q] + l * g.nvol + iv);
                if (recon) pf_l2(f.r[q] + l * g.nvol + iv);
            }
        constexpr int np = L > 0 ? 10 : 5;
        constexpr int pid[10] = {PM, PMU, PMUIPJP, PMUJPKP, PMUIPKP, PTAUP, PTAUS, PTAUSIPJP, PTAUSJPKP, PTAUSIPKP};
#pragma unroll
        for (int k = 0; k < np; k++) pf_l2(f.p[pid[k]] + ip);
        if (!g.bp2) {
            pf_l2(a.grad[GM] + ip);
            if (g.restype == 0) pf_l2(a.grad[GMU] + ip);
        }
    }
    int mq[4] = {-1, -1, -1, -1};
    if (recon) {
#pragma unroll
        for (int j = 0; j < 4; j++) mq[j] = inject_ind3d(g, gz0 + j, gy, gx);
    }
    const float *hc = g.hc;
    // adjoint velocity derivatives, with CPML
    Q4 vzzr = dbw_z<F>(ldw(a.wr[VZ], iv), hc), vyzr = dfw_z<F>(ldw(a.wr[VY], iv), hc);
    Q4 vxzr = dfw_z<F>(ldw(a.wr[VX], iv), hc);
    Q4 vzxr = dfw_q<F>(a.wr[VZ], iv, sx, hc), vzyr = dfw_q<F>(a.wr[VZ], iv, sy, hc);
    Q4 vyxr = dfw_q<F>(a.wr[VY], iv, sx, hc), vyyr = dbw_q<F>(a.wr[VY], iv, sy, hc);
    Q4 vxxr = dbw_q<F>(a.wr[VX], iv, sx, hc), vxyr = dfw_q<F>(a.wr[VX], iv, sy, hc);
    if (g.abs_type == 1) cpml_s3d_adj_q4(g, f, gz0, gy, gx, vxxr, vxyr, vxzr, vyxr, vyyr, vyzr, vzxr, vzyr, vzzr);
    Q4 rsh[3];   // adjoint shear sums vxy+vyx, vyz+vzy, vxz+vzx
#pragma unroll
    for (int j = 0; j < 4; j++) {
        rsh[0].v[j] = vxyr.v[j] + vyxr.v[j];
        rsh[1].v[j] = vyzr.v[j] + vzyr.v[j];
        rsh[2].v[j] = vxzr.v[j] + vzxr.v[j];
    }
    const Q4 qM = ldq(f.p[PM] + ip), qmu = ldq(f.p[PMU] + ip);
    float gM[4] = {0, 0, 0, 0}, gmu[4] = {0, 0, 0, 0};

    // ---- normal stresses (sxx, syy, szz) with rxx, ryy, rzz: the forward
    // reconstruction of the quad, then its adjoint update
    {
        const int wid[3] = {SXX, SYY, SZZ}, rid[3] = {RXX, RYY, RZZ};
        Q4 qtaup = {{0, 0, 0, 0}}, qtaus = qtaup;
        if (L > 0) { qtaup = ldq(f.p[PTAUP] + ip); qtaus = ldq(f.p[PTAUS] + ip); }
        Q4 s3[3] = {{{0, 0, 0, 0}}, {{0, 0, 0, 0}}, {{0, 0, 0, 0}}};
        if (g.ckpt) {
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int j = 0; j < 4; j++) s3[c].v[j] = fwd_at<T>(g, a, wid[c], iv + j);
        } else if (!g.bp2) {
            const Q4 vzz = dbw_z<F>(ldw(f.w[VZ], iv), hc);
            const Q4 vyy = dbw_q<F>(f.w[VY], iv, sy, hc);
            const Q4 vxx = dbw_q<F>(f.w[VX], iv, sx, hc);
#pragma unroll
            for (int c = 0; c < 3; c++) s3[c] = ldq_rw(f.w[wid[c]] + iv);
            Q4 rf[3][L > 0 ? L : 1];
            if constexpr (L > 0) {
#pragma unroll
                for (int c = 0; c < 3; c++)
#pragma unroll
                    for (int l = 0; l < L; l++) rf[c][l] = ldq_rw(f.r[rid[c]] + l * g.nvol + iv);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float lM = qM.v[j], lmu = qmu.v[j];
                float gm = lM, fm = 2.0f * lmu, d = 0, e = 0;
                if (L > 0) {
                    const float ltaup = qtaup.v[j], ltaus = qtaus.v[j];
                    gm = lM * (1.0f + (float)L * ltaup);
                    fm = 2.0f * lmu * (1.0f + (float)L * ltaus);
                    d = 2.0f * lmu * ltaus / g.dt; e = lM * ltaup / g.dt;
                }
                const float vxxyyzz = vxx.v[j] + vyy.v[j] + vzz.v[j], vyyzz = vyy.v[j] + vzz.v[j];
                const float vxxzz = vxx.v[j] + vzz.v[j], vxxyy = vxx.v[j] + vyy.v[j];
                const float fw[3] = {gm * vxxyyzz - fm * vyyzz, gm * vxxyyzz - fm * vxxzz, gm * vxxyyzz - fm * vxxyy};
                if (L == 0) {
#pragma unroll
                    for (int c = 0; c < 3; c++) s3[c].v[j] -= fw[c];
                } else {
                    const float dc[3] = {e * vxxyyzz - d * vyyzz, e * vxxyyzz - d * vxxzz, e * vxxyyzz - d * vxxyy};
#pragma unroll
                    for (int c = 0; c < 3; c++) {
                        float aa = 0;
#pragma unroll
                        for (int l = 0; l < L; l++) aa += rf[c][l].v[j];
                        const float ls = fw[c] + g.dt2 * aa;
                        aa = 0;
                        // 3D reconstruction keeps the forward-time coefficients (update_adjs3D.cl:357-359)
#pragma unroll
                        for (int l = 0; l < L; l++) {
                            const float el = g.eta[l];
                            const float b = 1.0f / (1.0f + el * 0.5f), cc = 1.0f - el * 0.5f;
                            aa += b * (rf[c][l].v[j] * cc - el * dc[c]);
                        }
                        s3[c].v[j] -= ls + g.dt2 * aa;
                    }
                }
                const int m = mq[j];
                if (m != -1) {
                    s3[0].v[j] = bnd_at<T>(g, a, SXX, m);
                    s3[1].v[j] = bnd_at<T>(g, a, SYY, m);
                    s3[2].v[j] = bnd_at<T>(g, a, SZZ, m);
                }
            }
#pragma unroll
            for (int c = 0; c < 3; c++) stq(f.w[wid[c]] + iv, s3[c]);
        }
        Q4 rr[3][L > 0 ? L : 1];
        if constexpr (L > 0) {
#pragma unroll
            for (int c = 0; c < 3; c++)
#pragma unroll
                for (int l = 0; l < L; l++) rr[c][l] = ldq_rw(a.rr[rid[c]] + l * g.nvol + iv);
        }
        Q4 w3[3];
#pragma unroll
        for (int c = 0; c < 3; c++) w3[c] = ldq_rw(a.wr[wid[c]] + iv);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float lM = qM.v[j], lmu = qmu.v[j];
            float gm = lM, fm = 2.0f * lmu, d = 0, e = 0;
            if (L > 0) {
                const float ltaup = qtaup.v[j], ltaus = qtaus.v[j];
                gm = lM * (1.0f + (float)L * ltaup);
                fm = 2.0f * lmu * (1.0f + (float)L * ltaus);
                d = 2.0f * lmu * ltaus / g.dt; e = lM * ltaup / g.dt;
            }
            const float vxxyyzzr = vxxr.v[j] + vyyr.v[j] + vzzr.v[j], vyyzzr = vyyr.v[j] + vzzr.v[j];
            const float vxxzzr = vxxr.v[j] + vzzr.v[j], vxxyyr = vxxr.v[j] + vyyr.v[j];
            float ls[3] = {gm * vxxyyzzr - fm * vyyzzr, gm * vxxyyzzr - fm * vxxzzr, gm * vxxyyzzr - fm * vxxyyr};
            if (L == 0) {
#pragma unroll
                for (int c = 0; c < 3; c++) w3[c].v[j] += ls[c];
            } else {
                const float dc[3] = {e * vxxyyzzr - d * vyyzzr, e * vxxyyzzr - d * vxxzzr, e * vxxyyzzr - d * vxxyyr};
#pragma unroll
                for (int c = 0; c < 3; c++) {
                    float aa = 0;
#pragma unroll
                    for (int l = 0; l < L; l++) aa += rr[c][l].v[j];
                    ls[c] += g.dt2 * aa;
                    // stored into the forward memory variables; the sum keeps the
                    // last adjoint value (update_adjs3D.cl:566-583); in the DFT
                    // adjoint both are one buffer, so that value is the new one
#pragma unroll
                    for (int l = 0; l < L; l++) {
                        const float el = g.eta[l];
                        const float b = 1.0f / (1.0f + el * 0.5f), cc = 1.0f - el * 0.5f;
                        const float n = b * (rr[c][l].v[j] * cc - el * dc[c]);
                        aa = g.bp2 ? n : rr[c][l].v[j];
                        rr[c][l].v[j] = n;
                    }
                    w3[c].v[j] += ls[c] + g.dt2 * aa;
                }
            }
            if (!g.bp2 && g.restype == 0) {
                const float c1 = 1.0f / (3.0f * lM - 4.0f * lmu) / (3.0f * lM - 4.0f * lmu);
                const float c3 = 1.0f / lmu / lmu;
                const float c5 = 1.0f / 6.0f * c3;
                const float sxx = s3[0].v[j], syy = s3[1].v[j], szz = s3[2].v[j];
                const float dM = c1 * (sxx + syy + szz) * (ls[0] + ls[1] + ls[2]);
                gM[j] = -dM;
                gmu[j] = 4.0f / 3.0f * dM - c5 * (ls[0] * (2.0f * sxx - syy - szz) + ls[1] * (2.0f * syy - sxx - szz) +
                                                  ls[2] * (2.0f * szz - sxx - syy));
            } else if (!g.bp2) {
                gM[j] = -((s3[0].v[j] + s3[1].v[j] + s3[2].v[j]) * (ls[0] + ls[1] + ls[2]));
            }
        }
        // the new adjoint memory values go to the forward arrays; a
        // checkpointed adjoint reloads those from a snapshot before they are
        // read again, so it skips the stores (its forward arrays may also be
        // FP16)
        if constexpr (L > 0) {
            if (!g.ckpt) {
#pragma unroll
                for (int c = 0; c < 3; c++)
#pragma unroll
                    for (int l = 0; l < L; l++) stq(f.r[rid[c]] + l * g.nvol + iv, rr[c][l]);
            }
        }
        if (g.abs_type == 2) {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float t3[3] = {w3[0].v[j], w3[1].v[j], w3[2].v[j]};
                taper_regs<3>(g, f.taper, gz0 + j, gy, gx, t3);
#pragma unroll
                for (int c = 0; c < 3; c++) w3[c].v[j] = t3[c];
            }
        }
#pragma unroll
        for (int c = 0; c < 3; c++) stq(a.wr[wid[c]] + iv, w3[c]);
    }

    // ---- shear stresses, one at a time: sxy (x,y), syz (y,z), sxz (x,z)
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const int wid = c == 0 ? SXY : (c == 1 ? SYZ : SXZ);
        const int rid = c == 0 ? RXY : (c == 1 ? RYZ : RXZ);
        const int pmu = c == 0 ? PMUIPJP : (c == 1 ? PMUJPKP : PMUIPKP);
        const int ptau = c == 0 ? PTAUSIPJP : (c == 1 ? PTAUSJPKP : PTAUSIPKP);
        const Q4 qmuc = ldq(f.p[pmu] + ip);
        Q4 qtauc = {{0, 0, 0, 0}};
        if (L > 0) qtauc = ldq(f.p[ptau] + ip);
        Q4 sc = {{0, 0, 0, 0}};
        if (g.ckpt) {
#pragma unroll
            for (int j = 0; j < 4; j++) sc.v[j] = fwd_at<T>(g, a, wid, iv + j);
        } else if (!g.bp2) {
            Q4 d1, d2;   // forward derivative pair (vxy+vyx, vyz+vzy, vxz+vzx)
            if (c == 0) { d1 = dfw_q<F>(f.w[VX], iv, sy, hc); d2 = dfw_q<F>(f.w[VY], iv, sx, hc); }
            else if (c == 1) { d1 = dfw_z<F>(ldw(f.w[VY], iv), hc); d2 = dfw_q<F>(f.w[VZ], iv, sy, hc); }
            else { d1 = dfw_z<F>(ldw(f.w[VX], iv), hc); d2 = dfw_q<F>(f.w[VZ], iv, sx, hc); }
            sc = ldq_rw(f.w[wid] + iv);
            Q4 rf[L > 0 ? L : 1];
            if constexpr (L > 0) {
#pragma unroll
                for (int l = 0; l < L; l++) rf[l] = ldq_rw(f.r[rid] + l * g.nvol + iv);
            }
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float fsum = d1.v[j] + d2.v[j];
                const float lmuc = qmuc.v[j];
                if (L == 0) {
                    sc.v[j] -= lmuc * fsum;
                } else {
                    const float lt = qtauc.v[j];
                    const float fc = lmuc * (1.0f + (float)L * lt), dc = lmuc * lt / g.dt;
                    float aa = 0;
#pragma unroll
                    for (int l = 0; l < L; l++) aa += rf[l].v[j];
                    const float ls = fc * fsum + g.dt2 * aa;
                    aa = 0;
#pragma unroll
                    for (int l = 0; l < L; l++) {
                        const float el = g.eta[l];
                        const float b = 1.0f / (1.0f + el * 0.5f), cc = 1.0f - el * 0.5f;
                        aa += b * (rf[l].v[j] * cc - el * (dc * fsum));
                    }
                    sc.v[j] -= ls + g.dt2 * aa;
                }
                const int m = mq[j];
                if (m != -1) sc.v[j] = bnd_at<T>(g, a, wid, m);
            }
            stq(f.w[wid] + iv, sc);
        }
        const Q4 rsum = rsh[c];
        Q4 rr[L > 0 ? L : 1];
        if constexpr (L > 0) {
#pragma unroll
            for (int l = 0; l < L; l++) rr[l] = ldq_rw(a.rr[rid] + l * g.nvol + iv);
        }
        Q4 wc = ldq_rw(a.wr[wid] + iv);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const float lmuc = qmuc.v[j];
            float fc = lmuc, dc = 0;
            if (L > 0) {
                const float lt = qtauc.v[j];
                fc = lmuc * (1.0f + (float)L * lt);
                dc = lmuc * lt / g.dt;
            }
            float ls = fc * rsum.v[j];
            if (L == 0) {
                wc.v[j] += ls;
            } else {
                float aa = 0;
#pragma unroll
                for (int l = 0; l < L; l++) aa += rr[l].v[j];
                ls += g.dt2 * aa;
#pragma unroll
                for (int l = 0; l < L; l++) {
                    const float el = g.eta[l];
                    const float b = 1.0f / (1.0f + el * 0.5f), cc = 1.0f - el * 0.5f;
                    const float n = b * (rr[l].v[j] * cc - el * (dc * rsum.v[j]));
                    aa = g.bp2 ? n : rr[l].v[j];
                    rr[l].v[j] = n;
                }
                wc.v[j] += ls + g.dt2 * aa;
            }
            if (!g.bp2 && g.restype == 0) {
                const float lmu = qmu.v[j];
                const float c3 = 1.0f / lmu / lmu;
                gmu[j] += -c3 * (sc.v[j] * ls);
            }
        }
        if constexpr (L > 0) {
#pragma unroll
            for (int l = 0; l < L; l++) stq(f.r[rid] + l * g.nvol + iv, rr[l]);
        }
        if (g.abs_type == 2) {
#pragma unroll
            for (int j = 0; j < 4; j++) {
                float t1[1] = {wc.v[j]};
                taper_regs<1>(g, f.taper, gz0 + j, gy, gx, t1);
                wc.v[j] = t1[0];
            }
        }
        stq(a.wr[wid] + iv, wc);
    }
    if (!g.bp2) {
        grad_add4(a.grad[GM], ip, gM);
        if (g.restype == 0) grad_add4(a.grad[GMU], ip, gmu);
    }
}

// true when the 4-cell kernels apply to this grid
static inline bool q4_ok(const Grid &g) { return g.nd == 3 && g.F == 4 && g.nz % 4 == 0; }

// Programmatic dependent launch for the single-shot 3D loop: the stress
// kernel, the sources and the receivers are launched with programmatic
// stream serialization, so each may be resident while the previous one
// drains its last wave (and the stress kernel asks L2 for its own streams
// meanwhile); every one of them waits (pdl_wait) before it reads or writes
// anything the previous kernels touch, and reads those fields with plain
// loads (a read-only-path load may be hoisted above the wait).  The
// velocity kernel is an ordinary launch that triggers its dependents
// early.  256^3, L=2: 1.004 against 1.015 ms per step.  The same for the
// 2D P-SV loop (velocity and fused stress-step kernels, 300 x 400) was
// slower, 7.17 against 7.39 Gcell/s, and is not done.  On unless the
// environment sets SEISCL_B200_PDL=0.
static bool pdl_enabled()
{
    static const bool on = [] {
        const char *e = std::getenv("SEISCL_B200_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

template <typename... KArgs, typename... Args>
static void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args &&...args)
{
    cudaLaunchConfig_t c = {};
    c.gridDim = grid;
    c.blockDim = block;
    c.dynamicSmemBytes = 0;
    c.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    c.attrs = at;
    c.numAttrs = 1;
    cudaLaunchKernelEx(&c, kernel, std::forward<Args>(args)...);
}

// kernel<<<grid, block, 0, st>>>(args...), with programmatic serialization when `pdl`
template <typename... KArgs, typename... Args>
static void launch_maybe_pdl(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st,
                             Args &&...args)
{
    if (pdl) launch_pdl(kernel, grid, block, st, std::forward<Args>(args)...);
    else kernel<<<grid, block, 0, st>>>(std::forward<Args>(args)...);
}

template <int F, int L, class T = float, bool MB = false>
__global__ void __launch_bounds__(256, 2) k_s3d_stream(Grid g, Fields f)
{
    CELL3D
    const float *hc = g.hc;
    // per-cell streams first: stresses, memory variables, parameters
    T *ws[6] = {fld<T>(f.w[SXY]), fld<T>(f.w[SYZ]), fld<T>(f.w[SXZ]),
                fld<T>(f.w[SXX]), fld<T>(f.w[SYY]), fld<T>(f.w[SZZ])};
    T *wr[6] = {fld<T>(f.r[RXY]), fld<T>(f.r[RYZ]), fld<T>(f.r[RXZ]),
                fld<T>(f.r[RXX]), fld<T>(f.r[RYY]), fld<T>(f.r[RZZ])};
    float s[6];
#pragma unroll
    for (int q = 0; q < 6; q++) s[q] = ldgv(ws[q] + iv);
    float r[6][L > 0 ? L : 1];
#pragma unroll
    for (int l = 0; l < L; l++) {
        const i64 ir = l * g.nvol + iv;
#pragma unroll
        for (int q = 0; q < 6; q++) r[q][l] = ldgv(wr[q] + ir);
    }
    const float lM = __ldg(f.p[PM] + ip), lmu = __ldg(f.p[PMU] + ip);
    const float lmuipkp = __ldg(f.p[PMUIPKP] + ip), lmuipjp = __ldg(f.p[PMUIPJP] + ip),
                lmujpkp = __ldg(f.p[PMUJPKP] + ip);
    float ltaup = 0, ltaus = 0, ltausipkp = 0, ltausipjp = 0, ltausjpkp = 0;
    if (L > 0) {
        ltaup = __ldg(f.p[PTAUP] + ip); ltaus = __ldg(f.p[PTAUS] + ip);
        ltausipkp = __ldg(f.p[PTAUSIPKP] + ip); ltausipjp = __ldg(f.p[PTAUSIPJP] + ip);
        ltausjpkp = __ldg(f.p[PTAUSJPKP] + ip);
    }
    const T *Vx = fld<T>(f.w[VX]), *Vy = fld<T>(f.w[VY]), *Vz = fld<T>(f.w[VZ]);
    float vzx = dfwT<F>(Vz, iv, sx, hc), vzy = dfwT<F>(Vz, iv, sy, hc), vzz = dbwT<F>(Vz, iv, 1, hc);
    float vyx = dfwT<F>(Vy, iv, sx, hc), vyy = dbwT<F>(Vy, iv, sy, hc), vyz = dfwT<F>(Vy, iv, 1, hc);
    float vxx = dbwT<F>(Vx, iv, sx, hc), vxy = dfwT<F>(Vx, iv, sy, hc), vxz = dfwT<F>(Vx, iv, 1, hc);
    if (g.abs_type == 1) cpml_s3d(g, f, gz, gy, gx, vxx, vxy, vxz, vyx, vyy, vyz, vzx, vzy, vzz, false);
    float vxyyx = vxy + vyx, vyzzy = vyz + vzy, vxzzx = vxz + vzx;
    float vxxyyzz = vxx + vyy + vzz, vyyzz = vyy + vzz, vxxzz = vxx + vzz, vxxyy = vxx + vyy;
    if (L == 0) {
        float gm = lM, fm = 2.0f * lmu;
        s[0] += lmuipjp * vxyyx;
        s[1] += lmujpkp * vyzzy;
        s[2] += lmuipkp * vxzzx;
        s[3] += gm * vxxyyzz - fm * vyyzz;
        s[4] += gm * vxxyyzz - fm * vxxzz;
        s[5] += gm * vxxyyzz - fm * vxxyy;
    } else {
        float fipjp = lmuipjp * (1.0f + (float)L * ltausipjp);
        float fjpkp = lmujpkp * (1.0f + (float)L * ltausjpkp);
        float fipkp = lmuipkp * (1.0f + (float)L * ltausipkp);
        float gm = lM * (1.0f + (float)L * ltaup);
        float fm = 2.0f * lmu * (1.0f + (float)L * ltaus);
        float dipjp = lmuipjp * ltausipjp / g.dt, djpkp = lmujpkp * ltausjpkp / g.dt, dipkp = lmuipkp * ltausipkp / g.dt;
        float d = 2.0f * lmu * ltaus / g.dt, e = lM * ltaup / g.dt;
        float a[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
        for (int l = 0; l < L; l++)
#pragma unroll
            for (int q = 0; q < 6; q++) a[q] += r[q][l];
        float ls[6] = {fipjp * vxyyx + g.dt2 * a[0], fjpkp * vyzzy + g.dt2 * a[1], fipkp * vxzzx + g.dt2 * a[2],
                       (gm * vxxyyzz - fm * vyyzz) + g.dt2 * a[3], (gm * vxxyyzz - fm * vxxzz) + g.dt2 * a[4],
                       (gm * vxxyyzz - fm * vxxyy) + g.dt2 * a[5]};
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
            const i64 ir = l * g.nvol + iv;
#pragma unroll
            for (int q = 0; q < 6; q++) stv(wr[q] + ir, r[q][l]);
        }
#pragma unroll
        for (int q = 0; q < 6; q++) s[q] += ls[q] + g.dt2 * a[q];
    }
    if (g.abs_type == 2) taper_regs<6>(g, f.taper, gz, gy, gx, s);
#pragma unroll
    for (int q = 0; q < 6; q++) stv(ws[q] + iv, s[q]);
}

// free surface 3D, one thread per (y, x) column (surface3D.cl:39-271)
// TR: storage type of the memory variables; values are read times
// g.rsci and stored times g.rsc (1 except with Grid::rhalf)
template <int F, class T = float, class TR = T>
__global__ void k_surf3d(Grid g, Fields f, int pdir)
{
    SHOT_F
    int gy = blockIdx.x * blockDim.x + threadIdx.x + F;
    int gx = blockIdx.y * blockDim.y + threadIdx.y + F;
    if (gy > g.NY - F - 1 || gx > g.NX - F - 1) return;
    int gz = F, NAB = g.nab, L = g.L;
    const i64 sx = (i64)g.NY * g.NZ, sy = g.NZ;
    i64 iv = gx * sx + (i64)gy * sy + gz;
    i64 ip = ((i64)(gx - F) * g.ny + (gy - F)) * g.nz + (gz - F);
    T *sxx = fld<T>(f.w[SXX]), *syy = fld<T>(f.w[SYY]), *szz = fld<T>(f.w[SZZ]), *syz = fld<T>(f.w[SYZ]),
      *sxz = fld<T>(f.w[SXZ]);
    TR *rxx = fld<TR>(f.r[RXX]), *ryy = fld<TR>(f.r[RYY]), *rzz = fld<TR>(f.r[RZZ]);
    stv(szz + iv, 0.0f);
    for (int l = 0; l < L; l++) stv(rzz + l * g.nvol + iv, 0.0f);
#pragma unroll
    for (int m = 1; m <= F; m++) {
        stv(szz + iv - m, -ldv(szz + iv + m));
        stv(sxz + iv - m, -ldv(sxz + iv + m - 1));
        stv(syz + iv - m, -ldv(syz + iv + m - 1));
    }
    float vxx = dbw_rwT<F>(fld<T>(f.w[VX]), iv, sx, g.hc);
    float vyy = dbw_rwT<F>(fld<T>(f.w[VY]), iv, sy, g.hc);
    float vzz = dbw_rwT<F>(fld<T>(f.w[VZ]), iv, 1, g.hc);
    if (g.abs_type == 1) {
        i64 nz = g.nz, ny = g.ny;
        if (gy - F < NAB) {
            i64 i = gx - F, j = gy - F;
            vyy = vyy * f.kinv[1][0][j] + f.psi[PVY_Y][(i * (2 * NAB) + j) * nz];
        } else if (gy > g.NY - NAB - F - 1) {
            i64 i = gx - F, j = gy - g.NY + NAB + F + NAB;
            int ind = 2 * NAB - 1 - (int)j;
            vyy = vyy * f.kinv[1][0][ind + 1] + f.psi[PVY_Y][(i * (2 * NAB) + j) * nz];
        }
        if (gx - F < NAB) {
            i64 i = gx - F, j = gy - F;
            vxx = vxx * f.kinv[0][0][i] + f.psi[PVX_X][(i * ny + j) * nz];
        }
        if (gx > g.NX - NAB - F - 1) {
            i64 i = gx - g.NX + NAB + F + NAB, j = gy - F;
            int ind = 2 * NAB - 1 - (int)i;
            vxx = vxx * f.kinv[0][0][ind + 1] + f.psi[PVX_X][(i * ny + j) * nz];
        }
    }
    if (L == 0) {
        float fm = f.p[PMU][ip] * 2.0f, gm = f.p[PM][ip];
        float h = -((gm - fm) * (gm - fm) * (vxx + vyy) / gm) - ((gm - fm) * vzz);
        // the reference adds h without the propagation direction (surface3D.cl:172-173)
        stv(sxx + iv, ldv(sxx + iv) + h);
        stv(syy + iv, ldv(syy + iv) + h);
    } else {
        float taus = f.p[PTAUS][ip], taup = f.p[PTAUP][ip], mu = f.p[PMU][ip], M = f.p[PM][ip];
        float fm = mu * 2.0f * (1.0f + L * taus);
        float gm = M * (1.0f + L * taup);
        float h = -((gm - fm) * (gm - fm) * (vxx + vyy) / gm) - ((gm - fm) * vzz);
        float sumx = 0, sumy = 0;
        for (int l = 0; l < L; l++) {
            sumx += ldv(rxx + l * g.nvol + iv) * g.rsci;
            sumy += ldv(ryy + l * g.nvol + iv) * g.rsci;
        }
        stv(sxx + iv, ldv(sxx + iv) + pdir * (h - g.dt2 * sumx));
        stv(syy + iv, ldv(syy + iv) + pdir * (h - g.dt2 * sumy));
        float d = 2.0f * mu * taus / g.dt, e = M * taup / g.dt;
        sumx = 0; sumy = 0;
        for (int l = 0; l < L; l++) {
            float b = g.eta[l] / (1.0f + g.eta[l] * 0.5f);
            float hh = b * (((d - e) * ((fm / gm) - 1.0f) * (vxx + vyy)) - ((d - e) * vzz));
            float rx = ldv(rxx + l * g.nvol + iv) * g.rsci + hh, ry = ldv(ryy + l * g.nvol + iv) * g.rsci + hh;
            stv(rxx + l * g.nvol + iv, rx * g.rsc);
            stv(ryy + l * g.nvol + iv, ry * g.rsc);
            sumx += rx; sumy += ry;
        }
        stv(sxx + iv, ldv(sxx + iv) + g.dt2 * sumx);
        stv(syy + iv, ldv(syy + iv) + g.dt2 * sumy);
    }
}


// ============================================================ 2D acoustic
// src/update_v2D_acc.cl:80-324, src/update_s2D_acc.cl:79-402; the pressure
// lives in the SXX slot, its memory variable in RXX, psi_p_x / psi_p_z in the
// PSXX_X / PSZZ_Z slots.
template <int F>
__global__ void __launch_bounds__(256) k_v2d_acc(Grid g, Fields f)
{
    SHOT_F
    int gz = blockIdx.x * blockDim.x + threadIdx.x + F;
    int gx = blockIdx.y * blockDim.y + threadIdx.y + F;
    if (gz > g.NZ - F - 1 || gx > g.NX - F - 1) return;
    i64 ip = (i64)(gx - F) * g.nz + (gz - F), iv = (i64)gx * g.NZ + gz;
    int NAB = g.nab, NZ = g.NZ, NX = g.NX;
    float p_x = dfw<F>(f.w[SXX], iv, NZ, g.hc);
    float p_z = dfw<F>(f.w[SXX], iv, 1, g.hc);
    if (g.abs_type == 1) {
        if (gz > NZ - NAB - F - 1) {
            int i = gx - F, k = gz - NZ + NAB + F + NAB, ind = 2 * NAB - 1 - k;
            cpml(f.psi[PSZZ_Z], (i64)i * (2 * NAB) + k, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, p_z);
        } else if (!g.freesurf && gz - F < NAB) {
            int i = gx - F, k = gz - F;
            cpml(f.psi[PSZZ_Z], (i64)i * (2 * NAB) + k, f.cz[CKH], f.cz[CAH], f.cz[CBH], k, p_z);
        }
        if (gx - F < NAB) {
            int i = gx - F, k = gz - F;
            cpml(f.psi[PSXX_X], (i64)i * g.nz + k, f.cx[CKH], f.cx[CAH], f.cx[CBH], i, p_x);
        }
        if (gx > NX - NAB - F - 1) {
            int i = gx - NX + NAB + F + NAB, k = gz - F, ind = 2 * NAB - 1 - i;
            cpml(f.psi[PSXX_X], (i64)i * g.nz + k, f.cx[CKH], f.cx[CAH], f.cx[CBH], ind, p_x);
        }
    }
    float vx = f.w[VX][iv] + p_x * __ldg(f.p[PRIP] + ip);
    float vz = f.w[VZ][iv] + p_z * __ldg(f.p[PRKP] + ip);
    if (g.abs_type == 2) {
        // the acoustic kernels taper the top even with a free surface
        const float *tp = f.taper;
        if (gz - F < NAB) { vx *= tp[gz - F]; vz *= tp[gz - F]; }
        if (gz > NZ - NAB - F - 1) { vx *= tp[NZ - F - gz - 1]; vz *= tp[NZ - F - gz - 1]; }
        if (gx - F < NAB) { vx *= tp[gx - F]; vz *= tp[gx - F]; }
        if (gx > NX - NAB - F - 1) { vx *= tp[NX - F - gx - 1]; vz *= tp[NX - F - gx - 1]; }
    }
    f.w[VX][iv] = vx;
    f.w[VZ][iv] = vz;
}

// one cell of the acoustic pressure update (update_s2D_acc.cl:79-402)
template <int F>
__device__ __forceinline__ void s2d_acc_cell(const Grid &g, const Fields &f, int gz, int gx)
{
    i64 ip = (i64)(gx - F) * g.nz + (gz - F), iv = (i64)gx * g.NZ + gz;
    int NAB = g.nab, NZ = g.NZ, NX = g.NX, L = g.L;
    float vxx = dbw<F>(f.w[VX], iv, NZ, g.hc);
    float vzz = dbw<F>(f.w[VZ], iv, 1, g.hc);
    if (g.abs_type == 1) {
        if (gz > NZ - NAB - F - 1) {
            int i = gx - F, k = gz - NZ + NAB + F + NAB, ind = 2 * NAB - 1 - k;
            cpml(f.psi[PVZ_Z], (i64)i * (2 * NAB) + k, f.cz[CK], f.cz[CA], f.cz[CB], ind + 1, vzz);
        } else if (!g.freesurf && gz - F < NAB) {
            int i = gx - F, k = gz - F;
            cpml(f.psi[PVZ_Z], (i64)i * (2 * NAB) + k, f.cz[CK], f.cz[CA], f.cz[CB], k, vzz);
        }
        if (gx - F < NAB) {
            int i = gx - F, k = gz - F;
            cpml(f.psi[PVX_X], (i64)i * g.nz + k, f.cx[CK], f.cx[CA], f.cx[CB], i, vxx);
        }
        if (gx > NX - NAB - F - 1) {
            int i = gx - NX + NAB + F + NAB, k = gz - F, ind = 2 * NAB - 1 - i;
            cpml(f.psi[PVX_X], (i64)i * g.nz + k, f.cx[CK], f.cx[CA], f.cx[CB], ind + 1, vxx);
        }
    }
    float p = f.w[SXX][iv];
    if (L == 0) {
        p += __ldg(f.p[PM] + ip) * (vxx + vzz);
    } else {
        float lM = __ldg(f.p[PM] + ip), ltaup = __ldg(f.p[PTAUP] + ip);
        float gm = lM * (1.0f + (float)L * ltaup);
        float e = lM * ltaup;  // no 1/dt, as update_s2D_acc.cl:333
        float sumrp = 0;
        for (int l = 0; l < L; l++) sumrp += f.r[RXX][l * g.nvol + iv];
        float lp = gm * (vxx + vzz) + g.dt2 * sumrp;
        sumrp = 0;
        for (int l = 0; l < L; l++) {
            float el = g.eta[l];
            float b = 1.0f / (1.0f + el * 0.5f), c = 1.0f - el * 0.5f;
            i64 ir = l * g.nvol + iv;
            float r = b * (f.r[RXX][ir] * c - el * e * (vxx + vzz));
            f.r[RXX][ir] = r;
            sumrp += r;
        }
        p += lp + g.dt2 * sumrp;
    }
    if (g.abs_type == 2) {
        const float *tp = f.taper;
        if (gz - F < NAB) p *= tp[gz - F];
        if (gz > NZ - NAB - F - 1) p *= tp[NZ - F - gz - 1];
        if (gx - F < NAB) p *= tp[gx - F];
        if (gx > NX - NAB - F - 1) p *= tp[NX - F - gx - 1];
    }
    f.w[SXX][iv] = p;
}

template <int F>
__global__ void __launch_bounds__(256) k_s2d_acc(Grid g, Fields f)
{
    SHOT_F
    int gz = blockIdx.x * blockDim.x + threadIdx.x + F;
    int gx = blockIdx.y * blockDim.y + threadIdx.y + F;
    if (gz <= g.NZ - F - 1 && gx <= g.NX - F - 1) s2d_acc_cell<F>(g, f, gz, gx);
}

// ================================================================== 2D SH
// src/update_v2D_SH.cl:106-356, src/update_s2D_SH.cl:109-421 (elastic).
// Buoyancy and shear modulus at the cell, unaveraged; the far-x CPML of the
// velocity uses the full-node coefficients at ind; at FDOH=1 the stress
// differences carry no coefficient; stresses are not tapered.
template <int F>
__global__ void __launch_bounds__(256) k_v2d_sh(Grid g, Fields f)
{
    int gz = blockIdx.x * blockDim.x + threadIdx.x + F;
    int gx = blockIdx.y * blockDim.y + threadIdx.y + F;
    if (gz > g.NZ - F - 1 || gx > g.NX - F - 1) return;
    i64 ip = (i64)(gx - F) * g.nz + (gz - F), iv = (i64)gx * g.NZ + gz;
    int NAB = g.nab, NZ = g.NZ, NX = g.NX;
    float sxy_x = dbw<F>(f.w[SXY], iv, NZ, g.hc);
    float syz_z = dbw<F>(f.w[SYZ], iv, 1, g.hc);
    if (g.abs_type == 1) {
        if (gz > NZ - NAB - F - 1) {
            int i = gx - F, k = gz - NZ + NAB + F + NAB, ind = 2 * NAB - 1 - k;
            cpml(f.psi[PSYZ_Z], (i64)i * (2 * NAB) + k, f.cz[CK], f.cz[CA], f.cz[CB], ind + 1, syz_z);
        } else if (!g.freesurf && gz - F < NAB) {
            int i = gx - F, k = gz - F;
            cpml(f.psi[PSYZ_Z], (i64)i * (2 * NAB) + k, f.cz[CK], f.cz[CA], f.cz[CB], k, syz_z);
        }
        if (gx - F < NAB) {
            int i = gx - F, k = gz - F;
            cpml(f.psi[PSXY_X], (i64)i * g.nz + k, f.cx[CK], f.cx[CA], f.cx[CB], i, sxy_x);
        }
        if (gx > NX - NAB - F - 1) {
            int i = gx - NX + NAB + F + NAB, k = gz - F, ind = 2 * NAB - 1 - i;
            cpml(f.psi[PSXY_X], (i64)i * g.nz + k, f.cx[CK], f.cx[CA], f.cx[CB], ind, sxy_x);
        }
    }
    float vy = f.w[VY][iv] + (sxy_x + syz_z) * __ldg(f.p[PRHO] + ip);
    if (g.abs_type == 2) {
        const float *tp = f.taper;
        if (!g.freesurf && gz - F < NAB) vy *= tp[gz - F];
        if (gz > NZ - NAB - F - 1) vy *= tp[NZ - F - gz - 1];
        if (gx - F < NAB) vy *= tp[gx - F];
        if (gx > NX - NAB - F - 1) vy *= tp[NX - F - gx - 1];
    }
    f.w[VY][iv] = vy;
}

template <int F>
__global__ void __launch_bounds__(256) k_s2d_sh(Grid g, Fields f)
{
    int gz = blockIdx.x * blockDim.x + threadIdx.x + F;
    int gx = blockIdx.y * blockDim.y + threadIdx.y + F;
    if (gz > g.NZ - F - 1 || gx > g.NX - F - 1) return;
    i64 ip = (i64)(gx - F) * g.nz + (gz - F), iv = (i64)gx * g.NZ + gz;
    int NAB = g.nab, NZ = g.NZ, NX = g.NX;
    float hone[6] = {1.0f, 0, 0, 0, 0, 0};
    const float *h = F == 1 ? hone : g.hc;
    float vyx = dfw<F>(f.w[VY], iv, NZ, h);
    float vyz = dfw<F>(f.w[VY], iv, 1, h);
    if (g.abs_type == 1) {
        if (gz > NZ - NAB - F - 1) {
            int i = gx - F, k = gz - NZ + NAB + F + NAB, ind = 2 * NAB - 1 - k;
            cpml(f.psi[PVY_Z], (i64)i * (2 * NAB) + k, f.cz[CKH], f.cz[CAH], f.cz[CBH], ind, vyz);
        } else if (!g.freesurf && gz - F < NAB) {
            int i = gx - F, k = gz - F;
            cpml(f.psi[PVY_Z], (i64)i * (2 * NAB) + k, f.cz[CKH], f.cz[CAH], f.cz[CBH], k, vyz);
        }
        if (gx - F < NAB) {
            int i = gx - F, k = gz - F;
            cpml(f.psi[PVY_X], (i64)i * g.nz + k, f.cx[CKH], f.cx[CAH], f.cx[CBH], i, vyx);
        }
        if (gx > NX - NAB - F - 1) {
            int i = gx - NX + NAB + F + NAB, k = gz - F, ind = 2 * NAB - 1 - i;
            cpml(f.psi[PVY_X], (i64)i * g.nz + k, f.cx[CKH], f.cx[CAH], f.cx[CBH], ind, vyx);
        }
    }
    float mu = __ldg(f.p[PMU] + ip);
    f.w[SXY][iv] += mu * vyx;
    f.w[SYZ][iv] += mu * vyz;
}

// SH free surface: image syz above the surface (src/surface2D_SH.cl:37-39)
template <int F>
__global__ void k_surf_sh(Grid g, Fields f)
{
    int gx = blockIdx.x * blockDim.x + threadIdx.x + F;
    if (gx > g.NX - F - 1) return;
    i64 iv = (i64)gx * g.NZ + F;
#pragma unroll
    for (int m = 1; m <= F; m++) f.w[SYZ][iv - m] = -f.w[SYZ][iv + m - 1];
}

// ---------------------------------------------------- boundary save (forward)
template <typename T>
__global__ void k_savebnd(Grid g, Fields f, BndSlot b, i64 tofs)
{
    SHOT_F
    int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= g.nbnd) return;
    const i64 sh = (i64)blockIdx.z * (g.sb_bnd / (i64)sizeof(T));
    int i, j, k;
    if (!shell_cell(g, gid, i, j, k)) return;
    i64 iv = ((i64)i * g.NY + j) * g.NZ + k;
    // every field index is a compile-time constant (a saved field has its
    // store in b.p[w]): indexing the parameter structs with a run-time field
    // id made each thread copy them to local memory (a 688-byte stack frame);
    // all loads go out before the stores
    float v[NW];
#pragma unroll
    for (int w = 0; w < NW; w++)
        if (b.p[w]) v[w] = f.w[w][iv];
#pragma unroll
    for (int w = 0; w < NW; w++)
        if (b.p[w]) ((T *)b.p[w])[sh + tofs + gid] = from_f<T>(v[w] * g.bsc[w]);
}

// ------------------------------------------------------- adjoint kernels 2D
template <int F, typename T>
__global__ void __launch_bounds__(256) k_adjv2d(Grid g, Fields f, AdjFields a)
{
    SHOT_FA
    int gz = blockIdx.x * blockDim.x + threadIdx.x + F;
    int gx = blockIdx.y * blockDim.y + threadIdx.y + F;
    if (gz > g.NZ - F - 1 || gx > g.NX - F - 1) return;
    i64 ip = (i64)(gx - F) * g.nz + (gz - F), iv = (i64)gx * g.NZ + gz;
    const float *hc = g.hc;
    float rip = __ldg(f.p[PRIP] + ip), rkp = __ldg(f.p[PRKP] + ip);
    float vx = 0.0f, vz = 0.0f;
    if (g.ckpt) {
        vx = fwd_at<T>(g, a, VX, iv);
        vz = fwd_at<T>(g, a, VZ, iv);
    } else if (!g.bp2) {  // backpropagate the forward velocities (update_adjv2D.cl:205-240)
        float sxx_x = dfw<F>(f.w[SXX], iv, g.NZ, hc);
        float szz_z = dfw<F>(f.w[SZZ], iv, 1, hc);
        float sxz_z = dbw<F>(f.w[SXZ], iv, 1, hc);
        float sxz_x = dbw<F>(f.w[SXZ], iv, g.NZ, hc);
        vx = f.w[VX][iv] - (sxx_x + sxz_z) * rip;
        vz = f.w[VZ][iv] - (szz_z + sxz_x) * rkp;
        int m = inject_ind2d(g, gz, gx);
        if (m != -1) {
            vx = bnd_at<T>(g, a, VX, m);
            vz = bnd_at<T>(g, a, VZ, m);
        }
        f.w[VX][iv] = vx;
        f.w[VZ][iv] = vz;
    }
    float sxx_xr = dfw<F>(a.wr[SXX], iv, g.NZ, hc);
    float szz_zr = dfw<F>(a.wr[SZZ], iv, 1, hc);
    float sxz_zr = dbw<F>(a.wr[SXZ], iv, 1, hc);
    float sxz_xr = dbw<F>(a.wr[SXZ], iv, g.NZ, hc);
    if (g.abs_type == 1) cpml_v2d(g, f, gz, gx, sxx_xr, szz_zr, sxz_xr, sxz_zr);
    float lvx = (sxx_xr + sxz_zr) * rip;
    float lvz = (szz_zr + sxz_xr) * rkp;
    a.wr[VX][iv] += lvx;
    a.wr[VZ][iv] += lvz;
    if (g.abs_type == 2) {
        float *fs[2] = {a.wr[VX], a.wr[VZ]};
        apply_taper<2>(g, f.taper, gz, 0, gx, fs, iv);
    }
    if (!g.bp2) a.grad[GRHO][ip] += (double)(-vx * lvx - vz * lvz);
}

template <int F, typename T>
__global__ void __launch_bounds__(256) k_adjs2d(Grid g, Fields f, AdjFields a)
{
    SHOT_FA
    int gz = blockIdx.x * blockDim.x + threadIdx.x + F;
    int gx = blockIdx.y * blockDim.y + threadIdx.y + F;
    if (gz > g.NZ - F - 1 || gx > g.NX - F - 1) return;
    i64 ip = (i64)(gx - F) * g.nz + (gz - F), iv = (i64)gx * g.NZ + gz;
    const float *hc = g.hc;
    float vxx = 0.0f, vxz = 0.0f, vzz = 0.0f, vzx = 0.0f;
    if (!g.bp2 && !g.ckpt) {
        vxx = dbw<F>(f.w[VX], iv, g.NZ, hc); vxz = dfw<F>(f.w[VX], iv, 1, hc);
        vzz = dbw<F>(f.w[VZ], iv, 1, hc); vzx = dfw<F>(f.w[VZ], iv, g.NZ, hc);
    }
    float vxxr = dbw<F>(a.wr[VX], iv, g.NZ, hc), vxzr = dfw<F>(a.wr[VX], iv, 1, hc);
    float vzzr = dbw<F>(a.wr[VZ], iv, 1, hc), vzxr = dfw<F>(a.wr[VZ], iv, g.NZ, hc);
    const int L = g.L;
    float lM = __ldg(f.p[PM] + ip), lmu = __ldg(f.p[PMU] + ip), fipkp, fm, gm, dipkp = 0, d = 0, e = 0;
    if (L == 0) {
        fipkp = __ldg(f.p[PMUIPKP] + ip);
        fm = 2.0f * lmu;
        gm = lM;
    } else {
        float lmuipkp = __ldg(f.p[PMUIPKP] + ip), ltaup = __ldg(f.p[PTAUP] + ip), ltaus = __ldg(f.p[PTAUS] + ip);
        float ltausipkp = __ldg(f.p[PTAUSIPKP] + ip);
        fipkp = lmuipkp * (1.0f + (float)L * ltausipkp);
        gm = lM * (1.0f + (float)L * ltaup);
        fm = 2.0f * lmu * (1.0f + (float)L * ltaus);
        dipkp = lmuipkp * ltausipkp / g.dt;
        d = 2.0f * lmu * ltaus / g.dt;
        e = lM * ltaup / g.dt;
    }
    float sxx = 0.0f, szz = 0.0f, sxz = 0.0f;
    // reconstruct the forward stresses (update_adjs2D.cl:222-278)
    if (g.bp2) {
    } else if (g.ckpt) {
        sxx = fwd_at<T>(g, a, SXX, iv); szz = fwd_at<T>(g, a, SZZ, iv); sxz = fwd_at<T>(g, a, SXZ, iv);
    } else if (L == 0) {
        sxx = f.w[SXX][iv]; szz = f.w[SZZ][iv]; sxz = f.w[SXZ][iv];
        sxz -= fipkp * (vxz + vzx);
        sxx -= gm * (vxx + vzz) - fm * vzz;
        szz -= gm * (vxx + vzz) - fm * vxx;
    } else {
        sxx = f.w[SXX][iv]; szz = f.w[SZZ][iv]; sxz = f.w[SXZ][iv];
        float *rxx = f.r[RXX], *rzz = f.r[RZZ], *rxz = f.r[RXZ];
        float s1 = 0, s2 = 0, s3 = 0;
        for (int l = 0; l < L; l++) { i64 ir = l * g.nvol + iv; s1 += rxz[ir]; s2 += rxx[ir]; s3 += rzz[ir]; }
        float lsxz = fipkp * (vxz + vzx) + g.dt2 * s1;
        float lsxx = (gm * (vxx + vzz) - fm * vzz) + g.dt2 * s2;
        float lszz = (gm * (vxx + vzz) - fm * vxx) + g.dt2 * s3;
        s1 = s2 = s3 = 0;
        for (int l = 0; l < L; l++) {
            float el = g.eta[l];
            float b = 1.0f / (1.0f - el * 0.5f), c = 1.0f + el * 0.5f;
            i64 ir = l * g.nvol + iv;
            float n1 = b * (rxz[ir] * c - el * (dipkp * (vxz + vzx)));
            float n2 = b * (rxx[ir] * c - el * (e * (vxx + vzz) - d * vzz));
            float n3 = b * (rzz[ir] * c - el * (e * (vxx + vzz) - d * vxx));
            rxz[ir] = n1; rxx[ir] = n2; rzz[ir] = n3;
            s1 += n1; s2 += n2; s3 += n3;
        }
        sxz -= lsxz + g.dt2 * s1;
        sxx -= lsxx + g.dt2 * s2;
        szz -= lszz + g.dt2 * s3;
    }
    if (!g.bp2 && !g.ckpt) {
        int m = inject_ind2d(g, gz, gx);
        if (m != -1) {
            sxx = bnd_at<T>(g, a, SXX, m);
            szz = bnd_at<T>(g, a, SZZ, m);
            sxz = bnd_at<T>(g, a, SXZ, m);
        }
        f.w[SXX][iv] = sxx; f.w[SZZ][iv] = szz; f.w[SXZ][iv] = sxz;
    }
    if (g.abs_type == 1) cpml_s2d(g, f, gz, gx, vxxr, vxzr, vzxr, vzzr);
    float lsxz, lsxx, lszz;
    if (L == 0) {
        lsxz = fipkp * (vxzr + vzxr);
        lsxx = gm * (vxxr + vzzr) - fm * vzzr;
        lszz = gm * (vxxr + vzzr) - fm * vxxr;
        a.wr[SXZ][iv] += lsxz;
        a.wr[SXX][iv] += lsxx;
        a.wr[SZZ][iv] += lszz;
    } else {
        float *rxxr = a.rr[RXX], *rzzr = a.rr[RZZ], *rxzr = a.rr[RXZ];
        float s1 = 0, s2 = 0, s3 = 0;
        for (int l = 0; l < L; l++) { i64 ir = l * g.nvol + iv; s1 += rxzr[ir]; s2 += rxxr[ir]; s3 += rzzr[ir]; }
        lsxz = fipkp * (vxzr + vzxr) + g.dt2 * s1;
        lsxx = (gm * (vxxr + vzzr) - fm * vzzr) + g.dt2 * s2;
        lszz = (gm * (vxxr + vzzr) - fm * vxxr) + g.dt2 * s3;
        s1 = s2 = s3 = 0;
        // every iteration updates the last mechanism's slot, as the reference
        // does (update_adjs2D.cl:379-391)
        i64 ir = (L - 1) * g.nvol + iv;
        for (int l = 0; l < L; l++) {
            float el = g.eta[l];
            float b = 1.0f / (1.0f + el * 0.5f), c = 1.0f - el * 0.5f;
            float n1 = b * (rxzr[ir] * c - el * (dipkp * (vxzr + vzxr)));
            float n2 = b * (rxxr[ir] * c - el * (e * (vxxr + vzzr) - d * vzzr));
            float n3 = b * (rzzr[ir] * c - el * (e * (vxxr + vzzr) - d * vxxr));
            rxzr[ir] = n1; rxxr[ir] = n2; rzzr[ir] = n3;
            s1 += n1; s2 += n2; s3 += n3;
        }
        a.wr[SXZ][iv] += lsxz + g.dt2 * s1;
        a.wr[SXX][iv] += lsxx + g.dt2 * s2;
        a.wr[SZZ][iv] += lszz + g.dt2 * s3;
    }
    if (g.abs_type == 2) {
        float *fs[3] = {a.wr[SXZ], a.wr[SXX], a.wr[SZZ]};
        apply_taper<3>(g, f.taper, gz, 0, gx, fs, iv);
    }
    if (g.bp2) {
    } else if (g.restype == 0) {
        float c1 = 1.0f / ((2.0f * lM - 2.0f * lmu) * (2.0f * lM - 2.0f * lmu));
        float c3 = 1.0f / (lmu * lmu);
        float c5 = 0.25f * c3;
        float dM = c1 * (sxx + szz) * (lsxx + lszz);
        a.grad[GM][ip] += (double)(-dM);
        a.grad[GMU][ip] += (double)(-c3 * (sxz * lsxz) + dM - c5 * ((sxx - szz) * (lsxx - lszz)));
        if (g.hout) {
            // update_adjs2D.cl:453-457 (the mu term subtracts the gradient's dM)
            float dMH = c1 * (sxx + szz) * (sxx + szz);
            a.hess[GM][ip] += (double)dMH;
            a.hess[GMU][ip] += (double)(c3 * sxz * sxz - dM + c5 * (sxx - szz) * (sxx - szz));
        }
    } else {
        float dM = (sxx + szz) * (lsxx + lszz);
        a.grad[GM][ip] += (double)(-dM);
        if (g.hout) a.hess[GM][ip] += (double)((sxx + szz) * (sxx + szz));
    }
}

// surface adjoint, split in two passes so no thread updates another
// column's cell (surface2D_adj.cl:35-148 lets neighbouring work-items add
// into the same vxr cells).  Pass 1: per column, the L transform, the vzr
// update of its own column, and q = hx * lsxx for pass 2.
template <int F>
__global__ void k_surfadj2d_a(Grid g, Fields f, AdjFields a, float *q)
{
    SHOT_FA
    q += blockIdx.z * g.sb_q;
    int gx = blockIdx.x * blockDim.x + threadIdx.x + F;
    if (gx > g.NX - F - 1) return;
    int gz = F;
    i64 iv = (i64)gx * g.NZ + gz, ip = (i64)(gx - F) * g.nz + (gz - F);
    float lszz = a.wr[SZZ][iv], lsxx = a.wr[SXX][iv];
    float lmu = f.p[PMU][ip], lM = f.p[PM][ip];
    float t1 = lsxx, t2 = lszz;
    float aa = 1.0f / (4.0f * lM * lmu - 4.0f * lmu * lmu);
    lsxx = -aa * (lM * t1 + (-lM + 2.0f * lmu) * t2);
    lszz = 0.0f;
    float hx = -((lM - lmu * 2.0f) * (lM - lmu * 2.0f) / lM);
    float hz = -(lM - lmu * 2.0f);
    for (int m = 0; m < F; m++)
        a.wr[VZ][iv + m] += g.hc[m] * hz * lsxx * f.p[PRKP][ip + m];
    q[gx - F] = hx * lsxx;
    a.wr[SZZ][iv] = -(lM * lszz + (lM - 2.0f * lmu) * lsxx);
    a.wr[SXX][iv] = -(lM * lsxx + (lM - 2.0f * lmu) * lszz);
}
// Pass 2: each column gathers the contributions of its neighbours.
template <int F>
__global__ void k_surfadj2d_b(Grid g, Fields f, AdjFields a, const float *q)
{
    SHOT_FA
    q += blockIdx.z * g.sb_q;
    int gx = blockIdx.x * blockDim.x + threadIdx.x + F;
    if (gx > g.NX - F - 1) return;
    int gz = F, x = gx - F, nx = g.nx;
    i64 iv = (i64)gx * g.NZ + gz, ip = (i64)(gx - F) * g.nz + (gz - F);
    float rip = f.p[PRIP][ip], acc = 0.0f;
    for (int m = 0; m < F; m++) {
        if (x - m >= 0) acc += g.hc[m] * q[x - m];
        if (x + m + 1 < nx) acc -= g.hc[m] * q[x + m + 1];
    }
    a.wr[VX][iv] += acc * rip;
}

// ------------------------------------------------------- adjoint kernels 3D
template <int F, typename T, bool MB = false>
__global__ void __launch_bounds__(256) k_adjv3d(Grid g, Fields f, AdjFields a)
{
    CELL3D
    if (MB) shot_adj(g, a, shot);
    const float *hc = g.hc;
    float rip = __ldg(f.p[PRIP] + ip), rjp = __ldg(f.p[PRJP] + ip), rkp = __ldg(f.p[PRKP] + ip);
    float vx = 0.0f, vy = 0.0f, vz = 0.0f;
    if (g.ckpt) {
        vx = fwd_at<T>(g, a, VX, iv); vy = fwd_at<T>(g, a, VY, iv); vz = fwd_at<T>(g, a, VZ, iv);
    } else if (!g.bp2) {  // backpropagate the forward velocities (update_adjv3D.cl:297-340)
        float szz_z = dfw<F>(f.w[SZZ], iv, 1, hc), sxx_x = dfw<F>(f.w[SXX], iv, sx, hc);
        float sxz_x = dbw<F>(f.w[SXZ], iv, sx, hc), sxz_z = dbw<F>(f.w[SXZ], iv, 1, hc);
        float syz_y = dbw<F>(f.w[SYZ], iv, sy, hc), syz_z = dbw<F>(f.w[SYZ], iv, 1, hc);
        float syy_y = dfw<F>(f.w[SYY], iv, sy, hc);
        float sxy_x = dbw<F>(f.w[SXY], iv, sx, hc), sxy_y = dbw<F>(f.w[SXY], iv, sy, hc);
        vx = f.w[VX][iv] - (sxx_x + sxy_y + sxz_z) * rip;
        vy = f.w[VY][iv] - (syy_y + sxy_x + syz_z) * rjp;
        vz = f.w[VZ][iv] - (szz_z + sxz_x + syz_y) * rkp;
        int m = inject_ind3d(g, gz, gy, gx);
        if (m != -1) {
            vx = bnd_at<T>(g, a, VX, m);
            vy = bnd_at<T>(g, a, VY, m);
            vz = bnd_at<T>(g, a, VZ, m);
        }
        f.w[VX][iv] = vx; f.w[VY][iv] = vy; f.w[VZ][iv] = vz;
    }
    float szz_zr = dfw<F>(a.wr[SZZ], iv, 1, hc), sxx_xr = dfw<F>(a.wr[SXX], iv, sx, hc);
    float sxz_xr = dbw<F>(a.wr[SXZ], iv, sx, hc), sxz_zr = dbw<F>(a.wr[SXZ], iv, 1, hc);
    float syz_yr = dbw<F>(a.wr[SYZ], iv, sy, hc), syz_zr = dbw<F>(a.wr[SYZ], iv, 1, hc);
    float syy_yr = dfw<F>(a.wr[SYY], iv, sy, hc);
    float sxy_xr = dbw<F>(a.wr[SXY], iv, sx, hc), sxy_yr = dbw<F>(a.wr[SXY], iv, sy, hc);
    if (g.abs_type == 1)
        cpml_v3d(g, f, gz, gy, gx, sxx_xr, syy_yr, szz_zr, sxy_yr, sxy_xr, syz_yr, syz_zr, sxz_xr, sxz_zr);
    float lvx = (sxx_xr + sxy_yr + sxz_zr) * rip;
    float lvy = (syy_yr + sxy_xr + syz_zr) * rjp;
    float lvz = (szz_zr + sxz_xr + syz_yr) * rkp;
    a.wr[VX][iv] += lvx; a.wr[VY][iv] += lvy; a.wr[VZ][iv] += lvz;
    if (g.abs_type == 2) {
        float *fs[3] = {a.wr[VX], a.wr[VY], a.wr[VZ]};
        apply_taper<3>(g, f.taper, gz, gy, gx, fs, iv);
    }
    if (!g.bp2) a.grad[GRHO][ip] += (double)(-vx * lvx - vy * lvy - vz * lvz);
}

template <int F, typename T, bool MB = false>
__global__ void __launch_bounds__(256) k_adjs3d(Grid g, Fields f, AdjFields a)
{
    CELL3D
    if (MB) shot_adj(g, a, shot);
    const float *hc = g.hc;
    float vzx = 0.0f, vzy = 0.0f, vzz = 0.0f, vyx = 0.0f, vyy = 0.0f, vyz = 0.0f, vxx = 0.0f, vxy = 0.0f, vxz = 0.0f;
    if (!g.bp2 && !g.ckpt) {
        vzx = dfw<F>(f.w[VZ], iv, sx, hc); vzy = dfw<F>(f.w[VZ], iv, sy, hc); vzz = dbw<F>(f.w[VZ], iv, 1, hc);
        vyx = dfw<F>(f.w[VY], iv, sx, hc); vyy = dbw<F>(f.w[VY], iv, sy, hc); vyz = dfw<F>(f.w[VY], iv, 1, hc);
        vxx = dbw<F>(f.w[VX], iv, sx, hc); vxy = dfw<F>(f.w[VX], iv, sy, hc); vxz = dfw<F>(f.w[VX], iv, 1, hc);
    }
    float vzxr = dfw<F>(a.wr[VZ], iv, sx, hc), vzyr = dfw<F>(a.wr[VZ], iv, sy, hc), vzzr = dbw<F>(a.wr[VZ], iv, 1, hc);
    float vyxr = dfw<F>(a.wr[VY], iv, sx, hc), vyyr = dbw<F>(a.wr[VY], iv, sy, hc), vyzr = dfw<F>(a.wr[VY], iv, 1, hc);
    float vxxr = dbw<F>(a.wr[VX], iv, sx, hc), vxyr = dfw<F>(a.wr[VX], iv, sy, hc), vxzr = dfw<F>(a.wr[VX], iv, 1, hc);
    const int L = g.L;
    float lM = __ldg(f.p[PM] + ip), lmu = __ldg(f.p[PMU] + ip);
    float fipjp, fjpkp, fipkp, gm, fm, dipjp = 0, djpkp = 0, dipkp = 0, d = 0, e = 0;
    if (L == 0) {
        fipjp = __ldg(f.p[PMUIPJP] + ip); fjpkp = __ldg(f.p[PMUJPKP] + ip); fipkp = __ldg(f.p[PMUIPKP] + ip);
        gm = lM; fm = 2.0f * lmu;
    } else {
        float lmuipkp = __ldg(f.p[PMUIPKP] + ip), lmuipjp = __ldg(f.p[PMUIPJP] + ip), lmujpkp = __ldg(f.p[PMUJPKP] + ip);
        float ltaup = __ldg(f.p[PTAUP] + ip), ltaus = __ldg(f.p[PTAUS] + ip);
        float ltausipkp = __ldg(f.p[PTAUSIPKP] + ip), ltausipjp = __ldg(f.p[PTAUSIPJP] + ip),
              ltausjpkp = __ldg(f.p[PTAUSJPKP] + ip);
        fipjp = lmuipjp * (1.0f + (float)L * ltausipjp);
        fjpkp = lmujpkp * (1.0f + (float)L * ltausjpkp);
        fipkp = lmuipkp * (1.0f + (float)L * ltausipkp);
        gm = lM * (1.0f + (float)L * ltaup);
        fm = 2.0f * lmu * (1.0f + (float)L * ltaus);
        dipjp = lmuipjp * ltausipjp / g.dt; djpkp = lmujpkp * ltausjpkp / g.dt; dipkp = lmuipkp * ltausipkp / g.dt;
        d = 2.0f * lmu * ltaus / g.dt; e = lM * ltaup / g.dt;
    }
    float vxyyx = vxy + vyx, vyzzy = vyz + vzy, vxzzx = vxz + vzx;
    float vxxyyzz = vxx + vyy + vzz, vyyzz = vyy + vzz, vxxzz = vxx + vzz, vxxyy = vxx + vyy;
    float s[6] = {0, 0, 0, 0, 0, 0};
    if (g.ckpt) {
        s[0] = fwd_at<T>(g, a, SXY, iv); s[1] = fwd_at<T>(g, a, SYZ, iv); s[2] = fwd_at<T>(g, a, SXZ, iv);
        s[3] = fwd_at<T>(g, a, SXX, iv); s[4] = fwd_at<T>(g, a, SYY, iv); s[5] = fwd_at<T>(g, a, SZZ, iv);
    } else if (!g.bp2) {
        s[0] = f.w[SXY][iv]; s[1] = f.w[SYZ][iv]; s[2] = f.w[SXZ][iv];
        s[3] = f.w[SXX][iv]; s[4] = f.w[SYY][iv]; s[5] = f.w[SZZ][iv];
    }
    float *const *r = f.r;
    if (g.bp2 || g.ckpt) {
    } else if (L == 0) {
        s[0] -= fipjp * vxyyx; s[1] -= fjpkp * vyzzy; s[2] -= fipkp * vxzzx;
        s[3] -= gm * vxxyyzz - fm * vyyzz; s[4] -= gm * vxxyyzz - fm * vxxzz; s[5] -= gm * vxxyyzz - fm * vxxyy;
    } else {
        float aa[6] = {0, 0, 0, 0, 0, 0};
        for (int l = 0; l < L; l++) {
            i64 ir = l * g.nvol + iv;
            aa[0] += r[RXY][ir]; aa[1] += r[RYZ][ir]; aa[2] += r[RXZ][ir];
            aa[3] += r[RXX][ir]; aa[4] += r[RYY][ir]; aa[5] += r[RZZ][ir];
        }
        float ls[6] = {fipjp * vxyyx + g.dt2 * aa[0], fjpkp * vyzzy + g.dt2 * aa[1], fipkp * vxzzx + g.dt2 * aa[2],
                       (gm * vxxyyzz - fm * vyyzz) + g.dt2 * aa[3], (gm * vxxyyzz - fm * vxxzz) + g.dt2 * aa[4],
                       (gm * vxxyyzz - fm * vxxyy) + g.dt2 * aa[5]};
        for (int q = 0; q < 6; q++) aa[q] = 0;
        // 3D reconstruction keeps the forward-time coefficients (update_adjs3D.cl:357-359)
        for (int l = 0; l < L; l++) {
            float el = g.eta[l];
            float b = 1.0f / (1.0f + el * 0.5f), c = 1.0f - el * 0.5f;
            i64 ir = l * g.nvol + iv;
            float n0 = b * (r[RXY][ir] * c - el * (dipjp * vxyyx));
            float n1 = b * (r[RYZ][ir] * c - el * (djpkp * vyzzy));
            float n2 = b * (r[RXZ][ir] * c - el * (dipkp * vxzzx));
            float n3 = b * (r[RXX][ir] * c - el * (e * vxxyyzz - d * vyyzz));
            float n4 = b * (r[RYY][ir] * c - el * (e * vxxyyzz - d * vxxzz));
            float n5 = b * (r[RZZ][ir] * c - el * (e * vxxyyzz - d * vxxyy));
            r[RXY][ir] = n0; r[RYZ][ir] = n1; r[RXZ][ir] = n2; r[RXX][ir] = n3; r[RYY][ir] = n4; r[RZZ][ir] = n5;
            aa[0] += n0; aa[1] += n1; aa[2] += n2; aa[3] += n3; aa[4] += n4; aa[5] += n5;
        }
        for (int q = 0; q < 6; q++) s[q] -= ls[q] + g.dt2 * aa[q];
    }
    if (!g.bp2 && !g.ckpt) {
        int m = inject_ind3d(g, gz, gy, gx);
        if (m != -1) {
            s[3] = bnd_at<T>(g, a, SXX, m); s[4] = bnd_at<T>(g, a, SYY, m);
            s[5] = bnd_at<T>(g, a, SZZ, m); s[0] = bnd_at<T>(g, a, SXY, m);
            s[1] = bnd_at<T>(g, a, SYZ, m); s[2] = bnd_at<T>(g, a, SXZ, m);
        }
        f.w[SXY][iv] = s[0]; f.w[SYZ][iv] = s[1]; f.w[SXZ][iv] = s[2];
        f.w[SXX][iv] = s[3]; f.w[SYY][iv] = s[4]; f.w[SZZ][iv] = s[5];
    }
    if (g.abs_type == 1) cpml_s3d(g, f, gz, gy, gx, vxxr, vxyr, vxzr, vyxr, vyyr, vyzr, vzxr, vzyr, vzzr, true);
    float vxyyxr = vxyr + vyxr, vyzzyr = vyzr + vzyr, vxzzxr = vxzr + vzxr;
    float vxxyyzzr = vxxr + vyyr + vzzr, vyyzzr = vyyr + vzzr, vxxzzr = vxxr + vzzr, vxxyyr = vxxr + vyyr;
    float ls[6];
    ls[0] = fipjp * vxyyxr; ls[1] = fjpkp * vyzzyr; ls[2] = fipkp * vxzzxr;
    ls[3] = gm * vxxyyzzr - fm * vyyzzr; ls[4] = gm * vxxyyzzr - fm * vxxzzr; ls[5] = gm * vxxyyzzr - fm * vxxyyr;
    float *const *wr = a.wr;
    const int sid[6] = {SXY, SYZ, SXZ, SXX, SYY, SZZ};
    if (L == 0) {
        for (int q = 0; q < 6; q++) wr[sid[q]][iv] += ls[q];
    } else {
        float *const *rr = a.rr;
        const int rid[6] = {RXY, RYZ, RXZ, RXX, RYY, RZZ};
        float aa[6] = {0, 0, 0, 0, 0, 0};
        for (int l = 0; l < L; l++) {
            i64 ir = l * g.nvol + iv;
            for (int q = 0; q < 6; q++) aa[q] += rr[rid[q]][ir];
        }
        for (int q = 0; q < 6; q++) ls[q] += g.dt2 * aa[q];
        // the reference stores these into the forward memory variables and
        // keeps only the last adjoint value of each sum (update_adjs3D.cl:566-583);
        // a checkpointed adjoint skips the stores (dead: the forward arrays are
        // reloaded from a snapshot before they are read)
        for (int l = 0; l < L; l++) {
            i64 ir = l * g.nvol + iv;
            if (!g.ckpt) {
                float el = g.eta[l];
                float b = 1.0f / (1.0f + el * 0.5f), c = 1.0f - el * 0.5f;
                r[RXY][ir] = b * (rr[RXY][ir] * c - el * (dipjp * vxyyxr));
                r[RYZ][ir] = b * (rr[RYZ][ir] * c - el * (djpkp * vyzzyr));
                r[RXZ][ir] = b * (rr[RXZ][ir] * c - el * (dipkp * vxzzxr));
                r[RXX][ir] = b * (rr[RXX][ir] * c - el * (e * vxxyyzzr - d * vyyzzr));
                r[RYY][ir] = b * (rr[RYY][ir] * c - el * (e * vxxyyzzr - d * vxxzzr));
                r[RZZ][ir] = b * (rr[RZZ][ir] * c - el * (e * vxxyyzzr - d * vxxyyr));
            }
            // after the stores: in the DFT adjoint r and rr are one buffer
            for (int q = 0; q < 6; q++) aa[q] = rr[rid[q]][ir];
        }
        for (int q = 0; q < 6; q++) wr[sid[q]][iv] += ls[q] + g.dt2 * aa[q];
    }
    if (g.abs_type == 2) {
        float *fs[6] = {wr[SXY], wr[SYZ], wr[SXZ], wr[SXX], wr[SYY], wr[SZZ]};
        apply_taper<6>(g, f.taper, gz, gy, gx, fs, iv);
    }
    float sxx = s[3], syy = s[4], szz = s[5], sxy = s[0], syz = s[1], sxz = s[2];
    float lsxy = ls[0], lsyz = ls[1], lsxz = ls[2], lsxx = ls[3], lsyy = ls[4], lszz = ls[5];
    if (g.bp2) {
    } else if (g.restype == 0) {
        float c1 = 1.0f / (3.0f * lM - 4.0f * lmu) / (3.0f * lM - 4.0f * lmu);
        float c3 = 1.0f / lmu / lmu;
        float c5 = 1.0f / 6.0f * c3;
        float dM = c1 * (sxx + syy + szz) * (lsxx + lsyy + lszz);
        a.grad[GM][ip] += (double)(-dM);
        a.grad[GMU][ip] += (double)(-c3 * (sxz * lsxz + sxy * lsxy + syz * lsyz) + 4.0f / 3.0f * dM -
                                    c5 * (lsxx * (2.0f * sxx - syy - szz) + lsyy * (2.0f * syy - sxx - szz) +
                                          lszz * (2.0f * szz - sxx - syy)));
    } else {
        float dM = (sxx + syy + szz) * (lsxx + lsyy + lszz);
        a.grad[GM][ip] += (double)(-dM);
    }
}

// surface adjoint 3D (surface3D_adj.cl:29-116), two passes like 2D.  The
// reference reads the syy component from sxxr (:62).
template <int F>
__global__ void k_surfadj3d_a(Grid g, Fields f, AdjFields a, float *q)
{
    SHOT_FA
    q += blockIdx.z * g.sb_q;
    int gy = blockIdx.x * blockDim.x + threadIdx.x + F;
    int gx = blockIdx.y * blockDim.y + threadIdx.y + F;
    if (gy > g.NY - F - 1 || gx > g.NX - F - 1) return;
    int gz = F;
    const i64 sx = (i64)g.NY * g.NZ, sy = g.NZ;
    i64 iv = gx * sx + (i64)gy * sy + gz;
    i64 ip = ((i64)(gx - F) * g.ny + (gy - F)) * g.nz + (gz - F);
    float lszz = -a.wr[SZZ][iv], lsxx = -a.wr[SXX][iv], lsyy = -a.wr[SXX][iv];
    float lmu = f.p[PMU][ip], lM = f.p[PM][ip];
    float t1 = lsxx, t2 = lsyy, t3 = lszz;
    float aa = 1.0f / (6.0f * lM * lmu - 8.0f * lmu * lmu);
    lsxx = aa * (2.0f * (lM - lmu) * t1 + (-lM + 2.0f * lmu) * (t2 + t3));
    lsyy = aa * (2.0f * (lM - lmu) * t2 + (-lM + 2.0f * lmu) * (t1 + t3));
    lszz = 0.0f;
    float h = -((lM - lmu * 2.0f) * (lM - lmu * 2.0f) / lM);
    float hz = -(lM - lmu * 2.0f);
    for (int m = 0; m < F; m++) a.wr[VZ][iv + m] += g.hc[m] * hz * (lsxx + lsyy) * f.p[PRKP][ip + m];
    q[(i64)(gx - F) * g.ny + (gy - F)] = h * (lsxx + lsyy);
    a.wr[SXX][iv] = -(lM * lsxx + (lM - 2.0f * lmu) * (lsyy + lszz));
    a.wr[SYY][iv] = -(lM * lsyy + (lM - 2.0f * lmu) * (lsxx + lszz));
    a.wr[SZZ][iv] = -(lM * lszz + (lM - 2.0f * lmu) * (lsxx + lsyy));
}
template <int F>
__global__ void k_surfadj3d_b(Grid g, Fields f, AdjFields a, const float *q)
{
    SHOT_FA
    q += blockIdx.z * g.sb_q;
    int gy = blockIdx.x * blockDim.x + threadIdx.x + F;
    int gx = blockIdx.y * blockDim.y + threadIdx.y + F;
    if (gy > g.NY - F - 1 || gx > g.NX - F - 1) return;
    int gz = F, x = gx - F, y = gy - F, nx = g.nx, ny = g.ny;
    const i64 sx = (i64)g.NY * g.NZ, sy = g.NZ;
    i64 iv = gx * sx + (i64)gy * sy + gz;
    i64 ip = ((i64)x * g.ny + y) * g.nz;
    float accx = 0.0f, accy = 0.0f;
    for (int m = 0; m < F; m++) {
        if (x - m >= 0) accx += g.hc[m] * q[(i64)(x - m) * ny + y];
        if (x + m + 1 < nx) accx -= g.hc[m] * q[(i64)(x + m + 1) * ny + y];
        if (y - m >= 0) accy += g.hc[m] * q[(i64)x * ny + (y - m)];
        if (y + m + 1 < ny) accy -= g.hc[m] * q[(i64)x * ny + (y + m + 1)];
    }
    a.wr[VX][iv] += accx * f.p[PRIP][ip];
    a.wr[VY][iv] += accy * f.p[PRJP][ip];
}

// ------------------------------------------------ point kernels (per shot)
// src/automatic_kernels.c:394-629; several sources may share a cell
template <class T>
__device__ __forceinline__ void source_point(const Fields &f, const PointSet &s, const float *src, int nt_total,
                                             int t, int pdir, float dt, int freesurf, int F, const WScale &ws,
                                             int gid)
{
    i64 cell = s.cell[gid];
    if (cell < 0) return;
    if (freesurf && pdir == -1 && s.kz[gid] < 2 * F) return;
    float amp = (float)pdir * (dt * src[(i64)gid * nt_total + t]);
    for (int q = 0; q < s.ntarget[gid]; q++) {
        float dv = s.div[gid * 3 + q];
        float val = dv == 0.0f ? amp : amp / dv;
        const int w = s.field[gid * 3 + q];
        atomicAdd(fld<T>(f.w[w]) + cell, (T)(val * ws.w[w]));
    }
}

template <class T = float>
__global__ void k_sources(Fields f, PointSet s, const float *src, int nt_total, int t, int pdir, float dt,
                          int freesurf, int F, WScale ws)
{
    pdl_trigger();
    pdl_wait();
    int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid < s.n) source_point<T>(f, s, src, nt_total, t, pdir, dt, freesurf, F, ws, gid);
}

// src/automatic_kernels.c:22-219; out is [nsel][nrec][NT].  L2: the loads
// bypass L1 (values stored by other blocks of the running kernel).
template <class T> __device__ __forceinline__ float ldv_l2(const T *p);
template <> __device__ __forceinline__ float ldv_l2<float>(const float *p) { return __ldcg(p); }
template <> __device__ __forceinline__ float ldv_l2<__half>(const __half *p) { return __half2float(__ldcg(p)); }

template <class T, bool L2>
__device__ __forceinline__ void record_point(const Fields &f, const PointSet &r, float *out, int nt_total, int t,
                                             unsigned outmask, int nd, const WScale &ws, int gid)
{
    i64 cell = r.cell[gid];
    if (cell < 0) return;
    auto ld = [](const T *q) { return L2 ? ldv_l2<T>(q) : ldv(q); };
    int slot = 0;
    for (int o = 0; o < SFD_NOUT; o++) {
        if (!(outmask & (1u << o))) continue;
        float v;
        if (o == SFD_OUT_P) {
            const T *xx = fld<T>(f.w[SXX]), *zz = fld<T>(f.w[SZZ]);
            if (nd == 3) v = (ld(xx + cell) + ld(zz + cell) + ld(fld<T>(f.w[SYY]) + cell)) / 3.0f;
            else if (nd == 22) v = ld(xx + cell);
            else v = (ld(xx + cell) + ld(zz + cell)) / 2.0f;
            v /= ws.w[SXX];
        } else {
            v = ld(fld<T>(f.w[o]) + cell) / ws.w[o];
        }
        out[((i64)slot * r.n + gid) * nt_total + t] = v;
        slot++;
    }
}

template <class T = float>
__global__ void k_record(Fields f, PointSet r, float *out, int nt_total, int t, unsigned outmask, int nd, WScale ws)
{
    pdl_trigger();
    pdl_wait();
    int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid < r.n) record_point<T, false>(f, r, out, nt_total, t, outmask, nd, ws, gid);
}

// ---------------------------------------------- fused 2D forward step tail
// The stress kernel of a fused 2D step ends with the receivers of step t
// and the sources of step t+1 (time_stepping.c:783-816 order: sources,
// update_v, update_s, surface, record), run by the block that finishes
// last: every block fences its stores and takes a ticket; the block with
// the last ticket sees all stores of the launch, records, adds the next
// step's sources and resets the ticket.  Nothing waits on another block.
template <class T = float>
__device__ __forceinline__ void step_tail(const Grid &g, const Fields &f, const StepTail &tl)
{
    __shared__ int s_last;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nth = blockDim.x * blockDim.y * blockDim.z;
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = atomicAdd(tl.ticket, 1) == (int)(gridDim.x * gridDim.y * gridDim.z) - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    for (int i = tid; i < tl.rec.n; i += nth)
        record_point<T, true>(f, tl.rec, tl.out, tl.nt_total, tl.t, tl.outmask, g.nd, g.ws, i);
    __syncthreads();
    if (tl.tsrc >= 0)
        for (int i = tid; i < tl.src.n; i += nth)
            source_point<T>(f, tl.src, tl.stf, tl.nt_total, tl.tsrc, 1, g.dt, g.freesurf, g.F, g.ws, i);
    if (tid == 0) *tl.ticket = 0;
}

// P-SV stress update, free surface (blocks of the top row: their 32 z
// rows hold every stress the surface reads, rows F..2F) and step tail.
// pdir (1) is a launch argument, as for the separate surface kernel, so
// that both contract and round alike.
template <int F, class T = float>
__global__ void __launch_bounds__(256) k_s2d_step(Grid g, Fields f, StepTail tl, int pdir)
{
    int gz = blockIdx.x * blockDim.x + threadIdx.x + F;
    int gx = blockIdx.y * blockDim.y + threadIdx.y + F;
    Fields fs = f;   // this block's shot; the tail's points carry their shot in their cells
    if (g.nb > 1) shot_fields(g, fs, blockIdx.z);
    if (gz <= g.NZ - F - 1 && gx <= g.NX - F - 1) s2d_cell<F, T>(g, fs, gz, gx);
    if (g.freesurf && blockIdx.x == 0) {
        __syncthreads();
        if (threadIdx.x == 0 && gx <= g.NX - F - 1) surf2d_column<F, T>(g, fs, gx, pdir);
    }
    step_tail<T>(g, f, tl);
}

// acoustic pressure update and step tail (no free-surface kernel)
template <int F>
__global__ void __launch_bounds__(256) k_s2d_acc_step(Grid g, Fields f, StepTail tl)
{
    int gz = blockIdx.x * blockDim.x + threadIdx.x + F;
    int gx = blockIdx.y * blockDim.y + threadIdx.y + F;
    Fields fs = f;
    if (g.nb > 1) shot_fields(g, fs, blockIdx.z);
    if (gz <= g.NZ - F - 1 && gx <= g.NX - F - 1) s2d_acc_cell<F>(g, fs, gz, gx);
    step_tail(g, f, tl);
}

// src/automatic_kernels.c:631-836; res is [nsel][nrec][NT]
__global__ void k_residuals(AdjFields a, PointSet r, const float *res, int nt_total, int t, unsigned outmask, int nd)
{
    int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= r.n) return;
    i64 cell = r.cell[gid];
    if (cell < 0) return;
    int slot = 0;
    for (int o = 0; o < SFD_NOUT; o++) {
        if (!(outmask & (1u << o))) continue;
        float v = res[((i64)slot * r.n + gid) * nt_total + t];
        if (o == SFD_OUT_P) {
            float n2 = nd == 3 ? 3.0f : 2.0f;
            atomicAdd(a.wr[SXX] + cell, v / n2);
            atomicAdd(a.wr[SZZ] + cell, v / n2);
            if (nd == 3) atomicAdd(a.wr[SYY] + cell, v / n2);
        } else {
            atomicAdd(a.wr[o] + cell, v);
        }
        slot++;
    }
}

// ------------------------------------------------------------- launchers
static inline unsigned cdiv(long a, long b) { return (unsigned)((a + b - 1) / b); }

// CTA shape (quads x y rows x x planes) of a 4-cell launch: the preferred
// shape, or half as many quads along z and twice the rows when that leaves
// fewer threads without a quad (nz = 200: 50 quads per column fill 56 slots
// of 8 instead of 64 of 16)
static dim3 q4_block(const Grid &g, unsigned bx, unsigned by, unsigned bz)
{
    const unsigned nq = (unsigned)(g.nz / 4);
    if (bx >= 16 && cdiv(nq, bx / 2) * (bx / 2) < cdiv(nq, bx) * bx) return dim3(bx / 2, by * 2, bz);
    return dim3(bx, by, bz);
}
static dim3 q4_grid(const Grid &g, dim3 b)
{
    return dim3(cdiv(g.nz / 4, b.x), cdiv(g.ny, b.y), cdiv(g.nx, b.z) * g.nb);
}

// batched launches (several shots) use the MB = true instantiations
#define MB_DISPATCH(g, ...)                                                     \
    if ((g).nb > 1) { constexpr bool MBV = true; __VA_ARGS__; }                  \
    else { constexpr bool MBV = false; __VA_ARGS__; }

#define DISPATCH_F(F, ...)                                                      \
    switch (F) {                                                               \
    case 1: { constexpr int FF = 1; __VA_ARGS__; } break;                      \
    case 2: { constexpr int FF = 2; __VA_ARGS__; } break;                      \
    case 3: { constexpr int FF = 3; __VA_ARGS__; } break;                      \
    case 4: { constexpr int FF = 4; __VA_ARGS__; } break;                      \
    case 5: { constexpr int FF = 5; __VA_ARGS__; } break;                      \
    case 6: { constexpr int FF = 6; __VA_ARGS__; } break;                      \
    default: break;                                                            \
    }

void launch_update_v(const Grid &g, const Fields &f, cudaStream_t st)
{
    if (g.fhalf && g.nd == 3) {   // FP16 storage: the vectorised or the streaming kernels
        if (q4_ok(g)) {
            dim3 b(8, 4, 4), gr(cdiv(g.nz / 4, 8), cdiv(g.ny, 4), cdiv(g.nx, 4) * g.nb);
            k_v3d_q4<__half><<<gr, b, 0, st>>>(g, f);
            return;
        }
        dim3 b(32, 4, 2), gr(cdiv(g.nz, 32), cdiv(g.ny, 4), cdiv(g.nx, 2) * g.nb);
        DISPATCH_F(g.F, k_v3d_stream<FF, __half><<<gr, b, 0, st>>>(g, f));
        return;
    }
    // kernels 0 takes the 4-cell vectorised kernel where it applies (0.43 ms
    // at 256^3, against 0.57 streaming, 0.58 general and 0.63 TMA), else the
    // streaming one; only kernels 3 takes the TMA path
    if (g.kernels == 3 && launch_update_v_tma(g, f, st)) return;
    if (g.kernels == 2 && launch_update_v_fast(g, f, st)) return;
    if (g.vasync && launch_update_v_async(g, f, st)) return;
    if (g.nd == 21 || g.nd == 22) {
        dim3 b(32, 8), gr(cdiv(g.nz, 32), cdiv(g.nx, 8), g.nb);
        if (g.nd == 21) DISPATCH_F(g.F, k_v2d_sh<FF><<<gr, b, 0, st>>>(g, f))
        else DISPATCH_F(g.F, k_v2d_acc<FF><<<gr, b, 0, st>>>(g, f))
        return;
    }
    if (g.nd == 3) {
        if ((g.kernels == 0 || g.kernels == 5) && q4_ok(g)) {
            // 16 quads (64 z cells) x 4 y x 2 x per CTA: the y and x stencil
            // rows of neighbouring threads share L1 lines.  Interior-only
            // timing at 256^3 on a B200: 0.268 ms, against 0.275 for 8 x 4 x
            // 4, 0.284 for 8 x 2 x 8 and 0.34 for 4 x 8 x 4 quads x y x x
            const dim3 b = q4_block(g, 16, 4, 2), gr = q4_grid(g, b);
            if (g.nb > 1) k_v3d_q4<float, true><<<gr, b, 0, st>>>(g, f);
            // an ordinary launch (after the sources, which are complete by
            // then) that lets the stress kernel launch early; launched with
            // programmatic serialization itself it would need plain loads:
            // 1.0062 against 1.0038 ms per step at 256^3, L=2
            else if (pdl_enabled()) k_v3d_q4_b4<true><<<gr, b, 0, st>>>(g, f);
            else k_v3d_q4_b4<<<gr, b, 0, st>>>(g, f);
            return;
        }
        dim3 b(32, 4, 2), gr(cdiv(g.nz, 32), cdiv(g.ny, 4), cdiv(g.nx, 2) * g.nb);
        if (g.kernels == 0 || g.kernels == 4 || g.kernels == 5) {
            DISPATCH_F(g.F, MB_DISPATCH(g, k_v3d_stream<FF, float, MBV><<<gr, b, 0, st>>>(g, f)));
            return;
        }
        DISPATCH_F(g.F, MB_DISPATCH(g, k_v3d<FF, MBV><<<gr, b, 0, st>>>(g, f)));
    } else {
        dim3 b(32, 8), gr(cdiv(g.nz, 32), cdiv(g.nx, 8), g.nb);
        if (g.fhalf) DISPATCH_F(g.F, k_v2d<FF, __half><<<gr, b, 0, st>>>(g, f))
        else DISPATCH_F(g.F, k_v2d<FF><<<gr, b, 0, st>>>(g, f));
    }
}

// the FP32 stream-prefetch stress kernel; TR: storage type of the memory variables
template <int L, class TR>
static void launch_s_pf(const Grid &g, const Fields &f, dim3 g4, dim3 b4, cudaStream_t st, bool surf, bool pdl)
{
    if (pdl) launch_pdl(k_s3d_q4_pf<L, float, true, TR>, g4, b4, st, g, f, surf);
    else k_s3d_q4_pf<L, float, false, TR><<<g4, b4, 0, st>>>(g, f, surf);
}

bool launch_update_s(const Grid &g, const Fields &f, cudaStream_t st, bool fold_surface)
{
    if (g.fhalf && g.nd == 3 && g.L <= 3) {   // FP16 storage: the vectorised or the streaming kernels
        if (q4_ok(g)) {
            const dim3 b4 = q4_block(g, 16, 8, 1), g4 = q4_grid(g, b4);
            if (g.kernels == 0 && g.nb == 1 && g.L > 0) {   // with the stream prefetch, as the FP32 default
                // ordinary launches: with programmatic serialization the FP16
                // velocities need plain loads, which cost this kernel more than
                // the overlap gives (0.510 against 0.489 ms at 256^3, L=2)
                switch (g.L) {
                case 0: k_s3d_q4_pf<0, __half><<<g4, b4, 0, st>>>(g, f, false); break;
                case 1: k_s3d_q4_pf<1, __half><<<g4, b4, 0, st>>>(g, f, false); break;
                case 2: k_s3d_q4_pf<2, __half><<<g4, b4, 0, st>>>(g, f, false); break;
                default: k_s3d_q4_pf<3, __half><<<g4, b4, 0, st>>>(g, f, false); break;
                }
                return false;
            }
            switch (g.L) {
            case 0: k_s3d_q4<0, __half><<<g4, b4, 0, st>>>(g, f, false); break;
            case 1: k_s3d_q4<1, __half><<<g4, b4, 0, st>>>(g, f, false); break;
            case 2: k_s3d_q4<2, __half><<<g4, b4, 0, st>>>(g, f, false); break;
            default: k_s3d_q4<3, __half><<<g4, b4, 0, st>>>(g, f, false); break;
            }
            return false;
        }
        dim3 b(32, 4, 2), gr(cdiv(g.nz, 32), cdiv(g.ny, 4), cdiv(g.nx, 2) * g.nb);
        switch (g.L) {
        case 0: DISPATCH_F(g.F, k_s3d_stream<FF, 0, __half><<<gr, b, 0, st>>>(g, f)); break;
        case 1: DISPATCH_F(g.F, k_s3d_stream<FF, 1, __half><<<gr, b, 0, st>>>(g, f)); break;
        case 2: DISPATCH_F(g.F, k_s3d_stream<FF, 2, __half><<<gr, b, 0, st>>>(g, f)); break;
        default: DISPATCH_F(g.F, k_s3d_stream<FF, 3, __half><<<gr, b, 0, st>>>(g, f)); break;
        }
        return false;
    }
    // kernels 0: the 4-cell vectorised kernel where it applies (0.74 ms at
    // 256^3, against 0.96 TMA and 0.98 streaming), else the streaming one
    if (g.kernels == 3 && launch_update_s_tma(g, f, st)) return false;
    if (g.kernels == 2 && launch_update_s_fast(g, f, st)) return false;
    // single-shot FP32 4-cell kernels apply the free surface in the same launch
    const bool surf = fold_surface && g.freesurf && g.nb == 1;
    if (g.nd == 21 || g.nd == 22) {
        dim3 b(32, 8), gr(cdiv(g.nz, 32), cdiv(g.nx, 8), g.nb);
        if (g.nd == 21) DISPATCH_F(g.F, k_s2d_sh<FF><<<gr, b, 0, st>>>(g, f))
        else DISPATCH_F(g.F, k_s2d_acc<FF><<<gr, b, 0, st>>>(g, f))
        return false;
    }
    if (g.nd == 3) {
        dim3 b(32, 4, 2), gr(cdiv(g.nz, 32), cdiv(g.ny, 4), cdiv(g.nx, 2) * g.nb);
        if ((g.kernels == 0 || g.kernels == 5) && q4_ok(g) && g.L <= 3) {
            const dim3 b4 = q4_block(g, 16, 8, 1), g4 = q4_grid(g, b4);  // 0.70 ms vs 0.71 (32 x 2 x 2)
            // the stream prefetch pays where memory variables add per-cell
            // streams: 256^3, L=2: 0.654 ms against 0.706; elastic (L=0):
            // 0.376 against 0.366 without it.  kernels 5 keeps k_s3d_q4.
            if (g.nb == 1 && g.kernels == 0 && g.L > 0) {
                const bool pdl = pdl_enabled();
                switch (g.L) {
                case 0: launch_s_pf<0, float>(g, f, g4, b4, st, surf, pdl); break;
                case 1: if (g.rhalf) launch_s_pf<1, __half>(g, f, g4, b4, st, surf, pdl);
                        else launch_s_pf<1, float>(g, f, g4, b4, st, surf, pdl);
                        break;
                case 2: if (g.rhalf) launch_s_pf<2, __half>(g, f, g4, b4, st, surf, pdl);
                        else launch_s_pf<2, float>(g, f, g4, b4, st, surf, pdl);
                        break;
                default: if (g.rhalf) launch_s_pf<3, __half>(g, f, g4, b4, st, surf, pdl);
                         else launch_s_pf<3, float>(g, f, g4, b4, st, surf, pdl);
                         break;
                }
                return surf;
            }
            switch (g.L) {
            case 0: MB_DISPATCH(g, k_s3d_q4<0, float, MBV><<<g4, b4, 0, st>>>(g, f, surf)) break;
            case 1: MB_DISPATCH(g, k_s3d_q4<1, float, MBV><<<g4, b4, 0, st>>>(g, f, surf)) break;
            case 2: MB_DISPATCH(g, k_s3d_q4<2, float, MBV><<<g4, b4, 0, st>>>(g, f, surf)) break;
            default: MB_DISPATCH(g, k_s3d_q4<3, float, MBV><<<g4, b4, 0, st>>>(g, f, surf)) break;
            }
            return surf;
        }
        if ((g.kernels == 0 || g.kernels == 4 || g.kernels == 5) && g.L <= 3) {
            switch (g.L) {
            case 0: DISPATCH_F(g.F, MB_DISPATCH(g, k_s3d_stream<FF, 0, float, MBV><<<gr, b, 0, st>>>(g, f))); break;
            case 1: DISPATCH_F(g.F, MB_DISPATCH(g, k_s3d_stream<FF, 1, float, MBV><<<gr, b, 0, st>>>(g, f))); break;
            case 2: DISPATCH_F(g.F, MB_DISPATCH(g, k_s3d_stream<FF, 2, float, MBV><<<gr, b, 0, st>>>(g, f))); break;
            default: DISPATCH_F(g.F, MB_DISPATCH(g, k_s3d_stream<FF, 3, float, MBV><<<gr, b, 0, st>>>(g, f))); break;
            }
            return false;
        }
        DISPATCH_F(g.F, MB_DISPATCH(g, k_s3d<FF, MBV><<<gr, b, 0, st>>>(g, f)));
    } else {
        dim3 b(32, 8), gr(cdiv(g.nz, 32), cdiv(g.nx, 8), g.nb);
        if (g.fhalf) DISPATCH_F(g.F, k_s2d<FF, __half><<<gr, b, 0, st>>>(g, f))
        else DISPATCH_F(g.F, k_s2d<FF><<<gr, b, 0, st>>>(g, f));
    }
    return false;
}

// movie snapshot (time_stepping.c:272-350): padded field -> [nx][ny][nz]
template <class T>
__global__ void k_movie(Grid g, const T *fld, float inv_scale, float *dst)
{
    const i64 n = (i64)g.nz * g.ny * g.nx;
    for (i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (i64)gridDim.x * blockDim.x) {
        const int k = (int)(idx % g.nz);
        const i64 r = idx / g.nz;
        const int j = (int)(r % g.ny), i = (int)(r / g.ny);
        const i64 iv = ((i64)(i + g.F) * g.NY + (g.nd == 3 ? j + g.F : 0)) * g.NZ + (k + g.F);
        dst[idx] = to_f<T>(fld[iv]) * inv_scale;
    }
}

// One wave field scanned for non-finite values (the reference tests the
// misfit for NaN once per run, src/residuals.c:444-448; here the field is
// tested every FINITE_CHECK_EVERY steps so a run reports the step near which
// it diverged).
template <class T>
__global__ void __launch_bounds__(256) k_finite(const T *__restrict__ v, i64 n, int t, int *first)
{
    bool bad = false;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        bad |= !isfinite(to_f<T>(v[i]));
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicMin(first, t);
}
__global__ void __launch_bounds__(256) k_finite4(const float4 *__restrict__ v, i64 n4, int t, int *first)
{
    bool bad = false;
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n4; i += (i64)gridDim.x * blockDim.x) {
        const float4 q = __ldg(v + i);
        bad |= !(isfinite(q.x) && isfinite(q.y) && isfinite(q.z) && isfinite(q.w));
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicMin(first, t);
}

void launch_finite_check(const Grid &g, const float *fld, int64_t n, int t, int *first, cudaStream_t st)
{
    if (!fld || n <= 0) return;
    const unsigned blocks = (unsigned)std::min<i64>((n + 1023) / 1024, 148 * 8);
    if (g.fhalf) k_finite<__half><<<blocks, 256, 0, st>>>(reinterpret_cast<const __half *>(fld), n, t, first);
    else if (n % 4 == 0 && ((uintptr_t)fld & 15) == 0)
        k_finite4<<<blocks, 256, 0, st>>>(reinterpret_cast<const float4 *>(fld), n / 4, t, first);
    else k_finite<float><<<blocks, 256, 0, st>>>(fld, n, t, first);
}

void launch_movie(const Grid &g, const float *fld, float inv_scale, float *dst, cudaStream_t st)
{
    const i64 n = (i64)g.nz * g.ny * g.nx;
    unsigned blocks = (unsigned)std::min<i64>((n + 255) / 256, 148 * 16);
    if (g.fhalf) k_movie<__half><<<blocks, 256, 0, st>>>(g, reinterpret_cast<const __half *>(fld), inv_scale, dst);
    else k_movie<float><<<blocks, 256, 0, st>>>(g, fld, inv_scale, dst);
}

int stress_family(const Grid &g, const Fields &f)
{
    // the same selection as launch_update_s
    if (g.nd != 3) return 0;
    if (g.fhalf && g.L <= 3) return q4_ok(g) ? 5 : 4;
    if (g.kernels == 3 && tma_ready(g, f)) return 3;
    if (g.kernels == 2) return 2;
    if ((g.kernels == 0 || g.kernels == 5) && q4_ok(g) && g.L <= 3) return 5;
    if ((g.kernels == 0 || g.kernels == 4 || g.kernels == 5) && g.L <= 3) return 4;
    return 1;
}

bool launch_update_s_step(const Grid &g, const Fields &f, const StepTail &tl, cudaStream_t st)
{
    if (g.nd != 2 && g.nd != 22) return false;
    dim3 b(32, 8), gr(cdiv(g.nz, 32), cdiv(g.nx, 8), g.nb);   // 32 z rows >= 2F + 1: the surface stays in its block
    if (g.nd == 2 && g.fhalf) DISPATCH_F(g.F, k_s2d_step<FF, __half><<<gr, b, 0, st>>>(g, f, tl, 1))
    else if (g.nd == 2) DISPATCH_F(g.F, k_s2d_step<FF><<<gr, b, 0, st>>>(g, f, tl, 1))
    else DISPATCH_F(g.F, k_s2d_acc_step<FF><<<gr, b, 0, st>>>(g, f, tl))
    return true;
}

void launch_surface(const Grid &g, const Fields &f, int pdir, cudaStream_t st)
{
    if (g.nd == 21) {
        DISPATCH_F(g.F, k_surf_sh<FF><<<cdiv(g.nx, 128), 128, 0, st>>>(g, f));
        return;
    }
    if (g.nd == 22) return;
    if (g.nd == 3) {
        dim3 b(32, 4), gr(cdiv(g.ny, 32), cdiv(g.nx, 4), g.nb);
        if (g.fhalf) DISPATCH_F(g.F, k_surf3d<FF, __half><<<gr, b, 0, st>>>(g, f, pdir))
        else if (g.rhalf) DISPATCH_F(g.F, (k_surf3d<FF, float, __half><<<gr, b, 0, st>>>(g, f, pdir)))
        else DISPATCH_F(g.F, k_surf3d<FF><<<gr, b, 0, st>>>(g, f, pdir))
    } else {
        if (g.fhalf) DISPATCH_F(g.F, k_surf2d<FF, __half><<<dim3(cdiv(g.nx, 128), 1, g.nb), 128, 0, st>>>(g, f, pdir))
        else DISPATCH_F(g.F, k_surf2d<FF><<<dim3(cdiv(g.nx, 128), 1, g.nb), 128, 0, st>>>(g, f, pdir));
    }
}

// S arrays (FP32 or FP16 wave fields) to T stores (pack) or FP32 arrays
// back from T stores (unpack), value times scale; one grid row per array, a
// grid-stride loop over its elements
template <class T, bool UNPACK, class S = float>
__global__ void k_pack(PackSet ps)
{
    const int q = blockIdx.y;
    const i64 n = ps.n[q];
    const float sc = ps.scale[q];
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        if (UNPACK) ((float *)ps.dst[q])[i] = to_f<T>(((const T *)ps.src[q])[i]) * sc;
        else ((T *)ps.dst[q])[i] = from_f<T>(to_f<S>(((const S *)ps.src[q])[i]) * sc);
    }
}

void launch_pack(const PackSet &ps, int prec, bool unpack, cudaStream_t st, bool half_src)
{
    if (ps.narr <= 0) return;
    i64 nmax = 0;
    for (int q = 0; q < ps.narr; q++) nmax = ps.n[q] > nmax ? ps.n[q] : nmax;
    dim3 gr((unsigned)std::min<i64>((nmax + 255) / 256, 148 * 8), (unsigned)ps.narr);
    if (gr.x == 0) return;
    if (half_src && !unpack) {
        if (prec == SFD_PREC_FP16) k_pack<__half, false, __half><<<gr, 256, 0, st>>>(ps);
        else if (prec == SFD_PREC_BF16) k_pack<__nv_bfloat16, false, __half><<<gr, 256, 0, st>>>(ps);
        else k_pack<float, false, __half><<<gr, 256, 0, st>>>(ps);
    } else if (prec == SFD_PREC_FP16) {
        if (unpack) k_pack<__half, true><<<gr, 256, 0, st>>>(ps);
        else k_pack<__half, false><<<gr, 256, 0, st>>>(ps);
    } else if (prec == SFD_PREC_BF16) {
        if (unpack) k_pack<__nv_bfloat16, true><<<gr, 256, 0, st>>>(ps);
        else k_pack<__nv_bfloat16, false><<<gr, 256, 0, st>>>(ps);
    } else {
        if (unpack) k_pack<float, true><<<gr, 256, 0, st>>>(ps);
        else k_pack<float, false><<<gr, 256, 0, st>>>(ps);
    }
}

void launch_savebnd(const Grid &g, const Fields &f, const BndSlot &b, int prec, int64_t tofs, cudaStream_t st)
{
    dim3 gr(cdiv(g.nbnd, 256), 1, g.nb);
    if (gr.x == 0) return;
    if (prec == SFD_PREC_FP16) k_savebnd<__half><<<gr, 256, 0, st>>>(g, f, b, tofs);
    else if (prec == SFD_PREC_BF16) k_savebnd<__nv_bfloat16><<<gr, 256, 0, st>>>(g, f, b, tofs);
    else k_savebnd<float><<<gr, 256, 0, st>>>(g, f, b, tofs);
}

template <typename T>
static void launch_adj_t(const Grid &g, const Fields &f, const AdjFields &a, bool stress, cudaStream_t st)
{
    if (g.nd == 3 && (g.kernels == 0 || g.kernels == 5) && q4_ok(g) && g.L <= 3) {
        const bool pf = g.kernels == 0 && g.nb == 1;   // kernels 5 keeps the kernels without the prefetch
        if (stress) {
            const dim3 b = q4_block(g, 16, 8, 1), gr = q4_grid(g, b);
            if (pf) {
                switch (g.L) {
                case 0: k_adjs3d_q4<0, T, false, true><<<gr, b, 0, st>>>(g, f, a); break;
                case 1: k_adjs3d_q4<1, T, false, true><<<gr, b, 0, st>>>(g, f, a); break;
                case 2: k_adjs3d_q4<2, T, false, true><<<gr, b, 0, st>>>(g, f, a); break;
                default: k_adjs3d_q4<3, T, false, true><<<gr, b, 0, st>>>(g, f, a); break;
                }
                return;
            }
            switch (g.L) {
            case 0: MB_DISPATCH(g, k_adjs3d_q4<0, T, MBV><<<gr, b, 0, st>>>(g, f, a)) break;
            case 1: MB_DISPATCH(g, k_adjs3d_q4<1, T, MBV><<<gr, b, 0, st>>>(g, f, a)) break;
            case 2: MB_DISPATCH(g, k_adjs3d_q4<2, T, MBV><<<gr, b, 0, st>>>(g, f, a)) break;
            default: MB_DISPATCH(g, k_adjs3d_q4<3, T, MBV><<<gr, b, 0, st>>>(g, f, a)) break;
            }
        } else {
            dim3 b(8, 4, 4), gr(cdiv(g.nz / 4, 8), cdiv(g.ny, 4), cdiv(g.nx, 4) * g.nb);
            if (pf) {
                k_adjv3d_q4<T, false, true><<<gr, b, 0, st>>>(g, f, a);
                return;
            }
            MB_DISPATCH(g, k_adjv3d_q4<T, MBV><<<gr, b, 0, st>>>(g, f, a))
        }
        return;
    }
    if (g.nd == 3) {
        dim3 b(32, 4, 2), gr(cdiv(g.nz, 32), cdiv(g.ny, 4), cdiv(g.nx, 2) * g.nb);
        if (stress) DISPATCH_F(g.F, MB_DISPATCH(g, k_adjs3d<FF, T, MBV><<<gr, b, 0, st>>>(g, f, a)))
        else DISPATCH_F(g.F, MB_DISPATCH(g, k_adjv3d<FF, T, MBV><<<gr, b, 0, st>>>(g, f, a)))
    } else {
        dim3 b(32, 8), gr(cdiv(g.nz, 32), cdiv(g.nx, 8), g.nb);
        if (stress) DISPATCH_F(g.F, k_adjs2d<FF, T><<<gr, b, 0, st>>>(g, f, a))
        else DISPATCH_F(g.F, k_adjv2d<FF, T><<<gr, b, 0, st>>>(g, f, a))
    }
}

void launch_update_adj(const Grid &g, const Fields &f, const AdjFields &a, bool stress, int prec, cudaStream_t st)
{
    if (prec == SFD_PREC_FP16) launch_adj_t<__half>(g, f, a, stress, st);
    else if (prec == SFD_PREC_BF16) launch_adj_t<__nv_bfloat16>(g, f, a, stress, st);
    else launch_adj_t<float>(g, f, a, stress, st);
}

void launch_surface_adj(const Grid &g, const Fields &f, const AdjFields &a, float *q, cudaStream_t st)
{
    if (g.nd == 3) {
        dim3 b(32, 4), gr(cdiv(g.ny, 32), cdiv(g.nx, 4), g.nb);
        DISPATCH_F(g.F, k_surfadj3d_a<FF><<<gr, b, 0, st>>>(g, f, a, q));
        DISPATCH_F(g.F, k_surfadj3d_b<FF><<<gr, b, 0, st>>>(g, f, a, q));
    } else {
        DISPATCH_F(g.F, k_surfadj2d_a<FF><<<dim3(cdiv(g.nx, 128), 1, g.nb), 128, 0, st>>>(g, f, a, q));
        DISPATCH_F(g.F, k_surfadj2d_b<FF><<<dim3(cdiv(g.nx, 128), 1, g.nb), 128, 0, st>>>(g, f, a, q));
    }
}

void launch_sources(const Grid &g, const Fields &f, const PointSet &s, const float *src, int nt_total, int t,
                    int pdir, cudaStream_t st)
{
    if (s.n == 0) return;
    const bool pdl = g.nd == 3 && g.nb == 1 && pdl_enabled();
    const dim3 gr(cdiv(s.n, 128)), b(128);
    if (g.fhalf)
        launch_maybe_pdl(pdl, k_sources<__half>, gr, b, st, f, s, src, nt_total, t, pdir, g.dt, g.freesurf, g.F, g.ws);
    else
        launch_maybe_pdl(pdl, k_sources<float>, gr, b, st, f, s, src, nt_total, t, pdir, g.dt, g.freesurf, g.F, g.ws);
}

void launch_record(const Grid &g, const Fields &f, const PointSet &r, float *out, int nt_total, int t,
                   unsigned outmask, cudaStream_t st)
{
    if (r.n == 0 || outmask == 0) return;
    const bool pdl = g.nd == 3 && g.nb == 1 && pdl_enabled();
    const dim3 gr(cdiv(r.n, 128)), b(128);
    if (g.fhalf) launch_maybe_pdl(pdl, k_record<__half>, gr, b, st, f, r, out, nt_total, t, outmask, g.nd, g.ws);
    else launch_maybe_pdl(pdl, k_record<float>, gr, b, st, f, r, out, nt_total, t, outmask, g.nd, g.ws);
}

void launch_residuals(const Grid &g, const AdjFields &a, const PointSet &r, const float *res, int nt_total, int t,
                      unsigned outmask, cudaStream_t st)
{
    if (r.n == 0 || outmask == 0) return;
    k_residuals<<<cdiv(r.n, 128), 128, 0, st>>>(a, r, res, nt_total, t, outmask, g.nd);
}

}  // namespace sfd
