// sfd_noalloc.cu -- forward modelling of one shot without any allocation.
//
// Some callers cannot call cudaMalloc on the path that runs a shot: a
// serving process that reserved its whole device memory budget up front and
// must not let a request grow it, or an embedding host whose allocator owns
// the device and forbids foreign allocations.  sfd_forward_noalloc serves
// them.  Its working memory -- wave fields, memory variables, CPML memory and
// the source/receiver maps -- lives in the fixed array below, which is part
// of the library image: every GPU that loads the library holds these
// SFD_NOALLOC_SCRATCH_BYTES until the process exits.  The caller passes its
// own device buffers for the shot inputs and for the seismograms.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "seiscl_b200.h"
#include "sfd_internal.h"
#include "sfd_kernels.h"
#include "sfd_setup.h"

using namespace sfd;

static __device__ __align__(256) unsigned char g_noalloc_scratch[SFD_NOALLOC_SCRATCH_BYTES];

namespace {

// Device address of the scratch array, looked up once per device.  In host
// code the symbol itself is only a host-side stand-in, never a device address.
constexpr int kMaxDevices = 64;
void *g_scratch_addr[kMaxDevices];
std::mutex g_scratch_lock;

int scratch_address(int device, void **out)
{
    if (device < 0 || device >= kMaxDevices) return SFD_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> guard(g_scratch_lock);
    if (!g_scratch_addr[device]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) return SFD_ERR_CUDA;
        g_scratch_addr[device] = ptr;
    }
    *out = g_scratch_addr[device];
    return SFD_OK;
}

// what a source of each type feeds (types 0..3, 100, anything else)
struct TargetTable {
    int n[6];
    int field[6][3];
    float div[6][3];
};

__device__ __forceinline__ int type_slot(int t) { return (t >= 0 && t < 4) ? t : (t == 100 ? 4 : 5); }

// cells of the shot's sources and receivers, (int)(pos/DH) + FDOH per axis
__global__ void k_noalloc_map(Grid g, double DH, const float *src_pos, int nsrc, const float *rec_pos, int nrec,
                              TargetTable tt, int64_t *scell, int *snt, int *sfield, float *sdiv, int *skz,
                              int64_t *rcell, int *bad)
{
    int gid = blockIdx.x * blockDim.x + threadIdx.x;
    const float *pos;
    if (gid < nsrc) pos = src_pos + 5 * gid;
    else if (gid < nsrc + nrec) pos = rec_pos + 8 * (gid - nsrc);
    else return;
    int i = (int)((double)pos[0] / DH) + g.F;
    int j = g.nd == 3 ? (int)((double)pos[1] / DH) + g.F : 0;
    int k = (int)((double)pos[2] / DH) + g.F;
    int64_t cell = -1;
    if (i >= g.F && i <= g.NX - g.F - 1) {
        if (j < 0 || j >= g.NY || k < 0 || k >= g.NZ) atomicExch(bad, 1);
        else cell = ((int64_t)i * g.NY + j) * g.NZ + k;
    }
    if (gid < nsrc) {
        int slot = type_slot((int)pos[4]);
        scell[gid] = cell;
        skz[gid] = k;
        snt[gid] = cell < 0 ? 0 : tt.n[slot];
        for (int q = 0; q < 3; q++) {
            sfield[3 * gid + q] = tt.field[slot][q];
            sdiv[3 * gid + q] = tt.div[slot][q];
        }
    } else {
        rcell[gid - nsrc] = cell;
    }
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

extern "C" int sfd_forward_noalloc(sfd_plan *p, const float *src_pos, const float *src, int nsrc,
                                   const float *rec_pos, int nrec, int mask, const int *outsel, float *seis,
                                   void *stream)
{
    if (!p) return SFD_ERR_ARG;
    if (!p->model_set) { p->err = "sfd_set_model must be called first"; return SFD_ERR_STATE; }
    if (p->g.fhalf || p->g.rhalf) {
        p->err = "sfd_forward_noalloc runs FP32 wave fields and memory variables only";
        return SFD_ERR_UNSUPPORTED;
    }
    if (nsrc < 0 || nrec < 0 || (nsrc && (!src_pos || !src)) || (nrec && !rec_pos)) {
        p->err = "invalid shot arrays";
        return SFD_ERR_ARG;
    }
    // one shot, whatever the plan's batch; a local copy leaves the plan's
    // state as it was
    Grid g = p->g;
    g.nb = 1;
    unsigned omask = 0;
    int nsel = 0;
    for (int o = 0; o < SFD_NOUT; o++) {
        if (!outsel || !outsel[o]) continue;
        bool ok = o == SFD_OUT_P ? g.nd != 21 : (p->f.w[o] != nullptr && !(g.nd == 22 && o == SFD_OUT_SXX));
        if (!ok) {
            p->err = "requested output variable does not exist in this physics";
            return SFD_ERR_ARG;
        }
        omask |= 1u << o;
        nsel++;
    }
    if (nsel && !seis) { p->err = "missing seismogram buffer"; return SFD_ERR_ARG; }

    // carve the scratch: the plan's own set of wave fields and memory
    // variables (which depends on the physics), CPML memory, maps
    int ids[NW], rids[NR], nwave = 0, nmem = 0;
    for (int w = 0; w < NW; w++)
        if (p->f.w[w]) ids[nwave++] = w;
    for (int r = 0; r < NR; r++)
        if (p->f.r[r]) rids[nmem++] = r;
    size_t need = 0;
    size_t off_w = need; need += align256(sizeof(float) * g.nvol * nwave);
    size_t off_r = need; need += align256(sizeof(float) * g.nvol * g.L * nmem);
    int64_t psi_total = 0;
    for (int i = 0; i < NPSI; i++) psi_total += psi_span(p->psi_size[i]);
    size_t off_psi = need; need += align256(sizeof(float) * psi_total);
    size_t off_map = need;
    need += align256(sizeof(int64_t) * (size_t)(nsrc + nrec)) + align256(sizeof(int) * 5 * (size_t)nsrc) +
            align256(sizeof(float) * 3 * (size_t)nsrc) + 256;
    if (need > (size_t)SFD_NOALLOC_SCRATCH_BYTES) {
        char buf[200];
        snprintf(buf, sizeof buf,
                 "shot needs %zu bytes of working memory; sfd_forward_noalloc holds at most %u (use sfd_forward)",
                 need, (unsigned)SFD_NOALLOC_SCRATCH_BYTES);
        p->err = buf;
        return SFD_ERR_MEMORY;
    }
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != p->device) {
        p->err = "make the plan's device current before sfd_forward_noalloc";
        return SFD_ERR_ARG;
    }
    void *base_v = nullptr;
    if (scratch_address(p->device, &base_v) != SFD_OK) {
        p->err = "cudaGetSymbolAddress failed for the no-allocation scratch";
        return SFD_ERR_CUDA;
    }
    unsigned char *base = (unsigned char *)base_v;
    cudaStream_t st = stream ? (cudaStream_t)stream : p->stream;

    Fields f = p->f;  // parameters, CPML constants and taper stay the plan's
    for (int w = 0; w < NW; w++) f.w[w] = nullptr;
    for (int q = 0; q < nwave; q++) f.w[ids[q]] = (float *)(base + off_w) + (int64_t)q * g.nvol;
    for (int r = 0; r < NR; r++) f.r[r] = nullptr;
    for (int q = 0; q < nmem; q++) f.r[rids[q]] = (float *)(base + off_r) + (int64_t)q * g.nvol * g.L;
    int64_t poff = 0;
    for (int i = 0; i < NPSI; i++) {
        f.psi[i] = p->psi_size[i] ? (float *)(base + off_psi) + poff : nullptr;
        poff += psi_span(p->psi_size[i]);
    }
    unsigned char *m = base + off_map;
    int64_t *scell = (int64_t *)m;
    int64_t *rcell = scell + nsrc;
    m += align256(sizeof(int64_t) * (size_t)(nsrc + nrec));
    int *snt = (int *)m, *skz = snt + nsrc, *sfield = skz + nsrc;
    m += align256(sizeof(int) * 5 * (size_t)nsrc);
    float *sdiv = (float *)m;
    m += align256(sizeof(float) * 3 * (size_t)nsrc);
    int *bad = (int *)m;

    TargetTable tt;
    memset(&tt, 0, sizeof tt);
    const int types[6] = {0, 1, 2, 3, 100, -1};
    for (int s = 0; s < 6; s++) tt.n[s] = source_targets(g.nd, mask, types[s], tt.field[s], tt.div[s]);

    // everything that must start at zero, every call: the array keeps the
    // previous call's contents
    cudaError_t e = cudaMemsetAsync(base, 0, off_map, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(bad, 0, sizeof(int), st);
    if (e == cudaSuccess && nsel && nrec)
        e = cudaMemsetAsync(seis, 0, sizeof(float) * (size_t)nsel * nrec * p->cfg.nt, st);
    if (e != cudaSuccess) { p->err = cudaGetErrorString(e); return SFD_ERR_CUDA; }
    if (nsrc + nrec > 0)
        k_noalloc_map<<<(nsrc + nrec + 127) / 128, 128, 0, st>>>(g, p->DH_lit, src_pos, nsrc, rec_pos, nrec, tt, scell,
                                                                 snt, sfield, sdiv, skz, rcell, bad);
    int hbad = 0;
    e = cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { p->err = cudaGetErrorString(e); return SFD_ERR_CUDA; }
    if (hbad) { p->err = "source or receiver position outside the padded grid"; return SFD_ERR_ARG; }

    PointSet S{nsrc, scell, snt, sfield, sdiv, skz};
    PointSet R{nrec, rcell, nullptr, nullptr, nullptr, nullptr};
    const int NT = p->cfg.nt;
    for (int t = 0; t < p->cfg.tmax; t++) {
        launch_sources(g, f, S, src, NT, t, 1, st);
        launch_update_v(g, f, st);
        launch_update_s(g, f, st);
        if (g.freesurf) launch_surface(g, f, 1, st);
        launch_record(g, f, R, seis, NT, t, omask, st);
    }
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { p->err = cudaGetErrorString(e); return SFD_ERR_CUDA; }
    // a TMA stage that gave up on its bounded wait leaves wrong seismograms
    // and raises the device status word; report it as sfd_forward does
    if (tma_take_status()) {
        p->err = "a TMA pipeline stage timed out (results invalid)";
        return SFD_ERR_CUDA;
    }
    return SFD_OK;
}
