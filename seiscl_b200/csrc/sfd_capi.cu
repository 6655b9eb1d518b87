// sfd_capi.cu -- the C ABI of the engine: plans, model upload, the forward
// and adjoint time loops (src/time_stepping.c:692-1012, single device).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "seiscl_b200.h"
#include "sfd_internal.h"
#include "sfd_kernels.h"
#include "sfd_setup.h"

using namespace sfd;

namespace {

int fail(sfd_plan *p, int code, const std::string &msg)
{
    if (p) p->err = msg;
    return code;
}

#define CKC(call)                                                                                     \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess)                                                                        \
            return fail(p, e_ == cudaErrorMemoryAllocation ? SFD_ERR_MEMORY : SFD_ERR_CUDA,           \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                           \
    } while (0)

// Device memory comes from the device's stream-ordered pool, ordered on the
// plan's stream: unlike cudaMalloc / cudaFree, allocating and freeing does
// not synchronize the device, so plans created and destroyed while others
// run (a serving process) leave the running ones alone.  The pool keeps
// freed memory for reuse (release threshold: unlimited).
void pool_setup(int dev)
{
    static std::atomic<uint64_t> done{0};
    if (dev < 0 || dev >= 64 || (done.load() >> dev) & 1) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    done.fetch_or(uint64_t(1) << dev);
}

// allocation owned by the caller (freed with dfree); tracked in dev_bytes
void *dalloc_raw(sfd_plan *p, size_t bytes, cudaError_t *err)
{
    void *ptr = nullptr;
    pool_setup(p->device);
    *err = cudaMallocAsync(&ptr, bytes ? bytes : 16, p->stream);
    if (*err == cudaSuccess) *err = cudaStreamSynchronize(p->stream);   // usable from any stream
    if (*err != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    p->dev_bytes += bytes;
    return ptr;
}

void dfree(sfd_plan *p, void *ptr, size_t bytes)
{
    if (!ptr) return;
    cudaFreeAsync(ptr, p->stream);
    p->dev_bytes -= bytes;
}

// allocation owned by the plan (freed with it)
void *dalloc(sfd_plan *p, size_t bytes, cudaError_t *err)
{
    void *ptr = dalloc_raw(p, bytes, err);
    if (ptr) p->allocs.push_back({ptr, bytes});
    return ptr;
}

bool is_wave_used(const Grid &g, int w)
{
    if (g.nd == 3) return true;
    if (g.nd == 21) return w == VY || w == SXY || w == SYZ;
    if (g.nd == 22) return w == VX || w == VZ || w == SXX;  // SXX holds the acoustic pressure
    return w == VX || w == VZ || w == SXX || w == SZZ || w == SXZ;
}
bool is_mem_used(const Grid &g, int r)
{
    if (g.L == 0) return false;
    if (g.nd == 3) return true;
    if (g.nd == 21) return r == RXY || r == RYZ;
    if (g.nd == 22) return r == RXX;
    return r == RXX || r == RZZ || r == RXZ;
}

unsigned outmask_of(const int *outsel, int nd, int *nsel)
{
    unsigned m = 0;
    int n = 0;
    for (int o = 0; o < SFD_NOUT; o++)
        if (outsel && outsel[o]) {
            m |= 1u << o;
            n++;
        }
    *nsel = n;
    return m;
}

int check_outsel(sfd_plan *p, const int *outsel)
{
    for (int o = 0; o < SFD_NOUT; o++) {
        if (!outsel || !outsel[o]) continue;
        if (o == SFD_OUT_P) {
            if (p->g.nd == 21) return fail(p, SFD_ERR_ARG, "Cannot output pressure for SH modeling");
            continue;
        }
        if (p->g.nd == 22 && o == SFD_OUT_SXX) return fail(p, SFD_ERR_ARG, "acoustic modeling records p, not sxx");
        if (!is_wave_used(p->g, o)) return fail(p, SFD_ERR_ARG, "requested output variable does not exist in this physics");
    }
    return SFD_OK;
}

// grow the per-shot device buffers
int ensure_shot_buffers(sfd_plan *p, int nsrc, int nrec, int nsel)
{
    cudaError_t e;
    if (nsrc > p->cap_src) {
        int cap = std::max(nsrc, 16);
        p->d_src_cell = (int64_t *)dalloc(p, sizeof(int64_t) * cap, &e); if (e) goto oom;
        p->d_src_nt = (int *)dalloc(p, sizeof(int) * cap, &e); if (e) goto oom;
        p->d_src_kz = (int *)dalloc(p, sizeof(int) * cap, &e); if (e) goto oom;
        p->d_src_field = (int *)dalloc(p, sizeof(int) * 3 * cap, &e); if (e) goto oom;
        p->d_src_div = (float *)dalloc(p, sizeof(float) * 3 * cap, &e); if (e) goto oom;
        p->d_src = (float *)dalloc(p, sizeof(float) * (size_t)cap * p->cfg.nt, &e); if (e) goto oom;
        p->cap_src = cap;
    }
    if ((int64_t)nrec * std::max(nsel, 1) > p->cap_rec) {
        int64_t cap = std::max<int64_t>((int64_t)nrec * std::max(nsel, 1), 16);
        p->d_rec_cell = (int64_t *)dalloc(p, sizeof(int64_t) * cap, &e); if (e) goto oom;
        p->d_seis = (float *)dalloc(p, sizeof(float) * (size_t)cap * p->cfg.nt, &e); if (e) goto oom;
        p->d_res = (float *)dalloc(p, sizeof(float) * (size_t)cap * p->cfg.nt, &e); if (e) goto oom;
        p->cap_rec = (int)cap;
    }
    return SFD_OK;
oom:
    return fail(p, SFD_ERR_MEMORY, std::string("device allocation failed: ") + cudaGetErrorString(e));
}

// host-side mapping of a shot's sources and receivers, uploaded to the device
int upload_shots(sfd_plan *p, int nshot, const sfd_shot *shots, int mask, PointSet &S, PointSet &R,
                 cudaStream_t st)
{
    const Grid &g = p->g;
    const int F = g.F, NT = p->cfg.nt;
    int nsrc = 0, nrec = 0;
    for (int b = 0; b < nshot; b++) { nsrc += shots[b].nsrc; nrec += shots[b].nrec; }
    std::vector<int64_t> scell(nsrc), rcell(nrec);
    std::vector<int> snt(nsrc), sfield(3 * nsrc), skz(nsrc);
    std::vector<float> sdiv(3 * nsrc), ssig((size_t)nsrc * NT);
    int s = 0, r = 0;
    for (int b = 0; b < nshot; b++) {
        const sfd_shot *shot = &shots[b];
        // shot b's points address copy b of the wave fields
        const int64_t base = (int64_t)b * g.nvol;
        for (int q = 0; q < shot->nsrc; q++, s++) {
            int i, j, k;
            point_cell(shot->src_pos + 5 * q, p->DH_lit, F, i, j, k);
            if (g.nd != 3) j = 0;  // 2D kernels index [(i)*NZ+k] (automatic_kernels.c:536-543)
            std::memcpy(&ssig[(size_t)s * NT], shot->src + (size_t)q * NT, sizeof(float) * NT);
            // sources outside [F, NX-F-1] along x are dropped (automatic_kernels.c:506-511)
            if (i < F || i > g.NX - F - 1) { scell[s] = -1; snt[s] = 0; continue; }
            if (j < 0 || j >= g.NY || k < 0 || k >= g.NZ)
                return fail(p, SFD_ERR_ARG, "source position outside the padded grid");
            scell[s] = base + ((int64_t)i * g.NY + j) * g.NZ + k;
            skz[s] = k;
            int type = (int)shot->src_pos[5 * q + 4];
            snt[s] = source_targets(g.nd, mask, type, &sfield[3 * s], &sdiv[3 * s]);
        }
        for (int q = 0; q < shot->nrec; q++, r++) {
            int i, j, k;
            point_cell(shot->rec_pos + 8 * q, p->DH_lit, F, i, j, k);
            if (g.nd != 3) j = 0;
            if (i < F || i > g.NX - F - 1) { rcell[r] = -1; continue; }
            if (j < 0 || j >= g.NY || k < 0 || k >= g.NZ)
                return fail(p, SFD_ERR_ARG, "receiver position outside the padded grid");
            rcell[r] = base + ((int64_t)i * g.NY + j) * g.NZ + k;
        }
    }
    {
        if (nsrc) {
            CKC(cudaMemcpyAsync(p->d_src_cell, scell.data(), sizeof(int64_t) * nsrc, cudaMemcpyHostToDevice, st));
            CKC(cudaMemcpyAsync(p->d_src_nt, snt.data(), sizeof(int) * nsrc, cudaMemcpyHostToDevice, st));
            CKC(cudaMemcpyAsync(p->d_src_kz, skz.data(), sizeof(int) * nsrc, cudaMemcpyHostToDevice, st));
            CKC(cudaMemcpyAsync(p->d_src_field, sfield.data(), sizeof(int) * 3 * nsrc, cudaMemcpyHostToDevice, st));
            CKC(cudaMemcpyAsync(p->d_src_div, sdiv.data(), sizeof(float) * 3 * nsrc, cudaMemcpyHostToDevice, st));
            CKC(cudaMemcpyAsync(p->d_src, ssig.data(), sizeof(float) * ssig.size(), cudaMemcpyHostToDevice, st));
        }
        if (nrec) CKC(cudaMemcpyAsync(p->d_rec_cell, rcell.data(), sizeof(int64_t) * nrec, cudaMemcpyHostToDevice, st));
        // pageable sources: wait so the host vectors may go out of scope
        CKC(cudaStreamSynchronize(st));
    }
    S = PointSet{nsrc, p->d_src_cell, p->d_src_nt, p->d_src_field, p->d_src_div, p->d_src_kz};
    R = PointSet{nrec, p->d_rec_cell, nullptr, nullptr, nullptr, nullptr};
    return SFD_OK;
}

int upload_shot(sfd_plan *p, const sfd_shot *shot, int mask, PointSet &S, PointSet &R, cudaStream_t st)
{
    return upload_shots(p, 1, shot, mask, S, R, st);
}

// bytes per stored wave-field / memory-variable value
size_t wave_elem(const Grid &g) { return g.fhalf ? 2 : sizeof(float); }
size_t mem_elem(const Grid &g) { return g.fhalf || g.rhalf ? 2 : sizeof(float); }

// CPML memory arrays of a grid (0: unused); returns the floats of their
// 256-byte aligned spans
int64_t psi_sizes(const Grid &g, int64_t size[NPSI])
{
    int64_t nab2 = 2 * (int64_t)g.nab;
    int64_t sx = nab2 * g.ny * g.nz, sy = (int64_t)g.nx * nab2 * g.nz, sz = (int64_t)g.nx * g.ny * nab2;
    int64_t sizes[NPSI] = {sx, sx, sx, sy, sy, sy, sz, sz, sz, sx, sx, sx, sy, sy, sy, sz, sz, sz};
    int64_t tot = 0;
    for (int i = 0; i < NPSI; i++) {
        bool used2 = i == PVX_X || i == PVZ_X || i == PVX_Z || i == PVZ_Z || i == PSXX_X || i == PSXZ_X ||
                     i == PSXZ_Z || i == PSZZ_Z;
        bool used21 = i == PSXY_X || i == PSYZ_Z || i == PVY_X || i == PVY_Z;
        bool used22 = i == PVX_X || i == PVZ_Z || i == PSXX_X || i == PSZZ_Z;  // + psi_p_x / psi_p_z
        bool used = g.abs_type == 1 && g.nab > 0 &&
                    (g.nd == 3 || (g.nd == 2 && used2) || (g.nd == 21 && used21) || (g.nd == 22 && used22));
        size[i] = used ? sizes[i] : 0;
        tot += psi_span(size[i]);
    }
    return tot;
}

int alloc_model(sfd_plan *p)
{
    const Grid &g = p->g;
    cudaError_t e;
    for (int w = 0; w < NW; w++) {
        p->f.w[w] = nullptr;
        if (!is_wave_used(g, w)) continue;
        p->f.w[w] = (float *)dalloc(p, wave_elem(g) * g.nvol * p->batch, &e);
        if (e) return fail(p, SFD_ERR_MEMORY, "wave field allocation failed");
    }
    for (int r = 0; r < NR; r++) {
        p->f.r[r] = nullptr;
        if (!is_mem_used(g, r)) continue;
        p->f.r[r] = (float *)dalloc(p, mem_elem(g) * g.nvol * g.L * p->batch, &e);
        if (e) return fail(p, SFD_ERR_MEMORY, "memory-variable allocation failed");
    }
    int64_t tot = psi_sizes(g, p->psi_size);
    p->d_psi_all = tot ? (float *)dalloc(p, sizeof(float) * tot * p->batch, &e) : nullptr;
    if (tot && e) return fail(p, SFD_ERR_MEMORY, "CPML allocation failed");
    int64_t off = 0;
    for (int i = 0; i < NPSI; i++) {
        p->f.psi[i] = p->psi_size[i] ? p->d_psi_all + off : nullptr;
        off += psi_span(p->psi_size[i]);
    }
    int64_t npar = (int64_t)g.nz * g.ny * g.nx;
    for (int k = 0; k < NPAR; k++) {
        p->f.p[k] = (const float *)dalloc(p, sizeof(float) * npar, &e);
        if (e) return fail(p, SFD_ERR_MEMORY, "parameter allocation failed");
    }
    int nc = std::max(2 * g.nab, 1);
    float *cst = (float *)dalloc(p, sizeof(float) * (3 * NC * nc + nc + 6 * nc), &e);
    if (e) return fail(p, SFD_ERR_MEMORY, "constant allocation failed");
    for (int k = 0; k < NC; k++) {
        p->f.cx[k] = cst + (0 * NC + k) * nc;
        p->f.cy[k] = cst + (1 * NC + k) * nc;
        p->f.cz[k] = cst + (2 * NC + k) * nc;
    }
    p->f.taper = cst + 3 * NC * nc;
    // block counter of the fused steps, instability flag
    p->d_ticket = (int *)dalloc(p, 2 * sizeof(int), &e);
    if (e) return fail(p, SFD_ERR_MEMORY, "step counter allocation failed");
    p->d_unstable = p->d_ticket + 1;
    // fused 3D step: ticket counter and per-unit flags (single-shot plans)
    const FusedShape fsh = fused_shape(g);
    p->d_fsync = nullptr;
    if (p->batch == 1 && fsh.units) {
        p->d_fsync = (int *)dalloc(p, sizeof(int) * (size_t)(1 + fsh.units), &e);
        if (e) return fail(p, SFD_ERR_MEMORY, "fused-step flag allocation failed");
    }
    for (int ax = 0; ax < 3; ax++)
        for (int h = 0; h < 2; h++) p->f.kinv[ax][h] = cst + 3 * NC * nc + nc + (2 * ax + h) * nc;
    return SFD_OK;
}

int upload_constants(sfd_plan *p)
{
    const Grid &g = p->g;
    const sfd_config &c = p->cfg;
    int nc = std::max(2 * g.nab, 1);
    std::vector<float> h(3 * NC * nc + nc + 6 * nc, 0.0f);
    if (g.abs_type == 1 && g.nab > 0) {
        for (int ax = 0; ax < 3; ax++) {
            float *b = h.data() + ax * NC * nc;
            if (!cpml_profiles(c.npower, c.k_max_cpml, c.fpml, c.vppml, c.dh, c.dt, g.nab, b + CK * nc, b + CA * nc,
                               b + CB * nc, b + CKH * nc, b + CAH * nc, b + CBH * nc))
                return fail(p, SFD_ERR_ARG, "invalid CPML parameters");
        }
    }
    if (g.abs_type == 2) cerjan_taper(c.abpc, g.nab, h.data() + 3 * NC * nc);
    // reciprocals of K and K_half for kernels that multiply instead of divide
    for (int ax = 0; ax < 3; ax++)
        for (int hh = 0; hh < 2; hh++) {
            const float *K = h.data() + ax * NC * nc + (hh ? CKH : CK) * nc;
            float *ki = h.data() + 3 * NC * nc + nc + (2 * ax + hh) * nc;
            for (int i = 0; i < nc; i++) ki[i] = K[i] != 0.0f ? 1.0f / K[i] : 0.0f;
        }
    CKC(cudaMemcpy((void *)p->f.cx[0], h.data(), sizeof(float) * h.size(), cudaMemcpyHostToDevice));
    return SFD_OK;
}

int zero_forward_state(sfd_plan *p, cudaStream_t st)
{
    const Grid &g = p->g;
    const size_t nb = (size_t)g.nb;   // the shots of this run
    for (int w = 0; w < NW; w++)
        if (p->f.w[w]) CKC(cudaMemsetAsync(p->f.w[w], 0, wave_elem(g) * g.nvol * nb, st));
    for (int r = 0; r < NR; r++)
        if (p->f.r[r]) CKC(cudaMemsetAsync(p->f.r[r], 0, mem_elem(g) * g.nvol * g.L * nb, st));
    int64_t tot = 0;
    for (int i = 0; i < NPSI; i++) tot += psi_span(p->psi_size[i]);
    if (tot) CKC(cudaMemsetAsync(p->d_psi_all, 0, sizeof(float) * tot * nb, st));
    return SFD_OK;
}

int alloc_adjoint(sfd_plan *p)
{
    const Grid &g = p->g;
    cudaError_t e;
    if (p->a.grad[0]) return SFD_OK;
    // the DFT adjoint runs in the forward buffers (no separate adjoint fields)
    const bool bp2 = p->cfg.back_prop_type == 2;
    for (int w = 0; w < NW; w++) {
        p->a.wr[w] = nullptr;
        if (bp2 || !is_wave_used(g, w)) continue;
        p->a.wr[w] = (float *)dalloc(p, sizeof(float) * g.nvol * p->batch, &e);
        if (e) return fail(p, SFD_ERR_MEMORY, "adjoint field allocation failed");
    }
    for (int r = 0; r < NR; r++) {
        p->a.rr[r] = nullptr;
        if (bp2 || !is_mem_used(g, r)) continue;
        p->a.rr[r] = (float *)dalloc(p, sizeof(float) * g.nvol * g.L * p->batch, &e);
        if (e) return fail(p, SFD_ERR_MEMORY, "adjoint memory-variable allocation failed");
    }
    int64_t npar = (int64_t)g.nz * g.ny * g.nx;
    for (int k = 0; k < NG; k++) {
        p->a.hess[k] = nullptr;
        if (!g.hout) continue;
        p->a.hess[k] = (double *)dalloc(p, sizeof(double) * npar * p->batch, &e);
        if (e) return fail(p, SFD_ERR_MEMORY, "Hessian allocation failed");
        CKC(cudaMemsetAsync(p->a.hess[k], 0, sizeof(double) * npar * p->batch, p->stream));
    }
    for (int k = 0; k < NG; k++) {
        p->a.grad[k] = nullptr;
        if ((k == GTAUP || k == GTAUS) && !(bp2 && g.L > 0)) continue;
        p->a.grad[k] = (double *)dalloc(p, sizeof(double) * npar * p->batch, &e);
        if (e) return fail(p, SFD_ERR_MEMORY, "gradient allocation failed");
        CKC(cudaMemsetAsync(p->a.grad[k], 0, sizeof(double) * npar * p->batch, p->stream));
    }
    int64_t nq = (int64_t)g.nx * g.ny;
    p->d_surf_q = (float *)dalloc(p, sizeof(float) * nq * p->batch, &e);
    if (e) return fail(p, SFD_ERR_MEMORY, "scratch allocation failed");
    return SFD_OK;
}

// ----------------------------------------------------------------- movie
// The movie films the call's selected wave fields (the reference films its
// output variables, time_stepping.c:284-292): output index -> wave field.
struct Movie {
    int n = 0;
    int out[SFD_NOUT];     // SFD_OUT_* index of each filmed variable
    int wave[SFD_NOUT];    // its wave field
    int nslot = 0;
    int64_t ncell = 0;
};

int movie_setup(sfd_plan *p, unsigned omask, Movie &mv)
{
    const Grid &g = p->g;
    mv.n = 0;
    if (p->movout <= 0) return SFD_OK;
    for (int o = 0; o < SFD_NOUT; o++) {
        if (!(omask & (1u << o)) || !p->mov_dst[o]) continue;
        int w = o;
        if (o == SFD_OUT_P) {
            if (g.nd != 22) continue;   // pressure is a wave field only in the acoustic model
            w = SXX;
        }
        if (!p->f.w[w]) continue;
        mv.out[mv.n] = o;
        mv.wave[mv.n] = w;
        mv.n++;
    }
    mv.nslot = p->cfg.nt / p->movout;
    mv.ncell = (int64_t)g.nz * g.ny * g.nx;
    if (!mv.n || !mv.nslot) { mv.n = 0; return SFD_OK; }
    size_t need = (size_t)mv.n * mv.nslot * mv.ncell;
    if (need > p->mov_cap) {
        dfree(p, p->d_mov, sizeof(float) * p->mov_cap);
        p->d_mov = nullptr;
        p->mov_cap = 0;
        cudaError_t e;
        p->d_mov = (float *)dalloc_raw(p, sizeof(float) * need, &e);
        if (!p->d_mov) return fail(p, SFD_ERR_MEMORY, "movie buffer does not fit in device memory");
        p->mov_cap = need;
    }
    CKC(cudaMemsetAsync(p->d_mov, 0, sizeof(float) * need, p->stream));
    CKC(cudaStreamSynchronize(p->stream));
    return SFD_OK;
}

void movie_snap(const sfd_plan *p, const Movie &mv, int slot, cudaStream_t st)
{
    for (int q = 0; q < mv.n; q++)
        launch_movie(p->g, p->f.w[mv.wave[q]], 1.0f / p->g.ws.w[mv.wave[q]],
                     p->d_mov + ((size_t)q * mv.nslot + slot) * mv.ncell, st);
}

int movie_out(sfd_plan *p, const Movie &mv, cudaStream_t st)
{
    for (int q = 0; q < mv.n; q++)
        CKC(cudaMemcpyAsync(p->mov_dst[mv.out[q]], p->d_mov + (size_t)q * mv.nslot * mv.ncell,
                            sizeof(float) * (size_t)mv.nslot * mv.ncell, cudaMemcpyDeviceToHost, st));
    return SFD_OK;
}

// ------------------------------------------------- instability detection
// Every FINITE_CHECK_EVERY steps (and after the last) a loop scans one
// velocity field of its shots for non-finite values; the first step at which
// one is seen is kept in p->d_unstable and turned into SFD_ERR_UNSTABLE when
// the loop has finished (the reference aborts on a NaN misfit,
// src/residuals.c:444-448).
const float *check_field(float *const *w)
{
    for (int q : {VX, VY, VZ})
        if (w[q]) return w[q];
    return nullptr;
}

int arm_unstable(sfd_plan *p, cudaStream_t st)
{
    CKC(cudaMemsetAsync(p->d_unstable, 0x7f, sizeof(int), st));
    return SFD_OK;
}

// call after the loop's stream has been synchronised
int take_unstable(sfd_plan *p, cudaStream_t st, const char *what)
{
    int v = 0;
    CKC(cudaMemcpyAsync(&v, p->d_unstable, sizeof(int), cudaMemcpyDeviceToHost, st));
    CKC(cudaStreamSynchronize(st));
    if (v == 0x7f7f7f7f) return SFD_OK;
    char buf[200];
    snprintf(buf, sizeof buf, "Simulation has become unstable: non-finite %s wave field at step %d", what, v);
    return fail(p, SFD_ERR_UNSTABLE, buf);
}

// ----------------------------------------------------------- loop graphs
// The bytes a time loop's launches bake in: kernel arguments by value and
// the buffers they point to.  Equal keys => the captured graph is valid.
struct LoopKey {
    std::string s;
    template <class T>
    void add(const T &v) { s.append(reinterpret_cast<const char *>(&v), sizeof v); }
    void add_points(const PointSet &q)
    {
        add(q.n); add(q.cell); add(q.ntarget); add(q.field); add(q.div); add(q.kz);
    }
};

bool graphs_on(const sfd_plan *p)
{
    const int m = p->cfg.loop_graphs;
    if (m == 2) return false;
    if (m == 1) return p->g.kernels != 3;   // the TMA path sets kernel attributes on first use
    return p->g.nd != 3 || (p->g.kernels != 3 && p->g.kernels != 2);
}

void drop_graph(sfd_plan::LoopGraph &lg)
{
    if (lg.exec) cudaGraphExecDestroy(lg.exec);
    lg.exec = nullptr;
    lg.key.clear();
}

// Run a time loop: its launches go to `st` directly, or -- when graphs are
// on -- through a graph captured from them and cached under `key`.
template <class Body>
int run_loop(sfd_plan *p, sfd_plan::LoopGraph &lg, const std::string &key, cudaStream_t st, Body body)
{
    if (!graphs_on(p)) {
        body(st);
        return SFD_OK;
    }
    if (!lg.exec || lg.key != key) {
        drop_graph(lg);
        // auto mode captures a loop the second time it runs unchanged: a plan
        // that runs one shot of a shape would only pay for the capture
        if (p->cfg.loop_graphs == 0 && lg.seen != key) {
            lg.seen = key;
            body(st);
            return SFD_OK;
        }
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            body(st);
            if (cudaStreamEndCapture(st, &graph) == cudaSuccess && graph) {
                if (cudaGraphInstantiate(&lg.exec, graph, 0) != cudaSuccess) lg.exec = nullptr;
                cudaGraphDestroy(graph);
            }
        }
        cudaGetLastError();
        if (!lg.exec) {   // capture not possible here: run the launches directly
            body(st);
            return SFD_OK;
        }
        lg.key = key;
    }
    CKC(cudaGraphLaunch(lg.exec, st));
    return SFD_OK;
}

// --------------------------------------------------- checkpointed gradients
// A snapshot holds the wave fields and memory variables in the store type of
// `precision` (FP16 with the power-of-two scales of the saved boundaries)
// and the CPML memory in FP32, in that order; the segment store holds the
// wave fields of each step of a K-step segment.
struct CkptSizes {
    int nwave, nmem, K, nseg;
    int64_t psi;            // CPML floats
    size_t elem, selem, snap, seg;   // bytes per stored value: segment store, snapshot fields
};
// FP16 wave-field storage: log2 of the factor a parameter carries (the
// moduli 2^-kshift, the buoyancies 2^kshift, the rest 1)
int param_exponent(int k, int kshift)
{
    if (k == PRIP || k == PRJP || k == PRKP) return kshift;
    if (k == PM || k == PMU || k == PMUIPKP || k == PMUIPJP || k == PMUJPKP) return -kshift;
    return 0;
}

CkptSizes ckpt_sizes(const Grid &g, const sfd_config &c)
{
    CkptSizes z;
    z.nwave = z.nmem = 0;
    for (int w = 0; w < NW; w++) z.nwave += is_wave_used(g, w);
    for (int r = 0; r < NR; r++) z.nmem += is_mem_used(g, r);
    int64_t psz[NPSI];
    z.psi = psi_sizes(g, psz);
    const int tmax = (c.tmax > 0 && c.tmax <= c.nt) ? c.tmax : c.nt;
    z.K = std::max(1, std::min(c.checkpoint, tmax));
    z.nseg = (tmax + z.K - 1) / z.K;
    z.elem = c.precision == SFD_PREC_FP32 ? 4 : 2;
    // FP16 wave-field storage: the snapshots copy the FP16 fields unchanged
    z.selem = g.fhalf ? 2 : z.elem;
    z.snap = z.selem * g.nvol * (z.nwave + (size_t)z.nmem * g.L) + sizeof(float) * z.psi;
    z.seg = z.elem * g.nvol * z.nwave * (size_t)z.K;
    return z;
}

int alloc_ckpt(sfd_plan *p)
{
    const CkptSizes z = ckpt_sizes(p->g, p->cfg);
    if (p->d_snap) return SFD_OK;
    cudaError_t e;
    p->d_snap = (char *)dalloc(p, z.snap * z.nseg, &e);
    if (!p->d_snap) return fail(p, SFD_ERR_MEMORY, "checkpoint snapshots do not fit in device memory");
    p->d_seg = (char *)dalloc(p, z.seg, &e);
    if (!p->d_seg) return fail(p, SFD_ERR_MEMORY, "checkpoint segment store does not fit in device memory");
    p->d_psi_adj = (float *)dalloc(p, sizeof(float) * std::max<int64_t>(z.psi, 1), &e);
    if (!p->d_psi_adj) return fail(p, SFD_ERR_MEMORY, "adjoint CPML allocation failed");
    p->snap_bytes = z.snap;
    p->seg_bytes = z.seg;
    p->nseg = z.nseg;
    return SFD_OK;
}

// FP16 wave-field storage: the unscaled parameters of the adjoint, uploaded
// once per model
int prepare_adjoint_params(sfd_plan *p)
{
    for (int k = 0; k < NPAR; k++) p->padj[k] = p->f.p[k];
    if (!p->g.fhalf) return SFD_OK;
    const Grid &g = p->g;
    const int64_t npar = (int64_t)g.nz * g.ny * g.nx;
    int nscaled = 0;
    for (int k = 0; k < NPAR; k++) nscaled += p->f.p[k] && param_exponent(k, 1) != 0;
    cudaError_t e;
    if (!p->d_padj) {
        p->d_padj = (float *)dalloc(p, sizeof(float) * npar * nscaled, &e);
        if (!p->d_padj) return fail(p, SFD_ERR_MEMORY, "unscaled adjoint parameters do not fit in device memory");
    }
    int q = 0;
    for (int k = 0; k < NPAR; k++) {
        if (!p->f.p[k] || param_exponent(k, 1) == 0) continue;
        float *dst = p->d_padj + npar * q++;
        if (!p->padj_valid)
            CKC(cudaMemcpy(dst, p->hp[k].data(), sizeof(float) * npar, cudaMemcpyHostToDevice));
        p->padj[k] = dst;
    }
    p->padj_valid = true;
    return SFD_OK;
}

// wave fields (and memory variables) <-> snapshot j
void ckpt_snapshot(sfd_plan *p, int j, bool load, cudaStream_t st)
{
    const Grid &g = p->g;
    const CkptSizes z = ckpt_sizes(g, p->cfg);
    char *base = p->d_snap + (size_t)j * p->snap_bytes;
    PackSet ps;
    memset(&ps, 0, sizeof ps);
    size_t off = 0;
    // FP16 wave-field storage: the fields are copied as they are (exact)
    auto copy = [&](void *field, size_t bytes) {
        if (load) cudaMemcpyAsync(field, base + off, bytes, cudaMemcpyDeviceToDevice, st);
        else cudaMemcpyAsync(base + off, field, bytes, cudaMemcpyDeviceToDevice, st);
        off += bytes;
    };
    for (int w = 0; w < NW; w++) {
        if (!p->f.w[w]) continue;
        if (g.fhalf) { copy(p->f.w[w], z.selem * g.nvol); continue; }
        ps.src[ps.narr] = load ? (const void *)(base + off) : (const void *)p->f.w[w];
        ps.dst[ps.narr] = load ? (void *)p->f.w[w] : (void *)(base + off);
        ps.n[ps.narr] = g.nvol;
        ps.scale[ps.narr] = load ? g.bsci[w] : g.bsc[w];
        ps.narr++;
        off += z.elem * g.nvol;
    }
    for (int r = 0; r < NR; r++) {   // memory variables: the scale of the stresses
        if (!p->f.r[r]) continue;
        if (g.fhalf) { copy(p->f.r[r], z.selem * g.nvol * g.L); continue; }
        ps.src[ps.narr] = load ? (const void *)(base + off) : (const void *)p->f.r[r];
        ps.dst[ps.narr] = load ? (void *)p->f.r[r] : (void *)(base + off);
        ps.n[ps.narr] = g.nvol * g.L;
        ps.scale[ps.narr] = load ? g.bsci[SXX] : g.bsc[SXX];
        ps.narr++;
        off += z.elem * g.nvol * g.L;
    }
    launch_pack(ps, p->cfg.precision, load, st);
    if (z.psi) {
        float *sp = (float *)(base + off);
        if (load) cudaMemcpyAsync(p->d_psi_all, sp, sizeof(float) * z.psi, cudaMemcpyDeviceToDevice, st);
        else cudaMemcpyAsync(sp, p->d_psi_all, sizeof(float) * z.psi, cudaMemcpyDeviceToDevice, st);
    }
}

// the wave fields now -> slot k of the segment store; the stored fields of
// slot k as the adjoint kernels read them
void ckpt_store(sfd_plan *p, int k, cudaStream_t st)
{
    const Grid &g = p->g;
    const CkptSizes z = ckpt_sizes(g, p->cfg);
    PackSet ps;
    memset(&ps, 0, sizeof ps);
    char *base = p->d_seg + (size_t)k * z.elem * g.nvol * z.nwave;
    for (int w = 0; w < NW; w++) {
        if (!p->f.w[w]) continue;
        ps.src[ps.narr] = p->f.w[w];
        ps.dst[ps.narr] = base + z.elem * g.nvol * ps.narr;
        ps.n[ps.narr] = g.nvol;
        // FP16 wave fields carry 2^a or 2^b: taken off before the store's own scale
        ps.scale[ps.narr] = g.fhalf ? g.bsc[w] / g.ws.w[w] : g.bsc[w];
        ps.narr++;
    }
    launch_pack(ps, p->cfg.precision, false, st, g.fhalf);
}
void ckpt_slot(const sfd_plan *p, int k, AdjFields &a)
{
    const Grid &g = p->g;
    const CkptSizes z = ckpt_sizes(g, p->cfg);
    const char *base = p->d_seg + (size_t)k * z.elem * g.nvol * z.nwave;
    int q = 0;
    for (int w = 0; w < NW; w++) {
        a.fwd[w] = nullptr;
        if (!p->f.w[w]) continue;
        a.fwd[w] = base + z.elem * g.nvol * q++;
    }
}

// The checkpointed adjoint: per K-step segment, from the last one, the
// forward run recomputed from the segment's snapshot (storing the wave
// fields of each step after its sources, before update_v: the fields that
// backpropagation would have reconstructed), then the adjoint steps of the
// segment, the same launches as the boundary-saving adjoint minus the
// reconstruction, injection and source removal.
int adjoint_ckpt(sfd_plan *p, const PointSet &S, const PointSet &R, unsigned omask, cudaStream_t st)
{
    const Grid &g = p->g;
    const CkptSizes z = ckpt_sizes(g, p->cfg);
    const int NT = p->cfg.nt, tmax = p->cfg.tmax, tmin = p->cfg.tmin;
    // the adjoint's CPML memory: the forward run's (the reference binds the
    // same buffers, src/clprogram.c:806-811) or zero
    if (z.psi) {
        if (p->cfg.adjoint_reset_psi) {
            CKC(cudaMemsetAsync(p->d_psi_adj, 0, sizeof(float) * z.psi, st));
        } else if (g.fhalf) {
            // the forward CPML memory is in the units of the FP16 fields:
            // psi of velocity derivatives carries 2^b, of stress derivatives 2^a
            PackSet ps;
            memset(&ps, 0, sizeof ps);
            for (int i = 0; i < NPSI; i++) {
                if (!p->f.psi[i] || !p->psi_size[i]) continue;
                ps.src[ps.narr] = p->f.psi[i];
                ps.dst[ps.narr] = p->d_psi_adj + (p->f.psi[i] - p->d_psi_all);
                ps.n[ps.narr] = p->psi_size[i];
                ps.scale[ps.narr] = 1.0f / g.ws.w[i < PSXX_X ? VX : SXX];
                if (++ps.narr == PackSet::MAXARR) { launch_pack(ps, SFD_PREC_FP32, false, st); ps.narr = 0; }
            }
            launch_pack(ps, SFD_PREC_FP32, false, st);
        } else {
            CKC(cudaMemcpyAsync(p->d_psi_adj, p->d_psi_all, sizeof(float) * z.psi, cudaMemcpyDeviceToDevice, st));
        }
    }
    Fields fa = p->f;
    for (int i = 0; i < NPSI; i++)
        fa.psi[i] = p->f.psi[i] ? p->d_psi_adj + (p->f.psi[i] - p->d_psi_all) : nullptr;
    int rc;
    if ((rc = prepare_adjoint_params(p))) return rc;
    for (int k = 0; k < NPAR; k++) fa.p[k] = p->padj[k];
    Grid ga = g;
    ga.ckpt = 1;
    ga.fhalf = false;   // the adjoint fields are FP32
    AdjFields a = p->a;
    for (int w = 0; w < NW; w++) a.bnd[w] = nullptr;
    LoopKey key;
    key.add(4); key.add(ga); key.add(p->f); key.add(fa); key.add(a); key.add_points(S); key.add_points(R);
    key.add(p->d_src); key.add(p->d_res); key.add(p->d_surf_q); key.add(omask); key.add(p->d_snap); key.add(p->d_seg);
    key.add(p->cfg.precision); key.add(tmax); key.add(tmin); key.add(z.K);
    const float *chk = check_field(a.wr);
    const int64_t nchk = g.nvol * g.nb;
    if ((rc = arm_unstable(p, st))) return rc;
    CKC(cudaEventRecord(p->ev0, st));
    int rcl = run_loop(p, p->gadj, key.s, st, [&](cudaStream_t s) {
        for (int j = z.nseg - 1; j >= 0; j--) {
            const int t0 = j * z.K, thi = std::min(t0 + z.K, tmax) - 1, tlo = std::max(t0, tmin + 1);
            if (thi < tlo) continue;
            ckpt_snapshot(p, j, true, s);
            for (int t = t0; t <= thi; t++) {
                launch_sources(g, p->f, S, p->d_src, NT, t, 1, s);
                ckpt_store(p, t - t0, s);
                if (t == thi) break;
                launch_update_v(g, p->f, s);
                launch_update_s(g, p->f, s);
                if (g.freesurf) launch_surface(g, p->f, 1, s);
            }
            for (int t = thi; t >= tlo; t--) {
                ckpt_slot(p, t - t0, a);
                if (g.freesurf) launch_surface_adj(ga, fa, a, p->d_surf_q, s);
                launch_residuals(ga, a, R, p->d_res, NT, t, omask, s);
                launch_update_adj(ga, fa, a, true, p->cfg.precision, s);
                launch_update_adj(ga, fa, a, false, p->cfg.precision, s);
                if (t % FINITE_CHECK_EVERY == 0 || t == tmin + 1)
                    launch_finite_check(ga, chk, nchk, t, p->d_unstable, s);
            }
        }
    });
    if (rcl) return rcl;
    CKC(cudaEventRecord(p->ev1, st));
    CKC(cudaGetLastError());
    CKC(cudaStreamSynchronize(st));
    cudaEventElapsedTime(&p->last_ms, p->ev0, p->ev1);
    p->have_forward = false;
    return take_unstable(p, st, "adjoint");
}

// ---------------------------------------------------------- DFT gradient
constexpr double PI_D = 3.141592653589793238462643383279502884197169;

void free_dft(sfd_plan *p)
{
    const size_t nf = (size_t)p->dft_nf;
    for (int s = 0; s < 2; s++) {
        for (int w = 0; w < NW; w++) {
            dfree(p, p->d_fw[s][w], sizeof(float2) * nf * p->g.nvol);
            p->d_fw[s][w] = nullptr;
        }
        for (int r = 0; r < NR; r++) {
            dfree(p, p->d_fr[s][r], sizeof(float2) * nf * p->g.nvol * p->g.L);
            p->d_fr[s][r] = nullptr;
        }
    }
    p->dft_nf = 0;
    p->have_dft = false;
}

// transforms of every wave field and memory variable, forward and adjoint
int alloc_dft(sfd_plan *p)
{
    const Grid &g = p->g;
    if (p->dft_nf == p->nfreqs) return SFD_OK;
    free_dft(p);
    const size_t nf = (size_t)p->nfreqs;
    p->dft_nf = p->nfreqs;   // the size free_dft releases
    cudaError_t e;
    for (int s = 0; s < 2; s++) {
        for (int w = 0; w < NW; w++) {
            if (!is_wave_used(g, w)) continue;
            p->d_fw[s][w] = (float2 *)dalloc_raw(p, sizeof(float2) * nf * g.nvol, &e);
            if (!p->d_fw[s][w]) {
                free_dft(p);
                return fail(p, SFD_ERR_MEMORY, "DFT gradient buffers do not fit in device memory");
            }
        }
        for (int r = 0; r < NR; r++) {
            if (!is_mem_used(g, r)) continue;
            p->d_fr[s][r] = (float2 *)dalloc_raw(p, sizeof(float2) * nf * g.nvol * g.L, &e);
            if (!p->d_fr[s][r]) {
                free_dft(p);
                return fail(p, SFD_ERR_MEMORY, "DFT gradient buffers do not fit in device memory");
            }
        }
    }
    return SFD_OK;
}

int zero_dft(sfd_plan *p, int slot, cudaStream_t st)
{
    const Grid &g = p->g;
    for (int w = 0; w < NW; w++)
        if (p->d_fw[slot][w]) CKC(cudaMemsetAsync(p->d_fw[slot][w], 0, sizeof(float2) * p->nfreqs * g.nvol, st));
    for (int r = 0; r < NR; r++)
        if (p->d_fr[slot][r])
            CKC(cudaMemsetAsync(p->d_fr[slot][r], 0, sizeof(float2) * p->nfreqs * g.nvol * g.L, st));
    return SFD_OK;
}

// Add sample `thist` of the current fields to the transforms of `slot`.
// Factors DTNYQ*DT*exp(-i pi 2 k n / NTNYQ) in FP64, stored FP32
// (src/automatic_kernels.c:1106-1110); cos/sin of pi x after an exact
// reduction of x modulo 2.
void dft_sample(sfd_plan *p, int slot, int thist, cudaStream_t st)
{
    const Grid &g = p->g;
    DftSet d;
    memset(&d, 0, sizeof d);
    d.nf = p->nfreqs;
    for (int k = 0; k < p->nfreqs; k++) {
        const double ph = std::fmod(2.0 * p->gradfreqsn[k] * thist / p->ntnyq, 2.0);
        d.re[k] = (float)(p->dtnyq * p->DT_lit * std::cos(PI_D * ph));
        d.im[k] = (float)(-p->dtnyq * p->DT_lit * std::sin(PI_D * ph));
    }
    int n = 0;
    for (int w = 0; w < NW; w++)
        if (p->d_fw[slot][w]) { d.v[n] = p->f.w[w]; d.f[n] = p->d_fw[slot][w]; d.n[n] = g.nvol; n++; }
    for (int r = 0; r < NR; r++)
        if (p->d_fr[slot][r]) { d.v[n] = p->f.r[r]; d.f[n] = p->d_fr[slot][r]; d.n[n] = g.nvol * g.L; n++; }
    d.nvar = n;
    launch_savefreqs(d, st);
}

// The DFT adjoint and gradient assembly (time_stepping.c:862-972 with
// BACK_PROP_TYPE=2): residuals are on the device already.
int adjoint_dft(sfd_plan *p, const PointSet &R, unsigned omask, cudaStream_t st)
{
    const Grid &g = p->g;
    const int NT = p->cfg.nt, tmin = p->cfg.tmin;
    int rc;
    // initsavefreqs + init_f (time_stepping.c:655-670): fields, memory
    // variables, CPML memory and the adjoint transforms start at zero
    if ((rc = zero_forward_state(p, st))) return rc;
    if ((rc = zero_dft(p, 1, st))) return rc;
    Grid ga = g;
    ga.bp2 = 1;
    AdjFields a = p->a;
    for (int w = 0; w < NW; w++) { a.wr[w] = p->f.w[w]; a.bnd[w] = nullptr; }
    for (int r = 0; r < NR; r++) a.rr[r] = p->f.r[r];
    LoopKey key;
    key.add(2); key.add(ga); key.add(p->f); key.add(a); key.add_points(R); key.add(omask); key.add(p->d_res);
    key.add(p->d_surf_q); key.add(p->cfg.tmax); key.add(tmin); key.add(p->nfreqs); key.add(p->dtnyq);
    key.add(p->ntnyq); key.add(p->gradfreqsn); key.add(p->d_fw); key.add(p->d_fr);
    const float *chk = check_field(a.wr);
    const int64_t nchk = g.nvol * g.nb;
    if ((rc = arm_unstable(p, st))) return rc;
    CKC(cudaEventRecord(p->ev0, st));
    int rc2 = run_loop(p, p->gadj, key.s, st, [&](cudaStream_t s) {
        for (int t = p->cfg.tmax - 1; t > tmin; t--) {
            if (g.freesurf) launch_surface_adj(ga, p->f, a, p->d_surf_q, s);
            launch_residuals(ga, a, R, p->d_res, NT, t, omask, s);
            launch_update_adj(ga, p->f, a, true, SFD_PREC_FP32, s);
            launch_update_adj(ga, p->f, a, false, SFD_PREC_FP32, s);
            if ((t - tmin) % p->dtnyq == 0) dft_sample(p, 1, (t - tmin) / p->dtnyq, s);
            if (t % FINITE_CHECK_EVERY == 0 || t == tmin + 1)
                launch_finite_check(g, chk, nchk, t, p->d_unstable, s);
        }
    });
    if (rc2) return rc2;
    // calc_grad (src/calc_grad.c:376-420 for the constants)
    GradDft d;
    memset(&d, 0, sizeof d);
    for (int s = 0; s < 2; s++) {
        for (int w = 0; w < NW; w++) d.fw[s][w] = p->d_fw[s][w];
        for (int r = 0; r < NR; r++) d.fr[s][r] = p->d_fr[s][r];
    }
    d.nf = p->nfreqs;
    d.par_type = p->cfg.param_type;
    for (int k = 0; k < p->nfreqs; k++) d.w[k] = (float)(2.0 * PI_D * p->df * p->gradfreqsn[k]);
    const float w0 = (float)(2.0 * PI_D * p->cfg.f0);
    float al = 0.0f;
    for (int l = 0; l < g.L; l++) {
        d.tausig[l] = (float)(1.0 / (2.0 * PI_D * p->cfg.fl[l]));
        const double q = std::pow(w0 / (2.0 * PI_D * p->cfg.fl[l]), 2);
        al = (float)(al + q / (1.0 + q));
    }
    d.al = al;
    d.ntnyq = (float)p->ntnyq;
    launch_calc_grad(g, p->f, p->a, d, st);
    CKC(cudaEventRecord(p->ev1, st));
    CKC(cudaGetLastError());
    CKC(cudaStreamSynchronize(st));
    cudaEventElapsedTime(&p->last_ms, p->ev0, p->ev1);
    p->have_forward = false;
    p->have_dft = false;
    return take_unstable(p, st, "adjoint");
}

}  // namespace

// ====================================================================== ABI
namespace {
int check_config(const sfd_config &c)
{
    if (c.nd != 2 && c.nd != 3 && c.nd != 21 && c.nd != 22) return SFD_ERR_UNSUPPORTED;
    // the reference has no acoustic free surface (assign_modeling_case.c:957-970) and its
    // viscoelastic SH stress kernel does not compile (update_s2D_SH.cl:290)
    if (c.nd == 22 && c.freesurf) return SFD_ERR_UNSUPPORTED;
    if (c.nd == 21 && c.L > 0) return SFD_ERR_UNSUPPORTED;
    if (c.fdorder < 2 || c.fdorder > 12 || c.fdorder % 2) return SFD_ERR_ARG;
    if (c.maxrelerror < 0 || c.maxrelerror > 4) return SFD_ERR_ARG;
    if (c.L < 0 || c.L > 8 || c.nt <= 0 || !(c.dt > 0) || !(c.dh > 0) || c.nab < 0) return SFD_ERR_ARG;
    if (c.abs_type != 1 && c.abs_type != 2 && c.abs_type != 0) return SFD_ERR_ARG;
    for (int i = 0; i < (c.nd == 3 ? 3 : 2); i++)
        if (c.n[i] <= 0) return SFD_ERR_ARG;
    // N[0] must be even (read_hdf5.c:535-540)
    if (c.n[0] % 2) return SFD_ERR_ARG;
    if (c.precision < 0 || c.precision > 2) return SFD_ERR_ARG;
    if (c.kernels < 0 || c.kernels > 7) return SFD_ERR_ARG;
    if (c.adjoint_reset_psi < 0 || c.adjoint_reset_psi > 1) return SFD_ERR_ARG;
    if (c.field_precision < 0 || c.field_precision > 2) return SFD_ERR_ARG;
    // FP16 memory variables with FP32 wave fields: the 4-cell stress kernel
    // of single-shot 3D viscoelastic modelling
    if (c.field_precision == 2 && (c.nd != 3 || c.L < 1 || c.L > 3 || c.fdorder != 8 || c.n[0] % 4 ||
                                   c.kernels != 0 || c.batch > 1 || c.checkpoint > 0 || c.hout))
        return SFD_ERR_UNSUPPORTED;
    // 16-bit fields: 3D (L <= 3, the 4-cell and streaming kernels) and 2D P-SV
    if (c.field_precision == 1 && ((c.nd != 3 && c.nd != 2) || c.L > 3)) return SFD_ERR_UNSUPPORTED;
    if (c.back_prop_type < 0 || c.back_prop_type > 2) return SFD_ERR_ARG;
    if (c.loop_graphs < 0 || c.loop_graphs > 2) return SFD_ERR_ARG;
    if (c.hout < 0 || c.hout > 1) return SFD_ERR_ARG;
    // the reference's 3D Hessian kernel does not compile (update_adjv3D.cl:486)
    if (c.hout && c.nd == 3 && c.back_prop_type != 2) return SFD_ERR_UNSUPPORTED;
    if (c.batch < 0 || c.batch > 64) return SFD_ERR_ARG;
    if (c.checkpoint < 0) return SFD_ERR_ARG;
    // checkpointed gradients: boundary-saving semantics on P-SV and 3D grids, one shot per launch
    if (c.checkpoint > 0 && (c.back_prop_type == 2 || (c.nd != 2 && c.nd != 3) || c.batch > 1 ||
                             (c.field_precision != 0 && c.hout)))
        return SFD_ERR_UNSUPPORTED;
    // batched shots: P-SV, acoustic and 3D one-cell / 4-cell kernels in FP32,
    // boundary-saving gradients
    if (c.batch > 1 && (c.nd == 21 || c.back_prop_type == 2 || c.field_precision != 0 || c.kernels == 2 ||
                        c.kernels == 3))
        return SFD_ERR_UNSUPPORTED;
    return SFD_OK;
}

void init_grid(const sfd_config &c, Grid &g)
{
    memset(&g, 0, sizeof g);
    g.nd = c.nd;
    g.F = c.fdorder / 2;
    g.nz = c.n[0];
    if (c.nd == 3) { g.ny = c.n[1]; g.nx = c.n[2]; }
    else { g.ny = 1; g.nx = c.n[1]; }
    g.NZ = g.nz + 2 * g.F;
    g.NX = g.nx + 2 * g.F;
    g.NY = c.nd == 3 ? g.ny + 2 * g.F : 1;
    g.nab = c.abs_type == 0 ? 0 : c.nab;
    g.abs_type = g.nab < 1 ? 0 : c.abs_type;  // NAB<1 disables absorption (assign_modeling_case.c:1045)
    g.L = c.L;
    g.freesurf = c.freesurf ? 1 : 0;
    g.restype = c.restype;
    // 6: the kernels of 0, plus the fused modelling step; 7: the kernels of 0
    // with the cp.async-staged velocity update
    g.kernels = (c.kernels == 6 || c.kernels == 7) ? 0 : c.kernels;
    g.fused = c.kernels == 6;
    g.vasync = c.kernels == 7;
    g.hout = c.hout;
    g.nvol = (int64_t)g.NZ * g.NY * g.NX;
    double hc[6];
    holberg(c.fdorder, c.maxrelerror, hc);
    for (int i = 0; i < 6; i++) g.hc[i] = (float)hc[i];
    g.dt = c.dt;
    g.dt2 = (float)((double)c.dt / 2.0);
    for (int l = 0; l < 8; l++) g.eta[l] = l < c.L ? (float)(2.0 * 3.141592653589793238462643 * c.fl[l] * (double)c.dt) : 0.0f;
    for (int l = 0; l < 8; l++) {
        volatile float half = g.eta[l] * 0.5f;   // FP32 steps, as a kernel would form them
        g.eta_b[l] = 1.0f / (1.0f + half);
        g.eta_c[l] = 1.0f - half;
    }
    g.inv_dt = 1.0f / c.dt;
    g.fhalf = c.field_precision == 1;
    g.rhalf = c.field_precision == 2;
    g.rsc = g.rsci = 1.0f;
    for (int w = 0; w < NW; w++) g.ws.w[w] = g.bsc[w] = g.bsci[w] = 1.0f;
    g.nbnd = nbnd_cells(g.nd, g.nz, g.ny, g.nx, g.F, g.nab, g.freesurf);
    g.nb = 1;
    g.sb_w = g.nvol;
    g.sb_r = g.nvol * g.L;
    int64_t psz[NPSI];
    g.sb_psi = psi_sizes(g, psz);
    g.sb_g = (int64_t)g.nz * g.ny * g.nx;
    g.sb_q = (int64_t)g.nx * g.ny;
    g.sb_bnd = (int64_t)(c.precision == SFD_PREC_FP32 ? 4 : 2) * c.nt * g.nbnd;
}
}  // namespace

extern "C" int sfd_plan_create(const sfd_config *cfg, sfd_plan **out)
{
    if (!cfg || !out) return SFD_ERR_ARG;
    *out = nullptr;
    const sfd_config &c = *cfg;
    int rc = check_config(c);
    if (rc) return rc;
    sfd_plan *p = new sfd_plan();
    p->cfg = c;
    Grid &g = p->g;
    init_grid(c, g);
    if (p->cfg.tmax <= 0 || p->cfg.tmax > c.nt) p->cfg.tmax = c.nt;
    if (p->cfg.tmin < 0) p->cfg.tmin = 0;
    p->DH_lit = literal9((double)c.dh);
    p->DT_lit = literal9((double)c.dt);
    p->model_set = false;
    p->have_forward = false;
    p->d_psi_all = nullptr;
    for (int w = 0; w < NW; w++) p->d_bnd[w] = nullptr;
    p->bnd_elem = c.precision == SFD_PREC_FP32 ? 4 : 2;
    p->cap_src = p->cap_rec = 0;
    p->d_surf_q = nullptr;
    p->d_ticket = nullptr;
    p->d_unstable = nullptr;
    p->d_fsync = nullptr;
    p->dev_bytes = 0;
    p->batch = std::max(1, c.batch);
    p->fwd_nb = 0;
    p->d_snap = p->d_seg = nullptr;
    p->d_psi_adj = nullptr;
    p->d_padj = nullptr;
    p->padj_valid = false;
    p->snap_bytes = p->seg_bytes = 0;
    p->nseg = 0;
    memset(&p->f, 0, sizeof p->f);
    memset(&p->a, 0, sizeof p->a);
    p->last_ms = 0.0f;
    p->kshift = p->bshift = 0;
    p->nfreqs = p->dtnyq = p->ntnyq = p->dft_nf = 0;
    p->df = 0.0f;
    memset(p->d_fw, 0, sizeof p->d_fw);
    p->movout = 0;
    memset(p->mov_dst, 0, sizeof p->mov_dst);
    p->d_mov = nullptr;
    p->mov_cap = 0;
    memset(p->d_fr, 0, sizeof p->d_fr);
    p->have_dft = false;
    if (cudaGetDevice(&p->device) != cudaSuccess) { delete p; return SFD_ERR_CUDA; }
    if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess) { delete p; return SFD_ERR_CUDA; }
    p->own_stream = true;
    cudaEventCreate(&p->ev0);
    cudaEventCreate(&p->ev1);
    *out = p;
    return SFD_OK;
}

extern "C" int sfd_footprint(const sfd_config *cfg, int gradient, int nsrc, int64_t nrec_sel, int nfreqs,
                             int64_t *bytes)
{
    if (!cfg || !bytes || nsrc < 0 || nrec_sel < 0 || nfreqs < 0 || nfreqs > MAXFREQ) return SFD_ERR_ARG;
    int rc = check_config(*cfg);
    if (rc) return rc;
    Grid g;
    init_grid(*cfg, g);
    const int64_t nt = cfg->nt, npar = (int64_t)g.nz * g.ny * g.nx;
    int nwave = 0, nmem = 0;
    for (int w = 0; w < NW; w++) nwave += is_wave_used(g, w);
    for (int r = 0; r < NR; r++) nmem += is_mem_used(g, r);
    // alloc_model: wave fields, memory variables, CPML memory, parameters, constants
    int64_t psz[NPSI];
    const int64_t nc = std::max(2 * g.nab, 1);
    const int64_t B = std::max(1, cfg->batch);   // copies of the per-shot arrays
    int64_t b = B * ((int64_t)wave_elem(g) * g.nvol * nwave + (int64_t)mem_elem(g) * g.nvol * nmem * g.L +
                     4 * psi_sizes(g, psz)) +
                4 * npar * NPAR + 4 * (3 * NC * nc + nc + 6 * nc);
    // ensure_shot_buffers: source maps and signatures, receiver maps, seismograms and residuals
    const int64_t cs = std::max<int64_t>(nsrc, 16), cr = std::max<int64_t>(nrec_sel, 16);
    b += cs * (8 + 4 + 12 + 4 + 12 + 4 * nt) + cr * (8 + 8 * nt);
    b += 2 * sizeof(int);   // fused-step block counter, instability flag
    {
        const FusedShape fsh = fused_shape(g);
        if (B == 1 && fsh.units) b += 4 * (1 + fsh.units);   // fused 3D step tickets and flags
    }
    if (gradient) {
        const bool bp2 = cfg->back_prop_type == 2;
        int ng = 0;
        for (int k = 0; k < NG; k++) ng += !((k == GTAUP || k == GTAUS) && !(bp2 && g.L > 0));
        b += B * (8 * npar * (ng + (cfg->hout ? NG : 0)) + 4 * (int64_t)g.nx * g.ny);
        if (bp2) {
            b += 2 * 8 * (int64_t)nfreqs * g.nvol * (nwave + (int64_t)nmem * g.L);
        } else {
            b += B * 4 * g.nvol * (nwave + (int64_t)nmem * g.L);
            if (cfg->checkpoint > 0) {   // snapshots, segment store, adjoint CPML memory
                const CkptSizes z = ckpt_sizes(g, *cfg);
                b += (int64_t)(z.snap * z.nseg + z.seg) + 4 * std::max<int64_t>(z.psi, 1);
                if (g.fhalf) b += 4 * npar * 8;   // the adjoint's unscaled moduli and buoyancies
            } else {
                b += B * (int64_t)(cfg->precision == SFD_PREC_FP32 ? 4 : 2) * nt * g.nbnd * nwave;
            }
        }
    }
    *bytes = b;
    return SFD_OK;
}

extern "C" int64_t sfd_plan_device_bytes(const sfd_plan *p)
{
    return p ? p->dev_bytes : SFD_ERR_ARG;
}

extern "C" int sfd_release_memory(void)
{
    int dev;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess)
        return SFD_ERR_CUDA;
    if (cudaDeviceSynchronize() != cudaSuccess || cudaMemPoolTrimTo(pool, 0) != cudaSuccess) return SFD_ERR_CUDA;
    return SFD_OK;
}

extern "C" int sfd_device_memory(int64_t *free_bytes, int64_t *total_bytes)
{
    size_t f = 0, t = 0;
    if (cudaMemGetInfo(&f, &t) != cudaSuccess) return SFD_ERR_CUDA;
    if (free_bytes) *free_bytes = (int64_t)f;
    if (total_bytes) *total_bytes = (int64_t)t;
    return SFD_OK;
}

extern "C" void sfd_plan_destroy(sfd_plan *p)
{
    if (!p) return;
    cudaStreamSynchronize(p->stream);
    drop_graph(p->gfwd);
    drop_graph(p->gadj);
    for (auto &a : p->allocs) dfree(p, a.first, a.second);
    for (int w = 0; w < NW; w++) dfree(p, p->d_bnd[w], p->bnd_elem * (size_t)p->cfg.nt * p->g.nbnd * p->batch);
    free_dft(p);
    dfree(p, p->d_mov, sizeof(float) * p->mov_cap);
    cudaStreamSynchronize(p->stream);
    cudaEventDestroy(p->ev0);
    cudaEventDestroy(p->ev1);
    if (p->own_stream) cudaStreamDestroy(p->stream);
    delete p;
}

extern "C" const char *sfd_last_error(const sfd_plan *p) { return p ? p->err.c_str() : "null plan"; }

extern "C" int sfd_set_model(sfd_plan *p, const float *const *params)
{
    if (!p || !params) return SFD_ERR_ARG;
    int rc = transform_model(p->cfg, p->g.nz, p->g.ny, p->g.nx, params, p->hp, p->err);
    if (rc) return rc;
    if (!p->model_set) {
        if ((rc = alloc_model(p))) return rc;
        if ((rc = upload_constants(p))) return rc;
    }
    int64_t npar = (int64_t)p->g.nz * p->g.ny * p->g.nx;
    // FP16 stores keep velocities as v * 2^b and stresses as s * 2^a with
    // b - a ~ log2 of the impedance, so both stay near the same magnitude
    {
        double acc = 0.0;
        int64_t n = 0, step = std::max<int64_t>(1, npar / 4096);
        for (int64_t i = 0; i < npar; i += step) {
            const double z = std::sqrt((double)p->hp[PM][i] / (double)p->hp[PRIP][i]);
            if (z > 0 && std::isfinite(z)) { acc += std::log2(z); n++; }
        }
        p->bshift = n ? (int)std::lround(acc / n) : 0;
    }
    {
        // the free-surface adjoint forms C^-1 at the top row with the factor
        // 1 / (4 M mu - 4 mu^2) in 2D and 1 / (6 M mu - 8 mu^2) in 3D
        // (surface2D_adj.cl, surface3D_adj.cl): undefined where mu = 0
        p->surf_mu_zero = false;
        const int64_t ncol = (int64_t)p->g.ny * p->g.nx;
        for (int64_t c = 0; c < ncol && !p->surf_mu_zero; c++)
            if (!(p->hp[PMU][c * p->g.nz] > 0.0f)) p->surf_mu_zero = true;
    }
    if (p->g.fhalf) {
        // FP16 wave fields: the moduli carry 2^-kshift and the buoyancies
        // 2^kshift (exact power-of-two scalings of the FP32 parameters).
        p->kshift = p->bshift;
        const int up[3] = {PRIP, PRJP, PRKP}, down[5] = {PM, PMU, PMUIPKP, PMUIPJP, PMUJPKP};
        std::vector<float> tmp(npar);
        for (int k = 0; k < NPAR; k++) {
            int e = 0;
            for (int q : up) if (q == k) e = p->kshift;
            for (int q : down) if (q == k) e = -p->kshift;
            for (int64_t i = 0; i < npar; i++) tmp[i] = std::ldexp(p->hp[k][i], e);
            CKC(cudaMemcpy((void *)p->f.p[k], tmp.data(), sizeof(float) * npar, cudaMemcpyHostToDevice));
        }
    } else {
        for (int k = 0; k < NPAR; k++)
            CKC(cudaMemcpy((void *)p->f.p[k], p->hp[k].data(), sizeof(float) * npar, cudaMemcpyHostToDevice));
    }
    p->model_set = true;
    p->padj_valid = false;
    p->have_forward = false;
    return SFD_OK;
}

extern "C" int sfd_source_type_mask(const float *src_pos, int nsrc_all)
{
    int m = 0;
    for (int s = 0; s < nsrc_all; s++) {
        int t = (int)src_pos[5 * s + 4];
        if (t >= 0 && t < 4) m |= 1 << t;
        if (t == 100) m |= 1 << 4;
    }
    return m;
}

namespace {
// the shots of one batched call: sources, receivers and their totals
struct ShotBatch {
    int n, nsrc, nrec;
    const sfd_shot *shots;
};
int check_batch(sfd_plan *p, int nshot, const sfd_shot *shots, ShotBatch &sb)
{
    if (nshot < 1 || !shots) return fail(p, SFD_ERR_ARG, "a batch needs at least one shot");
    if (nshot > p->batch) return fail(p, SFD_ERR_ARG, "more shots than the plan's batch");
    sb.n = nshot;
    sb.shots = shots;
    sb.nsrc = sb.nrec = 0;
    for (int b = 0; b < nshot; b++) {
        if (shots[b].nsrc < 0 || shots[b].nrec < 0) return fail(p, SFD_ERR_ARG, "negative source or receiver count");
        sb.nsrc += shots[b].nsrc;
        sb.nrec += shots[b].nrec;
    }
    return SFD_OK;
}
}  // namespace

extern "C" int sfd_forward(sfd_plan *p, const sfd_shot *shot, int mask, const int *outsel, float *const *seis,
                           int save_boundaries, void *stream)
{
    if (!p || !shot) return SFD_ERR_ARG;
    return sfd_forward_batch(p, 1, shot, mask, outsel, seis, save_boundaries, stream);
}

extern "C" int sfd_forward_batch(sfd_plan *p, int nshot, const sfd_shot *shots, int mask, const int *outsel,
                                 float *const *seis, int save_boundaries, void *stream)
{
    if (!p) return SFD_ERR_ARG;
    if (!p->model_set) return fail(p, SFD_ERR_STATE, "sfd_set_model must be called first");
    int rc;
    ShotBatch sb;
    if ((rc = check_batch(p, nshot, shots, sb))) return rc;
    if ((rc = check_outsel(p, outsel))) return rc;
    if (nshot > 1 && save_boundaries && p->cfg.back_prop_type == 2)
        return fail(p, SFD_ERR_UNSUPPORTED, "batched shots cover the boundary-saving gradient");
    if (nshot > 1 && p->movout > 0) return fail(p, SFD_ERR_UNSUPPORTED, "a movie films one shot per run");
    cudaStream_t st = stream ? (cudaStream_t)stream : p->stream;
    p->g.nb = nshot;
    const Grid &g = p->g;
    int nsel;
    unsigned omask = outmask_of(outsel, g.nd, &nsel);
    if ((rc = ensure_shot_buffers(p, sb.nsrc, sb.nrec, nsel))) return rc;
    PointSet S, R;
    if ((rc = upload_shots(p, nshot, shots, mask, S, R, st))) return rc;
    if ((rc = zero_forward_state(p, st))) return rc;
    // a batch without receivers has no seismogram buffer (none is allocated
    // for zero traces): no copy of zero bytes goes to a null pointer
    if (nsel && sb.nrec) CKC(cudaMemsetAsync(p->d_seis, 0, sizeof(float) * (size_t)nsel * sb.nrec * p->cfg.nt, st));
    BndSlot bs;
    memset(&bs, 0, sizeof bs);
    // FP16 stores: the source injects about 2^4 per step into the field it
    // feeds (velocities for force sources, stresses otherwise)
    auto store_exponents = [&](int shift, int &a, int &b) {
        float smax = 0.0f;
        bool force_only = sb.nsrc > 0;
        for (int q = 0; q < nshot; q++)
            for (int i = 0; i < shots[q].nsrc; i++) {
                const int ty = (int)shots[q].src_pos[5 * i + 4];
                if (ty != 0 && ty != 1 && ty != 2) force_only = false;
                for (int t = 0; t < p->cfg.nt; t++)
                    smax = std::max(smax, std::fabs(shots[q].src[(int64_t)i * p->cfg.nt + t]));
            }
        const double inj = (double)smax * p->cfg.dt;
        const int e0 = inj > 0 ? (int)std::lround(4.0 - std::log2(inj)) : 0;
        a = force_only ? e0 - shift : e0;
        b = a + shift;
    };
    if (g.fhalf) {
        if (save_boundaries && !(p->cfg.checkpoint > 0 && p->cfg.back_prop_type != 2))
            return fail(p, SFD_ERR_UNSUPPORTED,
                        "FP16 wave-field storage covers forward modelling and checkpointed gradients");
        int a, b;
        store_exponents(p->kshift, a, b);
        for (int w = 0; w < NW; w++) p->g.ws.w[w] = std::ldexp(1.0f, w <= VZ ? b : a);
    }
    if (g.rhalf) {
        // FP16 memory variables: stored times the stress scale FP16 wave
        // fields would take (about 2^4 injected per step for explosive sources)
        if (save_boundaries)
            return fail(p, SFD_ERR_UNSUPPORTED, "FP16 memory variables cover forward modelling only");
        int a, b;
        store_exponents(p->bshift, a, b);
        p->g.rsc = std::ldexp(1.0f, a);
        p->g.rsci = std::ldexp(1.0f, -a);
    }
    for (int w = 0; w < NW; w++) p->g.bsc[w] = p->g.bsci[w] = 1.0f;
    if (save_boundaries && p->cfg.precision == SFD_PREC_FP16) {
        // without a scale, velocities (~stress / impedance) fall below FP16's range
        int a, b;
        store_exponents(p->bshift, a, b);
        for (int w = 0; w < NW; w++) {
            p->g.bsc[w] = std::ldexp(1.0f, w <= VZ ? b : a);
            p->g.bsci[w] = std::ldexp(1.0f, w <= VZ ? -b : -a);
        }
    }
    // a gradient run keeps the boundary shells (BACK_PROP_TYPE 1) or the
    // forward transforms (2)
    const bool dft = save_boundaries && p->cfg.back_prop_type == 2;
    const bool ckpt = save_boundaries && !dft && p->cfg.checkpoint > 0;
    if (dft) {
        if (g.nd == 21 || g.nd == 22)
            return fail(p, SFD_ERR_UNSUPPORTED, "the adjoint path covers P-SV and 3D elastic/viscoelastic media");
        if (!p->nfreqs) return fail(p, SFD_ERR_STATE, "sfd_set_gradfreqs must be called before a DFT-gradient run");
        if ((rc = alloc_dft(p))) return rc;
        if ((rc = zero_dft(p, 0, st))) return rc;
    } else if (save_boundaries && p->cfg.checkpoint > 0) {
        if (p->movout > 0) return fail(p, SFD_ERR_UNSUPPORTED, "a checkpointed gradient films no movie");
        if ((rc = alloc_ckpt(p))) return rc;
    } else if (save_boundaries) {
        if (g.nd == 21 || g.nd == 22)
            return fail(p, SFD_ERR_UNSUPPORTED, "the adjoint path covers P-SV and 3D elastic/viscoelastic media");
        if (g.nab <= 0 || g.nbnd <= 0) return fail(p, SFD_ERR_ARG, "boundary saving needs an absorbing layer");
        for (int w = 0; w < NW; w++) {
            if (!p->f.w[w]) continue;
            if (!p->d_bnd[w]) {
                cudaError_t e;
                p->d_bnd[w] = dalloc_raw(p, p->bnd_elem * (size_t)p->cfg.nt * g.nbnd * p->batch, &e);
                if (!p->d_bnd[w]) return fail(p, SFD_ERR_MEMORY, "saved-boundary store does not fit in device memory");
            }
            bs.p[w] = p->d_bnd[w];
            bs.fields[bs.nfield++] = w;
        }
    }
    p->have_forward = false;
    p->have_dft = false;
    const int NT = p->cfg.nt, tmax = p->cfg.tmax, tmin = p->cfg.tmin;
    // the movie of a boundary-saving gradient run is filmed by its adjoint
    // (time_stepping.c:819-822)
    Movie mv;
    if (!(save_boundaries && !dft) && (rc = movie_setup(p, omask, mv))) return rc;
    // modelling runs of 2D P-SV / acoustic grids: two launches per step
    // (update_v; update_s with the free surface, the receivers and the next
    // step's sources, the last two done by the block that finishes last).
    // Not in 3D: there the last-block handshake costs each of the ~10^4
    // blocks of a launch a fence and an atomic round trip, and a surface
    // done by the top blocks of the stress kernel holds them on the SMs;
    // both made a 256^3 step slower (1.31 and 1.19 ms against 1.13).
    const bool fuse2d = (g.nd == 2 || g.nd == 22) && g.kernels != 1 && !save_boundaries && !dft && !mv.n;
    if (fuse2d) CKC(cudaMemsetAsync(p->d_ticket, 0, sizeof(int), st));
    // 3D modelling runs: one launch per step for the velocity, stress and
    // free-surface updates (sfd_kernels.cu, fused 3D forward step)
    const FusedShape fsh = fused_shape(g);
    const bool fuse3d = g.nd == 3 && nshot == 1 && p->d_fsync && fsh.units && !save_boundaries && !dft && !mv.n;
    const bool bnd_shells = save_boundaries && !dft && !ckpt;
    LoopKey key;
    key.add(mv.n); key.add(p->movout); key.add(p->d_mov); key.add(fuse2d); key.add(p->d_ticket); key.add(fuse3d);
    key.add(1); key.add(p->g); key.add(p->f); key.add_points(S); key.add_points(R); key.add(p->d_src);
    key.add(p->d_seis); key.add(omask); key.add(dft); key.add(save_boundaries != 0); key.add(bs);
    key.add(p->cfg.precision); key.add(tmax); key.add(tmin); key.add(ckpt); key.add(p->d_snap);
    if (dft) {
        key.add(p->nfreqs); key.add(p->dtnyq); key.add(p->ntnyq); key.add(p->gradfreqsn); key.add(p->d_fw);
        key.add(p->d_fr);
    }
    const float *chk = check_field(p->f.w);
    const int64_t nchk = g.nvol * g.nb;
    auto check = [&](int t, cudaStream_t s) {
        if ((t + 1) % FINITE_CHECK_EVERY == 0 || t == tmax - 1) launch_finite_check(g, chk, nchk, t, p->d_unstable, s);
    };
    if ((rc = arm_unstable(p, st))) return rc;
    CKC(cudaEventRecord(p->ev0, st));
    int rcl = run_loop(p, p->gfwd, key.s, st, [&](cudaStream_t s) {
        if (fuse2d) {
            if (tmax > 0) launch_sources(g, p->f, S, p->d_src, NT, 0, 1, s);
            for (int t = 0; t < tmax; t++) {
                launch_update_v(g, p->f, s);
                StepTail tl{p->d_ticket, R, p->d_seis, omask, t, S, p->d_src, t + 1 < tmax ? t + 1 : -1, NT};
                launch_update_s_step(g, p->f, tl, s);
                check(t, s);
            }
            return;
        }
        if (fuse3d) {
            cudaMemsetAsync(p->d_fsync, 0, sizeof(int) * (size_t)(1 + fsh.units), s);
            for (int t = 0; t < tmax; t++) {
                launch_sources(g, p->f, S, p->d_src, NT, t, 1, s);
                launch_fused_step(g, p->f, p->d_fsync, t, s);
                launch_record(g, p->f, R, p->d_seis, NT, t, omask, s);
                check(t, s);
            }
            return;
        }
        for (int t = 0; t < tmax; t++) {
            // the state after t steps, before the sources of step t (time_stepping.c:766-781)
            if (dft && t >= tmin && (t - tmin) % p->dtnyq == 0) dft_sample(p, 0, (t - tmin) / p->dtnyq, s);
            if (ckpt && t % p->cfg.checkpoint == 0) ckpt_snapshot(p, t / p->cfg.checkpoint, false, s);
            launch_sources(g, p->f, S, p->d_src, NT, t, 1, s);
            launch_update_v(g, p->f, s);
            // the stress kernel may apply the free surface itself, unless the
            // saved boundaries must see the stresses before it
            const bool folded = launch_update_s(g, p->f, s, !bnd_shells);
            if (bnd_shells) launch_savebnd(g, p->f, bs, p->cfg.precision, (int64_t)t * g.nbnd, s);
            if (g.freesurf && !folded) launch_surface(g, p->f, 1, s);
            launch_record(g, p->f, R, p->d_seis, NT, t, omask, s);
            if (mv.n && (t + 1) % p->movout == 0) movie_snap(p, mv, (t + 1) / p->movout - 1, s);
            check(t, s);
        }
    });
    if (rcl) return rcl;
    if (mv.n && (rc = movie_out(p, mv, st))) return rc;
    CKC(cudaEventRecord(p->ev1, st));
    CKC(cudaGetLastError());
    int slot = 0;
    for (int o = 0; o < SFD_NOUT; o++) {
        if (!(omask & (1u << o))) continue;
        if (seis && seis[o] && sb.nrec)
            CKC(cudaMemcpyAsync(seis[o], p->d_seis + (size_t)slot * sb.nrec * NT,
                                sizeof(float) * (size_t)sb.nrec * NT, cudaMemcpyDeviceToHost, st));
        slot++;
    }
    CKC(cudaStreamSynchronize(st));
    cudaEventElapsedTime(&p->last_ms, p->ev0, p->ev1);
    if (tma_take_status())
        return fail(p, SFD_ERR_CUDA, "a TMA stage of the 3D stencil kernels did not arrive within its time bound");
    if (fuse3d && fused_take_status())
        return fail(p, SFD_ERR_CUDA, "a fused 3D step did not see its neighbours' velocities within its time bound");
    if ((rc = take_unstable(p, st, "forward"))) return rc;
    p->have_forward = save_boundaries != 0;
    p->fwd_nb = nshot;
    p->have_dft = dft;
    return SFD_OK;
}

extern "C" int sfd_adjoint(sfd_plan *p, const sfd_shot *shot, int mask, const int *outsel,
                           const float *const *residuals, void *stream)
{
    if (!p || !shot) return SFD_ERR_ARG;
    return sfd_adjoint_batch(p, 1, shot, mask, outsel, residuals, stream);
}

extern "C" int sfd_adjoint_batch(sfd_plan *p, int nshot, const sfd_shot *shots, int mask, const int *outsel,
                                 const float *const *residuals, void *stream)
{
    if (!p) return SFD_ERR_ARG;
    int rc;
    ShotBatch sb;
    if ((rc = check_batch(p, nshot, shots, sb))) return rc;
    if (p->g.nd == 21 || p->g.nd == 22)
        return fail(p, SFD_ERR_UNSUPPORTED, "the adjoint path covers P-SV and 3D elastic/viscoelastic media");
    if (p->g.fhalf && p->cfg.checkpoint <= 0)
        return fail(p, SFD_ERR_UNSUPPORTED, "FP16 wave-field storage covers forward modelling and checkpointed gradients");
    if (p->g.rhalf) return fail(p, SFD_ERR_UNSUPPORTED, "FP16 memory variables cover forward modelling only");
    if (!p->have_forward) return fail(p, SFD_ERR_STATE, "sfd_adjoint needs a preceding sfd_forward with saved boundaries");
    if (nshot != p->fwd_nb) return fail(p, SFD_ERR_STATE, "the adjoint must follow a forward run of the same shots");
    if (p->g.freesurf && p->surf_mu_zero)
        return fail(p, SFD_ERR_UNSUPPORTED, "the free-surface adjoint divides by mu, which is zero at the surface "
                                            "(acoustic media: use a plan without a free surface)");
    if ((rc = check_outsel(p, outsel))) return rc;
    if ((rc = alloc_adjoint(p))) return rc;
    cudaStream_t st = stream ? (cudaStream_t)stream : p->stream;
    p->g.nb = nshot;
    const Grid &g = p->g;
    int nsel;
    unsigned omask = outmask_of(outsel, g.nd, &nsel);
    if ((rc = ensure_shot_buffers(p, sb.nsrc, sb.nrec, nsel))) return rc;
    PointSet S, R;
    if ((rc = upload_shots(p, nshot, shots, mask, S, R, st))) return rc;
    const int NT = p->cfg.nt;
    int slot = 0;
    for (int o = 0; o < SFD_NOUT; o++) {
        if (!(omask & (1u << o))) continue;
        if (!residuals || !residuals[o]) return fail(p, SFD_ERR_ARG, "missing residual array");
        if (sb.nrec)
            CKC(cudaMemcpyAsync(p->d_res + (size_t)slot * sb.nrec * NT, residuals[o],
                                sizeof(float) * (size_t)sb.nrec * NT, cudaMemcpyHostToDevice, st));
        slot++;
    }
    if (p->cfg.back_prop_type == 2) {
        if (!p->have_dft) return fail(p, SFD_ERR_STATE, "the forward transforms are missing (gradfreqs changed?)");
        return adjoint_dft(p, R, omask, st);
    }
    // adjoint fields start at zero; the CPML memory carries over from the
    // forward run (the reference binds the forward psi buffers by name)
    for (int w = 0; w < NW; w++)
        if (p->a.wr[w]) CKC(cudaMemsetAsync(p->a.wr[w], 0, sizeof(float) * g.nvol * nshot, st));
    for (int r = 0; r < NR; r++)
        if (p->a.rr[r]) CKC(cudaMemsetAsync(p->a.rr[r], 0, sizeof(float) * g.nvol * g.L * nshot, st));
    if (p->cfg.checkpoint > 0) return adjoint_ckpt(p, S, R, omask, st);
    if (p->cfg.adjoint_reset_psi) {
        // optional: start the adjoint with clean CPML memory instead
        int64_t tot = 0;
        for (int i = 0; i < NPSI; i++) tot += psi_span(p->psi_size[i]);
        if (tot) CKC(cudaMemsetAsync(p->d_psi_all, 0, sizeof(float) * tot * nshot, st));
    }
    AdjFields a = p->a;
    // the movie of a boundary-saving gradient: the reconstructed forward
    // field after each adjoint step with t % movout == 0 (time_stepping.c:927-929)
    Movie mv;
    if ((rc = movie_setup(p, omask, mv))) return rc;
    LoopKey key;
    key.add(mv.n); key.add(p->movout); key.add(p->d_mov);
    key.add(3); key.add(g); key.add(p->f); key.add(a); key.add_points(S); key.add_points(R); key.add(p->d_src);
    key.add(p->d_res); key.add(p->d_surf_q); key.add(omask); key.add(p->d_bnd); key.add(p->bnd_elem);
    key.add(p->cfg.precision); key.add(p->cfg.tmax); key.add(p->cfg.tmin);
    const float *chk = check_field(a.wr);
    const int64_t nchk = g.nvol * g.nb;
    if ((rc = arm_unstable(p, st))) return rc;
    CKC(cudaEventRecord(p->ev0, st));
    int rcl = run_loop(p, p->gadj, key.s, st, [&](cudaStream_t s) {
        for (int t = p->cfg.tmax - 1; t > p->cfg.tmin; t--) {
            for (int w = 0; w < NW; w++)
                a.bnd[w] = p->d_bnd[w] ? (const char *)p->d_bnd[w] + p->bnd_elem * (size_t)(t - 1) * g.nbnd : nullptr;
            if (g.freesurf) launch_surface_adj(g, p->f, a, p->d_surf_q, s);
            launch_residuals(g, a, R, p->d_res, NT, t, omask, s);
            launch_update_adj(g, p->f, a, true, p->cfg.precision, s);
            launch_update_adj(g, p->f, a, false, p->cfg.precision, s);
            launch_sources(g, p->f, S, p->d_src, NT, t, -1, s);
            if (mv.n && t % p->movout == 0) movie_snap(p, mv, (t + 1) / p->movout - 1, s);
            if (t % FINITE_CHECK_EVERY == 0 || t == p->cfg.tmin + 1)
                launch_finite_check(g, chk, nchk, t, p->d_unstable, s);
        }
    });
    if (rcl) return rcl;
    if (mv.n && (rc = movie_out(p, mv, st))) return rc;
    CKC(cudaEventRecord(p->ev1, st));
    CKC(cudaGetLastError());
    CKC(cudaStreamSynchronize(st));
    cudaEventElapsedTime(&p->last_ms, p->ev0, p->ev1);
    p->have_forward = false;
    return take_unstable(p, st, "adjoint");
}

namespace {
// the sum over the plan's shot copies of a device array of n doubles, in
// copy order
int fetch_sum(sfd_plan *p, const double *d, double *h, int64_t n)
{
    if (p->batch == 1) {
        CKC(cudaMemcpy(h, d, sizeof(double) * n, cudaMemcpyDeviceToHost));
        return SFD_OK;
    }
    std::vector<double> all((size_t)n * p->batch);
    CKC(cudaMemcpy(all.data(), d, sizeof(double) * all.size(), cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < n; i++) {
        double acc = all[i];
        for (int b = 1; b < p->batch; b++) acc += all[(size_t)b * n + i];
        h[i] = acc;
    }
    return SFD_OK;
}
}  // namespace

extern "C" int sfd_zero_gradient(sfd_plan *p)
{
    if (!p) return SFD_ERR_ARG;
    int rc;
    if ((rc = alloc_adjoint(p))) return rc;
    int64_t npar = (int64_t)p->g.nz * p->g.ny * p->g.nx * p->batch;
    for (int k = 0; k < NG; k++) {
        if (p->a.grad[k]) CKC(cudaMemsetAsync(p->a.grad[k], 0, sizeof(double) * npar, p->stream));
        if (p->a.hess[k]) CKC(cudaMemsetAsync(p->a.hess[k], 0, sizeof(double) * npar, p->stream));
    }
    return SFD_OK;
}

extern "C" int sfd_get_hessian(sfd_plan *p, int transform, float *const *out)
{
    if (!p || !out) return SFD_ERR_ARG;
    if (!p->g.hout) return fail(p, SFD_ERR_STATE, "the plan was not created with hout = 1");
    if (!p->a.hess[0]) return fail(p, SFD_ERR_STATE, "no Hessian has been accumulated");
    const int64_t n = (int64_t)p->g.nz * p->g.ny * p->g.nx;
    std::vector<double> h[NG];
    for (int k = 0; k < NG; k++) {
        h[k].resize(n);
        if (int rc_ = fetch_sum(p, p->a.hess[k], h[k].data(), n)) return rc_;
    }
    const int pt = p->cfg.param_type;
    if (transform && p->cfg.back_prop_type != 2 && (pt == 0 || pt == 2)) {
        // src/calc_grad.c:1004-1090 for the Hessian: the parameters rescaled
        // as for the gradient, no division by dt
        const double dt = p->cfg.dt, dh = p->cfg.dh;
        for (int64_t i = 0; i < n; i++) {
            const double rho = 1.0 / p->hp[PRHO][i] * dt / dh;
            const double M = p->hp[PM][i] * dh / dt, mu = p->hp[PMU][i] * dh / dt;
            h[GRHO][i] += M / rho * h[GM][i];
            if (mu > 0) h[GRHO][i] += mu / rho * h[GMU][i];
            const double sM = pt == 0 ? std::sqrt(rho * M) : std::sqrt(M / rho);
            const double smu = pt == 0 ? std::sqrt(rho * mu) : std::sqrt(mu / rho);
            h[GM][i] *= 2.0 * sM;
            h[GMU][i] *= 2.0 * smu;
        }
    }
    const int order[5] = {GM, GMU, GRHO, GTAUP, GTAUS};
    for (int q = 0; q < 5; q++)
        if (out[q])
            for (int64_t i = 0; i < n; i++) out[q][i] = (float)h[order[q]][i];
    return SFD_OK;
}

extern "C" int sfd_set_movie(sfd_plan *p, int movout, float *const *dst)
{
    if (!p) return SFD_ERR_ARG;
    if (movout > 0 && !dst) return fail(p, SFD_ERR_ARG, "movie destinations missing");
    p->movout = movout > 0 ? movout : 0;
    for (int o = 0; o < SFD_NOUT; o++) p->mov_dst[o] = p->movout ? dst[o] : nullptr;
    return SFD_OK;
}

extern "C" int sfd_set_gradfreqs(sfd_plan *p, const float *freqs, int nfreqs, int *info)
{
    if (!p || !freqs) return SFD_ERR_ARG;
    if (p->cfg.back_prop_type != 2) return fail(p, SFD_ERR_STATE, "the plan was not created with back_prop_type 2");
    if (nfreqs < 1 || nfreqs > MAXFREQ) return fail(p, SFD_ERR_ARG, "between 1 and 16 gradient frequencies");
    // src/assign_modeling_case.c:549-570
    float fmaxout = 0.0f;
    for (int j = 0; j < nfreqs; j++) {
        if (!std::isfinite(freqs[j]) || freqs[j] < 0.0f) return fail(p, SFD_ERR_ARG, "gradient frequencies must be >= 0");
        if (freqs[j] > fmaxout) fmaxout = freqs[j];
    }
    if (!(fmaxout > 0.0f)) return fail(p, SFD_ERR_ARG, "the highest gradient frequency must be positive");
    const float dt = p->cfg.dt;
    p->dtnyq = (int)std::ceil(0.0156 / fmaxout / dt);
    p->ntnyq = (p->cfg.tmax - p->cfg.tmin) / p->dtnyq + 1;
    p->df = (float)(1.0 / p->ntnyq / dt / p->dtnyq);
    for (int j = 0; j < nfreqs; j++) p->gradfreqsn[j] = std::floor(freqs[j] / p->df);
    p->nfreqs = nfreqs;
    p->have_dft = false;
    if (info) {
        info[0] = p->dtnyq;
        info[1] = p->ntnyq;
    }
    return SFD_OK;
}

extern "C" int sfd_get_gradient_q(sfd_plan *p, float *gtaup, float *gtaus)
{
    if (!p) return SFD_ERR_ARG;
    if (!p->a.grad[0]) return fail(p, SFD_ERR_STATE, "no gradient has been accumulated");
    int64_t n = (int64_t)p->g.nz * p->g.ny * p->g.nx;
    std::vector<double> h(n);
    float *outs[2] = {gtaup, gtaus};
    const int ids[2] = {GTAUP, GTAUS};
    for (int q = 0; q < 2; q++) {
        if (!outs[q]) continue;
        if (!p->a.grad[ids[q]]) {
            std::fill(outs[q], outs[q] + n, 0.0f);
            continue;
        }
        if (int rc_ = fetch_sum(p, p->a.grad[ids[q]], h.data(), n)) return rc_;
        for (int64_t i = 0; i < n; i++) outs[q][i] = (float)h[i];
    }
    return SFD_OK;
}

extern "C" int sfd_get_gradient(sfd_plan *p, int transform, float *g0, float *g1, float *g2)
{
    if (!p) return SFD_ERR_ARG;
    if (!p->a.grad[0]) return fail(p, SFD_ERR_STATE, "no gradient has been accumulated");
    int64_t n = (int64_t)p->g.nz * p->g.ny * p->g.nx;
    std::vector<double> gr(n), gM(n), gmu(n);
    if (int rc_ = fetch_sum(p, p->a.grad[GRHO], gr.data(), n)) return rc_;
    if (int rc_ = fetch_sum(p, p->a.grad[GM], gM.data(), n)) return rc_;
    if (int rc_ = fetch_sum(p, p->a.grad[GMU], gmu.data(), n)) return rc_;
    // the DFT gradient is already in the param_type's basis (no transf_grad)
    if (!transform || p->cfg.back_prop_type == 2) {
        for (int64_t i = 0; i < n; i++) {
            if (g0) g0[i] = (float)gM[i];
            if (g1) g1[i] = (float)gmu[i];
            if (g2) g2[i] = (float)gr[i];
        }
        return SFD_OK;
    }
    // src/calc_grad.c:975-1107
    const double dt = p->cfg.dt, dh = p->cfg.dh;
    const int pt = p->cfg.param_type;
    for (int64_t i = 0; i < n; i++) {
        double rho = 1.0 / p->hp[PRHO][i] * dt / dh;
        double M = p->hp[PM][i] * dh / dt, mu = p->hp[PMU][i] * dh / dt;
        double grho = gr[i] / dt, gm = gM[i] / dt, gs = gmu[i] / dt;
        if (pt == 0 || pt == 2) {
            grho += M / rho * gm;
            if (mu > 0) grho += mu / rho * gs;
        }
        if (pt == 0) {
            gm = 2.0 * std::sqrt(rho * M) * gm;
            gs = 2.0 * std::sqrt(rho * mu) * gs;
        } else if (pt == 2) {
            gm = 2.0 * std::sqrt(M / rho) * gm;
            gs = 2.0 * std::sqrt(mu / rho) * gs;
        }
        if (g0) g0[i] = (float)gm;
        if (g1) g1[i] = (float)gs;
        if (g2) g2[i] = (float)grho;
    }
    return SFD_OK;
}

extern "C" int sfd_residual_scale(sfd_plan *p, const sfd_shot *shot, const int *outsel, float *const *res)
{
    // src/residuals.c:452-568 in FP32 (par_scale 0).  For velocity outputs
    // the reference reads x, y and z from the first column of rec_pos
    // (:487-489); that index is kept.
    if (!p || !shot) return SFD_ERR_ARG;
    if (!p->model_set) return fail(p, SFD_ERR_STATE, "no model");
    const Grid &g = p->g;
    const int NT = p->cfg.nt, tmax = p->cfg.tmax;
    const float dh = p->cfg.dh, dt = p->cfg.dt;
    int64_t npar = (int64_t)g.nz * g.ny * g.nx;
    for (int o = 0; o < SFD_NOUT; o++) {
        if (!outsel || !outsel[o] || !res || !res[o]) continue;
        if (o != SFD_OUT_VX && o != SFD_OUT_VY && o != SFD_OUT_VZ && o != SFD_OUT_P) continue;
        for (int r = 0; r < shot->nrec; r++) {
            const float *rp = shot->rec_pos + 8 * r;
            int x, y, z;
            if (o == SFD_OUT_P) { x = (int)(rp[0] / dh); y = (int)(rp[1] / dh); z = (int)(rp[2] / dh); }
            else { x = (int)(rp[0] / dh); y = x; z = x; }
            int64_t pos = g.nd == 3 ? ((int64_t)x * g.ny + y) * g.nz + z : (int64_t)x * g.nz + z;
            if (pos < 0 || pos >= npar) return fail(p, SFD_ERR_ARG, "residual scaling index outside the model");
            float *row = res[o] + (int64_t)r * NT;
            if (o == SFD_OUT_P) {
                float parscal = -2.0 * (p->hp[PM][pos] - p->hp[PMU][pos]) * dh / dt;
                for (int t = 0; t < tmax; t++) row[t] *= parscal * dt;
            } else {
                int id = o == SFD_OUT_VX ? PRIP : (o == SFD_OUT_VY ? PRJP : PRKP);
                float parscal = 1.0 / p->hp[id][pos] * dh / dt;
                for (int t = 0; t < tmax; t++) row[t] *= 1.0 / parscal * dt;
            }
        }
    }
    return SFD_OK;
}

extern "C" int sfd_plan_info(const sfd_plan *p, int64_t *o)
{
    if (!p || !o) return SFD_ERR_ARG;
    o[0] = p->g.NZ; o[1] = p->g.NY; o[2] = p->g.NX; o[3] = p->g.nvol;
    o[4] = (int64_t)p->g.nz * p->g.ny * p->g.nx; o[5] = p->g.nbnd; o[6] = p->g.F; o[7] = p->cfg.tmax;
    return SFD_OK;
}

extern "C" int sfd_plan_uses_tma(const sfd_plan *p)
{
    if (!p) return SFD_ERR_ARG;
    if (cudaSetDevice(p->device) != cudaSuccess) return SFD_ERR_CUDA;
    return tma_ready(p->g, p->f) ? 1 : 0;
}

extern "C" int sfd_plan_kernel_family(const sfd_plan *p)
{
    if (!p) return SFD_ERR_ARG;
    if (!p->model_set) return 0;
    if (cudaSetDevice(p->device) != cudaSuccess) return SFD_ERR_CUDA;
    return stress_family(p->g, p->f);
}

extern "C" int64_t sfd_debug_copy(sfd_plan *p, int kind, int id, float *dst, int64_t cap)
{
    if (!p || !dst) return SFD_ERR_ARG;
    const Grid &g = p->g;
    const void *src = nullptr;
    int64_t n = 0;
    if (g.fhalf && kind >= 0 && kind <= 2) return fail(p, SFD_ERR_UNSUPPORTED, "wave fields are stored in FP16");
    if (g.rhalf && kind == 2) return fail(p, SFD_ERR_UNSUPPORTED, "memory variables are stored in FP16");
    if (kind == 0 && id >= 0 && id < NW) { src = p->f.w[id]; n = g.nvol; }
    else if (kind == 1 && id >= 0 && id < NW) { src = p->a.wr[id]; n = g.nvol; }
    else if (kind == 2 && id >= 0 && id < NR) { src = p->f.r[id]; n = g.nvol * g.L; }
    else if (kind == 3 && id >= 0 && id < NPAR) { src = p->f.p[id]; n = (int64_t)g.nz * g.ny * g.nx; }
    else if (kind == 4 && id >= 0 && id < 3) {
        src = id == 0 ? p->f.cx[0] : (id == 1 ? p->f.cy[0] : p->f.cz[0]);
        n = (int64_t)NC * std::max(2 * g.nab, 1);
    } else if (kind == 5 && id >= 0 && id < NPSI) { src = p->f.psi[id]; n = p->psi_size[id]; }
    else if ((kind == 6 || kind == 7) && id >= 0 && id < NW) { src = p->d_fw[kind - 6][id]; n = 2 * (int64_t)p->dft_nf * g.nvol; }
    else if ((kind == 8 || kind == 9) && id >= 0 && id < NR) {
        src = p->d_fr[kind - 8][id];
        n = 2 * (int64_t)p->dft_nf * g.nvol * g.L;
    }
    if (!src) return fail(p, SFD_ERR_ARG, "array not allocated");
    if (n > cap) return fail(p, SFD_ERR_ARG, "destination too small");
    cudaDeviceSynchronize();
    if (cudaMemcpy(dst, src, sizeof(float) * n, cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(p, SFD_ERR_CUDA, "copy failed");
    return n;
}

extern "C" int64_t sfd_debug_load(sfd_plan *p, int kind, int id, const float *src, int64_t n)
{
    if (!p || !src || n < 0) return SFD_ERR_ARG;
    if (!p->model_set) return fail(p, SFD_ERR_STATE, "sfd_set_model must be called first");
    const Grid &g = p->g;
    if (g.fhalf) return fail(p, SFD_ERR_UNSUPPORTED, "wave fields are stored in FP16");
    if (g.rhalf && kind == 2) return fail(p, SFD_ERR_UNSUPPORTED, "memory variables are stored in FP16");
    int rc;
    if (kind == 1 && (rc = alloc_adjoint(p))) return rc;
    void *dst = nullptr;
    int64_t cap = 0;
    if (kind == 0 && id >= 0 && id < NW) { dst = p->f.w[id]; cap = g.nvol; }
    else if (kind == 1 && id >= 0 && id < NW) { dst = p->a.wr[id]; cap = g.nvol; }
    else if (kind == 2 && id >= 0 && id < NR) { dst = p->f.r[id]; cap = g.nvol * g.L; }
    if (!dst) return fail(p, SFD_ERR_ARG, "array not allocated");
    if (n != cap) return fail(p, SFD_ERR_ARG, "size differs from the array's");
    cudaDeviceSynchronize();
    if (cudaMemcpy(dst, src, sizeof(float) * n, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(p, SFD_ERR_CUDA, "copy failed");
    return n;
}

extern "C" int sfd_debug_launch(sfd_plan *p, int which)
{
    if (!p) return SFD_ERR_ARG;
    if (!p->model_set) return fail(p, SFD_ERR_STATE, "sfd_set_model must be called first");
    cudaStream_t st = p->stream;
    p->g.nb = 1;
    const Grid &g = p->g;
    int rc;
    switch (which) {
    case 0: launch_update_v(g, p->f, st); break;
    case 1: launch_update_s(g, p->f, st); break;
    case 2:
        if (!g.freesurf) return fail(p, SFD_ERR_STATE, "the plan has no free surface");
        launch_surface(g, p->f, 1, st);
        break;
    case 3:
        if (!g.freesurf) return fail(p, SFD_ERR_STATE, "the plan has no free surface");
        if (g.nd == 21 || g.nd == 22) return fail(p, SFD_ERR_UNSUPPORTED, "no surface adjoint for this physics");
        if ((rc = alloc_adjoint(p))) return rc;
        launch_surface_adj(g, p->f, p->a, p->d_surf_q, st);
        break;
    default: return fail(p, SFD_ERR_ARG, "unknown kernel");
    }
    CKC(cudaGetLastError());
    CKC(cudaStreamSynchronize(st));
    return SFD_OK;
}

extern "C" float sfd_last_loop_ms(const sfd_plan *p) { return p ? p->last_ms : 0.0f; }

extern "C" int sfd_bench_kernels(sfd_plan *p, int nrep, float *out_ms)
{
    if (!p || !out_ms || nrep <= 0) return SFD_ERR_ARG;
    if (!p->model_set) return fail(p, SFD_ERR_STATE, "no model");
    cudaStream_t st = p->stream;
    p->g.nb = 1;
    const Grid &g = p->g;
    for (int k = 0; k < 4; k++) out_ms[k] = 0.0f;
    const bool fused = p->d_fsync && fused_shape(g).units;
    for (int which = 0; which < 4; which++) {
        if (which == 2 && !g.freesurf) continue;
        if (which == 3 && !fused) break;
        if (which == 3) CKC(cudaMemsetAsync(p->d_fsync, 0, sizeof(int) * (size_t)(1 + fused_shape(g).units), st));
        CKC(cudaEventRecord(p->ev0, st));
        for (int r = 0; r < nrep; r++) {
            if (which == 0) launch_update_v(g, p->f, st);
            else if (which == 1) launch_update_s(g, p->f, st);
            else if (which == 2) launch_surface(g, p->f, 1, st);
            else launch_fused_step(g, p->f, p->d_fsync, r, st);
        }
        CKC(cudaEventRecord(p->ev1, st));
        CKC(cudaEventSynchronize(p->ev1));
        CKC(cudaGetLastError());
        float ms = 0;
        cudaEventElapsedTime(&ms, p->ev0, p->ev1);
        out_ms[which] = ms / nrep;
    }
    if (fused && fused_take_status())
        return fail(p, SFD_ERR_CUDA, "a fused 3D step did not see its neighbours' velocities within its time bound");
    return SFD_OK;
}

extern "C" int sfd_plan_fused_step(const sfd_plan *p)
{
    if (!p) return SFD_ERR_ARG;
    return p->d_fsync && fused_shape(p->g).units ? 1 : 0;
}

// ------------------------------------------------------------ host-only
namespace {
int host_grid(const sfd_config *c, Grid &g)
{
    if (!c || (c->nd != 2 && c->nd != 3 && c->nd != 21 && c->nd != 22) || c->fdorder < 2 || c->fdorder > 12 ||
        c->fdorder % 2)
        return SFD_ERR_ARG;
    memset(&g, 0, sizeof g);
    g.nd = c->nd;
    g.F = c->fdorder / 2;
    g.nz = c->n[0];
    if (c->nd == 3) { g.ny = c->n[1]; g.nx = c->n[2]; }
    else { g.ny = 1; g.nx = c->n[1]; }
    if (g.nz <= 0 || g.ny <= 0 || g.nx <= 0) return SFD_ERR_ARG;
    g.NZ = g.nz + 2 * g.F;
    g.NX = g.nx + 2 * g.F;
    g.NY = c->nd == 3 ? g.ny + 2 * g.F : 1;
    return SFD_OK;
}
}  // namespace

extern "C" int sfd_host_transform(const sfd_config *cfg, const float *const *params, float *const *out)
{
    Grid g;
    int rc = host_grid(cfg, g);
    if (rc) return rc;
    std::vector<float> tmp[NPAR];
    std::string err;
    rc = transform_model(*cfg, g.nz, g.ny, g.nx, params, tmp, err);
    if (rc) return rc;
    for (int k = 0; k < NPAR; k++)
        if (out && out[k]) memcpy(out[k], tmp[k].data(), sizeof(float) * tmp[k].size());
    return SFD_OK;
}

extern "C" int sfd_host_point_cells(const sfd_config *cfg, const float *pos, int n, int stride, int64_t *cells)
{
    Grid g;
    int rc = host_grid(cfg, g);
    if (rc) return rc;
    double DH = literal9((double)cfg->dh);
    int kept = 0;
    for (int r = 0; r < n; r++) {
        int i, j, k;
        point_cell(pos + (int64_t)stride * r, DH, g.F, i, j, k);
        if (g.nd != 3) j = 0;
        if (i < g.F || i > g.NX - g.F - 1) { cells[r] = -1; continue; }
        cells[r] = ((int64_t)i * g.NY + j) * g.NZ + k;
        kept++;
    }
    return kept;
}

extern "C" int sfd_host_source_targets(int nd, int mask, int type, int *fields, float *div)
{
    return source_targets(nd, mask, type, fields, div);
}

extern "C" int sfd_host_cpml(const sfd_config *c, float *out)
{
    if (!c || !out || c->nab <= 0) return SFD_ERR_ARG;
    int n = 2 * c->nab;
    if (!cpml_profiles(c->npower, c->k_max_cpml, c->fpml, c->vppml, c->dh, c->dt, c->nab, out, out + n, out + 2 * n,
                       out + 3 * n, out + 4 * n, out + 5 * n))
        return SFD_ERR_ARG;
    return SFD_OK;
}
