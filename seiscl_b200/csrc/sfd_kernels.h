// sfd_kernels.h -- launchers of the FDTD kernels (host side).
#pragma once

#include <cuda_runtime.h>

#include "sfd_internal.h"

namespace sfd {

struct BndSlot {            // saved-boundary stores, by value
    void *p[NW];
    int nfield;
    int fields[NW];
};

void launch_update_v(const Grid &g, const Fields &f, cudaStream_t st);
bool launch_update_v_fast(const Grid &g, const Fields &f, cudaStream_t st);
bool launch_update_v_async(const Grid &g, const Fields &f, cudaStream_t st);
bool launch_update_s_fast(const Grid &g, const Fields &f, cudaStream_t st);
int fast3d_xchunk(const Grid &g);
bool launch_update_v_tma(const Grid &g, const Fields &f, cudaStream_t st);
bool launch_update_s_tma(const Grid &g, const Fields &f, cudaStream_t st);
bool tma_ready(const Grid &g, const Fields &f);  // the TMA kernels will run for this plan
int tma_take_status();      // 1 if a TMA stage of the last launches never arrived (and clears it)
// 3D stress-update family of a plan: 0 not 3D, 1 general, 2 register-blocked,
// 3 TMA-pipelined, 4 streaming, 5 4-cell vectorised
int stress_family(const Grid &g, const Fields &f);
// fold_surface: single-shot FP32 4-cell kernels may apply the free surface in
// the same launch (true returned: the caller skips launch_surface)
bool launch_update_s(const Grid &g, const Fields &f, cudaStream_t st, bool fold_surface = false);
// Fused 3D forward step (velocity, stress, free surface in one launch; see
// sfd_kernels.cu).  Work units = ntz x nty x nchunk; units = 0 when the plan's
// grid does not take it (sfd_config.kernels 6; 3D, 8th order, nz % 4 == 0,
// FP32 fields, L <= 3, nx >= 5).  nchunk = x planes (one unit per tile and
// plane).
struct FusedShape {
    int ntz, nty, nchunk;
    int64_t units;
};
FusedShape fused_shape(const Grid &g);
// sync: 1 + units ints (a ticket counter, one flag per unit), zeroed before
// step 0 of a run; t: the step's index in the run.  False: not launched.
bool launch_fused_step(const Grid &g, const Fields &f, int *sync, int t, cudaStream_t st);
int fused_take_status();    // 1 if a fused step's wait ran out (and clears it)
void launch_surface(const Grid &g, const Fields &f, int pdir, cudaStream_t st);
// 2D P-SV and acoustic forward: stress update, free surface, receivers of
// step tl.t and sources of step tl.tsrc in one launch (false: not 2D)
bool launch_update_s_step(const Grid &g, const Fields &f, const StepTail &tl, cudaStream_t st);
void launch_savebnd(const Grid &g, const Fields &f, const BndSlot &b, int prec, int64_t tofs, cudaStream_t st);
void launch_update_adj(const Grid &g, const Fields &f, const AdjFields &a, bool stress, int prec, cudaStream_t st);
void launch_surface_adj(const Grid &g, const Fields &f, const AdjFields &a, float *q, cudaStream_t st);
void launch_sources(const Grid &g, const Fields &f, const PointSet &s, const float *src, int nt_total, int t,
                    int pdir, cudaStream_t st);
void launch_record(const Grid &g, const Fields &f, const PointSet &r, float *out, int nt_total, int t,
                   unsigned outmask, cudaStream_t st);
void launch_residuals(const Grid &g, const AdjFields &a, const PointSet &r, const float *res, int nt_total, int t,
                      unsigned outmask, cudaStream_t st);

// instability detection: if any of the n values of a wave field (FP32, or
// FP16 when g.fhalf) is not finite, *first = min(*first, t)
void launch_finite_check(const Grid &g, const float *fld, int64_t n, int t, int *first, cudaStream_t st);
constexpr int FINITE_CHECK_EVERY = 64;   // time steps between checks

// movie snapshot: the physical cells of one wave field, divided by its
// storage scale, into dst [nx][ny][nz]
void launch_movie(const Grid &g, const float *fld, float inv_scale, float *dst, cudaStream_t st);

// checkpointed gradients: copies of wave fields / memory variables between
// their FP32 arrays and stores of the saved-boundary precision (FP16 stores
// scaled by powers of two)
struct PackSet {
    static constexpr int MAXARR = NW + NR;
    const void *src[MAXARR];
    void *dst[MAXARR];
    int64_t n[MAXARR];
    float scale[MAXARR];   // applied to each value on the way
    int narr;
};
void launch_pack(const PackSet &ps, int prec, bool unpack, cudaStream_t st, bool half_src = false);

// DFT gradient (sfd_dft.cu)
struct DftSet {             // variables transformed by one accumulation launch
    const float *v[NW + NR];
    float2 *f[NW + NR];
    int64_t n[NW + NR];     // elements of each variable (nvol, or L*nvol)
    int nvar, nf;
    float re[MAXFREQ], im[MAXFREQ];
};
void launch_savefreqs(const DftSet &d, cudaStream_t st);
struct GradDft {            // inputs of the per-cell assembly
    const float2 *fw[2][NW], *fr[2][NR];
    int nf, par_type;
    float w[MAXFREQ];       // angular frequency of each bin (FP32, as the reference forms it)
    float tausig[8];
    float al, ntnyq;
};
void launch_calc_grad(const Grid &g, const Fields &f, const AdjFields &a, const GradDft &d, cudaStream_t st);

}  // namespace sfd
