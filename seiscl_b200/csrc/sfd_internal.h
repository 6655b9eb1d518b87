// sfd_internal.h -- plan state and kernel argument blocks of the B200 FDTD
// engine (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <utility>
#include <vector>

#include "seiscl_b200.h"

namespace sfd {

// wave fields; the order doubles as the bit layout of masks
enum { VX, VY, VZ, SXX, SYY, SZZ, SXY, SYZ, SXZ, NW };
// memory variables
enum { RXX, RYY, RZZ, RXY, RYZ, RXZ, NR };
// CPML memory arrays psi_<field>_<axis>
enum {
    PVX_X, PVY_X, PVZ_X, PVX_Y, PVY_Y, PVZ_Y, PVX_Z, PVY_Z, PVZ_Z,
    PSXX_X, PSXY_X, PSXZ_X, PSXY_Y, PSYY_Y, PSYZ_Y, PSXZ_Z, PSYZ_Z, PSZZ_Z, NPSI
};
// transformed parameters
enum {
    PM, PMU, PRHO, PTAUP, PTAUS, PRIP, PRJP, PRKP, PMUIPKP, PMUIPJP, PMUJPKP,
    PTAUSIPKP, PTAUSIPJP, PTAUSJPKP, NPAR
};
// CPML constants per axis
enum { CK, CA, CB, CKH, CAH, CBH, NC };
// CPML memory arrays share one allocation; each starts on a 256-byte
// boundary so the 4-cell kernels can move them with 128-bit accesses
inline int64_t psi_span(int64_t n) { return (n + 63) & ~(int64_t)63; }
// gradient accumulators; taup and taus are filled by the DFT gradient only
enum { GRHO, GM, GMU, GTAUP, GTAUS, NG };
constexpr int MAXFREQ = 16;   // DFT gradient frequencies per plan

// Stored value = field x w[field]: 1 for FP32 storage; powers of two for
// FP16 storage (set per shot from the source amplitude).
struct WScale {
    float w[NW];
};

// Everything a stencil kernel needs, passed by value (a few hundred bytes of
// kernel parameter space).
struct Grid {
    int nd;                 // 2 or 3
    int F;                  // stencil half width
    int nz, ny, nx;         // physical sizes (ny = 1 in 2D)
    int NZ, NY, NX;         // padded sizes
    int nab, L, freesurf, abs_type;
    int64_t nvol;           // padded cell count
    float hc[6];            // FD coefficients
    float dt, dt2;          // dt and dt/2
    float eta[8];           // 2 pi FL dt
    float eta_b[8], eta_c[8];  // 1/(1+eta/2) and 1-eta/2, FP32 as the kernels would form them
    float inv_dt;           // 1/dt rounded to FP32
    int fhalf;              // 1: wave fields and memory variables stored in FP16 (3D forward)
    int rhalf;              // 1: memory variables alone stored in FP16, times rsc (3D forward)
    float rsc, rsci;        // that scale (a power of two, set per shot) and its inverse
    WScale ws;              // storage scale per wave field (all 1 for FP32)
    float bsc[NW], bsci[NW];  // saved-boundary store scale per wave field and its inverse
                              // (powers of two for FP16 stores, 1 otherwise)
    int nbnd;               // saved-boundary cells per field per step
    int restype;
    int kernels;            // 0: register-blocked 3D kernels where available, 1: general only
    int fused;              // 1: 3D modelling runs take the fused step kernel (sfd_config.kernels 6)
    int vasync;             // 1: 3D single-shot velocity updates take the cp.async-staged kernel (kernels 7)
    int bp2;                // adjoint kernels: 1 for the DFT gradient (no reconstruction,
                            // boundary injection or on-the-fly gradient)
    int hout;               // accumulate the approximate Hessian
    int ckpt;               // adjoint kernels: the forward field comes from a.fwd (checkpointed
                            // gradient), not from backpropagation and boundary injection
    // batched shots (2D): the launch covers nb shots, blockIdx.z = shot; shot
    // b works on copy b of each per-shot array, these strides apart
    int nb;
    int64_t sb_w, sb_r;     // wave fields (nvol), memory variables (L nvol)
    int64_t sb_psi;         // the CPML block (floats)
    int64_t sb_g;           // gradient / Hessian sums (physical cells)
    int64_t sb_q;           // surface-adjoint scratch (nx ny)
    int64_t sb_bnd;         // saved-boundary store of one field (bytes)
};

struct Fields {
    float *w[NW];
    float *r[NR];           // [L][nvol]
    float *psi[NPSI];
    const float *p[NPAR];
    const float *cx[NC], *cy[NC], *cz[NC];
    const float *kinv[3][2];  // 1/K and 1/K_half per axis (x, y, z), FP32-rounded on the host
    const float *taper;
};

struct AdjFields {
    float *wr[NW];
    float *rr[NR];
    double *grad[NG];
    double *hess[NG];       // approximate Hessian (HOUT), same layout as grad
    const void *bnd[NW];    // slice t-1 of the saved boundaries
    const void *fwd[NW];    // checkpointed gradients: the forward wave fields of the step
};

struct PointSet {           // sources or receivers of one shot, device side
    int n;
    const int64_t *cell;    // padded linear index, -1 when dropped
    const int *ntarget;     // sources: number of fed fields
    const int *field;       // sources: [n][3] wave-field ids
    const float *div;       // sources: [n][3] divisor (0 = none)
    const int *kz;          // z cell index (free-surface adjoint skip)
};

struct FusedSync {          // fused 3D step: work-unit tickets and flags
    unsigned *ticket;       // CTAs of the run so far (zeroed before step 0; wraps)
    int *flags;             // per unit: last step (+1) whose velocities are done
    unsigned base;          // tickets taken by the run's earlier steps (mod 2^32)
    int ntz, nty;           // tiles along z and y
    int units;              // work units of one step
};

struct StepTail {           // fused 2D forward step: the work of its last block
    int *ticket;            // blocks finished; 0 between launches
    PointSet rec;           // receivers recorded at step t into out [nsel][nrec][nt_total]
    float *out;
    unsigned outmask;
    int t;
    PointSet src;           // sources injected for step tsrc (< 0: none)
    const float *stf;       // [nsrc][nt_total]
    int tsrc;
    int nt_total;
};

}  // namespace sfd

struct sfd_plan {
    sfd_config cfg;
    sfd::Grid g;
    int device;
    cudaStream_t stream;
    bool own_stream;
    std::string err;
    double DH_lit;          // the reference's "%9.9f" dh literal
    double DT_lit;
    // host copies of the transformed parameters (for transf_grad, res_scale)
    std::vector<float> hp[sfd::NPAR];
    bool model_set;
    // device memory
    std::vector<std::pair<void *, size_t>> allocs;   // owned by the plan
    int64_t dev_bytes;      // device bytes the plan holds
    sfd::Fields f;
    sfd::AdjFields a;
    float *d_psi_all;
    int64_t psi_size[sfd::NPSI];
    void *d_bnd[sfd::NW];   // [nt][nbnd]
    size_t bnd_elem;        // bytes per stored value
    bool have_forward;      // boundaries of a forward run are on the device
    // per-shot device buffers (grown on demand)
    int cap_src, cap_rec;
    int64_t *d_src_cell, *d_rec_cell;
    int *d_src_nt, *d_src_field, *d_src_kz;
    float *d_src_div, *d_src, *d_seis, *d_res;
    float *d_surf_q;        // surface-adjoint scratch [nx][ny]
    int *d_ticket;          // fused 2D steps: block counter of the stress launch
    int *d_unstable;        // first checked step with a non-finite wave field (INT_MAX: none)
    int *d_fsync;           // fused 3D step: ticket counter + one flag per work unit
    // checkpointed gradients (cfg.checkpoint = K > 0)
    char *d_snap;           // [nseg] snapshots: wave fields, memory variables (store type; FP16 wave-field
                            // storage: the FP16 fields as they are), CPML (FP32)
    char *d_seg;            // [K][wave fields] of the segment being backpropagated (store type)
    float *d_psi_adj;       // the adjoint's CPML memory
    // FP16 wave-field storage: the parameters the adjoint reads, without the
    // power-of-two scalings of the moduli and buoyancies (the adjoint fields
    // are FP32 and unscaled); padj[k] is f.p[k] for the unscaled ones
    float *d_padj;
    const float *padj[sfd::NPAR];
    bool padj_valid;
    size_t snap_bytes, seg_bytes;
    int nseg;
    int batch;              // copies of the per-shot arrays (shots per launch)
    int fwd_nb;             // shots of the forward run whose boundaries are saved
    cudaEvent_t ev0, ev1;
    int kshift;             // FP16 storage: log2 ratio of velocity to stress scales
    int bshift;             // the same ratio for FP16 saved boundaries (set whatever the storage)
    bool surf_mu_zero;      // mu is zero somewhere on the top row (the free-surface adjoint is undefined)
    float last_ms;
    // DFT gradient (back_prop_type 2, src/assign_modeling_case.c:549-570)
    int nfreqs, dtnyq, ntnyq;
    float df;
    float gradfreqsn[sfd::MAXFREQ];
    float2 *d_fw[2][sfd::NW];   // [forward, adjoint] transforms [nfreqs][nvol]
    float2 *d_fr[2][sfd::NR];   // memory variables [nfreqs][L][nvol]
    int dft_nf;                 // frequencies the transform buffers were allocated for
    bool have_dft;              // a forward run left its transforms on the device
    // movie (MOVOUT): snapshots of the selected wave fields every movout steps
    int movout;
    float *mov_dst[SFD_NOUT];   // host destinations, [NT/movout][nx][ny][nz] each
    float *d_mov;               // device staging, [nsel][NT/movout][nx][ny][nz]
    size_t mov_cap;             // floats allocated at d_mov
    // time loops captured as CUDA graphs (small grids, where launches dominate);
    // each is reused while its key -- every value its launches bake in -- is unchanged
    struct LoopGraph {
        cudaGraphExec_t exec = nullptr;
        std::string key;
        std::string seen;   // key of the last loop run without a graph
    } gfwd, gadj;
};
