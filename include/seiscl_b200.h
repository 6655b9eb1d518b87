/*
 * seiscl_b200.h -- C ABI of the B200 staggered-grid FDTD engine.
 *
 * One plan = one grid, one physics case and one set of device buffers on the
 * current CUDA device.  All arrays crossing this boundary are plain host or
 * device pointers with sizes; nothing here depends on PyTorch.
 *
 * The entry points replace the single-device path of SeisCL:
 *   - sfd_plan_create/sfd_set_model replace readhdf5 + assign_modeling_case +
 *     Init_cst + Init_model + Init_CUDA (src/read_hdf5.c:554,
 *     src/assign_modeling_case.c:871, src/Init_cst.c:24, src/Init_model.c:40,
 *     src/Init_OpenCL.c:326);
 *   - sfd_forward replaces the forward half of
 *     int time_stepping(model*, device**, struct filenames)
 *     (src/time_stepping.c:692, loop at :747-860);
 *   - sfd_adjoint replaces its gradient half (src/time_stepping.c:862-972)
 *     for BACK_PROP_TYPE=1 (boundary-saving reconstruction) and
 *     BACK_PROP_TYPE=2 (DFT gradient, with calc_grad, src/calc_grad.c:376-960);
 *   - sfd_set_gradfreqs replaces the gradfreqs/gradfreqsn set-up
 *     (src/read_hdf5.c:546-549, src/assign_modeling_case.c:549-570);
 *   - sfd_get_gradient replaces transf_grad (src/calc_grad.c:975-1107) and
 *     the gradient output of src/writehdf5.c:262-275.
 *
 * Layout conventions are the reference host's (src/read_hdf5.c:606-625):
 * model parameters are [nx][ny][nz] (3D) or [nx][nz] (2D) with z fastest;
 * src_pos is [nsrc][5] = (x, y, z, srcid, type); rec_pos is [nrec][8] =
 * (x, y, z, srcid, recid, ...); src is [nsrc][NT]; a seismogram is
 * [nrec][NT] (src/writehdf5.c:209-220).
 *
 * Errors: every call returns 0 or a negative SFD_ERR_* code and leaves a
 * message in sfd_last_error(plan).  Nothing calls exit().  A plan must not
 * be used from two host threads at once; distinct plans are independent.
 */
#ifndef SEISCL_B200_H
#define SEISCL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SFD_OK 0
#define SFD_ERR_ARG (-1)       /* invalid argument or configuration */
#define SFD_ERR_CUDA (-2)      /* a CUDA call failed */
#define SFD_ERR_CFL (-3)       /* dt above the stability limit (assign_modeling_case.c:819) */
#define SFD_ERR_MEMORY (-4)    /* device memory exhausted or above the plan budget */
#define SFD_ERR_STATE (-5)     /* call out of order (e.g. adjoint without forward) */
#define SFD_ERR_UNSTABLE (-6)  /* non-finite wavefield detected (residuals.c:444-448) */
#define SFD_ERR_UNSUPPORTED (-7)

/* Output variable indices for the outsel/seis arrays. */
enum {
    SFD_OUT_VX = 0, SFD_OUT_VY, SFD_OUT_VZ, SFD_OUT_SXX, SFD_OUT_SYY, SFD_OUT_SZZ,
    SFD_OUT_SXY, SFD_OUT_SYZ, SFD_OUT_SXZ, SFD_OUT_P, SFD_NOUT
};

/* Storage precision of wave fields / saved boundaries (arithmetic is FP32). */
enum { SFD_PREC_FP32 = 0, SFD_PREC_FP16 = 1, SFD_PREC_BF16 = 2 };

/* The csts keys of SeisCL.py:23-30 that the single-device path reads
 * (src/read_hdf5.c:461-552). */
typedef struct sfd_config {
    int nd;            /* 2: P-SV, 3: 3D */
    int n[3];          /* N as in SeisCL: [NZ, NX] in 2D, [NZ, NY, NX] in 3D */
    int nt;            /* NT */
    int fdorder;       /* FDORDER: 2..12 */
    int maxrelerror;   /* MAXRELERROR: 0..4 */
    int L;             /* relaxation mechanisms (0 = elastic) */
    int freesurf;
    int abs_type;      /* 1: CPML, 2: Cerjan taper */
    int nab;
    float dt, dh, f0;
    float fl[8];       /* FL, L values */
    float vppml, fpml, npower, k_max_cpml, abpc;
    int tmin, tmax;    /* adjoint time window in steps; tmax <= 0 means NT */
    int param_type;    /* 0: vp,vs,rho  1: M,mu,rho  2: Ip,Is,rho */
    int restype;       /* 0: L2 (full gradient), 1: M only */
    int precision;     /* SFD_PREC_*: storage of the saved boundaries */
    int kernels;       /* 0: fastest measured: in 3D the 4-cell vectorised kernels where
                             they apply (8th order, nz a multiple of 4, L <= 3), else the
                             streaming ones; in 2D (P-SV, acoustic) modelling runs
                             without saved boundaries, DFT or movie, two launches per
                             step (the stress update carries the free surface, the
                             receivers and the next step's sources),
                          1: general one-thread-per-cell kernels only, one launch per
                             reference kernel,
                          2: register-blocked 3D kernels where available,
                          3: TMA-pipelined 3D velocity and stress updates,
                          4: streaming one-thread-per-cell 3D kernels (per-cell loads first),
                          5: 4-cell vectorised 3D kernels where they apply, else streaming,
                          6: as 0, and 3D modelling runs of one shot advance each step in
                             one fused launch (velocity, stress, memory variables, free
                             surface; sfd_plan_fused_step).  With 0 the single-shot 3D
                             modelling stress kernel applies the free surface itself. */
    int adjoint_reset_psi; /* 0: the adjoint continues with the forward run's CPML memory
                              (reference behaviour, src/clprogram.c:806-811); 1: it starts
                              from zeroed CPML memory.  With sources whose wave field is
                              large (forces), the carried-over memory dominates the adjoint
                              field inside the absorbing layers; 1 removes that. */
    int field_precision;   /* 0: wave fields and memory variables in FP32; 1: in FP16,
                              scaled by powers of two per shot (forward modelling of 3D
                              and 2D P-SV grids, L <= 3, and the forward and recomputed
                              runs of a checkpointed gradient, whose adjoint fields stay
                              FP32; arithmetic stays FP32); 2: memory variables alone
                              in FP16, times a power of two set per shot, wave fields
                              FP32 (3D viscoelastic forward modelling, FDORDER 8, NZ a
                              multiple of 4, kernels 0, batch 1).  No reference counterpart
                              in this form: the reference's FP16=2 mode also scales
                              by powers of two (src/assign_modeling_case.c:829-866). */
    int back_prop_type;    /* BACK_PROP_TYPE: 0 or 1 boundary-saving backpropagation,
                              2 DFT gradient at the frequencies of sfd_set_gradfreqs */
    int loop_graphs;       /* time loops as CUDA graphs: 0 (auto) for every loop but those
                              of the register-blocked and TMA 3D kernels, captured the
                              second time a loop runs unchanged (launches dominate small
                              grids; 1 % at 256^3), 1 always from the first run,
                              2 never.  A graph is captured on the first shot of a shape
                              and replayed while nothing its launches depend on changes.
                              No reference counterpart (launch mechanics). */
    int hout;              /* HOUT: also accumulate the approximate Hessian (2D; the
                              reference's 3D Hessian kernel does not compile,
                              update_adjv3D.cl:486, so 3D boundary-saving plans reject it) */
    int batch;             /* shots one launch advances together (0 or 1: one; P-SV,
                              acoustic and 3D with FP32 fields, kernels 0, 1, 4 or 5,
                              boundary-saving gradients).  The plan holds `batch` copies of every
                              per-shot array; sfd_forward_batch / sfd_adjoint_batch run
                              up to that many shots of the same model at once, each
                              launch covering all of them.  No reference counterpart
                              (the reference runs the shots of a group one by one,
                              time_stepping.c:705-722). */
    int checkpoint;        /* gradient recompute strategy: 0 saves the boundary shells and
                              backpropagates the forward field (BACK_PROP_TYPE 1, the
                              reference's); K > 0 keeps a snapshot of the whole forward
                              state every K steps and, during the adjoint, recomputes each
                              K-step segment forward from its snapshot, storing the wave
                              fields of every step of the segment: the adjoint reads the
                              forward field instead of reconstructing it (no boundary
                              store; memory: (nt/K) snapshots + K wave-field states, in
                              `precision`, CPML memory in FP32; with FP16 wave-field
                              storage the snapshots hold the FP16 fields as they are).
                              P-SV and 3D, batch 1.  The reference's INPUTRES checkpoint
                              (time_stepping.c:92-270) saves the final state and the
                              boundaries instead. */
} sfd_config;

typedef struct sfd_shot {
    int nsrc, nrec;
    const float *src_pos;  /* [nsrc][5] */
    const float *src;      /* [nsrc][NT] */
    const float *rec_pos;  /* [nrec][8] */
} sfd_shot;

typedef struct sfd_plan sfd_plan;

/* Create a plan for `cfg` on the current CUDA device.  No device memory is
 * allocated for the model until sfd_set_model. */
int sfd_plan_create(const sfd_config *cfg, sfd_plan **out);
void sfd_plan_destroy(sfd_plan *plan);
const char *sfd_last_error(const sfd_plan *plan);

/* Device bytes a plan for `cfg` allocates to run shots with up to nsrc
 * sources and nrec_sel = receivers x selected outputs: model, wave fields,
 * memory variables, CPML memory, constants and shot buffers; gradient != 0
 * adds what a gradient run holds (saved boundaries, adjoint fields and
 * gradient sums for back_prop_type 1; the transforms at nfreqs frequencies
 * for back_prop_type 2).  Computed from the configuration alone (no device
 * call), for admission control by a caller that shares one device among
 * many plans.  No counterpart in the reference. */
int sfd_footprint(const sfd_config *cfg, int gradient, int nsrc, int64_t nrec_sel, int nfreqs, int64_t *bytes);
/* Device bytes the plan holds now (every allocation it made and keeps). */
int64_t sfd_plan_device_bytes(const sfd_plan *plan);
/* Plans allocate from the current device's stream-ordered memory pool,
 * which keeps freed memory for the next plan; this returns what no plan
 * holds to the device (synchronises the device). */
int sfd_release_memory(void);
/* Free and total memory of the current device (cudaMemGetInfo). */
int sfd_device_memory(int64_t *free_bytes, int64_t *total_bytes);
/* Host-only self-check of the cache that keeps the 3D TMA kernels' tensor
 * maps between launches: `nthreads` threads make `iters` lookups each over
 * more keys than it holds and verify every value they copy out.  Returns the
 * number of bad copies (0 = sound).  Needs no device.  No counterpart in the
 * reference (which has no host state shared between threads). */
int64_t sfd_selftest_cache(int nthreads, int iters);

/* Upload the model.  params = {vp, vs, rho} (param_type 0), plus {taup, taus}
 * when L > 0, each a host array of nz*ny*nx floats in [nx][ny][nz] order.
 * vs may be NULL for zero shear.  Applies the reference transforms
 * (assign_modeling_case.c:305-535) and the CFL check (:730-827). */
int sfd_set_model(sfd_plan *plan, const float *const *params);

/* Bit t (t = 0..3) for each source type and bit 4 for type 100 over the
 * whole acquisition (automatic_kernels.c:416-437 scans all shots). */
int sfd_source_type_mask(const float *src_pos, int nsrc_all);

/* Forward modelling of one shot (time_stepping.c:747-835).  outsel[SFD_NOUT]
 * selects the recorded variables; seis[k] receives [nrec][NT] floats for each
 * selected k (host pointers).  save_boundaries != 0 keeps the boundary shells
 * and final state on the device for a following sfd_adjoint.  stream may be
 * NULL (the plan's own stream). */
int sfd_forward(sfd_plan *plan, const sfd_shot *shot, int srctype_mask, const int *outsel,
                float *const *seis, int save_boundaries, void *stream);

/* Adjoint of the shot last run by sfd_forward(save_boundaries=1):
 * residuals[k] are [nrec][NT] host arrays already scaled as adjoint sources
 * (see sfd_residual_scale); gradients accumulate in FP64 on the device.
 * With back_prop_type 2 the adjoint runs from zeroed fields without
 * reconstructing the forward field (src/time_stepping.c:862-972), its
 * transforms are taken at the forward's sampling times, and the shot's
 * gradient is assembled from both (calc_grad, src/calc_grad.c:376-960).
 * Returns SFD_ERR_UNSUPPORTED for a plan with a free surface whose model has
 * mu = 0 on the top row (the free-surface adjoint divides by mu there). */
int sfd_adjoint(sfd_plan *plan, const sfd_shot *shot, int srctype_mask, const int *outsel,
                const float *const *residuals, void *stream);

/* Zero the gradient accumulators (gradinit, automatic_kernels.c:840-930). */
int sfd_zero_gradient(sfd_plan *plan);

/* Gradients [nx][ny][nz] as floats.  back_prop_type 1: transformed
 * (transform=1: gradvp, gradvs, gradrho for param_type 0, calc_grad.c:975-1107)
 * or raw (transform=0: grad M, grad mu, grad rho of the stored parameters).
 * back_prop_type 2: the accumulated DFT gradient of the param_type's three
 * parameters, which calc_grad already expresses in that parametrisation (the
 * reference applies no transf_grad there, time_stepping.c:976-1002);
 * `transform` is ignored. */
int sfd_get_gradient(sfd_plan *plan, int transform, float *g0, float *g1, float *g2);

/* Movie (MOVOUT, time_stepping.c:272-350): every `movout` steps, the
 * physical cells of each wave field selected in a run's outsel (the
 * acoustic model's pressure included) are copied to dst[k] (k an SFD_OUT_*
 * index), a host array of [NT/movout][nx][ny][nz] floats: snapshot
 * (t+1)/movout - 1 after forward step t when (t+1) % movout == 0.  A
 * boundary-saving gradient run films its adjoint instead -- the
 * reconstructed forward field after adjoint step t when t % movout == 0,
 * into the same slot formula (:927-929).  movout <= 0 turns it off.  The
 * destinations must stay valid until the run that fills them returns. */
int sfd_set_movie(sfd_plan *plan, int movout, float *const *dst);

/* ---- DFT gradient (BACK_PROP_TYPE=2) ----
 *
 * Frequencies (Hz, 1..16 values) of the DFT gradient of a plan created with
 * back_prop_type 2: DTNYQ = ceil(0.0156 / max(freqs) / dt), NTNYQ =
 * (tmax - tmin) / DTNYQ + 1, df = 1 / (NTNYQ dt DTNYQ), and each frequency
 * is taken at bin floor(f / df) (src/assign_modeling_case.c:549-570).  A
 * bin of 0 Hz makes calc_grad divide by zero, as in the reference.  Device
 * memory for the transforms (2 x nfreqs x 8 bytes per wave-field cell, and
 * per memory-variable cell) is allocated by the next gradient forward run.
 * info (may be NULL) receives DTNYQ, NTNYQ. */
int sfd_set_gradfreqs(sfd_plan *plan, const float *freqs, int nfreqs, int *info);

/* Approximate Hessian (HOUT) accumulated with the gradient: out[0..4] =
 * H of the param_type's first and second parameters, rho, taup, taus
 * (entries may be NULL).  Boundary-saving plans: transform=1 applies
 * transf_grad's chain rule without the division by dt
 * (src/calc_grad.c:1004-1090), transform=0 gives the raw HM, Hmu, Hrho
 * (update_adjs2D.cl:453-470; Hrho stays 0 there as in the reference, whose
 * line is commented out).  DFT plans: calc_grad's 2D Hessian
 * (src/calc_grad.c:838-905), zero in 3D as in the reference. */
int sfd_get_hessian(sfd_plan *plan, int transform, float *const *out);

/* Gradients of the relaxation parameters taup and taus [nx][ny][nz], filled
 * by the DFT gradient of viscoelastic plans (src/calc_grad.c:729-739); zero
 * otherwise, as the reference leaves them. */
int sfd_get_gradient_q(sfd_plan *plan, float *gtaup, float *gtaus);

/* res_scale (residuals.c:452-568): scale residuals in place into adjoint
 * sources.  res[k] are [nrec][NT] host arrays for the selected outputs. */
int sfd_residual_scale(sfd_plan *plan, const sfd_shot *shot, const int *outsel, float *const *res);

/* Batched shots (cfg.batch > 1): nshot <= batch shots
 * of the plan's model advance together, each launch of the time loop
 * covering all of them.  Shot s works on copy s of every per-shot array, so
 * each shot's result is the one sfd_forward gives it alone.  seis[o] (and
 * residuals[o]) hold the traces of all shots in shot order, [sum nrec][NT];
 * the adjoint must follow a forward of the same shots.  The gradient
 * accumulates per shot copy and sfd_get_gradient returns the sum over
 * copies (in copy order).  sfd_forward / sfd_adjoint are the one-shot case. */
int sfd_forward_batch(sfd_plan *plan, int nshot, const sfd_shot *shots, int mask, const int *outsel,
                      float *const *seis, int save_boundaries, void *stream);
int sfd_adjoint_batch(sfd_plan *plan, int nshot, const sfd_shot *shots, int mask, const int *outsel,
                      const float *const *residuals, void *stream);

/* ---- forward modelling without allocation ----
 *
 * This entry point has no counterpart in the reference; SeisCL always
 * allocates its buffers per run.  It is for callers that cannot call
 * cudaMalloc when they run a shot -- a serving process that reserved its
 * device memory budget at start-up and must not grow it per request, or a
 * host application whose own allocator owns the device.  It runs the same
 * forward time loop as sfd_forward, but keeps its working memory (wave
 * fields, memory variables, CPML memory, source/receiver maps) in one fixed
 * array of SFD_NOALLOC_SCRATCH_BYTES compiled into the library, which every
 * GPU that loads the library holds until the process exits.  It calls no
 * cudaMalloc, cudaFree or other allocating routine.
 *
 * - The plan must hold a model (sfd_set_model, done beforehand) and its
 *   device must be current.  The shot's working memory must fit in the
 *   array; a larger grid is rejected with SFD_ERR_MEMORY and a message
 *   naming the size it needed.
 * - Inputs and outputs are caller-owned DEVICE buffers: src_pos [nsrc][5],
 *   src [nsrc][NT], rec_pos [nrec][8], and seis [nsel][nrec][NT] for the
 *   nsel selected outputs in SFD_OUT_* order.
 * - The first call on a device looks up the array's device address
 *   (cudaGetSymbolAddress) with that device current; make that first call
 *   before any stream capture.  Under CUDA's lazy module loading (the
 *   default since CUDA 12.2) that first call is also when the driver loads
 *   this part of the library onto the device and commits the array's
 *   SFD_NOALLOC_SCRATCH_BYTES: a caller that reserves the rest of the
 *   device afterwards should make its first call at start-up, before it
 *   takes that reservation.  Later calls commit nothing.
 * - Every call on a device shares the one array.  Each call clears what must
 *   start at zero, but calls that overlap on the GPU (different streams or
 *   threads at once) race on it: issue them one after another.
 * - The call returns after the shot has finished on `stream` (or the plan's
 *   stream when NULL). */
#define SFD_NOALLOC_SCRATCH_BYTES (16u << 20)
int sfd_forward_noalloc(sfd_plan *plan, const float *src_pos, const float *src, int nsrc, const float *rec_pos,
                        int nrec, int srctype_mask, const int *outsel, float *seis, void *stream);

/* ---- host-only set-up (no device needed) ---- */

/* The 14 transformed parameter arrays of sfd_set_model (M, mu, rho_b, taup,
 * taus, rip, rjp, rkp, muipkp, muipjp, mujpkp, tausipkp, tausipjp, tausjpkp;
 * src/assign_modeling_case.c:305-535), each nz*ny*nx floats.  out[k] may be
 * NULL.  Returns SFD_ERR_CFL when dt is above the stability limit. */
int sfd_host_transform(const sfd_config *cfg, const float *const *params, float *const *out);

/* Padded linear cell index ((i*NYp + j)*NZp + k) of n source or receiver rows
 * of `stride` floats, i = (int)(x/DH) + FDOH as the generated kernels compute
 * it (src/automatic_kernels.c:95-105, 501-511); -1 for rows dropped because
 * i is outside [FDOH, NXp-FDOH-1].  Returns the number kept. */
int sfd_host_point_cells(const sfd_config *cfg, const float *pos, int n, int stride, int64_t *cells);

/* Wave fields fed by a source of `type` under the acquisition's type mask
 * (src/automatic_kernels.c:416-614): fields[3] receive indices in
 * SFD_OUT_VX..SFD_OUT_SXZ order, div[3] the divisor (0 = none). */
int sfd_host_source_targets(int nd, int mask, int type, int *fields, float *div);

/* CPML profiles of one axis: 6 arrays of 2*nab floats (K, a, b, K_half,
 * a_half, b_half; src/third_party/SOFI3D/CPML_COEFF.c:26-200). */
int sfd_host_cpml(const sfd_config *cfg, float *out);

/* Introspection for tests: padded dims, counts, boundary cells. */
int sfd_plan_info(const sfd_plan *plan, int64_t *out8);

/* 1 when the plan's 3D updates run on the TMA-pipelined kernels (kernels = 3,
 * 8th order, nz a multiple of 4), 0 otherwise; negative on error.  No
 * counterpart in the reference (kernel selection is internal to this engine). */
int sfd_plan_uses_tma(const sfd_plan *plan);

/* Kernel family of the plan's 3D stress update (after sfd_set_model): 0 not
 * 3D, 1 general, 2 register-blocked, 3 TMA-pipelined, 4 streaming, 5 4-cell
 * vectorised; negative on error.  No counterpart in the reference. */
int sfd_plan_kernel_family(const sfd_plan *plan);

/* Copy a device array of the plan to the host (tests): kind 0 wave field,
 * 1 adjoint wave field, 2 memory variable, 3 transformed parameter,
 * 4 CPML constants of axis id (6 arrays of 2*nab), 5 psi array, 6/7 forward/
 * adjoint DFT of wave field id and 8/9 of memory variable id (interleaved
 * complex, [nfreqs][(L)][padded cells]).  Returns the number of floats
 * written, or a negative error. */
int64_t sfd_debug_copy(sfd_plan *plan, int kind, int id, float *dst, int64_t cap);

/* Tests of single kernels (adjoint dot products): copy n host floats into a
 * device array (kinds 0-2 of sfd_debug_copy; n must be the array's size;
 * kind 1 allocates the adjoint fields), and run one kernel on the plan's
 * arrays -- which 0 velocity update, 1 stress update, 2 free surface
 * (forward), 3 free-surface adjoint on the adjoint fields (the reference's
 * surface_adj, src/surface2D_adj.cl:35-148, src/surface3D_adj.cl:29-116) --
 * returning after it finished.  No counterpart in the reference. */
int64_t sfd_debug_load(sfd_plan *plan, int kind, int id, const float *src, int64_t n);
int sfd_debug_launch(sfd_plan *plan, int which);

/* Kernel timing for benchmarks: runs the velocity update, the stress update,
 * (with a free surface) the surface kernel and (where the plan has it) the
 * fused 3D step `nrep` times each on the plan's stream, bracketed by CUDA
 * events, and writes the mean milliseconds per launch to out_ms[0..3] (0 for
 * a kernel not run).  The wave fields are modified. */
int sfd_bench_kernels(sfd_plan *plan, int nrep, float *out_ms);

/* 1 when the plan's 3D modelling runs (sfd_forward without saved boundaries,
 * DFT or movie, one shot) advance each time step in one fused launch --
 * velocity, stress, memory variables and free surface (kernels 6; 3D, 8th
 * order, nz a multiple of 4, FP32 fields, L <= 3, batch 1) -- else 0.  No
 * counterpart in the reference, which launches update_v and update_s
 * separately (src/time_stepping.c:426-479). */
int sfd_plan_fused_step(const sfd_plan *plan);

/* Milliseconds spent in the device time loop of the last sfd_forward /
 * sfd_adjoint (CUDA events on the plan's stream). */
float sfd_last_loop_ms(const sfd_plan *plan);

#ifdef __cplusplus
}
#endif
#endif
