/*
 * fdo.h -- CPU oracle for the staggered-grid FDTD forward and adjoint path.
 *
 * TEST INFRASTRUCTURE ONLY.  This oracle is the checker for the CUDA product
 * path in seiscl_b200/.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load it.  The product never calls into it.
 *
 * It is a plain-C restatement of SeisCL's single-device algorithm:
 *   - the time loop of src/time_stepping.c:747-940 (forward then adjoint),
 *   - the generated kernels of src/automatic_kernels.c (sources 394-629,
 *     varsout 22-219, residuals 631-836),
 *   - the stencil kernels src/update_{v,s}{2D,3D}.cl, src/surface{2D,3D}.cl,
 *     src/update_adj{v,s}{2D,3D}.cl, src/surface2D_adj.cl, src/savebnd{2D,3D}.cl
 *     and src/header_injectbnd.cl,
 *   - the host transforms of src/assign_modeling_case.c:305-660 and the
 *     coefficient code of src/third_party/SOFI3D/{holbergcoeff,CPML_COEFF}.c.
 *
 * The restatement keeps the reference's mixed float/double expression trees
 * (the reference passes HC1..HC6, DT, DT2 and DH as double literals printed
 * with "%9.9f", src/clprogram.c:493-520), so that a build with
 * -ffp-contract=off reproduces the reference kernels compiled as C bit for
 * bit.  That is how the oracle is pinned: oracle/ref_glue.c compiles the
 * reference kernel sources in place and tests/test_oracle_pin.py compares.
 *
 * Sizes are runtime values here (the reference fixes them at compile time).
 *
 * Layout (identical to the reference, src/update_v2D.cl:98-99,
 * src/update_v3D.cl:128-129):
 *   wave fields   padded  [NXp][NYp][NZp], z fastest, NXp = nx + 2*fdoh ...
 *   memory vars   [L][NXp][NYp][NZp]
 *   parameters    unpadded [nx][ny][nz]
 *   CPML psi      x-type [2*nab][ny][nz], y-type [nx][2*nab][nz],
 *                 z-type [nx][ny][2*nab]
 * In 2D, ny = NYp = 1.
 */
#ifndef SEISCL_ORACLE_FDO_H
#define SEISCL_ORACLE_FDO_H

#include <stdint.h>

/* FDO_FP64: the FP64 build of the same restatement (every float of the
 * interface, the state and the arithmetic becomes double), the double
 * precision reference that FP32 and FP16-storage results are measured
 * against.  Files include this header after their system headers. */
#ifdef FDO_FP64
#define float double
#define sqrtf sqrt
#define powf pow
#define fabsf fabs
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* wave fields */
enum { W_VX, W_VY, W_VZ, W_SXX, W_SYY, W_SZZ, W_SXY, W_SYZ, W_SXZ, W_N };
/* memory variables (viscoelastic) */
enum { R_XX, R_YY, R_ZZ, R_XY, R_YZ, R_XZ, R_N };
/* CPML memory arrays, named after the reference (psi_<field>_<axis>) */
enum {
    PS_VX_X, PS_VY_X, PS_VZ_X, PS_VX_Y, PS_VY_Y, PS_VZ_Y, PS_VX_Z, PS_VY_Z, PS_VZ_Z,
    PS_SXX_X, PS_SXY_X, PS_SXZ_X, PS_SXY_Y, PS_SYY_Y, PS_SYZ_Y, PS_SXZ_Z, PS_SYZ_Z,
    PS_SZZ_Z, PS_N
};
/* transformed material parameters */
enum {
    P_M, P_MU, P_RHO, P_TAUP, P_TAUS, P_RIP, P_RJP, P_RKP, P_MUIPKP, P_MUIPJP,
    P_MUJPKP, P_TAUSIPKP, P_TAUSIPJP, P_TAUSJPKP, P_N
};
/* CPML / taper constants: per axis x,y,z: K, a, b, K_half, a_half, b_half */
enum { C_K, C_A, C_B, C_KH, C_AH, C_BH, C_N };
/* gradient outputs (per-parameter, in the reference's M/mu/rho basis; the
 * DFT gradient also fills taup and taus) */
enum { G_RHO, G_M, G_MU, G_TAUP, G_TAUS, G_N };
#define FDO_MAXFREQ 16

typedef struct fdo_cfg {
    int nd;            /* 2 (P-SV) or 3 */
    int nz, ny, nx;    /* physical grid (absorbing layers included); ny = 1 in 2D */
    int fdorder, fdoh; /* stencil order and half width */
    int maxrelerror;   /* Holberg table row */
    int nab, freesurf, abs_type, L;
    int nt;            /* number of time steps NT */
    int tmin, tmax;    /* time window of the adjoint loop (steps) */
    float dt, dh;
    float f0;          /* relaxation centre frequency */
    float fl[8];       /* relaxation frequencies FL */
    float vppml, fpml, npower, k_max_cpml, abpc;
    int param_type;    /* 0: vp,vs,rho  1: M,mu,rho  2: Ip,Is,rho */
    int restype;       /* 0 or 1 (src/update_adjs2D.cl:441-470) */
    int back_prop_type;/* 1: boundary-saving backpropagation, 2: DFT gradient */
    int nfreqs;        /* DFT gradient: number of frequencies (<= FDO_MAXFREQ) */
    float gradfreqs[FDO_MAXFREQ];  /* DFT gradient frequencies (Hz) */
    int hout;          /* HOUT: accumulate the approximate Hessian (2D) */
} fdo_cfg;

/* One shot: sources and receivers, the reference's src_pos [nsrc][5] and
 * rec_pos [nrec][8] row layout (src/read_hdf5.c:307-459). */
typedef struct fdo_shot {
    int nsrc, nrec;
    const float *src_pos;  /* nsrc*5 */
    const float *src;      /* nsrc*NT */
    const float *rec_pos;  /* nrec*8 */
} fdo_shot;

/* Output selection: one flag per recorded variable */
enum { O_VX, O_VY, O_VZ, O_SXX, O_SYY, O_SZZ, O_SXY, O_SYZ, O_SXZ, O_P, O_N };

/* Kernel table: the port (fdo_port.c) and the in-place reference build
 * (ref_glue.c) each provide one. */
struct fdo_state;
typedef struct fdo_kernels {
    void (*update_v)(struct fdo_state *s);
    void (*update_s)(struct fdo_state *s);
    void (*surface)(struct fdo_state *s, int pdir);
    void (*update_adjv)(struct fdo_state *s);
    void (*update_adjs)(struct fdo_state *s);
    void (*surface_adj)(struct fdo_state *s);
    void (*savebnd)(struct fdo_state *s, int t);
    const char *name;
} fdo_kernels;

typedef struct fdo_state {
    fdo_cfg c;
    int NZp, NYp, NXp;     /* padded sizes */
    int64_t nvol;          /* padded cell count */
    int64_t npar;          /* physical cell count */
    int nbnd;              /* saved-boundary cells per field per step */
    double hc[7];          /* FD coefficients as the reference's literals */
    double DT, DT2, DH;    /* the reference's "%9.9f" literals */
    float *w[W_N];         /* forward wave fields */
    float *r[R_N];         /* forward memory variables */
    float *wr[W_N];        /* adjoint wave fields */
    float *rr[R_N];        /* adjoint memory variables */
    float *psi[PS_N];
    float *p[P_N];
    float *cx[C_N], *cy[C_N], *cz[C_N];
    float *taper;
    float *eta;
    float *grad[G_N];      /* float accumulators as in the reference */
    float *hess[G_N];      /* approximate Hessian (HOUT), same layout */
    float *bnd[W_N];       /* [nt][nbnd] per wave field */
    float *bnd_cur[W_N];   /* slice injected during the current adjoint step */
    int nwave;             /* number of wave fields used */
    int wave_ids[W_N];
    int nmem;
    int mem_ids[R_N];
    /* DFT gradient (back_prop_type 2, src/assign_modeling_case.c:549-570) */
    int dtnyq, ntnyq;
    float df;
    float gradfreqsn[FDO_MAXFREQ];
    float *fw[2][W_N];     /* [forward, adjoint] DFT, complex [nfreqs][nvol] */
    float *fr[2][R_N];     /* memory variables, complex [nfreqs][L*nvol] */
} fdo_state;

/* ---- setup (fdo_setup.c) ---- */
int  fdo_holberg(int fdorder, int maxrelerror, double hc[7]);
int  fdo_cpml_coeff(float npower, float k_max, float fpml, float vppml, float dh,
                    float dt, int nab, float *K, float *b, float *a,
                    float *K_half, float *b_half, float *a_half);
int  fdo_state_init(fdo_state *s, const fdo_cfg *c);
void fdo_state_free(fdo_state *s);
/* params in: 2D [nx][nz], 3D [nx][ny][nz] (z fastest); pars: vp/vs/rho
 * (taup, taus when L>0) for param_type 0.  Returns 0 or an error code
 * (1 = CFL violated as in src/assign_modeling_case.c:819-823). */
int  fdo_set_model(fdo_state *s, const float *a, const float *b, const float *rho,
                   const float *taup, const float *taus);
void fdo_literal(double *out, float v);

/* ---- time loop (fdo_driver.c) ---- */
int fdo_forward(fdo_state *s, const fdo_kernels *k, const fdo_shot *shot,
                const int outsel[O_N], int alltypes_mask, float *const seis[O_N],
                int save_boundaries);
int fdo_adjoint(fdo_state *s, const fdo_kernels *k, const fdo_shot *shot,
                const int outsel[O_N], int alltypes_mask, float *const res[O_N]);
void fdo_zero_gradients(fdo_state *s);
/* ---- DFT gradient (fdo_dft.c) ---- */
void fdo_dft_factors(const fdo_state *s, int thist, float *re, float *im);
void fdo_savefreqs(fdo_state *s, int slot, int thist);
void fdo_zero_dft(fdo_state *s, int slot);
void fdo_calc_grad(fdo_state *s);
int  fdo_source_targets(int nd, int alltypes_mask, int type, int *fields, float *div);

extern const fdo_kernels fdo_port_kernels;

#ifdef __cplusplus
}
#endif
#endif
