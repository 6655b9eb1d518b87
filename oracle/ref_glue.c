/*
 * ref_glue.c -- kernel table that runs the reference's own kernel sources
 * (compiled in place as C by oracle/build_ref.py) over every work-item.
 *
 * TEST INFRASTRUCTURE ONLY.  It pins the oracle restatement (fdo_port.c):
 * tests/test_oracle_pin.py runs the same time loop through both tables and
 * requires identical bits.  Compiled with the same -D constants as the
 * kernels (ND, NX/NY/NZ padded, FDOH, ...).
 */
#include "fdo.h"

#include <stddef.h>
#include <stdint.h>

__thread int fdo_ref_gid[3];

/* The reference kernels' entry points, renamed at compile time.  Declared
 * without prototypes: each call below lists the arguments in the order of the
 * kernel's signature in the reference file. */
void ref_update_v();
void ref_update_s();
void ref_freesurface();
void ref_update_adjv();
void ref_update_adjs();
void ref_surface_adj();
void ref_savebnd();

#define W(s, id) ((s)->w[id])
#define WR(s, id) ((s)->wr[id])
#define PS(s, id) ((s)->psi[id])
#define PP(s, id) ((s)->p[id])
#define CX(s) (s)->cx[C_K], (s)->cx[C_A], (s)->cx[C_B], (s)->cx[C_KH], (s)->cx[C_AH], (s)->cx[C_BH]
#define CY(s) (s)->cy[C_K], (s)->cy[C_A], (s)->cy[C_B], (s)->cy[C_KH], (s)->cy[C_AH], (s)->cy[C_BH]
#define CZ(s) (s)->cz[C_K], (s)->cz[C_A], (s)->cz[C_B], (s)->cz[C_KH], (s)->cz[C_AH], (s)->cz[C_BH]

static int64_t ncells(const fdo_state *s) { return (int64_t)s->c.nz * s->c.ny * s->c.nx; }

#if ND == 21 || ND == 22
/* SH and acoustic: only the two update kernels exist as loadable kernels */
static void g_update_v(fdo_state *s)
{
    int64_t n = ncells(s);
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < n; g++) {
        fdo_ref_gid[0] = (int)g;
#if ND == 21
        ref_update_v(0, 0, W(s, W_VY), W(s, W_SXY), W(s, W_SYZ), PP(s, P_RHO), s->taper, CX(s), CZ(s),
                     PS(s, PS_SXY_X), PS(s, PS_SYZ_Z), NULL);
#else
        ref_update_v(0, W(s, W_VX), W(s, W_VZ), W(s, W_SXX), PP(s, P_RIP), PP(s, P_RKP), s->taper, CZ(s), CX(s),
                     PS(s, PS_SXX_X), PS(s, PS_SZZ_Z), NULL);
#endif
    }
}
static void g_update_s(fdo_state *s)
{
    int64_t n = ncells(s);
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < n; g++) {
        fdo_ref_gid[0] = (int)g;
#if ND == 21
        /* the reference would bind NULL for psi_vyx / psi_vyz; the intended
         * arrays are passed */
        ref_update_s(0, 0, W(s, W_VY), W(s, W_SXY), W(s, W_SYZ), PP(s, P_MU), s->r[R_XY], s->r[R_YZ],
                     PP(s, P_TAUS), s->eta, s->taper, CX(s), CZ(s), PS(s, PS_VY_X), PS(s, PS_VY_Z), NULL);
#else
        ref_update_s(0, W(s, W_VX), W(s, W_VZ), W(s, W_SXX), PP(s, P_M), s->r[R_XX], PP(s, P_TAUP), s->eta,
                     s->taper, CX(s), CZ(s), PS(s, PS_VX_X), PS(s, PS_VZ_Z), NULL);
#endif
    }
}
static void g_none_s(fdo_state *s) { (void)s; }
static void g_none_sp(fdo_state *s, int p) { (void)s; (void)p; }
static const fdo_kernels ref_kernels = {
    g_update_v, g_update_s, g_none_sp, g_none_s, g_none_s, g_none_s, g_none_sp, "reference",
};
#else
static void g_update_v(fdo_state *s)
{
    int64_t n = ncells(s);
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < n; g++) {
        fdo_ref_gid[0] = (int)g;
#if ND == 3
        ref_update_v(0, W(s, W_VX), W(s, W_VY), W(s, W_VZ), W(s, W_SXX), W(s, W_SYY), W(s, W_SZZ), W(s, W_SXY),
                     W(s, W_SYZ), W(s, W_SXZ), PP(s, P_RIP), PP(s, P_RJP), PP(s, P_RKP), s->taper, CX(s), CY(s),
                     CZ(s), PS(s, PS_SXX_X), PS(s, PS_SXY_X), PS(s, PS_SXY_Y), PS(s, PS_SXZ_X), PS(s, PS_SXZ_Z),
                     PS(s, PS_SYY_Y), PS(s, PS_SYZ_Y), PS(s, PS_SYZ_Z), PS(s, PS_SZZ_Z), NULL);
#else
        ref_update_v(0, W(s, W_VX), W(s, W_VZ), W(s, W_SXX), W(s, W_SZZ), W(s, W_SXZ), PP(s, P_RIP),
                     PP(s, P_RKP), s->taper, CZ(s), CX(s), PS(s, PS_SXX_X), PS(s, PS_SXZ_X), PS(s, PS_SXZ_Z),
                     PS(s, PS_SZZ_Z), NULL);
#endif
    }
}

static void g_update_s(fdo_state *s)
{
    int64_t n = ncells(s);
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < n; g++) {
        fdo_ref_gid[0] = (int)g;
#if ND == 3
        ref_update_s(0, 0, W(s, W_VX), W(s, W_VY), W(s, W_VZ), W(s, W_SXX), W(s, W_SYY), W(s, W_SZZ),
                     W(s, W_SXY), W(s, W_SYZ), W(s, W_SXZ), PP(s, P_M), PP(s, P_MU), PP(s, P_MUIPJP),
                     PP(s, P_MUJPKP), PP(s, P_MUIPKP), s->r[R_XX], s->r[R_YY], s->r[R_ZZ], s->r[R_XY],
                     s->r[R_YZ], s->r[R_XZ], PP(s, P_TAUS), PP(s, P_TAUSIPJP), PP(s, P_TAUSJPKP),
                     PP(s, P_TAUSIPKP), PP(s, P_TAUP), s->eta, NULL, NULL, s->taper, CX(s), CY(s), CZ(s),
                     PS(s, PS_VX_X), PS(s, PS_VX_Y), PS(s, PS_VX_Z), PS(s, PS_VY_X), PS(s, PS_VY_Y),
                     PS(s, PS_VY_Z), PS(s, PS_VZ_X), PS(s, PS_VZ_Y), PS(s, PS_VZ_Z), NULL);
#else
        ref_update_s(0, W(s, W_VX), W(s, W_VZ), W(s, W_SXX), W(s, W_SZZ), W(s, W_SXZ), PP(s, P_M), PP(s, P_MU),
                     PP(s, P_MUIPKP), s->r[R_XX], s->r[R_ZZ], s->r[R_XZ], PP(s, P_TAUS), PP(s, P_TAUSIPKP),
                     PP(s, P_TAUP), s->eta, s->taper, CX(s), CZ(s), PS(s, PS_VX_X), PS(s, PS_VX_Z),
                     PS(s, PS_VZ_X), PS(s, PS_VZ_Z), NULL);
#endif
    }
}

static void g_surface(fdo_state *s, int pdir)
{
#if ND == 3
#pragma omp parallel for collapse(2) schedule(static)
    for (int x = 0; x < s->c.nx; x++)
        for (int y = 0; y < s->c.ny; y++) {
            fdo_ref_gid[0] = y;
            fdo_ref_gid[1] = x;
            ref_freesurface(W(s, W_VX), W(s, W_VY), W(s, W_VZ), W(s, W_SXX), W(s, W_SYY), W(s, W_SZZ),
                            W(s, W_SXY), W(s, W_SYZ), W(s, W_SXZ), PP(s, P_M), PP(s, P_MU), s->r[R_XX],
                            s->r[R_YY], s->r[R_ZZ], PP(s, P_TAUS), PP(s, P_TAUP), s->eta, s->cx[C_K],
                            PS(s, PS_VX_X), s->cy[C_K], PS(s, PS_VY_Y), s->taper, pdir);
        }
#else
    for (int x = 0; x < s->c.nx; x++) {
        fdo_ref_gid[0] = x;
        ref_freesurface(W(s, W_VX), W(s, W_VZ), W(s, W_SXX), W(s, W_SZZ), W(s, W_SXZ), PP(s, P_M), PP(s, P_MU),
                        s->r[R_XX], s->r[R_ZZ], PP(s, P_TAUS), PP(s, P_TAUP), s->eta, s->cx[C_K],
                        PS(s, PS_VX_X), s->taper, pdir);
    }
#endif
}

#define BC(s, id) ((s)->bnd_cur[id])

static void g_update_adjv(fdo_state *s)
{
    int64_t n = ncells(s);
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < n; g++) {
        fdo_ref_gid[0] = (int)g;
#if ND == 3
        ref_update_adjv(0, W(s, W_VX), W(s, W_VY), W(s, W_VZ), W(s, W_SXX), W(s, W_SYY), W(s, W_SZZ),
                        W(s, W_SXY), W(s, W_SYZ), W(s, W_SXZ), BC(s, W_VX), BC(s, W_VY), BC(s, W_VZ),
                        BC(s, W_SXX), BC(s, W_SYY), BC(s, W_SZZ), BC(s, W_SXY), BC(s, W_SYZ), BC(s, W_SXZ),
                        WR(s, W_VX), WR(s, W_VY), WR(s, W_VZ), WR(s, W_SXX), WR(s, W_SYY), WR(s, W_SZZ),
                        WR(s, W_SXY), WR(s, W_SYZ), WR(s, W_SXZ), PP(s, P_RIP), PP(s, P_RJP), PP(s, P_RKP),
                        s->taper, CX(s), CY(s), CZ(s), PS(s, PS_SXX_X), PS(s, PS_SXY_X), PS(s, PS_SXY_Y),
                        PS(s, PS_SXZ_X), PS(s, PS_SXZ_Z), PS(s, PS_SYY_Y), PS(s, PS_SYZ_Y), PS(s, PS_SYZ_Z),
                        PS(s, PS_SZZ_Z), NULL, s->grad[G_RHO], NULL, NULL, NULL);
#else
        ref_update_adjv(0, W(s, W_VX), W(s, W_VZ), W(s, W_SXX), W(s, W_SZZ), W(s, W_SXZ), BC(s, W_VX),
                        BC(s, W_VZ), BC(s, W_SXX), BC(s, W_SZZ), BC(s, W_SXZ), WR(s, W_VX), WR(s, W_VZ),
                        WR(s, W_SXX), WR(s, W_SZZ), WR(s, W_SXZ), PP(s, P_RIP), PP(s, P_RKP), s->taper, CX(s),
                        CZ(s), PS(s, PS_SXX_X), PS(s, PS_SXZ_X), PS(s, PS_SXZ_Z), PS(s, PS_SZZ_Z),
                        s->grad[G_RHO], NULL, NULL, NULL, NULL);
#endif
    }
}

static void g_update_adjs(fdo_state *s)
{
    int64_t n = ncells(s);
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < n; g++) {
        fdo_ref_gid[0] = (int)g;
#if ND == 3
        ref_update_adjs(0, W(s, W_VX), W(s, W_VY), W(s, W_VZ), W(s, W_SXX), W(s, W_SYY), W(s, W_SZZ),
                        W(s, W_SXY), W(s, W_SYZ), W(s, W_SXZ), BC(s, W_VX), BC(s, W_VY), BC(s, W_VZ),
                        BC(s, W_SXX), BC(s, W_SYY), BC(s, W_SZZ), BC(s, W_SXY), BC(s, W_SYZ), BC(s, W_SXZ),
                        WR(s, W_VX), WR(s, W_VY), WR(s, W_VZ), WR(s, W_SXX), WR(s, W_SYY), WR(s, W_SZZ),
                        WR(s, W_SXY), WR(s, W_SYZ), WR(s, W_SXZ), s->r[R_XX], s->r[R_YY], s->r[R_ZZ],
                        s->r[R_XY], s->r[R_YZ], s->r[R_XZ], s->rr[R_XX], s->rr[R_YY], s->rr[R_ZZ], s->rr[R_XY],
                        s->rr[R_YZ], s->rr[R_XZ], PP(s, P_M), PP(s, P_MU), PP(s, P_MUIPJP), PP(s, P_MUJPKP),
                        PP(s, P_MUIPKP), PP(s, P_TAUS), PP(s, P_TAUSIPJP), PP(s, P_TAUSJPKP), PP(s, P_TAUSIPKP),
                        PP(s, P_TAUP), s->eta, s->taper, CX(s), CY(s), CZ(s), PS(s, PS_VX_X), PS(s, PS_VX_Y),
                        PS(s, PS_VX_Z), PS(s, PS_VY_X), PS(s, PS_VY_Y), PS(s, PS_VY_Z), PS(s, PS_VZ_X),
                        PS(s, PS_VZ_Y), PS(s, PS_VZ_Z), s->grad[G_RHO], s->grad[G_M], s->grad[G_MU], NULL,
                        NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL, NULL);
#else
        ref_update_adjs(0, W(s, W_VX), W(s, W_VZ), W(s, W_SXX), W(s, W_SZZ), W(s, W_SXZ), BC(s, W_VX),
                        BC(s, W_VZ), BC(s, W_SXX), BC(s, W_SZZ), BC(s, W_SXZ), WR(s, W_VX), WR(s, W_VZ),
                        WR(s, W_SXX), WR(s, W_SZZ), WR(s, W_SXZ), s->r[R_XX], s->r[R_ZZ], s->r[R_XZ],
                        s->rr[R_XX], s->rr[R_ZZ], s->rr[R_XZ], PP(s, P_M), PP(s, P_MU), PP(s, P_MUIPKP),
                        PP(s, P_TAUS), PP(s, P_TAUSIPKP), PP(s, P_TAUP), s->eta, s->taper, CX(s), CZ(s),
                        PS(s, PS_VX_X), PS(s, PS_VX_Z), PS(s, PS_VZ_X), PS(s, PS_VZ_Z), s->grad[G_RHO],
                        s->grad[G_M], s->grad[G_MU], NULL, NULL, NULL, s->hess[G_RHO], s->hess[G_M],
                        s->hess[G_MU], s->hess[G_TAUP], s->hess[G_TAUS], NULL, NULL);
#endif
    }
}

static void g_surface_adj(fdo_state *s)
{
    /* sequential: the kernel updates neighbouring columns */
#if ND == 3
    for (int x = 0; x < s->c.nx; x++)
        for (int y = 0; y < s->c.ny; y++) {
            fdo_ref_gid[0] = x;
            fdo_ref_gid[1] = y;
            ref_surface_adj(WR(s, W_VX), WR(s, W_VY), WR(s, W_VZ), WR(s, W_SXX), WR(s, W_SYY), WR(s, W_SZZ),
                            WR(s, W_SXY), WR(s, W_SYZ), WR(s, W_SXZ), PP(s, P_M), PP(s, P_RIP), PP(s, P_RJP),
                            PP(s, P_RKP), PP(s, P_MU), s->r[R_XX], s->r[R_ZZ], PP(s, P_TAUS), PP(s, P_TAUP),
                            s->eta);
        }
#else
    for (int x = 0; x < s->c.nx; x++) {
        fdo_ref_gid[0] = x;
        ref_surface_adj(WR(s, W_VX), WR(s, W_VZ), WR(s, W_SXX), WR(s, W_SZZ), WR(s, W_SXZ), PP(s, P_M),
                        PP(s, P_RIP), PP(s, P_RKP), PP(s, P_MU), s->r[R_XX], s->r[R_ZZ], PP(s, P_TAUS),
                        PP(s, P_TAUP), s->eta, s->cx[C_K], PS(s, PS_VX_X), s->taper);
    }
#endif
}

static void g_savebnd(fdo_state *s, int t)
{
    float *b[W_N];
    for (int i = 0; i < W_N; i++) b[i] = s->bnd[i] ? s->bnd[i] + (int64_t)t * s->nbnd : NULL;
    for (int g = 0; g < s->nbnd; g++) {
        fdo_ref_gid[0] = g;
#if ND == 3
        ref_savebnd(W(s, W_VX), W(s, W_VY), W(s, W_VZ), W(s, W_SXX), W(s, W_SYY), W(s, W_SZZ), W(s, W_SXY),
                    W(s, W_SYZ), W(s, W_SXZ), b[W_VX], b[W_VY], b[W_VZ], b[W_SXX], b[W_SYY], b[W_SZZ], b[W_SXY],
                    b[W_SYZ], b[W_SXZ]);
#else
        ref_savebnd(W(s, W_SXX), W(s, W_SXZ), W(s, W_SZZ), W(s, W_VX), W(s, W_VZ), b[W_SXX], b[W_SXZ],
                    b[W_SZZ], b[W_VX], b[W_VZ]);
#endif
    }
}

static const fdo_kernels ref_kernels = {
    g_update_v, g_update_s, g_surface, g_update_adjv, g_update_adjs, g_surface_adj, g_savebnd, "reference",
};
#endif

const fdo_kernels *fdo_ref_kernels_or_null(void) { return &ref_kernels; }

/* The grid this build was compiled for, to refuse mismatched state. */
void fdo_ref_grid(int *out)
{
    out[0] = NZ; out[1] = NX;
#if ND == 3
    out[2] = NY;
#else
    out[2] = 1;
#endif
    out[3] = FDOH;
}
