/*
 * ref_calc_grad_glue.c -- runs the reference's own calc_grad
 * (src/calc_grad.c, compiled in place by oracle/build.py:build_refcg) on
 * transforms supplied by a test.
 *
 * TEST INFRASTRUCTURE ONLY.  It fills the few fields of the reference's
 * model/device structures that calc_grad reads (src/calc_grad.c:376-560) and
 * provides the name lookups it calls.  tests/test_oracle_pin.py compares the
 * result with the oracle's restatement (oracle/fdo_dft.c).
 */
#include "F.h"

constants *get_cst(constants *csts, int ncsts, const char *name)
{
    for (int i = 0; i < ncsts; i++)
        if (strcmp(csts[i].name, name) == 0) return &csts[i];
    return NULL;
}

parameter *get_par(parameter *pars, int npars, const char *name)
{
    for (int i = 0; i < npars; i++)
        if (strcmp(pars[i].name, name) == 0) return &pars[i];
    return NULL;
}

/* fwd/adj: 15 complex buffers in the order vx vy vz sxx syy szz sxy syz sxz
 * rxx ryy rzz rxy ryz rxz (NULL where the model has none), each
 * [nfreqs][(L)][padded cells]; par and grad: M, mu, rho, taup, taus over the
 * physical cells; hess (NULL: HOUT off) the Hessian arrays in the same
 * order.  The buffers are modified in place, as the reference
 * modifies its host copies. */
int refcg_run(int nd, int nz, int ny, int nx, int fdorder, int L, int par_type, int nfreqs, int ntnyq,
              int dtnyq, float dt, float f0, const float *fl, const float *gradfreqsn, float **fwd, float **adj,
              float **par, float **grad, float **hess)
{
    static const char *vname[15] = {"vx", "vy", "vz", "sxx", "syy", "szz", "sxy", "syz", "sxz",
                                    "rxx", "ryy", "rzz", "rxy", "ryz", "rxz"};
    static const char *pname[5] = {"M", "mu", "rho", "taup", "taus"};
    model *m = calloc(1, sizeof(model));
    device *d = calloc(1, sizeof(device));
    variable vars[15];
    parameter pars[5];
    constants csts[2];
    float flc[8] = {0}, fnc[16] = {0};
    memset(vars, 0, sizeof vars);
    memset(pars, 0, sizeof pars);
    memset(csts, 0, sizeof csts);
    int nv = 0;
    for (int i = 0; i < 15; i++) {
        if (!fwd[i]) continue;
        vars[nv].name = vname[i];
        vars[nv].for_grad = 1;
        vars[nv].cl_fvar.host = fwd[i];
        vars[nv].cl_fvar_adj.host = adj[i];
        nv++;
    }
    int np = L > 0 ? 5 : 3;
    for (int i = 0; i < np; i++) {
        pars[i].name = pname[i];
        pars[i].cl_par.host = par[i];
        pars[i].cl_grad.host = grad[i];
        pars[i].cl_H.host = hess ? hess[i] : NULL;
        pars[i].to_grad = 1;
    }
    for (int l = 0; l < L && l < 8; l++) flc[l] = fl[l];
    for (int f = 0; f < nfreqs && f < 16; f++) fnc[f] = gradfreqsn[f];
    csts[0].name = "FL";
    csts[0].gl_cst = flc;
    csts[0].num_ele = L;
    csts[1].name = "gradfreqsn";
    csts[1].gl_cst = fnc;
    csts[1].num_ele = nfreqs;
    m->ND = nd;
    m->NDIM = nd == 3 ? 3 : 2;
    m->L = L;
    m->par_type = par_type;
    m->NFREQS = nfreqs;
    m->NTNYQ = ntnyq;
    m->DTNYQ = dtnyq;
    m->dt = dt;
    m->f0 = f0;
    m->FDORDER = fdorder;
    m->FDOH = fdorder / 2;
    m->HOUT = hess != NULL;
    m->csts = csts;
    m->ncsts = 2;
    m->nvars = nv;
    m->npars = np;
    d->vars = vars;
    d->nvars = nv;
    d->pars = pars;
    d->npars = np;
    d->N[0] = nz;
    if (nd == 3) { d->N[1] = ny; d->N[2] = nx; }
    else d->N[1] = nx;
    int rc = calc_grad(m, d);
    free(m);
    free(d);
    return rc;
}
