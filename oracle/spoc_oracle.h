/*
 * CPU oracle for the SPOC RK4 discontinuous-Galerkin shallow-water path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a line-by-line C restatement of the
 * reference Fortran 77 routines (dupontf/SPOC), kept in the reference loop
 * and summation order and compiled with -ffp-contract=off so that it is
 * deterministic.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it, and only as the checker / CPU baseline; the
 * product (spoc_b200/) never calls it.
 *
 * Parity pin status: the reference ships no golden vectors, no tests and no
 * fixtures, and it cannot be compiled here (Fortran 77, no Fortran compiler).
 * The oracle is therefore "parity unpinned" with respect to reference output;
 * it is pinned instead by known-answer properties (closed-form integrals of
 * Legendre products, Cholesky reconstruction, exact mass conservation, a
 * linear standing wave, constant-state invariance, polynomial exactness of the
 * face trace/lift) checked in tests/.
 *
 * Index conventions follow the Fortran: every integer connectivity array
 * stores 1-based ids, and every 2-D array is column-major with an explicit
 * leading dimension.
 */
#ifndef SPOC_ORACLE_H
#define SPOC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* The contents of the reference COMMON blocks /const/ /gauss/ /gaussf/
 * /gauss2/ /gauss3/ /matrices/ plus cip (src/shwwnl.f:60-71). */
typedef struct {
  int nc, nm, ng, ngf;
  const double *wi, *xi, *yi;   /* [ng] */
  const double *wif, *tif;      /* [ngf] */
  const double *pi2;  int ldq;  /* pi2(ldq, nm) */
  const double *pico; int ldg, ldp; /* pico(ldg, ldp, 3) */
  const double *amm, *amml, *agx, *agy, *ammo; int ldm; /* (ldm, nm); amm/amml upper Cholesky factors */
  const int *cip;               /* cip(2, 0:nc): cip[2*j + (r-1)] */
} ora_common;

/* Mesh pointers as cal_var receives them (src/calvarnl_fs.f:9-12). */
typedef struct {
  int ne, nf;
  const int *itm;      /* itm(3,ne)  face of each element side          */
  const int *its;      /* its(3,ne)  +1 if element is tseg(1,face), else -1 */
  const int *tseg;     /* tseg(2,nf) elements of a face, 0 = wall       */
  const int *ssit;     /* ssit(2,nf) side index of the face in each element */
  const double *norm;  /* norm(2,nf) (dy,-dx), length = edge length     */
  const double *vect;  /* vect(5,ne) ax,bx,ay,by,1/det                 */
  const double *normt; /* normt(2,ne) unit normal of side 1            */
  const int *bdl;      /* bdl(ne) wall element flag (logical)          */
} ora_mesh;

enum { ORA_LIN = 0, ORA_FS = 1, ORA_NS = 2, ORA_INV = 3 };

/* Contraction precision of the study mode: 64 (default, the reference) or 32
 * (float operands and accumulation in every contraction; solves and RK4 stay
 * double).  See tests/test_precision_study.py. */
void ora_set_contraction_precision(int bits);

/* ---- L1: basis, quadrature tables and reference operators ---- */
double ora_po(int n, double x);
double ora_dpo(int n, double x);
void ora_cal_p2(int nc, int ng, const double *xi, const double *yi, double *pi2, int ldq);
void ora_cal_pico(int nc, int ngf, const double *tif, double *pico, int ldg, int ldp);
void ora_calip(int nc, int *cip);
/* which: 0 f2 (mass), 1 fx, 2 fy, 3 dfx, 4 dfy */
void ora_cal_mat(int nc, int ng, int which, const double *xi, const double *yi,
                 const double *wi, double *mat, int ldm);
void ora_cal_matl(int nc, const double *amm, double *amml, int ldm);
int ora_dpotf2_upper(int n, double *a, int lda);
void ora_dtrsm4(int m, const double *a, int lda, double *b, const double *diag);

/* ---- L2: mesh ---- */
int ora_pointer_mesh(int nn, int ne, const int *in, int *itm, int *tseg, int *pseg, int nfmax);
int ora_check_mesh(int ne, int nf, const int *itm, const int *tseg);
void ora_cal_rotnf(int nf, const double *x, const double *y, double *norm, const int *pseg);
int ora_cal_its(int nf, const int *itm, int *its, const int *tseg, int *ssit);
void ora_calpre(int nn, int ne, int nf, const int *in, const double *xgr, const double *ygr,
                double *vect, const int *itm, const double *norm, double *normt, int *bdl,
                int *nint, int *pint, int *nbdl, int *pbdl, int *nebd, const int *tseg,
                const int *pseg);
void ora_coriolis(int nc, int ne, const int *in, const double *xgr, const double *ygr,
                  double *fc, int ld, double f0, double beta);
int ora_changemaille(int nn, int ne, int nf, int *in, int *itm, int *tseg, int *pseg);

/* ---- L1 hot kernels (exposed for unit pins) ---- */
void ora_cal_flu(const ora_common *c, int nf, const int *tseg, double *fbdy, int ldf,
                 const double *a0, int ld, const int *ssit, int nthreads);
void ora_tri_f(const ora_common *c, int tk, const int *itm, const int *its,
               const double *fbdy, int ldf, double *b, double coeff);
void ora_cal_b(const ora_common *c, double *b, const double *ak, const double *mat, double coeff);
void ora_spectoxy(const ora_common *c, double *mff, const double *ak);
void ora_xytospec(const ora_common *c, double *b, const double *mff);
void ora_reduc_gn(int nc, const double *gn, double *gnr, const int *cip);
void ora_reduc_inv_gn(int nc, double *gn, const double *gnr, const int *cip);

/* ---- L3: the physics right-hand side, one of four variants ---- */
int ora_cal_var(int variant, const ora_common *c, const ora_mesh *m, int ld,
                const double *u0, const double *v0, const double *h0,
                double *u1, double *v1, double *h1,
                const double *fc, const double *w0, const double *z0, const double *hb,
                double mu0, double mb0, double g0, int nthreads);

/* ---- L4: RK4 loop of src/shwwnl.f:233-286 (state updated in place) ---- */
int ora_rk4(int variant, const ora_common *c, const ora_mesh *m, int ld,
            double *u0, double *v0, double *h0,
            const double *fc, const double *w0, const double *z0, const double *hb,
            double mu0, double mb0, double g0, double dt, int nsteps, int nthreads);

/* ---- diagnostics ---- */
void ora_energy(const ora_common *c, int ne, int ld, const double *u0, const double *v0,
                const double *h0, double g0, const double *hb, double *ke, double *pe,
                double *mass, const int *in, const double *xgr, const double *ygr);
double ora_checkcfl(int nc, int ne, int ld, const double *hb, const int *in, double g0,
                    const double *xgr, const double *ygr, double *cflmin);

/* ---- initial conditions (src/init.f:290-344) ---- */
void ora_calh_points(const ora_common *c, int ne, const int *in, const double *xgr,
                     const double *ygr, double *px, double *py);
void ora_calh(const ora_common *c, int ne, const double *vals, double *h, int ld);

/* ---- L5: regridding (src/adapt.f) and the adaptive driver's CFL ---- */
void ora_checkconv(const ora_common *c, int nf, int ne, int ld, const double *a0,
                   const int *tseg, const int *ssit, double *amax);
void ora_cal_conv(const ora_common *c, int nf, int ne, int ld, const double *u0,
                  const double *v0, const double *h0, const int *tseg, const int *ssit,
                  double fac1, double fac2, double fac3, int *fconv, int *fderaff, int *flags,
                  double *supmax, double *umax, double *vmax, double *hmax);
void ora_inter_only_new(int ne, int nenew, const int *in, const int *innew, int *tinter);
int ora_interlin(const int *itt, const int *itm, const int *tseg, const int *pseg,
                 const double *x, const double *y, int *tk, double *xdp, double *ydp,
                 double *lab, int maxit);
int ora_interpol(const ora_common *c, int ne, const int *in, const int *itm, const int *tseg,
                 const int *pseg, const double *xgr, const double *ygr, const int *tinter,
                 const double *u, int ld, double *unew, int nenew, const double *xgrnew,
                 const double *ygrnew, const int *innew, int *loc_elem, double *loc_x,
                 double *loc_y);
void ora_verif_rot(const ora_common *c, int ne, int ld, double *u0, double *v0,
                   const double *normt, const int *bdl);
void ora_cal_pgraph(int nc, int n, double *pgraph);
void ora_eval_points(int nc, int ld, const double *u, const double *v, const double *h,
                     int npts, const int *elem, const double *px, const double *py,
                     double *out);
void ora_lattice(int nc, int ne, int ld, const double *u, const double *v, const double *h,
                 const int *in, const double *xgr, const double *ygr, int n,
                 const double *pgraph, double *out);
double ora_checkcfl2(int nc, int ne, int ld, const double *hb, const double *u,
                     const double *v, const int *in, double g0, const double *xgr,
                     const double *ygr, int n, const double *pgraph, double dt_in,
                     double *cflmin);

#ifdef __cplusplus
}
#endif
#endif
