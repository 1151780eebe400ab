/*
 * spoc_gpu.h -- C ABI of the B200 implementation of SPOC's RK4
 * discontinuous-Galerkin shallow-water right-hand side.
 *
 * The reference selects its physics at link time: every src/calvar*.f defines
 *   subroutine cal_var(nf,ne,u0,v0,h0,u1,v1,h1,tseg,pseg,ssit,itm,its,norm,
 *                      nbdl,pbdl,nint,pint,bdl,cip,vect,normt,
 *                      mu0,mb0,fc,beta,w0,z0,g0,hb,time)
 * (src/calvarnl_fs.f:9-12, src/calvar_lin.f:7-10) and reads its tables from
 * COMMON /const/ /gauss/ /gaussf/ /gauss2/ /gauss3/ /matrices/
 * (src/calvarnl_fs.f:16-64).  This header exposes:
 *   - spoc_create / spoc_cal_var / spoc_cal_var_dev / spoc_rk4_*: the handle
 *     API (tables and mesh uploaded once, state optionally device-resident);
 *   - cal_var_: the literal 31-argument drop-in with the gfortran by-reference
 *     ABI, reading the COMMON contents registered by spoc_register_commons;
 *   - spoc_build_* helpers: host restatements of the reference set-up routines
 *     (tables, mesh pointers, corner fix, L2 projection) for callers that do
 *     not keep the Fortran driver.
 *
 * Conventions: every integer connectivity array stores the reference's 1-based
 * ids; every 2-D array is Fortran column-major with an explicit leading
 * dimension; all functions return 0 on success or a positive SPOC_E* code and
 * never throw.  A handle owns one CUDA stream and is not re-entrant.
 */
#ifndef SPOC_GPU_H
#define SPOC_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define SPOC_OK 0
#define SPOC_E_ARG 1         /* bad argument or size */
#define SPOC_E_CUDA 2        /* CUDA runtime error (see spoc_last_error) */
#define SPOC_E_NONFINITE 3   /* the device non-finite flag was raised */
#define SPOC_E_MATRIX 4      /* a mass matrix is not positive definite */
#define SPOC_E_MESH 5        /* connectivity check failed */
#define SPOC_E_NOMEM 6       /* host or device allocation failed */
#define SPOC_E_UNSUPPORTED 7 /* variant / precision / size not built */

/* physics variants: the four link-time plug-ins of the reference */
#define SPOC_LIN 0 /* src/calvar_lin.f   */
#define SPOC_FS 1  /* src/calvarnl_fs.f  */
#define SPOC_NS 2  /* src/calvarnl_ns.f  */
#define SPOC_INV 3 /* src/calvarnl_inv.f */

/* precision modes */
#define SPOC_FP64 0     /* reference operation order, no contraction: bit-exact to the CPU restatement */
#define SPOC_FP64_FMA 1 /* reference order with fused multiply-adds in the contractions and
                           solves: FP64 accuracy, not bit-exact; untabulated (nc, ng, ngf)
                           run the SPOC_FP64 kernels */
#define SPOC_MIXED 2    /* FP32 contractions in the orthonormal basis psi = U^-T phi
                           (amm = U^T U), FP64 RK4 state and basis changes; tabulated
                           (nc, ng, ngf) only.  State, inputs and outputs stay in the
                           reference basis at the ABI. */

/* COMMON-block content, as the Fortran driver holds it (src/shwwnl.f:60-71).
 * amm and amml hold the upper Cholesky factors (src/shwwnl.f:153-156). */
typedef struct {
  int nc, nm, ng, ngf;
  const double *wi, *xi, *yi; /* [ng]  /gauss/  */
  const double *wif, *tif;    /* [ngf] /gaussf/ */
  const double *pi2;          /* pi2(ld_pi2, nm)            /gauss2/ */
  int ld_pi2;
  const double *pico;         /* pico(ld_pico1, ld_pico2, 3) /gauss3/ */
  int ld_pico1, ld_pico2;
  const double *amm, *amml, *agx, *agy, *ammo; /* (ld_mat, nm) /matrices/ */
  int ld_mat;
  const int *cip;             /* cip(2, 0:ncip-1), ncip >= nc+1 */
} spoc_tables;

/* mesh pointers, exactly as cal_var receives them (src/calvarnl_fs.f:22-61) */
typedef struct {
  int ne, nf;
  const int *itm;      /* itm(3,ne)  */
  const int *its;      /* its(3,ne)  */
  const int *tseg;     /* tseg(2,nf) (0 = wall) */
  const int *ssit;     /* ssit(2,nf) */
  const double *norm;  /* norm(2,nf) */
  const double *vect;  /* vect(5,ne) */
  const double *normt; /* normt(2,ne) */
  const int *bdl;      /* bdl(ne), LOGICAL*4 */
} spoc_mesh;

/* physical parameters and time-constant fields (ld, ne) */
typedef struct {
  double mu0, mb0, g0;
  const double *fc, *w0, *z0, *hb;
  int ld;
} spoc_params;

typedef struct spoc_handle spoc_handle;

/* Upload tables and mesh; allocate device work space for ne elements.
 * Replaces the per-call COMMON/argument reads of cal_var (src/calvarnl_fs.f:9-64). */
int spoc_create(const spoc_tables *tables, const spoc_mesh *mesh, int variant, int precision,
                spoc_handle **out);
void spoc_destroy(spoc_handle *h);
/* Kernel family (no reference counterpart; results are identical):
 * SPOC_PATH_AUTO picks the compile-time-sized kernels when (nc, ng, ngf) is
 * one of the tabulated combinations, else the generic runtime-sized ones. */
#define SPOC_PATH_AUTO 0
#define SPOC_PATH_GENERIC 1
#define SPOC_PATH_TEMPLATED 2
#define SPOC_PATH_TENSOR 3 /* SPOC_MIXED only: nonlinear volume work on the tcgen05 tensor
                              cores (three-term TF32 products); SPOC_PATH_AUTO and
                              SPOC_PATH_TEMPLATED keep it on the FP32 pipes, which are more
                              accurate (FP32 fused multiply-adds) */
int spoc_set_kernel_path(spoc_handle *h, int path);
/* Use an external cudaStream_t (0 = the handle's own stream). */
int spoc_set_stream(spoc_handle *h, void *stream);
/* Upload mu0, mb0, g0 and fc, w0, z0, hb (arguments of cal_var, src/calvarnl_fs.f:12). */
int spoc_set_params(spoc_handle *h, const spoc_params *p);

/* One right-hand-side evaluation with HOST arrays (ld, ne): the literal
 * replacement of `call cal_var(...)` in the RK4 loop (src/shwwnl.f:238-274). */
int spoc_cal_var(spoc_handle *h, int ld, const double *u0, const double *v0, const double *h0,
                 double *u1, double *v1, double *h1);
/* Same with DEVICE arrays (ld, ne), on the handle's stream. */
int spoc_cal_var_dev(spoc_handle *h, int ld, const double *u0, const double *v0,
                     const double *h0, double *u1, double *v1, double *h1);

/* Device-resident state (src/shwwnl.f:180-188 init.bin layout, ld = nm packed or 45). */
int spoc_set_state(spoc_handle *h, int ld, const double *u, const double *v, const double *hh);
int spoc_get_state(spoc_handle *h, int ld, double *u, double *v, double *hh);
/* nsteps classical RK4 steps on the resident state (src/shwwnl.f:233-286). */
int spoc_rk4_steps(spoc_handle *h, double dt, int nsteps);
/* H2D of (u,v,hh), nsteps RK4 steps, D2H back: the host-buffer entry point.
   With FP64 handles and mapped pinned arrays (cudaHostAlloc, cudaMallocHost,
   registered memory) the last stage kernel stores the new state into the
   arrays directly; only the rows' first nm values are written. */
int spoc_rk4_steps_host(spoc_handle *h, int ld, double *u, double *v, double *hh, double dt,
                        int nsteps);
/* Kinetic/potential energy and mass of the resident state (src/energy.f:3-96). */
int spoc_energy(spoc_handle *h, double *ke, double *pe, double *mass);
/* CFL time step of src/cfl.f:4-52 on the device (in(3,ne), node coordinates). */
int spoc_cfl(spoc_handle *h, int nn, const int *in, const double *xgr, const double *ygr,
             double *cflmin, double *dt);
/* ---- solution-driven regridding (src/adapt.f; the adaptive driver
 * src/shwwnl_adap.f:375-450) ----
 * spoc_checkconv: checkconv (src/adapt.f:1260-1334) of the resident u, v, h
 *   on the device: per element, the largest jump of the trace across its
 *   interior faces, divided by the field's max |mode 0| (0 when <= 1e-6);
 *   umax / vmax / hmax are host arrays of ne.
 * spoc_cal_conv: cal_conv (src/adapt.f:1122-1193): fconv[e] = some field's
 *   jump > fac1 (refine), fderaff[e] = all three < fac2 (coarsen), host int
 *   arrays of ne; flags[0] conv, flags[1] deraff, flags[2] timedir; *supmax
 *   (may be null) the largest jump.
 * spoc_interpol: interpol (src/adapt.f:1662-1745) on the device: dst's
 *   resident state becomes src's re-projected onto dst's mesh.  tinter[ne_dst]
 *   (from spoc_inter_only_new): the src element (1-based) a dst element
 *   copies, or 0 to project; pt_elem / pt_x / pt_y (ng x ne_dst, from
 *   spoc_locate_points; may be null when nothing projects) the src element
 *   and reference coordinates of each quadrature point.  Both handles must
 *   share the degree and the quadrature rule.
 * spoc_verif_rot: verif_rot (src/shwwnl_adap.f:481-596) on the resident u, v:
 *   the mass-matrix load is solved again, in the rotated wall sub-basis on
 *   wall elements.
 * spoc_cfl2: checkcfl2 (src/cfl.f:57-140) of the resident state on the
 *   ngraph-point lattice (the reference uses 10); *dt = dt_in when no
 *   rounding branch applies. */
int spoc_checkconv(spoc_handle *h, double *umax, double *vmax, double *hmax);
int spoc_cal_conv(spoc_handle *h, double fac1, double fac2, double fac3, int *fconv,
                  int *fderaff, int *flags, double *supmax);
int spoc_interpol(spoc_handle *dst, spoc_handle *src, const int *tinter, const int *pt_elem,
                  const double *pt_x, const double *pt_y);
/* Same with DEVICE arrays, enqueued on dst's stream (after src's stream is
 * drained when the streams differ); ids outside 1..ne_src are not read and
 * make the call return SPOC_E_ARG. */
int spoc_interpol_dev(spoc_handle *dst, spoc_handle *src, const int *tinter, const int *pt_elem,
                      const double *pt_x, const double *pt_y);
int spoc_verif_rot(spoc_handle *h);
int spoc_cfl2(spoc_handle *h, int ngraph, int nn, const int *in, const double *xgr,
              const double *ygr, double dt_in, double *cflmin, double *dt);
/* Point evaluation of the resident state (fsol, src/compare.f:203-219):
 * elem (1-based) and reference coordinates of npts points (host arrays);
 * out[f * npts + i], f = u, v, h. */
int spoc_eval_points(spoc_handle *h, int npts, const int *elem, const double *px,
                     const double *py, double *out);
/* write_gra's values (src/visu2.f:86-149) on the device: for every element
 * and every point of the ngraph-point lattice (k outer, l inner) the
 * physical point and u, v, h: out[(e * np + p) * 5 + c], np = ngraph
 * (ngraph + 1) / 2, c = x, y, u, v, h. */
int spoc_lattice(spoc_handle *h, int ngraph, int nn, const int *in, const double *xgr,
                 const double *ygr, double *out);
/* Number of kernels this handle launched so far (telemetry). */
long long spoc_kernel_launches(spoc_handle *h);
/* Diagnostics (no reference counterpart): run nsteps RK4 steps like
 * spoc_rk4_steps, timing every kernel with CUDA events on the handle's stream;
 * kernel_ms[k] receives the total milliseconds of kernel kind k (nonlinear:
 * 0 q-phase, 1 nonlinear volume, 2 tendency+RK4; linear: 0), *nkinds the
 * number of kinds. */
int spoc_profile_rk4(spoc_handle *h, double dt, int nsteps, double *kernel_ms, int *nkinds);
/* ---- ensemble of basins (no reference counterpart: the reference runs one
 * basin per process).  Members are SPOC_MIXED handles of the free-slip variant
 * (degree 3-6, tabulated rules), each with its own mesh, parameters, state and
 * time step, set through the handle API.  spoc_ensemble_steps advances every
 * member by nsteps RK4 steps with one cooperative launch per RK4 stage for
 * all members together (replayed from a CUDA graph when use_graph != 0 and
 * capture succeeds); the members' states are then read with spoc_get_state.
 * Work layout: blocks_per_sm resident blocks per SM (1 .. max), dealt to the
 * members in proportion to their work modelled as ne nm^p, p = 2, 1, 0.5, 0
 * for weight 0, 1, 2, 3, or measured (weight 4, after spoc_ensemble_balance);
 * spoc_ensemble_configure sets it, spoc_ensemble_info reports it (graph: 1
 * when steps run from a graph; member_blocks: blocks per member, or null).
 * spoc_ensemble_balance runs `rounds` steps (they advance the members) with
 * per-block cycle counters and after each deals the blocks again in
 * proportion to every member's measured block cycles (weight 4). */
typedef struct spoc_ensemble spoc_ensemble;
int spoc_ensemble_create(int nmem, spoc_handle *const *members, spoc_ensemble **out);
void spoc_ensemble_destroy(spoc_ensemble *e);
int spoc_ensemble_configure(spoc_ensemble *e, int blocks_per_sm, int weight);
int spoc_ensemble_info(spoc_ensemble *e, int *blocks_per_sm, int *max_blocks_per_sm, int *weight,
                       int *blocks, int *graph, int *member_blocks);
int spoc_ensemble_steps(spoc_ensemble *e, const double *dt, int nsteps, int use_graph);
int spoc_ensemble_balance(spoc_ensemble *e, const double *dt, int rounds);

/* Self-test of the tcgen05 TF32 tensor-core path the mixed kernels use (no
 * reference counterpart): D (128 x n) = A (128 x K) B^T (B: n x K), row-major
 * host arrays, as one TF32 product (split 0) or the three-term hi/lo split
 * (split 1), onto dinit (128 x n) when not null.  (kpad, n) in {(8, 16),
 * (32, 32), (40, 48), (48, 144)}, K <= kpad. */
int spoc_tc_selftest(int K, int kpad, int n, int split, const float *A, const float *B,
                     const float *dinit, float *D);
/* Measured throughput of this GPU in TFLOP/s (2 flops per multiply-add);
 * mode 0: FP64 fused multiply-add, mode 1: FP64 separately rounded multiply
 * and add, mode 2: FP32 fused multiply-add. */
int spoc_fp64_peak(int mode, double *tflops);
/* Energy diagnostic that allocates nothing.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc: cudaMalloc and cudaFree are
 * prohibited while a stream is captured into a CUDA graph (default capture
 * mode) and cudaFree synchronises the device, or the host program owns all
 * device memory itself.  The result is the one spoc_energy gives.
 * Every argument is a DEVICE pointer owned by the caller: u, v, h, hb are
 * (ld, ne) fields, vect is (5, ne), pi2 is (ng, nm), wi is [ng], ammo1 is
 * column 1 of the mass matrix ammo [nm]; out receives (ke, pe, mass).  Work
 * is queued on `stream` (0 = legacy default stream) and nothing is allocated:
 * the per-element scratch is a static device array holding at most
 * SPOC_NOALLOC_MAX_NE elements (3 MiB on every GPU that loads the library);
 * larger ne returns SPOC_E_UNSUPPORTED.  The first call on a device (and
 * the first after cudaDeviceReset) looks up that array's device address and
 * should come before any stream capture.  All calls on a device share the
 * array and it keeps the last call's contents (each call overwrites what it
 * reads): calls that overlap on the GPU race on it. */
#define SPOC_NOALLOC_MAX_NE 131072
int spoc_energy_noalloc(int nc, int ng, int ne, int ld, double g0, const double *u,
                        const double *v, const double *h, const double *hb, const double *vect,
                        const double *pi2, const double *wi, const double *ammo1, double *out,
                        void *stream);
/* Message for the last SPOC_E_CUDA / SPOC_E_ARG on this thread. */
const char *spoc_last_error(void);

/* ---- tangent-linear model, adjoint, gradient (no reference counterpart) ----
 * All arrays are HOST arrays (ld, ne).  These calls use the handle's resident
 * state buffers as work space (call spoc_set_state again afterwards).
 * spoc_tlm_rhs: (ou,ov,oh) = J(u,v,hh) (du,dv,dh), J the Jacobian of cal_var.
 * spoc_adj_rhs: (ou,ov,oh) = J(u,v,hh)^T (bu,bv,bh).
 * spoc_tlm_steps: (du,dv,dh) <- the perturbation after nsteps RK4 steps from
 *   the base state (u0,v0,h0).
 * spoc_adj_steps: (bu,bv,bh) <- the adjoint at step 0 of the adjoint given at
 *   step nsteps (recomputing the trajectory from (u0,v0,h0)).
 * spoc_set_observations: nobs points, point o in element elem[o] (1-based)
 *   with basis values basis[o*nm + n] = phi_n(xi_o, eta_o); observed eta
 *   values[t*nobs + o] at RK4 step steps[t].
 * spoc_fwd_window / spoc_bwd_window: the forward / backward pair of the cost
 *   J = 1/2 sum_t sum_o (eta(x_o, step_t) - values[t*nobs+o])^2 over nsteps
 *   RK4 steps from (u0,v0,h0): fwd returns J; bwd returns J and its gradient
 *   with respect to the initial modal coefficients (gu,gv,gh), reversing the
 *   window with binomial checkpointing in `snaps` device snapshots.
 * spoc_adjoint_counters: forward and adjoint RK4 steps run since the last
 *   call (recomputation included).
 * spoc_set_adjoint_sweeps (no reference counterpart): precision of the
 *   forward steps that spoc_fwd_window, spoc_bwd_window, spoc_tlm_steps and
 *   spoc_adj_steps run (the cost sweep, the checkpoint sweeps and the
 *   re-advances of the reversal): SPOC_FP64 (default) or SPOC_MIXED (the
 *   mixed-precision form, built from `tables`, which must be the handle's).
 *   The tangent-linear and adjoint kernels stay FP64; with SPOC_MIXED they
 *   are linearised about the mixed-precision trajectory. */
int spoc_tlm_rhs(spoc_handle *h, int ld, const double *u, const double *v, const double *hh,
                 const double *du, const double *dv, const double *dh, double *ou, double *ov,
                 double *oh);
int spoc_adj_rhs(spoc_handle *h, int ld, const double *u, const double *v, const double *hh,
                 const double *bu, const double *bv, const double *bh, double *ou, double *ov,
                 double *oh);
int spoc_tlm_steps(spoc_handle *h, int ld, const double *u0, const double *v0, const double *h0,
                   double *du, double *dv, double *dh, double dt, int nsteps);
int spoc_adj_steps(spoc_handle *h, int ld, const double *u0, const double *v0, const double *h0,
                   double *bu, double *bv, double *bh, double dt, int nsteps);
int spoc_set_observations(spoc_handle *h, int nobs, const int *elem, const double *basis,
                          int ntimes, const int *steps, const double *values);
int spoc_fwd_window(spoc_handle *h, int ld, const double *u0, const double *v0, const double *h0,
                    double dt, int nsteps, double *cost);
int spoc_bwd_window(spoc_handle *h, int ld, const double *u0, const double *v0, const double *h0,
                    double dt, int nsteps, int snaps, double *cost, double *gu, double *gv,
                    double *gh);
int spoc_adjoint_counters(spoc_handle *h, long long *fwd_steps, long long *adj_steps);
int spoc_set_adjoint_sweeps(spoc_handle *h, const spoc_tables *tables, int precision);

/* ---- Fortran drop-in ----
 * Register the COMMON contents once (after dpotrf), then link this library
 * instead of calvar*.o: cal_var_ has the reference argument list
 * (src/calvarnl_fs.f:9-12) with gfortran's by-reference, trailing-underscore
 * ABI.  A handle is created on the first call and reused while nf, ne, a
 * content key of the mesh arrays (tseg, ssit, itm, its, bdl, norm, vect,
 * normt: the adaptive driver rewrites them in place at a regrid) and the
 * addresses of fc, w0, z0, hb are unchanged; spoc_cal_var_refresh() makes the
 * next call upload everything (fields rewritten in place on the same mesh).
 * Errors set *spoc_cal_var_status() (the reference `stop`s instead). */
int spoc_register_commons(const spoc_tables *tables, int variant, int precision);
void cal_var_(int *nf, int *ne, double *u0, double *v0, double *h0, double *u1, double *v1,
              double *h1, int *tseg, int *pseg, int *ssit, int *itm, int *its, double *norm,
              int *nbdl, int *pbdl, int *nint, int *pint, int *bdl, int *cip, double *vect,
              double *normt, double *mu0, double *mb0, double *fc, double *beta, double *w0,
              double *z0, double *g0, double *hb, double *time);
int *spoc_cal_var_status(void);
void spoc_cal_var_refresh(void);
void spoc_release_commons(void);

/* ---- host set-up helpers (no CUDA) ----
 * Tables: read_gauss values in, then cal_p2 (src/nonlin.f:10-30), cal_pico
 * (src/mat1.f:214-259), calip (src/mat1.f:383-410), cal_mat x5
 * (src/mat1.f:90-142), cal_matl (src/mat1.f:285-368) and the two dpotrf
 * (src/shwwnl.f:153-156).  Output arrays, caller-allocated:
 *   pi2[ng*nm] (ld ng), pico[ngf*nm*3] (ld ngf, nm), amm/amml/agx/agy/ammo/
 *   ammx/ammy[nm*nm] (ld nm), cip[2*(nc+1)].
 * Returns 0, or SPOC_E_MATRIX with *info = the dpotrf info (column of failure,
 * +1000 for amml). */
int spoc_build_tables(int nc, int ng, int ngf, const double *wi, const double *xi,
                      const double *yi, const double *wif, const double *tif, double *pi2,
                      double *pico, double *amm, double *amml, double *agx, double *agy,
                      double *ammo, double *ammx, double *ammy, int *cip, int *info);
/* Mesh pointers: pointer_mesh (src/cmal_s.f:88-216), check_mesh (:222-277),
 * cal_rotnf (src/mat1.f:7-23), cal_its (:28-64), calpre (src/shwwnl.f:350-422)
 * and coriolis (src/mat1.f:69-83).  Face arrays are sized for nfmax faces
 * (3*ne suffices); fc is (ld, ne) and is zeroed first. */
int spoc_build_mesh(int nn, int ne, const int *in, const double *xgr, const double *ygr,
                    int nc, double f0, double beta, int nfmax, int *nf, int *itm, int *its,
                    int *tseg, int *pseg, int *ssit, double *norm, double *vect, double *normt,
                    int *bdl, double *fc, int ld);
/* Corner fix of src/chmal.f:240-330: flip the diagonal of each element with
 * two wall faces, then rotate local numbering so a wall face is side 1. */
int spoc_fix_mesh(int nn, int ne, int *in);
/* L2 projection of calh (src/init.f:290-344): vals(ng, ne) are the function at
 * the points returned by spoc_projection_points; out is (ld, ne).  amm is the
 * Cholesky factor from spoc_build_tables. */
int spoc_projection_points(int ne, const int *in, const double *xgr, const double *ygr, int ng,
                           const double *xi, const double *yi, double *px, double *py);
int spoc_project(int nc, int ng, const double *wi, const double *pi2, const double *amm,
                 int ne, const double *vals, double *out, int ld);
/* Regridding set-up on the host.  inter_only_new (src/adapt.f:1233-1258):
 * tinter[i] = the old element (1-based) new element i repeats, else 0.
 * Point location of interpol (src/adapt.f:1690-1718, interlin :1747-1830):
 * the quadrature points of every new element with tinter == 0 located in the
 * old mesh (arrays of spoc_build_mesh), the walk continuing from the previous
 * point's element; pt_elem / pt_x / pt_y are (ng, nenew).  SPOC_E_MESH when a
 * walk does not end. */
int spoc_inter_only_new(int ne, int nenew, const int *in, const int *innew, int *tinter);
/* Sequential point location of compare.f (src/compare.f:118-150): interlin
 * from *tk (updated) for each point; coordinates summing below 0.5 count as
 * outside (inside[i] = 0) and restart the walk at reset_tk. */
int spoc_locate_xy(int ne, const int *in, const int *itm, const int *tseg, const int *pseg,
                   const double *xgr, const double *ygr, int npts, const double *px,
                   const double *py, int *tk, int reset_tk, int *elem, double *x1, double *y1,
                   int *inside);
int spoc_locate_points(int ne, const int *in, const int *itm, const int *tseg, const int *pseg,
                       const double *xgr, const double *ygr, int nenew, const int *innew,
                       const double *xgrnew, const double *ygrnew, const int *tinter, int ng,
                       const double *xi, const double *yi, int *pt_elem, double *pt_x,
                       double *pt_y);

#ifdef __cplusplus
}
#endif
#endif /* SPOC_GPU_H */
