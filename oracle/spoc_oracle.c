/*
 * CPU oracle for the SPOC RK4 DG shallow-water path -- TEST INFRASTRUCTURE.
 *
 * Restates the reference Fortran routines in their loop and summation order.
 * Each function names the reference file:line it follows.  Build with
 * -O2 -ffp-contract=off (see oracle/Makefile): no fused multiply-adds, so the
 * serial and OpenMP builds are bit-identical (element and face loops carry no
 * cross-iteration reductions).  Parity with reference output is unpinned (the
 * reference ships no golden data and cannot be compiled here); the oracle is
 * pinned by known-answer tests in tests/.
 */
#include "spoc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Contraction precision: 64 (default) evaluates the reference in double; 32
 * rounds both operands of every contraction (cal_b, spectoxy, xytospec,
 * cal_flu, tri_f) to float and accumulates in float, leaving the solves, the
 * pointwise terms and RK4 in double.  32 models the best case of a tensor-core
 * form that computes the contractions to FP32 accuracy (TF32 with a hi/lo
 * split); it exists to measure how the mass solves amplify that error. */
static int g_contract32 = 0;
void ora_set_contraction_precision(int bits) { g_contract32 = (bits == 32); }

#define NNMAX 66   /* local vector capacity: degree <= 10 */
#define NGMAX 80   /* triangle quadrature points */
#define NGFMAX 16  /* edge quadrature points */

/* 1-based column-major accessors */
#define M2(a, ld, i, j) ((a)[((size_t)(j) - 1) * (size_t)(ld) + (size_t)(i) - 1])
#define I2(a, i, j, n1) ((a)[((size_t)(j) - 1) * (size_t)(n1) + (size_t)(i) - 1])
#define PICO(c, j, i1, k) \
  ((c)->pico[(((size_t)(k) - 1) * (size_t)(c)->ldp + (size_t)(i1) - 1) * (size_t)(c)->ldg + (size_t)(j) - 1])
#define PI2(c, i, i1) ((c)->pi2[((size_t)(i1) - 1) * (size_t)(c)->ldq + (size_t)(i) - 1])
#define CIP(cip, r, j) ((cip)[2 * (j) + (r) - 1])

/* ------------------------------------------------------------------ */
/* Legendre polynomial and derivative: src/legendre2.f:5-30, :32-62     */
/* ------------------------------------------------------------------ */
double ora_po(int n, double x) {
  double p0 = 1.0, p1 = x, po = 0.0;
  if (n == 0) po = p0;
  if (n == 1) {
    po = p1;
  } else {
    int i = 1;
    while (i < n) {
      i = i + 1;
      double a0 = (double)i, a2 = (double)(2 * i - 1), a3 = (double)(i - 1);
      po = (a2 * x * p1 - a3 * p0) / a0;
      p0 = p1;
      p1 = po;
    }
  }
  return po;
}

double ora_dpo(int n, double x) {
  double p0 = 1.0, p1 = x, dp0 = 0.0, dp1 = 1.0, dpo = 0.0;
  if (n == 0) dpo = dp0;
  if (n == 1) {
    dpo = dp1;
  } else {
    int i = 1;
    while (i < n) {
      i = i + 1;
      double a0 = (double)i, a2 = (double)(2 * i - 1), a3 = (double)(i - 1);
      dpo = (a2 * x * dp1 + a2 * p1 - a3 * dp0) / a0;
      double p2 = (a2 * x * p1 - a3 * p0) / a0;
      p0 = p1;
      p1 = p2;
      dp0 = dp1;
      dp1 = dpo;
    }
  }
  return dpo;
}

/* cal_p2: src/nonlin.f:10-30 */
void ora_cal_p2(int nc, int ng, const double *xi, const double *yi, double *pi2, int ldq) {
  int i1 = 0;
  for (int kc1 = 0; kc1 <= nc; kc1++)
    for (int kc2 = 0; kc2 <= nc - kc1; kc2++) {
      i1++;
      for (int i = 1; i <= ng; i++) {
        double y = yi[i - 1], x = xi[i - 1];
        M2(pi2, ldq, i, i1) = ora_po(kc1, x) * ora_po(kc2, y);
      }
    }
}

/* cal_pico: src/mat1.f:214-259 (side 1: (t,-1); side 2: (-t,t); side 3: (-1,-t)) */
void ora_cal_pico(int nc, int ngf, const double *ti, double *pico, int ldg, int ldp) {
#define PK(j, i1, k) pico[(((size_t)(k) - 1) * (size_t)ldp + (size_t)(i1) - 1) * (size_t)ldg + (size_t)(j) - 1]
  int i1 = 0;
  for (int kc1 = 0; kc1 <= nc; kc1++)
    for (int kc2 = 0; kc2 <= nc - kc1; kc2++) {
      i1++;
      for (int j = 1; j <= ngf; j++) {
        double x = ti[j - 1], y = -1.0;
        PK(j, i1, 1) = ora_po(kc1, x) * ora_po(kc2, y);
      }
    }
  i1 = 0;
  for (int kc1 = 0; kc1 <= nc; kc1++)
    for (int kc2 = 0; kc2 <= nc - kc1; kc2++) {
      i1++;
      for (int j = 1; j <= ngf; j++) {
        double x = -ti[j - 1], y = ti[j - 1];
        PK(j, i1, 2) = ora_po(kc1, x) * ora_po(kc2, y);
      }
    }
  i1 = 0;
  for (int kc1 = 0; kc1 <= nc; kc1++)
    for (int kc2 = 0; kc2 <= nc - kc1; kc2++) {
      i1++;
      for (int j = 1; j <= ngf; j++) {
        double x = -1.0, y = -ti[j - 1];
        PK(j, i1, 3) = ora_po(kc1, x) * ora_po(kc2, y);
      }
    }
#undef PK
}

/* calip: src/mat1.f:383-410 */
void ora_calip(int nc, int *cip) {
  for (int i = 0; i <= nc; i++) {
    int ip = 0, j = 0;
    while (j < i) {
      ip = ip + nc + 1 - j;
      j++;
    }
    CIP(cip, 1, i) = ip;
  }
  int nc2 = nc - 1;
  for (int i = 0; i <= nc2; i++) {
    int ip = 0, j = 0;
    while (j < i) {
      ip = ip + nc2 + 1 - j;
      j++;
    }
    CIP(cip, 2, i) = ip;
  }
  if (nc2 + 1 <= nc) CIP(cip, 2, nc) = 0;
}

/* integrands f2/fx/fy/dfx/dfy: src/mat1.f:513-576 */
static double integrand(int which, int kc1, int kc2, int kc3, int kc4, double x, double y) {
  switch (which) {
    case 0: return ora_po(kc1, x) * ora_po(kc2, y) * ora_po(kc3, x) * ora_po(kc4, y);
    case 1: return ora_po(kc1, x) * ora_po(kc2, y) * ora_po(kc3, x) * ora_po(kc4, y) * x;
    case 2: return ora_po(kc1, x) * ora_po(kc2, y) * ora_po(kc3, x) * ora_po(kc4, y) * y;
    case 3: return ora_po(kc1, x) * ora_po(kc2, y) * ora_dpo(kc3, x) * ora_po(kc4, y);
    default: return ora_po(kc1, x) * ora_po(kc2, y) * ora_po(kc3, x) * ora_dpo(kc4, y);
  }
}

/* cal_mat + inttri: src/mat1.f:90-142, :266-279.  mat(i1,i2) = sum_q w_q phi_i1 op(phi_i2) */
void ora_cal_mat(int nc, int ng, int which, const double *xi, const double *yi,
                 const double *wi, double *mat, int ldm) {
  int nm = (nc + 1) * (nc + 2) / 2;
  for (int j = 1; j <= nm; j++)
    for (int i = 1; i <= nm; i++) M2(mat, ldm, i, j) = 0.0;
  int i1 = 0;
  for (int kc1 = 0; kc1 <= nc; kc1++)
    for (int kc2 = 0; kc2 <= nc - kc1; kc2++) {
      i1++;
      int i2 = 0;
      for (int kc3 = 0; kc3 <= nc; kc3++)
        for (int kc4 = 0; kc4 <= nc - kc3; kc4++) {
          i2++;
          double ans = 0.0;
          for (int j = 1; j <= ng; j++) {
            double y = yi[j - 1], x = xi[j - 1];
            ans = ans + wi[j - 1] * integrand(which, kc1, kc2, kc3, kc4, x, y);
          }
          M2(mat, ldm, i1, i2) = ans;
        }
    }
}

/* ip: src/mat1.f:372-381 */
static int ip_(int nc, int i) {
  int ip = 0, j = 0;
  while (j < i) {
    ip = ip + nc + 1 - j;
    j++;
  }
  return ip;
}

/* cal_matl: src/mat1.f:285-368 (mass matrix of the basis vanishing on side 1) */
void ora_cal_matl(int nc, const double *amm, double *amml, int ldm) {
  for (int pass = 0; pass < 4; pass++) {
    int j0s = (pass == 1 || pass == 3) ? 1 : 0;
    int l0s = (pass == 2 || pass == 3) ? 1 : 0;
    for (int i = 0; i <= nc - 1; i++)
      for (int j = j0s; j <= nc - 1 - i; j += 2)
        for (int k = 0; k <= nc - 1; k++)
          for (int l = l0s; l <= nc - 1 - k; l += 2) {
            int i1 = ip_(nc - 1, i) + j + 1;
            int i2 = ip_(nc, i) + j + 2;
            int j1 = ip_(nc - 1, k) + l + 1;
            int j2 = ip_(nc, k) + l + 2;
            int i0 = ip_(nc, i) + 1;
            int jj0 = ip_(nc, k) + 1;
            double v;
            if (pass == 0)
              v = M2(amm, ldm, i2, j2) + M2(amm, ldm, i0, j2) + M2(amm, ldm, i2, jj0) + M2(amm, ldm, i0, jj0);
            else if (pass == 1)
              v = M2(amm, ldm, i2, j2) - M2(amm, ldm, i0, j2) + M2(amm, ldm, i2, jj0) - M2(amm, ldm, i0, jj0);
            else if (pass == 2)
              v = M2(amm, ldm, i2, j2) + M2(amm, ldm, i0, j2) - M2(amm, ldm, i2, jj0) - M2(amm, ldm, i0, jj0);
            else
              v = M2(amm, ldm, i2, j2) - M2(amm, ldm, i0, j2) - M2(amm, ldm, i2, jj0) + M2(amm, ldm, i0, jj0);
            M2(amml, ldm, i1, j1) = v;
          }
  }
}

/* DPOTF2 upper: src/solve.f:276-440, with the vendored DDOT (src/solve.f:1378,
 * unrolled by 5 but accumulated left to right, i.e. sequentially), DGEMV 'T'
 * (src/solve2.f:314, column dot products then y += alpha*temp) and DSCAL
 * (src/solve2.f:575, stride lda). */
int ora_dpotf2_upper(int n, double *a, int lda) {
  for (int j = 1; j <= n; j++) {
    double dot = 0.0;
    for (int k = 1; k <= j - 1; k++) dot = dot + M2(a, lda, k, j) * M2(a, lda, k, j);
    double ajj = M2(a, lda, j, j) - dot;
    if (ajj <= 0.0) {
      M2(a, lda, j, j) = ajj;
      return j;
    }
    ajj = sqrt(ajj);
    M2(a, lda, j, j) = ajj;
    if (j < n) {
      /* DGEMV('T', j-1, n-j, -1, A(1,j+1), lda, A(1,j), 1, 1, A(j,j+1), lda) */
      for (int jj = j + 1; jj <= n; jj++) {
        double temp = 0.0;
        for (int i = 1; i <= j - 1; i++) temp = temp + M2(a, lda, i, jj) * M2(a, lda, i, j);
        M2(a, lda, j, jj) = M2(a, lda, j, jj) + (-1.0) * temp;
      }
      double r = 1.0 / ajj;
      for (int jj = j + 1; jj <= n; jj++) M2(a, lda, j, jj) = r * M2(a, lda, j, jj);
    }
  }
  return 0;
}

/* DTRSM4: src/dtrsm1.f:47-82.  b := (U^T U)^{-1} b, diag = 1/diag(U). */
void ora_dtrsm4(int m, const double *a, int lda, double *b, const double *diag) {
  for (int i = 1; i <= m; i++) {
    double temp = b[i - 1];
    for (int k = 1; k <= i - 1; k++) temp = temp - M2(a, lda, k, i) * b[k - 1];
    temp = temp * diag[i - 1];
    b[i - 1] = temp;
  }
  for (int k = m; k >= 1; k--) {
    b[k - 1] = b[k - 1] * diag[k - 1];
    for (int i = 1; i <= k - 1; i++) b[i - 1] = b[i - 1] - b[k - 1] * M2(a, lda, i, k);
  }
}

/* ------------------------------------------------------------------ */
/* Mesh pointers: src/cmal_s.f:88-216, :222-277; src/mat1.f:7-83      */
/* ------------------------------------------------------------------ */

/* pointer_mesh: node->element lists (tmit/imit, sorted by element), then a face
 * search over earlier elements around the end node of each side
 * (src/cmal_s.f:164-208).  Faces are numbered in order of first appearance.
 * Returns nf, or -1 if nfmax is exceeded. */
int ora_pointer_mesh(int nn, int ne, const int *in, int *itm, int *tseg, int *pseg, int nfmax) {
  int *cnt = (int *)calloc((size_t)nn + 2, sizeof(int));
  int *nmit = (int *)calloc((size_t)nn + 2, sizeof(int));
  int *tmit = (int *)malloc(sizeof(int) * (3 * (size_t)ne + 2));
  int *imit = (int *)malloc(sizeof(int) * (3 * (size_t)ne + 2));
  for (int i = 1; i <= ne; i++)
    for (int k = 1; k <= 3; k++) cnt[I2(in, k, i, 3)]++;
  nmit[1] = 1;
  for (int i = 1; i <= nn; i++) nmit[i + 1] = nmit[i] + cnt[i];
  int *fill = (int *)malloc(sizeof(int) * ((size_t)nn + 2));
  for (int i = 1; i <= nn + 1; i++) fill[i] = nmit[i];
  for (int i = 1; i <= ne; i++)
    for (int k = 1; k <= 3; k++) {
      int n1 = I2(in, k, i, 3);
      tmit[fill[n1]] = i;
      imit[fill[n1]] = k;
      fill[n1]++;
    }
  /* sentinel: the list of the end node always contains the current element
   * itself, so the search below stops inside the list; guard anyway. */
  tmit[3 * ne + 1] = ne + 1;
  imit[3 * ne + 1] = 1;
  for (int i = 1; i <= nfmax; i++) {
    I2(tseg, 1, i, 2) = 0;
    I2(tseg, 2, i, 2) = 0;
  }
  int nf = 0;
  for (int i = 1; i <= ne; i++) {
    for (int j = 1; j <= 3; j++) {
      int ne1 = I2(in, j, i, 3);
      int ne2 = (j == 3) ? I2(in, 1, i, 3) : I2(in, j + 1, i, 3);
      int k = nmit[ne2];
      int tk = tmit[k];
      int trouve = 1;
      int ik = imit[k];
      while (tk < i && trouve) {
        int ne3 = (ik + 1 < 4) ? I2(in, ik + 1, tk, 3) : I2(in, 1, tk, 3);
        if (ne1 == ne3) {
          int lk = I2(itm, ik, tk, 3);
          I2(tseg, 2, lk, 2) = i;
          I2(itm, j, i, 3) = lk;
          trouve = 0;
        }
        k++;
        tk = tmit[k];
        ik = imit[k];
      }
      if (trouve) {
        nf++;
        if (nf > nfmax) {
          free(cnt); free(nmit); free(tmit); free(imit); free(fill);
          return -1;
        }
        I2(itm, j, i, 3) = nf;
        I2(tseg, 1, nf, 2) = i;
        I2(pseg, 1, nf, 2) = ne1;
        I2(pseg, 2, nf, 2) = ne2;
      }
    }
  }
  free(cnt); free(nmit); free(tmit); free(imit); free(fill);
  return nf;
}

/* check_mesh: src/cmal_s.f:222-277.  0 ok; 1 an element has >1 wall face;
 * 2 a wall face is not side 1 of its element (the reference only warns). */
int ora_check_mesh(int ne, int nf, const int *itm, const int *tseg) {
  int *pebd = (int *)calloc((size_t)ne + 1, sizeof(int));
  int rc = 0;
  for (int i = 1; i <= nf; i++)
    if (I2(tseg, 2, i, 2) == 0) pebd[I2(tseg, 1, i, 2)]++;
  for (int i = 1; i <= ne; i++)
    if (pebd[i] > 1) rc = 1;
  if (!rc)
    for (int i = 1; i <= nf; i++)
      if (I2(tseg, 2, i, 2) == 0) {
        int tk = I2(tseg, 1, i, 2), j = 1;
        while (j <= 3 && I2(itm, j, tk, 3) != i) j++;
        if (j != 1) rc = 2;
      }
  free(pebd);
  return rc;
}

/* cal_rotnf: src/mat1.f:7-23 */
void ora_cal_rotnf(int nf, const double *x, const double *y, double *norm, const int *pseg) {
  for (int i = 1; i <= nf; i++) {
    int ne1 = I2(pseg, 1, i, 2), ne2 = I2(pseg, 2, i, 2);
    double nx = (y[ne2 - 1] - y[ne1 - 1]);
    double ny = -(x[ne2 - 1] - x[ne1 - 1]);
    I2(norm, 1, i, 2) = nx;
    I2(norm, 2, i, 2) = ny;
  }
}

/* cal_its: src/mat1.f:28-64.  Returns 0, or the face id with bad connectivity. */
int ora_cal_its(int nf, const int *itm, int *its, const int *tseg, int *ssit) {
  for (int i = 1; i <= nf; i++) {
    I2(ssit, 1, i, 2) = 0;
    I2(ssit, 2, i, 2) = 0;
  }
  for (int i = 1; i <= nf; i++) {
    int tk = I2(tseg, 1, i, 2);
    int j = 1;
    while (j < 4 && I2(itm, j, tk, 3) != i) j++;
    if (j == 4) return i;
    I2(its, j, tk, 3) = 1;
    I2(ssit, 1, i, 2) = j;
    tk = I2(tseg, 2, i, 2);
    if (tk > 0) {
      j = 1;
      while (j < 4 && I2(itm, j, tk, 3) != i) j++;
      if (j == 4) return i;
      I2(its, j, tk, 3) = -1;
      I2(ssit, 2, i, 2) = j;
    }
  }
  return 0;
}

/* calpre: src/shwwnl.f:350-422 (no NBEDIM limit: arrays are sized by the caller) */
void ora_calpre(int nn, int ne, int nf, const int *in, const double *xgr, const double *ygr,
                double *vect, const int *itm, const double *norm, double *normt, int *bdl,
                int *nint, int *pint, int *nbdl, int *pbdl, int *nebd, const int *tseg,
                const int *pseg) {
  (void)nn; (void)pseg;
  for (int i = 1; i <= ne; i++) bdl[i - 1] = 0;
  *nebd = 0;
  for (int i = 1; i <= nf; i++)
    if (I2(tseg, 2, i, 2) == 0) {
      (*nebd)++;
      bdl[I2(tseg, 1, i, 2) - 1] = 1;
    }
  for (int i = 1; i <= ne; i++) {
    int i1 = I2(in, 1, i, 3), i2 = I2(in, 2, i, 3), i3 = I2(in, 3, i, 3);
    double ax = (xgr[i2 - 1] - xgr[i1 - 1]) * 0.5;
    double bx = (xgr[i3 - 1] - xgr[i1 - 1]) * 0.5;
    double ay = (ygr[i2 - 1] - ygr[i1 - 1]) * 0.5;
    double by = (ygr[i3 - 1] - ygr[i1 - 1]) * 0.5;
    double deta = ax * by - ay * bx;
    double detai = 1.0 / deta;
    I2(vect, 1, i, 5) = ax;
    I2(vect, 2, i, 5) = bx;
    I2(vect, 3, i, 5) = ay;
    I2(vect, 4, i, 5) = by;
    I2(vect, 5, i, 5) = detai;
    int ns1 = I2(itm, 1, i, 3);
    double dnx = I2(norm, 1, ns1, 2), dny = I2(norm, 2, ns1, 2);
    double dis = sqrt(dnx * dnx + dny * dny);
    dnx = dnx / dis;
    dny = dny / dis;
    I2(normt, 1, i, 2) = dnx;
    I2(normt, 2, i, 2) = dny;
  }
  *nbdl = 0;
  *nint = 0;
  for (int i = 1; i <= ne; i++) {
    if (bdl[i - 1]) {
      (*nbdl)++;
      pbdl[*nbdl - 1] = i;
    } else {
      (*nint)++;
      pint[*nint - 1] = i;
    }
  }
}

/* coriolis: src/mat1.f:69-83 (fc must be zeroed by the caller, as the
 * reference relies on zero-initialised static storage) */
void ora_coriolis(int nc, int ne, const int *in, const double *xgr, const double *ygr,
                  double *fc, int ld, double f0, double beta) {
  (void)xgr;
  for (int i = 1; i <= ne; i++) {
    int n1 = I2(in, 1, i, 3), n2 = I2(in, 2, i, 3), n3 = I2(in, 3, i, 3);
    M2(fc, ld, 1, i) = f0 + 0.5 * beta * (ygr[n3 - 1] + ygr[n2 - 1]);
    M2(fc, ld, 2, i) = 0.5 * beta * (ygr[n3 - 1] - ygr[n1 - 1]);
    M2(fc, ld, nc + 2, i) = 0.5 * beta * (ygr[n2 - 1] - ygr[n1 - 1]);
  }
}

/* cit: src/chmal.f:334-342 */
static int cit_(int n, int k, int np) {
  int k1 = k + np;
  if (k1 > n) k1 -= n;
  if (k1 < 1) k1 += n;
  return k1;
}

/* changemaille: src/chmal.f:240-330.  Flips the diagonal of every element with
 * two wall faces, then rotates local numbering so the wall face is side 1.
 * Operates on in/itm/tseg/pseg from ora_pointer_mesh; only `in` is meaningful
 * afterwards (the reference saves it and recomputes the pointers).
 * Returns 0, or -1 if a search leaves the element (malformed input). */
int ora_changemaille(int nn, int ne, int nf, int *in, int *itm, int *tseg, int *pseg) {
  (void)nn;
  int nfbd = 0;
  int *sbd = (int *)malloc(sizeof(int) * ((size_t)nf + 1));
  int *pebd = (int *)calloc((size_t)ne + 1, sizeof(int));
  for (int i = 1; i <= nf; i++)
    if (I2(tseg, 2, i, 2) == 0) sbd[++nfbd] = i;
  for (int i = 1; i <= nfbd; i++) pebd[I2(tseg, 1, sbd[i], 2)]++;
  int rc = 0;
  for (int i = 1; i <= ne && !rc; i++) {
    if (pebd[i] > 1) {
      int j = 1, ns1 = I2(itm, j, i, 3);
      while (I2(tseg, 2, ns1, 2) == 0) {
        j++;
        if (j > 3) { rc = -1; break; }
        ns1 = I2(itm, j, i, 3);
      }
      if (rc) break;
      int tk1 = I2(tseg, 1, ns1, 2), tk2 = I2(tseg, 2, ns1, 2);
      int j1 = 1;
      while (j1 <= 3 && I2(itm, j1, tk1, 3) != ns1) j1++;
      int j2 = 1;
      while (j2 <= 3 && I2(itm, j2, tk2, 3) != ns1) j2++;
      if (j1 > 3 || j2 > 3) { rc = -1; break; }
      int k1 = cit_(3, j1, 1), k2 = cit_(3, j2, -1), k3 = cit_(3, j2, 1), k4 = cit_(3, j1, -1);
      int i2 = I2(in, k2, tk2, 3);
      int i4 = I2(in, k4, tk1, 3);
      I2(in, k1, tk1, 3) = i2;
      I2(in, k3, tk2, 3) = i4;
      I2(itm, j1, tk1, 3) = I2(itm, k3, tk2, 3);
      I2(itm, j2, tk2, 3) = I2(itm, k1, tk1, 3);
      I2(itm, k1, tk1, 3) = ns1;
      I2(itm, k3, tk2, 3) = ns1;
      I2(pseg, 1, ns1, 2) = i2;
      I2(pseg, 2, ns1, 2) = i4;
      if (i == tk1)
        I2(tseg, 1, I2(itm, j2, tk2, 3), 2) = tk2;
      else
        I2(tseg, 1, I2(itm, j1, tk1, 3), 2) = tk1;
    }
  }
  for (int i = 1; i <= nfbd && !rc; i++) {
    int ns1 = sbd[i], tk1 = I2(tseg, 1, ns1, 2), j = 1;
    while (j <= 3 && I2(itm, j, tk1, 3) != ns1) j++;
    if (j > 3) { rc = -1; break; }
    int pp[3], pf[3];
    for (int k = 1; k <= 3; k++) {
      int l = cit_(3, k, j - 1);
      pp[k - 1] = I2(in, l, tk1, 3);
      pf[k - 1] = I2(itm, l, tk1, 3);
    }
    for (int k = 1; k <= 3; k++) {
      I2(in, k, tk1, 3) = pp[k - 1];
      I2(itm, k, tk1, 3) = pf[k - 1];
    }
  }
  free(sbd);
  free(pebd);
  return rc;
}

/* ------------------------------------------------------------------ */
/* L1 hot kernels                                                      */
/* ------------------------------------------------------------------ */

/* cal_flu: src/calflu.f:6-71 (central trace at the ngf edge points) */
void ora_cal_flu(const ora_common *c, int nf, const int *tseg, double *fbdy, int ldf,
                 const double *a0, int ld, const int *ssit, int nthreads) {
  const int nm = c->nm, ngf = c->ngf;
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
  for (int i = 1; i <= nf; i++) {
    for (int j = 1; j <= ngf; j++) M2(fbdy, ldf, j, i) = 0.0;
    int k1 = I2(tseg, 1, i, 2), k2 = I2(tseg, 2, i, 2);
    if (g_contract32) {
      for (int j = 1; j <= ngf; j++) {
        float t1 = 0.f, t2 = 0.f;
        int s1 = k2 == 0 ? 1 : I2(ssit, 1, i, 2);
        for (int i1 = 1; i1 <= nm; i1++) t1 = t1 + (float)M2(a0, ld, i1, k1) * (float)PICO(c, j, i1, s1);
        if (k2 != 0) {
          int s2 = I2(ssit, 2, i, 2);
          for (int i1 = 1; i1 <= nm; i1++)
            t2 = t2 + (float)M2(a0, ld, i1, k2) * (float)PICO(c, ngf - j + 1, i1, s2);
          M2(fbdy, ldf, j, i) = 0.5f * (t1 + t2);
        } else {
          M2(fbdy, ldf, j, i) = t1;
        }
      }
      continue;
    }
    if (k2 == 0) {
      for (int i1 = 1; i1 <= nm; i1++)
        for (int j = 1; j <= ngf; j++)
          M2(fbdy, ldf, j, i) = M2(fbdy, ldf, j, i) + M2(a0, ld, i1, k1) * PICO(c, j, i1, 1);
    } else {
      int cote = I2(ssit, 1, i, 2);
      for (int i1 = 1; i1 <= nm; i1++)
        for (int j = 1; j <= ngf; j++)
          M2(fbdy, ldf, j, i) = M2(fbdy, ldf, j, i) + M2(a0, ld, i1, k1) * PICO(c, j, i1, cote);
      cote = I2(ssit, 2, i, 2);
      for (int i1 = 1; i1 <= nm; i1++)
        for (int j = 1; j <= ngf; j++)
          M2(fbdy, ldf, j, i) = M2(fbdy, ldf, j, i) + M2(a0, ld, i1, k2) * PICO(c, ngf - j + 1, i1, cote);
      for (int j = 1; j <= ngf; j++) M2(fbdy, ldf, j, i) = 0.5 * M2(fbdy, ldf, j, i);
    }
  }
}

/* tri_f: src/mat1.f:172-209 (lift of the three face fluxes) */
void ora_tri_f(const ora_common *c, int tk, const int *itm, const int *its,
               const double *fbdy, int ldf, double *b, double coeff) {
  const int nm = c->nm, ngf = c->ngf;
  for (int k = 1; k <= 3; k++) {
    int ns1 = I2(itm, k, tk, 3);
    int isg = I2(its, k, tk, 3);
    int isg2 = (ngf + 1) * (1 - isg) / 2;
    double sig = (double)isg * coeff * 0.5;
    for (int i1 = 1; i1 <= nm; i1++) {
      double ans = 0.0;
      if (g_contract32) {
        float a = 0.f;
        for (int j = 1; j <= ngf; j++) {
          int j1 = isg2 + isg * j;
          a = a + (float)(c->wif[j - 1] * PICO(c, j1, i1, k)) * (float)M2(fbdy, ldf, j, ns1);
        }
        ans = a;
      } else
      for (int j = 1; j <= ngf; j++) {
        int j1 = isg2 + isg * j;
        double var = PICO(c, j1, i1, k) * M2(fbdy, ldf, j, ns1);
        ans = ans + c->wif[j - 1] * var;
      }
      b[i1 - 1] = b[i1 - 1] + ans * sig;
    }
  }
}

/* cal_b: src/calb2.f:3-24  (b += coeff * mat^T ak) */
void ora_cal_b(const ora_common *c, double *b, const double *ak, const double *mat, double coeff) {
  const int nm = c->nm, ldm = c->ldm;
  for (int i = 1; i <= nm; i++) {
    double ans = 0.0;
    if (g_contract32) {
      float a = 0.f;
      for (int j = 1; j <= nm; j++) a = a + (float)M2(mat, ldm, j, i) * (float)ak[j - 1];
      ans = a;
    } else {
      for (int j = 1; j <= nm; j++) ans = ans + M2(mat, ldm, j, i) * ak[j - 1];
    }
    b[i - 1] = b[i - 1] + ans * coeff;
  }
}

/* spectoxy: src/nonlin.f:62-86 */
void ora_spectoxy(const ora_common *c, double *mff, const double *ak) {
  const int ng = c->ng, nm = c->nm;
  for (int j = 1; j <= ng; j++) mff[j - 1] = 0.0;
  if (g_contract32) {
    for (int j = 1; j <= ng; j++) {
      float a = 0.f;
      for (int i1 = 1; i1 <= nm; i1++) a = a + (float)ak[i1 - 1] * (float)PI2(c, j, i1);
      mff[j - 1] = a;
    }
    return;
  }
  for (int i1 = 1; i1 <= nm; i1++)
    for (int j = 1; j <= ng; j++) mff[j - 1] = mff[j - 1] + ak[i1 - 1] * PI2(c, j, i1);
}

/* xytospec + inttri2: src/nonlin.f:35-57, :91-107 */
void ora_xytospec(const ora_common *c, double *b, const double *mff) {
  const int ng = c->ng, nm = c->nm;
  for (int i1 = 1; i1 <= nm; i1++) {
    double ans = 0.0;
    if (g_contract32) {
      float a = 0.f;
      for (int i = 1; i <= ng; i++) a = a + (float)(c->wi[i - 1] * mff[i - 1]) * (float)PI2(c, i, i1);
      ans = a;
    } else {
      for (int i = 1; i <= ng; i++) ans = ans + c->wi[i - 1] * mff[i - 1] * PI2(c, i, i1);
    }
    b[i1 - 1] = ans;
  }
}

/* multiply / divide: src/nonlin.f:111-133 */
static void multiply_(int ng, double *mff, const double *m1, const double *m2) {
  for (int j = 0; j < ng; j++) mff[j] = m1[j] * m2[j];
}
static void divide_(int ng, double *mff, const double *m1, const double *m2) {
  for (int j = 0; j < ng; j++) mff[j] = m1[j] / m2[j];
}

/* reduc_gn: src/mat1.f:418-439 */
void ora_reduc_gn(int nc, const double *gn, double *gnr, const int *cip) {
  for (int j = 0; j <= nc - 1; j++) {
    int ind0 = CIP(cip, 1, j) + 1;
    for (int l = 0; l <= nc - 1 - j; l += 2) {
      int k = CIP(cip, 1, j) + l + 2, ind = CIP(cip, 2, j) + l + 1;
      gnr[ind - 1] = gn[k - 1] + gn[ind0 - 1];
    }
    for (int l = 1; l <= nc - 1 - j; l += 2) {
      int k = CIP(cip, 1, j) + l + 2, ind = CIP(cip, 2, j) + l + 1;
      gnr[ind - 1] = gn[k - 1] - gn[ind0 - 1];
    }
  }
}

/* reduc_inv_gn: src/mat1.f:445-473 */
void ora_reduc_inv_gn(int nc, double *gn, const double *gnr, const int *cip) {
  int nm = (nc + 1) * (nc + 2) / 2;
  for (int j = 0; j <= nc - 1; j++) {
    int k = CIP(cip, 1, j) + 1;
    gn[k - 1] = 0.0;
    for (int l = 0; l <= nc - j - 1; l += 2) gn[k - 1] = gn[k - 1] + gnr[CIP(cip, 2, j) + l];
    for (int l = 1; l <= nc - j - 1; l += 2) gn[k - 1] = gn[k - 1] - gnr[CIP(cip, 2, j) + l];
    for (int l = 0; l <= nc - j - 1; l++) {
      k = CIP(cip, 1, j) + l + 2;
      gn[k - 1] = gnr[CIP(cip, 2, j) + l];
    }
  }
  gn[nm - 1] = 0.0;
}

/* rot_vec: src/mat1.f:478-488 */
static void rot_vec_(int nm, double *gn, double *gt, const double *gx, const double *gy,
                     double dnx, double dny) {
  for (int j = 0; j < nm; j++) {
    double a = gx[j], b = gy[j];
    gn[j] = a * dnx + b * dny;
    gt[j] = a * dny - b * dnx;
  }
}

/* ------------------------------------------------------------------ */
/* L3: cal_var                                                          */
/* ------------------------------------------------------------------ */

typedef struct {
  double *qxx, *qxy, *qyx, *qyy, *fxx, *fxy, *fyx, *fyy;
  double *adu, *adv, *uh, *vh, *w1, *z1;
  double *fbd, *fbdxx, *fbdxy, *fbdyx, *fbdyy, *fbdx, *fbdy;
} work_t;

static int work_alloc(work_t *w, int nm, int ne, int ngf, int nf) {
  size_t en = (size_t)nm * (size_t)ne, fn = (size_t)ngf * (size_t)nf;
  double **ev[] = {&w->qxx, &w->qxy, &w->qyx, &w->qyy, &w->fxx, &w->fxy, &w->fyx,
                   &w->fyy, &w->adu, &w->adv, &w->uh, &w->vh, &w->w1, &w->z1};
  double **fv[] = {&w->fbd, &w->fbdxx, &w->fbdxy, &w->fbdyx, &w->fbdyy, &w->fbdx, &w->fbdy};
  int ok = 1;
  for (size_t i = 0; i < sizeof(ev) / sizeof(ev[0]); i++) {
    *ev[i] = (double *)malloc(sizeof(double) * (en ? en : 1));
    ok = ok && *ev[i];
  }
  for (size_t i = 0; i < sizeof(fv) / sizeof(fv[0]); i++) {
    *fv[i] = (double *)malloc(sizeof(double) * (fn ? fn : 1));
    ok = ok && *fv[i];
  }
  return ok;
}

static void work_free(work_t *w) {
  double *all[] = {w->qxx, w->qxy, w->qyx, w->qyy, w->fxx, w->fxy, w->fyx, w->fyy, w->adu,
                   w->adv, w->uh, w->vh, w->w1, w->z1, w->fbd, w->fbdxx, w->fbdxy,
                   w->fbdyx, w->fbdyy, w->fbdx, w->fbdy};
  for (size_t i = 0; i < sizeof(all) / sizeof(all[0]); i++) free(all[i]);
}

/* fbdo(j,i) = fbd(j,i) * norm(comp,i) [* scale] */
static void scale_faces(int nf, int ngf, const double *fbd, double *out, const double *norm,
                        int comp, int use_scale, double scale) {
  for (int i = 1; i <= nf; i++)
    for (int j = 1; j <= ngf; j++) {
      double v = M2(fbd, ngf, j, i) * I2(norm, comp, i, 2);
      if (use_scale) v = v * scale;
      M2(out, ngf, j, i) = v;
    }
}

static void solve_amm(const ora_common *c, double *b, const double *dia1) {
  ora_dtrsm4(c->nm, c->amm, c->ldm, b, dia1);
}
static void solve_amml(const ora_common *c, double *b, const double *dia2) {
  ora_dtrsm4(c->nm - c->nc - 1, c->amml, c->ldm, b, dia2);
}

/* free-slip/inviscid wall solve of a vector field (gx,gy): rotate to
 * (normal, tangent), solve the normal part in the wall-vanishing sub-basis. */
static void wall_solve_rot(const ora_common *c, double *gx, double *gy, double dnx, double dny,
                           const double *dia1, const double *dia2) {
  double gn[NNMAX] = {0}, gt[NNMAX] = {0}, bu[NNMAX] = {0};
  const int nm = c->nm, nc = c->nc;
  rot_vec_(nm, gn, gt, gx, gy, dnx, dny);
  ora_reduc_gn(nc, gn, bu, c->cip);
  solve_amml(c, bu, dia2);
  solve_amm(c, gt, dia1);
  ora_reduc_inv_gn(nc, gn, bu, c->cip);
  rot_vec_(nm, gx, gy, gn, gt, dnx, dny);
}

/* no-slip wall solve: both components in the wall-vanishing sub-basis */
static void wall_solve_zero(const ora_common *c, double *gx, double *gy, const double *dia2) {
  double bu[NNMAX], bv[NNMAX];
  const int nc = c->nc;
  ora_reduc_gn(nc, gx, bu, c->cip);
  ora_reduc_gn(nc, gy, bv, c->cip);
  solve_amml(c, bu, dia2);
  solve_amml(c, bv, dia2);
  ora_reduc_inv_gn(nc, gx, bu, c->cip);
  ora_reduc_inv_gn(nc, gy, bv, c->cip);
}

#define VEC(v, i) (&(v)[((size_t)(i) - 1) * (size_t)ld])
#define WVEC(v, i) (&(v)[((size_t)(i) - 1) * (size_t)nm])

/* calvar_lin.f:7-287 */
static void cal_var_lin(const ora_common *c, const ora_mesh *m, int ld, const double *u0,
                        const double *v0, const double *h0, double *u1, double *v1, double *h1,
                        const double *hb, double g0, const double *dia1, const double *dia2,
                        work_t *w, int nthreads) {
  const int nm = c->nm, ngf = c->ngf, ne = m->ne, nf = m->nf;
  double hh0 = hb[0];
  for (int i = 1; i <= ne; i++)
    for (int j = 1; j <= nm; j++) {
      WVEC(w->fxx, i)[j - 1] = -(g0 * VEC(h0, i)[j - 1]);
      WVEC(w->fxy, i)[j - 1] = 0.0;
      WVEC(w->fyx, i)[j - 1] = 0.0;
      WVEC(w->fyy, i)[j - 1] = -(g0 * VEC(h0, i)[j - 1]);
    }
  ora_cal_flu(c, nf, m->tseg, w->fbd, ngf, w->fxx, nm, m->ssit, nthreads);
  scale_faces(nf, ngf, w->fbd, w->fbdxx, m->norm, 1, 0, 0.0);
  ora_cal_flu(c, nf, m->tseg, w->fbd, ngf, w->fxy, nm, m->ssit, nthreads);
  scale_faces(nf, ngf, w->fbd, w->fbdxy, m->norm, 2, 0, 0.0);
  ora_cal_flu(c, nf, m->tseg, w->fbd, ngf, w->fyx, nm, m->ssit, nthreads);
  scale_faces(nf, ngf, w->fbd, w->fbdyx, m->norm, 1, 0, 0.0);
  ora_cal_flu(c, nf, m->tseg, w->fbd, ngf, w->fyy, nm, m->ssit, nthreads);
  scale_faces(nf, ngf, w->fbd, w->fbdyy, m->norm, 2, 0, 0.0);

#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
  for (int i = 1; i <= ne; i++) {
    double gx[NNMAX], gy[NNMAX];
    const double *vp = &m->vect[5 * (size_t)(i - 1)];
    double ax = vp[0], bx = vp[1], ay = vp[2], by = vp[3], detai = vp[4];
    for (int j = 0; j < nm; j++) gx[j] = gy[j] = 0.0;
    const double *gxx = WVEC(w->fxx, i), *gxy = WVEC(w->fxy, i);
    const double *gyx = WVEC(w->fyx, i), *gyy = WVEC(w->fyy, i);
    ora_cal_b(c, gx, gxx, c->agx, -(by * detai));
    ora_cal_b(c, gx, gxx, c->agy, ay * detai);
    ora_cal_b(c, gx, gxy, c->agx, bx * detai);
    ora_cal_b(c, gx, gxy, c->agy, -(ax * detai));
    ora_tri_f(c, i, m->itm, m->its, w->fbdxx, ngf, gx, detai);
    ora_tri_f(c, i, m->itm, m->its, w->fbdxy, ngf, gx, detai);
    double coeff = by * detai;
    ora_cal_b(c, gy, gyx, c->agx, -coeff);
    coeff = -(ay * detai);
    ora_cal_b(c, gy, gyx, c->agy, -coeff);
    coeff = -(bx * detai);
    ora_cal_b(c, gy, gyy, c->agx, -coeff);
    coeff = ax * detai;
    ora_cal_b(c, gy, gyy, c->agy, -coeff);
    ora_tri_f(c, i, m->itm, m->its, w->fbdyx, ngf, gy, detai);
    ora_tri_f(c, i, m->itm, m->its, w->fbdyy, ngf, gy, detai);
    if (m->bdl[i - 1]) {
      wall_solve_rot(c, gx, gy, I2(m->normt, 1, i, 2), I2(m->normt, 2, i, 2), dia1, dia2);
    } else {
      solve_amm(c, gx, dia1);
      solve_amm(c, gy, dia1);
    }
    for (int j = 0; j < nm; j++) {
      VEC(u1, i)[j] = gx[j];
      VEC(v1, i)[j] = gy[j];
    }
  }

  ora_cal_flu(c, nf, m->tseg, w->fbd, ngf, u0, ld, m->ssit, nthreads);
  scale_faces(nf, ngf, w->fbd, w->fbdx, m->norm, 1, 1, hh0);
  ora_cal_flu(c, nf, m->tseg, w->fbd, ngf, v0, ld, m->ssit, nthreads);
  scale_faces(nf, ngf, w->fbd, w->fbdy, m->norm, 2, 1, hh0);

#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
  for (int i = 1; i <= ne; i++) {
    double b[NNMAX], ak[NNMAX];
    const double *vp = &m->vect[5 * (size_t)(i - 1)];
    double ax = vp[0], bx = vp[1], ay = vp[2], by = vp[3], detai = vp[4];
    for (int j = 0; j < nm; j++) b[j] = 0.0;
    for (int j = 0; j < nm; j++) ak[j] = VEC(u0, i)[j] * hh0;
    ora_cal_b(c, b, ak, c->agx, by * detai);
    ora_cal_b(c, b, ak, c->agy, -(ay * detai));
    for (int j = 0; j < nm; j++) ak[j] = VEC(v0, i)[j] * hh0;
    ora_cal_b(c, b, ak, c->agx, -(bx * detai));
    ora_cal_b(c, b, ak, c->agy, ax * detai);
    ora_tri_f(c, i, m->itm, m->its, w->fbdx, ngf, b, -detai);
    ora_tri_f(c, i, m->itm, m->its, w->fbdy, ngf, b, -detai);
    solve_amm(c, b, dia1);
    for (int j = 0; j < nm; j++) VEC(h1, i)[j] = b[j];
  }
}

/* calvarnl_fs.f:9-549, calvarnl_ns.f:9, calvarnl_inv.f:6 */
static void cal_var_nl(int variant, const ora_common *c, const ora_mesh *m, int ld,
                       const double *u0, const double *v0, const double *h0, double *u1,
                       double *v1, double *h1, const double *fc, const double *w0,
                       const double *z0, const double *hb, double mu0, double mb0, double g0,
                       const double *dia1, const double *dia2, work_t *w, int nthreads) {
  const int nm = c->nm, nc = c->nc, ng = c->ng, ngf = c->ngf, ne = m->ne, nf = m->nf;

  /* Phase A: face traces of u, v (calvarnl_fs.f:88-101) */
  ora_cal_flu(c, nf, m->tseg, w->fbd, ngf, u0, ld, m->ssit, nthreads);
  scale_faces(nf, ngf, w->fbd, w->fbdxx, m->norm, 1, 0, 0.0);
  scale_faces(nf, ngf, w->fbd, w->fbdxy, m->norm, 2, 0, 0.0);
  ora_cal_flu(c, nf, m->tseg, w->fbd, ngf, v0, ld, m->ssit, nthreads);
  scale_faces(nf, ngf, w->fbd, w->fbdyx, m->norm, 1, 0, 0.0);
  scale_faces(nf, ngf, w->fbd, w->fbdyy, m->norm, 2, 0, 0.0);

  /* q = grad(u), grad(v) in weak DG form (calvarnl_fs.f:115-226) */
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
  for (int i = 1; i <= ne; i++) {
    double uk[NNMAX], vk[NNMAX], gx1[NNMAX], gy1[NNMAX];
    double gxx[NNMAX], gxy[NNMAX], gyx[NNMAX], gyy[NNMAX];
    for (int j = 0; j < nm; j++) {
      uk[j] = VEC(u0, i)[j];
      vk[j] = VEC(v0, i)[j];
    }
    const double *vp = &m->vect[5 * (size_t)(i - 1)];
    double ax = vp[0], bx = vp[1], ay = vp[2], by = vp[3], detai = vp[4];
    for (int j = 0; j < nm; j++) gx1[j] = gy1[j] = 0.0;
    ora_cal_b(c, gx1, uk, c->agx, -1.0);
    ora_cal_b(c, gy1, uk, c->agy, -1.0);
    for (int j = 0; j < nm; j++) {
      gxx[j] = (by * gx1[j] - ay * gy1[j]) * detai;
      gxy[j] = (-(bx * gx1[j]) + ax * gy1[j]) * detai;
    }
    ora_tri_f(c, i, m->itm, m->its, w->fbdxx, ngf, gxx, detai);
    ora_tri_f(c, i, m->itm, m->its, w->fbdxy, ngf, gxy, detai);
    for (int j = 0; j < nm; j++) gx1[j] = gy1[j] = 0.0;
    ora_cal_b(c, gx1, vk, c->agx, -1.0);
    ora_cal_b(c, gy1, vk, c->agy, -1.0);
    for (int j = 0; j < nm; j++) {
      gyx[j] = (by * gx1[j] - ay * gy1[j]) * detai;
      gyy[j] = (-(bx * gx1[j]) + ax * gy1[j]) * detai;
    }
    ora_tri_f(c, i, m->itm, m->its, w->fbdyx, ngf, gyx, detai);
    ora_tri_f(c, i, m->itm, m->its, w->fbdyy, ngf, gyy, detai);
    if (variant == ORA_FS && m->bdl[i - 1]) {
      /* calvarnl_fs.f:165-205 */
      double dnx = I2(m->normt, 1, i, 2), dny = I2(m->normt, 2, i, 2);
      double gnx[NNMAX], gtx[NNMAX], gny[NNMAX], gty[NNMAX];
      double gnn[NNMAX], gnt[NNMAX], gtn[NNMAX], gtt[NNMAX], bu[NNMAX];
      rot_vec_(nm, gnx, gtx, gxx, gyx, dnx, dny);
      rot_vec_(nm, gny, gty, gxy, gyy, dnx, dny);
      rot_vec_(nm, gnn, gnt, gnx, gny, dnx, dny);
      rot_vec_(nm, gtn, gtt, gtx, gty, dnx, dny);
      ora_reduc_gn(nc, gtn, bu, c->cip);
      solve_amm(c, gnn, dia1);
      solve_amm(c, gnt, dia1);
      solve_amml(c, bu, dia2);
      solve_amm(c, gtt, dia1);
      ora_reduc_inv_gn(nc, gtn, bu, c->cip);
      rot_vec_(nm, gnx, gny, gnn, gnt, dnx, dny);
      rot_vec_(nm, gtx, gty, gtn, gtt, dnx, dny);
      rot_vec_(nm, gxx, gyx, gnx, gtx, dnx, dny);
      rot_vec_(nm, gxy, gyy, gny, gty, dnx, dny);
    } else {
      solve_amm(c, gxx, dia1);
      solve_amm(c, gxy, dia1);
      solve_amm(c, gyx, dia1);
      solve_amm(c, gyy, dia1);
    }
    for (int j = 0; j < nm; j++) {
      WVEC(w->qxx, i)[j] = gxx[j];
      WVEC(w->qxy, i)[j] = gxy[j];
      WVEC(w->qyx, i)[j] = gyx[j];
      WVEC(w->qyy, i)[j] = gyy[j];
    }
  }

  /* Phase B: nonlinear terms at quadrature points (calvarnl_fs.f:243-332) */
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
  for (int i = 1; i <= ne; i++) {
    double uk[NNMAX], vk[NNMAX], hk[NNMAX], wk[NNMAX], zk[NNMAX];
    double gxx[NNMAX], gxy[NNMAX], gyx[NNMAX], gyy[NNMAX];
    double uux[NNMAX], vuy[NNMAX], uvx[NNMAX], vvy[NNMAX], uhk[NNMAX], vhk[NNMAX];
    double mff[NGMAX], mff1[NGMAX], mff2[NGMAX], mff3[NGMAX], mff4[NGMAX];
    for (int j = 0; j < nm; j++) {
      uk[j] = VEC(u0, i)[j];
      vk[j] = VEC(v0, i)[j];
      hk[j] = VEC(h0, i)[j] + VEC(hb, i)[j];
      wk[j] = VEC(w0, i)[j] - mb0 * uk[j];
      zk[j] = VEC(z0, i)[j] - mb0 * vk[j];
      gxx[j] = WVEC(w->qxx, i)[j];
      gxy[j] = WVEC(w->qxy, i)[j] - VEC(fc, i)[j];
      gyx[j] = WVEC(w->qyx, i)[j] + VEC(fc, i)[j];
      gyy[j] = WVEC(w->qyy, i)[j];
    }
    ora_spectoxy(c, mff1, uk);
    ora_spectoxy(c, mff2, vk);
    ora_spectoxy(c, mff3, gxx);
    ora_spectoxy(c, mff4, gxy);
    multiply_(ng, mff, mff1, mff3);
    ora_xytospec(c, uux, mff);
    multiply_(ng, mff, mff2, mff4);
    ora_xytospec(c, vuy, mff);
    ora_spectoxy(c, mff3, gyx);
    ora_spectoxy(c, mff4, gyy);
    multiply_(ng, mff, mff1, mff3);
    ora_xytospec(c, uvx, mff);
    multiply_(ng, mff, mff2, mff4);
    ora_xytospec(c, vvy, mff);
    ora_spectoxy(c, mff3, hk);
    multiply_(ng, mff, mff1, mff3);
    ora_xytospec(c, uhk, mff);
    multiply_(ng, mff, mff2, mff3);
    ora_xytospec(c, vhk, mff);
    ora_spectoxy(c, mff4, wk);
    divide_(ng, mff, mff4, mff3);
    ora_xytospec(c, wk, mff);
    ora_spectoxy(c, mff4, zk);
    divide_(ng, mff, mff4, mff3);
    ora_xytospec(c, zk, mff);
    if (m->bdl[i - 1]) {
      if (variant == ORA_NS)
        wall_solve_zero(c, uhk, vhk, dia2); /* calvarnl_ns.f:249-265 */
      else
        wall_solve_rot(c, uhk, vhk, I2(m->normt, 1, i, 2), I2(m->normt, 2, i, 2), dia1, dia2);
    } else {
      solve_amm(c, uhk, dia1);
      solve_amm(c, vhk, dia1);
    }
    for (int j = 0; j < nm; j++) {
      WVEC(w->adu, i)[j] = uux[j] + vuy[j];
      WVEC(w->adv, i)[j] = uvx[j] + vvy[j];
      WVEC(w->uh, i)[j] = uhk[j];
      WVEC(w->vh, i)[j] = vhk[j];
      WVEC(w->w1, i)[j] = wk[j];
      WVEC(w->z1, i)[j] = zk[j];
    }
  }

  /* Phase C: u, v tendencies (calvarnl_fs.f:341-478) */
  for (int i = 1; i <= ne; i++)
    for (int j = 0; j < nm; j++) {
      WVEC(w->fxx, i)[j] = mu0 * WVEC(w->qxx, i)[j] - g0 * VEC(h0, i)[j];
      WVEC(w->fxy, i)[j] = mu0 * WVEC(w->qxy, i)[j];
      WVEC(w->fyx, i)[j] = mu0 * WVEC(w->qyx, i)[j];
      WVEC(w->fyy, i)[j] = mu0 * WVEC(w->qyy, i)[j] - g0 * VEC(h0, i)[j];
    }
  ora_cal_flu(c, nf, m->tseg, w->fbd, ngf, w->fxx, nm, m->ssit, nthreads);
  scale_faces(nf, ngf, w->fbd, w->fbdxx, m->norm, 1, 0, 0.0);
  ora_cal_flu(c, nf, m->tseg, w->fbd, ngf, w->fxy, nm, m->ssit, nthreads);
  scale_faces(nf, ngf, w->fbd, w->fbdxy, m->norm, 2, 0, 0.0);
  ora_cal_flu(c, nf, m->tseg, w->fbd, ngf, w->fyx, nm, m->ssit, nthreads);
  scale_faces(nf, ngf, w->fbd, w->fbdyx, m->norm, 1, 0, 0.0);
  ora_cal_flu(c, nf, m->tseg, w->fbd, ngf, w->fyy, nm, m->ssit, nthreads);
  scale_faces(nf, ngf, w->fbd, w->fbdyy, m->norm, 2, 0, 0.0);

#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
  for (int i = 1; i <= ne; i++) {
    double gx[NNMAX], gy[NNMAX];
    const double *vp = &m->vect[5 * (size_t)(i - 1)];
    double ax = vp[0], bx = vp[1], ay = vp[2], by = vp[3], detai = vp[4];
    for (int j = 0; j < nm; j++) {
      gx[j] = -WVEC(w->adu, i)[j] + WVEC(w->w1, i)[j];
      gy[j] = -WVEC(w->adv, i)[j] + WVEC(w->z1, i)[j];
    }
    const double *gxx = WVEC(w->fxx, i), *gxy = WVEC(w->fxy, i);
    const double *gyx = WVEC(w->fyx, i), *gyy = WVEC(w->fyy, i);
    ora_cal_b(c, gx, gxx, c->agx, -(by * detai));
    ora_cal_b(c, gx, gxx, c->agy, ay * detai);
    ora_cal_b(c, gx, gxy, c->agx, bx * detai);
    ora_cal_b(c, gx, gxy, c->agy, -(ax * detai));
    ora_tri_f(c, i, m->itm, m->its, w->fbdxx, ngf, gx, detai);
    ora_tri_f(c, i, m->itm, m->its, w->fbdxy, ngf, gx, detai);
    ora_cal_b(c, gy, gyx, c->agx, -(by * detai));
    ora_cal_b(c, gy, gyx, c->agy, ay * detai);
    ora_cal_b(c, gy, gyy, c->agx, bx * detai);
    ora_cal_b(c, gy, gyy, c->agy, -(ax * detai));
    ora_tri_f(c, i, m->itm, m->its, w->fbdyx, ngf, gy, detai);
    ora_tri_f(c, i, m->itm, m->its, w->fbdyy, ngf, gy, detai);
    if (m->bdl[i - 1]) {
      if (variant == ORA_NS)
        wall_solve_zero(c, gx, gy, dia2); /* calvarnl_ns.f:404-421 */
      else
        wall_solve_rot(c, gx, gy, I2(m->normt, 1, i, 2), I2(m->normt, 2, i, 2), dia1, dia2);
    } else {
      solve_amm(c, gx, dia1);
      solve_amm(c, gy, dia1);
    }
    for (int j = 0; j < nm; j++) {
      VEC(u1, i)[j] = gx[j];
      VEC(v1, i)[j] = gy[j];
    }
  }

  /* Phase D: h tendency (calvarnl_fs.f:487-544) */
  ora_cal_flu(c, nf, m->tseg, w->fbd, ngf, w->uh, nm, m->ssit, nthreads);
  scale_faces(nf, ngf, w->fbd, w->fbdx, m->norm, 1, 0, 0.0);
  ora_cal_flu(c, nf, m->tseg, w->fbd, ngf, w->vh, nm, m->ssit, nthreads);
  scale_faces(nf, ngf, w->fbd, w->fbdy, m->norm, 2, 0, 0.0);

#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
  for (int i = 1; i <= ne; i++) {
    double b[NNMAX], ak[NNMAX];
    const double *vp = &m->vect[5 * (size_t)(i - 1)];
    double ax = vp[0], bx = vp[1], ay = vp[2], by = vp[3], detai = vp[4];
    for (int j = 0; j < nm; j++) b[j] = 0.0;
    for (int j = 0; j < nm; j++) ak[j] = WVEC(w->uh, i)[j];
    ora_cal_b(c, b, ak, c->agx, by * detai);
    ora_cal_b(c, b, ak, c->agy, -(ay * detai));
    for (int j = 0; j < nm; j++) ak[j] = WVEC(w->vh, i)[j];
    ora_cal_b(c, b, ak, c->agx, -(bx * detai));
    ora_cal_b(c, b, ak, c->agy, ax * detai);
    ora_tri_f(c, i, m->itm, m->its, w->fbdx, ngf, b, -detai);
    ora_tri_f(c, i, m->itm, m->its, w->fbdy, ngf, b, -detai);
    solve_amm(c, b, dia1);
    for (int j = 0; j < nm; j++) VEC(h1, i)[j] = b[j];
  }
}

int ora_cal_var(int variant, const ora_common *c, const ora_mesh *m, int ld,
                const double *u0, const double *v0, const double *h0,
                double *u1, double *v1, double *h1,
                const double *fc, const double *w0, const double *z0, const double *hb,
                double mu0, double mb0, double g0, int nthreads) {
  if (c->nm > NNMAX || c->ng > NGMAX || c->ngf > NGFMAX || ld < c->nm) return 1;
  if (nthreads < 1) nthreads = 1;
  double dia1[NNMAX], dia2[NNMAX];
  for (int i = 1; i <= c->nm; i++) dia1[i - 1] = 1.0 / M2(c->amm, c->ldm, i, i);
  for (int i = 1; i <= c->nm - c->nc - 1; i++) dia2[i - 1] = 1.0 / M2(c->amml, c->ldm, i, i);
  work_t w;
  if (!work_alloc(&w, c->nm, m->ne, c->ngf, m->nf)) {
    work_free(&w);
    return 2;
  }
  if (variant == ORA_LIN)
    cal_var_lin(c, m, ld, u0, v0, h0, u1, v1, h1, hb, g0, dia1, dia2, &w, nthreads);
  else
    cal_var_nl(variant, c, m, ld, u0, v0, h0, u1, v1, h1, fc, w0, z0, hb, mu0, mb0, g0, dia1,
               dia2, &w, nthreads);
  work_free(&w);
  return 0;
}

/* RK4 loop body: src/shwwnl.f:238-284 */
int ora_rk4(int variant, const ora_common *c, const ora_mesh *m, int ld,
            double *u0, double *v0, double *h0,
            const double *fc, const double *w0, const double *z0, const double *hb,
            double mu0, double mb0, double g0, double dt, int nsteps, int nthreads) {
  const int nm = c->nm, ne = m->ne;
  size_t n = (size_t)ld * (size_t)ne;
  double *buf = (double *)calloc(15 * n, sizeof(double));
  if (!buf) return 2;
  double *u1 = buf, *v1 = buf + n, *h1 = buf + 2 * n;
  double *d[4][3];
  for (int s = 0; s < 4; s++)
    for (int f = 0; f < 3; f++) d[s][f] = buf + (3 + 3 * s + f) * n;
  int rc = 0;
  for (int ite = 0; ite < nsteps && !rc; ite++) {
    rc = ora_cal_var(variant, c, m, ld, u0, v0, h0, d[0][0], d[0][1], d[0][2], fc, w0, z0, hb,
                     mu0, mb0, g0, nthreads);
    for (int i = 1; i <= ne; i++)
      for (int j = 0; j < nm; j++) {
        VEC(u1, i)[j] = VEC(u0, i)[j] + dt * VEC(d[0][0], i)[j] * 0.5;
        VEC(v1, i)[j] = VEC(v0, i)[j] + dt * VEC(d[0][1], i)[j] * 0.5;
        VEC(h1, i)[j] = VEC(h0, i)[j] + dt * VEC(d[0][2], i)[j] * 0.5;
      }
    if (!rc)
      rc = ora_cal_var(variant, c, m, ld, u1, v1, h1, d[1][0], d[1][1], d[1][2], fc, w0, z0, hb,
                       mu0, mb0, g0, nthreads);
    for (int i = 1; i <= ne; i++)
      for (int j = 0; j < nm; j++) {
        VEC(u1, i)[j] = VEC(u0, i)[j] + dt * VEC(d[1][0], i)[j] * 0.5;
        VEC(v1, i)[j] = VEC(v0, i)[j] + dt * VEC(d[1][1], i)[j] * 0.5;
        VEC(h1, i)[j] = VEC(h0, i)[j] + dt * VEC(d[1][2], i)[j] * 0.5;
      }
    if (!rc)
      rc = ora_cal_var(variant, c, m, ld, u1, v1, h1, d[2][0], d[2][1], d[2][2], fc, w0, z0, hb,
                       mu0, mb0, g0, nthreads);
    for (int i = 1; i <= ne; i++)
      for (int j = 0; j < nm; j++) {
        VEC(u1, i)[j] = VEC(u0, i)[j] + dt * VEC(d[2][0], i)[j];
        VEC(v1, i)[j] = VEC(v0, i)[j] + dt * VEC(d[2][1], i)[j];
        VEC(h1, i)[j] = VEC(h0, i)[j] + dt * VEC(d[2][2], i)[j];
      }
    if (!rc)
      rc = ora_cal_var(variant, c, m, ld, u1, v1, h1, d[3][0], d[3][1], d[3][2], fc, w0, z0, hb,
                       mu0, mb0, g0, nthreads);
    double dt6 = dt / 6.0;
    for (int f = 0; f < 3; f++) {
      double *s = f == 0 ? u0 : (f == 1 ? v0 : h0);
      for (int i = 1; i <= ne; i++)
        for (int j = 0; j < nm; j++)
          VEC(s, i)[j] = VEC(s, i)[j] + dt6 * (VEC(d[0][f], i)[j] + 2.0 * VEC(d[1][f], i)[j] +
                                               2.0 * VEC(d[2][f], i)[j] + VEC(d[3][f], i)[j]);
    }
  }
  free(buf);
  return rc;
}

/* energy: src/energy.f:3-96 */
void ora_energy(const ora_common *c, int ne, int ld, const double *u0, const double *v0,
                const double *h0, double g0, const double *hb, double *ke, double *pe,
                double *mass, const int *in, const double *xgr, const double *ygr) {
  const int nm = c->nm, ng = c->ng;
  double k = 0.0, p = 0.0, ms = 0.0;
  for (int i = 1; i <= ne; i++) {
    int i1 = I2(in, 1, i, 3), i2 = I2(in, 2, i, 3), i3 = I2(in, 3, i, 3);
    double ax = (xgr[i2 - 1] - xgr[i1 - 1]) * 0.5;
    double bx = (xgr[i3 - 1] - xgr[i1 - 1]) * 0.5;
    double ay = (ygr[i2 - 1] - ygr[i1 - 1]) * 0.5;
    double by = (ygr[i3 - 1] - ygr[i1 - 1]) * 0.5;
    double deta = ax * by - ay * bx;
    double uk[NNMAX], vk[NNMAX], hk[NNMAX], hbk[NNMAX];
    for (int j = 0; j < nm; j++) {
      uk[j] = VEC(u0, i)[j];
      vk[j] = VEC(v0, i)[j];
      hk[j] = VEC(h0, i)[j];
      hbk[j] = VEC(h0, i)[j] + VEC(hb, i)[j];
    }
    for (int j = 1; j <= nm; j++) ms = ms + M2(c->ammo, c->ldm, j, 1) * deta * hk[j - 1];
    double mff[NGMAX], mu[NGMAX], mv[NGMAX], mh[NGMAX], mhb[NGMAX];
    for (int j = 0; j < ng; j++) mff[j] = mu[j] = mh[j] = mhb[j] = mv[j] = 0.0;
    for (int q = 1; q <= nm; q++)
      for (int j = 1; j <= ng; j++) {
        double pp = PI2(c, j, q);
        mu[j - 1] = mu[j - 1] + uk[q - 1] * pp;
        mv[j - 1] = mv[j - 1] + vk[q - 1] * pp;
        mh[j - 1] = mh[j - 1] + hk[q - 1] * pp;
        mhb[j - 1] = mhb[j - 1] + hbk[q - 1] * pp;
      }
    for (int j = 0; j < ng; j++) mff[j] = mhb[j] * (mu[j] * mu[j] + mv[j] * mv[j]);
    double ans = 0.0;
    for (int j = 1; j <= ng; j++) ans = ans + c->wi[j - 1] * mff[j - 1] * PI2(c, j, 1);
    k = k + ans * deta * 0.5;
    for (int j = 0; j < ng; j++) mff[j] = mh[j] * mh[j];
    ans = 0.0;
    for (int j = 1; j <= ng; j++) ans = ans + c->wi[j - 1] * mff[j - 1] * PI2(c, j, 1);
    p = p + ans * deta * 0.5 * g0;
  }
  *ke = k;
  *pe = p;
  *mass = ms;
}

/* checkcfl: src/cfl.f:4-52.  Returns dt; *cflmin gets the raw bound. */
double ora_checkcfl(int nc, int ne, int ld, const double *hb, const int *in, double g0,
                    const double *xgr, const double *ygr, double *cflmin_out) {
  double cflmin = 6000.0, ra = 0.30, dt = 0.0;
  for (int i = 1; i <= ne; i++) {
    int i1 = I2(in, 1, i, 3), i2 = I2(in, 2, i, 3), i3 = I2(in, 3, i, 3);
    double ax = (xgr[i2 - 1] - xgr[i1 - 1]), ay = (ygr[i2 - 1] - ygr[i1 - 1]);
    double dd1 = sqrt(ax * ax + ay * ay) / (double)nc * ra;
    ax = (xgr[i3 - 1] - xgr[i1 - 1]);
    ay = (ygr[i3 - 1] - ygr[i1 - 1]);
    double dd2 = sqrt(ax * ax + ay * ay) / (double)nc * ra;
    ax = (xgr[i3 - 1] - xgr[i2 - 1]);
    ay = (ygr[i3 - 1] - ygr[i2 - 1]);
    double dd3 = sqrt(ax * ax + ay * ay) / (double)nc * ra;
    double cc0 = sqrt(g0 * M2(hb, ld, 1, i));
    cflmin = fmin(cflmin, dd1 / cc0);
    cflmin = fmin(cflmin, dd2 / cc0);
    cflmin = fmin(cflmin, dd3 / cc0);
  }
  if (cflmin >= 100)
    dt = (double)(10 * (int)(cflmin / 10));
  else if (cflmin >= 10 && cflmin < 100)
    dt = (double)(2 * (int)(cflmin / 2));
  else if (cflmin < 10 && cflmin >= 1)
    dt = (double)((int)cflmin);
  else if (cflmin < 1)
    dt = (double)((int)(cflmin * 10) / 10); /* integer division, as in the reference */
  if (cflmin_out) *cflmin_out = cflmin;
  return dt;
}

/* calh quadrature-point coordinates: src/init.f:315-333 (px,py are (ng,ne)) */
void ora_calh_points(const ora_common *c, int ne, const int *in, const double *xgr,
                     const double *ygr, double *px, double *py) {
  const int ng = c->ng;
  for (int i = 1; i <= ne; i++) {
    int i1 = I2(in, 1, i, 3), i2 = I2(in, 2, i, 3), i3 = I2(in, 3, i, 3);
    double agx = (xgr[i2 - 1] - xgr[i1 - 1]) * 0.5, agy = (ygr[i2 - 1] - ygr[i1 - 1]) * 0.5;
    double bgx = (xgr[i3 - 1] - xgr[i1 - 1]) * 0.5, bgy = (ygr[i3 - 1] - ygr[i1 - 1]) * 0.5;
    double xof = xgr[i1 - 1], yof = ygr[i1 - 1];
    for (int j = 1; j <= ng; j++) {
      double x = c->xi[j - 1], y = c->yi[j - 1];
      M2(px, ng, j, i) = agx * (x + 1.0) + bgx * (y + 1.0) + xof;
      M2(py, ng, j, i) = agy * (x + 1.0) + bgy * (y + 1.0) + yof;
    }
  }
}

/* calh projection: src/init.f:335-341 (vals are the function at ora_calh_points) */
void ora_calh(const ora_common *c, int ne, const double *vals, double *h, int ld) {
  const int nm = c->nm, ng = c->ng;
  double dia1[NNMAX];
  for (int i = 1; i <= nm; i++) dia1[i - 1] = 1.0 / M2(c->amm, c->ldm, i, i);
  for (int i = 1; i <= ne; i++) {
    double b[NNMAX];
    ora_xytospec(c, b, &vals[(size_t)(i - 1) * ng]);
    ora_dtrsm4(nm, c->amm, c->ldm, b, dia1);
    for (int j = 0; j < nm; j++) VEC(h, i)[j] = b[j];
  }
}

/* ------------------------------------------------------------------ */
/* L5: solution-driven regridding and the adaptive driver's CFL        */
/* ------------------------------------------------------------------ */

/* checkconv: src/adapt.f:1260-1334.  amax(ne): per element, the largest jump
 * of a0's trace across its interior faces at the ngf edge points, divided by
 * max |a0(1,i)| (0 when that is <= 1e-6). */
void ora_checkconv(const ora_common *c, int nf, int ne, int ld, const double *a0,
                   const int *tseg, const int *ssit, double *amax) {
  const int nm = c->nm, ngf = c->ngf;
  double fbdy1[NGFMAX], fbdy2[NGFMAX];
  for (int i = 1; i <= ne; i++) amax[i - 1] = 0.0;
  for (int i = 1; i <= nf; i++) {
    for (int j = 1; j <= ngf; j++) fbdy1[j - 1] = fbdy2[j - 1] = 0.0;
    const int k1 = I2(tseg, 1, i, 2), k2 = I2(tseg, 2, i, 2);
    if (k2 > 0) {
      int cote = I2(ssit, 1, i, 2);
      for (int i1 = 1; i1 <= nm; i1++)
        for (int j = 1; j <= ngf; j++)
          fbdy1[j - 1] = fbdy1[j - 1] + VEC(a0, k1)[i1 - 1] * PICO(c, j, i1, cote);
      cote = I2(ssit, 2, i, 2);
      for (int i1 = 1; i1 <= nm; i1++)
        for (int j = 1; j <= ngf; j++)
          fbdy2[j - 1] = fbdy2[j - 1] + VEC(a0, k2)[i1 - 1] * PICO(c, ngf - j + 1, i1, cote);
      for (int j = 1; j <= ngf; j++) {
        const double dif = fabs(fbdy2[j - 1] - fbdy1[j - 1]);
        if (amax[k1 - 1] < dif) amax[k1 - 1] = dif;
        if (amax[k2 - 1] < dif) amax[k2 - 1] = dif;
      }
    }
  }
  double vmax = fabs(VEC(a0, 1)[0]);
  for (int i = 2; i <= ne; i++) vmax = fmax(fabs(VEC(a0, i)[0]), vmax);
  for (int i = 1; i <= ne; i++) amax[i - 1] = vmax > 1.0e-6 ? amax[i - 1] / vmax : 0.0;
}

/* cal_conv: src/adapt.f:1122-1193.  fconv(i): some field's jump > fac1
 * (refine); fderaff(i): all three < fac2 (coarsen); flags[0] conv, flags[1]
 * deraff, flags[2] timedir; *supmax the largest jump. */
void ora_cal_conv(const ora_common *c, int nf, int ne, int ld, const double *u0,
                  const double *v0, const double *h0, const int *tseg, const int *ssit,
                  double fac1, double fac2, double fac3, int *fconv, int *fderaff, int *flags,
                  double *supmax_out, double *umax, double *vmax, double *hmax) {
  ora_checkconv(c, nf, ne, ld, u0, tseg, ssit, umax);
  ora_checkconv(c, nf, ne, ld, v0, tseg, ssit, vmax);
  ora_checkconv(c, nf, ne, ld, h0, tseg, ssit, hmax);
  int deraff = 0;
  double supmax = umax[0];
  for (int i = 0; i < ne; i++) {
    fconv[i] = (umax[i] > fac1) || (vmax[i] > fac1) || (hmax[i] > fac1);
    fderaff[i] = (umax[i] < fac2) && (vmax[i] < fac2) && (hmax[i] < fac2);
    if (fderaff[i]) deraff = 1;
    supmax = fmax(supmax, umax[i]);
    supmax = fmax(supmax, vmax[i]);
    supmax = fmax(supmax, hmax[i]);
  }
  flags[2] = !(supmax > fac3);
  flags[0] = (supmax > fac1) || deraff;
  flags[1] = deraff;
  if (supmax_out) *supmax_out = supmax;
}

/* inter_only_new: src/adapt.f:1233-1258.  tinter(i) = the old element that
 * new element i repeats (same three nodes, in order), else 0. */
void ora_inter_only_new(int ne, int nenew, const int *in, const int *innew, int *tinter) {
  for (int i = 0; i < nenew; i++) tinter[i] = 0;
  int tk = 1;
  for (int i = 1; i <= ne && tk <= nenew; i++) {
    int k = 0;
    for (int j = 1; j <= 3; j++)
      if (I2(in, j, i, 3) == I2(innew, j, tk, 3)) k++;
    if (k == 3) {
      tinter[tk - 1] = i;
      tk++;
    }
  }
}

/* interlin: src/adapt.f:1747-1830.  Walks from element *tk to the element
 * holding (xdp, ydp) (a point outside the mesh is moved onto the wall edge it
 * crossed), returning its barycentric coordinates lab(3).  The walk is capped
 * at maxit moves; returns 0, or -1 when the cap is reached. */
int ora_interlin(const int *itt, const int *itm, const int *tseg, const int *pseg,
                 const double *x, const double *y, int *tk_io, double *xdp_io, double *ydp_io,
                 double *lab, int maxit) {
  const double eps = 1.0e-9;
  int tk = *tk_io;
  double xdp = *xdp_io, ydp = *ydp_io;
  for (int it = 0; it < maxit; it++) {
    double x1 = x[I2(itt, 1, tk, 3) - 1], y1 = y[I2(itt, 1, tk, 3) - 1];
    double x2 = x[I2(itt, 2, tk, 3) - 1], y2 = y[I2(itt, 2, tk, 3) - 1];
    const double x3 = x[I2(itt, 3, tk, 3) - 1], y3 = y[I2(itt, 3, tk, 3) - 1];
    const double aire = (x2 - x3) * (y2 - y1) - (x2 - x1) * (y2 - y3);
    lab[0] = (xdp - x2) * (ydp - y3) - (xdp - x3) * (ydp - y2);
    lab[1] = (xdp - x3) * (ydp - y1) - (xdp - x1) * (ydp - y3);
    lab[2] = (xdp - x1) * (ydp - y2) - (xdp - x2) * (ydp - y1);
    for (int k = 0; k < 3; k++) {
      lab[k] = lab[k] / aire;
      if (fabs(lab[k]) < eps) lab[k] = 0.0;
    }
    int tk1, ns1 = 0;
    if (lab[0] >= 0 && lab[1] >= 0 && lab[2] >= 0) {
      *tk_io = tk;
      *xdp_io = xdp;
      *ydp_io = ydp;
      return 0;
    }
    if (lab[0] < 0.0) ns1 = I2(itm, 2, tk, 3);
    else if (lab[1] < 0.0) ns1 = I2(itm, 3, tk, 3);
    else ns1 = I2(itm, 1, tk, 3);
    tk1 = I2(tseg, 1, ns1, 2);
    if (tk1 == tk) tk1 = I2(tseg, 2, ns1, 2);
    if (tk1 > 0) {
      tk = tk1;
    } else {
      const int n1 = I2(pseg, 1, ns1, 2), n2 = I2(pseg, 2, ns1, 2);
      x1 = x[n1 - 1];
      y1 = y[n1 - 1];
      x2 = x[n2 - 1];
      y2 = y[n2 - 1];
      const double d = (x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2);
      double pr = (x1 - xdp) * (x1 - x2) + (y1 - ydp) * (y1 - y2);
      pr = pr / d;
      xdp = x1 * (1.0 - pr) + x2 * pr;
      ydp = y1 * (1.0 - pr) + y2 * pr;
    }
  }
  *tk_io = tk;
  return -1;
}

/* fsol: src/compare.f:203-219 (the modal expansion of element i at (x, y)) */
static double fsol_(int nc, double x, double y, const double *b, int ld, int i) {
  int j = 0;
  double s = 0.0;
  for (int kc1 = 0; kc1 <= nc; kc1++)
    for (int kc2 = 0; kc2 <= nc - kc1; kc2++) {
      j++;
      s = s + VEC(b, i)[j - 1] * ora_po(kc1, x) * ora_po(kc2, y);
    }
  return s;
}

/* interpol: src/adapt.f:1662-1745.  unew(ld, nenew) on the new mesh from
 * u(ld, ne) on the old one: elements with tinter > 0 copy their old element;
 * the others are the L2 projection of u evaluated at their quadrature points
 * (located by interlin, the walk continuing from the previous point's
 * element).  loc_elem / loc_x / loc_y (ng x nenew, may be null) receive the
 * located element and reference coordinates.  Returns 0, or -1 if a walk hit
 * its cap. */
int ora_interpol(const ora_common *c, int ne, const int *in, const int *itm, const int *tseg,
                 const int *pseg, const double *xgr, const double *ygr, const int *tinter,
                 const double *u, int ld, double *unew, int nenew, const double *xgrnew,
                 const double *ygrnew, const int *innew, int *loc_elem, double *loc_x,
                 double *loc_y) {
  const int nm = c->nm, ng = c->ng, nc = c->nc;
  double dia1[NNMAX], mff[NGMAX], b[NNMAX], lab[3];
  for (int i = 1; i <= nm; i++) dia1[i - 1] = 1.0 / M2(c->amm, c->ldm, i, i);
  int tk = 1;
  for (int i = 1; i <= nenew; i++) {
    if (tinter[i - 1] == 0) {
      const int i1 = I2(innew, 1, i, 3), i2 = I2(innew, 2, i, 3), i3 = I2(innew, 3, i, 3);
      const double agx = (xgrnew[i2 - 1] - xgrnew[i1 - 1]) * 0.5;
      const double bgx = (xgrnew[i3 - 1] - xgrnew[i1 - 1]) * 0.5;
      const double agy = (ygrnew[i2 - 1] - ygrnew[i1 - 1]) * 0.5;
      const double bgy = (ygrnew[i3 - 1] - ygrnew[i1 - 1]) * 0.5;
      const double xof = xgrnew[i1 - 1], yof = ygrnew[i1 - 1];
      for (int j = 1; j <= ng; j++) {
        const double y = c->yi[j - 1], x = c->xi[j - 1];
        double x0 = agx * (x + 1.0) + bgx * (y + 1.0) + xof;
        double y0 = agy * (x + 1.0) + bgy * (y + 1.0) + yof;
        if (ora_interlin(in, itm, tseg, pseg, xgr, ygr, &tk, &x0, &y0, lab, 16 * ne + 64))
          return -1;
        const double x1 = 2.0 * lab[1] - 1.0, y1 = 2.0 * lab[2] - 1.0;
        mff[j - 1] = fsol_(nc, x1, y1, u, ld, tk);
        if (loc_elem) {
          M2(loc_elem, ng, j, i) = tk;
          M2(loc_x, ng, j, i) = x1;
          M2(loc_y, ng, j, i) = y1;
        }
      }
      ora_xytospec(c, b, mff);
      ora_dtrsm4(nm, c->amm, c->ldm, b, dia1);
      for (int j = 0; j < nm; j++) VEC(unew, i)[j] = b[j];
    } else {
      for (int j = 0; j < nm; j++) VEC(unew, i)[j] = VEC(u, tinter[i - 1])[j];
    }
  }
  return 0;
}

/* verif_rot: src/shwwnl_adap.f:481-596.  Re-projects (u0, v0) after a regrid:
 * the mass-matrix load (cal_b with ammo) is solved again, in the rotated
 * wall-vanishing sub-basis for the normal component on wall elements. */
void ora_verif_rot(const ora_common *c, int ne, int ld, double *u0, double *v0,
                   const double *normt, const int *bdl) {
  const int nm = c->nm, nmr = nm - c->nc - 1;
  double dia1[NNMAX], dia2[NNMAX];
  for (int i = 1; i <= nm; i++) dia1[i - 1] = 1.0 / M2(c->amm, c->ldm, i, i);
  for (int i = 1; i <= nmr; i++) dia2[i - 1] = 1.0 / M2(c->amml, c->ldm, i, i);
  for (int i = 1; i <= ne; i++) {
    double gx[NNMAX] = {0}, gy[NNMAX] = {0};
    ora_cal_b(c, gx, VEC(u0, i), c->ammo, 1.0);
    ora_cal_b(c, gy, VEC(v0, i), c->ammo, 1.0);
    if (bdl[i - 1]) {
      wall_solve_rot(c, gx, gy, I2(normt, 1, i, 2), I2(normt, 2, i, 2), dia1, dia2);
    } else {
      solve_amm(c, gx, dia1);
      solve_amm(c, gy, dia1);
    }
    for (int j = 0; j < nm; j++) {
      VEC(u0, i)[j] = gx[j];
      VEC(v0, i)[j] = gy[j];
    }
  }
}

/* cal_pgraph: src/visu2.f:4-25.  pgraph(nm, n, n): the basis on the n-point
 * lattice of the reference triangle, (l, k) with l <= n - k + 1. */
void ora_cal_pgraph(int nc, int n, double *pgraph) {
  const int nm = (nc + 1) * (nc + 2) / 2;
  for (int k = 1; k <= n; k++)
    for (int l = 1; l <= n - k + 1; l++) {
      const double y = (double)(2 * k - n - 1) / (double)(n - 1);
      const double x = (double)(2 * l - n - 1) / (double)(n - 1);
      int i1 = 0;
      for (int kc1 = 0; kc1 <= nc; kc1++)
        for (int kc2 = 0; kc2 <= nc - kc1; kc2++) {
          i1++;
          pgraph[((size_t)(k - 1) * n + (l - 1)) * nm + i1 - 1] = ora_po(kc1, x) * ora_po(kc2, y);
        }
    }
}

/* checkcfl2: src/cfl.f:57-140.  Time step from the gravity-wave speed of the
 * largest depth plus the largest velocity on the lattice of each element.
 * dt_in is returned unchanged when no branch applies (a NaN bound). */
double ora_checkcfl2(int nc, int ne, int ld, const double *hb, const double *u,
                     const double *v, const int *in, double g0, const double *xgr,
                     const double *ygr, int n, const double *pgraph, double dt_in,
                     double *cflmin_out) {
  const int nm = (nc + 1) * (nc + 2) / 2;
  const double ra = 0.35;
  double cflmin = 6000.0;
  for (int i = 1; i <= ne; i++) {
    double maxdepth = 0.0, maxvel = 0.0;
    for (int k = 1; k <= n; k++)
      for (int l = 1; l <= n - k + 1; l++) {
        double sol0 = 0.0, sol1 = 0.0, sol2 = 0.0;
        for (int i1 = 1; i1 <= nm; i1++) {
          const double pp = pgraph[((size_t)(k - 1) * n + (l - 1)) * nm + i1 - 1];
          sol0 = sol0 + VEC(hb, i)[i1 - 1] * pp;
          sol1 = sol1 + VEC(u, i)[i1 - 1] * pp;
          sol2 = sol2 + VEC(v, i)[i1 - 1] * pp;
        }
        maxdepth = fmax(maxdepth, sol0);
        maxvel = fmax(maxvel, sqrt(sol1 * sol1 + sol2 * sol2));
      }
    const int i1 = I2(in, 1, i, 3), i2 = I2(in, 2, i, 3), i3 = I2(in, 3, i, 3);
    double ax = xgr[i2 - 1] - xgr[i1 - 1], ay = ygr[i2 - 1] - ygr[i1 - 1];
    const double dd1 = sqrt(ax * ax + ay * ay) / (double)nc * ra;
    ax = xgr[i3 - 1] - xgr[i1 - 1];
    ay = ygr[i3 - 1] - ygr[i1 - 1];
    const double dd2 = sqrt(ax * ax + ay * ay) / (double)nc * ra;
    ax = xgr[i3 - 1] - xgr[i2 - 1];
    ay = ygr[i3 - 1] - ygr[i2 - 1];
    const double dd3 = sqrt(ax * ax + ay * ay) / (double)nc * ra;
    const double cc0 = sqrt(g0 * maxdepth) + maxvel;
    cflmin = fmin(cflmin, dd1 / cc0);
    cflmin = fmin(cflmin, dd2 / cc0);
    cflmin = fmin(cflmin, dd3 / cc0);
  }
  if (cflmin_out) *cflmin_out = cflmin;
  double dt = dt_in;
  if (cflmin >= 100) dt = (double)(10 * (int)(cflmin / 10));
  else if (cflmin >= 10 && cflmin < 100) dt = (double)(2 * (int)(cflmin / 2));
  else if (cflmin < 10 && cflmin >= 1) dt = (double)(int)cflmin;
  else if (cflmin < 1) dt = (double)((int)(cflmin * 10) / 10);
  return dt;
}

/* fsol at npts points: out[f * npts + i] for u, v, h (src/compare.f:203-219) */
void ora_eval_points(int nc, int ld, const double *u, const double *v, const double *h,
                     int npts, const int *elem, const double *px, const double *py,
                     double *out) {
  for (int i = 0; i < npts; i++) {
    out[i] = fsol_(nc, px[i], py[i], u, ld, elem[i]);
    out[(size_t)npts + i] = fsol_(nc, px[i], py[i], v, ld, elem[i]);
    out[2 * (size_t)npts + i] = fsol_(nc, px[i], py[i], h, ld, elem[i]);
  }
}

/* write_gra's values (src/visu2.f:86-149): out[(e*np + p)*5 + c], c = x, y,
 * then the field values of u, v, h at lattice point p (k outer, l inner). */
void ora_lattice(int nc, int ne, int ld, const double *u, const double *v, const double *h,
                 const int *in, const double *xgr, const double *ygr, int n,
                 const double *pgraph, double *out) {
  const int nm = (nc + 1) * (nc + 2) / 2, np = n * (n + 1) / 2;
  for (int i = 1; i <= ne; i++) {
    const int i1 = I2(in, 1, i, 3), i2 = I2(in, 2, i, 3), i3 = I2(in, 3, i, 3);
    const double ax = (xgr[i2 - 1] - xgr[i1 - 1]) * 0.5, bx = (xgr[i3 - 1] - xgr[i1 - 1]) * 0.5;
    const double ay = (ygr[i2 - 1] - ygr[i1 - 1]) * 0.5, by = (ygr[i3 - 1] - ygr[i1 - 1]) * 0.5;
    const double xof = xgr[i1 - 1], yof = ygr[i1 - 1];
    int p = 0;
    for (int k = 1; k <= n; k++)
      for (int l = 1; l <= n - k + 1; l++, p++) {
        const double y1 = (double)(2 * k - n - 1) / (double)(n - 1);
        const double x1 = (double)(2 * l - n - 1) / (double)(n - 1);
        double *o = &out[(((size_t)(i - 1)) * np + p) * 5];
        o[0] = xof + ax * (x1 + 1.0) + bx * (y1 + 1.0);
        o[1] = yof + ay * (x1 + 1.0) + by * (y1 + 1.0);
        const double *fld[3] = {u, v, h};
        for (int f = 0; f < 3; f++) {
          double sol = 0.0;
          for (int j = 1; j <= nm; j++)
            sol = sol + VEC(fld[f], i)[j - 1] * pgraph[((size_t)(k - 1) * n + (l - 1)) * nm + j - 1];
          o[2 + f] = sol;
        }
      }
  }
}
