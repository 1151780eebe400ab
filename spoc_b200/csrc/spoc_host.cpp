// Host-side set-up of the SPOC DG operators and mesh pointers.
//
// These run once per run on the CPU, exactly like the Fortran driver's set-up
// (src/shwwnl.f:127-174), and produce the arrays the RK4 right-hand side
// consumes.  Arithmetic follows the reference order with separately rounded
// products (compiled with -ffp-contract=off), so the tables are bit-identical
// to what the Fortran driver would pass through COMMON.
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/spoc_gpu.h"

namespace {

// Legendre polynomial P_n(x) by the three-term recurrence (src/legendre2.f:5-30).
double legendre(int n, double x) {
  if (n == 0) return 1.0;
  double pm1 = 1.0, p = x;
  for (int i = 2; i <= n; ++i) {
    const double a0 = double(i), a2 = double(2 * i - 1), a3 = double(i - 1);
    const double pn = (a2 * x * p - a3 * pm1) / a0;
    pm1 = p;
    p = pn;
  }
  return p;
}

// P_n'(x) by the differentiated recurrence (src/legendre2.f:32-62).
double legendre_d(int n, double x) {
  if (n == 0) return 0.0;
  double pm1 = 1.0, p = x, dpm1 = 0.0, dp = 1.0;
  for (int i = 2; i <= n; ++i) {
    const double a0 = double(i), a2 = double(2 * i - 1), a3 = double(i - 1);
    const double dpn = (a2 * x * dp + a2 * p - a3 * dpm1) / a0;
    const double pn = (a2 * x * p - a3 * pm1) / a0;
    pm1 = p;
    p = pn;
    dpm1 = dp;
    dp = dpn;
  }
  return dp;
}

// Mode ordering shared by every table: kc1 outer 0..nc, kc2 inner 0..nc-kc1
// (src/nonlin.f:325-327).
struct Modes {
  std::vector<int> k1, k2;
  explicit Modes(int nc) {
    for (int a = 0; a <= nc; ++a)
      for (int b = 0; b <= nc - a; ++b) {
        k1.push_back(a);
        k2.push_back(b);
      }
  }
  int size() const { return int(k1.size()); }
};

// Offset of the kc1 = i block: sum_{j<i} (nc+1-j) (src/mat1.f:372-381).
int block_offset(int nc, int i) {
  int off = 0;
  for (int j = 0; j < i; ++j) off += nc + 1 - j;
  return off;
}

// Upper Cholesky, unblocked (DPOTF2 with the vendored DDOT/DGEMV/DSCAL order,
// src/solve.f:276-440).  Returns 0 or the failing column (1-based).
int cholesky_upper(int n, double *a, int lda) {
  auto A = [&](int i, int j) -> double & { return a[size_t(j) * lda + i]; };
  for (int j = 0; j < n; ++j) {
    double dot = 0.0;
    for (int k = 0; k < j; ++k) dot = dot + A(k, j) * A(k, j);
    double ajj = A(j, j) - dot;
    if (ajj <= 0.0) {
      A(j, j) = ajj;
      return j + 1;
    }
    ajj = std::sqrt(ajj);
    A(j, j) = ajj;
    if (j + 1 < n) {
      for (int c = j + 1; c < n; ++c) {
        double t = 0.0;
        for (int i = 0; i < j; ++i) t = t + A(i, c) * A(i, j);
        A(j, c) = A(j, c) + (-1.0) * t;
      }
      const double r = 1.0 / ajj;
      for (int c = j + 1; c < n; ++c) A(j, c) = r * A(j, c);
    }
  }
  return 0;
}

}  // namespace

extern "C" int spoc_build_tables(int nc, int ng, int ngf, const double *wi, const double *xi,
                                 const double *yi, const double *wif, const double *tif,
                                 double *pi2, double *pico, double *amm, double *amml,
                                 double *agx, double *agy, double *ammo, double *ammx,
                                 double *ammy, int *cip, int *info) {
  (void)wif;
  if (info) *info = 0;
  if (nc < 1 || ng < 1 || ngf < 1 || !wi || !xi || !yi || !tif || !pi2 || !pico || !amm ||
      !amml || !agx || !agy || !ammo || !ammx || !ammy || !cip)
    return SPOC_E_ARG;
  const Modes md(nc);
  const int nm = md.size();

  // pi2(q, n) = P_k1(x_q) P_k2(y_q)   (src/nonlin.f:10-30)
  for (int n = 0; n < nm; ++n)
    for (int q = 0; q < ng; ++q)
      pi2[size_t(n) * ng + q] = legendre(md.k1[n], xi[q]) * legendre(md.k2[n], yi[q]);

  // pico(j, n, side) on the three reference edges (src/mat1.f:214-259)
  for (int side = 0; side < 3; ++side)
    for (int n = 0; n < nm; ++n)
      for (int j = 0; j < ngf; ++j) {
        double x, y;
        if (side == 0) {
          x = tif[j];
          y = -1.0;
        } else if (side == 1) {
          x = -tif[j];
          y = tif[j];
        } else {
          x = -1.0;
          y = -tif[j];
        }
        pico[(size_t(side) * nm + n) * ngf + j] = legendre(md.k1[n], x) * legendre(md.k2[n], y);
      }

  // cip(1,i) / cip(2,i) block offsets of the full and reduced bases (src/mat1.f:383-410)
  for (int i = 0; i <= nc; ++i) {
    cip[2 * i] = block_offset(nc, i);
    cip[2 * i + 1] = (i <= nc - 1) ? block_offset(nc - 1, i) : 0;
  }

  // Reference-element operators by quadrature (src/mat1.f:90-142, integrands :513-576):
  // mat(a, b) = sum_q w_q phi_a(q) * op(phi_b)(q)
  double *mats[5] = {amm, ammx, ammy, agx, agy};
  for (int which = 0; which < 5; ++which) {
    double *m = mats[which];
    for (int a = 0; a < nm; ++a)
      for (int b = 0; b < nm; ++b) {
        double s = 0.0;
        for (int q = 0; q < ng; ++q) {
          const double x = xi[q], y = yi[q];
          double f;
          switch (which) {
            case 0:
              f = legendre(md.k1[a], x) * legendre(md.k2[a], y) * legendre(md.k1[b], x) *
                  legendre(md.k2[b], y);
              break;
            case 1:
              f = legendre(md.k1[a], x) * legendre(md.k2[a], y) * legendre(md.k1[b], x) *
                  legendre(md.k2[b], y) * x;
              break;
            case 2:
              f = legendre(md.k1[a], x) * legendre(md.k2[a], y) * legendre(md.k1[b], x) *
                  legendre(md.k2[b], y) * y;
              break;
            case 3:
              f = legendre(md.k1[a], x) * legendre(md.k2[a], y) * legendre_d(md.k1[b], x) *
                  legendre(md.k2[b], y);
              break;
            default:
              f = legendre(md.k1[a], x) * legendre(md.k2[a], y) * legendre(md.k1[b], x) *
                  legendre_d(md.k2[b], y);
              break;
          }
          s = s + wi[q] * f;
        }
        m[size_t(b) * nm + a] = s;
      }
  }
  std::memcpy(ammo, amm, sizeof(double) * size_t(nm) * nm);

  // amml: mass matrix of the sub-basis (P_{l+1}(y) +/- P_0(y)) P_i(x) that
  // vanishes on side 1 (src/mat1.f:285-368).  Four parity passes, same order.
  std::memset(amml, 0, sizeof(double) * size_t(nm) * nm);
  auto AM = [&](int i, int j) { return amm[size_t(j - 1) * nm + (i - 1)]; };
  for (int pass = 0; pass < 4; ++pass) {
    const int jstart = (pass & 1) ? 1 : 0;  // odd l on the row side
    const int lstart = (pass & 2) ? 1 : 0;  // odd l on the column side
    for (int i = 0; i <= nc - 1; ++i)
      for (int j = jstart; j <= nc - 1 - i; j += 2)
        for (int k = 0; k <= nc - 1; ++k)
          for (int l = lstart; l <= nc - 1 - k; l += 2) {
            const int i1 = block_offset(nc - 1, i) + j + 1, i2 = block_offset(nc, i) + j + 2;
            const int j1 = block_offset(nc - 1, k) + l + 1, j2 = block_offset(nc, k) + l + 2;
            const int i0 = block_offset(nc, i) + 1, j0 = block_offset(nc, k) + 1;
            const double sr = (pass & 1) ? -1.0 : 1.0, sc = (pass & 2) ? -1.0 : 1.0;
            // pass 0: a+b+c+d; 1: a-b+c-d; 2: a+b-c-d; 3: a-b-c+d (a=(i2,j2) b=(i0,j2) c=(i2,j0) d=(i0,j0))
            double v = AM(i2, j2);
            v = (sr > 0) ? v + AM(i0, j2) : v - AM(i0, j2);
            v = (sc > 0) ? v + AM(i2, j0) : v - AM(i2, j0);
            v = (sr * sc > 0) ? v + AM(i0, j0) : v - AM(i0, j0);
            amml[size_t(j1 - 1) * nm + (i1 - 1)] = v;
          }
  }

  // Cholesky factors in place (src/shwwnl.f:153-156)
  int r = cholesky_upper(nm, amm, nm);
  if (r) {
    if (info) *info = r;
    return SPOC_E_MATRIX;
  }
  r = cholesky_upper(nm - nc - 1, amml, nm);
  if (r) {
    if (info) *info = 1000 + r;
    return SPOC_E_MATRIX;
  }
  return SPOC_OK;
}

extern "C" int spoc_build_mesh(int nn, int ne, const int *in, const double *xgr,
                               const double *ygr, int nc, double f0, double beta, int nfmax,
                               int *nf_out, int *itm, int *its, int *tseg, int *pseg, int *ssit,
                               double *norm, double *vect, double *normt, int *bdl, double *fc,
                               int ld) {
  if (nn < 3 || ne < 1 || !in || !xgr || !ygr || !nf_out || !itm || !its || !tseg || !pseg ||
      !ssit || !norm || !vect || !normt || !bdl || nfmax < 1)
    return SPOC_E_ARG;
  for (int i = 0; i < 3 * ne; ++i)
    if (in[i] < 1 || in[i] > nn) return SPOC_E_MESH;

  // Node -> elements incidence, sorted by element (src/cmal_s.f:121-160).
  std::vector<int> start(size_t(nn) + 2, 0), lst_t(size_t(3) * ne + 1), lst_k(size_t(3) * ne + 1);
  for (int i = 0; i < 3 * ne; ++i) start[in[i]]++;
  {
    int acc = 0;
    for (int n = 1; n <= nn; ++n) {
      const int c = start[n];
      start[n] = acc;
      acc += c;
    }
    start[nn + 1] = acc;
  }
  {
    std::vector<int> fill(start.begin(), start.end());
    for (int e = 1; e <= ne; ++e)
      for (int k = 1; k <= 3; ++k) {
        const int n = in[size_t(e - 1) * 3 + (k - 1)];
        lst_t[fill[n]] = e;
        lst_k[fill[n]] = k;
        fill[n]++;
      }
  }

  // Faces in order of first appearance; a side matches the reversed side of an
  // earlier element around its end node (src/cmal_s.f:164-208).
  for (int f = 0; f < nfmax; ++f) tseg[2 * f] = tseg[2 * f + 1] = 0;
  int nf = 0;
  for (int e = 1; e <= ne; ++e)
    for (int j = 1; j <= 3; ++j) {
      const int a = in[size_t(e - 1) * 3 + (j - 1)];
      const int b = in[size_t(e - 1) * 3 + (j == 3 ? 0 : j)];
      int found = 0;
      for (int p = start[b]; p < start[b + 1]; ++p) {
        const int t = lst_t[p], k = lst_k[p];
        if (t >= e) break;
        const int c = in[size_t(t - 1) * 3 + (k == 3 ? 0 : k)];
        if (c == a) {
          found = itm[size_t(t - 1) * 3 + (k - 1)];
          break;
        }
      }
      if (found) {
        tseg[2 * (found - 1) + 1] = e;
        itm[size_t(e - 1) * 3 + (j - 1)] = found;
      } else {
        if (nf >= nfmax) return SPOC_E_ARG;
        ++nf;
        itm[size_t(e - 1) * 3 + (j - 1)] = nf;
        tseg[2 * (nf - 1)] = e;
        pseg[2 * (nf - 1)] = a;
        pseg[2 * (nf - 1) + 1] = b;
      }
    }
  *nf_out = nf;

  // check_mesh: one wall face per element at most, and it must be side 1 (src/cmal_s.f:222-277)
  {
    std::vector<int> walls(size_t(ne) + 1, 0);
    for (int f = 0; f < nf; ++f)
      if (tseg[2 * f + 1] == 0) walls[tseg[2 * f]]++;
    for (int e = 1; e <= ne; ++e)
      if (walls[e] > 1) return SPOC_E_MESH;
    for (int f = 0; f < nf; ++f)
      if (tseg[2 * f + 1] == 0 && itm[size_t(tseg[2 * f] - 1) * 3] != f + 1) return SPOC_E_MESH;
  }

  // Unnormalised face normals (dy, -dx) (src/mat1.f:7-23)
  for (int f = 0; f < nf; ++f) {
    const int n1 = pseg[2 * f], n2 = pseg[2 * f + 1];
    norm[2 * f] = (ygr[n2 - 1] - ygr[n1 - 1]);
    norm[2 * f + 1] = -(xgr[n2 - 1] - xgr[n1 - 1]);
  }

  // Side orientation and side-in-element of each face (src/mat1.f:28-64)
  for (int f = 0; f < nf; ++f) ssit[2 * f] = ssit[2 * f + 1] = 0;
  for (int f = 1; f <= nf; ++f)
    for (int s = 0; s < 2; ++s) {
      const int t = tseg[2 * (f - 1) + s];
      if (t == 0) continue;
      int j = 1;
      while (j <= 3 && itm[size_t(t - 1) * 3 + (j - 1)] != f) ++j;
      if (j > 3) return SPOC_E_MESH;
      its[size_t(t - 1) * 3 + (j - 1)] = s == 0 ? 1 : -1;
      ssit[2 * (f - 1) + s] = j;
    }

  // Element geometry and side-1 unit normal (src/shwwnl.f:361-406)
  for (int e = 0; e < ne; ++e) bdl[e] = 0;
  for (int f = 0; f < nf; ++f)
    if (tseg[2 * f + 1] == 0) bdl[tseg[2 * f] - 1] = 1;
  for (int e = 0; e < ne; ++e) {
    const int i1 = in[3 * size_t(e)], i2 = in[3 * size_t(e) + 1], i3 = in[3 * size_t(e) + 2];
    const double ax = (xgr[i2 - 1] - xgr[i1 - 1]) * 0.5;
    const double bx = (xgr[i3 - 1] - xgr[i1 - 1]) * 0.5;
    const double ay = (ygr[i2 - 1] - ygr[i1 - 1]) * 0.5;
    const double by = (ygr[i3 - 1] - ygr[i1 - 1]) * 0.5;
    const double deta = ax * by - ay * bx;
    double *v = vect + 5 * size_t(e);
    v[0] = ax;
    v[1] = bx;
    v[2] = ay;
    v[3] = by;
    v[4] = 1.0 / deta;
    const int f1 = itm[3 * size_t(e)];
    double dnx = norm[2 * (f1 - 1)], dny = norm[2 * (f1 - 1) + 1];
    const double dis = std::sqrt(dnx * dnx + dny * dny);
    normt[2 * size_t(e)] = dnx / dis;
    normt[2 * size_t(e) + 1] = dny / dis;
  }

  // Coriolis modal coefficients of f0 + beta*y (src/mat1.f:69-83)
  if (fc) {
    const int nm = (nc + 1) * (nc + 2) / 2;
    if (ld < nm || nc + 2 > nm) return SPOC_E_ARG;
    for (int e = 0; e < ne; ++e) {
      double *c = fc + size_t(e) * ld;
      for (int j = 0; j < ld; ++j) c[j] = 0.0;
      const int n1 = in[3 * size_t(e)], n2 = in[3 * size_t(e) + 1], n3 = in[3 * size_t(e) + 2];
      c[0] = f0 + 0.5 * beta * (ygr[n3 - 1] + ygr[n2 - 1]);
      c[1] = 0.5 * beta * (ygr[n3 - 1] - ygr[n1 - 1]);
      c[nc + 1] = 0.5 * beta * (ygr[n2 - 1] - ygr[n1 - 1]);
    }
  }
  return SPOC_OK;
}

// Corner fix (src/chmal.f:240-330).  The diagonal shared by an element with two
// wall faces and its neighbour is flipped; afterwards every wall element's
// local numbering is rotated so its wall face is side 1.
extern "C" int spoc_fix_mesh(int nn, int ne, int *in) {
  if (nn < 3 || ne < 1 || !in) return SPOC_E_ARG;
  const int nfmax = 3 * ne;
  std::vector<int> itm(size_t(3) * ne), its(size_t(3) * ne), tseg(2 * size_t(nfmax)),
      pseg(2 * size_t(nfmax));
  // Pointers of the unfixed mesh: same face search as spoc_build_mesh, without checks.
  std::vector<int> start(size_t(nn) + 2, 0), lst_t(size_t(3) * ne), lst_k(size_t(3) * ne);
  for (int i = 0; i < 3 * ne; ++i) {
    if (in[i] < 1 || in[i] > nn) return SPOC_E_MESH;
    start[in[i]]++;
  }
  {
    int acc = 0;
    for (int n = 1; n <= nn; ++n) {
      const int c = start[n];
      start[n] = acc;
      acc += c;
    }
    start[nn + 1] = acc;
    std::vector<int> fill(start.begin(), start.end());
    for (int e = 1; e <= ne; ++e)
      for (int k = 1; k <= 3; ++k) {
        const int n = in[size_t(e - 1) * 3 + (k - 1)];
        lst_t[fill[n]] = e;
        lst_k[fill[n]] = k;
        fill[n]++;
      }
  }
  auto IN = [&](int k, int e) -> int & { return in[size_t(e - 1) * 3 + (k - 1)]; };
  auto ITM = [&](int k, int e) -> int & { return itm[size_t(e - 1) * 3 + (k - 1)]; };
  auto TSEG = [&](int s, int f) -> int & { return tseg[size_t(f - 1) * 2 + (s - 1)]; };
  int nf = 0;
  for (int e = 1; e <= ne; ++e)
    for (int j = 1; j <= 3; ++j) {
      const int a = IN(j, e), b = IN(j == 3 ? 1 : j + 1, e);
      int found = 0;
      for (int p = start[b]; p < start[b + 1]; ++p) {
        const int t = lst_t[p], k = lst_k[p];
        if (t >= e) break;
        if (IN(k == 3 ? 1 : k + 1, t) == a) {
          found = ITM(k, t);
          break;
        }
      }
      if (found) {
        TSEG(2, found) = e;
        ITM(j, e) = found;
      } else {
        ++nf;
        ITM(j, e) = nf;
        TSEG(1, nf) = e;
        TSEG(2, nf) = 0;
      }
    }
  auto wrap = [](int k) { return k > 3 ? k - 3 : (k < 1 ? k + 3 : k); };
  std::vector<int> walls, nwall(size_t(ne) + 1, 0);
  for (int f = 1; f <= nf; ++f)
    if (TSEG(2, f) == 0) {
      walls.push_back(f);
      nwall[TSEG(1, f)]++;
    }
  for (int e = 1; e <= ne; ++e) {
    if (nwall[e] <= 1) continue;
    int j = 1;
    while (j <= 3 && TSEG(2, ITM(j, e)) == 0) ++j;
    if (j > 3) return SPOC_E_MESH;
    const int f = ITM(j, e), t1 = TSEG(1, f), t2 = TSEG(2, f);
    int j1 = 1, j2 = 1;
    while (j1 <= 3 && ITM(j1, t1) != f) ++j1;
    while (j2 <= 3 && ITM(j2, t2) != f) ++j2;
    if (j1 > 3 || j2 > 3) return SPOC_E_MESH;
    const int k1 = wrap(j1 + 1), k2 = wrap(j2 - 1), k3 = wrap(j2 + 1), k4 = wrap(j1 - 1);
    const int opp2 = IN(k2, t2), opp1 = IN(k4, t1);
    IN(k1, t1) = opp2;
    IN(k3, t2) = opp1;
    ITM(j1, t1) = ITM(k3, t2);
    ITM(j2, t2) = ITM(k1, t1);
    ITM(k1, t1) = f;
    ITM(k3, t2) = f;
    if (e == t1)
      TSEG(1, ITM(j2, t2)) = t2;
    else
      TSEG(1, ITM(j1, t1)) = t1;
  }
  for (int f : walls) {
    const int t = TSEG(1, f);
    int j = 1;
    while (j <= 3 && ITM(j, t) != f) ++j;
    if (j > 3) return SPOC_E_MESH;
    int pp[3], pf[3];
    for (int k = 1; k <= 3; ++k) {
      const int l = wrap(k + j - 1);
      pp[k - 1] = IN(l, t);
      pf[k - 1] = ITM(l, t);
    }
    for (int k = 1; k <= 3; ++k) {
      IN(k, t) = pp[k - 1];
      ITM(k, t) = pf[k - 1];
    }
  }
  (void)its;
  (void)pseg;
  return SPOC_OK;
}

extern "C" int spoc_projection_points(int ne, const int *in, const double *xgr,
                                      const double *ygr, int ng, const double *xi,
                                      const double *yi, double *px, double *py) {
  if (ne < 1 || ng < 1 || !in || !xgr || !ygr || !xi || !yi || !px || !py) return SPOC_E_ARG;
  for (int e = 0; e < ne; ++e) {
    const int i1 = in[3 * size_t(e)], i2 = in[3 * size_t(e) + 1], i3 = in[3 * size_t(e) + 2];
    const double agx = (xgr[i2 - 1] - xgr[i1 - 1]) * 0.5, agy = (ygr[i2 - 1] - ygr[i1 - 1]) * 0.5;
    const double bgx = (xgr[i3 - 1] - xgr[i1 - 1]) * 0.5, bgy = (ygr[i3 - 1] - ygr[i1 - 1]) * 0.5;
    const double xof = xgr[i1 - 1], yof = ygr[i1 - 1];
    for (int q = 0; q < ng; ++q) {
      const double x = xi[q], y = yi[q];
      px[size_t(e) * ng + q] = agx * (x + 1.0) + bgx * (y + 1.0) + xof;
      py[size_t(e) * ng + q] = agy * (x + 1.0) + bgy * (y + 1.0) + yof;
    }
  }
  return SPOC_OK;
}

extern "C" int spoc_project(int nc, int ng, const double *wi, const double *pi2,
                            const double *amm, int ne, const double *vals, double *out, int ld) {
  const int nm = (nc + 1) * (nc + 2) / 2;
  if (nc < 1 || ng < 1 || ld < nm || !wi || !pi2 || !amm || !vals || !out) return SPOC_E_ARG;
  std::vector<double> dia(nm), b(nm);
  for (int i = 0; i < nm; ++i) dia[i] = 1.0 / amm[size_t(i) * nm + i];
  for (int e = 0; e < ne; ++e) {
    const double *f = vals + size_t(e) * ng;
    // load vector b_n = sum_q (w_q f_q) pi2(q,n)   (src/nonlin.f:35-57, :91-107)
    for (int n = 0; n < nm; ++n) {
      double s = 0.0;
      for (int q = 0; q < ng; ++q) s = s + wi[q] * f[q] * pi2[size_t(n) * ng + q];
      b[n] = s;
    }
    // (U^T U) x = b   (src/dtrsm1.f:47-82)
    for (int i = 0; i < nm; ++i) {
      double t = b[i];
      for (int k = 0; k < i; ++k) t = t - amm[size_t(i) * nm + k] * b[k];
      b[i] = t * dia[i];
    }
    for (int k = nm - 1; k >= 0; --k) {
      b[k] = b[k] * dia[k];
      for (int i = 0; i < k; ++i) b[i] = b[i] - b[k] * amm[size_t(k) * nm + i];
    }
    for (int n = 0; n < nm; ++n) out[size_t(e) * ld + n] = b[n];
  }
  return SPOC_OK;
}

// inter_only_new (src/adapt.f:1233-1258): tinter[i] = the old element (1-based)
// that new element i repeats with the same nodes in the same order, else 0.
// Old elements are matched in order against the new list, as the reference
// does, so unchanged elements must keep their relative order.
extern "C" int spoc_inter_only_new(int ne, int nenew, const int *in, const int *innew,
                                   int *tinter) {
  if (ne < 1 || nenew < 1 || !in || !innew || !tinter) return SPOC_E_ARG;
  for (int i = 0; i < nenew; ++i) tinter[i] = 0;
  int tk = 0;
  for (int i = 0; i < ne && tk < nenew; ++i) {
    int k = 0;
    for (int j = 0; j < 3; ++j)
      if (in[3 * size_t(i) + j] == innew[3 * size_t(tk) + j]) ++k;
    if (k == 3) tinter[tk++] = i + 1;
  }
  return SPOC_OK;
}

namespace {

// interlin (src/adapt.f:1747-1830): walk from element *tk (1-based) towards
// (xdp, ydp) through the faces whose barycentric coordinate is negative; a
// point pushed out through a wall is moved onto that wall edge.  Barycentric
// coordinates within 1e-9 of zero count as zero.  At most maxit moves.
bool interlin(const int *in, const int *itm, const int *tseg, const int *pseg, const double *x,
              const double *y, int *tk_io, double *xdp_io, double *ydp_io, double lab[3],
              long maxit) {
  const double eps = 1.0e-9;
  int tk = *tk_io;
  double xdp = *xdp_io, ydp = *ydp_io;
  for (long it = 0; it < maxit; ++it) {
    const size_t b = 3 * size_t(tk - 1);
    double x1 = x[in[b] - 1], y1 = y[in[b] - 1];
    double x2 = x[in[b + 1] - 1], y2 = y[in[b + 1] - 1];
    const double x3 = x[in[b + 2] - 1], y3 = y[in[b + 2] - 1];
    const double aire = (x2 - x3) * (y2 - y1) - (x2 - x1) * (y2 - y3);
    lab[0] = (xdp - x2) * (ydp - y3) - (xdp - x3) * (ydp - y2);
    lab[1] = (xdp - x3) * (ydp - y1) - (xdp - x1) * (ydp - y3);
    lab[2] = (xdp - x1) * (ydp - y2) - (xdp - x2) * (ydp - y1);
    for (int k = 0; k < 3; ++k) {
      lab[k] = lab[k] / aire;
      if (std::fabs(lab[k]) < eps) lab[k] = 0.0;
    }
    if (lab[0] >= 0 && lab[1] >= 0 && lab[2] >= 0) {
      *tk_io = tk;
      *xdp_io = xdp;
      *ydp_io = ydp;
      return true;
    }
    // side 2 faces vertex 1, side 3 vertex 2, side 1 vertex 3
    const int side = lab[0] < 0.0 ? 1 : (lab[1] < 0.0 ? 2 : 0);
    const int ns1 = itm[b + side];
    int tk1 = tseg[2 * size_t(ns1 - 1)];
    if (tk1 == tk) tk1 = tseg[2 * size_t(ns1 - 1) + 1];
    if (tk1 > 0) {
      tk = tk1;
    } else {
      const int n1 = pseg[2 * size_t(ns1 - 1)], n2 = pseg[2 * size_t(ns1 - 1) + 1];
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
  return false;
}

}  // namespace

// Point location of interpol (src/adapt.f:1690-1718): for every new element
// with tinter == 0, its quadrature points (the calh map of the new element)
// are located in the old mesh by interlin, the walk starting from the
// element the previous point ended in (element 1 first), exactly as the
// reference's loop runs.  pt_elem (1-based old element) and the reference
// coordinates pt_x = 2 lab2 - 1, pt_y = 2 lab3 - 1 are (ng, nenew); rows of
// inherited elements are set to 0.  Old-mesh arrays are those of
// spoc_build_mesh (1-based, tseg 0 on walls).  Returns SPOC_E_MESH when a
// walk does not end.
extern "C" int spoc_locate_points(int ne, const int *in, const int *itm, const int *tseg,
                                  const int *pseg, const double *xgr, const double *ygr,
                                  int nenew, const int *innew, const double *xgrnew,
                                  const double *ygrnew, const int *tinter, int ng,
                                  const double *xi, const double *yi, int *pt_elem,
                                  double *pt_x, double *pt_y) {
  if (ne < 1 || nenew < 1 || ng < 1 || !in || !itm || !tseg || !pseg || !xgr || !ygr ||
      !innew || !xgrnew || !ygrnew || !tinter || !xi || !yi || !pt_elem || !pt_x || !pt_y)
    return SPOC_E_ARG;
  const long maxit = 16L * ne + 64;
  int tk = 1;
  double lab[3];
  for (int i = 0; i < nenew; ++i) {
    const size_t o = size_t(i) * ng;
    if (tinter[i] != 0) {
      for (int j = 0; j < ng; ++j) {
        pt_elem[o + j] = 0;
        pt_x[o + j] = pt_y[o + j] = 0.0;
      }
      continue;
    }
    const int i1 = innew[3 * size_t(i)], i2 = innew[3 * size_t(i) + 1], i3 = innew[3 * size_t(i) + 2];
    const double agx = (xgrnew[i2 - 1] - xgrnew[i1 - 1]) * 0.5;
    const double bgx = (xgrnew[i3 - 1] - xgrnew[i1 - 1]) * 0.5;
    const double agy = (ygrnew[i2 - 1] - ygrnew[i1 - 1]) * 0.5;
    const double bgy = (ygrnew[i3 - 1] - ygrnew[i1 - 1]) * 0.5;
    const double xof = xgrnew[i1 - 1], yof = ygrnew[i1 - 1];
    for (int j = 0; j < ng; ++j) {
      const double yq = yi[j], xq = xi[j];
      double x0 = agx * (xq + 1.0) + bgx * (yq + 1.0) + xof;
      double y0 = agy * (xq + 1.0) + bgy * (yq + 1.0) + yof;
      if (!interlin(in, itm, tseg, pseg, xgr, ygr, &tk, &x0, &y0, lab, maxit)) return SPOC_E_MESH;
      pt_elem[o + j] = tk;
      pt_x[o + j] = 2.0 * lab[1] - 1.0;
      pt_y[o + j] = 2.0 * lab[2] - 1.0;
    }
  }
  return SPOC_OK;
}

// Sequential point location of compare.f (src/compare.f:118-150): each point
// (px[i], py[i]) is located by interlin from the element the previous walk
// ended in (*tk on entry, updated); a result whose barycentric coordinates sum
// below 0.5 counts as outside (inside[i] = 0) and the walk restarts from
// reset_tk.  elem (1-based), x1 = 2 lab2 - 1, y1 = 2 lab3 - 1.
extern "C" int spoc_locate_xy(int ne, const int *in, const int *itm, const int *tseg,
                              const int *pseg, const double *xgr, const double *ygr, int npts,
                              const double *px, const double *py, int *tk, int reset_tk,
                              int *elem, double *x1, double *y1, int *inside) {
  if (ne < 1 || npts < 0 || !in || !itm || !tseg || !pseg || !xgr || !ygr || !tk ||
      (npts && (!px || !py || !elem || !x1 || !y1 || !inside)) || *tk < 1 || *tk > ne ||
      reset_tk < 1 || reset_tk > ne)
    return SPOC_E_ARG;
  const long maxit = 16L * ne + 64;
  double lab[3];
  for (int i = 0; i < npts; ++i) {
    double x = px[i], y = py[i];
    if (!interlin(in, itm, tseg, pseg, xgr, ygr, tk, &x, &y, lab, maxit)) return SPOC_E_MESH;
    const double sum = lab[0] + lab[1] + lab[2];
    if (sum < 0.5) {
      inside[i] = 0;
      elem[i] = 0;
      x1[i] = y1[i] = 0.0;
      *tk = reset_tk;
    } else {
      inside[i] = 1;
      elem[i] = *tk;
      x1[i] = 2.0 * lab[1] - 1.0;
      y1[i] = 2.0 * lab[2] - 1.0;
    }
  }
  return SPOC_OK;
}
