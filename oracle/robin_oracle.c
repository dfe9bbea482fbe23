/* CPU ORACLE -- test infrastructure, not product code.
 *
 * Plain-C restatement of EMerge's Robin (third-kind) boundary term on
 * Nedelec-2 (SECOND_MIXED_VOLAKIS) triangles, the port / absorbing-boundary
 * matrix the microwave assembler adds into A:
 *
 *   ned2_tri_stiff      physics/microwave/assembly/robinbc.py:316-378
 *   construct_local_vertices                     robinbc.py:165-183
 *   tri_coefficients                             robinbc.py:200-221
 *   DPTS (6-point triangle rule)                 robinbc.py:189-196
 *   compute_bc_entries                           robinbc.py:381-402
 *   ned2_tri_force / compute_force_entries       robinbc.py:220-313
 *   2-D basis functions _ne0_2d, _ne2_2d, _nf0_2d, _nf1_2d
 *                                                compiled/ccbf.py:81,107,269,284
 *   second-order ABC correction _abc_order_2_terms / _matrix_builder
 *                                physics/microwave/assembly/robin_abc_order2.py:143-251
 *   its tri_coefficients and 6-point rule (14 digits)     robin_abc_order2.py:100-122, 89-98
 *   2-D curls _curl_ne0_2d, _curl_ne2_2d, _curl_nf0_2d, _curl_nf1_2d
 *                                                compiled/ccbf.py:168,178,386,397
 *
 * dofcodes2d of the Volakis set are [64, 64, 64, 66, 66, 66, 128, 129]
 * (elements/dofsets.py:39,114-115): three ne0 edge functions on the local
 * vertex pairs (0,1), (1,2), (0,2), three ne2 on the same pairs, then nf0 and
 * nf1 on (0,1,2). The triangle matrix is
 *   B[a][b] = gamma * A * sum_q w_q (f_a . f_b)(x_q)
 * in the triangle's own plane (unconjugated dot product, A = area).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef double complex cplx;

/* robinbc.py:189-196, digit for digit: weights and barycentric rows L1..L3 */
static const double TRI_DPTS[4][6] = {
    {0.10995174365532200, 0.10995174365532200, 0.10995174365532200, 0.22338158967801100, 0.22338158967801100,
     0.22338158967801100},
    {0.81684757298045896, 0.09157621350977101, 0.09157621350977101, 0.10810301816807000, 0.44594849091596500,
     0.44594849091596500},
    {0.09157621350977101, 0.81684757298045896, 0.09157621350977101, 0.44594849091596500, 0.10810301816807000,
     0.44594849091596500},
    {0.09157621350977004, 0.09157621350977008, 0.81684757298045807, 0.44594849091596500, 0.44594849091596500,
     0.10810301816807000},
};

static void cross3(const double a[3], const double b[3], double out[3]) {
  out[0] = a[1] * b[2] - a[2] * b[1];
  out[1] = a[2] * b[0] - a[0] * b[2];
  out[2] = a[0] * b[1] - a[1] * b[0];
}

static void normalize3(double a[3]) {
  const double n = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  a[0] /= n;
  a[1] /= n;
  a[2] /= n;
}

/* The triangle's local frame (construct_local_vertices), coefficients
 * (tri_coefficients) and the 8 Volakis functions at the 6 points.
 * X[d][v]: vertex v (0..2) coordinates. Returns the area; basis rows are
 * xhat, yhat, zhat. */
/* construct_local_vertices (robinbc.py:165-183): origin at vertex 0, x along
 * edge 0->1, z the normal; the vertices' local coordinates tx, ty */
static void tri_local(const double X[3][3], double basis[3][3], double tx[3], double ty[3]) {
  double e1[3], e2[3], xh[3], yh[3], zh[3];
  for (int d = 0; d < 3; ++d) {
    e1[d] = X[d][1] - X[d][0];
    e2[d] = X[d][2] - X[d][0];
  }
  cross3(e1, e2, zh);
  normalize3(zh);
  memcpy(xh, e1, sizeof xh);
  normalize3(xh);
  cross3(zh, xh, yh);
  normalize3(yh);
  for (int d = 0; d < 3; ++d) {
    basis[0][d] = xh[d];
    basis[1][d] = yh[d];
    basis[2][d] = zh[d];
  }
  for (int v = 0; v < 3; ++v) {
    double rx = 0.0, ry = 0.0;
    for (int d = 0; d < 3; ++d) {
      const double r = X[d][v] - X[d][0];
      rx += xh[d] * r;
      ry += yh[d] * r;
    }
    tx[v] = rx;
    ty[v] = ry;
  }
}

static double tri_frame_basis(const double X[3][3], double basis[3][3], double f[8][2][6]) {
  double tx[3], ty[3];
  tri_local(X, basis, tx, ty);
  /* tri_coefficients */
  const double x1 = tx[0], x2 = tx[1], x3 = tx[2], y1 = ty[0], y2 = ty[1], y3 = ty[2];
  const double a[3] = {x2 * y3 - y2 * x3, x3 * y1 - y3 * x1, x1 * y2 - y1 * x2};
  const double b[3] = {y2 - y3, y3 - y1, y1 - y2};
  const double c[3] = {x3 - x2, x1 - x3, x2 - x1};
  const double sA = 0.5 * (b[0] * c[1] - b[1] * c[0]);
  double ca[3], cb[3], cc[3];
  for (int m = 0; m < 3; ++m) {
    ca[m] = a[m] / (2 * sA);
    cb[m] = b[m] / (2 * sA);
    cc[m] = c[m] / (2 * sA);
  }
  /* the 8 basis functions at the 6 points */
  static const int EI[3] = {0, 1, 0}, EJ[3] = {1, 2, 2};
  for (int q = 0; q < 6; ++q) {
    const double xs = tx[0] * TRI_DPTS[1][q] + tx[1] * TRI_DPTS[2][q] + tx[2] * TRI_DPTS[3][q];
    const double ys = ty[0] * TRI_DPTS[1][q] + ty[1] * TRI_DPTS[2][q] + ty[2] * TRI_DPTS[3][q];
    double L[3];
    for (int m = 0; m < 3; ++m) L[m] = ca[m] + cb[m] * xs + cc[m] * ys;
    for (int e = 0; e < 3; ++e) {
      const int i = EI[e], j = EJ[e];
      /* ne0: L_i grad L_j - L_j grad L_i */
      f[e][0][q] = L[i] * cb[j] - L[j] * cb[i];
      f[e][1][q] = L[i] * cc[j] - L[j] * cc[i];
      /* ne2: (L_i - L_j)(L_i grad L_j - L_j grad L_i) */
      const double s = L[i] - L[j];
      f[3 + e][0][q] = s * (L[i] * cb[j] - L[j] * cb[i]);
      f[3 + e][1][q] = s * (L[i] * cc[j] - L[j] * cc[i]);
    }
    /* nf0: L_0 (L_1 grad L_2 - L_2 grad L_1); nf1: L_1 (L_0 grad L_2 - L_2 grad L_0) */
    f[6][0][q] = L[0] * (L[1] * cb[2] - L[2] * cb[1]);
    f[6][1][q] = L[0] * (L[1] * cc[2] - L[2] * cc[1]);
    f[7][0][q] = L[1] * (L[0] * cb[2] - L[2] * cb[0]);
    f[7][1][q] = L[1] * (L[0] * cc[2] - L[2] * cc[0]);
  }
  return fabs(sA);
}

/* X[d][v]: vertex v (0..2) coordinates. out[64] row-major, gamma applied. */
void oracle_tri_stiff(const double X[3][3], double g_re, double g_im, cplx *out) {
  double basis[3][3], f[8][2][6];
  const double area = tri_frame_basis(X, basis, f);
  const cplx g = g_re + I * g_im;
  for (int p = 0; p < 8; ++p)
    for (int r = 0; r < 8; ++r) {
      double sum = 0.0;
      for (int q = 0; q < 6; ++q) sum += (f[p][0][q] * f[r][0][q] + f[p][1][q] * f[r][1][q]) * TRI_DPTS[0][q];
      out[8 * p + r] = g * sum * area;
    }
}

/* compute_bc_entries: Bmat[itri*64 .. +64] += B(itri) for every listed tri.
 * nodes f64 [3][nN], tris i64 [3][F] (sorted vertex ids). */
int oracle_robin_entries(const double *nodes, int64_t nN, const int64_t *tris, int64_t F, const int64_t *btris,
                         int64_t nb, double g_re, double g_im, cplx *Bmat) {
  for (int64_t i = 0; i < nb; ++i) {
    const int64_t t = btris[i];
    if (t < 0 || t >= F) return -1;
    for (int v = 0; v < 3; ++v)
      if (tris[v * F + t] < 0 || tris[v * F + t] >= nN) return -1;
  }
  for (int64_t i = 0; i < nb; ++i) {
    const int64_t t = btris[i];
    double X[3][3];
    for (int d = 0; d < 3; ++d)
      for (int v = 0; v < 3; ++v) X[d][v] = nodes[d * nN + tris[v * F + t]];
    cplx B[64];
    oracle_tri_stiff(X, g_re, g_im, B);
    for (int k = 0; k < 64; ++k) Bmat[t * 64 + k] += B[k];
  }
  return 0;
}

/* ned2_tri_force: out[8] = -A sum_q w_q f_a(q) . U2(q), with U2 the first two
 * components of the incident field in the triangle's frame (basis @ U).
 * U: complex [3][6] (component, point). */
void oracle_tri_force(const double X[3][3], const cplx *U, cplx *out) {
  double basis[3][3], f[8][2][6];
  const double area = tri_frame_basis(X, basis, f);
  cplx u2[2][6];
  for (int a = 0; a < 2; ++a)
    for (int q = 0; q < 6; ++q) u2[a][q] = basis[a][0] * U[0 * 6 + q] + basis[a][1] * U[1 * 6 + q] + basis[a][2] * U[2 * 6 + q];
  for (int p = 0; p < 8; ++p) {
    cplx sum = 0.0;
    for (int q = 0; q < 6; ++q) sum += TRI_DPTS[0][q] * (f[p][0][q] * u2[0][q] + f[p][1][q] * u2[1][q]);
    out[p] = -area * sum;
  }
}

/* compute_force_entries: b[tri_to_field[:, itri]] += force(itri) for every
 * listed tri, U: complex [3][6][nb] (the reference's U_global_all layout),
 * t2f: int64 [8][F]. */
int oracle_force_entries(const double *nodes, int64_t nN, const int64_t *tris, int64_t F, const int64_t *t2f,
                         const int64_t *btris, int64_t nb, const cplx *U, int64_t N, cplx *b) {
  for (int64_t i = 0; i < nb; ++i) {
    const int64_t t = btris[i];
    if (t < 0 || t >= F) return -1;
    for (int v = 0; v < 3; ++v)
      if (tris[v * F + t] < 0 || tris[v * F + t] >= nN) return -1;
    for (int k = 0; k < 8; ++k)
      if (t2f[k * F + t] < 0 || t2f[k * F + t] >= N) return -1;
  }
  for (int64_t i = 0; i < nb; ++i) {
    const int64_t t = btris[i];
    double X[3][3];
    for (int d = 0; d < 3; ++d)
      for (int v = 0; v < 3; ++v) X[d][v] = nodes[d * nN + tris[v * F + t]];
    cplx Ui[18];
    for (int d = 0; d < 3; ++d)
      for (int q = 0; q < 6; ++q) Ui[d * 6 + q] = U[(d * 6 + q) * nb + i];
    cplx bv[8];
    oracle_tri_force(X, Ui, bv);
    for (int k = 0; k < 8; ++k) b[t2f[k * F + t]] += bv[k];
  }
  return 0;
}

/* robin_abc_order2.py:89-98, its own copy of the rule: weights, L1..L3 */
static const double ABC2_DPTS[4][6] = {
    {0.10995174365532, 0.10995174365532, 0.10995174365532, 0.22338158967801, 0.22338158967801, 0.22338158967801},
    {0.81684757298046, 0.09157621350977, 0.09157621350977, 0.10810301816807, 0.44594849091597, 0.44594849091597},
    {0.09157621350977, 0.81684757298046, 0.09157621350977, 0.44594849091597, 0.10810301816807, 0.44594849091597},
    {0.09157621350977, 0.09157621350977, 0.81684757298046, 0.44594849091597, 0.44594849091597, 0.10810301816807}};

/* _abc_order_2_terms: B[a][b] = cf * A * sum_q w_q c_a(q) c_b(q) with c the
 * scalar 2-D curls of the 8 functions in the triangle's plane. The reference
 * also forms a divergence matrix, but writes the first function's divergence
 * into the second function's buffer, which the inner loop overwrites before
 * use, so that matrix is identically zero; it is left out here. */
void oracle_abc2_block(const double X[3][3], double cf_re, double cf_im, cplx *out) {
  double basis[3][3], tx[3], ty[3];
  tri_local(X, basis, tx, ty);
  const double x1 = tx[0], x2 = tx[1], x3 = tx[2], y1 = ty[0], y2 = ty[1], y3 = ty[2];
  const double a[3] = {x2 * y3 - y2 * x3, x3 * y1 - y3 * x1, x1 * y2 - y1 * x2};
  const double b[3] = {y2 - y3, y3 - y1, y1 - y2};
  const double c[3] = {x3 - x2, x1 - x3, x2 - x1};
  const double sA = 0.5 * ((x1 - x3) * (y2 - y1) - (x1 - x2) * (y3 - y1));
  const double sign = sA > 0 ? 1.0 : (sA < 0 ? -1.0 : 0.0);
  const double A = fabs(sA);
  double ca[3], cb[3], cc[3];
  for (int m = 0; m < 3; ++m) {
    ca[m] = a[m] * sign / (2 * A);
    cb[m] = b[m] * sign / (2 * A);
    cc[m] = c[m] * sign / (2 * A);
  }
  static const int EI[3] = {0, 1, 0}, EJ[3] = {1, 2, 2};
  double C[8][6];
  for (int q = 0; q < 6; ++q) {
    const double xs = x1 * ABC2_DPTS[1][q] + x2 * ABC2_DPTS[2][q] + x3 * ABC2_DPTS[3][q];
    const double ys = y1 * ABC2_DPTS[1][q] + y2 * ABC2_DPTS[2][q] + y3 * ABC2_DPTS[3][q];
    for (int e = 0; e < 3; ++e) {
      const int i = EI[e], j = EJ[e];
      const double ai = ca[i], bi = cb[i], ci = cc[i], aj = ca[j], bj = cb[j], cj = cc[j];
      /* _curl_ne0_2d */
      C[e][q] = 2 * bi * cj - 2 * bj * ci;
      /* _curl_ne2_2d */
      const double t0 = bj * xs, t1 = cj * ys, t2 = t0 + t1 + aj, t3 = ai + bi * xs + ci * ys;
      C[3 + e][q] = -(bi - bj) * (t2 * ci - t3 * cj) + (ci - cj) * (t2 * bi - t3 * bj) +
                    2 * (bi * cj - bj * ci) * (-t0 - t1 + t3 - aj);
    }
    {  /* _curl_nf0_2d on (0, 1, 2) */
      const double t0 = ca[2] + cb[2] * xs + cc[2] * ys, t1 = ca[1] + cb[1] * xs + cc[1] * ys;
      C[6][q] = -cb[0] * (t0 * cc[1] - t1 * cc[2]) + cc[0] * (t0 * cb[1] - t1 * cb[2]) +
                2 * (cb[1] * cc[2] - cb[2] * cc[1]) * (ca[0] + cb[0] * xs + cc[0] * ys);
    }
    {  /* _curl_nf1_2d on (0, 1, 2) */
      const double t0 = ca[2] + cb[2] * xs + cc[2] * ys, t1 = ca[0] + cb[0] * xs + cc[0] * ys;
      C[7][q] = -cb[1] * (t0 * cc[0] - t1 * cc[2]) + cc[1] * (t0 * cb[0] - t1 * cb[2]) +
                2 * (cb[0] * cc[2] - cb[2] * cc[0]) * (ca[1] + cb[1] * xs + cc[1] * ys);
    }
  }
  const cplx cf = cf_re + cf_im * I;
  for (int i = 0; i < 8; ++i)
    for (int j = 0; j < 8; ++j) {
      double s = 0.0;
      for (int q = 0; q < 6; ++q) s += C[i][q] * C[j][q] * ABC2_DPTS[0][q];
      out[8 * i + j] = cf * s * A;
    }
}

/* _matrix_builder of robin_abc_order2.py: Mat[itri*64 .. +64] += B(itri) */
int oracle_abc2_entries(const double *nodes, int64_t nN, const int64_t *tris, int64_t F, const int64_t *btris,
                        int64_t nb, double cf_re, double cf_im, cplx *Mat) {
  for (int64_t i = 0; i < nb; ++i) {
    const int64_t t = btris[i];
    if (t < 0 || t >= F) return -1;
    for (int v = 0; v < 3; ++v)
      if (tris[v * F + t] < 0 || tris[v * F + t] >= nN) return -1;
  }
  for (int64_t i = 0; i < nb; ++i) {
    const int64_t t = btris[i];
    double X[3][3];
    for (int d = 0; d < 3; ++d)
      for (int v = 0; v < 3; ++v) X[d][v] = nodes[d * nN + tris[v * F + t]];
    cplx B[64];
    oracle_abc2_block(X, cf_re, cf_im, B);
    for (int k = 0; k < 64; ++k) Mat[t * 64 + k] += B[k];
  }
  return 0;
}
