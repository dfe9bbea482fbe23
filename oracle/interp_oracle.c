/* CPU ORACLE -- test infrastructure, not product code.
 *
 * Plain-C restatement of EMerge's Nedelec-2 field interpolation and the port
 * overlap integral of its S-parameter post-processing:
 *
 *   ned2_tet_interp        compiled/base/interp.py:286-387 (the solution at
 *                          points inside given tets; NaN outside)
 *   tet_coefficients       compiled/base/interp.py:82-166 (its own copy: the
 *                          determinant's terms are divided by 6 one by one)
 *   local_mapping          compiled/base/interp.py:192-226
 *   _ne0_3d/_ne2_3d/_nf0_3d/_nf1_3d  compiled/ccbf.py:537,569,790,808
 *   surface_integral /     mth/integrals.py:13-24,64-103 with
 *   generate_int_points_tri / calc_area  mth/optimized.py
 *   sparam_field_power     physics/microwave/sparam.py:62-97 (integrand
 *                          (E - Q U) . conj(U), without the 1/(2 Z0))
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>

typedef double complex cplx;

static void tet_coefficients_interp(const double *xs, const double *ys, const double *zs, double aa[4],
                                    double bb[4], double cc[4], double dd[4], double *V) {
  double x1 = xs[0], x2 = xs[1], x3 = xs[2], x4 = xs[3];
  double y1 = ys[0], y2 = ys[1], y3 = ys[2], y4 = ys[3];
  double z1 = zs[0], z2 = zs[1], z3 = zs[2], z4 = zs[3];
  double v = -x1 * y2 * z3 / 6 + x1 * y2 * z4 / 6 + x1 * y3 * z2 / 6 - x1 * y3 * z4 / 6 - x1 * y4 * z2 / 6 +
             x1 * y4 * z3 / 6 + x2 * y1 * z3 / 6 - x2 * y1 * z4 / 6 - x2 * y3 * z1 / 6 + x2 * y3 * z4 / 6 +
             x2 * y4 * z1 / 6 - x2 * y4 * z3 / 6 - x3 * y1 * z2 / 6 + x3 * y1 * z4 / 6 + x3 * y2 * z1 / 6 -
             x3 * y2 * z4 / 6 - x3 * y4 * z1 / 6 + x3 * y4 * z2 / 6 + x4 * y1 * z2 / 6 - x4 * y1 * z3 / 6 -
             x4 * y2 * z1 / 6 + x4 * y2 * z3 / 6 + x4 * y3 * z1 / 6 - x4 * y3 * z2 / 6;
  *V = fabs(v);
  aa[0] = x2 * y3 * z4 - x2 * y4 * z3 - x3 * y2 * z4 + x3 * y4 * z2 + x4 * y2 * z3 - x4 * y3 * z2;
  aa[1] = -x1 * y3 * z4 + x1 * y4 * z3 + x3 * y1 * z4 - x3 * y4 * z1 - x4 * y1 * z3 + x4 * y3 * z1;
  aa[2] = x1 * y2 * z4 - x1 * y4 * z2 - x2 * y1 * z4 + x2 * y4 * z1 + x4 * y1 * z2 - x4 * y2 * z1;
  aa[3] = -x1 * y2 * z3 + x1 * y3 * z2 + x2 * y1 * z3 - x2 * y3 * z1 - x3 * y1 * z2 + x3 * y2 * z1;
  bb[0] = -y2 * z3 + y2 * z4 + y3 * z2 - y3 * z4 - y4 * z2 + y4 * z3;
  bb[1] = y1 * z3 - y1 * z4 - y3 * z1 + y3 * z4 + y4 * z1 - y4 * z3;
  bb[2] = -y1 * z2 + y1 * z4 + y2 * z1 - y2 * z4 - y4 * z1 + y4 * z2;
  bb[3] = y1 * z2 - y1 * z3 - y2 * z1 + y2 * z3 + y3 * z1 - y3 * z2;
  cc[0] = x2 * z3 - x2 * z4 - x3 * z2 + x3 * z4 + x4 * z2 - x4 * z3;
  cc[1] = -x1 * z3 + x1 * z4 + x3 * z1 - x3 * z4 - x4 * z1 + x4 * z3;
  cc[2] = x1 * z2 - x1 * z4 - x2 * z1 + x2 * z4 + x4 * z1 - x4 * z2;
  cc[3] = -x1 * z2 + x1 * z3 + x2 * z1 - x2 * z3 - x3 * z1 + x3 * z2;
  dd[0] = -x2 * y3 + x2 * y4 + x3 * y2 - x3 * y4 - x4 * y2 + x4 * y3;
  dd[1] = x1 * y3 - x1 * y4 - x3 * y1 + x3 * y4 + x4 * y1 - x4 * y3;
  dd[2] = -x1 * y2 + x1 * y4 + x2 * y1 - x2 * y4 - x4 * y1 + x4 * y2;
  dd[3] = x1 * y2 - x1 * y3 - x2 * y1 + x2 * y3 + x3 * y1 - x3 * y2;
}

static int local_of(const int64_t g[4], int64_t id) {
  for (int q = 0; q < 4; ++q)
    if (g[q] == id) return q;
  return -1;
}

/* E at one point of tet t: sum over the 20 DoFs in dofcode order */
static void interp_point(const double *nodes, int64_t nN, const int64_t *tets, int64_t nT, const int64_t *edges,
                         int64_t E, const int64_t *tris, int64_t F, const int64_t *t2e, const int64_t *t2t,
                         const cplx *x, int64_t t, double px, double py, double pz, cplx out[3]) {
  int64_t g[4];
  double xs[4], ys[4], zs[4];
  for (int q = 0; q < 4; ++q) {
    g[q] = tets[q * nT + t];
    xs[q] = nodes[0 * nN + g[q]];
    ys[q] = nodes[1 * nN + g[q]];
    zs[q] = nodes[2 * nN + g[q]];
  }
  double a[4], b[4], c[4], d[4], V;
  tet_coefficients_interp(xs, ys, zs, a, b, c, d, &V);
  double co[4][4];
  for (int m = 0; m < 4; ++m) {
    co[0][m] = a[m] / (6 * V);
    co[1][m] = b[m] / (6 * V);
    co[2][m] = c[m] / (6 * V);
    co[3][m] = d[m] / (6 * V);
  }
  cplx ex = 0, ey = 0, ez = 0;
  for (int idof = 0; idof < 20; ++idof) {
    int kind, i, j, k = 0;
    int64_t dof;
    if (idof < 12) {
      const int s = idof % 6;
      const int64_t e = t2e[s * nT + t];
      i = local_of(g, edges[0 * E + e]);
      j = local_of(g, edges[1 * E + e]);
      kind = idof < 6 ? 0 : 1;
      dof = idof < 6 ? e : e + E;
    } else {
      const int f = (idof - 12) % 4;
      const int64_t tr = t2t[f * nT + t];
      i = local_of(g, tris[0 * F + tr]);
      j = local_of(g, tris[1 * F + tr]);
      k = local_of(g, tris[2 * F + tr]);
      kind = idof < 16 ? 2 : 3;
      dof = idof < 16 ? 2 * E + tr : 2 * E + F + tr;
    }
    const double Li = co[0][i] + co[1][i] * px + co[2][i] * py + co[3][i] * pz;
    const double Lj = co[0][j] + co[1][j] * px + co[2][j] * py + co[3][j] * pz;
    const double Lk = co[0][k] + co[1][k] * px + co[2][k] * py + co[3][k] * pz;
    double f0, f1, f2;
    if (kind == 0) {
      f0 = -Lj * co[1][i] + Li * co[1][j];
      f1 = -Lj * co[2][i] + Li * co[2][j];
      f2 = -Lj * co[3][i] + Li * co[3][j];
    } else if (kind == 1) {
      const double t4 = Li - Lj;
      f0 = t4 * (Li * co[1][j] - Lj * co[1][i]);
      f1 = t4 * (Li * co[2][j] - Lj * co[2][i]);
      f2 = t4 * (Li * co[3][j] - Lj * co[3][i]);
    } else if (kind == 2) {
      f0 = -Li * (Lk * co[1][j] - Lj * co[1][k]);
      f1 = -Li * (Lk * co[2][j] - Lj * co[2][k]);
      f2 = -Li * (Lk * co[3][j] - Lj * co[3][k]);
    } else {
      f0 = -Lj * (Lk * co[1][i] - Li * co[1][k]);
      f1 = -Lj * (Lk * co[2][i] - Li * co[2][k]);
      f2 = -Lj * (Lk * co[3][i] - Li * co[3][k]);
    }
    ex += f0 * x[dof];
    ey += f1 * x[dof];
    ez += f2 * x[dof];
  }
  out[0] = ex;
  out[1] = ey;
  out[2] = ez;
}

/* ned2_tet_interp: Eout[3][np] for points pts[3][np] lying in tets tet_of[np]
 * (-1: outside, NaN as in the reference) */
void oracle_ned2_interp(const double *nodes, int64_t nN, const int64_t *tets, int64_t nT, const int64_t *edges,
                        int64_t E, const int64_t *tris, int64_t F, const int64_t *t2e, const int64_t *t2t,
                        const cplx *x, const double *pts, int64_t np, const int64_t *tet_of, cplx *Eout) {
  for (int64_t n = 0; n < np; ++n) {
    cplx e[3] = {NAN, NAN, NAN};
    if (tet_of[n] >= 0 && tet_of[n] < nT)
      interp_point(nodes, nN, tets, nT, edges, E, tris, F, t2e, t2t, x, tet_of[n], pts[n], pts[np + n],
                   pts[2 * np + n], e);
    for (int c = 0; c < 3; ++c) Eout[c * np + n] = e[c];
  }
}

/* The port overlap of sparam_field_power: per boundary tri btris[i] (lying on
 * a face of tet btet[i]) the Dunavant-rule points x = v1 L1 + v2 L2 + v3 L3
 * (rule[4][nq]: weights, L1, L2, L3), the integrand (E - q U) . conj(U) with
 * U[3][nq][nb], and per_tri[i] = area * sum_q w_q integrand (surface_integral
 * with unit constants); *total = their sum in list order. */
void oracle_port_overlap(const double *nodes, int64_t nN, const int64_t *tets, int64_t nT, const int64_t *edges,
                         int64_t E, const int64_t *tris, int64_t F, const int64_t *t2e, const int64_t *t2t,
                         const cplx *x, const int64_t *btris, const int64_t *btet, int64_t nb, const double *rule,
                         int nq, const cplx *U, double q, cplx *per_tri, cplx *total) {
  cplx tot = 0;
  for (int64_t i = 0; i < nb; ++i) {
    const int64_t tr = btris[i];
    double v[3][3];
    for (int a = 0; a < 3; ++a)
      for (int d = 0; d < 3; ++d) v[a][d] = nodes[d * nN + tris[a * F + tr]];
    double e1[3], e2[3];
    for (int d = 0; d < 3; ++d) {
      e1[d] = v[1][d] - v[0][d];
      e2[d] = v[2][d] - v[0][d];
    }
    const double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2],
                 cz = e1[0] * e2[1] - e1[1] * e2[0];
    const double area = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
    cplx field = 0;
    for (int k = 0; k < nq; ++k) {
      const double L1 = rule[1 * nq + k], L2 = rule[2 * nq + k], L3 = rule[3 * nq + k];
      const double px = v[0][0] * L1 + v[1][0] * L2 + v[2][0] * L3;
      const double py = v[0][1] * L1 + v[1][1] * L2 + v[2][1] * L3;
      const double pz = v[0][2] * L1 + v[1][2] * L2 + v[2][2] * L3;
      cplx e[3];
      interp_point(nodes, nN, tets, nT, edges, E, tris, F, t2e, t2t, x, btet[i], px, py, pz, e);
      cplx s = 0;
      for (int c = 0; c < 3; ++c) {
        const cplx u = U[(c * nq + k) * nb + i];
        s += (e[c] - q * u) * conj(u);
      }
      field += rule[k] * s;
    }
    per_tri[i] = field * area;
    tot += per_tri[i];
  }
  *total = tot;
}
