/* CPU ORACLE -- test infrastructure, not product code.
 *
 * Plain-C restatement of EMerge's heat-conduction volume assembly on
 * Lagrange-2 tetrahedra (physics/heatconduction/assembly/grad.py):
 *
 *   tet_coefficients      grad.py:23-111 (determinant terms divided by 6)
 *   grad_n1 / grad_n2     grad.py:115-146 (vertex and edge function gradients)
 *   LOCAL_EDGE_MAP, DPTS  grad.py:178-189 (the rule's digits exactly as given)
 *   leg2_tet_stiff        grad.py:199-260: K_ij = V sum_q w_q (k grad N_i) . grad N_j
 *   leg2_tet_mass         grad.py:263-330: M_ij = rho_cp V sum_q w_q N_i N_j
 *   _stiff/_mass_matrix_builder  grad.py:333-400 (COO, 100 slots per tet,
 *                         rows[p + 10 ii + jj] = t2f[ii], cols = t2f[jj])
 */
#include <math.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static const double HEAT_DPTS[5][11] = {
    {-0.078933, 0.04573333, 0.04573333, 0.04573333, 0.04573333, 0.14933333, 0.14933333, 0.14933333, 0.14933333,
     0.14933333, 0.14933333},
    {0.25, 0.78571429, 0.07142857, 0.07142857, 0.07142857, 0.39940358, 0.39940358, 0.39940358, 0.10059642, 0.10059642,
     0.10059642},
    {0.25, 0.07142857, 0.07142857, 0.07142857, 0.78571429, 0.10059642, 0.10059642, 0.39940358, 0.39940358, 0.39940358,
     0.10059642},
    {0.25, 0.07142857, 0.07142857, 0.78571429, 0.07142857, 0.39940358, 0.10059642, 0.10059642, 0.39940358, 0.10059642,
     0.39940358},
    {0.25, 0.07142857, 0.78571429, 0.07142857, 0.07142857, 0.10059642, 0.39940358, 0.10059642, 0.10059642, 0.39940358,
     0.39940358},
};
static const int LEM[2][6] = {{0, 0, 0, 1, 1, 2}, {1, 2, 3, 2, 3, 3}};

static void heat_coefficients(const double X[3][4], double co[4][4], double *Vout) {
  const double x1 = X[0][0], x2 = X[0][1], x3 = X[0][2], x4 = X[0][3];
  const double y1 = X[1][0], y2 = X[1][1], y3 = X[1][2], y4 = X[1][3];
  const double z1 = X[2][0], z2 = X[2][1], z3 = X[2][2], z4 = X[2][3];
  const double V = fabs(-x1 * y2 * z3 / 6 + x1 * y2 * z4 / 6 + x1 * y3 * z2 / 6 - x1 * y3 * z4 / 6 -
                        x1 * y4 * z2 / 6 + x1 * y4 * z3 / 6 + x2 * y1 * z3 / 6 - x2 * y1 * z4 / 6 -
                        x2 * y3 * z1 / 6 + x2 * y3 * z4 / 6 + x2 * y4 * z1 / 6 - x2 * y4 * z3 / 6 -
                        x3 * y1 * z2 / 6 + x3 * y1 * z4 / 6 + x3 * y2 * z1 / 6 - x3 * y2 * z4 / 6 -
                        x3 * y4 * z1 / 6 + x3 * y4 * z2 / 6 + x4 * y1 * z2 / 6 - x4 * y1 * z3 / 6 -
                        x4 * y2 * z1 / 6 + x4 * y2 * z3 / 6 + x4 * y3 * z1 / 6 - x4 * y3 * z2 / 6);
  double a[4], b[4], c[4], d[4];
  a[0] = x2 * y3 * z4 - x2 * y4 * z3 - x3 * y2 * z4 + x3 * y4 * z2 + x4 * y2 * z3 - x4 * y3 * z2;
  a[1] = -x1 * y3 * z4 + x1 * y4 * z3 + x3 * y1 * z4 - x3 * y4 * z1 - x4 * y1 * z3 + x4 * y3 * z1;
  a[2] = x1 * y2 * z4 - x1 * y4 * z2 - x2 * y1 * z4 + x2 * y4 * z1 + x4 * y1 * z2 - x4 * y2 * z1;
  a[3] = -x1 * y2 * z3 + x1 * y3 * z2 + x2 * y1 * z3 - x2 * y3 * z1 - x3 * y1 * z2 + x3 * y2 * z1;
  b[0] = -y2 * z3 + y2 * z4 + y3 * z2 - y3 * z4 - y4 * z2 + y4 * z3;
  b[1] = y1 * z3 - y1 * z4 - y3 * z1 + y3 * z4 + y4 * z1 - y4 * z3;
  b[2] = -y1 * z2 + y1 * z4 + y2 * z1 - y2 * z4 - y4 * z1 + y4 * z2;
  b[3] = y1 * z2 - y1 * z3 - y2 * z1 + y2 * z3 + y3 * z1 - y3 * z2;
  c[0] = x2 * z3 - x2 * z4 - x3 * z2 + x3 * z4 + x4 * z2 - x4 * z3;
  c[1] = -x1 * z3 + x1 * z4 + x3 * z1 - x3 * z4 - x4 * z1 + x4 * z3;
  c[2] = x1 * z2 - x1 * z4 - x2 * z1 + x2 * z4 + x4 * z1 - x4 * z2;
  c[3] = -x1 * z2 + x1 * z3 + x2 * z1 - x2 * z3 - x3 * z1 + x3 * z2;
  d[0] = -x2 * y3 + x2 * y4 + x3 * y2 - x3 * y4 - x4 * y2 + x4 * y3;
  d[1] = x1 * y3 - x1 * y4 - x3 * y1 + x3 * y4 + x4 * y1 - x4 * y3;
  d[2] = -x1 * y2 + x1 * y4 + x2 * y1 - x2 * y4 - x4 * y1 + x4 * y2;
  d[3] = x1 * y2 - x1 * y3 - x2 * y1 + x2 * y3 + x3 * y1 - x3 * y2;
  for (int m = 0; m < 4; ++m) {
    co[0][m] = a[m] / (6 * V);
    co[1][m] = b[m] / (6 * V);
    co[2][m] = c[m] / (6 * V);
    co[3][m] = d[m] / (6 * V);
  }
  *Vout = V;
}

/* gradient of function iv (0-3 vertex, 4-9 edge) at point (x, y, z) */
static void heat_grad(const double co[4][4], int iv, double x, double y, double z, double g[3]) {
  if (iv < 4) {
    const double a = co[0][iv], b = co[1][iv], c = co[2][iv], d = co[3][iv];
    const double q = 4 * (b * x + c * y + d * z) + (4 * a - 1);
    g[0] = q * b;
    g[1] = q * c;
    g[2] = q * d;
  } else {
    const int i = LEM[0][iv - 4], j = LEM[1][iv - 4];
    const double L1 = 4 * (co[0][i] + co[1][i] * x + co[2][i] * y + co[3][i] * z);
    const double L2 = 4 * (co[0][j] + co[1][j] * x + co[2][j] * y + co[3][j] * z);
    g[0] = L2 * co[1][i] + L1 * co[1][j];
    g[1] = L2 * co[2][i] + L1 * co[2][j];
    g[2] = L2 * co[3][i] + L1 * co[3][j];
  }
}

/* leg2_tet_stiff: out[100] row-major, k row-major 3x3 */
void oracle_leg2_stiff(const double X[3][4], const double k[9], double *out) {
  double co[4][4], V;
  heat_coefficients(X, co, &V);
  double xs[11], ys[11], zs[11];
  for (int q = 0; q < 11; ++q) {
    xs[q] = X[0][0] * HEAT_DPTS[1][q] + X[0][1] * HEAT_DPTS[2][q] + X[0][2] * HEAT_DPTS[3][q] + X[0][3] * HEAT_DPTS[4][q];
    ys[q] = X[1][0] * HEAT_DPTS[1][q] + X[1][1] * HEAT_DPTS[2][q] + X[1][2] * HEAT_DPTS[3][q] + X[1][3] * HEAT_DPTS[4][q];
    zs[q] = X[2][0] * HEAT_DPTS[1][q] + X[2][1] * HEAT_DPTS[2][q] + X[2][2] * HEAT_DPTS[3][q] + X[2][3] * HEAT_DPTS[4][q];
  }
  for (int i = 0; i < 10; ++i)
    for (int j = 0; j < 10; ++j) {
      double s = 0.0;
      for (int q = 0; q < 11; ++q) {
        double gi[3], gj[3];
        heat_grad(co, i, xs[q], ys[q], zs[q], gi);
        heat_grad(co, j, xs[q], ys[q], zs[q], gj);
        const double kg0 = k[0] * gi[0] + k[1] * gi[1] + k[2] * gi[2];
        const double kg1 = k[3] * gi[0] + k[4] * gi[1] + k[5] * gi[2];
        const double kg2 = k[6] * gi[0] + k[7] * gi[1] + k[8] * gi[2];
        s += (kg0 * gj[0] + kg1 * gj[1] + kg2 * gj[2]) * HEAT_DPTS[0][q];
      }
      out[10 * i + j] = s * V;
    }
}

/* leg2_tet_mass: out[100] row-major */
void oracle_leg2_mass(const double X[3][4], double rho_cp, double *out) {
  double co[4][4], V;
  heat_coefficients(X, co, &V);
  for (int i = 0; i < 10; ++i)
    for (int j = i; j < 10; ++j) {
      double val = 0.0;
      for (int q = 0; q < 11; ++q) {
        const double x = X[0][0] * HEAT_DPTS[1][q] + X[0][1] * HEAT_DPTS[2][q] + X[0][2] * HEAT_DPTS[3][q] +
                         X[0][3] * HEAT_DPTS[4][q];
        const double y = X[1][0] * HEAT_DPTS[1][q] + X[1][1] * HEAT_DPTS[2][q] + X[1][2] * HEAT_DPTS[3][q] +
                         X[1][3] * HEAT_DPTS[4][q];
        const double z = X[2][0] * HEAT_DPTS[1][q] + X[2][1] * HEAT_DPTS[2][q] + X[2][2] * HEAT_DPTS[3][q] +
                         X[2][3] * HEAT_DPTS[4][q];
        double L[4];
        for (int m = 0; m < 4; ++m) L[m] = co[0][m] + co[1][m] * x + co[2][m] * y + co[3][m] * z;
        const double N1 = i < 4 ? L[i] * (2.0 * L[i] - 1.0) : 4.0 * L[LEM[0][i - 4]] * L[LEM[1][i - 4]];
        const double N2 = j < 4 ? L[j] * (2.0 * L[j] - 1.0) : 4.0 * L[LEM[0][j - 4]] * L[LEM[1][j - 4]];
        val += HEAT_DPTS[0][q] * N1 * N2;
      }
      out[10 * i + j] = val * rho_cp * V;
      out[10 * j + i] = val * rho_cp * V;
    }
}

/* _stiff_matrix_builder / _mass_matrix_builder: values[100 nT] in the
 * reference's COO layout. coef: kind 0 -> conductivity [3][3][nT], kind 1 ->
 * rho_cp [nT]. */
int oracle_leg2_builder(const double *nodes, int64_t nN, const int64_t *tets, int64_t nT, const double *coef, int kind,
                        double *values) {
#pragma omp parallel for schedule(static)
  for (int64_t t = 0; t < nT; ++t) {
    double X[3][4];
    for (int d = 0; d < 3; ++d)
      for (int v = 0; v < 4; ++v) X[d][v] = nodes[d * nN + tets[v * nT + t]];
    if (kind == 0) {
      double k[9];
      for (int r = 0; r < 9; ++r) k[r] = coef[r * nT + t];
      oracle_leg2_stiff(X, k, values + 100 * t);
    } else {
      oracle_leg2_mass(X, coef[t], values + 100 * t);
    }
  }
  return 0;
}

/* scatter_to_csc_f8 (mth/csc_cast.py:150-177) for real data: the CSC value of
 * each entry is the sum of its COO slots in the pattern's slot order */
void oracle_scatter_f8(const double *data, const int64_t *perm, const int64_t *target, const int64_t *col_offsets,
                       int64_t N, double *data_csc, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < N; ++i)
    for (int64_t k = col_offsets[i]; k < col_offsets[i + 1]; ++k) data_csc[target[k]] += data[perm[k]];
}
