// postproc.cu -- Nedelec-2 field interpolation and the port overlap integral
// of the S-parameter post-processing, on the device.
//
// Replaces ned2_tet_interp (compiled/base/interp.py:286-387) for points whose
// tet is known, and the port-face integral of sparam_field_power
// (physics/microwave/sparam.py:62-97 through mth/integrals.py
// surface_integral :64-103): per port triangle sum_k w_k (E - Q U) . conj(U)
// times its area, E interpolated in the triangle's tet. Built with
// -fmad=false: the arithmetic follows the reference's operation order
// without fused multiply-adds, as its own CPU code does.
#include "common.cuh"

namespace emg {
namespace {

constexpr int MAX_RULE = 16;
struct TriRule {
  int nq;
  double w[MAX_RULE], l1[MAX_RULE], l2[MAX_RULE], l3[MAX_RULE];
};

struct C128 {
  double re, im;
};

// the solution at point (px, py, pz) of tet t; false for an index outside
// its array (the caller writes NaN)
__device__ bool interp_point(const double *nodes, int64_t nN, const int32_t *tets, int64_t nT, const int32_t *t2e,
                             const int32_t *t2t, int64_t E, int64_t F, const double2 *x, int64_t t, double px,
                             double py, double pz, C128 out[3]) {
  if (t < 0 || t >= nT) return false;
  int64_t g[4];
  double xs[4], ys[4], zs[4];
  for (int q = 0; q < 4; ++q) {
    g[q] = tets[q * nT + t];
    if (g[q] < 0 || g[q] >= nN) return false;
    xs[q] = nodes[g[q]];
    ys[q] = nodes[nN + g[q]];
    zs[q] = nodes[2 * nN + g[q]];
  }
  const double x1 = xs[0], x2 = xs[1], x3 = xs[2], x4 = xs[3];
  const double y1 = ys[0], y2 = ys[1], y3 = ys[2], y4 = ys[3];
  const double z1 = zs[0], z2 = zs[1], z3 = zs[2], z4 = zs[3];
  // tet_coefficients of interp.py:82-166: each determinant term divided by 6
  const double v = -x1 * y2 * z3 / 6 + x1 * y2 * z4 / 6 + x1 * y3 * z2 / 6 - x1 * y3 * z4 / 6 - x1 * y4 * z2 / 6 +
                   x1 * y4 * z3 / 6 + x2 * y1 * z3 / 6 - x2 * y1 * z4 / 6 - x2 * y3 * z1 / 6 + x2 * y3 * z4 / 6 +
                   x2 * y4 * z1 / 6 - x2 * y4 * z3 / 6 - x3 * y1 * z2 / 6 + x3 * y1 * z4 / 6 + x3 * y2 * z1 / 6 -
                   x3 * y2 * z4 / 6 - x3 * y4 * z1 / 6 + x3 * y4 * z2 / 6 + x4 * y1 * z2 / 6 - x4 * y1 * z3 / 6 -
                   x4 * y2 * z1 / 6 + x4 * y2 * z3 / 6 + x4 * y3 * z1 / 6 - x4 * y3 * z2 / 6;
  const double V6 = 6 * fabs(v);
  double co[4][4];
  co[0][0] = x2 * y3 * z4 - x2 * y4 * z3 - x3 * y2 * z4 + x3 * y4 * z2 + x4 * y2 * z3 - x4 * y3 * z2;
  co[0][1] = -x1 * y3 * z4 + x1 * y4 * z3 + x3 * y1 * z4 - x3 * y4 * z1 - x4 * y1 * z3 + x4 * y3 * z1;
  co[0][2] = x1 * y2 * z4 - x1 * y4 * z2 - x2 * y1 * z4 + x2 * y4 * z1 + x4 * y1 * z2 - x4 * y2 * z1;
  co[0][3] = -x1 * y2 * z3 + x1 * y3 * z2 + x2 * y1 * z3 - x2 * y3 * z1 - x3 * y1 * z2 + x3 * y2 * z1;
  co[1][0] = -y2 * z3 + y2 * z4 + y3 * z2 - y3 * z4 - y4 * z2 + y4 * z3;
  co[1][1] = y1 * z3 - y1 * z4 - y3 * z1 + y3 * z4 + y4 * z1 - y4 * z3;
  co[1][2] = -y1 * z2 + y1 * z4 + y2 * z1 - y2 * z4 - y4 * z1 + y4 * z2;
  co[1][3] = y1 * z2 - y1 * z3 - y2 * z1 + y2 * z3 + y3 * z1 - y3 * z2;
  co[2][0] = x2 * z3 - x2 * z4 - x3 * z2 + x3 * z4 + x4 * z2 - x4 * z3;
  co[2][1] = -x1 * z3 + x1 * z4 + x3 * z1 - x3 * z4 - x4 * z1 + x4 * z3;
  co[2][2] = x1 * z2 - x1 * z4 - x2 * z1 + x2 * z4 + x4 * z1 - x4 * z2;
  co[2][3] = -x1 * z2 + x1 * z3 + x2 * z1 - x2 * z3 - x3 * z1 + x3 * z2;
  co[3][0] = -x2 * y3 + x2 * y4 + x3 * y2 - x3 * y4 - x4 * y2 + x4 * y3;
  co[3][1] = x1 * y3 - x1 * y4 - x3 * y1 + x3 * y4 + x4 * y1 - x4 * y3;
  co[3][2] = -x1 * y2 + x1 * y4 + x2 * y1 - x2 * y4 - x4 * y1 + x4 * y2;
  co[3][3] = x1 * y2 - x1 * y3 - x2 * y1 + x2 * y3 + x3 * y1 - x3 * y2;
  for (int r = 0; r < 4; ++r)
    for (int m = 0; m < 4; ++m) co[r][m] = co[r][m] / V6;
  double L[4];
  for (int m = 0; m < 4; ++m) L[m] = co[0][m] + co[1][m] * px + co[2][m] * py + co[3][m] * pz;
  // local orientation (local_mapping): an edge runs from its lower global
  // vertex, a face's vertices are taken in ascending global order
  const int EU[6] = {0, 0, 0, 1, 3, 2}, EV[6] = {1, 2, 3, 2, 1, 3};
  const int FA[4] = {0, 0, 0, 1}, FB[4] = {1, 2, 3, 2}, FC[4] = {2, 3, 1, 3};
  double ex_r = 0, ex_i = 0, ey_r = 0, ey_i = 0, ez_r = 0, ez_i = 0;
  for (int idof = 0; idof < 20; ++idof) {
    int kind, i, j, k = 0;
    int64_t dof;
    if (idof < 12) {
      const int s = idof % 6;
      const int64_t e = t2e[s * nT + t];
      if (e < 0 || e >= E) return false;
      const int u = EU[s], w = EV[s];
      i = g[u] < g[w] ? u : w;
      j = g[u] < g[w] ? w : u;
      kind = idof < 6 ? 0 : 1;
      dof = idof < 6 ? e : e + E;
    } else {
      const int fs = (idof - 12) % 4;
      const int64_t tr = t2t[fs * nT + t];
      if (tr < 0 || tr >= F) return false;
      int a = FA[fs], b = FB[fs], c = FC[fs], tmp;
      if (g[a] > g[b]) tmp = a, a = b, b = tmp;
      if (g[b] > g[c]) tmp = b, b = c, c = tmp;
      if (g[a] > g[b]) tmp = a, a = b, b = tmp;
      i = a, j = b, k = c;
      kind = idof < 16 ? 2 : 3;
      dof = idof < 16 ? 2 * E + tr : 2 * E + F + tr;
    }
    const double Li = L[i], Lj = L[j], Lk = L[k];
    double f0, f1, f2;
    if (kind == 0) {  // ne0: Li grad Lj - Lj grad Li
      f0 = -Lj * co[1][i] + Li * co[1][j];
      f1 = -Lj * co[2][i] + Li * co[2][j];
      f2 = -Lj * co[3][i] + Li * co[3][j];
    } else if (kind == 1) {  // ne2: (Li - Lj)(Li grad Lj - Lj grad Li)
      const double t4 = Li - Lj;
      f0 = t4 * (Li * co[1][j] - Lj * co[1][i]);
      f1 = t4 * (Li * co[2][j] - Lj * co[2][i]);
      f2 = t4 * (Li * co[3][j] - Lj * co[3][i]);
    } else if (kind == 2) {  // nf0: Li (Lj grad Lk - Lk grad Lj)
      f0 = -Li * (Lk * co[1][j] - Lj * co[1][k]);
      f1 = -Li * (Lk * co[2][j] - Lj * co[2][k]);
      f2 = -Li * (Lk * co[3][j] - Lj * co[3][k]);
    } else {  // nf1: Lj (Li grad Lk - Lk grad Li)
      f0 = -Lj * (Lk * co[1][i] - Li * co[1][k]);
      f1 = -Lj * (Lk * co[2][i] - Li * co[2][k]);
      f2 = -Lj * (Lk * co[3][i] - Li * co[3][k]);
    }
    const double2 xv = x[dof];
    ex_r += f0 * xv.x, ex_i += f0 * xv.y;
    ey_r += f1 * xv.x, ey_i += f1 * xv.y;
    ez_r += f2 * xv.x, ez_i += f2 * xv.y;
  }
  out[0] = {ex_r, ex_i};
  out[1] = {ey_r, ey_i};
  out[2] = {ez_r, ez_i};
  return true;
}

__global__ void k_ned2_interp(const double *nodes, int64_t nN, const int32_t *tets, int64_t nT, const int32_t *t2e,
                              const int32_t *t2t, int64_t E, int64_t F, const double2 *x, const double *pts,
                              int64_t np, const int32_t *tet_of, double2 *out) {
  const int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= np) return;
  C128 e[3];
  if (!interp_point(nodes, nN, tets, nT, t2e, t2t, E, F, x, tet_of[n], pts[n], pts[np + n], pts[2 * np + n], e))
    e[0] = e[1] = e[2] = {nan(""), nan("")};
  for (int c = 0; c < 3; ++c) out[c * np + n] = make_double2(e[c].re, e[c].im);
}

// one port triangle per thread: area * sum_k w_k (E - q U) . conj(U)
__global__ void k_port_overlap(const double *nodes, int64_t nN, const int32_t *tets, int64_t nT, const int32_t *t2e,
                               const int32_t *t2t, const int32_t *tris, int64_t E, int64_t F, const double2 *x,
                               const int32_t *btris, const int32_t *btets, int64_t nb, TriRule rule,
                               const double2 *U, double q, double2 *per_tri, int64_t *st) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  const int64_t tr = btris[i];
  bool ok = tr >= 0 && tr < F;
  double v[3][3];
  for (int a = 0; a < 3 && ok; ++a) {
    const int64_t n = tris[a * F + tr];
    ok = n >= 0 && n < nN;
    for (int d = 0; d < 3 && ok; ++d) v[a][d] = nodes[d * nN + n];
  }
  double fr = 0.0, fi = 0.0, area = 0.0;
  if (ok) {
    double e1[3], e2[3];
    for (int d = 0; d < 3; ++d) {
      e1[d] = v[1][d] - v[0][d];
      e2[d] = v[2][d] - v[0][d];
    }
    const double cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2],
                 cz = e1[0] * e2[1] - e1[1] * e2[0];
    area = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
    for (int k = 0; k < rule.nq && ok; ++k) {
      const double px = v[0][0] * rule.l1[k] + v[1][0] * rule.l2[k] + v[2][0] * rule.l3[k];
      const double py = v[0][1] * rule.l1[k] + v[1][1] * rule.l2[k] + v[2][1] * rule.l3[k];
      const double pz = v[0][2] * rule.l1[k] + v[1][2] * rule.l2[k] + v[2][2] * rule.l3[k];
      C128 e[3];
      ok = interp_point(nodes, nN, tets, nT, t2e, t2t, E, F, x, btets[i], px, py, pz, e);
      double sr = 0.0, si = 0.0;
      for (int c = 0; c < 3; ++c) {
        const double2 u = U[((int64_t)c * rule.nq + k) * nb + i];
        const double dr = e[c].re - q * u.x, di = e[c].im - q * u.y;
        // (dr + j di)(u.x - j u.y)
        sr += dr * u.x + di * u.y;
        si += di * u.x - dr * u.y;
      }
      fr += rule.w[k] * sr;
      fi += rule.w[k] * si;
    }
  }
  if (!ok) flag(st, EMG_ST_INDEX, i);
  per_tri[i] = ok ? make_double2(fr * area, fi * area) : make_double2(0.0, 0.0);
}

// deterministic total: 1024 threads, strided partial sums, fixed tree
__global__ void __launch_bounds__(1024) k_sum_c128(const double2 *v, int64_t n, double2 *total) {
  __shared__ double sr[1024], si[1024];
  double a = 0.0, b = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += 1024) a += v[i].x, b += v[i].y;
  sr[threadIdx.x] = a;
  si[threadIdx.x] = b;
  __syncthreads();
  for (int s = 512; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sr[threadIdx.x] += sr[threadIdx.x + s], si[threadIdx.x] += si[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = make_double2(sr[0], si[0]);
}

}  // namespace
}  // namespace emg

using namespace emg;

extern "C" {

int emg_ned2_interp(const double *d_nodes, int64_t n_nodes, const int32_t *d_tets, int64_t n_tets,
                    const int32_t *d_tet_to_edge, const int32_t *d_tet_to_tri, int64_t n_edges, int64_t n_tris,
                    const void *d_x, const double *d_points, int64_t n_points, const int32_t *d_tet_of, void *d_E,
                    emg_stream_t stream) {
  if (n_points < 0 || n_nodes < 0 || n_tets < 0) return fail(EMG_EINVAL, "negative size");
  if (n_points == 0) return EMG_OK;
  if (!d_nodes || !d_tets || !d_tet_to_edge || !d_tet_to_tri || !d_x || !d_points || !d_tet_of || !d_E)
    return fail(EMG_EINVAL, "null pointer");
  k_ned2_interp<<<grid_for(n_points, 128), 128, 0, S(stream)>>>(
      d_nodes, n_nodes, d_tets, n_tets, d_tet_to_edge, d_tet_to_tri, n_edges, n_tris,
      static_cast<const double2 *>(d_x), d_points, n_points, d_tet_of, static_cast<double2 *>(d_E));
  return launch_check("k_ned2_interp");
}

int emg_port_overlap(const double *d_nodes, int64_t n_nodes, const int32_t *d_tets, int64_t n_tets,
                     const int32_t *d_tet_to_edge, const int32_t *d_tet_to_tri, const int32_t *d_tris, int64_t n_edges,
                     int64_t n_tris, const void *d_x, const int32_t *d_btris, const int32_t *d_btets, int64_t n_btris,
                     const double *h_rule, int nq, const void *d_U, double q, void *d_per_tri, void *d_total,
                     int64_t *d_status, emg_stream_t stream) {
  if (!h_rule || nq < 1 || nq > MAX_RULE) return fail(EMG_EINVAL, "rule needs 1..%d points", MAX_RULE);
  if (n_btris < 0) return fail(EMG_EINVAL, "negative size");
  if (!d_total) return fail(EMG_EINVAL, "null pointer");
  cudaStream_t s = S(stream);
  if (n_btris == 0) {
    CUDA_TRY(cudaMemsetAsync(d_total, 0, 16, s));
    return EMG_OK;
  }
  if (!d_nodes || !d_tets || !d_tet_to_edge || !d_tet_to_tri || !d_tris || !d_x || !d_btris || !d_btets || !d_U ||
      !d_per_tri)
    return fail(EMG_EINVAL, "null pointer");
  TriRule rule{};
  rule.nq = nq;
  for (int k = 0; k < nq; ++k) {
    rule.w[k] = h_rule[k];
    rule.l1[k] = h_rule[nq + k];
    rule.l2[k] = h_rule[2 * nq + k];
    rule.l3[k] = h_rule[3 * nq + k];
  }
  k_port_overlap<<<grid_for(n_btris, 128), 128, 0, s>>>(
      d_nodes, n_nodes, d_tets, n_tets, d_tet_to_edge, d_tet_to_tri, d_tris, n_edges, n_tris,
      static_cast<const double2 *>(d_x), d_btris, d_btets, n_btris, rule, static_cast<const double2 *>(d_U), q,
      static_cast<double2 *>(d_per_tri), d_status);
  int rc = launch_check("k_port_overlap");
  if (rc) return rc;
  k_sum_c128<<<1, 1024, 0, s>>>(static_cast<const double2 *>(d_per_tri), n_btris, static_cast<double2 *>(d_total));
  return launch_check("k_sum_c128");
}

}  // extern "C"
