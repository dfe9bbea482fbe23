// robin.cu -- the Robin (third-kind) boundary term of ports and absorbing
// boundaries on Nedelec-2 triangles, scattered into A's pattern.
//
// Replaces assemble_robin_bc / compute_bc_entries / ned2_tri_stiff
// (physics/microwave/assembly/robinbc.py:316-451) and the caller's
// K += field.generate_csc(B_matrix_robin) (assembler.py:576-630,
// elements/femdata.py:104-118). The triangle block is linear in gamma, so it
// is built once for gamma = 1 and every frequency adds gamma(f) times it.
#include "common.cuh"

namespace emg {
namespace {

// 6-point triangle rule of robinbc.py:189-196 (weights, barycentric L1..L3)
__constant__ double kTW[6] = {0.10995174365532200, 0.10995174365532200, 0.10995174365532200,
                              0.22338158967801100, 0.22338158967801100, 0.22338158967801100};
__constant__ double kTL[3][6] = {
    {0.81684757298045896, 0.09157621350977101, 0.09157621350977101, 0.10810301816807000, 0.44594849091596500,
     0.44594849091596500},
    {0.09157621350977101, 0.81684757298045896, 0.09157621350977101, 0.44594849091596500, 0.10810301816807000,
     0.44594849091596500},
    {0.09157621350977004, 0.09157621350977008, 0.81684757298045807, 0.44594849091596500, 0.44594849091596500,
     0.10810301816807000}};

// the second-order ABC correction's own copy of the rule, 14 digits
// (robin_abc_order2.py:89-98)
__constant__ double kAW[6] = {0.10995174365532, 0.10995174365532, 0.10995174365532,
                              0.22338158967801, 0.22338158967801, 0.22338158967801};
__constant__ double kAL[3][6] = {
    {0.81684757298046, 0.09157621350977, 0.09157621350977, 0.10810301816807, 0.44594849091597, 0.44594849091597},
    {0.09157621350977, 0.81684757298046, 0.09157621350977, 0.44594849091597, 0.10810301816807, 0.44594849091597},
    {0.09157621350977, 0.09157621350977, 0.81684757298046, 0.44594849091597, 0.44594849091597, 0.10810301816807}};

// position of row `row` in column `col` of the CSC pattern, or -1
__device__ __forceinline__ int64_t find_in_column(const int32_t *indptr, const int32_t *indices, int64_t col,
                                                  int32_t row) {
  int64_t lo = indptr[col], hi = (int64_t)indptr[col + 1] - 1;
  while (lo <= hi) {
    const int64_t mid = (lo + hi) >> 1;
    const int32_t v = indices[mid];
    if (v == row) return mid;
    if (v < row) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

// The triangle's own frame (origin at vertex 0, x along edge 0->1, z the
// normal; construct_local_vertices, robinbc.py:165-183) and its barycentric
// coefficients (tri_coefficients :200-221). Returns the area.
struct TriFrame {
  double xh[3], yh[3], tx[3], ty[3], ca[3], cb[3], cc[3];
};

// abc2: the coefficients as robin_abc_order2.py's tri_coefficients forms them
// (:100-122: its own signed-area expression, sign and |area| applied apart)
__device__ double tri_frame(const double *nodes, int64_t nN, const int32_t v[3], TriFrame &T, bool abc2 = false) {
  double X[3][3];
  for (int d = 0; d < 3; ++d)
    for (int k = 0; k < 3; ++k) X[d][k] = nodes[d * nN + v[k]];
  double e1[3], e2[3], zh[3];
  for (int d = 0; d < 3; ++d) {
    e1[d] = X[d][1] - X[d][0];
    e2[d] = X[d][2] - X[d][0];
  }
  zh[0] = e1[1] * e2[2] - e1[2] * e2[1];
  zh[1] = e1[2] * e2[0] - e1[0] * e2[2];
  zh[2] = e1[0] * e2[1] - e1[1] * e2[0];
  const double nz = sqrt(zh[0] * zh[0] + zh[1] * zh[1] + zh[2] * zh[2]);
  const double nx = sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
  for (int d = 0; d < 3; ++d) {
    zh[d] /= nz;
    T.xh[d] = e1[d] / nx;
  }
  T.yh[0] = zh[1] * T.xh[2] - zh[2] * T.xh[1];
  T.yh[1] = zh[2] * T.xh[0] - zh[0] * T.xh[2];
  T.yh[2] = zh[0] * T.xh[1] - zh[1] * T.xh[0];
  const double ny = sqrt(T.yh[0] * T.yh[0] + T.yh[1] * T.yh[1] + T.yh[2] * T.yh[2]);
  for (int d = 0; d < 3; ++d) T.yh[d] /= ny;
  for (int k = 0; k < 3; ++k) {
    double rx = 0.0, ry = 0.0;
    for (int d = 0; d < 3; ++d) {
      const double r = X[d][k] - X[d][0];
      rx += T.xh[d] * r;
      ry += T.yh[d] * r;
    }
    T.tx[k] = rx;
    T.ty[k] = ry;
  }
  const double *tx = T.tx, *ty = T.ty;
  const double a0 = tx[1] * ty[2] - ty[1] * tx[2], a1 = tx[2] * ty[0] - ty[2] * tx[0], a2 = tx[0] * ty[1] - ty[0] * tx[1];
  const double b0 = ty[1] - ty[2], b1 = ty[2] - ty[0], b2 = ty[0] - ty[1];
  const double c0 = tx[2] - tx[1], c1 = tx[0] - tx[2], c2 = tx[1] - tx[0];
  if (abc2) {
    const double sA = 0.5 * ((tx[0] - tx[2]) * (ty[1] - ty[0]) - (tx[0] - tx[1]) * (ty[2] - ty[0]));
    const double sg = sA > 0.0 ? 1.0 : (sA < 0.0 ? -1.0 : 0.0), A2 = 2 * fabs(sA);
    T.ca[0] = a0 * sg / A2, T.ca[1] = a1 * sg / A2, T.ca[2] = a2 * sg / A2;
    T.cb[0] = b0 * sg / A2, T.cb[1] = b1 * sg / A2, T.cb[2] = b2 * sg / A2;
    T.cc[0] = c0 * sg / A2, T.cc[1] = c1 * sg / A2, T.cc[2] = c2 * sg / A2;
    return fabs(sA);
  }
  const double sA = 0.5 * (b0 * c1 - b1 * c0);
  const double s2 = 2 * sA;
  T.ca[0] = a0 / s2, T.ca[1] = a1 / s2, T.ca[2] = a2 / s2;
  T.cb[0] = b0 / s2, T.cb[1] = b1 / s2, T.cb[2] = b2 / s2;
  T.cc[0] = c0 / s2, T.cc[1] = c1 / s2, T.cc[2] = c2 / s2;
  return fabs(sA);
}

// the scalar 2-D curls of the 8 functions at point q of the ABC rule
// (_curl_ne0_2d, _curl_ne2_2d, _curl_nf0_2d, _curl_nf1_2d, ccbf.py:168-410)
__device__ __forceinline__ void tri_curls(const TriFrame &T, int q, double C[8]) {
  const double xs = T.tx[0] * kAL[0][q] + T.tx[1] * kAL[1][q] + T.tx[2] * kAL[2][q];
  const double ys = T.ty[0] * kAL[0][q] + T.ty[1] * kAL[1][q] + T.ty[2] * kAL[2][q];
  const int EI[3] = {0, 1, 0}, EJ[3] = {1, 2, 2};
  const double *a = T.ca, *b = T.cb, *c = T.cc;
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    const int i = EI[e], j = EJ[e];
    C[e] = 2 * b[i] * c[j] - 2 * b[j] * c[i];
    const double t0 = b[j] * xs, t1 = c[j] * ys, t2 = t0 + t1 + a[j], t3 = a[i] + b[i] * xs + c[i] * ys;
    C[3 + e] = -(b[i] - b[j]) * (t2 * c[i] - t3 * c[j]) + (c[i] - c[j]) * (t2 * b[i] - t3 * b[j]) +
               2 * (b[i] * c[j] - b[j] * c[i]) * (-t0 - t1 + t3 - a[j]);
  }
  {
    const double t0 = a[2] + b[2] * xs + c[2] * ys, t1 = a[1] + b[1] * xs + c[1] * ys;
    C[6] = -b[0] * (t0 * c[1] - t1 * c[2]) + c[0] * (t0 * b[1] - t1 * b[2]) +
           2 * (b[1] * c[2] - b[2] * c[1]) * (a[0] + b[0] * xs + c[0] * ys);
  }
  {
    const double t0 = a[2] + b[2] * xs + c[2] * ys, t1 = a[0] + b[0] * xs + c[0] * ys;
    C[7] = -b[1] * (t0 * c[0] - t1 * c[2]) + c[1] * (t0 * b[0] - t1 * b[2]) +
           2 * (b[0] * c[2] - b[2] * c[0]) * (a[1] + b[1] * xs + c[1] * ys);
  }
}

// the 8 Volakis functions (ne0, ne2 on (0,1), (1,2), (0,2); nf0, nf1) at point q
__device__ __forceinline__ void tri_functions(const TriFrame &T, int q, double f[8][2]) {
  const double xs = T.tx[0] * kTL[0][q] + T.tx[1] * kTL[1][q] + T.tx[2] * kTL[2][q];
  const double ys = T.ty[0] * kTL[0][q] + T.ty[1] * kTL[1][q] + T.ty[2] * kTL[2][q];
  double L[3];
  for (int m = 0; m < 3; ++m) L[m] = T.ca[m] + T.cb[m] * xs + T.cc[m] * ys;
  const int EI[3] = {0, 1, 0}, EJ[3] = {1, 2, 2};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int a = EI[k], b = EJ[k];
    const double wx = L[a] * T.cb[b] - L[b] * T.cb[a], wy = L[a] * T.cc[b] - L[b] * T.cc[a];
    f[k][0] = wx;
    f[k][1] = wy;
    const double s = L[a] - L[b];
    f[3 + k][0] = s * wx;
    f[3 + k][1] = s * wy;
  }
  f[6][0] = L[0] * (L[1] * T.cb[2] - L[2] * T.cb[1]);
  f[6][1] = L[0] * (L[1] * T.cc[2] - L[2] * T.cc[1]);
  f[7][0] = L[1] * (L[0] * T.cb[2] - L[2] * T.cb[0]);
  f[7][1] = L[1] * (L[0] * T.cc[2] - L[2] * T.cc[0]);
}

// DoFs of the triangle (nedelec2.py:69-79): edges, edges + E, tri + 2E, tri + 2E + F
__device__ __forceinline__ void tri_dofs(const int32_t e[3], int64_t t, int64_t E, int64_t F, int64_t dof[8]) {
  for (int k = 0; k < 3; ++k) {
    dof[k] = e[k];
    dof[3 + k] = e[k] + E;
  }
  dof[6] = 2 * E + t;
  dof[7] = 2 * E + F + t;
}

// load and check a boundary triangle's vertices and edges
__device__ __forceinline__ bool tri_load(const int32_t *tris, const int32_t *tri_to_edge, int64_t F, int64_t nN,
                                         int64_t E, int64_t t, int32_t v[3], int32_t e[3]) {
  bool ok = t >= 0 && t < F;
  for (int k = 0; k < 3; ++k) {
    v[k] = ok ? tris[k * F + t] : 0;
    e[k] = ok ? tri_to_edge[k * F + t] : 0;
    ok = ok && v[k] >= 0 && v[k] < nN && e[k] >= 0 && e[k] < E;
  }
  return ok;
}

// One boundary triangle per thread: the 8x8 block for gamma = 1 in the
// triangle's own plane (origin at vertex 0, x along edge 0->1), the 2-D
// Volakis functions ne0, ne2 on the vertex pairs (0,1), (1,2), (0,2) and
// nf0, nf1 on (0,1,2) at the 6 points, B[a][b] = A * sum_q w_q f_a . f_b
// (computed for a <= b and mirrored), and each slot's position in A.
// ABC2: the second-order ABC correction instead (_abc_order_2_terms,
// robin_abc_order2.py:143-217), B[a][b] = A * sum_q w_q c_a c_b with c the
// scalar 2-D curls; the reference's divergence matrix is identically zero
// (it writes the first function's divergence into a buffer the inner loop
// overwrites), so the block is the curl term alone.
template <bool ABC2>
__global__ void __launch_bounds__(128)
    k_robin_build(const double *nodes, int64_t nN, const int32_t *tris, const int32_t *tri_to_edge, int64_t F,
                  int64_t E, const int32_t *btris, int64_t nb, const int32_t *tri_dofs_in, const int32_t *indptr,
                  const int32_t *indices, int64_t N, uint64_t *keys, double2 *vals, int64_t *st) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  uint64_t *my_keys = keys + i * 64;
  double2 *my_vals = vals + i * 64;
  const int64_t t = btris[i];
  int32_t v[3], e[3];
  if (!tri_load(tris, tri_to_edge, F, nN, E, t, v, e)) {
    flag(st, EMG_ST_INDEX, i);
    for (int k = 0; k < 64; ++k) {
      my_keys[k] = ~0ull;
      my_vals[k] = make_double2(0.0, 0.0);
    }
    return;
  }
  TriFrame T;
  const double area = tri_frame(nodes, nN, v, T, ABC2);
  if (!(area > 0.0) || !isfinite(area)) flag(st, EMG_ST_DEGENERATE, i);
  double B[36];
  for (int k = 0; k < 36; ++k) B[k] = 0.0;
#pragma unroll 1
  for (int q = 0; q < 6; ++q) {
    if constexpr (ABC2) {
      double C[8];
      tri_curls(T, q, C);
      const double w = kAW[q];
      int k = 0;
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = a; b < 8; ++b, ++k) B[k] += C[a] * C[b] * w;
    } else {
      double f[8][2];
      tri_functions(T, q, f);
      const double w = kTW[q];
      int k = 0;
#pragma unroll
      for (int a = 0; a < 8; ++a)
#pragma unroll
        for (int b = a; b < 8; ++b, ++k) B[k] += (f[a][0] * f[b][0] + f[a][1] * f[b][1]) * w;
    }
  }
  int64_t dof[8];
  tri_dofs(e, t, E, F, dof);
  if (tri_dofs_in)  // the caller's numbering (a partitioned field's other side)
    for (int a = 0; a < 8; ++a) dof[a] = tri_dofs_in[i * 8 + a];
  int k = 0;
  for (int a = 0; a < 8; ++a)
    for (int b = a; b < 8; ++b, ++k) {
      const double val = B[k] * area;
      for (int pass = 0; pass < (a == b ? 1 : 2); ++pass) {
        const int r = pass ? b : a, c = pass ? a : b;  // slot (r, c): row dof[r] in column dof[c]
        const int slot = 8 * r + c;
        int64_t pos = -1;
        if (dof[c] >= 0 && dof[r] >= 0 && dof[c] < N && dof[r] < N)
          pos = find_in_column(indptr, indices, dof[c], (int32_t)dof[r]);
        if (pos < 0) flag(st, EMG_ST_INDEX, i);
        my_keys[slot] = pos < 0 ? ~0ull : (((uint64_t)pos << 32) | (uint64_t)(i * 64 + slot));
        my_vals[slot] = make_double2(val, 0.0);
      }
    }
}

// Port forcing vector (ned2_tri_force, robinbc.py:220-277): per boundary
// triangle b_a = -A sum_q w_q f_a(q) . (U projected on the triangle's plane),
// U complex [3][6][nb] at the points of generate_points_3d (:104-135); one
// key (DoF << 32 | slot) and value per (triangle, DoF).
__global__ void __launch_bounds__(128)
    k_robin_force(const double *nodes, int64_t nN, const int32_t *tris, const int32_t *tri_to_edge, int64_t F,
                  int64_t E, const int32_t *btris, int64_t nb, const double2 *U, uint64_t *keys, double2 *vals,
                  int64_t *st) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  const int64_t t = btris[i];
  int32_t v[3], e[3];
  if (!tri_load(tris, tri_to_edge, F, nN, E, t, v, e)) {
    flag(st, EMG_ST_INDEX, i);
    for (int k = 0; k < 8; ++k) {
      keys[i * 8 + k] = ~0ull;
      vals[i * 8 + k] = make_double2(0.0, 0.0);
    }
    return;
  }
  TriFrame T;
  const double area = tri_frame(nodes, nN, v, T);
  if (!(area > 0.0) || !isfinite(area)) flag(st, EMG_ST_DEGENERATE, i);
  double br[8], bi[8];
  for (int k = 0; k < 8; ++k) br[k] = bi[k] = 0.0;
#pragma unroll 1
  for (int q = 0; q < 6; ++q) {
    double f[8][2];
    tri_functions(T, q, f);
    double ux_r = 0.0, ux_i = 0.0, uy_r = 0.0, uy_i = 0.0;
    for (int d = 0; d < 3; ++d) {
      const double2 u = U[(d * 6 + q) * nb + i];
      ux_r += T.xh[d] * u.x;
      ux_i += T.xh[d] * u.y;
      uy_r += T.yh[d] * u.x;
      uy_i += T.yh[d] * u.y;
    }
    const double w = kTW[q];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      br[k] += w * (f[k][0] * ux_r + f[k][1] * uy_r);
      bi[k] += w * (f[k][0] * ux_i + f[k][1] * uy_i);
    }
  }
  int64_t dof[8];
  tri_dofs(e, t, E, F, dof);
  for (int k = 0; k < 8; ++k) {
    keys[i * 8 + k] = ((uint64_t)dof[k] << 32) | (uint64_t)(i * 8 + k);
    vals[i * 8 + k] = make_double2(-area * br[k], -area * bi[k]);
  }
}

__global__ void k_pad_keys(uint64_t *keys, int64_t from, int64_t n_keys) {
  const int64_t k = from + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n_keys) keys[k] = ~0ull;
}

// A[p] += gamma * (sum of the slots of target p, in slot order); one thread
// per sorted slot, the first slot of each target sums its run
__global__ void k_robin_apply(const uint64_t *keys, int64_t n_slots, const double2 *vals, double gr, double gi,
                              double2 *A, int64_t nnz) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_slots) return;
  const uint64_t key = keys[i];
  if (key == ~0ull) return;
  const uint64_t p = key >> 32;
  if (i > 0 && (keys[i - 1] >> 32) == p) return;
  if ((int64_t)p >= nnz) return;
  double sr = 0.0, si = 0.0;
  for (int64_t j = i; j < n_slots; ++j) {
    const uint64_t kj = keys[j];
    if ((kj >> 32) != p || kj == ~0ull) break;
    const uint64_t slot = kj & 0xffffffffu;
    if ((int64_t)slot >= n_slots) continue;
    const double2 v = vals[slot];
    sr += v.x;
    si += v.y;
  }
  double2 a = A[p];
  a.x += gr * sr - gi * si;
  a.y += gr * si + gi * sr;
  A[p] = a;
}

}  // namespace
}  // namespace emg

using namespace emg;

extern "C" {

int emg_robin_init(int64_t n_btris, emg_robin *r) {
  if (!r) return fail(EMG_EINVAL, "null robin descriptor");
  if (n_btris < 0) return fail(EMG_EINVAL, "negative triangle count");
  if (n_btris * 64 >= (1LL << 32)) return fail(EMG_ERANGE, "more than 2^26 boundary triangles");
  r->n_btris = n_btris;
  r->n_slots = n_btris * 64;
  r->n_keys = n_btris > 0 ? pow2_at_least(r->n_slots) : 0;
  r->keys_bytes = (size_t)r->n_keys * 8;
  r->values_bytes = (size_t)r->n_slots * 16;
  r->n_fslots = n_btris * 8;
  r->n_fkeys = n_btris > 0 ? pow2_at_least(r->n_fslots) : 0;
  r->fkeys_bytes = (size_t)r->n_fkeys * 8;
  r->fvalues_bytes = (size_t)r->n_fslots * 16;
  return EMG_OK;
}

}  // extern "C"

namespace {
int robin_build(bool abc2, const emg_robin *r, const double *d_nodes, int64_t n_nodes, const int32_t *d_tris,
                const int32_t *d_tri_to_edge, int64_t n_tris, int64_t n_edges, const int32_t *d_btris,
                const int32_t *d_tri_dofs, const int32_t *d_indptr, const int32_t *d_indices, int64_t N,
                uint64_t *d_keys, void *d_values, int64_t *d_status, emg_stream_t stream) {
  if (!r) return fail(EMG_EINVAL, "null robin descriptor");
  if (r->n_btris == 0) return EMG_OK;
  if (!d_nodes || !d_tris || !d_tri_to_edge || !d_btris || !d_indptr || !d_indices || !d_keys || !d_values)
    return fail(EMG_EINVAL, "null pointer");
  if (n_nodes <= 0 || n_tris <= 0 || n_edges <= 0 || N < 2 * n_edges + 2 * n_tris || N >= (1LL << 31))
    return fail(EMG_EINVAL, "bad sizes (N must be at least 2 E + 2 F and below 2^31)");
  cudaStream_t s = S(stream);
  auto *vals = static_cast<double2 *>(d_values);
  if (abc2)
    k_robin_build<true><<<grid_for(r->n_btris, 128), 128, 0, s>>>(
        d_nodes, n_nodes, d_tris, d_tri_to_edge, n_tris, n_edges, d_btris, r->n_btris, d_tri_dofs, d_indptr, d_indices,
        N, d_keys, vals, d_status);
  else
    k_robin_build<false><<<grid_for(r->n_btris, 128), 128, 0, s>>>(
        d_nodes, n_nodes, d_tris, d_tri_to_edge, n_tris, n_edges, d_btris, r->n_btris, d_tri_dofs, d_indptr, d_indices,
        N, d_keys, vals, d_status);
  int rc = launch_check("k_robin_build");
  if (rc) return rc;
  if (r->n_keys > r->n_slots) {
    k_pad_keys<<<grid_for(r->n_keys - r->n_slots, 256), 256, 0, s>>>(d_keys, r->n_slots, r->n_keys);
    if ((rc = launch_check("k_pad_keys"))) return rc;
  }
  return sort_u64(d_keys, r->n_keys, s);
}
}  // namespace

extern "C" {

int emg_robin_build(const emg_robin *r, const double *d_nodes, int64_t n_nodes, const int32_t *d_tris,
                    const int32_t *d_tri_to_edge, int64_t n_tris, int64_t n_edges, const int32_t *d_btris,
                    const int32_t *d_indptr, const int32_t *d_indices, int64_t N, uint64_t *d_keys, void *d_values,
                    int64_t *d_status, emg_stream_t stream) {
  return robin_build(false, r, d_nodes, n_nodes, d_tris, d_tri_to_edge, n_tris, n_edges, d_btris, nullptr, d_indptr,
                     d_indices, N, d_keys, d_values, d_status, stream);
}

int emg_robin_build_dofs(const emg_robin *r, const double *d_nodes, int64_t n_nodes, const int32_t *d_tris,
                         const int32_t *d_tri_to_edge, int64_t n_tris, int64_t n_edges, const int32_t *d_btris,
                         const int32_t *d_tri_dofs, const int32_t *d_indptr, const int32_t *d_indices, int64_t N,
                         uint64_t *d_keys, void *d_values, int64_t *d_status, emg_stream_t stream) {
  if (!d_tri_dofs && r && r->n_btris) return fail(EMG_EINVAL, "null triangle DoF array");
  return robin_build(false, r, d_nodes, n_nodes, d_tris, d_tri_to_edge, n_tris, n_edges, d_btris, d_tri_dofs, d_indptr,
                     d_indices, N, d_keys, d_values, d_status, stream);
}

int emg_abc2_build(const emg_robin *r, const double *d_nodes, int64_t n_nodes, const int32_t *d_tris,
                   const int32_t *d_tri_to_edge, int64_t n_tris, int64_t n_edges, const int32_t *d_btris,
                   const int32_t *d_indptr, const int32_t *d_indices, int64_t N, uint64_t *d_keys, void *d_values,
                   int64_t *d_status, emg_stream_t stream) {
  return robin_build(true, r, d_nodes, n_nodes, d_tris, d_tri_to_edge, n_tris, n_edges, d_btris, nullptr, d_indptr,
                     d_indices, N, d_keys, d_values, d_status, stream);
}

int emg_robin_apply(const emg_robin *r, const uint64_t *d_keys, const void *d_values, double gamma_re,
                    double gamma_im, void *d_A, int64_t nnz, emg_stream_t stream) {
  if (!r) return fail(EMG_EINVAL, "null robin descriptor");
  if (r->n_btris == 0) return EMG_OK;
  if (!d_keys || !d_values || !d_A) return fail(EMG_EINVAL, "null pointer");
  k_robin_apply<<<grid_for(r->n_slots, 256), 256, 0, S(stream)>>>(
      d_keys, r->n_slots, static_cast<const double2 *>(d_values), gamma_re, gamma_im, static_cast<double2 *>(d_A),
      nnz);
  return launch_check("k_robin_apply");
}

int emg_robin_force(const emg_robin *r, const double *d_nodes, int64_t n_nodes, const int32_t *d_tris,
                    const int32_t *d_tri_to_edge, int64_t n_tris, int64_t n_edges, const int32_t *d_btris,
                    const void *d_U, uint64_t *d_fkeys, void *d_fvalues, void *d_b, int64_t N, int64_t *d_status,
                    emg_stream_t stream) {
  if (!r) return fail(EMG_EINVAL, "null robin descriptor");
  if (r->n_btris == 0) return EMG_OK;
  if (!d_nodes || !d_tris || !d_tri_to_edge || !d_btris || !d_U || !d_fkeys || !d_fvalues || !d_b)
    return fail(EMG_EINVAL, "null pointer");
  if (n_nodes <= 0 || n_tris <= 0 || n_edges <= 0 || N < 2 * n_edges + 2 * n_tris)
    return fail(EMG_EINVAL, "bad sizes (N must be at least 2 E + 2 F)");
  cudaStream_t s = S(stream);
  k_robin_force<<<grid_for(r->n_btris, 128), 128, 0, s>>>(d_nodes, n_nodes, d_tris, d_tri_to_edge, n_tris, n_edges,
                                                          d_btris, r->n_btris, static_cast<const double2 *>(d_U),
                                                          d_fkeys, static_cast<double2 *>(d_fvalues), d_status);
  int rc = launch_check("k_robin_force");
  if (rc) return rc;
  if (r->n_fkeys > r->n_fslots) {
    k_pad_keys<<<grid_for(r->n_fkeys - r->n_fslots, 256), 256, 0, s>>>(d_fkeys, r->n_fslots, r->n_fkeys);
    if ((rc = launch_check("k_pad_keys"))) return rc;
  }
  if ((rc = sort_u64(d_fkeys, r->n_fkeys, s))) return rc;
  k_robin_apply<<<grid_for(r->n_fslots, 256), 256, 0, s>>>(d_fkeys, r->n_fslots,
                                                           static_cast<const double2 *>(d_fvalues), 1.0, 0.0,
                                                           static_cast<double2 *>(d_b), N);
  return launch_check("k_robin_apply");
}

}  // extern "C"
