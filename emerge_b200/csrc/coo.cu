// coo.cu -- a general COO -> CSC mapping on the device, and the Lagrange-2
// heat-conduction element kernels that use it.
//
// Replaces CSCMapping.from_rowcol / precompute_csc_pattern / to_csc for any
// (rows, cols) slot list (mth/csc_cast.py:51-177), as the heat-conduction
// assembly calls them (physics/heatconduction/assembly/grad.py:403-460), and
// leg2_tet_stiff / leg2_tet_mass with their COO builders (grad.py:199-400).
// Pattern: slots counted per column, scattered into column buckets, each
// bucket sorted by (row, slot) -- a fixed order, whatever order the scatter
// left them in -- and its distinct rows become the column's entries; the value
// of an entry is the sum of its slots in that order. Built with -fmad=false:
// the element arithmetic follows the reference's CPU operation order.
#include "common.cuh"

namespace emg {
namespace {

__global__ void k_coo_count(const int32_t *cols, int64_t S, int64_t N, int32_t *cnt, int64_t *st) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const int32_t c = cols[s];
  if (c < 0 || c >= N) {
    flag(st, EMG_ST_INDEX, s);
    return;
  }
  atomicAdd(&cnt[c], 1);
}

__global__ void k_coo_scatter(const int32_t *cols, int64_t S, int64_t N, const int32_t *col_off, int32_t *cursor,
                              int32_t *perm) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  const int32_t c = cols[s];
  if (c < 0 || c >= N) return;
  perm[col_off[c] + atomicAdd(&cursor[c], 1)] = (int32_t)s;
}

// sort each column's slots by (row, slot) and count its distinct rows
__global__ void k_coo_sort_count(const int32_t *rows, const int32_t *col_off, int64_t N, int32_t *perm,
                                 int32_t *col_nnz, int64_t *st) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int32_t b = col_off[c], e = col_off[c + 1];
  for (int32_t i = b + 1; i < e; ++i) {  // insertion sort, stable on the slot index
    const int32_t v = perm[i];
    const int64_t kv = ((int64_t)rows[v] << 32) | (uint32_t)v;
    int32_t j = i - 1;
    while (j >= b && (((int64_t)rows[perm[j]] << 32) | (uint32_t)perm[j]) > kv) {
      perm[j + 1] = perm[j];
      --j;
    }
    perm[j + 1] = v;
  }
  int32_t n = 0;
  for (int32_t i = b; i < e; ++i) {
    const int32_t r = rows[perm[i]];
    if (r < 0 || r >= N) flag(st, EMG_ST_INDEX, perm[i]);
    if (i == b || r != rows[perm[i - 1]]) ++n;
  }
  col_nnz[c] = n;
}

// indices (distinct rows) and, per entry, the first of its sorted slots
__global__ void k_coo_fill(const int32_t *rows, const int32_t *col_off, int64_t N, const int32_t *perm,
                           const int32_t *indptr, int32_t *indices, int32_t *run) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int32_t b = col_off[c], e = col_off[c + 1];
  int32_t q = indptr[c];
  for (int32_t i = b; i < e; ++i) {
    const int32_t r = rows[perm[i]];
    if (i == b || r != rows[perm[i - 1]]) {
      indices[q] = r;
      run[q] = i;
      ++q;
    }
  }
}

__global__ void k_coo_run_end(const int32_t *run, int64_t nnz, int64_t S, int32_t *run_end) {
  if (blockIdx.x == 0 && threadIdx.x == 0) run_end[nnz] = (int32_t)S;
}

template <typename V>
__global__ void k_coo_gather(const int32_t *perm, const int32_t *run, int64_t nnz, int64_t S, const V *vals, V *out);

template <>
__global__ void k_coo_gather<double>(const int32_t *perm, const int32_t *run, int64_t nnz, int64_t S,
                                     const double *vals, double *out) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x) {
    const int32_t b = run[p], e = run[p + 1];
    double s = 0.0;
    for (int32_t i = b; i < e && i < S; ++i) s += vals[perm[i]];
    out[p] = s;
  }
}

template <>
__global__ void k_coo_gather<double2>(const int32_t *perm, const int32_t *run, int64_t nnz, int64_t S,
                                      const double2 *vals, double2 *out) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x) {
    const int32_t b = run[p], e = run[p + 1];
    double sr = 0.0, si = 0.0;
    for (int32_t i = b; i < e && i < S; ++i) {
      const double2 v = vals[perm[i]];
      sr += v.x;
      si += v.y;
    }
    out[p] = make_double2(sr, si);
  }
}

// rows/cols of an element with D DoFs per tet in the reference layout
// (femdata.py:58-73, grad.py:350-354): slot p = D^2 t + D ii + jj
__global__ void k_coo_rowcol(const int32_t *t2f, int D, int64_t nT, int32_t *rows, int32_t *cols) {
  const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t D2 = (int64_t)D * D;
  if (s >= D2 * nT) return;
  const int64_t t = s / D2;
  const int r = (int)(s % D2);
  rows[s] = t2f[(int64_t)(r / D) * nT + t];
  cols[s] = t2f[(int64_t)(r % D) * nT + t];
}

// ---------------------------------------------------------------------------
// Lagrange-2 heat elements (grad.py:178-330)
__constant__ double kHW[11] = {-0.078933,  0.04573333, 0.04573333, 0.04573333, 0.04573333, 0.14933333,
                               0.14933333, 0.14933333, 0.14933333, 0.14933333, 0.14933333};
__constant__ double kHP[4][11] = {
    {0.25, 0.78571429, 0.07142857, 0.07142857, 0.07142857, 0.39940358, 0.39940358, 0.39940358, 0.10059642, 0.10059642,
     0.10059642},
    {0.25, 0.07142857, 0.07142857, 0.07142857, 0.78571429, 0.10059642, 0.10059642, 0.39940358, 0.39940358, 0.39940358,
     0.10059642},
    {0.25, 0.07142857, 0.07142857, 0.78571429, 0.07142857, 0.39940358, 0.10059642, 0.10059642, 0.39940358, 0.10059642,
     0.39940358},
    {0.25, 0.07142857, 0.78571429, 0.07142857, 0.07142857, 0.10059642, 0.39940358, 0.10059642, 0.10059642, 0.39940358,
     0.39940358}};
__constant__ int kLEM[2][6] = {{0, 0, 0, 1, 1, 2}, {1, 2, 3, 2, 3, 3}};

__device__ bool leg2_coefficients(const double X[3][4], double co[4][4], double &Vout) {
  const double x1 = X[0][0], x2 = X[0][1], x3 = X[0][2], x4 = X[0][3];
  const double y1 = X[1][0], y2 = X[1][1], y3 = X[1][2], y4 = X[1][3];
  const double z1 = X[2][0], z2 = X[2][1], z3 = X[2][2], z4 = X[2][3];
  const double V = fabs(-x1 * y2 * z3 / 6 + x1 * y2 * z4 / 6 + x1 * y3 * z2 / 6 - x1 * y3 * z4 / 6 -
                        x1 * y4 * z2 / 6 + x1 * y4 * z3 / 6 + x2 * y1 * z3 / 6 - x2 * y1 * z4 / 6 -
                        x2 * y3 * z1 / 6 + x2 * y3 * z4 / 6 + x2 * y4 * z1 / 6 - x2 * y4 * z3 / 6 -
                        x3 * y1 * z2 / 6 + x3 * y1 * z4 / 6 + x3 * y2 * z1 / 6 - x3 * y2 * z4 / 6 -
                        x3 * y4 * z1 / 6 + x3 * y4 * z2 / 6 + x4 * y1 * z2 / 6 - x4 * y1 * z3 / 6 -
                        x4 * y2 * z1 / 6 + x4 * y2 * z3 / 6 + x4 * y3 * z1 / 6 - x4 * y3 * z2 / 6);
  double c4[4][4];
  c4[0][0] = x2 * y3 * z4 - x2 * y4 * z3 - x3 * y2 * z4 + x3 * y4 * z2 + x4 * y2 * z3 - x4 * y3 * z2;
  c4[0][1] = -x1 * y3 * z4 + x1 * y4 * z3 + x3 * y1 * z4 - x3 * y4 * z1 - x4 * y1 * z3 + x4 * y3 * z1;
  c4[0][2] = x1 * y2 * z4 - x1 * y4 * z2 - x2 * y1 * z4 + x2 * y4 * z1 + x4 * y1 * z2 - x4 * y2 * z1;
  c4[0][3] = -x1 * y2 * z3 + x1 * y3 * z2 + x2 * y1 * z3 - x2 * y3 * z1 - x3 * y1 * z2 + x3 * y2 * z1;
  c4[1][0] = -y2 * z3 + y2 * z4 + y3 * z2 - y3 * z4 - y4 * z2 + y4 * z3;
  c4[1][1] = y1 * z3 - y1 * z4 - y3 * z1 + y3 * z4 + y4 * z1 - y4 * z3;
  c4[1][2] = -y1 * z2 + y1 * z4 + y2 * z1 - y2 * z4 - y4 * z1 + y4 * z2;
  c4[1][3] = y1 * z2 - y1 * z3 - y2 * z1 + y2 * z3 + y3 * z1 - y3 * z2;
  c4[2][0] = x2 * z3 - x2 * z4 - x3 * z2 + x3 * z4 + x4 * z2 - x4 * z3;
  c4[2][1] = -x1 * z3 + x1 * z4 + x3 * z1 - x3 * z4 - x4 * z1 + x4 * z3;
  c4[2][2] = x1 * z2 - x1 * z4 - x2 * z1 + x2 * z4 + x4 * z1 - x4 * z2;
  c4[2][3] = -x1 * z2 + x1 * z3 + x2 * z1 - x2 * z3 - x3 * z1 + x3 * z2;
  c4[3][0] = -x2 * y3 + x2 * y4 + x3 * y2 - x3 * y4 - x4 * y2 + x4 * y3;
  c4[3][1] = x1 * y3 - x1 * y4 - x3 * y1 + x3 * y4 + x4 * y1 - x4 * y3;
  c4[3][2] = -x1 * y2 + x1 * y4 + x2 * y1 - x2 * y4 - x4 * y1 + x4 * y2;
  c4[3][3] = x1 * y2 - x1 * y3 - x2 * y1 + x2 * y3 + x3 * y1 - x3 * y2;
  for (int r = 0; r < 4; ++r)
    for (int m = 0; m < 4; ++m) co[r][m] = c4[r][m] / (6 * V);
  Vout = V;
  return V > 0.0 && isfinite(V);
}

__device__ __forceinline__ void leg2_grad(const double co[4][4], int iv, double x, double y, double z, double g[3]) {
  if (iv < 4) {
    const double a = co[0][iv], b = co[1][iv], c = co[2][iv], d = co[3][iv];
    const double q = 4 * (b * x + c * y + d * z) + (4 * a - 1);
    g[0] = q * b, g[1] = q * c, g[2] = q * d;
  } else {
    const int i = kLEM[0][iv - 4], j = kLEM[1][iv - 4];
    const double L1 = 4 * (co[0][i] + co[1][i] * x + co[2][i] * y + co[3][i] * z);
    const double L2 = 4 * (co[0][j] + co[1][j] * x + co[2][j] * y + co[3][j] * z);
    g[0] = L2 * co[1][i] + L1 * co[1][j];
    g[1] = L2 * co[2][i] + L1 * co[2][j];
    g[2] = L2 * co[3][i] + L1 * co[3][j];
  }
}

// one tet per thread: the 10x10 block in the reference's row-major COO slots
__global__ void __launch_bounds__(128) k_leg2_element(const double *nodes, int64_t nN, const int32_t *tets, int64_t nT,
                                                      const double *coef, int kind, double *out, int64_t *st) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nT) return;
  double X[3][4];
  bool ok = true;
  for (int v = 0; v < 4; ++v) {
    const int64_t n = tets[v * nT + t];
    ok = ok && n >= 0 && n < nN;
    for (int d = 0; d < 3; ++d) X[d][v] = ok ? nodes[d * nN + n] : 0.0;
  }
  double co[4][4], V = 0.0;
  if (ok) ok = leg2_coefficients(X, co, V);
  double *o = out + 100 * t;
  if (!ok) {
    flag(st, EMG_ST_DEGENERATE, t);
    for (int k = 0; k < 100; ++k) o[k] = 0.0;
    return;
  }
  double px[11], py[11], pz[11];
  for (int q = 0; q < 11; ++q) {
    px[q] = X[0][0] * kHP[0][q] + X[0][1] * kHP[1][q] + X[0][2] * kHP[2][q] + X[0][3] * kHP[3][q];
    py[q] = X[1][0] * kHP[0][q] + X[1][1] * kHP[1][q] + X[1][2] * kHP[2][q] + X[1][3] * kHP[3][q];
    pz[q] = X[2][0] * kHP[0][q] + X[2][1] * kHP[1][q] + X[2][2] * kHP[2][q] + X[2][3] * kHP[3][q];
  }
  if (kind == 0) {
    double k[9];
    for (int r = 0; r < 9; ++r) k[r] = coef[r * nT + t];
#pragma unroll 1
    for (int i = 0; i < 10; ++i)
#pragma unroll 1
      for (int j = 0; j < 10; ++j) {
        double s = 0.0;
#pragma unroll 1
        for (int q = 0; q < 11; ++q) {
          double gi[3], gj[3];
          leg2_grad(co, i, px[q], py[q], pz[q], gi);
          leg2_grad(co, j, px[q], py[q], pz[q], gj);
          const double kg0 = k[0] * gi[0] + k[1] * gi[1] + k[2] * gi[2];
          const double kg1 = k[3] * gi[0] + k[4] * gi[1] + k[5] * gi[2];
          const double kg2 = k[6] * gi[0] + k[7] * gi[1] + k[8] * gi[2];
          s += (kg0 * gj[0] + kg1 * gj[1] + kg2 * gj[2]) * kHW[q];
        }
        o[10 * i + j] = s * V;
      }
  } else {
    const double rho = coef[t];
#pragma unroll 1
    for (int i = 0; i < 10; ++i)
#pragma unroll 1
      for (int j = i; j < 10; ++j) {
        double val = 0.0;
#pragma unroll 1
        for (int q = 0; q < 11; ++q) {
          double L[4];
          for (int m = 0; m < 4; ++m) L[m] = co[0][m] + co[1][m] * px[q] + co[2][m] * py[q] + co[3][m] * pz[q];
          const double N1 = i < 4 ? L[i] * (2.0 * L[i] - 1.0) : 4.0 * L[kLEM[0][i - 4]] * L[kLEM[1][i - 4]];
          const double N2 = j < 4 ? L[j] * (2.0 * L[j] - 1.0) : 4.0 * L[kLEM[0][j - 4]] * L[kLEM[1][j - 4]];
          val += kHW[q] * N1 * N2;
        }
        o[10 * i + j] = val * rho * V;
        o[10 * j + i] = val * rho * V;
      }
  }
}

struct CooWs {
  int32_t *cnt, *col_off, *cursor, *col_nnz;
  long long *bsum;
};

CooWs coo_ws(void *d_ws, int64_t N) {
  char *w = static_cast<char *>(d_ws);
  CooWs r;
  size_t o = 0;
  r.cnt = reinterpret_cast<int32_t *>(w + o);
  o = align_up(o + (size_t)(N + 1) * 4, 256);
  r.col_off = reinterpret_cast<int32_t *>(w + o);
  o = align_up(o + (size_t)(N + 1) * 4, 256);
  r.cursor = reinterpret_cast<int32_t *>(w + o);
  o = align_up(o + (size_t)(N + 1) * 4, 256);
  r.col_nnz = reinterpret_cast<int32_t *>(w + o);
  o = align_up(o + (size_t)(N + 1) * 4, 256);
  r.bsum = reinterpret_cast<long long *>(w + o);
  return r;
}

}  // namespace
}  // namespace emg

using namespace emg;

extern "C" {

int emg_coo_init(int64_t S, int64_t N, emg_coo_map *m) {
  if (!m) return fail(EMG_EINVAL, "null descriptor");
  if (S < 0 || N < 0) return fail(EMG_EINVAL, "negative size");
  if (S >= INT32_MAX || N >= INT32_MAX) return fail(EMG_ERANGE, "more than 2^31 slots or columns");
  memset(m, 0, sizeof(*m));
  m->S = S;
  m->N = N;
  m->perm_bytes = align_up((size_t)(S > 0 ? S : 1) * 4, 256);
  m->run_bytes = align_up((size_t)(S + 1) * 4, 256);
  m->workspace_bytes = align_up((size_t)(N + 1) * 4, 256) * 4 + scan_i32_bsum_bytes(N + 1);
  return EMG_OK;
}

int emg_coo_rowcol(const int32_t *d_tet_to_field, int dofs_per_tet, int64_t n_tets, int32_t *d_rows, int32_t *d_cols,
                   emg_stream_t stream) {
  if (dofs_per_tet <= 0 || n_tets < 0) return fail(EMG_EINVAL, "bad sizes");
  const int64_t n = (int64_t)dofs_per_tet * dofs_per_tet * n_tets;
  if (n == 0) return EMG_OK;
  if (n >= INT32_MAX) return fail(EMG_ERANGE, "more than 2^31 slots");
  if (!d_tet_to_field || !d_rows || !d_cols) return fail(EMG_EINVAL, "null pointer");
  k_coo_rowcol<<<grid_for(n, 256), 256, 0, S(stream)>>>(d_tet_to_field, dofs_per_tet, n_tets, d_rows, d_cols);
  return launch_check("k_coo_rowcol");
}

int emg_coo_build(emg_coo_map *m, const int32_t *d_rows, const int32_t *d_cols, int32_t *d_perm, void *d_ws,
                  int32_t *d_indptr, int64_t *d_status, emg_stream_t stream) {
  if (!m || !d_perm || !d_ws || !d_indptr || !d_status || (m->S > 0 && (!d_rows || !d_cols)))
    return fail(EMG_EINVAL, "null pointer");
  cudaStream_t s = S(stream);
  CooWs w = coo_ws(d_ws, m->N);
  int rc;
  if ((rc = status_reset(d_status, s))) return rc;
  CUDA_TRY(cudaMemsetAsync(w.cnt, 0, (size_t)(m->N + 1) * 4, s));
  CUDA_TRY(cudaMemsetAsync(w.cursor, 0, (size_t)(m->N + 1) * 4, s));
  if (m->S > 0) {
    k_coo_count<<<grid_for(m->S, 256), 256, 0, s>>>(d_cols, m->S, m->N, w.cnt, d_status);
    if ((rc = launch_check("k_coo_count"))) return rc;
  }
  if ((rc = scan_i32(w.cnt, m->N, w.col_off, w.bsum, d_status, s))) return rc;
  if (m->S > 0) {
    k_coo_scatter<<<grid_for(m->S, 256), 256, 0, s>>>(d_cols, m->S, m->N, w.col_off, w.cursor, d_perm);
    if ((rc = launch_check("k_coo_scatter"))) return rc;
  }
  if (m->N > 0) {
    k_coo_sort_count<<<grid_for(m->N, 128), 128, 0, s>>>(d_rows, w.col_off, m->N, d_perm, w.col_nnz, d_status);
    if ((rc = launch_check("k_coo_sort_count"))) return rc;
  }
  if ((rc = scan_i32(w.col_nnz, m->N, d_indptr, w.bsum, d_status, s))) return rc;
  int32_t nnz = 0;
  int64_t h_st[2] = {0, 0};
  CUDA_TRY(cudaMemcpyAsync(&nnz, d_indptr + m->N, 4, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(h_st, d_status, 16, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (h_st[0]) return fail(EMG_EMESH, "COO pattern: index out of range at slot %lld", (long long)h_st[1]);
  m->nnz = nnz;
  return EMG_OK;
}

int emg_coo_finish(const emg_coo_map *m, const int32_t *d_rows, const int32_t *d_perm, void *d_ws,
                   const int32_t *d_indptr, int32_t *d_indices, int32_t *d_run, emg_stream_t stream) {
  if (!m || !d_perm || !d_ws || !d_indptr || !d_run) return fail(EMG_EINVAL, "null pointer");
  if (m->nnz > 0 && (!d_indices || !d_rows)) return fail(EMG_EINVAL, "null pointer");
  cudaStream_t s = S(stream);
  CooWs w = coo_ws(d_ws, m->N);
  if (m->N > 0) {
    k_coo_fill<<<grid_for(m->N, 128), 128, 0, s>>>(d_rows, w.col_off, m->N, d_perm, d_indptr, d_indices, d_run);
    const int rc = launch_check("k_coo_fill");
    if (rc) return rc;
  }
  k_coo_run_end<<<1, 32, 0, s>>>(d_run, m->nnz, m->S, d_run);
  return launch_check("k_coo_run_end");
}

int emg_coo_gather(const emg_coo_map *m, const int32_t *d_perm, const int32_t *d_run, int is_complex,
                   const void *d_values, void *d_out, emg_stream_t stream) {
  if (!m) return fail(EMG_EINVAL, "null descriptor");
  if (m->nnz == 0) return EMG_OK;
  if (!d_perm || !d_run || !d_values || !d_out) return fail(EMG_EINVAL, "null pointer");
  const int g = persistent_ctas(8);
  if (is_complex)
    k_coo_gather<double2><<<g, 256, 0, S(stream)>>>(d_perm, d_run, m->nnz, m->S,
                                                    static_cast<const double2 *>(d_values),
                                                    static_cast<double2 *>(d_out));
  else
    k_coo_gather<double><<<g, 256, 0, S(stream)>>>(d_perm, d_run, m->nnz, m->S, static_cast<const double *>(d_values),
                                                   static_cast<double *>(d_out));
  return launch_check("k_coo_gather");
}

int emg_leg2_element(const double *d_nodes, int64_t n_nodes, const int32_t *d_tets, int64_t n_tets,
                     const double *d_coef, int kind, double *d_values, int64_t *d_status, emg_stream_t stream) {
  if (kind != 0 && kind != 1) return fail(EMG_EINVAL, "kind must be 0 (stiffness) or 1 (mass)");
  if (n_tets < 0 || n_nodes < 0) return fail(EMG_EINVAL, "negative size");
  if (n_tets == 0) return EMG_OK;
  if (!d_nodes || !d_tets || !d_coef || !d_values) return fail(EMG_EINVAL, "null pointer");
  k_leg2_element<<<grid_for(n_tets, 128), 128, 0, S(stream)>>>(d_nodes, n_nodes, d_tets, n_tets, d_coef, kind,
                                                               d_values, d_status);
  return launch_check("k_leg2_element");
}

}  // extern "C"
