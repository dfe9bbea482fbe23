// coo.cu -- a general COO -> CSC mapping on the device.
//
// Replaces CSCMapping.from_rowcol / precompute_csc_pattern / to_csc for any
// (rows, cols) slot list (mth/csc_cast.py:51-177), as the heat-conduction
// assembly calls them (physics/heatconduction/assembly/grad.py:403-460).
// Pattern: slots counted per column, scattered into column buckets, each
// bucket sorted by (row, slot) -- a fixed order, whatever order the scatter
// left them in -- and its distinct rows become the column's entries; the value
// of an entry is the sum of its slots in that order.
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

// the value index of slot s: s itself, or, for values stored as transposed
// D x D blocks (slot D^2 t + D i + j at D^2 t + D j + i), the swapped one
template <int D>
__device__ __forceinline__ int64_t value_index(int32_t s) {
  if constexpr (D == 0) {
    return s;
  } else {
    const int32_t t = s / (D * D), r = s - t * (D * D);
    const int32_t i = r / D, j = r - i * D;
    return (int64_t)t * (D * D) + j * D + i;
  }
}

template <int D>
__global__ void __launch_bounds__(256, 8) k_coo_gather_f8(const int32_t *perm, const int32_t *run, int64_t nnz,
                                                          int64_t S, const double *vals, double *out) {
  // the run bounds of this thread's next entry are loaded while the current
  // entry is summed (one dependent load off each entry's chain)
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int32_t nb = 0, ne = 0;
  if (p < nnz) {
    nb = run[p];
    ne = run[p + 1];
  }
  for (; p < nnz; p += stride) {
    const int32_t b = nb, e = min((int64_t)ne, S);
    if (p + stride < nnz) {
      nb = run[p + stride];
      ne = run[p + stride + 1];
    }
    double s = 0.0;
    int32_t i = b;
    for (; i + 4 <= e; i += 4) {  // four loads in flight, summed in slot order
      const int32_t p0 = perm[i], p1 = perm[i + 1], p2 = perm[i + 2], p3 = perm[i + 3];
      const double v0 = vals[value_index<D>(p0)], v1 = vals[value_index<D>(p1)];
      const double v2 = vals[value_index<D>(p2)], v3 = vals[value_index<D>(p3)];
      s += v0;
      s += v1;
      s += v2;
      s += v3;
    }
    if (i + 2 <= e) {
      const int32_t p0 = perm[i], p1 = perm[i + 1];
      const double v0 = vals[value_index<D>(p0)], v1 = vals[value_index<D>(p1)];
      s += v0;
      s += v1;
      i += 2;
    }
    if (i < e) s += vals[value_index<D>(perm[i])];
    out[p] = s;
  }
}

template <int D>
__global__ void __launch_bounds__(256) k_coo_gather_c16(const int32_t *perm, const int32_t *run, int64_t nnz,
                                                        int64_t S, const double2 *vals, double2 *out) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x) {
    const int32_t b = run[p], e = run[p + 1];
    double sr = 0.0, si = 0.0;
    for (int32_t i = b; i < e && i < S; ++i) {
      const double2 v = vals[value_index<D>(perm[i])];
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

int emg_coo_gather(const emg_coo_map *m, const int32_t *d_perm, const int32_t *d_run, int is_complex, int block_dofs,
                   const void *d_values, void *d_out, emg_stream_t stream) {
  if (!m) return fail(EMG_EINVAL, "null descriptor");
  if (block_dofs != 0 && block_dofs != 10) return fail(EMG_EINVAL, "block_dofs must be 0 or 10");
  if (block_dofs && m->S % 100) return fail(EMG_EINVAL, "slot count is not a multiple of the block size");
  if (m->nnz == 0) return EMG_OK;
  if (!d_perm || !d_run || !d_values || !d_out) return fail(EMG_EINVAL, "null pointer");
  const int g = persistent_ctas(8);
  cudaStream_t s = S(stream);
  const int64_t n = m->nnz, S_ = m->S;
  if (is_complex) {
    auto v = static_cast<const double2 *>(d_values);
    auto o = static_cast<double2 *>(d_out);
    if (block_dofs)
      k_coo_gather_c16<10><<<g, 256, 0, s>>>(d_perm, d_run, n, S_, v, o);
    else
      k_coo_gather_c16<0><<<g, 256, 0, s>>>(d_perm, d_run, n, S_, v, o);
  } else {
    auto v = static_cast<const double *>(d_values);
    auto o = static_cast<double *>(d_out);
    if (block_dofs)
      k_coo_gather_f8<10><<<g, 256, 0, s>>>(d_perm, d_run, n, S_, v, o);
    else
      k_coo_gather_f8<0><<<g, 256, 0, s>>>(d_perm, d_run, n, S_, v, o);
  }
  return launch_check("k_coo_gather");
}

}  // extern "C"
