// select.cu -- the solve-DoF submatrix of A on the device.
//
// Replaces the host-side slicing the reference does before every solve,
// Asel = A[:, solve_ids][solve_ids, :] (solver.py:2071; solve_ids = all DoFs
// minus the PEC DoFs, assembler.py:543-564,742), so that a GPU solver gets the
// reduced system without A crossing to the host. The pattern part (which
// positions of A survive, their new row numbers) is built once; per frequency
// only the values are gathered.
#include "common.cuh"

namespace emg {
namespace {

__global__ void k_keep_flags(const uint8_t *keep, int64_t N, int32_t *flags) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) flags[i] = keep[i] ? 1 : 0;
}

// kept column j: number of its rows that are kept (removed columns: 0)
__global__ void k_sel_count(const int32_t *indptr, const int32_t *indices, const uint8_t *keep, int64_t N,
                            int32_t *cnt, int64_t *st) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  int32_t c = 0;
  if (keep[j]) {
    for (int32_t p = indptr[j]; p < indptr[j + 1]; ++p) {
      const int32_t r = indices[p];
      if (r < 0 || r >= N) {
        flag(st, EMG_ST_INDEX, p);
        continue;
      }
      c += keep[r] ? 1 : 0;
    }
  }
  cnt[j] = c;
}

// compact the per-column counts of kept columns into the new column order
__global__ void k_sel_compact(const int32_t *cnt, const uint8_t *keep, const int32_t *newid, int64_t N,
                              int32_t *cnt_sel) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j < N && keep[j]) cnt_sel[newid[j]] = cnt[j];
}

// rows of kept column j, renumbered, in A's (ascending) order; take[q] = the
// position in A of selected entry q
__global__ void k_sel_fill(const int32_t *indptr, const int32_t *indices, const uint8_t *keep, const int32_t *newid,
                           int64_t N, const int32_t *indptr_sel, int32_t *indices_sel, int32_t *take) {
  const int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N || !keep[j]) return;
  int32_t q = indptr_sel[newid[j]];
  for (int32_t p = indptr[j]; p < indptr[j + 1]; ++p) {
    const int32_t r = indices[p];
    if (r < 0 || r >= N || !keep[r]) continue;
    indices_sel[q] = newid[r];
    take[q] = p;
    ++q;
  }
}

__global__ void k_take_c128(const double2 *A, const int32_t *take, int64_t n, int64_t nnz, double2 *out) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
    const int32_t p = take[q];
    out[q] = (p >= 0 && p < nnz) ? A[p] : make_double2(0.0, 0.0);
  }
}

struct SelWs {
  int32_t *newid, *cnt;
  long long *bsum;
};

SelWs sel_ws(void *d_ws, int64_t N) {
  char *w = static_cast<char *>(d_ws);
  SelWs r;
  size_t o = 0;
  r.newid = reinterpret_cast<int32_t *>(w + o);
  o = align_up(o + (size_t)(N + 1) * 4, 256);
  r.cnt = reinterpret_cast<int32_t *>(w + o);
  o = align_up(o + (size_t)(N + 1) * 4, 256);
  r.bsum = reinterpret_cast<long long *>(w + o);
  return r;
}

}  // namespace
}  // namespace emg

using namespace emg;

extern "C" {

int emg_select_init(int64_t N, emg_select *sel) {
  if (!sel) return fail(EMG_EINVAL, "null descriptor");
  if (N < 0 || N >= INT32_MAX) return fail(EMG_ERANGE, "N out of range");
  memset(sel, 0, sizeof(*sel));
  sel->N = N;
  sel->workspace_bytes = align_up((size_t)(N + 1) * 4, 256) * 2 + scan_i32_bsum_bytes(N + 1);
  return EMG_OK;
}

int emg_select_build(emg_select *sel, const int32_t *d_indptr, const int32_t *d_indices, const uint8_t *d_keep,
                     void *d_ws, int32_t *d_indptr_sel, int64_t *d_status, emg_stream_t stream) {
  if (!sel || !d_indptr || !d_indices || !d_keep || !d_ws || !d_indptr_sel || !d_status)
    return fail(EMG_EINVAL, "null pointer");
  const int64_t N = sel->N;
  cudaStream_t s = S(stream);
  SelWs w = sel_ws(d_ws, N);
  int rc;
  if ((rc = status_reset(d_status, s))) return rc;
  if (N > 0) {
    k_keep_flags<<<grid_for(N, 256), 256, 0, s>>>(d_keep, N, w.newid);
    if ((rc = launch_check("k_keep_flags"))) return rc;
  }
  if ((rc = scan_i32(w.newid, N, w.newid, w.bsum, d_status, s))) return rc;  // newid[i] = kept DoFs before i
  int32_t M = 0;
  CUDA_TRY(cudaMemcpyAsync(&M, w.newid + N, 4, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (N > 0) {
    k_sel_count<<<grid_for(N, 256), 256, 0, s>>>(d_indptr, d_indices, d_keep, N, w.cnt, d_status);
    if ((rc = launch_check("k_sel_count"))) return rc;
    k_sel_compact<<<grid_for(N, 256), 256, 0, s>>>(w.cnt, d_keep, w.newid, N, d_indptr_sel);
    if ((rc = launch_check("k_sel_compact"))) return rc;
  }
  if ((rc = scan_i32(d_indptr_sel, M, d_indptr_sel, w.bsum, d_status, s))) return rc;
  int32_t nnz = 0;
  int64_t h_st[2] = {0, 0};
  CUDA_TRY(cudaMemcpyAsync(&nnz, d_indptr_sel + M, 4, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(h_st, d_status, 16, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (h_st[0]) return fail(EMG_EMESH, "submatrix build: status flags 0x%llx", (long long)h_st[0]);
  sel->M = M;
  sel->nnz_sel = nnz;
  return EMG_OK;
}

int emg_select_finish(const emg_select *sel, const int32_t *d_indptr, const int32_t *d_indices, const uint8_t *d_keep,
                      void *d_ws, const int32_t *d_indptr_sel, int32_t *d_indices_sel, int32_t *d_take,
                      emg_stream_t stream) {
  if (!sel || !d_indptr || !d_indices || !d_keep || !d_ws || !d_indptr_sel) return fail(EMG_EINVAL, "null pointer");
  if (sel->nnz_sel > 0 && (!d_indices_sel || !d_take)) return fail(EMG_EINVAL, "null pointer");
  if (sel->N == 0) return EMG_OK;
  SelWs w = sel_ws(d_ws, sel->N);
  k_sel_fill<<<grid_for(sel->N, 256), 256, 0, S(stream)>>>(d_indptr, d_indices, d_keep, w.newid, sel->N,
                                                             d_indptr_sel, d_indices_sel, d_take);
  return launch_check("k_sel_fill");
}

int emg_select_values(const emg_select *sel, const int32_t *d_take, const void *d_A, int64_t nnz, void *d_A_sel,
                      emg_stream_t stream) {
  if (!sel) return fail(EMG_EINVAL, "null descriptor");
  if (sel->nnz_sel == 0) return EMG_OK;
  if (!d_take || !d_A || !d_A_sel) return fail(EMG_EINVAL, "null pointer");
  k_take_c128<<<persistent_ctas(8), 256, 0, S(stream)>>>(static_cast<const double2 *>(d_A), d_take, sel->nnz_sel, nnz,
                                                           static_cast<double2 *>(d_A_sel));
  return launch_check("k_take_c128");
}

}  // extern "C"
