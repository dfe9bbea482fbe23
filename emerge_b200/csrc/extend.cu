// extend.cu -- growing a CSC pattern by a few extra entries: the pattern of
// K + generate_csc(B2, empty_tri_rowcol(other_side=True)) for a field whose
// DoFs are split across a ThinConductor surface (assembler.py:636-639,
// femdata.py:86-104 and :110-124; the split DoFs of nedelec2.py:114-172).
//
// The reference adds two scipy matrices; their sum's pattern is the union of
// both. Here the union is laid out once (emg_csc_lookup finds which entries
// are new and where they go) and every assembly moves A's values to their
// union positions in one pass (emg_csc_shift), the new entries zeroed, before
// the other-side term is added with emg_robin_apply.
#include "common.cuh"

namespace emg {
namespace {

// position of (row, col) in the pattern, else -(1 + insertion point)
__global__ void k_csc_lookup(const int32_t *indptr, const int32_t *indices, int64_t N, const int64_t *cols,
                             const int64_t *rows, int64_t n, int64_t *out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t c = cols[i], r = rows[i];
  if (c < 0 || c >= N || r < 0 || r >= N) {
    out[i] = INT64_MIN;
    return;
  }
  int64_t lo = indptr[c], hi = indptr[c + 1];  // first index with indices[.] >= r
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (indices[mid] < r) lo = mid + 1;
    else hi = mid;
  }
  const bool found = lo < indptr[c + 1] && indices[lo] == r;
  out[i] = found ? lo : -(1 + lo);
}

constexpr int kShiftThreads = 256;
constexpr int kShiftPer = 8;  // elements per thread in a copy tile
constexpr int64_t kShiftTile = (int64_t)kShiftThreads * kShiftPer;

// last segment whose start is <= p (seg_start[0] == 0, ascending)
__device__ __forceinline__ int seg_of(const int64_t *seg_start, int lo, int hi, int64_t p) {
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (seg_start[mid] <= p) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// dst[p + shift(p)] = src[p] for p < n_src, the shift constant over each
// segment; then dst[xpos[e]] = xval[e] (or zero). Copy tiles first, one
// binary search per tile unless a segment boundary falls inside it.
template <typename T>
__global__ void __launch_bounds__(kShiftThreads)
    k_csc_shift(const T *src, int64_t n_src, const int64_t *seg_start, const int64_t *seg_shift, int n_seg,
                const int64_t *xpos, const T *xval, int64_t n_x, T *dst, int64_t n_dst, int64_t n_copy_blocks) {
  const int64_t b = blockIdx.x;
  if (b < n_copy_blocks) {
    const int64_t t0 = b * kShiftTile, t1 = min(t0 + kShiftTile, n_src);
    __shared__ int s_lo, s_hi;
    if (threadIdx.x == 0) {
      s_lo = seg_of(seg_start, 0, n_seg - 1, t0);
      s_hi = seg_of(seg_start, s_lo, n_seg - 1, t1 - 1);
    }
    __syncthreads();
    const int lo = s_lo, hi = s_hi;
    for (int64_t p = t0 + threadIdx.x; p < t1; p += kShiftThreads) {
      const int s = lo == hi ? lo : seg_of(seg_start, lo, hi, p);
      const int64_t q = p + seg_shift[s];
      if (q >= 0 && q < n_dst) dst[q] = src[p];
    }
    return;
  }
  const int64_t e = (b - n_copy_blocks) * kShiftThreads + threadIdx.x;
  if (e >= n_x) return;
  const int64_t q = xpos[e];
  if (q >= 0 && q < n_dst) dst[q] = xval ? xval[e] : T{};
}

template <typename T>
int launch_shift(const void *src, int64_t n_src, const int64_t *seg_start, const int64_t *seg_shift, int n_seg,
                 const int64_t *xpos, const void *xval, int64_t n_x, void *dst, int64_t n_dst, cudaStream_t s) {
  const int64_t nb_copy = (n_src + kShiftTile - 1) / kShiftTile;
  const int64_t nb_x = (n_x + kShiftThreads - 1) / kShiftThreads;
  const int64_t nb = nb_copy + nb_x;
  if (nb == 0) return EMG_OK;
  if (nb >= (1LL << 31)) return fail(EMG_ERANGE, "pattern too large for one shift launch");
  k_csc_shift<T><<<(unsigned)nb, kShiftThreads, 0, s>>>(static_cast<const T *>(src), n_src, seg_start, seg_shift,
                                                        n_seg, xpos, static_cast<const T *>(xval), n_x,
                                                        static_cast<T *>(dst), n_dst, nb_copy);
  return launch_check("k_csc_shift");
}

}  // namespace
}  // namespace emg

using namespace emg;

extern "C" {

int emg_csc_lookup(const int32_t *d_indptr, const int32_t *d_indices, int64_t N, const int64_t *d_cols,
                   const int64_t *d_rows, int64_t n, int64_t *d_out, emg_stream_t stream) {
  if (n < 0 || N < 0) return fail(EMG_EINVAL, "negative size");
  if (n == 0) return EMG_OK;
  if (!d_indptr || !d_indices || !d_cols || !d_rows || !d_out) return fail(EMG_EINVAL, "null pointer");
  k_csc_lookup<<<grid_for(n, 256), 256, 0, S(stream)>>>(d_indptr, d_indices, N, d_cols, d_rows, n, d_out);
  return launch_check("k_csc_lookup");
}

int emg_csc_shift(const void *d_src, int64_t n_src, int elem_bytes, const int64_t *d_seg_start,
                  const int64_t *d_seg_shift, int n_seg, const int64_t *d_xpos, const void *d_xval, int64_t n_x,
                  void *d_dst, int64_t n_dst, emg_stream_t stream) {
  if (n_src < 0 || n_x < 0 || n_dst < 0) return fail(EMG_EINVAL, "negative size");
  if (n_src > 0 && (n_seg < 1 || !d_seg_start || !d_seg_shift || !d_src))
    return fail(EMG_EINVAL, "a copy needs its segment table");
  if (n_x > 0 && !d_xpos) return fail(EMG_EINVAL, "null extra positions");
  if ((n_src > 0 || n_x > 0) && !d_dst) return fail(EMG_EINVAL, "null destination");
  cudaStream_t s = S(stream);
  if (elem_bytes == 16)
    return launch_shift<double2>(d_src, n_src, d_seg_start, d_seg_shift, n_seg, d_xpos, d_xval, n_x, d_dst, n_dst, s);
  if (elem_bytes == 8)
    return launch_shift<float2>(d_src, n_src, d_seg_start, d_seg_shift, n_seg, d_xpos, d_xval, n_x, d_dst, n_dst, s);
  if (elem_bytes == 4)
    return launch_shift<int32_t>(d_src, n_src, d_seg_start, d_seg_shift, n_seg, d_xpos, d_xval, n_x, d_dst, n_dst, s);
  return fail(EMG_EINVAL, "elem_bytes must be 4, 8 or 16");
}

}  // extern "C"
