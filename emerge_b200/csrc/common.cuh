// common.cuh -- shared definitions of the emgpu translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <utility>

#include "../../include/emgpu.h"

namespace emg {

// error message of the last failing C-ABI call in this thread (api.cu)
int fail(int code, const char *fmt, ...);

#define CUDA_TRY(expr)                                                                           \
  do {                                                                                           \
    cudaError_t _e = (expr);                                                                     \
    if (_e != cudaSuccess) return ::emg::fail(EMG_ECUDA, "%s: %s", #expr, cudaGetErrorString(_e)); \
  } while (0)

inline int launch_check(const char *what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(EMG_ECUDA, "launch of %s failed: %s", what, cudaGetErrorString(e));
  return EMG_OK;
}

inline cudaStream_t S(emg_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

inline int grid_for(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  return (int)(g < 1 ? 1 : g);
}

// canonical edge index of rank pair r1 != r2 in (0,1),(0,2),(0,3),(1,2),(1,3),(2,3)
__host__ __device__ __forceinline__ int canon_edge(int a, int b) {
  int r1 = a < b ? a : b, r2 = a < b ? b : a;
  return r1 == 0 ? r2 - 1 : (r1 == 1 ? r2 + 1 : 5);
}

// Canonical DoF (0..19) of reference DoF slot r of a tet whose vertex ranks
// are packed 2 bits per local vertex: edge slots use local vertex pairs
// (0,1),(0,2),(0,3),(1,2),(3,1),(2,3) and face slots miss vertex 3,1,2,0
// (mesh3d.py:760-761); canonical edges are rank pairs, canonical faces are
// numbered 3 - (rank of the missing vertex).
__host__ __device__ __forceinline__ int canon_dof(int ranks, int r) {
  if (r < 12) {
    const int e = r < 6 ? r : r - 6;
    const int u = e < 3 ? 0 : (e == 3 ? 1 : (e == 4 ? 3 : 2));
    const int v = e < 3 ? e + 1 : (e == 3 ? 2 : (e == 4 ? 1 : 3));
    return (r < 6 ? 0 : 6) + canon_edge((ranks >> (2 * u)) & 3, (ranks >> (2 * v)) & 3);
  }
  const int f = r < 16 ? r - 12 : r - 16;
  const int miss = f == 0 ? 3 : (f == 1 ? 1 : (f == 2 ? 2 : 0));
  return (r < 16 ? 12 : 16) + 3 - ((ranks >> (2 * miss)) & 3);
}

// index of canonical pair (x, y), x <= y, in the packed upper triangle
__host__ __device__ __forceinline__ int packed_index(int x, int y) { return x * (41 - x) / 2 + (y - x); }

// Entity-pair block layout (EMG_LAYOUT_BLOCK): block (i, j), i <= j, of the
// tet's canonical entities (0-5 edges, 6-9 faces) at 4 * block_index(i, j)
// holds [(i1,j1), (i1,j2), (i2,j1), (i2,j2)] of the entities' first and second
// canonical DoFs; 55 blocks, 220 values per tet.
constexpr int kBlockValues = 220;
__host__ __device__ __forceinline__ constexpr int block_index(int i, int j) { return i * (21 - i) / 2 + (j - i); }
__host__ __device__ __forceinline__ constexpr int ent_dof1(int i) { return i < 6 ? i : 12 + (i - 6); }
__host__ __device__ __forceinline__ constexpr int ent_dof2(int i) { return i < 6 ? i + 6 : 16 + (i - 6); }
// Block gather record: ia * 55 + block_index(min(a, b), max(a, b)) of row
// entity a and column entity b, bit 31 set when a > b (the block is stored
// transposed: its middle two values swap).
__host__ __device__ __forceinline__ bool block_record_fits(int64_t n_assy) { return n_assy * 55 < (1LL << 31); }

// Compact gather record (emg_plan.record_bytes = 4; one uint32 per
// contribution instead of an int2 of both value indices): the packed index of
// the contribution's first-column value, ia * 210 + p0, with bit 31 set when
// the row DoF sorts first in p0's (min, max) pair. The owner entity's second
// column DoF is its first plus 6 (edges) or 4 (faces), so p0 and that bit
// determine the second value's slot p1 = kSecondSlot[bit][p0].
struct SecondSlotTable {
  uint8_t v[2][210];
};
constexpr SecondSlotTable make_second_slot_table() {
  SecondSlotTable t{};
  int lo_of[210] = {}, hi_of[210] = {};
  for (int x = 0; x < 20; ++x)
    for (int y = x; y < 20; ++y) {
      lo_of[x * (41 - x) / 2 + (y - x)] = x;
      hi_of[x * (41 - x) / 2 + (y - x)] = y;
    }
  for (int f = 0; f < 2; ++f)
    for (int p = 0; p < 210; ++p) {
      const int b0 = f ? hi_of[p] : lo_of[p], row = f ? lo_of[p] : hi_of[p];
      const bool first = b0 < 6 || (b0 >= 12 && b0 < 16);
      const int b1 = b0 < 6 ? b0 + 6 : b0 + 4;
      const int x = row < b1 ? row : b1, y = row < b1 ? b1 : row;
      t.v[f][p] = first ? (uint8_t)(x * (41 - x) / 2 + (y - x)) : (uint8_t)0;
    }
  return t;
}
__host__ __device__ __forceinline__ bool pidx_compact_fits(int64_t n_assy) { return n_assy * 210 < (1LL << 31); }

// status word: [0] flags (EMG_ST_*), [1] smallest offending index
__device__ __forceinline__ void flag(int64_t *st, int64_t bit, int64_t index) {
  if (st) {
    atomicOr(reinterpret_cast<unsigned long long *>(st), (unsigned long long)bit);
    atomicMin(reinterpret_cast<long long *>(st + 1), (long long)index);
  }
}

// Item record, 16 bytes: assembled tet index, entity slot (0-5 edge, 6-9 face)
// of the owning entity in that tet, and for each of the tet's 10 entity slots
// its index in the owner's sorted adjacent-edge (slots 0-5) or adjacent-face
// (slots 6-9) list.
struct __align__(16) Item {
  int32_t ia;
  uint8_t slot;
  uint8_t pos[10];
  uint8_t ranks;  // vertex ranks of the tet by global node id: 2 bits per local vertex
};
static_assert(sizeof(Item) == 16, "item record must be 16 bytes");

struct ElemArgs {
  const double *nodes;
  int64_t nN;
  const int32_t *tets;
  int64_t nT;
  const int32_t *tetids;
  int64_t nA;
  const void *er;
  const void *ur;
  double ar, ai, br, bi;
  void *out;
  int64_t *st;
};

// one job of a batched packed gather (emg_gather_batch)
struct GatherJob {
  const int32_t *ent_ptr, *order;
  const void *pidx;       // packed: int2 records; block: uint32 block records
  const uint16_t *posoff; // packed: list start per position; block: per row pair
  const int32_t *indptr;
  const uint32_t *ent_cnt;  // block layout: adjacent edges | faces << 16 per entity
  const void *values;
  double2 *A;
  int64_t E, F, n_values, n_ctas;  // n_values: value slots (packed) or blocks (block layout)
};

// Gather chunks: a warp owns CHUNK consecutive entities of one kind. Their
// items are contiguous in the plan and their first-DoF (second-DoF) columns
// are consecutive, so each chunk's output is two contiguous runs of A.
constexpr int CHUNK = 8;
constexpr int CHUNK_MAX_POS = 1024;   // positions per run of a chunk (plan capacity)
constexpr int CHUNK_MAX_ITEMS = 1023; // items per chunk (10-bit item index)

__host__ __device__ __forceinline__ int64_t n_edge_chunks(int64_t E) { return (E + CHUNK - 1) / CHUNK; }
__host__ __device__ __forceinline__ int64_t n_chunks(int64_t E, int64_t F) {
  return n_edge_chunks(E) + (F + CHUNK - 1) / CHUNK;
}

// Default processing order g -> chunk. Edge chunks and face chunks are each
// sorted by their entities' lowest node; interleaving them in proportion keeps
// the edge and face chunks of one mesh region together.
__host__ __device__ __forceinline__ int64_t chunk_at(int64_t g, int64_t nec, int64_t nch) {
  const int64_t ce0 = (g * nec) / nch, ce1 = ((g + 1) * nec) / nch;
  return ce1 > ce0 ? ce0 : nec + (g - ce0);
}

// CTAs of a persistent grid: per_sm per SM of the current device
inline int persistent_ctas(int per_sm) {
  static int sms[64] = {0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148 * per_sm;
  if (!sms[dev] && cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms[dev] = 0;
  return (sms[dev] > 0 ? sms[dev] : 148) * per_sm;
}

// element kernel launchers, one translation unit per (form, material kind);
// form 0 = reference-faithful FP64, 1 = mixed, 2 = exact closed form
#define EMG_DECLARE_ELEM(F, K) int launch_element_##F##_##K(const ElemArgs &a, int layout, cudaStream_t s);
EMG_DECLARE_ELEM(0, 0)
EMG_DECLARE_ELEM(0, 1)
EMG_DECLARE_ELEM(0, 2)
EMG_DECLARE_ELEM(1, 0)
EMG_DECLARE_ELEM(1, 1)
EMG_DECLARE_ELEM(1, 2)
EMG_DECLARE_ELEM(2, 0)
EMG_DECLARE_ELEM(2, 1)
EMG_DECLARE_ELEM(2, 2)

#define EMG_DECLARE_ELEM_BATCH(F, K)                                                                      \
  int launch_element_batch_##F##_##K(const ElemArgs *d_jobs, const int64_t *d_cta_start, int n_jobs, \
                                     int64_t total_ctas, int layout, cudaStream_t s);
EMG_DECLARE_ELEM_BATCH(0, 0)
EMG_DECLARE_ELEM_BATCH(0, 1)
EMG_DECLARE_ELEM_BATCH(0, 2)
EMG_DECLARE_ELEM_BATCH(1, 0)
EMG_DECLARE_ELEM_BATCH(1, 1)
EMG_DECLARE_ELEM_BATCH(1, 2)
EMG_DECLARE_ELEM_BATCH(2, 0)
EMG_DECLARE_ELEM_BATCH(2, 1)
EMG_DECLARE_ELEM_BATCH(2, 2)

// element values are complex64 for the mixed form, complex128 otherwise
inline bool values_fp32(int precision) { return precision == EMG_MIXED; }

// plan.cu
size_t plan_workspace_bytes(const emg_plan *p);
size_t plan_layout(emg_plan *p);
int plan_build(emg_plan *p, const int32_t *tets, const int32_t *t2e, const int32_t *t2t, const int32_t *tetids,
               void *d_plan, void *d_ws, int32_t *indptr, int64_t *st, cudaStream_t s);
int plan_finish(const emg_plan *p, const int32_t *t2e, const int32_t *t2t, const int32_t *tetids, void *d_plan,
                const int32_t *indptr, int32_t *indices, int64_t *st, cudaStream_t s);
int plan_order(const emg_plan *p, void *d_plan, const double *nodes, int64_t nN, const int32_t *tets,
               const int32_t *tetids, void *d_ws, cudaStream_t s);
// exclusive prefix sum of n int32 counts into out[0..n] (out[n] = total; in
// and out may alias); bsum: scan_i32_bsum_bytes(n) of scratch
int scan_i32(const int32_t *in, int64_t n, int32_t *out, long long *bsum, int64_t *st, cudaStream_t s);
size_t scan_i32_bsum_bytes(int64_t n);

// ascending bitonic sort of n2 (a power of two) 64-bit keys in place
int sort_u64(uint64_t *keys, int64_t n2, cudaStream_t s);
inline int64_t pow2_at_least(int64_t n) {
  int64_t v = 1;
  while (v < n) v <<= 1;
  return v;
}
int status_reset(int64_t *st, cudaStream_t s);

// gather.cu
int launch_gather(const emg_plan *p, const void *d_plan, const int32_t *indptr, const void *v1, const void *v2,
                  int precision, int layout, double ar, double ai, double br, double bi, void *A, int64_t *st,
                  cudaStream_t s);
int gather_job_fill(const emg_plan *p, const void *d_plan, const int32_t *d_indptr, const void *d_values, void *d_A,
                    GatherJob *out);
int launch_gather_batch(const GatherJob *d_jobs, const int64_t *d_cta_start, int n_jobs, int64_t total_ctas,
                        int precision, int layout, cudaStream_t s);
int launch_form_sweep(const void *K, const void *M, const void *P, int64_t nnz, const double *coef, int nf,
                      void *out, int64_t stride, cudaStream_t s);
int launch_form_batch(const emg_form_item *items, const int64_t *tile_start, const int32_t *n_items, int max_items,
                      cudaStream_t s);

}  // namespace emg
