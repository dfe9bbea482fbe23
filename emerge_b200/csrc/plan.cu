// plan.cu -- sparsity pattern and column-gather plan of the Nedelec-2 system.
//
// Replaces CSCMapping.from_rowcol / precompute_csc_pattern (mth/csc_cast.py:51-160)
// for the structured Nedelec-2 pattern: the rows of the columns of entity x
// (edge or face) are the DoFs of every entity that shares an assembled tet
// with x, in four sorted blocks [edges | edges+E | faces+2E | faces+2E+F]
// (the DoF numbering of elements/nedelec2.py:65-79).
#include "common.cuh"

namespace emg {
namespace {

__global__ void k_status_reset(int64_t *st) {
  st[0] = 0;
  st[1] = INT64_MAX;
}

// ---------------------------------------------------------------------------
// exclusive scan int32 counts -> int32 offsets (n + 1 entries), int64 guard
// ---------------------------------------------------------------------------
constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_PER_THREAD = 4;
constexpr int SCAN_BLOCK = SCAN_THREADS * SCAN_PER_THREAD;

__device__ __forceinline__ long long block_exclusive_scan(long long v, long long *warp_sums, long long *total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  long long x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[w] = x;
  __syncthreads();
  if (w == 0) {
    long long s = (lane < (int)(blockDim.x >> 5)) ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      long long y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    warp_sums[lane] = s;  // inclusive
  }
  __syncthreads();
  long long base = (w > 0) ? warp_sums[w - 1] : 0;
  *total = warp_sums[(blockDim.x >> 5) - 1];
  __syncthreads();
  return base + x - v;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const int32_t *in, int64_t n, long long *bsum) {
  __shared__ long long ws[32];
  int64_t base = (int64_t)blockIdx.x * SCAN_BLOCK + (int64_t)threadIdx.x * SCAN_PER_THREAD;
  long long s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; ++k)
    if (base + k < n) s += in[base + k];
  long long tot;
  block_exclusive_scan(s, ws, &tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_bsums(long long *bsum, int64_t nb) {
  __shared__ long long ws[32];
  long long carry = 0;
  for (int64_t b0 = 0; b0 < nb; b0 += SCAN_THREADS) {
    int64_t i = b0 + threadIdx.x;
    long long v = (i < nb) ? bsum[i] : 0;
    long long tot;
    long long ex = block_exclusive_scan(v, ws, &tot);
    if (i < nb) bsum[i] = carry + ex;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) bsum[nb] = carry;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_apply(const int32_t *in, int64_t n, const long long *bsum,
                                                             int32_t *out, int64_t *st) {
  __shared__ long long ws[32];
  int64_t base = (int64_t)blockIdx.x * SCAN_BLOCK + (int64_t)threadIdx.x * SCAN_PER_THREAD;
  long long v[SCAN_PER_THREAD];
  long long s = 0;
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    s += v[k];
  }
  long long tot;
  long long ex = block_exclusive_scan(s, ws, &tot) + bsum[blockIdx.x];
#pragma unroll
  for (int k = 0; k < SCAN_PER_THREAD; ++k) {
    if (base + k < n) {
      if (ex > INT32_MAX) flag(st, EMG_ST_CAPACITY, base + k);
      out[base + k] = (int32_t)ex;
    }
    ex += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
    long long total = bsum[gridDim.x];
    if (total > INT32_MAX) flag(st, EMG_ST_CAPACITY, n);
    out[n] = (int32_t)total;
  }
}

// in and out may alias (in-place scan of counts stored in out[0..n))
int exclusive_scan(const int32_t *in, int64_t n, int32_t *out, long long *bsum, int64_t *st, cudaStream_t s) {
  int64_t nb = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
  if (nb == 0) nb = 1;
  k_scan_reduce<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, bsum);
  k_scan_bsums<<<1, SCAN_THREADS, 0, s>>>(bsum, nb);
  k_scan_apply<<<(unsigned)nb, SCAN_THREADS, 0, s>>>(in, n, bsum, out, st);
  return launch_check("exclusive_scan");
}

size_t scan_bsum_bytes(int64_t n) { return (size_t)((n + SCAN_BLOCK - 1) / SCAN_BLOCK + 2) * sizeof(long long); }

// ---------------------------------------------------------------------------
// plan: entity -> incident (tet, slot) items and column positions
// ---------------------------------------------------------------------------
constexpr int MAX_ADJ = 255;  // adjacent edges (faces) per entity: uint8 positions

__device__ __forceinline__ int64_t tet_of(const int32_t *tetids, int64_t ia) { return tetids ? tetids[ia] : ia; }


__global__ void k_count_incidence(const int32_t *t2e, const int32_t *t2t, const int32_t *tetids, int64_t nT,
                                  int64_t nA, int64_t E, int64_t F, int32_t *cnt, int64_t *st) {
  int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nA * 10) return;
  int64_t ia = g / 10;
  int s = (int)(g % 10);
  int64_t it = tet_of(tetids, ia);
  if (it < 0 || it >= nT) {
    flag(st, EMG_ST_INDEX, ia);
    return;
  }
  int64_t raw = s < 6 ? (int64_t)t2e[(int64_t)s * nT + it] : (int64_t)t2t[(int64_t)(s - 6) * nT + it];
  if (raw < 0 || raw >= (s < 6 ? E : F)) {
    flag(st, EMG_ST_INDEX, ia);
    return;
  }
  atomicAdd(&cnt[s < 6 ? raw : E + raw], 1);
}

__global__ void k_fill_items(const int32_t *tets, const int32_t *t2e, const int32_t *t2t, const int32_t *tetids,
                             int64_t nT, int64_t nA, int64_t E, int64_t F, const int32_t *ent_ptr, int32_t *cursor,
                             Item *items) {
  int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= nA * 10) return;
  int64_t ia = g / 10;
  int s = (int)(g % 10);
  int64_t it = tet_of(tetids, ia);
  if (it < 0 || it >= nT) return;
  int64_t raw = s < 6 ? (int64_t)t2e[(int64_t)s * nT + it] : (int64_t)t2t[(int64_t)(s - 6) * nT + it];
  if (raw < 0 || raw >= (s < 6 ? E : F)) return;
  int64_t x = s < 6 ? raw : E + raw;
  int32_t p = ent_ptr[x] + atomicAdd(&cursor[x], 1);
  Item rec;
  rec.ia = (int32_t)ia;
  rec.slot = (uint8_t)s;
#pragma unroll
  for (int k = 0; k < 10; ++k) rec.pos[k] = 0;
  // vertex ranks by global id (a repeated vertex is caught by the element kernel)
  int32_t v[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) v[q] = tets[(int64_t)q * nT + it];
  uint32_t ranks = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int r = 0;
#pragma unroll
    for (int o = 0; o < 4; ++o) r += (v[o] < v[q] || (v[o] == v[q] && o < q)) ? 1 : 0;
    ranks |= (uint32_t)r << (2 * q);
  }
  rec.ranks = (uint8_t)ranks;
  items[p] = rec;
}

// insertion sort of each entity's items by assembled tet index (deterministic order)
__global__ void k_sort_items(const int32_t *ent_ptr, int64_t n_ent, Item *items) {
  int64_t x = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= n_ent) return;
  int32_t b = ent_ptr[x], e = ent_ptr[x + 1];
  for (int32_t i = b + 1; i < e; ++i) {
    Item v = items[i];
    int32_t j = i - 1;
    while (j >= b && items[j].ia > v.ia) {
      items[j + 1] = items[j];
      --j;
    }
    items[j + 1] = v;
  }
}

// Warp per entity. Candidates = the 6 edges / 4 faces of every incident tet;
// unique values counted (count pass) or ranked (fill pass) by comparison in
// shared memory.
constexpr int ROWS_WARPS = 4;
constexpr int CAND_CAP = 640;   // edge candidates per entity (6 per tet) => up to 106 incident tets
constexpr int CAND_CAP_F = 432; // face candidates (4 per tet)

template <bool FILL>
__global__ void __launch_bounds__(ROWS_WARPS * 32)
    k_entity_rows(const int32_t *t2e, const int32_t *t2t, const int32_t *tetids, int64_t nT, int64_t E, int64_t F,
                  const int32_t *ent_ptr, Item *items, int64_t n_ent, int32_t *col_len, uint32_t *ent_cnt,
                  const int32_t *indptr, int32_t *indices, int64_t *st) {
  __shared__ int32_t cand_e[ROWS_WARPS][CAND_CAP];
  __shared__ int32_t cand_f[ROWS_WARPS][CAND_CAP_F];
  __shared__ uint8_t first_e[ROWS_WARPS][CAND_CAP];
  __shared__ uint8_t first_f[ROWS_WARPS][CAND_CAP_F];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int64_t x = (int64_t)blockIdx.x * ROWS_WARPS + w;
  if (x >= n_ent) return;
  int32_t b = ent_ptr[x], e = ent_ptr[x + 1];
  int nitem = e - b;
  int ne = nitem * 6, nf = nitem * 4;
  if (ne > CAND_CAP || nf > CAND_CAP_F) {
    if (lane == 0) flag(st, EMG_ST_CAPACITY, x);
    return;
  }
  int32_t *ce = cand_e[w], *cf = cand_f[w];
  uint8_t *fe = first_e[w], *ff = first_f[w];
  for (int i = lane; i < ne; i += 32) {
    int64_t it = tet_of(tetids, items[b + i / 6].ia);
    ce[i] = t2e[(int64_t)(i % 6) * nT + it];
  }
  for (int i = lane; i < nf; i += 32) {
    int64_t it = tet_of(tetids, items[b + i / 4].ia);
    cf[i] = t2t[(int64_t)(i % 4) * nT + it];
  }
  __syncwarp();
  // first occurrences -> number of distinct adjacent edges / faces
  int ue = 0, uf = 0;
  for (int i = lane; i < ne; i += 32) {
    int32_t v = ce[i];
    bool first = true;
    for (int j = 0; j < i; ++j) first &= (ce[j] != v);
    fe[i] = first;
    ue += first;
  }
  for (int i = lane; i < nf; i += 32) {
    int32_t v = cf[i];
    bool first = true;
    for (int j = 0; j < i; ++j) first &= (cf[j] != v);
    ff[i] = first;
    uf += first;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ue += __shfl_xor_sync(0xffffffffu, ue, o);
    uf += __shfl_xor_sync(0xffffffffu, uf, o);
  }
  if (ue > MAX_ADJ || uf > MAX_ADJ) {
    if (lane == 0) flag(st, EMG_ST_CAPACITY, x);
    return;
  }
  const bool is_edge = x < E;
  const int64_t c0 = is_edge ? x : E + x;          // 2E + (x - E)
  const int64_t c1 = is_edge ? x + E : E + F + x;  // 2E + F + (x - E)
  if (!FILL) {
    if (lane == 0) {
      int32_t L = 2 * (ue + uf);
      col_len[c0] = L;
      col_len[c1] = L;
      ent_cnt[x] = (uint32_t)ue | ((uint32_t)uf << 16);
    }
    return;
  }
  __syncwarp();
  // rank = number of distinct smaller values; rows of the four column blocks
  const int64_t s0 = indptr[c0], s1 = indptr[c1];
  for (int i = lane; i < ne; i += 32) {
    int32_t v = ce[i];
    int r = 0;
    for (int j = 0; j < ne; ++j) r += (fe[j] && ce[j] < v) ? 1 : 0;
    if (fe[i]) {
      indices[s0 + r] = v;
      indices[s0 + ue + r] = v + (int32_t)E;
      indices[s1 + r] = v;
      indices[s1 + ue + r] = v + (int32_t)E;
    }
    items[b + i / 6].pos[i % 6] = (uint8_t)r;
  }
  for (int i = lane; i < nf; i += 32) {
    int32_t v = cf[i];
    int r = 0;
    for (int j = 0; j < nf; ++j) r += (ff[j] && cf[j] < v) ? 1 : 0;
    if (ff[i]) {
      int32_t r0 = v + 2 * (int32_t)E, r1 = v + 2 * (int32_t)E + (int32_t)F;
      indices[s0 + 2 * ue + r] = r0;
      indices[s0 + 2 * ue + uf + r] = r1;
      indices[s1 + 2 * ue + r] = r0;
      indices[s1 + 2 * ue + uf + r] = r1;
    }
    items[b + i / 4].pos[6 + i % 4] = (uint8_t)r;
  }
}

__global__ void k_max_col(const int32_t *col_len, int64_t n, int32_t *out) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int32_t m = 0;
  for (; i < n; i += (int64_t)gridDim.x * blockDim.x) m = max(m, col_len[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// Gather lists, warp per chunk: every (item, row) of the chunk contributes to
// one position of the chunk's first-DoF run (and the same position of its
// second-DoF run). Count per position, scan, then place the contributions in
// item order (items of an entity are sorted by tet), so each output sums its
// contributions in a fixed order.
constexpr int CC_WARPS = 8;

__global__ void __launch_bounds__(CC_WARPS * 32)
    k_chunk_contrib(const int32_t *ent_ptr, const Item *items, const uint32_t *ent_cnt, int64_t E, int64_t F,
                    const int32_t *indptr, uint16_t *contrib, uint16_t *posoff, void *pidx_v, bool compact,
                    int64_t *st) {
  __shared__ int32_t cnt_all[CC_WARPS][CHUNK_MAX_POS];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t chunk = (int64_t)blockIdx.x * CC_WARPS + w;
  const int64_t nec = n_edge_chunks(E);
  if (chunk >= n_chunks(E, F)) return;
  const bool edges = chunk < nec;
  const int64_t x0 = edges ? chunk * CHUNK : E + (chunk - nec) * CHUNK;
  const int nx = (int)min((int64_t)CHUNK, (edges ? E : E + F) - x0);
  const int64_t cb0 = edges ? x0 : E + x0;
  const int32_t my_ptr = lane <= nx ? ent_ptr[x0 + lane] : 0;
  const int32_t my_c0 = lane <= nx ? indptr[cb0 + lane] : 0;
  const uint32_t my_cnt = lane < nx ? ent_cnt[x0 + lane] : 0u;
  const int32_t I0 = __shfl_sync(0xffffffffu, my_ptr, 0), I1 = __shfl_sync(0xffffffffu, my_ptr, nx);
  const int32_t A0 = __shfl_sync(0xffffffffu, my_c0, 0), A0e = __shfl_sync(0xffffffffu, my_c0, nx);
  const int Lsum = A0e - A0;
  if (Lsum > CHUNK_MAX_POS || I1 - I0 > CHUNK_MAX_ITEMS) {
    if (lane == 0) flag(st, EMG_ST_CAPACITY, x0);
    return;
  }
  const int64_t hbase = edges ? (int64_t)A0 : (int64_t)indptr[E] + (A0 - indptr[2 * E]);
  int32_t *cnt = cnt_all[w];
  for (int i = lane; i < Lsum; i += 32) cnt[i] = 0;
  const int r = lane;
  const int sl = r < 6 ? r : (r < 12 ? r - 6 : (r < 16 ? r - 6 : r - 10));
  const int blk = r < 6 ? 0 : (r < 12 ? 1 : (r < 16 ? 2 : 3));
  __syncwarp();
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1) {
      // exclusive scan of the counts into start offsets (lane-serial blocks of 32)
      int32_t carry = 0;
      for (int b0 = 0; b0 < Lsum; b0 += 32) {
        const int i = b0 + lane;
        const int32_t v = i < Lsum ? cnt[i] : 0;
        int32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
          if (lane >= o) x += y;
        }
        if (i < Lsum) {
          cnt[i] = carry + x - v;  // becomes the cursor
          posoff[hbase + i] = (uint16_t)(carry + x - v);
        }
        carry += __shfl_sync(0xffffffffu, x, 31);
      }
      __syncwarp();
    }
    for (int32_t k = I0; k < I1; ++k) {
      if (r < 20) {
        int e = 0;
        for (int q = 1; q < nx; ++q)
          if (k >= __shfl_sync(0x000fffffu, my_ptr, q)) e = q;
        const int32_t ce = __shfl_sync(0x000fffffu, my_c0, e);
        const uint32_t c = __shfl_sync(0x000fffffu, my_cnt, e);
        const int ne = (int)(c & 0xffffu), nf = (int)(c >> 16);
        const int off = blk == 0 ? 0 : (blk == 1 ? ne : (blk == 2 ? 2 * ne : 2 * ne + nf));
        const Item rec = items[k];
        const int p = (ce - A0) + off + rec.pos[sl];
        if (pass == 0) {
          cnt[p] += 1;  // distinct p across the 20 lanes of one item
        } else {
          const int32_t at = cnt[p]++;
          contrib[(int64_t)20 * I0 + at] = (uint16_t)(((k - I0) << 5) | r);
          const int s = rec.slot;
          const int a0 = s < 6 ? s : 12 + (s - 6), a1 = s < 6 ? s + 6 : 16 + (s - 6);
          const int al = canon_dof(rec.ranks, r);
          const int b0 = canon_dof(rec.ranks, a0), b1 = canon_dof(rec.ranks, a1);
          const int64_t base = (int64_t)rec.ia * 210;
          if (pidx_v && compact)
            static_cast<uint32_t *>(pidx_v)[(int64_t)20 * I0 + at] =
                (uint32_t)(base + packed_index(min(al, b0), max(al, b0))) | (al <= b0 ? 0x80000000u : 0u);
          else if (pidx_v)
            static_cast<int2 *>(pidx_v)[(int64_t)20 * I0 + at] =
                make_int2((int)(base + packed_index(min(al, b0), max(al, b0))),
                          (int)(base + packed_index(min(al, b1), max(al, b1))));
        }
      }
      __syncwarp();
    }
  }
}

// Block gather lists (EMG_LAYOUT_BLOCK), warp per chunk: every (item, row
// entity) of the chunk contributes the tet's block of that entity pair to one
// row pair (the row entity's first-DoF row and its partner row, which hold the
// same tets); counted per row pair, scanned into hoff (list start relative to
// the chunk's first record, 10 * I0), then placed in item order, so each
// output sums its contributions in the order of the packed lists.
__global__ void __launch_bounds__(CC_WARPS * 32)
    k_chunk_blocks(const int32_t *ent_ptr, const Item *items, const uint32_t *ent_cnt, int64_t E, int64_t F,
                   const int32_t *indptr, uint16_t *hoff, uint32_t *brec, int64_t *st) {
  __shared__ int32_t cnt_all[CC_WARPS][CHUNK_MAX_POS / 2];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t chunk = (int64_t)blockIdx.x * CC_WARPS + w;
  const int64_t nec = n_edge_chunks(E);
  if (chunk >= n_chunks(E, F)) return;
  const bool edges = chunk < nec;
  const int64_t x0 = edges ? chunk * CHUNK : E + (chunk - nec) * CHUNK;
  const int nx = (int)min((int64_t)CHUNK, (edges ? E : E + F) - x0);
  const int64_t cb0 = edges ? x0 : E + x0;
  const int32_t my_ptr = lane <= nx ? ent_ptr[x0 + lane] : 0;
  const int32_t my_c0 = lane <= nx ? indptr[cb0 + lane] : 0;
  const uint32_t my_cnt = lane < nx ? ent_cnt[x0 + lane] : 0u;
  const int32_t I0 = __shfl_sync(0xffffffffu, my_ptr, 0), I1 = __shfl_sync(0xffffffffu, my_ptr, nx);
  const int32_t A0 = __shfl_sync(0xffffffffu, my_c0, 0), A0e = __shfl_sync(0xffffffffu, my_c0, nx);
  const int Lsum = A0e - A0, Hsum = Lsum / 2;
  if (Lsum > CHUNK_MAX_POS || I1 - I0 > CHUNK_MAX_ITEMS) {
    if (lane == 0) flag(st, EMG_ST_CAPACITY, x0);
    return;
  }
  const int64_t hb = (edges ? (int64_t)A0 : (int64_t)indptr[E] + (A0 - indptr[2 * E])) / 2;
  int32_t *cnt = cnt_all[w];
  for (int i = lane; i < Hsum; i += 32) cnt[i] = 0;
  const int r = lane;  // row entity slot (0-5 edges, 6-9 faces) of the item's tet
  __syncwarp();
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1) {
      int32_t carry = 0;
      for (int b0 = 0; b0 < Hsum; b0 += 32) {
        const int i = b0 + lane;
        const int32_t v = i < Hsum ? cnt[i] : 0;
        int32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
          if (lane >= o) x += y;
        }
        if (i < Hsum) {
          cnt[i] = carry + x - v;
          hoff[hb + i] = (uint16_t)(carry + x - v);
        }
        carry += __shfl_sync(0xffffffffu, x, 31);
      }
      __syncwarp();
    }
    for (int32_t k = I0; k < I1; ++k) {
      if (r < 10) {
        int e = 0;
        for (int q = 1; q < nx; ++q)
          if (k >= __shfl_sync(0x3ffu, my_ptr, q)) e = q;
        const int32_t ce = __shfl_sync(0x3ffu, my_c0, e);
        const uint32_t c = __shfl_sync(0x3ffu, my_cnt, e);
        const int ne = (int)(c & 0xffffu);
        const Item rec = items[k];
        const int h = (ce - A0) / 2 + (r < 6 ? 0 : ne) + rec.pos[r];
        if (pass == 0) {
          cnt[h] += 1;  // distinct h across the 10 lanes of one item
        } else {
          const int32_t at = cnt[h]++;
          const int s = rec.slot;
          const int cb = s < 6 ? canon_dof(rec.ranks, s) : canon_dof(rec.ranks, 12 + (s - 6)) - 6;
          const int ca = r < 6 ? canon_dof(rec.ranks, r) : canon_dof(rec.ranks, 12 + (r - 6)) - 6;
          const int lo = ca < cb ? ca : cb, hi = ca < cb ? cb : ca;
          brec[(int64_t)10 * I0 + at] =
              (uint32_t)((int64_t)rec.ia * 55 + block_index(lo, hi)) | (ca > cb ? 0x80000000u : 0u);
        }
      }
      __syncwarp();
    }
  }
}

__global__ void k_default_order(int32_t *order, int64_t nec, int64_t nch) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < nch) order[g] = (int32_t)chunk_at(g, nec, nch);
}

// bounding box of the nodes (SoA [3][nN]): per-block partials, then one block
__global__ void __launch_bounds__(256) k_bbox_partial(const double *nodes, int64_t nN, double *part) {
  __shared__ double sm[6][256];
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nN; i += (int64_t)gridDim.x * blockDim.x)
    for (int d = 0; d < 3; ++d) {
      const double x = nodes[d * nN + i];
      lo[d] = fmin(lo[d], x);
      hi[d] = fmax(hi[d], x);
    }
  for (int d = 0; d < 3; ++d) {
    sm[d][threadIdx.x] = lo[d];
    sm[3 + d][threadIdx.x] = hi[d];
  }
  __syncthreads();
  for (int st = 128; st > 0; st >>= 1) {
    if ((int)threadIdx.x < st)
      for (int d = 0; d < 3; ++d) {
        sm[d][threadIdx.x] = fmin(sm[d][threadIdx.x], sm[d][threadIdx.x + st]);
        sm[3 + d][threadIdx.x] = fmax(sm[3 + d][threadIdx.x], sm[3 + d][threadIdx.x + st]);
      }
    __syncthreads();
  }
  if (threadIdx.x < 6) part[blockIdx.x * 6 + threadIdx.x] = sm[threadIdx.x][0];
}

__global__ void k_bbox_final(const double *part, int nblk, double *box) {
  if (threadIdx.x < 6) {
    double v = part[threadIdx.x];
    for (int b = 1; b < nblk; ++b) {
      const double x = part[b * 6 + threadIdx.x];
      v = threadIdx.x < 3 ? fmin(v, x) : fmax(v, x);
    }
    box[threadIdx.x] = v;
  }
}

__device__ __forceinline__ uint32_t spread_bits10(uint32_t x) {  // bit i -> bit 3i
  x &= 0x3ffu;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

// key of chunk c = Morton code of the centroid of its first incident tet in
// the high 32 bits, c in the low 32 bits; chunks without items and the
// padding up to the power of two sort last
__global__ void k_chunk_keys(const int32_t *ent_ptr, const Item *items, const double *nodes, int64_t nN,
                             const int32_t *tets, int64_t nT, const int32_t *tetids, int64_t nA, const double *box,
                             int64_t E, int64_t F, int64_t nch, int64_t n2, uint64_t *keys) {
  const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n2) return;
  uint64_t key = ~0ull;
  if (c < nch) {
    const int64_t nec = n_edge_chunks(E);
    const int64_t x0 = c < nec ? c * CHUNK : E + (c - nec) * CHUNK;
    const int64_t xe = min(x0 + CHUNK, c < nec ? E : E + F);
    const int32_t i0 = ent_ptr[x0], i1 = ent_ptr[xe];
    uint32_t code = 0xffffffffu;
    if (i1 > i0) {
      const int64_t ia = items[i0].ia;
      const int64_t t = (ia >= 0 && ia < nA) ? (tetids ? (int64_t)tetids[ia] : ia) : -1;
      if (t >= 0 && t < nT) {
        const double ext = fmax(fmax(box[3] - box[0], box[4] - box[1]), fmax(box[5] - box[2], 1e-300));
        uint32_t q[3];
        for (int d = 0; d < 3; ++d) {
          double x = 0.0;
          for (int k = 0; k < 4; ++k) {
            const int64_t v = tets[k * nT + t];
            x += (v >= 0 && v < nN) ? nodes[d * nN + v] : box[d];
          }
          const double u = (0.25 * x - box[d]) / ext * 1024.0;
          q[d] = (uint32_t)fmin(fmax(u, 0.0), 1023.0);
        }
        code = spread_bits10(q[0]) | (spread_bits10(q[1]) << 1) | (spread_bits10(q[2]) << 2);
      }
    }
    key = ((uint64_t)code << 32) | (uint64_t)c;
  }
  keys[c] = key;
}

// one compare-exchange step (k, j) of a bitonic sort of n2 = 2^m keys
__global__ void k_bitonic_step(uint64_t *keys, int64_t n2, int64_t j, int64_t k) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n2) return;
  const int64_t l = i ^ j;
  if (l > i) {
    const uint64_t a = keys[i], b = keys[l];
    const bool up = (i & k) == 0;
    if ((a > b) == up) {
      keys[i] = b;
      keys[l] = a;
    }
  }
}

__global__ void k_write_order(const uint64_t *keys, int64_t nch, int32_t *order) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g < nch) order[g] = (int32_t)(keys[g] & 0xffffffffu);
}

}  // namespace

int status_reset(int64_t *st, cudaStream_t s) {
  k_status_reset<<<1, 1, 0, s>>>(st);
  return launch_check("k_status_reset");
}

int scan_i32(const int32_t *in, int64_t n, int32_t *out, long long *bsum, int64_t *st, cudaStream_t s) {
  return exclusive_scan(in, n, out, bsum, st, s);
}
size_t scan_i32_bsum_bytes(int64_t n) { return scan_bsum_bytes(n); }

size_t plan_layout(emg_plan *p) {
  size_t o = 0;
  p->off_ent_ptr = o;
  o = align_up(o + (size_t)(p->n_ent + 1) * 4, 256);
  p->off_item = o;
  o = align_up(o + (size_t)p->n_items * sizeof(Item), 256);
  p->off_item_pos = p->off_item;  // positions live inside the item records
  p->off_ent_cnt = o;
  o = align_up(o + (size_t)p->n_ent * 4, 256);
  // 20 contributions (uint16: item-in-chunk << 5 | row) per item, and one
  // uint16 start offset per first-DoF output position; a column of entity x
  // has 2 (n_adj_edges + n_adj_faces) <= 20 * items(x) entries, so 20 per item
  // bounds the positions before nnz is known
  p->off_contrib = o;
  o = align_up(o + (size_t)p->n_items * 20 * 2, 256);
  p->off_posoff = o;
  o = align_up(o + (size_t)p->n_items * 20 * 2, 256);
  // per contribution the packed-layout indices of its two values (first- and
  // second-DoF column), in the same order as contrib; block layout: one
  // 4-byte block record per (item, row entity) and a uint16 list start per
  // row pair (at most 10 per item)
  const bool block = p->value_layout == EMG_LAYOUT_BLOCK;
  p->off_pidx = o;
  o = align_up(o + (size_t)p->n_items * (block ? 10 * 4 : 20 * (p->record_bytes == 4 ? 4 : 8)), 256);
  p->off_hoff = o;
  o = align_up(o + (block ? (size_t)p->n_items * 10 * 2 : 0), 256);
  // the gather's chunk processing order
  p->off_order = o;
  o = align_up(o + (size_t)n_chunks(p->n_edges, p->n_tris) * 4, 256);
  p->plan_bytes = o;
  return o;
}

// chunk-order scratch: bounding-box partials and the sort keys (power of two)
constexpr int BBOX_BLOCKS = 296;
static size_t order_workspace_bytes(const emg_plan *p) {
  return align_up((size_t)BBOX_BLOCKS * 6 * 8 + 64, 256) +
         (size_t)pow2_at_least(n_chunks(p->n_edges, p->n_tris)) * 8;
}

// workspace: per-entity counters, per-column lengths, scan block sums, max
// (plan build); bounding box and sort keys (chunk order); the larger of both
size_t plan_workspace_bytes(const emg_plan *p) {
  size_t w = 0;
  w = align_up(w + (size_t)p->n_ent * 4, 256);
  w = align_up(w + (size_t)(p->N + 1) * 4, 256);
  w = align_up(w + scan_bsum_bytes(p->N > p->n_ent ? p->N : p->n_ent), 256);
  w = align_up(w + 16, 256);
  const size_t wo = order_workspace_bytes(p);
  return w > wo ? w : wo;
}

int plan_build(emg_plan *p, const int32_t *d_tets, const int32_t *d_t2e, const int32_t *d_t2t,
               const int32_t *d_tetids, void *d_plan, void *d_ws, int32_t *d_indptr, int64_t *d_status,
               cudaStream_t s) {
  char *plan = static_cast<char *>(d_plan);
  char *ws = static_cast<char *>(d_ws);
  int32_t *ent_ptr = reinterpret_cast<int32_t *>(plan + p->off_ent_ptr);
  Item *items = reinterpret_cast<Item *>(plan + p->off_item);
  uint32_t *ent_cnt = reinterpret_cast<uint32_t *>(plan + p->off_ent_cnt);
  size_t o = 0;
  int32_t *cnt = reinterpret_cast<int32_t *>(ws + o);
  o = align_up(o + (size_t)p->n_ent * 4, 256);
  int32_t *col_len = reinterpret_cast<int32_t *>(ws + o);
  o = align_up(o + (size_t)(p->N + 1) * 4, 256);
  long long *bsum = reinterpret_cast<long long *>(ws + o);
  o = align_up(o + scan_bsum_bytes(p->N > p->n_ent ? p->N : p->n_ent), 256);
  int32_t *maxc = reinterpret_cast<int32_t *>(ws + o);
  int rc;
  if ((rc = status_reset(d_status, s))) return rc;
  if (p->n_ent > 0) CUDA_TRY(cudaMemsetAsync(cnt, 0, (size_t)p->n_ent * 4, s));
  CUDA_TRY(cudaMemsetAsync(maxc, 0, 4, s));
  const int64_t nI = p->n_items;
  if (nI > 0) {
    k_count_incidence<<<grid_for(nI, 256), 256, 0, s>>>(d_t2e, d_t2t, d_tetids, p->n_tets, p->n_assy, p->n_edges,
                                                         p->n_tris, cnt, d_status);
    if ((rc = launch_check("k_count_incidence"))) return rc;
  }
  if ((rc = exclusive_scan(cnt, p->n_ent, ent_ptr, bsum, d_status, s))) return rc;
  if (p->n_ent > 0) CUDA_TRY(cudaMemsetAsync(cnt, 0, (size_t)p->n_ent * 4, s));
  if (nI > 0) {
    k_fill_items<<<grid_for(nI, 256), 256, 0, s>>>(d_tets, d_t2e, d_t2t, d_tetids, p->n_tets, p->n_assy,
                                                    p->n_edges, p->n_tris, ent_ptr, cnt, items);
    if ((rc = launch_check("k_fill_items"))) return rc;
  }
  CUDA_TRY(cudaMemsetAsync(col_len, 0, (size_t)(p->N + 1) * 4, s));
  if (p->n_ent > 0) {
    k_sort_items<<<grid_for(p->n_ent, 256), 256, 0, s>>>(ent_ptr, p->n_ent, items);
    if ((rc = launch_check("k_sort_items"))) return rc;
    k_entity_rows<false><<<grid_for(p->n_ent, ROWS_WARPS), ROWS_WARPS * 32, 0, s>>>(
        d_t2e, d_t2t, d_tetids, p->n_tets, p->n_edges, p->n_tris, ent_ptr, items, p->n_ent, col_len, ent_cnt,
        nullptr, nullptr, d_status);
    if ((rc = launch_check("k_entity_rows<count>"))) return rc;
    k_max_col<<<296, 256, 0, s>>>(col_len, p->N, maxc);
    if ((rc = launch_check("k_max_col"))) return rc;
  }
  if ((rc = exclusive_scan(col_len, p->N, d_indptr, bsum, d_status, s))) return rc;
  int32_t h_nnz = 0, h_max = 0;
  int64_t h_st[2] = {0, 0};
  CUDA_TRY(cudaMemcpyAsync(&h_nnz, d_indptr + p->N, 4, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(&h_max, maxc, 4, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(h_st, d_status, 16, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (h_st[0])
    return fail(EMG_EMESH, "plan build: status flags 0x%llx at index %lld", (long long)h_st[0], (long long)h_st[1]);
  p->nnz = h_nnz;
  p->max_col = h_max;
  return EMG_OK;
}

int plan_finish(const emg_plan *p, const int32_t *d_t2e, const int32_t *d_t2t, const int32_t *d_tetids,
                void *d_plan, const int32_t *d_indptr, int32_t *d_indices, int64_t *d_status, cudaStream_t s) {
  char *plan = static_cast<char *>(d_plan);
  const int64_t nch = n_chunks(p->n_edges, p->n_tris);
  if (nch > 0) {
    k_default_order<<<grid_for(nch, 256), 256, 0, s>>>(reinterpret_cast<int32_t *>(plan + p->off_order),
                                                        n_edge_chunks(p->n_edges), nch);
    const int rc = launch_check("k_default_order");
    if (rc) return rc;
  }
  if (p->n_ent == 0 || p->n_assy == 0) return EMG_OK;
  const int32_t *ent_ptr = reinterpret_cast<const int32_t *>(plan + p->off_ent_ptr);
  Item *items = reinterpret_cast<Item *>(plan + p->off_item);
  uint32_t *ent_cnt = reinterpret_cast<uint32_t *>(plan + p->off_ent_cnt);
  k_entity_rows<true><<<grid_for(p->n_ent, ROWS_WARPS), ROWS_WARPS * 32, 0, s>>>(
      d_t2e, d_t2t, d_tetids, p->n_tets, p->n_edges, p->n_tris, ent_ptr, items, p->n_ent, nullptr, ent_cnt,
      d_indptr, d_indices, d_status);
  int rc = launch_check("k_entity_rows<fill>");
  if (rc) return rc;
  uint16_t *contrib = reinterpret_cast<uint16_t *>(plan + p->off_contrib);
  uint16_t *posoff = reinterpret_cast<uint16_t *>(plan + p->off_posoff);
  void *pidx = plan + p->off_pidx;
  const bool compact = p->record_bytes == 4;
  const bool block = p->value_layout == EMG_LAYOUT_BLOCK;
  // the block layout keeps the (item, row) lists for the COO gather and puts
  // its own records where the packed records would be
  k_chunk_contrib<<<grid_for(n_chunks(p->n_edges, p->n_tris), CC_WARPS), CC_WARPS * 32, 0, s>>>(
      ent_ptr, items, ent_cnt, p->n_edges, p->n_tris, d_indptr, contrib, posoff, block ? nullptr : pidx, compact,
      d_status);
  if ((rc = launch_check("k_chunk_contrib"))) return rc;
  if (!block) return EMG_OK;
  k_chunk_blocks<<<grid_for(n_chunks(p->n_edges, p->n_tris), CC_WARPS), CC_WARPS * 32, 0, s>>>(
      ent_ptr, items, ent_cnt, p->n_edges, p->n_tris, d_indptr, reinterpret_cast<uint16_t *>(plan + p->off_hoff),
      static_cast<uint32_t *>(pidx), d_status);
  return launch_check("k_chunk_blocks");
}

int sort_u64(uint64_t *keys, int64_t n2, cudaStream_t s) {
  if (n2 & (n2 - 1)) return fail(EMG_EINVAL, "sort length %lld is not a power of two", (long long)n2);
  for (int64_t k = 2; k <= n2; k <<= 1)
    for (int64_t j = k >> 1; j > 0; j >>= 1) {
      k_bitonic_step<<<grid_for(n2, 256), 256, 0, s>>>(keys, n2, j, k);
      const int rc = launch_check("k_bitonic_step");
      if (rc) return rc;
    }
  return EMG_OK;
}

int plan_order(const emg_plan *p, void *d_plan, const double *nodes, int64_t nN, const int32_t *tets,
               const int32_t *tetids, void *d_ws, cudaStream_t s) {
  const int64_t nch = n_chunks(p->n_edges, p->n_tris);
  if (nch == 0 || p->n_assy == 0 || nN == 0) return EMG_OK;
  char *plan = static_cast<char *>(d_plan);
  char *ws = static_cast<char *>(d_ws);
  double *part = reinterpret_cast<double *>(ws);
  double *box = part + (size_t)BBOX_BLOCKS * 6;
  uint64_t *keys = reinterpret_cast<uint64_t *>(ws + align_up((size_t)BBOX_BLOCKS * 6 * 8 + 64, 256));
  const int64_t n2 = pow2_at_least(nch);
  k_bbox_partial<<<BBOX_BLOCKS, 256, 0, s>>>(nodes, nN, part);
  int rc = launch_check("k_bbox_partial");
  if (rc) return rc;
  k_bbox_final<<<1, 32, 0, s>>>(part, BBOX_BLOCKS, box);
  if ((rc = launch_check("k_bbox_final"))) return rc;
  k_chunk_keys<<<grid_for(n2, 256), 256, 0, s>>>(
      reinterpret_cast<const int32_t *>(plan + p->off_ent_ptr), reinterpret_cast<const Item *>(plan + p->off_item),
      nodes, nN, tets, p->n_tets, tetids, p->n_assy, box, p->n_edges, p->n_tris, nch, n2, keys);
  if ((rc = launch_check("k_chunk_keys"))) return rc;
  if ((rc = sort_u64(keys, n2, s))) return rc;
  k_write_order<<<grid_for(nch, 256), 256, 0, s>>>(keys, nch, reinterpret_cast<int32_t *>(plan + p->off_order));
  return launch_check("k_write_order");
}

}  // namespace emg
