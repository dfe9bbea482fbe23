// gather.cu -- column gather + segmented sum, and the frequency-sweep form.
//
// Replaces CSCMapping.to_csc / scatter_to_csc_c16 (mth/csc_cast.py:55-63,
// 162-177) and the caller's COO combination Evec - Bvec*k0^2
// (physics/microwave/assembly/assembler.py:494).
#include <type_traits>
#include "common.cuh"

namespace emg {
namespace {

struct C64 {
  double re, im;
};


// L2 eviction priority "evict last" for the element values: each
// off-diagonal block is read twice, by the chunks of its two entities, and
// the second read comes after some of A and of the records have streamed
// through L2. Marking the value reads evict-last (createpolicy, a per-load
// hint; no device setting changes) keeps more of them resident for that
// second read (complex64 gather 4.15 -> 3.70 ms on the 2.01M-tet box, complex128
// unchanged); the same hint on A's stores or the records measured slower.
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

template <typename R>
__device__ __forceinline__ C64 load_val_last(const void *p, int64_t idx, uint64_t pol) {
  if constexpr (sizeof(R) == 8) {
    double2 v;
    asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
                 : "=d"(v.x), "=d"(v.y)
                 : "l"(reinterpret_cast<const double2 *>(p) + idx), "l"(pol));
    return {v.x, v.y};
  } else {
    float2 v;
    asm volatile("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
                 : "=f"(v.x), "=f"(v.y)
                 : "l"(reinterpret_cast<const float2 *>(p) + idx), "l"(pol));
    return {(double)v.x, (double)v.y};
  }
}

template <typename R>
__device__ __forceinline__ C64 load_val(const void *p, int64_t idx) {
  if constexpr (sizeof(R) == 8) {
    double2 v = reinterpret_cast<const double2 *>(p)[idx];
    return {v.x, v.y};
  } else {
    float2 v = reinterpret_cast<const float2 *>(p)[idx];
    return {(double)v.x, (double)v.y};
  }
}

// Pull gather (every layout). A warp owns one entity chunk (CHUNK consecutive
// entities of one kind, see common.cuh); its two output runs are contiguous.
// Lane l owns positions l, l+32, ... of the runs: it reads the position's
// contribution list from the plan (item of the chunk, element row), sums the
// contributing element values in that fixed order (items ascending, so tets
// ascending), and writes the first-DoF and second-DoF entries once. No shared
// memory, no atomics; each nonzero is produced by exactly one lane.
constexpr int PG_WARPS = 8;

// element slots (row r, column a0) and (row r, column a1) of the reference COO
// block: the item's contributions to its entity's two columns
template <typename R>
__device__ __forceinline__ void load_coo_pair(const void *v, int ia, int slot, int r, C64 &u0, C64 &u1) {
  const int a0 = slot < 6 ? slot : 12 + (slot - 6);
  const int a1 = slot < 6 ? slot + 6 : 16 + (slot - 6);
  const int64_t base = (int64_t)ia * 400 + r * 20;
  u0 = load_val<R>(v, base + a0);
  u1 = load_val<R>(v, base + a1);
}

struct ChunkMeta {
  int32_t I0, I1, A0, A1, Lsum;
  int64_t hbase;
  int64_t x0, cb0;  // first entity of the chunk and its first-DoF column
  int nx;           // entities in the chunk
};

// Processing position g -> chunk through the plan's order array (the default
// interleave, or a spatial order from emg_plan_order), so that the element
// values of a region's tets are read while still in L2.
__device__ __forceinline__ bool chunk_meta(const int32_t *ent_ptr, const int32_t *order, const int32_t *indptr,
                                           int64_t E, int64_t F, int64_t g, ChunkMeta &m) {
  const int lane = threadIdx.x & 31;
  const int64_t nec = n_edge_chunks(E);
  const int64_t nch = n_chunks(E, F);
  if (g >= nch) return false;
  const int64_t chunk = __ldg(order + g);
  if (chunk < 0 || chunk >= nch) return false;  // only a corrupted plan can hold this
  const bool edges = chunk < nec;
  const int64_t x0 = edges ? chunk * CHUNK : E + (chunk - nec) * CHUNK;
  const int nx = (int)min((int64_t)CHUNK, (edges ? E : E + F) - x0);
  const int64_t cb0 = edges ? x0 : E + x0;          // first-DoF column of x0 (faces: 2E + (x0 - E))
  const int64_t cb1 = edges ? x0 + E : E + F + x0;  // second-DoF column of x0
  int32_t meta = 0;
  if (lane == 0) meta = ent_ptr[x0];
  else if (lane == 1) meta = ent_ptr[x0 + nx];
  else if (lane == 2) meta = indptr[cb0];
  else if (lane == 3) meta = indptr[cb0 + nx];
  else if (lane == 4) meta = indptr[cb1];
  else if (lane == 5) meta = edges ? 0 : indptr[E];
  else if (lane == 6) meta = edges ? 0 : indptr[2 * E];
  m.I0 = __shfl_sync(0xffffffffu, meta, 0);
  m.I1 = __shfl_sync(0xffffffffu, meta, 1);
  m.A0 = __shfl_sync(0xffffffffu, meta, 2);
  m.Lsum = __shfl_sync(0xffffffffu, meta, 3) - m.A0;
  m.A1 = __shfl_sync(0xffffffffu, meta, 4);
  const int32_t cE = __shfl_sync(0xffffffffu, meta, 5), c2E = __shfl_sync(0xffffffffu, meta, 6);
  m.hbase = edges ? (int64_t)m.A0 : (int64_t)cE + (m.A0 - c2E);
  m.x0 = x0;
  m.cb0 = cb0;
  m.nx = nx;
  return true;
}

// reference COO layout (any COO data of this field's slot layout)
template <typename R, bool TWO>
__global__ void __launch_bounds__(PG_WARPS * 32)
    k_gather_coo(const int32_t *ent_ptr, const int32_t *order, const Item *items, const uint16_t *contrib,
                 const uint16_t *posoff, int64_t E, int64_t F, const int32_t *indptr, const void *v1, const void *v2, double ar, double ai,
                 double br, double bi, double2 *A) {
  const int lane = threadIdx.x & 31;
  ChunkMeta m;
  if (!chunk_meta(ent_ptr, order, indptr, E, F, (int64_t)blockIdx.x * PG_WARPS + (threadIdx.x >> 5), m)) return;
  const int total = 20 * (m.I1 - m.I0);
  const uint16_t *clist = contrib + (int64_t)20 * m.I0;
  const Item *it = items + m.I0;
  for (int p = lane; p < m.Lsum; p += 32) {
    const int o0 = posoff[m.hbase + p];
    const int o1 = min(p + 1 < m.Lsum ? (int)posoff[m.hbase + p + 1] : total, total);
    double s0r = 0.0, s0i = 0.0, s1r = 0.0, s1i = 0.0;
    for (int k = o0; k < o1; ++k) {
      const uint32_t c = clist[k];
      if ((int)(c >> 5) >= m.I1 - m.I0) continue;  // only a plan whose build was flagged can hold this
      const uint4 rec = __ldg(reinterpret_cast<const uint4 *>(it + (c >> 5)));
      const int r = (int)(c & 31u);
      C64 u0, u1;
      load_coo_pair<R>(v1, (int)rec.x, (int)(rec.y & 0xffu), r, u0, u1);
      s0r += ar * u0.re - ai * u0.im;
      s0i += ar * u0.im + ai * u0.re;
      s1r += ar * u1.re - ai * u1.im;
      s1i += ar * u1.im + ai * u1.re;
      if (TWO) {
        C64 t0, t1;
        load_coo_pair<R>(v2, (int)rec.x, (int)(rec.y & 0xffu), r, t0, t1);
        s0r += br * t0.re - bi * t0.im;
        s0i += br * t0.im + bi * t0.re;
        s1r += br * t1.re - bi * t1.im;
        s1i += br * t1.im + bi * t1.re;
      }
    }
    A[m.A0 + p] = make_double2(s0r, s0i);
    A[m.A1 + p] = make_double2(s1r, s1i);
  }
}

// packed layout (the assembly path): per contribution the two value indices
// come from the plan, as an int2 or as one compact uint32 (first index + a
// bit, the second slot from kSecondSlot)
__constant__ SecondSlotTable kSecondSlot = make_second_slot_table();

// Complex128 values (R = double): the list bounds of a lane's next position
// are loaded while the current one is summed, which takes one dependent load
// off each position's chain, with the register count held for six CTAs per
// SM. Complex64 values keep the plain loop (32 registers and eight CTAs per SM
// with 8-byte records), where the prefetch measured slower.
// Warps per CTA and CTAs per SM. A warp's time follows its chunk's list
// lengths, and a CTA's slot frees only when its slowest warp ends, so small
// CTAs keep more warps resident: 4-warp CTAs, 12 per SM at 40 registers
// (complex128) or 16 at 32 (complex64). Compact records keep 8-warp CTAs.
template <typename R, bool COMPACT>
struct PackedShape {
  static constexpr bool c128 = std::is_same<R, double>::value;
  static constexpr int warps = !COMPACT ? 4 : PG_WARPS;
  static constexpr int min_blocks = (c128 && !COMPACT) ? 12 : (!COMPACT ? 16 : 6);
};

// One warp's chunk of the packed gather (chunk meta already read).
template <typename R, bool COMPACT>
__device__ __forceinline__ void gather_packed_chunk(const ChunkMeta &m, const void *pidx_v, const uint16_t *posoff,
                                                    int64_t n_values, const void *v, double ar, double ai,
                                                    double2 *A, const uint8_t (*slot2)[210]) {
  const int lane = threadIdx.x & 31;
  const int total = 20 * (m.I1 - m.I0);
  constexpr bool PREFETCH = std::is_same<R, double>::value;
  int n0 = 0, n1 = 0;
  if (PREFETCH && lane < m.Lsum) {
    n0 = posoff[m.hbase + lane];
    n1 = lane + 1 < m.Lsum ? (int)posoff[m.hbase + lane + 1] : total;
  }
  for (int p = lane; p < m.Lsum; p += 32) {
    int o0, o1;
    if constexpr (PREFETCH) {
      o0 = n0;
      o1 = min(n1, total);
      if (p + 32 < m.Lsum) {
        n0 = posoff[m.hbase + p + 32];
        n1 = p + 33 < m.Lsum ? (int)posoff[m.hbase + p + 33] : total;
      }
    } else {
      o0 = posoff[m.hbase + p];
      o1 = min(p + 1 < m.Lsum ? (int)posoff[m.hbase + p + 1] : total, total);
    }
    double s0r = 0.0, s0i = 0.0, s1r = 0.0, s1i = 0.0;
    for (int k = o0; k < o1; ++k) {
      int64_t qx, qy;
      if constexpr (COMPACT) {
        const uint32_t c = __ldg(static_cast<const uint32_t *>(pidx_v) + (int64_t)20 * m.I0 + k);
        const uint32_t x = c & 0x7fffffffu;
        const uint32_t p0 = x % 210u;
        qx = x;
        qy = (int64_t)(x - p0) + slot2[c >> 31][p0];
      } else {
        const int2 q = __ldg(static_cast<const int2 *>(pidx_v) + (int64_t)20 * m.I0 + k);
        qx = (uint32_t)q.x;
        qy = (uint32_t)q.y;
      }
      if (qx >= n_values || qy >= n_values) continue;
      const C64 u0 = load_val<R>(v, qx), u1 = load_val<R>(v, qy);
      s0r += u0.re;
      s0i += u0.im;
      s1r += u1.re;
      s1i += u1.im;
    }
    A[m.A0 + p] = make_double2(ar * s0r - ai * s0i, ar * s0i + ai * s0r);
    A[m.A1 + p] = make_double2(ar * s1r - ai * s1i, ar * s1i + ai * s1r);
  }
}


template <typename R, bool COMPACT>
__global__ void __launch_bounds__(PackedShape<R, COMPACT>::warps * 32, PackedShape<R, COMPACT>::min_blocks)
    k_gather_packed(const int32_t *ent_ptr, const int32_t *order, const void *pidx_v, const uint16_t *posoff,
                    int64_t E, int64_t F, int64_t n_values, const int32_t *indptr, const void *v, double ar,
                    double ai, double2 *A) {
  __shared__ uint8_t slot2[2][210];
  if constexpr (COMPACT) {
    for (int i = threadIdx.x; i < 420; i += blockDim.x) slot2[i / 210][i % 210] = kSecondSlot.v[i / 210][i % 210];
    __syncthreads();
  }
  ChunkMeta m;
  if (!chunk_meta(ent_ptr, order, indptr, E, F,
                  (int64_t)blockIdx.x * PackedShape<R, COMPACT>::warps + (threadIdx.x >> 5), m))
    return;
  gather_packed_chunk<R, COMPACT>(m, pidx_v, posoff, n_values, v, ar, ai, A, slot2);
}

// ---- entity-pair block layout (EMG_LAYOUT_BLOCK). A lane owns a row pair of
// the chunk's first-DoF runs -- the first-DoF row p of an adjacent entity and
// its partner row p' (the entity's second DoF) -- and sums, over the tets of
// its list in item order, the 2x2 blocks of that entity pair: the entries of
// rows p, p' in the chunk entity's two columns. One 4-byte record and one
// contiguous 64-byte (32-byte) read give four entries of A; every entry sums
// the same values in the same order as the packed gather.
constexpr int BG_WARPS = 4;

template <typename R>
__device__ __forceinline__ void gather_block_chunk(const ChunkMeta &m, const uint32_t *brec, const uint16_t *hoff,
                                                   const int32_t *indptr, const uint32_t *ent_cnt, int64_t n_blocks,
                                                   const void *v, double ar, double ai, double2 *A,
                                                   int32_t *se /* 3 * CHUNK + 1 ints of this warp */) {
  const int lane = threadIdx.x & 31;
  int32_t *hs = se;                  // half start of entity e in the chunk, hs[nx] = all row pairs
  int32_t *nes = se + CHUNK + 1;     // adjacent edges of entity e
  int32_t *cs = se + 2 * CHUNK + 1;  // first-DoF column start of entity e, relative to A0
  if (lane < m.nx) {
    const int32_t c = indptr[m.cb0 + lane] - m.A0;
    cs[lane] = c;
    hs[lane] = c / 2;
    nes[lane] = (int32_t)(ent_cnt[m.x0 + lane] & 0xffffu);
  }
  if (lane == 0) hs[m.nx] = m.Lsum / 2;
  __syncwarp();
  const uint64_t pv = policy_evict_last();
  const int H = m.Lsum / 2;
  const int total = 10 * (m.I1 - m.I0);
  const uint32_t *rl = brec + (int64_t)10 * m.I0;
  const int64_t hb = m.hbase / 2;
  int e = 0;
  // list bounds of the lane's next row pair are loaded while the current one is summed
  // complex64 values: the first record of the lane's next row pair is also
  // loaded ahead (measured 2% faster; slower for complex128)
  constexpr bool RECORD_AHEAD = !std::is_same<R, double>::value;
  int n0 = 0, n1 = 0;
  uint32_t r0n = 0;
  if (lane < H) {
    n0 = hoff[hb + lane];
    n1 = lane + 1 < H ? (int)hoff[hb + lane + 1] : total;
    if (RECORD_AHEAD && n0 < min(n1, total)) r0n = __ldg(rl + n0);
  }
  for (int h = lane; h < H; h += 32) {
    while (e + 1 < m.nx && h >= hs[e + 1]) ++e;  // h only grows along a lane
    const int hl = h - hs[e], ne = nes[e];
    const int nf = hs[e + 1] - hs[e] - ne;
    const int p = hl < ne ? cs[e] + hl : cs[e] + ne + hl;
    const int pp = hl < ne ? p + ne : p + nf;
    const int o0 = n0;
    const int o1 = min(n1, total);
    const uint32_t r0 = r0n;
    if (h + 32 < H) {
      n0 = hoff[hb + h + 32];
      n1 = h + 33 < H ? (int)hoff[hb + h + 33] : total;
    }
    double s0r = 0.0, s0i = 0.0, s1r = 0.0, s1i = 0.0, s2r = 0.0, s2i = 0.0, s3r = 0.0, s3i = 0.0;
    for (int k = o0; k < o1; ++k) {
      const uint32_t rec = (RECORD_AHEAD && k == o0) ? r0 : __ldg(rl + k);
      const int64_t b = rec & 0x7fffffffu;
      if (b >= n_blocks) continue;  // only a plan whose build was flagged can hold this
      const C64 u0 = load_val_last<R>(v, 4 * b, pv), u3 = load_val_last<R>(v, 4 * b + 3, pv);
      C64 u1 = load_val_last<R>(v, 4 * b + 1, pv), u2 = load_val_last<R>(v, 4 * b + 2, pv);
      if (rec >> 31) {
        const C64 t = u1;
        u1 = u2;
        u2 = t;
      }
      s0r += u0.re;
      s0i += u0.im;
      s1r += u1.re;
      s1i += u1.im;
      s2r += u2.re;
      s2i += u2.im;
      s3r += u3.re;
      s3i += u3.im;
    }
    if (RECORD_AHEAD && h + 32 < H && n0 < min(n1, total)) r0n = __ldg(rl + n0);
    A[m.A0 + p] = make_double2(ar * s0r - ai * s0i, ar * s0i + ai * s0r);
    A[m.A1 + p] = make_double2(ar * s1r - ai * s1i, ar * s1i + ai * s1r);
    A[m.A0 + pp] = make_double2(ar * s2r - ai * s2i, ar * s2i + ai * s2r);
    A[m.A1 + pp] = make_double2(ar * s3r - ai * s3i, ar * s3i + ai * s3r);
  }
}

template <typename R>
__global__ void __launch_bounds__(BG_WARPS * 32, 10)
    k_gather_block(const int32_t *ent_ptr, const int32_t *order, const uint32_t *brec, const uint16_t *hoff,
                   const uint32_t *ent_cnt, int64_t E, int64_t F, int64_t n_blocks, const int32_t *indptr,
                   const void *v, double ar, double ai, double2 *A) {
  __shared__ int32_t se[BG_WARPS][3 * CHUNK + 1];
  ChunkMeta m;
  if (!chunk_meta(ent_ptr, order, indptr, E, F, (int64_t)blockIdx.x * BG_WARPS + (threadIdx.x >> 5), m)) return;
  gather_block_chunk<R>(m, brec, hoff, indptr, ent_cnt, n_blocks, v, ar, ai, A, se[threadIdx.x >> 5]);
}

// Several jobs' packed gathers (8-byte records, alpha = 1) in one launch: job
// j owns the CTAs [cta_start[j], cta_start[j + 1]) and its chunks in CTA
// order, as if launched alone.
template <typename R>
__global__ void __launch_bounds__(PackedShape<R, false>::warps * 32, PackedShape<R, false>::min_blocks)
    k_gather_packed_batch(const GatherJob *jobs, const int64_t *cta_start, int n_jobs) {
  const int64_t b = blockIdx.x;
  int lo = 0, hi = n_jobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cta_start[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  if (n_jobs <= 0 || b >= cta_start[n_jobs]) return;
  const GatherJob &j = jobs[lo];
  ChunkMeta m;
  if (!chunk_meta(j.ent_ptr, j.order, j.indptr, j.E, j.F,
                  (b - cta_start[lo]) * PackedShape<R, false>::warps + (threadIdx.x >> 5), m))
    return;
  gather_packed_chunk<R, false>(m, j.pidx, j.posoff, j.n_values, j.values, 1.0, 0.0, j.A, nullptr);
}

// Several jobs' block gathers (alpha = 1) in one launch, as k_gather_packed_batch.
template <typename R>
__global__ void __launch_bounds__(BG_WARPS * 32, 10)
    k_gather_block_batch(const GatherJob *jobs, const int64_t *cta_start, int n_jobs) {
  __shared__ int32_t se[BG_WARPS][3 * CHUNK + 1];
  const int64_t b = blockIdx.x;
  int lo = 0, hi = n_jobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cta_start[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  if (n_jobs <= 0 || b >= cta_start[n_jobs]) return;
  const GatherJob &j = jobs[lo];
  ChunkMeta m;
  if (!chunk_meta(j.ent_ptr, j.order, j.indptr, j.E, j.F, (b - cta_start[lo]) * BG_WARPS + (threadIdx.x >> 5), m))
    return;
  gather_block_chunk<R>(m, static_cast<const uint32_t *>(j.pidx), j.posoff, j.indptr, j.ent_cnt, j.n_values,
                        j.values, 1.0, 0.0, j.A, se[threadIdx.x >> 5]);
}

// ---------------------------------------------------------------------------
// frequency sweep: A_f = a_f K + b_f M (+ c_f P)
// ---------------------------------------------------------------------------
constexpr int SWEEP_MAX = 32;
struct SweepCoef {
  double c[SWEEP_MAX][6];
};

// Four elements per thread per pass: their loads are independent of the
// previous pass's stores (restrict), so they are in flight together; the
// arithmetic per value is unchanged.
template <bool HASP>
__global__ void __launch_bounds__(256) k_form_sweep(const double2 *__restrict__ K, const double2 *__restrict__ M,
                                                    const double2 *__restrict__ P, int64_t nnz, SweepCoef cf, int nf,
                                                    double2 *__restrict__ out, int64_t stride) {
  constexpr int U = 4;
  const int64_t T = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < nnz; i0 += U * T) {
    double2 k[U], m[U], p[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = i0 + u * T;
      const bool in = i < nnz;
      k[u] = in ? __ldg(K + i) : make_double2(0.0, 0.0);
      m[u] = in ? __ldg(M + i) : make_double2(0.0, 0.0);
      p[u] = (HASP && in) ? __ldg(P + i) : make_double2(0.0, 0.0);
    }
    for (int f = 0; f < nf; ++f) {
      const double *c = cf.c[f];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t i = i0 + u * T;
        if (i >= nnz) break;
        double2 o;
        o.x = c[0] * k[u].x - c[1] * k[u].y + c[2] * m[u].x - c[3] * m[u].y;
        o.y = c[0] * k[u].y + c[1] * k[u].x + c[2] * m[u].y + c[3] * m[u].x;
        if (HASP) {
          o.x += c[4] * p[u].x - c[5] * p[u].y;
          o.y += c[4] * p[u].y + c[5] * p[u].x;
        }
        out[(int64_t)f * stride + i] = o;
      }
    }
  }
}

// serving batch: grid-stride over tiles of all items
constexpr int FORM_TILE = 32768;

__global__ void __launch_bounds__(256) k_form_batch(const emg_form_item *items, const int64_t *tile_start,
                                                    const int32_t *n_items_p, int max_items) {
  const int n = min(*n_items_p, max_items);
  if (n <= 0) return;
  const int64_t total = tile_start[n];
  for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
    int lo = 0, hi = n - 1;  // item with tile_start[i] <= t < tile_start[i+1]
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (tile_start[mid] <= t) lo = mid; else hi = mid - 1;
    }
    const emg_form_item &it = items[lo];
    const int64_t b = (t - tile_start[lo]) * FORM_TILE;
    const int64_t e = min(b + FORM_TILE, it.nnz);
    const int g = max(1, min(it.group, n - lo));  // the group's items share K, M, P: read them once
    const double2 *K = static_cast<const double2 *>(it.K);
    const double2 *M = static_cast<const double2 *>(it.M);
    const double2 *P = static_cast<const double2 *>(it.P);
    for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) {
      const double2 k = K[i], m = M[i];
      const double2 p = P ? P[i] : make_double2(0.0, 0.0);
      for (int f = 0; f < g; ++f) {
        const double *c = items[lo + f].coef;
        double2 o;
        o.x = c[0] * k.x - c[1] * k.y + c[2] * m.x - c[3] * m.y;
        o.y = c[0] * k.y + c[1] * k.x + c[2] * m.y + c[3] * m.x;
        if (P) {
          o.x += c[4] * p.x - c[5] * p.y;
          o.y += c[4] * p.y + c[5] * p.x;
        }
        static_cast<double2 *>(items[lo + f].out)[i] = o;
      }
    }
  }
}

}  // namespace

int launch_gather(const emg_plan *p, const void *d_plan, const int32_t *d_indptr, const void *d_v1, const void *d_v2,
                  int precision, int layout, double ar, double ai, double br, double bi, void *d_A, int64_t *d_status,
                  cudaStream_t s) {
  (void)d_status;
  if (p->n_ent == 0) return EMG_OK;
  if (precision < EMG_FP64 || precision > EMG_EXACT) return fail(EMG_EINVAL, "bad precision %d", precision);
  if (layout != EMG_LAYOUT_COO && layout != EMG_LAYOUT_PACKED && layout != EMG_LAYOUT_BLOCK)
    return fail(EMG_EINVAL, "bad layout %d", layout);
  const char *plan = static_cast<const char *>(d_plan);
  const int32_t *ent_ptr = reinterpret_cast<const int32_t *>(plan + p->off_ent_ptr);
  const Item *items = reinterpret_cast<const Item *>(plan + p->off_item);
  const int32_t *order = reinterpret_cast<const int32_t *>(plan + p->off_order);
  const uint16_t *contrib = reinterpret_cast<const uint16_t *>(plan + p->off_contrib);
  const uint16_t *posoff = reinterpret_cast<const uint16_t *>(plan + p->off_posoff);
  const int g = grid_for(n_chunks(p->n_edges, p->n_tris), PG_WARPS);
  double2 *A = static_cast<double2 *>(d_A);
  const bool two = d_v2 != nullptr;
  const bool f32 = values_fp32(precision);
  if (layout == EMG_LAYOUT_BLOCK) {
    if (two) return fail(EMG_EINVAL, "the block layout takes one value array");
    const uint32_t *brec = reinterpret_cast<const uint32_t *>(plan + p->off_pidx);
    const uint16_t *hoff = reinterpret_cast<const uint16_t *>(plan + p->off_hoff);
    const uint32_t *ent_cnt = reinterpret_cast<const uint32_t *>(plan + p->off_ent_cnt);
    const int gb = grid_for(n_chunks(p->n_edges, p->n_tris), BG_WARPS);
    const int64_t nb = p->n_assy * 55;
    if (f32)
      k_gather_block<float><<<gb, BG_WARPS * 32, 0, s>>>(ent_ptr, order, brec, hoff, ent_cnt, p->n_edges, p->n_tris,
                                                          nb, d_indptr, d_v1, ar, ai, A);
    else
      k_gather_block<double><<<gb, BG_WARPS * 32, 0, s>>>(ent_ptr, order, brec, hoff, ent_cnt, p->n_edges,
                                                           p->n_tris, nb, d_indptr, d_v1, ar, ai, A);
    return launch_check("k_gather_block");
  }
  if (layout == EMG_LAYOUT_PACKED) {
    if (two) return fail(EMG_EINVAL, "the packed layout takes one value array");
    const void *pidx = plan + p->off_pidx;
    const int64_t nv = p->n_assy * 210;
    const bool compact = p->record_bytes == 4;
#define EMG_PK(R, C)                                                                                    \
  k_gather_packed<R, C><<<grid_for(n_chunks(p->n_edges, p->n_tris), PackedShape<R, C>::warps),           \
                          PackedShape<R, C>::warps * 32, 0, s>>>(ent_ptr, order, pidx, posoff, p->n_edges,  \
                                                                 p->n_tris, nv, d_indptr, d_v1, ar, ai, A)
    if (f32) {
      if (compact) EMG_PK(float, true); else EMG_PK(float, false);
    } else {
      if (compact) EMG_PK(double, true); else EMG_PK(double, false);
    }
#undef EMG_PK
    return launch_check("k_gather_packed");
  }
#define EMG_COO(R, TWO)                                                                                           \
  k_gather_coo<R, TWO><<<g, PG_WARPS * 32, 0, s>>>(ent_ptr, order, items, contrib, posoff, p->n_edges, p->n_tris, \
                                                   d_indptr, d_v1, d_v2, ar, ai, br, bi, A)
  if (f32) {
    if (two) EMG_COO(float, true); else EMG_COO(float, false);
  } else {
    if (two) EMG_COO(double, true); else EMG_COO(double, false);
  }
#undef EMG_COO
  return launch_check("k_gather_coo");
}

int gather_job_fill(const emg_plan *p, const void *d_plan, const int32_t *d_indptr, const void *d_values, void *d_A,
                    GatherJob *out) {
  const bool block = p->value_layout == EMG_LAYOUT_BLOCK;
  if (!block && p->record_bytes != 8)
    return fail(EMG_EINVAL, "batched gathers take block-layout plans or packed ones with 8-byte records");
  const char *plan = static_cast<const char *>(d_plan);
  out->ent_ptr = reinterpret_cast<const int32_t *>(plan + p->off_ent_ptr);
  out->order = reinterpret_cast<const int32_t *>(plan + p->off_order);
  out->pidx = plan + p->off_pidx;
  out->posoff = reinterpret_cast<const uint16_t *>(plan + (block ? p->off_hoff : p->off_posoff));
  out->indptr = d_indptr;
  out->ent_cnt = reinterpret_cast<const uint32_t *>(plan + p->off_ent_cnt);
  out->values = d_values;
  out->A = static_cast<double2 *>(d_A);
  out->E = p->n_edges;
  out->F = p->n_tris;
  out->n_values = p->n_assy * (block ? 55 : 210);
  const int warps = block ? BG_WARPS : PackedShape<double, false>::warps;
  out->n_ctas = (n_chunks(p->n_edges, p->n_tris) + warps - 1) / warps;
  return EMG_OK;
}

int launch_gather_batch(const GatherJob *d_jobs, const int64_t *d_cta_start, int n_jobs, int64_t total_ctas,
                        int precision, int layout, cudaStream_t s) {
  if (n_jobs == 0 || total_ctas == 0) return EMG_OK;
  if (total_ctas > INT32_MAX) return fail(EMG_ERANGE, "too many CTAs (%lld)", (long long)total_ctas);
  if (layout == EMG_LAYOUT_BLOCK) {
    if (values_fp32(precision))
      k_gather_block_batch<float><<<(unsigned)total_ctas, BG_WARPS * 32, 0, s>>>(d_jobs, d_cta_start, n_jobs);
    else
      k_gather_block_batch<double><<<(unsigned)total_ctas, BG_WARPS * 32, 0, s>>>(d_jobs, d_cta_start, n_jobs);
    return launch_check("k_gather_block_batch");
  }
  static_assert(PackedShape<double, false>::warps == PackedShape<float, false>::warps, "same chunks per CTA");
  if (values_fp32(precision))
    k_gather_packed_batch<float><<<(unsigned)total_ctas, PackedShape<float, false>::warps * 32, 0, s>>>(
        d_jobs, d_cta_start, n_jobs);
  else
    k_gather_packed_batch<double><<<(unsigned)total_ctas, PackedShape<double, false>::warps * 32, 0, s>>>(
        d_jobs, d_cta_start, n_jobs);
  return launch_check("k_gather_packed_batch");
}

int launch_form_batch(const emg_form_item *items, const int64_t *tile_start, const int32_t *n_items, int max_items,
                      cudaStream_t s) {
  // many short-lived CTAs (a few tiles each) rather than a persistent grid,
  // so that kernels of higher-priority streams are scheduled between them
  k_form_batch<<<persistent_ctas(16), 256, 0, s>>>(items, tile_start, n_items, max_items);
  return launch_check("k_form_batch");
}

int launch_form_sweep(const void *d_K, const void *d_M, const void *d_P, int64_t nnz, const double *h_coef, int nf,
                      void *d_out, int64_t out_stride, cudaStream_t s) {
  for (int f0 = 0; f0 < nf; f0 += SWEEP_MAX) {
    int n = nf - f0 < SWEEP_MAX ? nf - f0 : SWEEP_MAX;
    SweepCoef c;
    memcpy(c.c, h_coef + (size_t)f0 * 6, (size_t)n * 6 * sizeof(double));
    double2 *o = static_cast<double2 *>(d_out) + (int64_t)f0 * out_stride;
    const int g = persistent_ctas(8);  // oversubscribed: measured faster than one resident wave
    if (d_P)
      k_form_sweep<true><<<g, 256, 0, s>>>((const double2 *)d_K, (const double2 *)d_M, (const double2 *)d_P, nnz, c,
                                           n, o, out_stride);
    else
      k_form_sweep<false><<<g, 256, 0, s>>>((const double2 *)d_K, (const double2 *)d_M, nullptr, nnz, c, n, o,
                                            out_stride);
    int rc = launch_check("k_form_sweep");
    if (rc) return rc;
  }
  return EMG_OK;
}

}  // namespace emg
