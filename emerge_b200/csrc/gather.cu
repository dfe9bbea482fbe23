// gather.cu -- column gather + segmented sum, and the frequency-sweep form.
//
// Replaces CSCMapping.to_csc / scatter_to_csc_c16 (mth/csc_cast.py:55-63,
// 162-177) and the caller's COO combination Evec - Bvec*k0^2
// (physics/microwave/assembly/assembler.py:494).
#include "common.cuh"

namespace emg {
namespace {

struct C64 {
  double re, im;
};

constexpr int GATHER_WARPS = 8;
constexpr int COL_CAP = 160;  // column entries buffered in shared memory per column

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

template <typename R, bool TWO>
__global__ void __launch_bounds__(GATHER_WARPS * 32)
    k_gather(const int32_t *ent_ptr, const Item *items, const uint32_t *ent_cnt, int64_t n_ent, int64_t E, int64_t F,
             const int32_t *indptr, const void *v1, const void *v2, double ar, double ai, double br, double bi,
             double2 *A, int64_t *st) {
  __shared__ double2 buf_all[GATHER_WARPS][2][COL_CAP];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int64_t x = (int64_t)blockIdx.x * GATHER_WARPS + w;
  if (x >= n_ent) return;
  const uint32_t cnt = ent_cnt[x];
  const int ne = (int)(cnt & 0xffffu), nf = (int)(cnt >> 16);
  const int L = 2 * (ne + nf);
  const bool is_edge = x < E;
  const int64_t c0 = is_edge ? x : E + x;
  const int64_t c1 = is_edge ? x + E : E + F + x;
  const int64_t s0 = indptr[c0], s1 = indptr[c1];
  const bool in_smem = L <= COL_CAP;
  double2 *b0 = in_smem ? buf_all[w][0] : A + s0;
  double2 *b1 = in_smem ? buf_all[w][1] : A + s1;
  for (int i = lane; i < L; i += 32) {
    b0[i] = make_double2(0.0, 0.0);
    b1[i] = make_double2(0.0, 0.0);
  }
  __syncwarp();
  const int32_t ib = ent_ptr[x], ie = ent_ptr[x + 1];
  // row r of an element block -> entity slot and block offset in the column
  const int r = lane;
  const int sl = r < 6 ? r : (r < 12 ? r - 6 : (r < 16 ? r - 6 : r - 10));
  const int off = r < 6 ? 0 : (r < 12 ? ne : (r < 16 ? 2 * ne : 2 * ne + nf));
  for (int32_t k = ib; k < ie; ++k) {
    const Item rec = items[k];
    if (r < 20) {
      const int s = rec.slot;
      const int a0 = s < 6 ? s : 12 + (s - 6);
      const int a1 = s < 6 ? s + 6 : 16 + (s - 6);
      const int64_t base = (int64_t)rec.ia * 400;
      C64 u0 = load_val<R>(v1, base + a0 * 20 + r);
      C64 u1 = load_val<R>(v1, base + a1 * 20 + r);
      C64 y0, y1;
      y0 = {ar * u0.re - ai * u0.im, ar * u0.im + ai * u0.re};
      y1 = {ar * u1.re - ai * u1.im, ar * u1.im + ai * u1.re};
      if (TWO) {
        C64 w0 = load_val<R>(v2, base + a0 * 20 + r);
        C64 w1 = load_val<R>(v2, base + a1 * 20 + r);
        y0.re += br * w0.re - bi * w0.im;
        y0.im += br * w0.im + bi * w0.re;
        y1.re += br * w1.re - bi * w1.im;
        y1.im += br * w1.im + bi * w1.re;
      }
      const int p = off + rec.pos[sl];
      double2 t0 = b0[p], t1 = b1[p];
      t0.x += y0.re;
      t0.y += y0.im;
      t1.x += y1.re;
      t1.y += y1.im;
      b0[p] = t0;
      b1[p] = t1;
    }
    __syncwarp();
  }
  if (in_smem) {
    for (int i = lane; i < L; i += 32) {
      A[s0 + i] = b0[i];
      A[s1 + i] = b1[i];
    }
  }
}

// ---------------------------------------------------------------------------
// frequency sweep: A_f = a_f K + b_f M (+ c_f P)
// ---------------------------------------------------------------------------
constexpr int SWEEP_MAX = 32;
struct SweepCoef {
  double c[SWEEP_MAX][6];
};

template <bool HASP>
__global__ void k_form_sweep(const double2 *K, const double2 *M, const double2 *P, int64_t nnz, SweepCoef cf, int nf,
                             double2 *out, int64_t stride) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nnz; i += (int64_t)gridDim.x * blockDim.x) {
    double2 k = K[i], m = M[i];
    double2 p = HASP ? P[i] : make_double2(0.0, 0.0);
    for (int f = 0; f < nf; ++f) {
      const double *c = cf.c[f];
      double2 o;
      o.x = c[0] * k.x - c[1] * k.y + c[2] * m.x - c[3] * m.y;
      o.y = c[0] * k.y + c[1] * k.x + c[2] * m.y + c[3] * m.x;
      if (HASP) {
        o.x += c[4] * p.x - c[5] * p.y;
        o.y += c[4] * p.y + c[5] * p.x;
      }
      out[(int64_t)f * stride + i] = o;
    }
  }
}

}  // namespace

int launch_gather(const emg_plan *p, const void *d_plan, const int32_t *d_indptr, const void *d_v1, const void *d_v2,
                  int precision, double ar, double ai, double br, double bi, void *d_A, int64_t *d_status,
                  cudaStream_t s) {
  if (p->n_ent == 0) return EMG_OK;
  const char *plan = static_cast<const char *>(d_plan);
  const int32_t *ent_ptr = reinterpret_cast<const int32_t *>(plan + p->off_ent_ptr);
  const Item *items = reinterpret_cast<const Item *>(plan + p->off_item);
  const uint32_t *ent_cnt = reinterpret_cast<const uint32_t *>(plan + p->off_ent_cnt);
  const int g = grid_for(p->n_ent, GATHER_WARPS);
  double2 *A = static_cast<double2 *>(d_A);
#define EMG_GATHER(R, TWO)                                                                                         \
  k_gather<R, TWO><<<g, GATHER_WARPS * 32, 0, s>>>(ent_ptr, items, ent_cnt, p->n_ent, p->n_edges, p->n_tris,      \
                                                   d_indptr, d_v1, d_v2, ar, ai, br, bi, A, d_status)
  if (precision < EMG_FP64 || precision > EMG_EXACT) return fail(EMG_EINVAL, "bad precision %d", precision);
  if (!values_fp32(precision)) {
    if (d_v2) EMG_GATHER(double, true); else EMG_GATHER(double, false);
  } else {
    if (d_v2) EMG_GATHER(float, true); else EMG_GATHER(float, false);
  }
#undef EMG_GATHER
  return launch_check("k_gather");
}

int launch_form_sweep(const void *d_K, const void *d_M, const void *d_P, int64_t nnz, const double *h_coef, int nf,
                      void *d_out, int64_t out_stride, cudaStream_t s) {
  for (int f0 = 0; f0 < nf; f0 += SWEEP_MAX) {
    int n = nf - f0 < SWEEP_MAX ? nf - f0 : SWEEP_MAX;
    SweepCoef c;
    memcpy(c.c, h_coef + (size_t)f0 * 6, (size_t)n * 6 * sizeof(double));
    double2 *o = static_cast<double2 *>(d_out) + (int64_t)f0 * out_stride;
    const int g = 148 * 8;
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
