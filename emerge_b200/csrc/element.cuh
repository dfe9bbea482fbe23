// element.cuh -- per-tet Nedelec-2 element kernel (closed-form K_e, M_e).
//
// Replaces _matrix_builder + ned2_tet_stiff_mass + tet_coefficients +
// local_mapping + matinv (physics/microwave/assembly/curlcurl.py:127-214,
// 285-456; mth/optimized.py:262-357). Thread per assembled tet:
//  * FP64: vertex ranks (the reference orients every edge/face by ascending
//    global node id), barycentric gradients, |det| (V) and sign(det) in the
//    tet's own vertex order (the reference's L = cofactor/|det| convention),
//    material tensors and mu^-1 (the reference's matinv);
//  * the element integrals are exact closed forms (KEAST4 integrates every
//    integrand of this element space exactly), evaluated as straight-line
//    multiply-adds on the per-tet tensors G = V (eps g_m).g_n and
//    H = V (mu^-1 X_P).X_Q, in FP64 (EMG_FP64) or FP32 (EMG_MIXED);
//  * one 20-value row of the block at a time goes to shared memory and the
//    warp writes its 32 rows as contiguous runs of the [tet][a][b] layout.
#pragma once
#include "common.cuh"

namespace emg {
namespace {

struct C64 {
  double re, im;
};
struct C32 {
  float re, im;
};

__device__ __forceinline__ C64 cmul(C64 a, C64 b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ C64 cadd(C64 a, C64 b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ C64 csub(C64 a, C64 b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ C64 crecip(C64 a) {
  double d = a.re * a.re + a.im * a.im;
  return {a.re / d, -a.im / d};
}
__device__ __forceinline__ C64 cdiv(C64 a, C64 b) {
  double d = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
__device__ __forceinline__ bool cis0(C64 a) { return a.re == 0.0 && a.im == 0.0; }

__device__ __forceinline__ C64 ld_c64(const void *p, int64_t idx) {
  const double2 v = reinterpret_cast<const double2 *>(p)[idx];
  return {v.x, v.y};
}

// matinv of the reference (optimized.py:315-357): 3x3 complex inverse with the
// diagonal fast path.
__device__ void matinv3(const C64 M[9], C64 out[9]) {
  if (cis0(M[1]) && cis0(M[2]) && cis0(M[3]) && cis0(M[5]) && cis0(M[6]) && cis0(M[7])) {
#pragma unroll
    for (int i = 0; i < 9; ++i) out[i] = {0.0, 0.0};
    out[0] = crecip(M[0]);
    out[4] = crecip(M[4]);
    out[8] = crecip(M[8]);
    return;
  }
  C64 det = csub(csub(cmul(cmul(M[0], M[4]), M[8]), cmul(cmul(M[0], M[5]), M[7])), cmul(cmul(M[1], M[3]), M[8]));
  det = cadd(det, cmul(cmul(M[1], M[5]), M[6]));
  det = cadd(det, cmul(cmul(M[2], M[3]), M[7]));
  det = csub(det, cmul(cmul(M[2], M[4]), M[6]));
  C64 a[9];
  a[0] = csub(cmul(M[4], M[8]), cmul(M[5], M[7]));
  a[1] = csub(cmul(M[2], M[7]), cmul(M[1], M[8]));
  a[2] = csub(cmul(M[1], M[5]), cmul(M[2], M[4]));
  a[3] = csub(cmul(M[5], M[6]), cmul(M[3], M[8]));
  a[4] = csub(cmul(M[0], M[8]), cmul(M[2], M[6]));
  a[5] = csub(cmul(M[2], M[3]), cmul(M[0], M[5]));
  a[6] = csub(cmul(M[3], M[7]), cmul(M[4], M[6]));
  a[7] = csub(cmul(M[1], M[6]), cmul(M[0], M[7]));
  a[8] = csub(cmul(M[0], M[4]), cmul(M[1], M[3]));
#pragma unroll
  for (int i = 0; i < 9; ++i) out[i] = cdiv(a[i], det);
}

// Per-tet geometry in the canonical (vertex-rank) frame.
struct Geo {
  double g[4][3];  // grad(lambda_r), r = rank of the vertex's global id
  double V;        // |det| / 6
  double sig;      // sign(det) in the tet's own vertex order
  uint64_t inv;    // nibble c (0..9 canonical entity) -> reference entity slot (0..9)
};

// canonical edge index of rank pair r1 < r2 in (0,1),(0,2),(0,3),(1,2),(1,3),(2,3)
__device__ __forceinline__ int canon_edge(int a, int b) {
  int r1 = min(a, b), r2 = max(a, b);
  return r1 == 0 ? r2 - 1 : (r1 == 1 ? r2 + 1 : 5);
}

// returns false for a degenerate tet (repeated vertex, zero/non-finite det)
__device__ __forceinline__ bool tet_geometry(const double X[3][4], const int64_t v[4], Geo &G) {
  int rank[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int r = 0;
#pragma unroll
    for (int p = 0; p < 4; ++p) r += (v[p] < v[q]) ? 1 : 0;
    rank[q] = r;
  }
  bool distinct = (v[0] != v[1]) && (v[0] != v[2]) && (v[0] != v[3]) && (v[1] != v[2]) && (v[1] != v[3]) &&
                  (v[2] != v[3]);
  double e1[3], e2[3], e3[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    e1[d] = X[d][1] - X[d][0];
    e2[d] = X[d][2] - X[d][0];
    e3[d] = X[d][3] - X[d][0];
  }
  double c23[3] = {e2[1] * e3[2] - e2[2] * e3[1], e2[2] * e3[0] - e2[0] * e3[2], e2[0] * e3[1] - e2[1] * e3[0]};
  double c31[3] = {e3[1] * e1[2] - e3[2] * e1[1], e3[2] * e1[0] - e3[0] * e1[2], e3[0] * e1[1] - e3[1] * e1[0]};
  double c12[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
  double det = e1[0] * c23[0] + e1[1] * c23[1] + e1[2] * c23[2];
  if (!distinct || !(det != 0.0) || !isfinite(det)) return false;
  double id = 1.0 / det;
  double gl[4][3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    gl[1][d] = c23[d] * id;
    gl[2][d] = c31[d] * id;
    gl[3][d] = c12[d] * id;
    gl[0][d] = -(gl[1][d] + gl[2][d] + gl[3][d]);
  }
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      // scatter by rank without dynamic register indexing
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (rank[q] == r) G.g[r][d] = gl[q][d];
    }
  G.V = fabs(det) / 6.0;
  G.sig = det > 0.0 ? 1.0 : -1.0;
  // reference edge slots (local vertex pairs) and the vertex missing from each face slot
  const int eu[6] = {0, 0, 0, 1, 3, 2}, ev[6] = {1, 2, 3, 2, 1, 3};
  const int fmiss[4] = {3, 1, 2, 0};
  uint64_t inv = 0;
#pragma unroll
  for (int s = 0; s < 6; ++s) inv |= (uint64_t)s << (4 * canon_edge(rank[eu[s]], rank[ev[s]]));
#pragma unroll
  for (int f = 0; f < 4; ++f) inv |= (uint64_t)(6 + f) << (4 * (6 + 3 - rank[fmiss[f]]));
  G.inv = inv;
  return true;
}

// reference DoF index (0..19) of canonical DoF y
__device__ __forceinline__ int ref_dof(uint64_t inv, int y) {
  int c = y < 6 ? y : (y < 12 ? y - 6 : (y < 16 ? y - 6 : y - 10));  // canonical entity 0..9
  int s = (int)((inv >> (4 * c)) & 15ull);                             // reference entity slot 0..9
  return y < 6 ? s : (y < 12 ? 6 + s : (y < 16 ? 12 + (s - 6) : 16 + (s - 6)));
}

template <typename R>
struct CR {
  R re, im;
};

// multiply-add used by the generated tables: acc += c * v
__device__ __forceinline__ void emg_mac(double &acc, double c, double v) { acc = fma(c, v, acc); }
__device__ __forceinline__ void emg_mac(float &acc, double c, float v) { acc = fmaf((float)c, v, acc); }
__device__ __forceinline__ void emg_mac(CR<double> &acc, double c, const CR<double> &v) {
  acc.re = fma(c, v.re, acc.re);
  acc.im = fma(c, v.im, acc.im);
}
__device__ __forceinline__ void emg_mac(CR<float> &acc, double c, const CR<float> &v) {
  acc.re = fmaf((float)c, v.re, acc.re);
  acc.im = fmaf((float)c, v.im, acc.im);
}

}  // namespace

// the generated tables call emg_mac unqualified: include them inside emg
#include "nedelec_tables.cuh"

namespace {

// Contractions: real symmetric (ISO) and complex (DIAG symmetric, FULL general).
// Tensor T_G[m][n] = (eps g_m).g_n * V, T_H[P][Q] = (mu^-1 X_P).X_Q * V.
template <int KIND, typename R>
struct Tensors;

template <typename R>
struct Tensors<EMG_MAT_ISO, R> {
  R G[4][4], H[6][6];  // real, symmetric, V folded in; material scalars applied per entry
};
template <typename R>
struct Tensors<EMG_MAT_DIAG, R> {
  CR<R> G[4][4], H[6][6];
};
template <typename R>
struct Tensors<EMG_MAT_FULL, R> {
  CR<R> G[4][4], H[6][6];
};

__device__ __forceinline__ void cross3(const double a[3], const double b[3], double o[3]) {
  o[0] = a[1] * b[2] - a[2] * b[1];
  o[1] = a[2] * b[0] - a[0] * b[2];
  o[2] = a[0] * b[1] - a[1] * b[0];
}

template <typename R>
__device__ __forceinline__ void build_iso(const Geo &Gm, Tensors<EMG_MAT_ISO, R> &T) {
  double X[6][3];
  const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {1, 2, 3, 2, 3, 3};
#pragma unroll
  for (int p = 0; p < 6; ++p) cross3(Gm.g[pa[p]], Gm.g[pb[p]], X[p]);
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int n = m; n < 4; ++n) {
      double s = (Gm.g[m][0] * Gm.g[n][0] + Gm.g[m][1] * Gm.g[n][1] + Gm.g[m][2] * Gm.g[n][2]) * Gm.V;
      T.G[m][n] = T.G[n][m] = (R)s;
    }
#pragma unroll
  for (int p = 0; p < 6; ++p)
#pragma unroll
    for (int q = p; q < 6; ++q) {
      double s = (X[p][0] * X[q][0] + X[p][1] * X[q][1] + X[p][2] * X[q][2]) * Gm.V;
      T.H[p][q] = T.H[q][p] = (R)s;
    }
}

// general complex tensors: eps, minv are 3x3 row-major complex
template <int KIND, typename R>
__device__ __forceinline__ void build_cplx(const Geo &Gm, const C64 eps[9], const C64 minv[9],
                                           Tensors<KIND, R> &T) {
  double X[6][3];
  const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {1, 2, 3, 2, 3, 3};
#pragma unroll
  for (int p = 0; p < 6; ++p) cross3(Gm.g[pa[p]], Gm.g[pb[p]], X[p]);
  // (A u).w = sum_r w_r sum_c A[r][c] u_c
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int n = 0; n < 4; ++n) {
      if (KIND == EMG_MAT_DIAG && n < m) {
        T.G[m][n] = T.G[n][m];
        continue;
      }
      double sr = 0, si = 0;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (KIND == EMG_MAT_DIAG && r != c) continue;
          double w = Gm.g[n][r] * Gm.g[m][c];
          sr += eps[3 * r + c].re * w;
          si += eps[3 * r + c].im * w;
        }
      T.G[m][n] = {(R)(sr * Gm.V), (R)(si * Gm.V)};
    }
#pragma unroll
  for (int p = 0; p < 6; ++p)
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      if (KIND == EMG_MAT_DIAG && q < p) {
        T.H[p][q] = T.H[q][p];
        continue;
      }
      double sr = 0, si = 0;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (KIND == EMG_MAT_DIAG && r != c) continue;
          double w = X[q][r] * X[p][c];
          sr += minv[3 * r + c].re * w;
          si += minv[3 * r + c].im * w;
        }
      T.H[p][q] = {(R)(sr * Gm.V), (R)(si * Gm.V)};
    }
}

// entry (first=f, second=s) of K and M in the canonical frame
template <int f, int s, typename R>
__device__ __forceinline__ void entry_iso(const Tensors<EMG_MAT_ISO, R> &T, R sig, R &k, R &m) {
  R ak = 0, am = 0;
  emg_tables::Pair<f, s>::stiff(ak, T.H);
  emg_tables::Pair<f, s>::mass(am, T.G);
  if (emg_tables::odd(f) != emg_tables::odd(s)) {
    ak *= sig;
    am *= sig;
  }
  k = ak;
  m = am;
}

template <int f, int s, int KIND, typename R>
__device__ __forceinline__ void entry_cplx(const Tensors<KIND, R> &T, R sig, CR<R> &k, CR<R> &m) {
  CR<R> ak{0, 0}, am{0, 0};
  emg_tables::Pair<f, s>::stiff(ak, T.H);
  emg_tables::Pair<f, s>::mass(am, T.G);
  if (emg_tables::odd(f) != emg_tables::odd(s)) {
    ak.re *= sig;
    ak.im *= sig;
    am.re *= sig;
    am.im *= sig;
  }
  k = ak;
  m = am;
}

template <typename R>
struct StoreT;
template <>
struct StoreT<double> {
  using T = double2;
};
template <>
struct StoreT<float> {
  using T = float2;
};

constexpr int ELEM_THREADS = 128;
constexpr int ELEM_WARPS = ELEM_THREADS / 32;


// per-tet complex scale factors for the ISO kind: value = cK*K0 + cM*M0
template <int KIND, int OUT, typename R>
struct RowCtx;

template <int x, int y, int KIND, int OUT, typename R>
__device__ __forceinline__ void compute_store(const Tensors<KIND, R> &T, R sig, const CR<R> &cK, const CR<R> &cM,
                                              uint64_t inv, int rx, typename StoreT<R>::T *row) {
  using ST = typename StoreT<R>::T;
  const int b = ref_dof(inv, y);
  ST v;
  if constexpr (KIND == EMG_MAT_ISO) {
    R k0, m0;
    entry_iso<(x < y ? x : y), (x < y ? y : x)>(T, sig, k0, m0);
    v.x = cK.re * k0 + cM.re * m0;
    v.y = cK.im * k0 + cM.im * m0;
  } else {
    CR<R> k, m;
    if constexpr (KIND == EMG_MAT_DIAG) {
      entry_cplx<(x < y ? x : y), (x < y ? y : x), KIND>(T, sig, k, m);
    } else {
      // first = the DoF with the lower reference index (curlcurl.py:358-376)
      if (rx <= b) {
        entry_cplx<x, y, KIND>(T, sig, k, m);
      } else {
        entry_cplx<y, x, KIND>(T, sig, k, m);
      }
    }
    // value = cK*K + cM*M, cK/cM = (alpha, beta) or (1,0)/(0,1)
    v.x = cK.re * k.re - cK.im * k.im + cM.re * m.re - cM.im * m.im;
    v.y = cK.re * k.im + cK.im * k.re + cM.re * m.im + cM.im * m.re;
  }
  row[b] = v;
}

template <int x, int KIND, int OUT, typename R, int... Ys>
__device__ __forceinline__ void compute_row(const Tensors<KIND, R> &T, R sig, const CR<R> &cK, const CR<R> &cM,
                                            uint64_t inv, int rx, typename StoreT<R>::T *row,
                                            std::integer_sequence<int, Ys...>) {
  (compute_store<x, Ys, KIND, OUT, R>(T, sig, cK, cM, inv, rx, row), ...);
}

template <int KIND, int OUT, typename R, int X>
__device__ __forceinline__ void do_row(const Tensors<KIND, R> &T, R sig, const CR<R> &cK, const CR<R> &cM,
                                       uint64_t inv, bool active, int ia, typename StoreT<R>::T *stage,
                                       typename StoreT<R>::T *out) {
  using ST = typename StoreT<R>::T;
  const int lane = threadIdx.x & 31;
  const int rx = ref_dof(inv, X);
  if (active) compute_row<X, KIND, OUT, R>(T, sig, cK, cM, inv, rx, stage + lane * 20,
                                          std::make_integer_sequence<int, 20>{});
  __syncwarp();
  // cooperative, coalesced write of the warp's 32 rows (each 20 contiguous values)
#pragma unroll 4
  for (int it = 0; it < 20; ++it) {
    int e = it * 32 + lane;
    int r = e / 20, c = e - r * 20;
    int ia_r = __shfl_sync(0xffffffffu, ia, r);
    int a_r = __shfl_sync(0xffffffffu, rx, r);
    bool act_r = __shfl_sync(0xffffffffu, (int)active, r);
    if (act_r) out[(int64_t)ia_r * 400 + a_r * 20 + c] = stage[r * 20 + c];
  }
  __syncwarp();
}

template <int KIND, int OUT, typename R, int... Xs>
__device__ __forceinline__ void all_rows(const Tensors<KIND, R> &T, R sig, const CR<R> &cK, const CR<R> &cM,
                                         uint64_t inv, bool active, int ia, typename StoreT<R>::T *stage,
                                         typename StoreT<R>::T *out, std::integer_sequence<int, Xs...>) {
  (do_row<KIND, OUT, R, Xs>(T, sig, cK, cM, inv, active, ia, stage, out), ...);
}

template <int KIND, int OUT, typename R>
__global__ void __launch_bounds__(ELEM_THREADS) k_element(ElemArgs a) {
  using ST = typename StoreT<R>::T;
  __shared__ ST stage_all[ELEM_WARPS][32 * 20];
  ST *stage = stage_all[threadIdx.x >> 5];
  ST *out = reinterpret_cast<ST *>(a.out);
  const int64_t ia64 = (int64_t)blockIdx.x * ELEM_THREADS + threadIdx.x;
  bool active = ia64 < a.nA;
  const int ia = (int)ia64;
  Geo G;
  Tensors<KIND, R> T;
  CR<R> cK{0, 0}, cM{0, 0};
  R sig = 1;
  uint64_t inv = 0;
  if (active) {
    int64_t it = a.tetids ? (int64_t)a.tetids[ia] : ia64;
    int64_t v[4];
    bool ok = (it >= 0 && it < a.nT);
    if (ok) {
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        v[q] = a.tets[(int64_t)q * a.nT + it];
        ok &= (v[q] >= 0 && v[q] < a.nN);
      }
    }
    if (!ok) {
      flag(a.st, EMG_ST_INDEX, ia64);
      active = false;
    } else {
      double X[3][4];
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int d = 0; d < 3; ++d) X[d][q] = a.nodes[(int64_t)d * a.nN + v[q]];
      if (!tet_geometry(X, v, G)) {
        flag(a.st, EMG_ST_DEGENERATE, ia64);
        active = false;
      } else {
        sig = (R)G.sig;
        inv = G.inv;
        C64 alpha{a.ar, a.ai}, beta{a.br, a.bi};
        if (OUT == EMG_OUT_K) {
          alpha = {1.0, 0.0};
          beta = {0.0, 0.0};
        } else if (OUT == EMG_OUT_M) {
          alpha = {0.0, 0.0};
          beta = {1.0, 0.0};
        }
        if constexpr (KIND == EMG_MAT_ISO) {
          C64 eps = ld_c64(a.er, it);
          C64 minv = a.ur ? crecip(ld_c64(a.ur, it)) : C64{1.0, 0.0};
          C64 k = cmul(alpha, minv), m = cmul(beta, eps);
          cK = {(R)k.re, (R)k.im};
          cM = {(R)m.re, (R)m.im};
          build_iso<R>(G, T);
        } else {
          C64 eps[9], mu[9], minv[9];
#pragma unroll
          for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              // DIAG: compact diagonals [3][nT]; FULL: the reference's [3][3][nT]
              const bool need = (KIND == EMG_MAT_FULL) || r == c;
              const int64_t o = (KIND == EMG_MAT_FULL) ? (int64_t)(3 * r + c) * a.nT + it : (int64_t)r * a.nT + it;
              eps[3 * r + c] = need ? ld_c64(a.er, o) : C64{0.0, 0.0};
              mu[3 * r + c] = (need && a.ur) ? ld_c64(a.ur, o) : C64{(r == c) ? 1.0 : 0.0, 0.0};
            }
          matinv3(mu, minv);
          cK = {(R)alpha.re, (R)alpha.im};
          cM = {(R)beta.re, (R)beta.im};
          build_cplx<KIND, R>(G, eps, minv, T);
        }
      }
    }
  }
  all_rows<KIND, OUT, R>(T, sig, cK, cM, inv, active, ia, stage, out, std::make_integer_sequence<int, 20>{});
}

template <int KIND, int OUT, typename R>
int launch_element_t(const ElemArgs &a, cudaStream_t s) {
  if (a.nA == 0) return EMG_OK;
  k_element<KIND, OUT, R><<<grid_for(a.nA, ELEM_THREADS), ELEM_THREADS, 0, s>>>(a);
  return launch_check("k_element");
}

template <int KIND, typename R>
int launch_element_k(const ElemArgs &a, int out, cudaStream_t s) {
  switch (out) {
    case EMG_OUT_LINCOMB: return launch_element_t<KIND, EMG_OUT_LINCOMB, R>(a, s);
    case EMG_OUT_K: return launch_element_t<KIND, EMG_OUT_K, R>(a, s);
    case EMG_OUT_M: return launch_element_t<KIND, EMG_OUT_M, R>(a, s);
  }
  return fail(EMG_EINVAL, "bad output selector %d", out);
}

}  // namespace
}  // namespace emg
