// element.cuh -- per-tet Nedelec-2 element kernel.
//
// Replaces _matrix_builder + ned2_tet_stiff_mass + tet_coefficients +
// local_mapping + matinv (physics/microwave/assembly/curlcurl.py:127-214,
// 285-456; mth/optimized.py:262-357). Thread per assembled tet, three forms:
//
//  FORM_REF64 (EMG_FP64, plain) reproduces the reference's arithmetic: its
//    barycentric coefficients from absolute-coordinate cofactors, its KEAST4
//    points and its values L~ of the four barycentric functions at them, all
//    in FP64 without fused multiply-adds in the reference's operation order.
//    The 11-point sums are then evaluated exactly as the per-tet quadrature
//    moments mu[alpha] = sum_q w_q L~_q^alpha (degree <= 4) contracted with
//    the tensors G = V (eps grad L~_m).grad L~_n and H = V (mu^-1 X_P).X_Q
//    through generated tables (nedelec_moment_tables.cuh).
//  FORM_REF32 (EMG_MIXED): FP64 geometry from edge vectors (Jacobian,
//    determinant, gradients, orientation sign), the tensors G and H formed in
//    FP64 and rounded to FP32, then contracted in FP32 with FP32 accumulation
//    against the closed-form tables (nedelec_tables.cuh). KEAST4 integrates
//    every product of two basis values or curls of this element exactly, so
//    its 11-point sums are fixed rational combinations of the tensors; the
//    tables hold them, evaluated once when the tables are generated. Element
//    values complex64.
//  FORM_EXACT (EMG_EXACT): exact closed-form integrals (nedelec_tables.cuh)
//    on accurate edge-vector geometry, free of the reference's cancellation.
//
// Every form writes one of three layouts (element_cta): the reference's COO
// block value[ia*400 + 20*a + b], the packed canonical upper triangle
// [ia][210], or the entity-pair blocks [ia][220] of the assembly path. One row
// of the block at a time is staged in shared memory and the warp writes its
// 32 tets' rows as contiguous runs.
#pragma once
#include "common.cuh"

namespace emg {
namespace {

enum { FORM_REF64 = 0, FORM_REF32 = 1, FORM_EXACT = 2 };
template <int FORM>
struct FormReal {
  using T = double;
};
template <>
struct FormReal<FORM_REF32> {
  using T = float;
};

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


// KEAST4 11-point rule exactly as the reference prints it (curlcurl.py:277-283):
// row 0 weights, rows 1-4 barycentric coordinates of the points.
__constant__ double kDP[5][11] = {
    {-0.07893333333333329982, 0.04573333333333329948, 0.04573333333333329948, 0.04573333333333329948,
     0.04573333333333329948, 0.14933333333333329018, 0.14933333333333329018, 0.14933333333333329018,
     0.14933333333333329018, 0.14933333333333329018, 0.14933333333333329018},
    {0.25000000000000000000, 0.78571428571428569843, 0.07142857142857139685, 0.07142857142857139685,
     0.07142857142857139685, 0.10059642383320080428, 0.39940357616679922348, 0.39940357616679922348,
     0.39940357616679922348, 0.10059642383320080428, 0.10059642383320080428},
    {0.25000000000000000000, 0.07142857142857139685, 0.07142857142857139685, 0.07142857142857139685,
     0.78571428571428569843, 0.39940357616679922348, 0.10059642383320080428, 0.39940357616679922348,
     0.10059642383320080428, 0.39940357616679922348, 0.10059642383320080428},
    {0.25000000000000000000, 0.07142857142857139685, 0.07142857142857139685, 0.78571428571428569843,
     0.07142857142857139685, 0.39940357616679922348, 0.39940357616679922348, 0.10059642383320080428,
     0.10059642383320080428, 0.10059642383320080428, 0.39940357616679922348},
    {0.25000000000000000000, 0.07142857142857150787, 0.78571428571428580945, 0.07142857142857150787,
     0.07142857142857150787, 0.10059642383320077652, 0.10059642383320077652, 0.10059642383320074877,
     0.39940357616679922348, 0.39940357616679922348, 0.39940357616679922348},
};

// Per-tet geometry in the canonical (vertex-rank) frame.
struct Geo {
  double g[4][3];  // gradients by vertex rank: reference forms grad L~, exact form grad lambda
  double V;        // |det| / 6 (reference determinant in the reference forms)
  double sig;      // sign(det) in the tet's own vertex order (exact form only)
  uint64_t inv;    // nibble c (0..9 canonical entity) -> reference entity slot (0..9)
};


// Barycentric coefficients exactly as the reference forms them
// (tet_coefficients, curlcurl.py:127-214): 24-term determinant and signed
// cofactors in ABSOLUTE coordinates, evaluated left to right without fused
// multiply-adds, V = |det| / 6, coefficient = cofactor / (6 V). These
// expressions cancel heavily (terms ~|x|^3 against det ~h^3), so the
// reference's element matrices carry that rounding; reproducing the same
// operation order keeps the GPU values within ulps of the reference's
// instead of differing by the cancellation error.
#define EMG_M2(a, b) __dmul_rn((a), (b))
#define EMG_M3(a, b, c) __dmul_rn(__dmul_rn((a), (b)), (c))
#define EMG_A(a, b) __dadd_rn((a), (b))
#define EMG_S(a, b) __dsub_rn((a), (b))

__device__ __forceinline__ void ref_coefficients(const double X[3][4], double ca[4], double cb[4], double cc[4],
                                                 double cd[4], double &det) {
  const double x1 = X[0][0], x2 = X[0][1], x3 = X[0][2], x4 = X[0][3];
  const double y1 = X[1][0], y2 = X[1][1], y3 = X[1][2], y4 = X[1][3];
  const double z1 = X[2][0], z2 = X[2][1], z3 = X[2][2], z4 = X[2][3];
  double d = EMG_M3(-x1, y2, z3);
  d = EMG_A(d, EMG_M3(x1, y2, z4));
  d = EMG_A(d, EMG_M3(x1, y3, z2));
  d = EMG_S(d, EMG_M3(x1, y3, z4));
  d = EMG_S(d, EMG_M3(x1, y4, z2));
  d = EMG_A(d, EMG_M3(x1, y4, z3));
  d = EMG_A(d, EMG_M3(x2, y1, z3));
  d = EMG_S(d, EMG_M3(x2, y1, z4));
  d = EMG_S(d, EMG_M3(x2, y3, z1));
  d = EMG_A(d, EMG_M3(x2, y3, z4));
  d = EMG_A(d, EMG_M3(x2, y4, z1));
  d = EMG_S(d, EMG_M3(x2, y4, z3));
  d = EMG_S(d, EMG_M3(x3, y1, z2));
  d = EMG_A(d, EMG_M3(x3, y1, z4));
  d = EMG_A(d, EMG_M3(x3, y2, z1));
  d = EMG_S(d, EMG_M3(x3, y2, z4));
  d = EMG_S(d, EMG_M3(x3, y4, z1));
  d = EMG_A(d, EMG_M3(x3, y4, z2));
  d = EMG_A(d, EMG_M3(x4, y1, z2));
  d = EMG_S(d, EMG_M3(x4, y1, z3));
  d = EMG_S(d, EMG_M3(x4, y2, z1));
  d = EMG_A(d, EMG_M3(x4, y2, z3));
  d = EMG_A(d, EMG_M3(x4, y3, z1));
  d = EMG_S(d, EMG_M3(x4, y3, z2));
  det = d;
  // six-term cofactor sums (the reference's bbs, ccs, dds)
#define EMG_C6(s1, a1, b1, s2, a2, b2, s3, a3, b3, s4, a4, b4, s5, a5, b5, s6, a6, b6)                   \
  EMG_##s6(EMG_##s5(EMG_##s4(EMG_##s3(EMG_##s2(EMG_M2(s1 a1, b1), EMG_M2(a2, b2)), EMG_M2(a3, b3)),       \
                             EMG_M2(a4, b4)),                                                             \
                    EMG_M2(a5, b5)),                                                                      \
           EMG_M2(a6, b6))
  cb[0] = EMG_C6(-, y2, z3, A, y2, z4, A, y3, z2, S, y3, z4, S, y4, z2, A, y4, z3);
  cb[1] = EMG_C6(+, y1, z3, S, y1, z4, S, y3, z1, A, y3, z4, A, y4, z1, S, y4, z3);
  cb[2] = EMG_C6(-, y1, z2, A, y1, z4, A, y2, z1, S, y2, z4, S, y4, z1, A, y4, z2);
  cb[3] = EMG_C6(+, y1, z2, S, y1, z3, S, y2, z1, A, y2, z3, A, y3, z1, S, y3, z2);
  cc[0] = EMG_C6(+, x2, z3, S, x2, z4, S, x3, z2, A, x3, z4, A, x4, z2, S, x4, z3);
  cc[1] = EMG_C6(-, x1, z3, A, x1, z4, A, x3, z1, S, x3, z4, S, x4, z1, A, x4, z3);
  cc[2] = EMG_C6(+, x1, z2, S, x1, z4, S, x2, z1, A, x2, z4, A, x4, z1, S, x4, z2);
  cc[3] = EMG_C6(-, x1, z2, A, x1, z3, A, x2, z1, S, x2, z3, S, x3, z1, A, x3, z2);
  cd[0] = EMG_C6(-, x2, y3, A, x2, y4, A, x3, y2, S, x3, y4, S, x4, y2, A, x4, y3);
  cd[1] = EMG_C6(+, x1, y3, S, x1, y4, S, x3, y1, A, x3, y4, A, x4, y1, S, x4, y3);
  cd[2] = EMG_C6(-, x1, y2, A, x1, y4, A, x2, y1, S, x2, y4, S, x4, y1, A, x4, y2);
  cd[3] = EMG_C6(+, x1, y2, S, x1, y3, S, x2, y1, A, x2, y3, A, x3, y1, S, x3, y2);
#undef EMG_C6
  // six-term triple-product sums (the reference's aas)
#define EMG_T6(s1, a1, b1, c1, s2, a2, b2, c2, s3, a3, b3, c3, s4, a4, b4, c4, s5, a5, b5, c5, s6, a6, b6, c6)   \
  EMG_##s6(EMG_##s5(EMG_##s4(EMG_##s3(EMG_##s2(EMG_M3(s1 a1, b1, c1), EMG_M3(a2, b2, c2)), EMG_M3(a3, b3, c3)),     \
                             EMG_M3(a4, b4, c4)),                                                                \
                    EMG_M3(a5, b5, c5)),                                                                         \
           EMG_M3(a6, b6, c6))
  ca[0] = EMG_T6(+, x2, y3, z4, S, x2, y4, z3, S, x3, y2, z4, A, x3, y4, z2, A, x4, y2, z3, S, x4, y3, z2);
  ca[1] = EMG_T6(-, x1, y3, z4, A, x1, y4, z3, A, x3, y1, z4, S, x3, y4, z1, S, x4, y1, z3, A, x4, y3, z1);
  ca[2] = EMG_T6(+, x1, y2, z4, S, x1, y4, z2, S, x2, y1, z4, A, x2, y4, z1, A, x4, y1, z2, S, x4, y2, z1);
  ca[3] = EMG_T6(-, x1, y2, z3, A, x1, y3, z2, A, x2, y1, z3, S, x2, y3, z1, S, x3, y1, z2, A, x3, y2, z1);
#undef EMG_T6
}


// vertex ranks by global id, and the canonical -> reference entity map
__device__ __forceinline__ bool ranks_and_map(const int64_t v[4], int rank[4], uint64_t &inv) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int r = 0;
#pragma unroll
    for (int p = 0; p < 4; ++p) r += (v[p] < v[q]) ? 1 : 0;
    rank[q] = r;
  }
  const bool distinct = (v[0] != v[1]) && (v[0] != v[2]) && (v[0] != v[3]) && (v[1] != v[2]) && (v[1] != v[3]) &&
                        (v[2] != v[3]);
  // reference edge slots (local vertex pairs) and the vertex missing from each face slot
  const int eu[6] = {0, 0, 0, 1, 3, 2}, ev[6] = {1, 2, 3, 2, 1, 3};
  const int fmiss[4] = {3, 1, 2, 0};
  uint64_t m = 0;
  if (distinct) {
#pragma unroll
    for (int s = 0; s < 6; ++s) m |= (uint64_t)s << (4 * canon_edge(rank[eu[s]], rank[ev[s]]));
#pragma unroll
    for (int f = 0; f < 4; ++f) m |= (uint64_t)(6 + f) << (4 * (6 + 3 - rank[fmiss[f]]));
  }
  inv = m;
  return distinct;
}

template <typename T>
__device__ __forceinline__ void scatter_rank(const T in[4], const int rank[4], T out[4]) {
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int r = 0; r < 4; ++r)
      if (rank[q] == r) out[r] = in[q];
}

}  // namespace

// the generated tables call emg_mac unqualified: include them inside emg
template <typename R>
struct CR {
  R re, im;
};
// Every multiply-add of the generated tables goes through rounding
// intrinsics, which the compiler neither re-associates nor re-contracts: the
// (x, y) and (y, x) entries, computed in different rows, are then bitwise
// equal, so the element blocks and A stay exactly symmetric.
__device__ __forceinline__ void emg_mac(double &acc, double a, double b) { acc = __fma_rn(a, b, acc); }
__device__ __forceinline__ void emg_mac(float &acc, double c, float v) { acc = __fmaf_rn((float)c, v, acc); }
__device__ __forceinline__ void emg_mac(float &acc, float a, float b) { acc = __fmaf_rn(a, b, acc); }
__device__ __forceinline__ void emg_mac(CR<double> &acc, double c, const CR<double> &v) {
  acc.re = __fma_rn(c, v.re, acc.re);
  acc.im = __fma_rn(c, v.im, acc.im);
}
__device__ __forceinline__ void emg_mac(CR<float> &acc, double c, const CR<float> &v) {
  acc.re = __fmaf_rn((float)c, v.re, acc.re);
  acc.im = __fmaf_rn((float)c, v.im, acc.im);
}
__device__ __forceinline__ void emg_mac(CR<double> &acc, const CR<double> &t, double w) {
  acc.re = __fma_rn(t.re, w, acc.re);
  acc.im = __fma_rn(t.im, w, acc.im);
}
__device__ __forceinline__ void emg_mac(CR<float> &acc, const CR<float> &t, float w) {
  acc.re = __fmaf_rn(t.re, w, acc.re);
  acc.im = __fmaf_rn(t.im, w, acc.im);
}
// inner moment sums of the generated tables: c0*mu0, then fma(c, mu, t)
__device__ __forceinline__ double emg_mul(double c, double m) { return __dmul_rn(c, m); }
__device__ __forceinline__ float emg_mul(double c, float m) { return __fmul_rn((float)c, m); }
__device__ __forceinline__ double emg_fma(double t, double c, double m) { return __fma_rn(c, m, t); }
__device__ __forceinline__ float emg_fma(float t, double c, float m) { return __fmaf_rn((float)c, m, t); }
#include "nedelec_moment_tables.cuh"
#include "nedelec_tables.cuh"

namespace {

constexpr int NMOM = emg_mtables::kNumMoments;

// Reference forms: coefficients, quadrature points and L~ exactly as the
// reference computes them, then the quadrature moments. Returns false for a
// degenerate tet.
template <typename R>
__device__ __forceinline__ bool ref_geometry(const double X[3][4], const int64_t v[4], Geo &G, R mu[NMOM]) {
  int rank[4];
  uint64_t inv;
  const bool distinct = ranks_and_map(v, rank, inv);
  double ca[4], cb[4], cc[4], cd[4], det;
  ref_coefficients(X, ca, cb, cc, cd, det);
  if (!distinct || !(det != 0.0) || !isfinite(det)) return false;
  const double V = fabs(det) / 6.0;
  const double six_v = __dmul_rn(6.0, V);
  double a[4], b[4], c[4], d[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    a[q] = ca[q] / six_v;
    b[q] = cb[q] / six_v;
    c[q] = cc[q] / six_v;
    d[q] = cd[q] / six_v;
  }
  double br[4], cr[4], dr[4];
  scatter_rank(b, rank, br);
  scatter_rank(c, rank, cr);
  scatter_rank(d, rank, dr);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    G.g[r][0] = br[r];
    G.g[r][1] = cr[r];
    G.g[r][2] = dr[r];
  }
  G.V = V;
  G.sig = 1.0;
  G.inv = inv;
#pragma unroll
  for (int i = 0; i < NMOM; ++i) mu[i] = (R)0;
  // rolled on purpose: the kernel is instruction-fetch bound, and the point
  // loop body is the same for all 11 points
#pragma unroll 1
  for (int q = 0; q < 11; ++q) {
    const double p1 = kDP[1][q], p2 = kDP[2][q], p3 = kDP[3][q], p4 = kDP[4][q];
    double xq[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
      xq[k] = EMG_A(EMG_A(EMG_A(EMG_M2(X[k][0], p1), EMG_M2(X[k][1], p2)), EMG_M2(X[k][2], p3)), EMG_M2(X[k][3], p4));
    double L[4];
#pragma unroll
    for (int m = 0; m < 4; ++m)
      L[m] = EMG_A(EMG_A(EMG_A(a[m], EMG_M2(b[m], xq[0])), EMG_M2(c[m], xq[1])), EMG_M2(d[m], xq[2]));
    double Lr[4];
    scatter_rank(L, rank, Lr);
    R Lq[4] = {(R)Lr[0], (R)Lr[1], (R)Lr[2], (R)Lr[3]};
    emg_mtables::emg_moments<R>(Lq, (R)kDP[0][q], mu);
  }
  return true;
}

// Exact form: accurate gradients from edge vectors (relative to vertex 0).
__device__ __forceinline__ bool exact_geometry(const double X[3][4], const int64_t v[4], Geo &G) {
  int rank[4];
  uint64_t inv;
  const bool distinct = ranks_and_map(v, rank, inv);
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
  const double id = 1.0 / det;
  double gx[4], gy[4], gz[4];
  gx[1] = c23[0] * id, gy[1] = c23[1] * id, gz[1] = c23[2] * id;
  gx[2] = c31[0] * id, gy[2] = c31[1] * id, gz[2] = c31[2] * id;
  gx[3] = c12[0] * id, gy[3] = c12[1] * id, gz[3] = c12[2] * id;
  gx[0] = -(gx[1] + gx[2] + gx[3]);
  gy[0] = -(gy[1] + gy[2] + gy[3]);
  gz[0] = -(gz[1] + gz[2] + gz[3]);
  double rx[4], ry[4], rz[4];
  scatter_rank(gx, rank, rx);
  scatter_rank(gy, rank, ry);
  scatter_rank(gz, rank, rz);
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    G.g[r][0] = rx[r];
    G.g[r][1] = ry[r];
    G.g[r][2] = rz[r];
  }
  G.V = fabs(det) / 6.0;
  G.sig = det > 0.0 ? 1.0 : -1.0;
  G.inv = inv;
  return true;
}

// reference DoF index (0..19) of canonical DoF y
__device__ __forceinline__ int ref_dof(uint64_t inv, int y) {
  int c = y < 6 ? y : (y < 12 ? y - 6 : (y < 16 ? y - 6 : y - 10));  // canonical entity 0..9
  int s = (int)((inv >> (4 * c)) & 15ull);                             // reference entity slot 0..9
  return y < 6 ? s : (y < 12 ? 6 + s : (y < 16 ? 12 + (s - 6) : 16 + (s - 6)));
}

// Per-tet tensors, V folded in: G[m][n] = V (eps g_m).g_n, H[P][Q] = V (mu^-1 X_P).X_Q.
// ISO: real (material scalars applied per entry); DIAG symmetric / FULL general: complex.
template <int KIND, typename R>
struct Tensors {
  CR<R> G[4][4], H[6][6];
};
template <typename R>
struct Tensors<EMG_MAT_ISO, R> {
  R G[4][4], H[6][6];
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

// complex tensors: eps, minv are 3x3 row-major complex; (A u).w = sum_r w_r sum_c A[r][c] u_c
template <int KIND, typename R>
__device__ __forceinline__ void build_cplx(const Geo &Gm, const C64 eps[9], const C64 minv[9], Tensors<KIND, R> &T) {
  double X[6][3];
  const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {1, 2, 3, 2, 3, 3};
#pragma unroll
  for (int p = 0; p < 6; ++p) cross3(Gm.g[pa[p]], Gm.g[pb[p]], X[p]);
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

template <int KIND, typename R>
struct EntryT {
  using T = CR<R>;
};
template <typename R>
struct EntryT<EMG_MAT_ISO, R> {
  using T = R;
};

template <typename A>
__device__ __forceinline__ void scale_sign(A &x, double s);
template <>
__device__ __forceinline__ void scale_sign(double &x, double s) { x *= s; }
template <>
__device__ __forceinline__ void scale_sign(float &x, double s) { x *= (float)s; }
template <>
__device__ __forceinline__ void scale_sign(CR<double> &x, double s) { x.re *= s, x.im *= s; }
template <>
__device__ __forceinline__ void scale_sign(CR<float> &x, double s) { x.re *= (float)s, x.im *= (float)s; }

// entry (first=f, second=s) of K and M in the canonical frame
template <int f, int s, int FORM, int KIND, typename R>
__device__ __forceinline__ void entry(const Tensors<KIND, R> &T, const R *mu, double sig,
                                      typename EntryT<KIND, R>::T &k, typename EntryT<KIND, R>::T &m) {
  using E = typename EntryT<KIND, R>::T;
  E ak{}, am{};
  if constexpr (FORM != FORM_REF64) {
    emg_tables::Pair<f, s>::stiff(ak, T.H);
    emg_tables::Pair<f, s>::mass(am, T.G);
    if (emg_tables::odd(f) != emg_tables::odd(s)) {
      scale_sign(ak, sig);
      scale_sign(am, sig);
    }
  } else {
    emg_mtables::MPair<f, s>::stiff(ak, T.H, mu);
    emg_mtables::MPair<f, s>::mass(am, T.G, mu);
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

__device__ __forceinline__ double cfma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float cfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double cmul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float cmul_rn(float a, float b) { return __fmul_rn(a, b); }

template <int x, int y, int FORM, int KIND, typename R>
__device__ __forceinline__ void compute_store(const Tensors<KIND, R> &T, const R *mu, double sig, const CR<R> &cK,
                                              const CR<R> &cM, uint64_t inv, int rx, typename StoreT<R>::T *row) {
  using ST = typename StoreT<R>::T;
  const int b = ref_dof(inv, y);
  ST v;
  if constexpr (KIND == EMG_MAT_ISO) {
    R k0, m0;
    entry<(x < y ? x : y), (x < y ? y : x), FORM, KIND, R>(T, mu, sig, k0, m0);
    v.x = cfma(cK.re, k0, cmul_rn(cM.re, m0));
    v.y = cfma(cK.im, k0, cmul_rn(cM.im, m0));
  } else {
    CR<R> k, m;
    if constexpr (KIND == EMG_MAT_DIAG) {
      entry<(x < y ? x : y), (x < y ? y : x), FORM, KIND, R>(T, mu, sig, k, m);
    } else {
      // first = the DoF with the lower reference index (curlcurl.py:358-376)
      if (rx <= b) {
        entry<x, y, FORM, KIND, R>(T, mu, sig, k, m);
      } else {
        entry<y, x, FORM, KIND, R>(T, mu, sig, k, m);
      }
    }
    v.x = cfma(cK.re, k.re, cfma(-cK.im, k.im, cfma(cM.re, m.re, cmul_rn(-cM.im, m.im))));
    v.y = cfma(cK.re, k.im, cfma(cK.im, k.re, cfma(cM.re, m.im, cmul_rn(cM.im, m.re))));
  }
  row[b] = v;
}

template <int x, int FORM, int KIND, typename R, int... Ys>
__device__ __forceinline__ void compute_row(const Tensors<KIND, R> &T, const R *mu, double sig, const CR<R> &cK,
                                            const CR<R> &cM, uint64_t inv, int rx, typename StoreT<R>::T *row,
                                            std::integer_sequence<int, Ys...>) {
  (compute_store<x, Ys, FORM, KIND, R>(T, mu, sig, cK, cM, inv, rx, row), ...);
}

template <int FORM, int KIND, typename R, int X>
__device__ __forceinline__ void do_row(const Tensors<KIND, R> &T, const R *mu, double sig, const CR<R> &cK,
                                       const CR<R> &cM, uint64_t inv, bool active, int ia,
                                       typename StoreT<R>::T *stage, typename StoreT<R>::T *out) {
  const int lane = threadIdx.x & 31;
  const int rx = ref_dof(inv, X);
  if (active)
    compute_row<X, FORM, KIND, R>(T, mu, sig, cK, cM, inv, rx, stage + lane * 21,
                                  std::make_integer_sequence<int, 20>{});
  __syncwarp();
  // cooperative, coalesced write of the warp's 32 rows (each 20 contiguous values)
#pragma unroll 1
  for (int it = 0; it < 20; ++it) {
    int e = it * 32 + lane;
    int r = e / 20, c = e - r * 20;
    int ia_r = __shfl_sync(0xffffffffu, ia, r);
    int a_r = __shfl_sync(0xffffffffu, rx, r);
    bool act_r = __shfl_sync(0xffffffffu, (int)active, r);
    if (act_r) out[(int64_t)ia_r * 400 + a_r * 20 + c] = stage[r * 21 + c];
  }
  __syncwarp();
}

template <int FORM, int KIND, typename R, int... Xs>
__device__ __forceinline__ void all_rows(const Tensors<KIND, R> &T, const R *mu, double sig, const CR<R> &cK,
                                         const CR<R> &cM, uint64_t inv, bool active, int ia,
                                         typename StoreT<R>::T *stage, typename StoreT<R>::T *out,
                                         std::integer_sequence<int, Xs...>) {
  (do_row<FORM, KIND, R, Xs>(T, mu, sig, cK, cM, inv, active, ia, stage, out), ...);
}

// ---- packed canonical layout: value[ia*210 + packed_index(x, y)], x <= y,
// canonical DoFs. Each unique pair is computed once; canonical row X (its
// 20 - X upper-triangle entries) is staged in shared memory and the warp
// writes its 32 row segments as contiguous runs.
template <int x, int y, int FORM, int KIND, typename R>
__device__ __forceinline__ void compute_store_packed(const Tensors<KIND, R> &T, const R *mu, double sig,
                                                     const CR<R> &cK, const CR<R> &cM, uint64_t inv,
                                                     typename StoreT<R>::T *row) {
  using ST = typename StoreT<R>::T;
  ST v;
  if constexpr (KIND == EMG_MAT_ISO) {
    R k0, m0;
    entry<x, y, FORM, KIND, R>(T, mu, sig, k0, m0);
    v.x = cfma(cK.re, k0, cmul_rn(cM.re, m0));
    v.y = cfma(cK.im, k0, cmul_rn(cM.im, m0));
  } else {
    CR<R> k, m;
    if constexpr (KIND == EMG_MAT_DIAG) {
      entry<x, y, FORM, KIND, R>(T, mu, sig, k, m);
    } else {
      // first = the DoF with the lower reference index (curlcurl.py:358-376)
      if (ref_dof(inv, x) <= ref_dof(inv, y)) {
        entry<x, y, FORM, KIND, R>(T, mu, sig, k, m);
      } else {
        entry<y, x, FORM, KIND, R>(T, mu, sig, k, m);
      }
    }
    v.x = cfma(cK.re, k.re, cfma(-cK.im, k.im, cfma(cM.re, m.re, cmul_rn(-cM.im, m.im))));
    v.y = cfma(cK.re, k.im, cfma(cK.im, k.re, cfma(cM.re, m.im, cmul_rn(cM.im, m.re))));
  }
  row[y - x] = v;
}

template <int x, int FORM, int KIND, typename R, int... Ds>
__device__ __forceinline__ void compute_row_packed(const Tensors<KIND, R> &T, const R *mu, double sig,
                                                   const CR<R> &cK, const CR<R> &cM, uint64_t inv,
                                                   typename StoreT<R>::T *row, std::integer_sequence<int, Ds...>) {
  (compute_store_packed<x, x + Ds, FORM, KIND, R>(T, mu, sig, cK, cM, inv, row), ...);
}

template <int FORM, int KIND, typename R, int X>
__device__ __forceinline__ void do_row_packed(const Tensors<KIND, R> &T, const R *mu, double sig, const CR<R> &cK,
                                              const CR<R> &cM, uint64_t inv, bool active, int ia,
                                              typename StoreT<R>::T *stage, typename StoreT<R>::T *out) {
  constexpr int W = 20 - X;
  const int lane = threadIdx.x & 31;
  if (active)
    compute_row_packed<X, FORM, KIND, R>(T, mu, sig, cK, cM, inv, stage + lane * (W | 1),
                                         std::make_integer_sequence<int, W>{});
  // the warp's 32 tets are consecutive assembled indices: lane r's is ia - lane + r
  const unsigned act = __ballot_sync(0xffffffffu, active);
  const int64_t ia_w = (int64_t)ia - lane;
  __syncwarp();
#pragma unroll 2
  for (int it = 0; it < W; ++it) {
    const int e = it * 32 + lane;
    const int r = e / W, c = e - r * W;
    if ((act >> r) & 1u) out[(ia_w + r) * 210 + packed_index(X, X) + c] = stage[r * (W | 1) + c];
  }
  __syncwarp();
}

template <int FORM, int KIND, typename R, int... Xs>
__device__ __forceinline__ void all_rows_packed(const Tensors<KIND, R> &T, const R *mu, double sig, const CR<R> &cK,
                                                const CR<R> &cM, uint64_t inv, bool active, int ia,
                                                typename StoreT<R>::T *stage, typename StoreT<R>::T *out,
                                                std::integer_sequence<int, Xs...>) {
  (do_row_packed<FORM, KIND, R, Xs>(T, mu, sig, cK, cM, inv, active, ia, stage, out), ...);
}

// ---- entity-pair block layout: value[ia*220 + 4*block_index(i, j) + k] for
// canonical entities i <= j. Block row i (its 10 - i blocks, 4 values each)
// is staged in shared memory and the warp writes its 32 block rows as
// contiguous runs. Each value is the packed layout's (min, max) entry.
template <int x, int y, int FORM, int KIND, typename R>
__device__ __forceinline__ void compute_store_any(const Tensors<KIND, R> &T, const R *mu, double sig, const CR<R> &cK,
                                                  const CR<R> &cM, uint64_t inv, typename StoreT<R>::T *dst) {
  constexpr int lo = x < y ? x : y, hi = x < y ? y : x;
  compute_store_packed<lo, hi, FORM, KIND, R>(T, mu, sig, cK, cM, inv, dst - (hi - lo));
}

template <int i, int FORM, int KIND, typename R, int... Js>
__device__ __forceinline__ void compute_block_row(const Tensors<KIND, R> &T, const R *mu, double sig,
                                                  const CR<R> &cK, const CR<R> &cM, uint64_t inv,
                                                  typename StoreT<R>::T *row, std::integer_sequence<int, Js...>) {
  // the first DoF's entries of the block row, then the second's (row order of the packed triangle)
  ((compute_store_any<ent_dof1(i), ent_dof1(i + Js), FORM, KIND, R>(T, mu, sig, cK, cM, inv, row + 4 * Js + 0),
    compute_store_any<ent_dof1(i), ent_dof2(i + Js), FORM, KIND, R>(T, mu, sig, cK, cM, inv, row + 4 * Js + 1)),
   ...);
  ((compute_store_any<ent_dof2(i), ent_dof1(i + Js), FORM, KIND, R>(T, mu, sig, cK, cM, inv, row + 4 * Js + 2),
    compute_store_any<ent_dof2(i), ent_dof2(i + Js), FORM, KIND, R>(T, mu, sig, cK, cM, inv, row + 4 * Js + 3)),
   ...);
}

template <int FORM, int KIND, typename R, int I>
__device__ __forceinline__ void do_row_block(const Tensors<KIND, R> &T, const R *mu, double sig, const CR<R> &cK,
                                             const CR<R> &cM, uint64_t inv, bool active, int ia,
                                             typename StoreT<R>::T *stage, typename StoreT<R>::T *out) {
  constexpr int W = 4 * (10 - I);
  const int lane = threadIdx.x & 31;
  if (active)
    compute_block_row<I, FORM, KIND, R>(T, mu, sig, cK, cM, inv, stage + lane * (W | 1),
                                        std::make_integer_sequence<int, 10 - I>{});
  // the warp's 32 tets are consecutive assembled indices: lane r's is ia - lane + r
  const unsigned act = __ballot_sync(0xffffffffu, active);
  const int64_t ia_w = (int64_t)ia - lane;
  __syncwarp();
#pragma unroll 2
  for (int it = 0; it < W; ++it) {
    const int e = it * 32 + lane;
    const int r = e / W, c = e - r * W;
    if ((act >> r) & 1u) out[(ia_w + r) * kBlockValues + 4 * block_index(I, I) + c] = stage[r * (W | 1) + c];
  }
  __syncwarp();
}

template <int FORM, int KIND, typename R, int... Is>
__device__ __forceinline__ void all_rows_block(const Tensors<KIND, R> &T, const R *mu, double sig, const CR<R> &cK,
                                               const CR<R> &cM, uint64_t inv, bool active, int ia,
                                               typename StoreT<R>::T *stage, typename StoreT<R>::T *out,
                                               std::integer_sequence<int, Is...>) {
  (do_row_block<FORM, KIND, R, Is>(T, mu, sig, cK, cM, inv, active, ia, stage, out), ...);
}

// LAYOUT 0: the reference's COO block [ia][a][b] (400 values, each entry
//           computed in both of its rows);
// LAYOUT 1: the packed canonical upper triangle [ia][210] (each unique
//           entry computed once);
// LAYOUT 2: the entity-pair blocks [ia][220] (the assembly path)
// One CTA's 128 tets, assembled indices ia0 .. ia0 + 127 of the job a (every
// thread of the CTA calls it with the same ia0).
template <int FORM, int KIND, int LAYOUT>
__device__ __forceinline__ void element_cta(const ElemArgs &a, int64_t ia0, unsigned char *stage_raw) {
  using R = typename FormReal<FORM>::T;
  using ST = typename StoreT<R>::T;
  // values per lane: a row's stride is odd (in values), so the 32 lanes'
  // stores of one value position fall in distinct shared-memory bank groups
  constexpr int STAGE = LAYOUT == 2 ? 41 : 21;
  ST *stage = reinterpret_cast<ST *>(stage_raw) + (threadIdx.x >> 5) * (32 * STAGE);
  ST *out = reinterpret_cast<ST *>(a.out);
  const int64_t ia64 = ia0 + threadIdx.x;
  bool active = ia64 < a.nA;
  const int ia = (int)ia64;
  Geo G;
  Tensors<KIND, R> T;
  R mu[FORM == FORM_REF64 ? NMOM : 1];
  CR<R> cK{0, 0}, cM{0, 0};
  double sig = 1.0;
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
      bool good;
      if constexpr (FORM != FORM_REF64) {
        good = exact_geometry(X, v, G);
      } else {
        good = ref_geometry<R>(X, v, G, mu);
      }
      if (!good) {
        flag(a.st, EMG_ST_DEGENERATE, ia64);
        active = false;
      } else {
        sig = G.sig;
        inv = G.inv;
        const C64 alpha{a.ar, a.ai}, beta{a.br, a.bi};
        if constexpr (KIND == EMG_MAT_ISO) {
          C64 eps = ld_c64(a.er, it);
          C64 minv = a.ur ? crecip(ld_c64(a.ur, it)) : C64{1.0, 0.0};
          C64 k = cmul(alpha, minv), m = cmul(beta, eps);
          cK = {(R)k.re, (R)k.im};
          cM = {(R)m.re, (R)m.im};
          build_iso<R>(G, T);
        } else {
          C64 eps[9], mu3[9], minv[9];
#pragma unroll
          for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              // DIAG: compact diagonals [3][nT]; FULL: the reference's [3][3][nT]
              const bool need = (KIND == EMG_MAT_FULL) || r == c;
              const int64_t o = (KIND == EMG_MAT_FULL) ? (int64_t)(3 * r + c) * a.nT + it : (int64_t)r * a.nT + it;
              eps[3 * r + c] = need ? ld_c64(a.er, o) : C64{0.0, 0.0};
              mu3[3 * r + c] = (need && a.ur) ? ld_c64(a.ur, o) : C64{(r == c) ? 1.0 : 0.0, 0.0};
            }
          matinv3(mu3, minv);
          cK = {(R)alpha.re, (R)alpha.im};
          cM = {(R)beta.re, (R)beta.im};
          build_cplx<KIND, R>(G, eps, minv, T);
        }
      }
    }
  }
  if constexpr (LAYOUT == 0) {
    all_rows<FORM, KIND, R>(T, mu, sig, cK, cM, inv, active, ia, stage, out, std::make_integer_sequence<int, 20>{});
  } else if constexpr (LAYOUT == 2) {
    all_rows_block<FORM, KIND, R>(T, mu, sig, cK, cM, inv, active, ia, stage, out,
                                  std::make_integer_sequence<int, 10>{});
  } else {
    all_rows_packed<FORM, KIND, R>(T, mu, sig, cK, cM, inv, active, ia, stage, out,
                                   std::make_integer_sequence<int, 20>{});
  }
}

// CTAs per SM the compiler must fit. Measured on the 2.01M-tet box: the
// FP64 forms at their natural 242-255 registers (two CTAs) beat every cap (a
// three-CTA cap: 1.84 -> 3.68 ms, 1.9 KB of spills); the mixed form needs 88-254
// registers with no cap (five CTAs per SM for the isotropic instance, set by
// its 42 KB stage as much as by registers).
template <int FORM, int KIND>
constexpr int elem_min_blocks() {
  return 1;
}

template <int FORM, int KIND, int LAYOUT>
__global__ void __launch_bounds__(ELEM_THREADS, elem_min_blocks<FORM, KIND>()) k_element(ElemArgs a) {
  extern __shared__ __align__(16) unsigned char stage_raw[];
  element_cta<FORM, KIND, LAYOUT>(a, (int64_t)blockIdx.x * ELEM_THREADS, stage_raw);
}

// Several jobs (meshes, materials, coefficients, outputs) in one launch of
// the packed form: job j owns the CTAs [cta_start[j], cta_start[j + 1]) and
// its tets in CTA order, as if launched alone.
template <int FORM, int KIND, int LAYOUT>
__global__ void __launch_bounds__(ELEM_THREADS, elem_min_blocks<FORM, KIND>())
    k_element_batch(const ElemArgs *jobs, const int64_t *cta_start, int n_jobs) {
  extern __shared__ __align__(16) unsigned char stage_raw[];
  const int64_t b = blockIdx.x;
  int lo = 0, hi = n_jobs - 1;  // the job with cta_start[j] <= b < cta_start[j + 1]
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cta_start[mid] <= b) lo = mid;
    else hi = mid - 1;
  }
  if (n_jobs <= 0 || b >= cta_start[n_jobs]) return;
  element_cta<FORM, KIND, LAYOUT>(jobs[lo], (b - cta_start[lo]) * ELEM_THREADS, stage_raw);
}

template <int FORM, int KIND, int LAYOUT>
int launch_element_t(const ElemArgs &a, cudaStream_t s) {
  using ST = typename StoreT<typename FormReal<FORM>::T>::T;
  constexpr size_t smem = (size_t)ELEM_WARPS * 32 * (LAYOUT == 2 ? 41 : 21) * sizeof(ST);
  // the attribute belongs to the current device: set once per device (benign
  // race: every thread that gets here sets the same value)
  static bool configured[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) dev = 0;
  if (dev >= 64 || !configured[dev]) {
    cudaError_t e = cudaFuncSetAttribute(k_element<FORM, KIND, LAYOUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return fail(EMG_ECUDA, "cudaFuncSetAttribute(k_element): %s", cudaGetErrorString(e));
    if (dev < 64) configured[dev] = true;
  }
  if (a.nA == 0) return EMG_OK;
  k_element<FORM, KIND, LAYOUT><<<grid_for(a.nA, ELEM_THREADS), ELEM_THREADS, smem, s>>>(a);
  return launch_check("k_element");
}

template <int FORM, int KIND, int LAYOUT>
int launch_element_batch_t(const ElemArgs *d_jobs, const int64_t *d_cta_start, int n_jobs, int64_t total_ctas,
                           cudaStream_t s) {
  using ST = typename StoreT<typename FormReal<FORM>::T>::T;
  constexpr size_t smem = (size_t)ELEM_WARPS * 32 * (LAYOUT == 2 ? 41 : 21) * sizeof(ST);  // element_cta's stage
  static bool configured[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) dev = 0;
  if (dev >= 64 || !configured[dev]) {
    cudaError_t e =
        cudaFuncSetAttribute(k_element_batch<FORM, KIND, LAYOUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return fail(EMG_ECUDA, "cudaFuncSetAttribute(k_element_batch): %s", cudaGetErrorString(e));
    if (dev < 64) configured[dev] = true;
  }
  if (n_jobs == 0 || total_ctas == 0) return EMG_OK;
  if (total_ctas > INT32_MAX) return fail(EMG_ERANGE, "too many CTAs (%lld)", (long long)total_ctas);
  k_element_batch<FORM, KIND, LAYOUT><<<(unsigned)total_ctas, ELEM_THREADS, smem, s>>>(d_jobs, d_cta_start,
                                                                                       n_jobs);
  return launch_check("k_element_batch");
}

template <int FORM, int KIND>
int launch_element_k(const ElemArgs &a, int layout, cudaStream_t s) {
  if (layout == EMG_LAYOUT_COO) return launch_element_t<FORM, KIND, 0>(a, s);
  if (layout == EMG_LAYOUT_PACKED) return launch_element_t<FORM, KIND, 1>(a, s);
  if (layout == EMG_LAYOUT_BLOCK) return launch_element_t<FORM, KIND, 2>(a, s);
  return fail(EMG_EINVAL, "bad layout %d", layout);
}

}  // namespace
}  // namespace emg
