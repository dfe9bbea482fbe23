// heat.cu -- Lagrange-2 heat-conduction element kernels: per tet the 10x10
// stiffness block (k grad N_i) . grad N_j and capacity block rho_cp N_i N_j
// (leg2_tet_stiff / leg2_tet_mass and their COO builders,
// physics/heatconduction/assembly/grad.py:199-400).
//
// Two forms.
//  * EMG_FP64: the reference's quadrature loop, expression for expression
//    (built with -fmad=false). Ten threads share a tet, one per basis
//    function: each evaluates its function's gradient (or value) at the 11
//    points once into shared memory, then forms its row of the block from
//    them -- the same operations per entry as the reference, which
//    re-evaluates both gradients for every entry.
//  * EMG_EXACT: the same rule folded into moments. Every gradient is linear
//    in the barycentrics, so K_ij is a fixed combination of the 16 products
//    S_pq = (k grad lam_p) . grad lam_q and the capacity block is rho_cp V
//    times a constant 10x10 matrix; the tables come from the same 8-digit
//    rule. Translation invariant (edge vectors), no cancellation in lam.
// In the fp64 form the basis values and gradients, where the reference's
// arithmetic cancels, are formed without fused multiply-adds; the sums that
// form an entry from them use fma (rounding-level differences only).
// Both stage a block's output in shared memory and store it coalesced, in
// the reference's row-major block (EMG_LAYOUT_COO) or transposed per tet
// (EMG_LAYOUT_COO_T: the 10 values of one column of one tet contiguous,
// which is what the COO -> CSC gather reads together).
#include "common.cuh"

namespace emg {
namespace {

// the 11-point rule with the reference's 8-digit weights and points
// (grad.py:177-188): row 0 weights, rows 1-4 barycentric coordinates
#define EMG_HEAT_W                                                                                                   \
  {-0.078933, 0.04573333, 0.04573333, 0.04573333, 0.04573333, 0.14933333, 0.14933333, 0.14933333, 0.14933333,       \
   0.14933333, 0.14933333}
#define EMG_HEAT_P                                                                                                   \
  {{0.25, 0.78571429, 0.07142857, 0.07142857, 0.07142857, 0.39940358, 0.39940358, 0.39940358, 0.10059642,           \
    0.10059642, 0.10059642},                                                                                         \
   {0.25, 0.07142857, 0.07142857, 0.07142857, 0.78571429, 0.10059642, 0.10059642, 0.39940358, 0.39940358,           \
    0.39940358, 0.10059642},                                                                                         \
   {0.25, 0.07142857, 0.07142857, 0.78571429, 0.07142857, 0.39940358, 0.10059642, 0.10059642, 0.39940358,           \
    0.10059642, 0.39940358},                                                                                         \
   {0.25, 0.07142857, 0.78571429, 0.07142857, 0.07142857, 0.10059642, 0.39940358, 0.10059642, 0.10059642,           \
    0.39940358, 0.39940358}}
__constant__ double kHW[11] = EMG_HEAT_W;
__constant__ double kHP[4][11] = EMG_HEAT_P;
static const double hHW[11] = EMG_HEAT_W;
static const double hHP[4][11] = EMG_HEAT_P;
// LOCAL_EDGE_MAP (grad.py:175)
__constant__ int kLEM[2][6] = {{0, 0, 0, 1, 1, 2}, {1, 2, 3, 2, 3, 3}};
static const int hLEM[2][6] = {{0, 0, 0, 1, 1, 2}, {1, 2, 3, 2, 3, 3}};

constexpr int kFp64Tets = 16;                 // tets per block, fp64 form
constexpr int kFp64Threads = kFp64Tets * 10;  // one thread per basis function
constexpr int kExactTets = 32;                // tets (threads) per block, exact form

__device__ __forceinline__ bool leg2_load(const double *nodes, int64_t nN, const int32_t *tets, int64_t nT, int64_t t,
                                          double X[3][4]) {
  bool ok = true;
  for (int v = 0; v < 4; ++v) {
    const int64_t n = tets[v * nT + t];
    const bool in = n >= 0 && n < nN;
    ok = ok && in;
    for (int d = 0; d < 3; ++d) X[d][v] = in ? nodes[d * nN + n] : 0.0;
  }
  return ok;
}

// tet_coefficients (grad.py:64-128): the volume ...
__device__ double leg2_volume(const double X[3][4]) {
  const double x1 = X[0][0], x2 = X[0][1], x3 = X[0][2], x4 = X[0][3];
  const double y1 = X[1][0], y2 = X[1][1], y3 = X[1][2], y4 = X[1][3];
  const double z1 = X[2][0], z2 = X[2][1], z3 = X[2][2], z4 = X[2][3];
  return fabs(-x1 * y2 * z3 / 6 + x1 * y2 * z4 / 6 + x1 * y3 * z2 / 6 - x1 * y3 * z4 / 6 - x1 * y4 * z2 / 6 +
              x1 * y4 * z3 / 6 + x2 * y1 * z3 / 6 - x2 * y1 * z4 / 6 - x2 * y3 * z1 / 6 + x2 * y3 * z4 / 6 +
              x2 * y4 * z1 / 6 - x2 * y4 * z3 / 6 - x3 * y1 * z2 / 6 + x3 * y1 * z4 / 6 + x3 * y2 * z1 / 6 -
              x3 * y2 * z4 / 6 - x3 * y4 * z1 / 6 + x3 * y4 * z2 / 6 + x4 * y1 * z2 / 6 - x4 * y1 * z3 / 6 -
              x4 * y2 * z1 / 6 + x4 * y2 * z3 / 6 + x4 * y3 * z1 / 6 - x4 * y3 * z2 / 6);
}

// ... and column m of (aas, bbs, ccs, dds), before the division by 6V
__device__ void leg2_column_raw(const double X[3][4], int m, double c[4]) {
  const double x1 = X[0][0], x2 = X[0][1], x3 = X[0][2], x4 = X[0][3];
  const double y1 = X[1][0], y2 = X[1][1], y3 = X[1][2], y4 = X[1][3];
  const double z1 = X[2][0], z2 = X[2][1], z3 = X[2][2], z4 = X[2][3];
  switch (m) {
    case 0:
      c[0] = x2 * y3 * z4 - x2 * y4 * z3 - x3 * y2 * z4 + x3 * y4 * z2 + x4 * y2 * z3 - x4 * y3 * z2;
      c[1] = -y2 * z3 + y2 * z4 + y3 * z2 - y3 * z4 - y4 * z2 + y4 * z3;
      c[2] = x2 * z3 - x2 * z4 - x3 * z2 + x3 * z4 + x4 * z2 - x4 * z3;
      c[3] = -x2 * y3 + x2 * y4 + x3 * y2 - x3 * y4 - x4 * y2 + x4 * y3;
      break;
    case 1:
      c[0] = -x1 * y3 * z4 + x1 * y4 * z3 + x3 * y1 * z4 - x3 * y4 * z1 - x4 * y1 * z3 + x4 * y3 * z1;
      c[1] = y1 * z3 - y1 * z4 - y3 * z1 + y3 * z4 + y4 * z1 - y4 * z3;
      c[2] = -x1 * z3 + x1 * z4 + x3 * z1 - x3 * z4 - x4 * z1 + x4 * z3;
      c[3] = x1 * y3 - x1 * y4 - x3 * y1 + x3 * y4 + x4 * y1 - x4 * y3;
      break;
    case 2:
      c[0] = x1 * y2 * z4 - x1 * y4 * z2 - x2 * y1 * z4 + x2 * y4 * z1 + x4 * y1 * z2 - x4 * y2 * z1;
      c[1] = -y1 * z2 + y1 * z4 + y2 * z1 - y2 * z4 - y4 * z1 + y4 * z2;
      c[2] = x1 * z2 - x1 * z4 - x2 * z1 + x2 * z4 + x4 * z1 - x4 * z2;
      c[3] = -x1 * y2 + x1 * y4 + x2 * y1 - x2 * y4 - x4 * y1 + x4 * y2;
      break;
    default:
      c[0] = -x1 * y2 * z3 + x1 * y3 * z2 + x2 * y1 * z3 - x2 * y3 * z1 - x3 * y1 * z2 + x3 * y2 * z1;
      c[1] = y1 * z2 - y1 * z3 - y2 * z1 + y2 * z3 + y3 * z1 - y3 * z2;
      c[2] = -x1 * z2 + x1 * z3 + x2 * z1 - x2 * z3 - x3 * z1 + x3 * z2;
      c[3] = x1 * y2 - x1 * y3 - x2 * y1 + x2 * y3 + x3 * y1 - x3 * y2;
      break;
  }
}

__device__ __forceinline__ void quad_point(const double X[3][4], int q, double &x, double &y, double &z) {
  x = X[0][0] * kHP[0][q] + X[0][1] * kHP[1][q] + X[0][2] * kHP[2][q] + X[0][3] * kHP[3][q];
  y = X[1][0] * kHP[0][q] + X[1][1] * kHP[1][q] + X[1][2] * kHP[2][q] + X[1][3] * kHP[3][q];
  z = X[2][0] * kHP[0][q] + X[2][1] * kHP[1][q] + X[2][2] * kHP[2][q] + X[2][3] * kHP[3][q];
}

// stage -> global: the block's tets are contiguous in the output
__device__ __forceinline__ void store_block(const double *stage, int64_t t0, int64_t nT, int per_block,
                                            double *out) {
  const int64_t n = min((int64_t)per_block, nT - t0) * 100;
  double *o = out + t0 * 100;
  for (int k = threadIdx.x; k < n; k += blockDim.x) o[k] = stage[k];
}

// The 24 terms of the reference's volume expression (grad.py:76-101), in its
// order: sign, and the vertices of the x, y and z factors. The sum is taken
// left to right over sign * ((x * y) * z) / 6, as the expression parses.
__constant__ signed char kVolTerm[24][4] = {
    {-1, 0, 1, 2}, {1, 0, 1, 3}, {1, 0, 2, 1}, {-1, 0, 2, 3}, {-1, 0, 3, 1}, {1, 0, 3, 2},
    {1, 1, 0, 2},  {-1, 1, 0, 3}, {-1, 1, 2, 0}, {1, 1, 2, 3},  {1, 1, 3, 0},  {-1, 1, 3, 2},
    {-1, 2, 0, 1}, {1, 2, 0, 3}, {1, 2, 1, 0},  {-1, 2, 1, 3}, {-1, 2, 3, 0}, {1, 2, 3, 1},
    {1, 3, 0, 1},  {-1, 3, 0, 2}, {-1, 3, 1, 0}, {1, 3, 1, 2},  {1, 3, 2, 0},  {-1, 3, 2, 1}};

// What the ten threads of a tet share: coeff = (aas, bbs, ccs, dds) / (6V)
// (grad.py:217-221), the 11 quadrature points (xs, ys, zs) and V. Each value
// is formed once, by the reference's expression: the volume's 24 divided
// terms and the 16 divisions by 6V are spread over the ten threads, the
// volume summed in the expression's order by one of them.
struct TetShared {
  double co[4][4];  // co[r][m]: row r (a, b, c, d) of vertex m; raw (undivided) until the last step
  double pt[11][3];
  double V;
  int ok;
};

// scratch: 24 doubles per tet of the block, free again when this returns
__device__ void fp64_prologue(const double *nodes, int64_t nN, const int32_t *tets, int64_t nT, int64_t t, int tl,
                              int i, TetShared *sh, double *scratch, int64_t *st) {
  double X[3][4];
  const bool in = t < nT && leg2_load(nodes, nN, tets, nT, t, X);
  TetShared &T = sh[tl];
  double *vt = scratch + 24 * tl;
  if (in) {
    for (int k = i; k < 24; k += 10) {
      const double x = X[0][kVolTerm[k][1]], y = X[1][kVolTerm[k][2]], z = X[2][kVolTerm[k][3]];
      vt[k] = kVolTerm[k][0] < 0 ? (-x * y * z) / 6 : (x * y * z) / 6;
    }
    if (i < 4) {
      double raw[4];
      leg2_column_raw(X, i, raw);
      for (int r = 0; r < 4; ++r) T.co[r][i] = raw[r];
    }
    for (int q = i; q < 11; q += 10) quad_point(X, q, T.pt[q][0], T.pt[q][1], T.pt[q][2]);
  }
  __syncthreads();
  if (i == 4) {
    double V = 0.0;
    if (in) {
      double sum = vt[0];
      for (int k = 1; k < 24; ++k) sum = sum + vt[k];
      V = fabs(sum);
    }
    T.V = V;
    T.ok = in && V > 0.0 && isfinite(V);
    if (t < nT && !T.ok) flag(st, in ? EMG_ST_DEGENERATE : EMG_ST_INDEX, t);
  }
  __syncthreads();
  if (T.ok) {
    const double V = T.V;
    for (int v = i; v < 16; v += 10) (&T.co[0][0])[v] = (&T.co[0][0])[v] / (6 * V);
  }
  __syncthreads();
}

// leg2_tet_stiff (grad.py:199-260), one thread per (tet, row i)
__global__ void __launch_bounds__(kFp64Threads, 4) k_leg2_stiff_fp64(const double *nodes, int64_t nN,
                                                                   const int32_t *tets, int64_t nT,
                                                                   const double *cond, int transposed, double *out,
                                                                   int64_t *st) {
  __shared__ TetShared sh[kFp64Tets];
  __shared__ double sg[kFp64Tets * 10 * 33];  // grad N_j at the 11 points; then the output stage
  const int tl = threadIdx.x / 10, i = threadIdx.x - tl * 10;
  const int64_t t0 = (int64_t)blockIdx.x * kFp64Tets, t = t0 + tl;
  fp64_prologue(nodes, nN, tets, nT, t, tl, i, sh, sg, st);
  const bool ok = sh[tl].ok;
  const double V = sh[tl].V;
  double kg[11][3];
  if (ok) {
    const int a = i < 4 ? i : kLEM[0][i - 4], b = i < 4 ? i : kLEM[1][i - 4];
    const double ca[4] = {sh[tl].co[0][a], sh[tl].co[1][a], sh[tl].co[2][a], sh[tl].co[3][a]};
    const double cb[4] = {sh[tl].co[0][b], sh[tl].co[1][b], sh[tl].co[2][b], sh[tl].co[3][b]};
    double k[9];
    for (int r = 0; r < 9; ++r) k[r] = cond[r * nT + t];
#pragma unroll
    for (int q = 0; q < 11; ++q) {
      const double x = sh[tl].pt[q][0], y = sh[tl].pt[q][1], z = sh[tl].pt[q][2];
      double g[3];
      if (i < 4) {  // grad_n1 (grad.py:139-151)
        const double qq = 4 * (ca[1] * x + ca[2] * y + ca[3] * z) + (4 * ca[0] - 1);
        g[0] = qq * ca[1], g[1] = qq * ca[2], g[2] = qq * ca[3];
      } else {  // grad_n2 (grad.py:154-172)
        const double L1 = 4 * (ca[0] + ca[1] * x + ca[2] * y + ca[3] * z);
        const double L2 = 4 * (cb[0] + cb[1] * x + cb[2] * y + cb[3] * z);
        g[0] = L2 * ca[1] + L1 * cb[1];
        g[1] = L2 * ca[2] + L1 * cb[2];
        g[2] = L2 * ca[3] + L1 * cb[3];
      }
      double *sp = sg + (tl * 10 + i) * 33 + q * 3;
      sp[0] = g[0], sp[1] = g[1], sp[2] = g[2];
      // matmul(cond_tet, grad) for row i
      kg[q][0] = __fma_rn(k[2], g[2], __fma_rn(k[1], g[1], k[0] * g[0]));
      kg[q][1] = __fma_rn(k[5], g[2], __fma_rn(k[4], g[1], k[3] * g[0]));
      kg[q][2] = __fma_rn(k[8], g[2], __fma_rn(k[7], g[1], k[6] * g[0]));
    }
  }
  __syncthreads();
  double row[10];
  // two entries at a time: independent sums, each in the reference's order
#pragma unroll 1
  for (int j = 0; j < 10; j += 2) {
    double s0 = 0.0, s1 = 0.0;
    if (ok) {
      const double *g0 = sg + (tl * 10 + j) * 33, *g1 = g0 + 33;
#pragma unroll
      for (int q = 0; q < 11; ++q) {
        const double d0 = __fma_rn(kg[q][2], g0[3 * q + 2], __fma_rn(kg[q][1], g0[3 * q + 1], kg[q][0] * g0[3 * q]));
        const double d1 = __fma_rn(kg[q][2], g1[3 * q + 2], __fma_rn(kg[q][1], g1[3 * q + 1], kg[q][0] * g1[3 * q]));
        s0 = __fma_rn(d0, kHW[q], s0);
        s1 = __fma_rn(d1, kHW[q], s1);
      }
    }
    row[j] = s0 * V;
    row[j + 1] = s1 * V;
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 10; ++j) sg[tl * 100 + (transposed ? 10 * j + i : 10 * i + j)] = ok ? row[j] : 0.0;
  __syncthreads();
  store_block(sg, t0, nT, kFp64Tets, out);
}

// leg2_tet_mass (grad.py:263-338), one thread per (tet, row i); entry (i, j)
// is the reference's val of (min, max) -- sum_q (w_q N_lo) N_hi -- times
// rho_cp, times V
__global__ void __launch_bounds__(kFp64Threads) k_leg2_mass_fp64(const double *nodes, int64_t nN,
                                                                  const int32_t *tets, int64_t nT,
                                                                  const double *rho_cp, int transposed, double *out,
                                                                  int64_t *st) {
  __shared__ TetShared sh[kFp64Tets];
  __shared__ double snv[kFp64Tets * 110];  // N_j at the 11 points
  __shared__ double sn[kFp64Tets * 100];   // output stage
  const int tl = threadIdx.x / 10, i = threadIdx.x - tl * 10;
  const int64_t t0 = (int64_t)blockIdx.x * kFp64Tets, t = t0 + tl;
  fp64_prologue(nodes, nN, tets, nT, t, tl, i, sh, snv, st);
  const bool ok = sh[tl].ok;
  const double V = sh[tl].V;
  double Ni[11];
  if (ok) {
    const int a = i < 4 ? i : kLEM[0][i - 4], b = i < 4 ? i : kLEM[1][i - 4];
    const double ca[4] = {sh[tl].co[0][a], sh[tl].co[1][a], sh[tl].co[2][a], sh[tl].co[3][a]};
    const double cb[4] = {sh[tl].co[0][b], sh[tl].co[1][b], sh[tl].co[2][b], sh[tl].co[3][b]};
#pragma unroll
    for (int q = 0; q < 11; ++q) {
      const double x = sh[tl].pt[q][0], y = sh[tl].pt[q][1], z = sh[tl].pt[q][2];
      const double La = ca[0] + ca[1] * x + ca[2] * y + ca[3] * z;
      double N;
      if (i < 4) {
        N = La * (2.0 * La - 1.0);
      } else {
        const double Lb = cb[0] + cb[1] * x + cb[2] * y + cb[3] * z;
        N = 4.0 * La * Lb;
      }
      Ni[q] = N;
      snv[(tl * 10 + i) * 11 + q] = N;
    }
  }
  __syncthreads();
  double row[10];
  const double rho = ok ? rho_cp[t] : 0.0;
#pragma unroll 1
  for (int j = 0; j < 10; j += 2) {
    double v0 = 0.0, v1 = 0.0;
    if (ok) {
      const double *n0 = snv + (tl * 10 + j) * 11, *n1 = n0 + 11;
      const bool f0 = i <= j, f1 = i <= j + 1;  // which factor is the lower-numbered function
#pragma unroll
      for (int q = 0; q < 11; ++q) {
        const double a0 = n0[q], a1 = n1[q];
        v0 = __fma_rn(kHW[q] * (f0 ? Ni[q] : a0), f0 ? a0 : Ni[q], v0);
        v1 = __fma_rn(kHW[q] * (f1 ? Ni[q] : a1), f1 ? a1 : Ni[q], v1);
      }
    }
    row[j] = v0 * rho * V;
    row[j + 1] = v1 * rho * V;
  }
#pragma unroll
  for (int j = 0; j < 10; ++j) sn[tl * 100 + (transposed ? 10 * j + i : 10 * i + j)] = ok ? row[j] : 0.0;
  __syncthreads();
  store_block(sn, t0, nT, kFp64Tets, out);
}

// the moment tables of the rule
struct HeatRule {
  double kvv[4][4];  // 16 Wm_ij - 4 r_i - 4 r_j + T
  double kve[4][4];  // 4 (4 Wm_ix - r_x)
  double w16[4][4];  // 16 Wm
  double c[100];     // C_ij = sum_q w_q N_i N_j
};

HeatRule make_heat_rule() {
  HeatRule h;
  double W[4][4], r[4] = {0, 0, 0, 0}, T = 0.0;
  for (int m = 0; m < 4; ++m)
    for (int n = 0; n < 4; ++n) {
      double a = 0.0;
      for (int q = 0; q < 11; ++q) a += hHW[q] * hHP[m][q] * hHP[n][q];
      W[m][n] = a;
    }
  for (int m = 0; m < 4; ++m) {
    for (int n = 0; n < 4; ++n) r[m] += W[m][n];
    T += r[m];
  }
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      h.kvv[i][j] = 16 * W[i][j] - 4 * r[i] - 4 * r[j] + T;
      h.kve[i][j] = 4 * (4 * W[i][j] - r[j]);
      h.w16[i][j] = 16 * W[i][j];
    }
  for (int i = 0; i < 10; ++i)
    for (int j = 0; j < 10; ++j) {
      double a = 0.0;
      for (int q = 0; q < 11; ++q) {
        double L[4];
        for (int m = 0; m < 4; ++m) L[m] = hHP[m][q];
        const double Ni = i < 4 ? L[i] * (2.0 * L[i] - 1.0) : 4.0 * L[hLEM[0][i - 4]] * L[hLEM[1][i - 4]];
        const double Nj = j < 4 ? L[j] * (2.0 * L[j] - 1.0) : 4.0 * L[hLEM[0][j - 4]] * L[hLEM[1][j - 4]];
        a += hHW[q] * Ni * Nj;
      }
      h.c[10 * i + j] = a;
    }
  return h;
}

// one thread per tet, its 100 values staged per block (value-major, so the
// staging writes do not conflict) and stored coalesced
// one entry of the stiffness block from S_pq = V (k grad lam_p) . grad lam_q
// and the rule's tables (i, j compile-time after unrolling)
__device__ __forceinline__ double exact_stiff(const double (&S)[4][4], const HeatRule &h, int i, int j) {
  constexpr int A[6] = {0, 0, 0, 1, 1, 2}, B[6] = {1, 2, 3, 2, 3, 3};
  if (i < 4 && j < 4) return S[i][j] * h.kvv[i][j];
  if (i < 4) {
    const int a = A[j - 4], b = B[j - 4];
    return S[i][a] * h.kve[i][b] + S[i][b] * h.kve[i][a];
  }
  if (j < 4) {
    const int a = A[i - 4], b = B[i - 4];
    return S[a][j] * h.kve[j][b] + S[b][j] * h.kve[j][a];
  }
  const int a = A[i - 4], b = B[i - 4], c = A[j - 4], d = B[j - 4];
  return h.w16[b][d] * S[a][c] + h.w16[b][c] * S[a][d] + h.w16[a][d] * S[b][c] + h.w16[a][c] * S[b][d];
}

// KIND 0 stiffness, 1 capacity; TR 1 writes each tet's block transposed. The
// 100 values of a tet are staged in two halves of 50 (13.2 KB per warp; the
// stiffness kernel at 126 registers), so 16 one-warp CTAs share an SM.
// Quarters, for 32 capacity CTAs per SM, measured 1.9x slower.
template <int KIND, int TR>
__global__ void __launch_bounds__(kExactTets, 16) k_leg2_exact(const double *nodes, int64_t nN, const int32_t *tets,
                                                               int64_t nT, const double *coef,
                                                               const __grid_constant__ HeatRule h, double *out,
                                                               int64_t *st) {
  constexpr int LD = kExactTets + 1;  // padded: the coalesced read walks values of one tet
  constexpr int PART = 50;
  __shared__ double stage[PART * LD];
  const int tl = threadIdx.x;
  const int64_t t0 = (int64_t)blockIdx.x * kExactTets, t = t0 + tl;
  double X[4][3];
  bool ok = false;
  double V = 0.0, det = 0.0, g[4][3];
  if (t < nT) {
    bool idx_ok = true;
    for (int v = 0; v < 4; ++v) {
      const int64_t n = tets[v * nT + t];
      const bool in = n >= 0 && n < nN;
      idx_ok = idx_ok && in;
      for (int d = 0; d < 3; ++d) X[v][d] = in ? nodes[d * nN + n] : 0.0;
    }
    double e[3][3];
    for (int v = 0; v < 3; ++v)
      for (int d = 0; d < 3; ++d) e[v][d] = X[v + 1][d] - X[0][d];
    // grad lam_1..3 = rows of the inverse edge matrix (cofactors / det)
    g[1][0] = e[1][1] * e[2][2] - e[1][2] * e[2][1];
    g[1][1] = e[1][2] * e[2][0] - e[1][0] * e[2][2];
    g[1][2] = e[1][0] * e[2][1] - e[1][1] * e[2][0];
    g[2][0] = e[2][1] * e[0][2] - e[2][2] * e[0][1];
    g[2][1] = e[2][2] * e[0][0] - e[2][0] * e[0][2];
    g[2][2] = e[2][0] * e[0][1] - e[2][1] * e[0][0];
    g[3][0] = e[0][1] * e[1][2] - e[0][2] * e[1][1];
    g[3][1] = e[0][2] * e[1][0] - e[0][0] * e[1][2];
    g[3][2] = e[0][0] * e[1][1] - e[0][1] * e[1][0];
    det = e[0][0] * g[1][0] + e[0][1] * g[1][1] + e[0][2] * g[1][2];
    V = fabs(det) / 6.0;
    ok = idx_ok && V > 0.0 && isfinite(V);
    if (!ok) flag(st, idx_ok ? EMG_ST_DEGENERATE : EMG_ST_INDEX, t);
  }
  double S[4][4];
  double rv = 0.0;
  if constexpr (KIND == 1) {
    rv = ok ? coef[t] * V : 0.0;
  } else {
    if (ok) {
      const double inv = 1.0 / det;
      for (int p = 1; p < 4; ++p)
        for (int d = 0; d < 3; ++d) g[p][d] *= inv;
      for (int d = 0; d < 3; ++d) g[0][d] = -(g[1][d] + g[2][d] + g[3][d]);
      double k[9];
      for (int r = 0; r < 9; ++r) k[r] = coef[r * nT + t];
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const double kg0 = k[0] * g[p][0] + k[1] * g[p][1] + k[2] * g[p][2];
        const double kg1 = k[3] * g[p][0] + k[4] * g[p][1] + k[5] * g[p][2];
        const double kg2 = k[6] * g[p][0] + k[7] * g[p][1] + k[8] * g[p][2];
#pragma unroll
        for (int q = 0; q < 4; ++q) S[p][q] = (kg0 * g[q][0] + kg1 * g[q][1] + kg2 * g[q][2]) * V;
      }
    } else {
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) S[p][q] = 0.0;
    }
  }
  const int64_t nt = min((int64_t)kExactTets, nT - t0);
  double *o = out + t0 * 100;
#pragma unroll
  for (int part = 0; part < 100 / PART; ++part) {
    // output position o_k = 10 r + c of the stored block; (i, j) is (r, c),
    // or (c, r) when the block is stored transposed
#pragma unroll
    for (int q = 0; q < PART; ++q) {
      const int ok_ = part * PART + q, r = ok_ / 10, c = ok_ % 10;
      const int i = TR ? c : r, j = TR ? r : c;
      stage[q * LD + tl] = KIND == 1 ? h.c[10 * i + j] * rv : exact_stiff(S, h, i, j);
    }
    __syncthreads();
    for (int k = tl; k < nt * PART; k += kExactTets) {
      const int tt = k / PART, e = k - tt * PART;
      o[(int64_t)tt * 100 + part * PART + e] = stage[e * LD + tt];
    }
    __syncthreads();
  }
}

}  // namespace
}  // namespace emg

using namespace emg;

extern "C" int emg_leg2_element(const double *d_nodes, int64_t n_nodes, const int32_t *d_tets, int64_t n_tets,
                                const double *d_coef, int kind, int precision, int layout, double *d_values,
                                int64_t *d_status, emg_stream_t stream) {
  if (kind != 0 && kind != 1) return fail(EMG_EINVAL, "kind must be 0 (stiffness) or 1 (mass)");
  if (precision != EMG_FP64 && precision != EMG_EXACT)
    return fail(EMG_EINVAL, "precision must be EMG_FP64 or EMG_EXACT");
  if (layout != EMG_LAYOUT_COO && layout != EMG_LAYOUT_COO_T)
    return fail(EMG_EINVAL, "layout must be EMG_LAYOUT_COO or EMG_LAYOUT_COO_T");
  if (n_tets < 0 || n_nodes < 0) return fail(EMG_EINVAL, "negative size");
  if (n_tets >= INT32_MAX / 100) return fail(EMG_ERANGE, "more than 21,474,836 tets");
  if (n_tets == 0) return EMG_OK;
  if (!d_nodes || !d_tets || !d_coef || !d_values || !d_status) return fail(EMG_EINVAL, "null pointer");
  const int tr = layout == EMG_LAYOUT_COO_T;
  cudaStream_t s = S(stream);
  if (precision == EMG_EXACT) {
    static const HeatRule rule = make_heat_rule();
    const int64_t blocks = (n_tets + kExactTets - 1) / kExactTets;
#define EMG_EX(K, T) \
  k_leg2_exact<K, T><<<(unsigned)blocks, kExactTets, 0, s>>>(d_nodes, n_nodes, d_tets, n_tets, d_coef, rule, d_values, \
                                                             d_status)
    if (kind == 1) {
      if (tr) EMG_EX(1, 1); else EMG_EX(1, 0);
    } else {
      if (tr) EMG_EX(0, 1); else EMG_EX(0, 0);
    }
#undef EMG_EX
    return launch_check("k_leg2_exact");
  }
  // prefer shared memory over L1 for the fp64 kernels, once per device (a
  // hint: a failure only costs occupancy, so its status is not an error)
  static bool carveout[64] = {false};
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess && dev >= 0 && dev < 64 && !carveout[dev]) {
    if (cudaFuncSetAttribute(k_leg2_stiff_fp64, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared) != cudaSuccess ||
        cudaFuncSetAttribute(k_leg2_mass_fp64, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared) != cudaSuccess)
      (void)cudaGetLastError();  // leave no error behind for the launch check
    carveout[dev] = true;
  }
  const int64_t blocks = (n_tets + kFp64Tets - 1) / kFp64Tets;
  if (kind == 0) {
    k_leg2_stiff_fp64<<<(unsigned)blocks, kFp64Threads, 0, s>>>(d_nodes, n_nodes, d_tets, n_tets, d_coef, tr,
                                                                d_values, d_status);
    return launch_check("k_leg2_stiff_fp64");
  }
  k_leg2_mass_fp64<<<(unsigned)blocks, kFp64Threads, 0, s>>>(d_nodes, n_nodes, d_tets, n_tets, d_coef, tr,
                                                             d_values, d_status);
  return launch_check("k_leg2_mass_fp64");
}
