/*
 * CPU ORACLE -- test infrastructure, not product code.
 *
 * Plain-C restatement of the reference's Nedelec-2 curl-curl assembly path
 * (biruichen/EMerge v2.8.0). Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py load this library, as the
 * checker and the timed CPU baseline. The product path never calls it.
 *
 * Parity: pinned against golden fixtures produced by running the reference's
 * own numba functions (tests/golden/make_golden.py).
 *
 * Functions restated, with the reference file:line they follow:
 *   tet_coefficients      physics/microwave/assembly/curlcurl.py:127-214
 *   local_mapping         mth/optimized.py:262-296
 *   matinv                mth/optimized.py:315-357
 *   basis fns / curls     compiled/ccbf.py:537 (_ne0_3d), :569 (_ne2_3d),
 *                         :790 (_nf0_3d), :808 (_nf1_3d), :644, :659, :928, :949
 *   ned2_tet_stiff_mass   physics/microwave/assembly/curlcurl.py:285-380
 *   _matrix_builder       physics/microwave/assembly/curlcurl.py:387-456
 *   precompute_csc_pattern mth/csc_cast.py:65-160
 *   scatter_to_csc_c16    mth/csc_cast.py:162-177
 *
 * Only the SECOND_MIXED_VOLAKIS dofcodes [64]*6+[66]*6+[128]*4+[129]*4 are
 * supported (elements/dofsets.py:114-115), which is what Microwave3D uses.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

/* KEAST4 11-point rule as printed in curlcurl.py:277-283 (weights, then the
 * four barycentric rows). */
static const double DPTS[5][11] = {
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

#define NQ 11
#define NDOF 20

/* tet_coefficients (curlcurl.py:127-214): signed cofactors, V = |det| / 6 */
static void tet_coefficients(const double *xs, const double *ys, const double *zs, double aa[4], double bb[4],
                             double cc[4], double dd[4], double *V) {
  double x1 = xs[0], x2 = xs[1], x3 = xs[2], x4 = xs[3];
  double y1 = ys[0], y2 = ys[1], y3 = ys[2], y4 = ys[3];
  double z1 = zs[0], z2 = zs[1], z3 = zs[2], z4 = zs[3];
  double det = -x1 * y2 * z3 + x1 * y2 * z4 + x1 * y3 * z2 - x1 * y3 * z4 - x1 * y4 * z2 + x1 * y4 * z3 +
               x2 * y1 * z3 - x2 * y1 * z4 - x2 * y3 * z1 + x2 * y3 * z4 + x2 * y4 * z1 - x2 * y4 * z3 -
               x3 * y1 * z2 + x3 * y1 * z4 + x3 * y2 * z1 - x3 * y2 * z4 - x3 * y4 * z1 + x3 * y4 * z2 +
               x4 * y1 * z2 - x4 * y1 * z3 - x4 * y2 * z1 + x4 * y2 * z3 + x4 * y3 * z1 - x4 * y3 * z2;
  *V = fabs(det) / 6.0;
  aa[0] = x2 * y3 * z4 - x2 * y4 * z3 - x3 * y2 * z4 + x3 * y4 * z2 + x4 * y2 * z3 - x4 * y3 * z2;
  aa[1] = -x1 * y3 * z4 + x1 * y4 * z3 + x3 * y1 * z4 - x3 * y4 * z1 - x4 * y1 * z3 + x4 * y3 * z1;
  aa[2] = x1 * y2 * z4 - x1 * y4 * z2 - x2 * y1 * z4 + x2 * y4 * z1 + x4 * y1 * z2 - x4 * y2 * z1;
  aa[3] = -x1 * y2 * z3 + x1 * y3 * z2 + x2 * y1 * z3 - x2 * y3 * z1 - x3 * y1 * z2 + x3 * y2 * z1;
  bb[0] = -y2 * z3 + y2 * z4 + y3 * z2 - y3 * z4 - y4 * z2 + y4 * z3;
  bb[1] = y1 * z3 - y1 * z4 - y3 * z1 + y3 * z4 + y4 * z1 - y4 * z3;
  bb[2] = -y1 * z2 + y1 * z4 + y2 * z1 - y2 * z4 - y4 * z1 + y4 * z2;
  bb[3] = y1 * z2 - y1 * z3 - y2 * z1 + y2 * z3 + y3 * z1 - y3 * z2;
  cc[0] = x2 * z3 - x2 * z4 - x3 * z2 + x3 * z4 + x4 * z2 - x4 * z3;
  cc[1] = -x1 * z3 + x1 * z4 + x3 * z1 - x3 * z4 - x4 * z1 + x4 * z3;
  cc[2] = x1 * z2 - x1 * z4 - x2 * z1 + x2 * z4 + x4 * z1 - x4 * z2;
  cc[3] = -x1 * z2 + x1 * z3 + x2 * z1 - x2 * z3 - x3 * z1 + x3 * z2;
  dd[0] = -x2 * y3 + x2 * y4 + x3 * y2 - x3 * y4 - x4 * y2 + x4 * y3;
  dd[1] = x1 * y3 - x1 * y4 - x3 * y1 + x3 * y4 + x4 * y1 - x4 * y3;
  dd[2] = -x1 * y2 + x1 * y4 + x2 * y1 - x2 * y4 - x4 * y1 + x4 * y2;
  dd[3] = x1 * y2 - x1 * y3 - x2 * y1 + x2 * y3 + x3 * y1 - x3 * y2;
}

/* matinv (optimized.py:315-357): 3x3 complex inverse, diagonal fast path */
static void matinv3(const cplx M[9], cplx out[9]) {
  if (M[1] == 0 && M[2] == 0 && M[3] == 0 && M[5] == 0 && M[6] == 0 && M[7] == 0) {
    memset(out, 0, 9 * sizeof(cplx));
    out[0] = 1.0 / M[0];
    out[4] = 1.0 / M[4];
    out[8] = 1.0 / M[8];
    return;
  }
  cplx det = M[0] * M[4] * M[8] - M[0] * M[5] * M[7] - M[1] * M[3] * M[8] + M[1] * M[5] * M[6] +
             M[2] * M[3] * M[7] - M[2] * M[4] * M[6];
  out[0] = M[4] * M[8] - M[5] * M[7];
  out[1] = -M[1] * M[8] + M[2] * M[7];
  out[2] = M[1] * M[5] - M[2] * M[4];
  out[3] = -M[3] * M[8] + M[5] * M[6];
  out[4] = M[0] * M[8] - M[2] * M[6];
  out[5] = -M[0] * M[5] + M[2] * M[3];
  out[6] = M[3] * M[7] - M[4] * M[6];
  out[7] = -M[0] * M[7] + M[1] * M[6];
  out[8] = M[0] * M[4] - M[1] * M[3];
  for (int i = 0; i < 9; ++i) out[i] = out[i] / det;
}

/* evaluate basis value (kind 0..3 = ne0, ne2, nf0, nf1) and curl at the 11
 * points; coeff[r][m]: r = 0 (a), 1 (b), 2 (c), 3 (d); (ccbf.py closed forms) */
static void eval_basis(int kind, const double co[4][4], const double *xs, const double *ys, const double *zs,
                       int i, int j, int k, double val[3][NQ], double curl[3][NQ]) {
  double ai = co[0][i], bi = co[1][i], ci = co[2][i], di = co[3][i];
  double aj = co[0][j], bj = co[1][j], cj = co[2][j], dj = co[3][j];
  double ak = co[0][k], bk = co[1][k], ck = co[2][k], dk = co[3][k];
  for (int n = 0; n < NQ; ++n) {
    double x = xs[n], y = ys[n], z = zs[n];
    double Li = ai + bi * x + ci * y + di * z;
    double Lj = aj + bj * x + cj * y + dj * z;
    double Lk = ak + bk * x + ck * y + dk * z;
    if (kind == 0) { /* _ne0_3d :537, _curl_ne0_3d :644 */
      val[0][n] = -Lj * bi + Li * bj;
      val[1][n] = -Lj * ci + Li * cj;
      val[2][n] = -Lj * di + Li * dj;
      curl[0][n] = 2 * ci * dj - 2 * cj * di;
      curl[1][n] = -2 * bi * dj + 2 * bj * di;
      curl[2][n] = 2 * bi * cj - 2 * bj * ci;
    } else if (kind == 1) { /* _ne2_3d :569, _curl_ne2_3d :659 */
      double t4 = Li - Lj;
      val[0][n] = t4 * (Li * bj - Lj * bi);
      val[1][n] = t4 * (Li * cj - Lj * ci);
      val[2][n] = t4 * (Li * dj - Lj * di);
      double t6 = Lj * ci - Li * cj, t8 = Lj * di - Li * dj, t10 = Lj * bi - Li * bj;
      double t9 = 2 * (Li - Lj);
      curl[0][n] = (di - dj) * t6 - (ci - cj) * t8 + t9 * (ci * dj - cj * di);
      curl[1][n] = -(di - dj) * t10 + (bi - bj) * t8 - t9 * (bi * dj - bj * di);
      curl[2][n] = t10 * (ci - cj) - (bi - bj) * t6 + t9 * (bi * cj - bj * ci);
    } else if (kind == 2) { /* _nf0_3d :790, _curl_nf0_3d :928 */
      val[0][n] = -Li * (Lk * bj - Lj * bk);
      val[1][n] = -Li * (Lk * cj - Lj * ck);
      val[2][n] = -Li * (Lk * dj - Lj * dk);
      double t0 = 2 * Li, t3 = Lk * cj - Lj * ck, t4 = Lk * dj - Lj * dk, t5 = Lk * bj - Lj * bk;
      curl[0][n] = t0 * (cj * dk - ck * dj) + t3 * di - t4 * ci;
      curl[1][n] = -t0 * (bj * dk - bk * dj) + t4 * bi - t5 * di;
      curl[2][n] = t0 * (bj * ck - bk * cj) - t3 * bi + t5 * ci;
    } else { /* _nf1_3d :808, _curl_nf1_3d :949 */
      val[0][n] = -Lj * (Lk * bi - Li * bk);
      val[1][n] = -Lj * (Lk * ci - Li * ck);
      val[2][n] = -Lj * (Lk * di - Li * dk);
      double t0 = 2 * Lj, t3 = Lk * ci - Li * ck, t4 = Lk * di - Li * dk, t5 = Lk * bi - Li * bk;
      curl[0][n] = t0 * (ci * dk - ck * di) + t3 * dj - t4 * cj;
      curl[1][n] = -t0 * (bi * dk - bk * di) + t4 * bj - t5 * dj;
      curl[2][n] = t0 * (bi * ck - bk * ci) - t3 * bj + t5 * cj;
    }
  }
}

/* ned2_tet_stiff_mass (curlcurl.py:285-380) for the Volakis DoF set.
 * X[3][4] vertex coords (tet order), lem[2][6], ltm[3][4] local maps,
 * Ms = ur^-1, Mm = er (row-major 3x3). K, M: 20x20 row-major. */
void oracle_tet_stiff_mass(const double X[3][4], const int64_t lem[2][6], const int64_t ltm[3][4], const cplx Ms[9],
                           const cplx Mm[9], cplx *K, cplx *M) {
  double aa[4], bb[4], cc[4], dd[4], V;
  tet_coefficients(X[0], X[1], X[2], aa, bb, cc, dd, &V);
  double co[4][4];
  for (int m = 0; m < 4; ++m) {
    co[0][m] = aa[m] / (6 * V);
    co[1][m] = bb[m] / (6 * V);
    co[2][m] = cc[m] / (6 * V);
    co[3][m] = dd[m] / (6 * V);
  }
  double xs[NQ], ys[NQ], zs[NQ];
  for (int n = 0; n < NQ; ++n) {
    xs[n] = X[0][0] * DPTS[1][n] + X[0][1] * DPTS[2][n] + X[0][2] * DPTS[3][n] + X[0][3] * DPTS[4][n];
    ys[n] = X[1][0] * DPTS[1][n] + X[1][1] * DPTS[2][n] + X[1][2] * DPTS[3][n] + X[1][3] * DPTS[4][n];
    zs[n] = X[2][0] * DPTS[1][n] + X[2][1] * DPTS[2][n] + X[2][2] * DPTS[3][n] + X[2][3] * DPTS[4][n];
  }
  static const int kinds[NDOF] = {0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 3};
  double fv[NDOF][3][NQ], fc[NDOF][3][NQ];
  cplx msc[NDOF][3][NQ], mmv[NDOF][3][NQ];
  for (int a = 0; a < NDOF; ++a) {
    int i, j, k;
    if (a < 12) {
      int e = a % 6;
      i = (int)lem[0][e];
      j = (int)lem[1][e];
      k = 0;
    } else {
      int f = (a - 12) % 4;
      i = (int)ltm[0][f];
      j = (int)ltm[1][f];
      k = (int)ltm[2][f];
    }
    eval_basis(kinds[a], co, xs, ys, zs, i, j, k, fv[a], fc[a]);
    for (int n = 0; n < NQ; ++n) { /* matmul_inplace curlcurl.py:110-119, weights :353-356 */
      for (int r = 0; r < 3; ++r) {
        cplx s = Ms[3 * r] * fc[a][0][n] + Ms[3 * r + 1] * fc[a][1][n] + Ms[3 * r + 2] * fc[a][2][n];
        cplx m = Mm[3 * r] * fv[a][0][n] + Mm[3 * r + 1] * fv[a][1][n] + Mm[3 * r + 2] * fv[a][2][n];
        msc[a][r][n] = s * DPTS[0][n];
        mmv[a][r][n] = m * DPTS[0][n];
      }
    }
  }
  for (int a = 0; a < NDOF; ++a) {
    for (int b = a; b < NDOF; ++b) { /* :358-376 */
      cplx accS = 0, accM = 0;
      for (int n = 0; n < NQ; ++n) {
        accS += msc[a][0][n] * fc[b][0][n] + msc[a][1][n] * fc[b][1][n] + msc[a][2][n] * fc[b][2][n];
        accM += mmv[a][0][n] * fv[b][0][n] + mmv[a][1][n] * fv[b][1][n] + mmv[a][2][n] * fv[b][2][n];
      }
      K[a * NDOF + b] = K[b * NDOF + a] = accS * V; /* :378-379 */
      M[a * NDOF + b] = M[b * NDOF + a] = accM * V;
    }
  }
}

/* local_mapping (optimized.py:262-296) for one entity with `nd` vertex ids */
static int64_t local_index(const int64_t v[4], int64_t gid) {
  for (int k = 0; k < 4; ++k)
    if (v[k] == gid) return k;
  return 0; /* the reference leaves 0 when not found */
}

/* _matrix_builder (curlcurl.py:387-456). Arrays are the reference layouts,
 * C-contiguous: nodes[3][nN], tets[4][nT], tris[3][F], edges[2][E],
 * t2f[20][nT], t2e[6][nT], t2tri[4][nT], ur/er[3][3][nT] (complex128).
 * Writes dataE/dataB (complex, 400*nA) and rows/cols (int64, 400*nA). */
int oracle_matrix_builder(const double *nodes, int64_t nN, const int64_t *tets, int64_t nT, const int64_t *tris,
                          int64_t F, const int64_t *edges, int64_t E, const int64_t *t2f, const int64_t *t2e,
                          const int64_t *t2tri, const cplx *ur, const cplx *er, const int64_t *tetids, int64_t nA,
                          cplx *dataE, cplx *dataB, int64_t *rows, int64_t *cols, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  (void)nN;
  (void)F;
  (void)E;
  int err = 0;
#pragma omp parallel for schedule(static) reduction(| : err)
  for (int64_t ia = 0; ia < nA; ++ia) {
    int64_t it = tetids[ia];
    if (it < 0 || it >= nT) {
      err |= 1;
      continue;
    }
    int64_t p = ia * 400;
    int64_t v[4];
    for (int q = 0; q < 4; ++q) v[q] = tets[q * nT + it];
    int64_t lem[2][6], ltm[3][4];
    for (int e = 0; e < 6; ++e) {
      int64_t ge = t2e[e * nT + it];
      lem[0][e] = local_index(v, edges[0 * E + ge]);
      lem[1][e] = local_index(v, edges[1 * E + ge]);
    }
    for (int f = 0; f < 4; ++f) {
      int64_t gf = t2tri[f * nT + it];
      for (int q = 0; q < 3; ++q) ltm[q][f] = local_index(v, tris[q * F + gf]);
    }
    double X[3][4];
    for (int d = 0; d < 3; ++d)
      for (int q = 0; q < 4; ++q) X[d][q] = nodes[d * nN + v[q]];
    cplx urt[9], ert[9], Ms[9];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) {
        urt[3 * r + c] = ur[(r * 3 + c) * nT + it];
        ert[3 * r + c] = er[(r * 3 + c) * nT + it];
      }
    matinv3(urt, Ms);
    oracle_tet_stiff_mass((const double(*)[4])X, (const int64_t(*)[6])lem, (const int64_t(*)[4])ltm, Ms, ert,
                          dataE + p, dataB + p);
    for (int ii = 0; ii < NDOF; ++ii)
      for (int jj = 0; jj < NDOF; ++jj) {
        rows[p + NDOF * ii + jj] = t2f[ii * nT + it];
        cols[p + NDOF * ii + jj] = t2f[jj * nT + it];
      }
  }
  return err ? -1 : 0;
}

/* precompute_csc_pattern (csc_cast.py:65-160): counting sort by column, then
 * per-column sort by row (stable here; the reference's np.argsort order among
 * equal rows is unspecified, which only changes the summation order). */
typedef struct {
  int64_t row, k;
} rk_t;

static int cmp_rk(const void *a, const void *b) {
  const rk_t *x = (const rk_t *)a, *y = (const rk_t *)b;
  if (x->row != y->row) return x->row < y->row ? -1 : 1;
  return x->k < y->k ? -1 : (x->k > y->k);
}

/* Pass 1: returns nnz; fills col_offsets[N+1], perm[S], target[S],
 * unique_counts tmp. Pass 2 (oracle_csc_fill) writes indptr/indices. */
int64_t oracle_csc_pattern(const int64_t *rows, const int64_t *cols, int64_t S, int64_t N, int64_t *col_offsets,
                           int64_t *perm, int64_t *indptr, int64_t *target, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  int64_t *cnt = (int64_t *)calloc((size_t)N, sizeof(int64_t));
  int64_t *grouped = (int64_t *)malloc((size_t)(S ? S : 1) * sizeof(int64_t));
  int64_t *uniq = (int64_t *)calloc((size_t)N, sizeof(int64_t));
  if (!cnt || !grouped || !uniq) {
    free(cnt);
    free(grouped);
    free(uniq);
    return -1;
  }
  for (int64_t k = 0; k < S; ++k) cnt[cols[k]]++;
  col_offsets[0] = 0;
  for (int64_t i = 0; i < N; ++i) col_offsets[i + 1] = col_offsets[i] + cnt[i];
  for (int64_t i = 0; i < N; ++i) cnt[i] = col_offsets[i];
  for (int64_t k = 0; k < S; ++k) grouped[cnt[cols[k]]++] = k;
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < N; ++i) {
    int64_t st = col_offsets[i], n = col_offsets[i + 1] - st;
    if (n == 0) continue;
    rk_t *loc = (rk_t *)malloc((size_t)n * sizeof(rk_t));
    for (int64_t j = 0; j < n; ++j) {
      loc[j].k = grouped[st + j];
      loc[j].row = rows[loc[j].k];
    }
    qsort(loc, (size_t)n, sizeof(rk_t), cmp_rk);
    int64_t u = 1;
    perm[st] = loc[0].k;
    for (int64_t j = 1; j < n; ++j) {
      if (loc[j].row != loc[j - 1].row) u++;
      perm[st + j] = loc[j].k;
    }
    uniq[i] = u;
    free(loc);
  }
  indptr[0] = 0;
  for (int64_t i = 0; i < N; ++i) indptr[i + 1] = indptr[i] + uniq[i];
  /* target positions (Phase 4) */
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < N; ++i) {
    int64_t st = col_offsets[i], n = col_offsets[i + 1] - st;
    if (n == 0) continue;
    int64_t pos = indptr[i];
    int64_t prev = rows[perm[st]];
    target[st] = pos;
    for (int64_t j = 1; j < n; ++j) {
      int64_t r = rows[perm[st + j]];
      if (r != prev) {
        pos++;
        prev = r;
      }
      target[st + j] = pos;
    }
  }
  free(cnt);
  free(grouped);
  free(uniq);
  return indptr[N];
}

void oracle_csc_indices(const int64_t *rows, const int64_t *perm, const int64_t *target, int64_t S, int64_t *indices) {
  for (int64_t k = 0; k < S; ++k) indices[target[k]] = rows[perm[k]];
}

/* scatter_to_csc_c16 (csc_cast.py:162-177): gather by perm, column-owned
 * accumulation. data_csc must be zeroed by the caller. */
void oracle_scatter_c16(const cplx *data, const int64_t *perm, const int64_t *target, const int64_t *col_offsets,
                        int64_t N, cplx *data_csc, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < N; ++i)
    for (int64_t k = col_offsets[i]; k < col_offsets[i + 1]; ++k) data_csc[target[k]] += data[perm[k]];
}

/* the caller's combination A = E - k0^2 B (assembler.py:494), fused with the
 * scatter: data = alpha*dataE + beta*dataB */
void oracle_scatter_lincomb_c16(const cplx *dataE, const cplx *dataB, double alpha_re, double alpha_im,
                                double beta_re, double beta_im, const int64_t *perm, const int64_t *target,
                                const int64_t *col_offsets, int64_t N, cplx *data_csc, int nthreads) {
  const cplx alpha = alpha_re + alpha_im * I, beta = beta_re + beta_im * I;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < N; ++i)
    for (int64_t k = col_offsets[i]; k < col_offsets[i + 1]; ++k) {
      int64_t s = perm[k];
      data_csc[target[k]] += alpha * dataE[s] + beta * dataB[s];
    }
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
