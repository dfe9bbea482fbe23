/*
 * CPU ORACLE -- test infrastructure, not product code (the timed CPU
 * baseline of bench.py, and a checker in tests/).
 *
 * The reference's cached-pattern assembly of one frequency,
 *
 *   dataE, dataB, rows, cols = _matrix_builder(..., tetids)   curlcurl.py:387-456
 *   A = cscmap.to_csc(dataE - dataB * k0**2)                  assembler.py:494,
 *                                                             csc_cast.py:55-63, 162-177
 *
 * for a mesh whose full COO arrays (19.2 KB per tet) do not fit in host
 * memory at once: the assembled tets are taken in chunks of consecutive
 * tetids, each chunk's element matrices built by oracle_matrix_builder
 * (nedelec_oracle.c) and its slots added into the one CSC value array in the
 * reference scatter's order -- by column, then row, then slot, which is
 * precompute_csc_pattern's sorted order (csc_cast.py:65-160) -- so every
 * nonzero sums its slots in the order the one-piece to_csc sums them and the
 * chunked result equals it bit for bit.
 *
 * Setup (untimed in the benchmark, as the reference caches its CSCMapping):
 *   oracle_dof_incidence  DoF -> assembled tets (counting sort)
 *   oracle_pattern_rows   indptr / indices of the pattern: the rows of column
 *                         d are the DoFs of every assembled tet holding d,
 *                         sorted, without repeats (the arrays
 *                         precompute_csc_pattern derives from rows/cols)
 *   oracle_chunk_order    a chunk's slots in scatter order with their nonzero
 *                         positions, and the thread split points between runs
 *                         of one position
 * Per step:
 *   oracle_matrix_builder per chunk, then oracle_chunk_scatter.
 */
#include <complex.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

static void set_threads(int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
}

/* dptr[N+1], dtet[20*nA]: the assembled tets holding DoF d, ascending. */
int oracle_dof_incidence(const int64_t *t2f, int64_t nT, const int64_t *tetids, int64_t nA, int64_t N,
                         int64_t *dptr, int32_t *dtet) {
  memset(dptr, 0, (size_t)(N + 1) * sizeof(int64_t));
  for (int64_t a = 0; a < nA; ++a) {
    const int64_t t = tetids[a];
    if (t < 0 || t >= nT) return -1;
    for (int i = 0; i < 20; ++i) {
      const int64_t d = t2f[i * nT + t];
      if (d < 0 || d >= N) return -1;
      dptr[d + 1]++;
    }
  }
  for (int64_t d = 0; d < N; ++d) dptr[d + 1] += dptr[d];
  int64_t *cur = (int64_t *)malloc((size_t)(N ? N : 1) * sizeof(int64_t));
  if (!cur) return -2;
  memcpy(cur, dptr, (size_t)N * sizeof(int64_t));
  for (int64_t a = 0; a < nA; ++a) {
    const int64_t t = tetids[a];
    for (int i = 0; i < 20; ++i) dtet[cur[t2f[i * nT + t]]++] = (int32_t)a;
  }
  free(cur);
  return 0;
}

static int cmp_i64(const void *a, const void *b) {
  const int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
  return (x > y) - (x < y);
}

/* The sorted distinct rows of column d into buf; returns their count. */
static int64_t column_rows(const int64_t *t2f, int64_t nT, const int64_t *tetids, const int64_t *dptr,
                           const int32_t *dtet, int64_t d, int64_t *buf) {
  int64_t n = 0;
  for (int64_t k = dptr[d]; k < dptr[d + 1]; ++k) {
    const int64_t t = tetids[dtet[k]];
    for (int i = 0; i < 20; ++i) buf[n++] = t2f[i * nT + t];
  }
  qsort(buf, (size_t)n, sizeof(int64_t), cmp_i64);
  int64_t u = 0;
  for (int64_t k = 0; k < n; ++k)
    if (k == 0 || buf[k] != buf[k - 1]) buf[u++] = buf[k];
  return u;
}

/* indices == NULL: fills indptr[N+1] and returns nnz. Otherwise writes
 * indices[nnz] (int32) for that indptr and returns nnz. max_deg: the largest
 * dptr[d+1] - dptr[d] (bounds the per-thread buffer). */
int64_t oracle_pattern_rows(const int64_t *t2f, int64_t nT, const int64_t *tetids, const int64_t *dptr,
                            const int32_t *dtet, int64_t N, int64_t max_deg, int64_t *indptr, int32_t *indices,
                            int nthreads) {
  set_threads(nthreads);
  int err = 0;
  if (!indices) indptr[0] = 0;
#pragma omp parallel reduction(| : err)
  {
    int64_t *buf = (int64_t *)malloc((size_t)(20 * (max_deg > 0 ? max_deg : 1)) * sizeof(int64_t));
    if (!buf) err |= 1;
#pragma omp for schedule(dynamic, 1024)
    for (int64_t d = 0; d < N; ++d) {
      if (!buf) continue;
      const int64_t u = column_rows(t2f, nT, tetids, dptr, dtet, d, buf);
      if (!indices) {
        indptr[d + 1] = u;
      } else {
        for (int64_t k = 0; k < u; ++k) indices[indptr[d] + k] = (int32_t)buf[k];
      }
    }
    free(buf);
  }
  if (err) return -1;
  if (!indices)
    for (int64_t d = 0; d < N; ++d) indptr[d + 1] += indptr[d];
  return indptr[N];
}

/* Chunk of assembled tets [a0, a1): its 400*(a1-a0) slots (slot s of the
 * chunk = slot 400*a0 + s of _matrix_builder's COO) in scatter order --
 * column, row, slot -- as perm[k] (the chunk slot) and tgt[k] (its nonzero
 * position); splits[0..nsplit] cut k into nsplit ranges that never split a
 * run of one position (per-thread ranges of the scatter). */
int oracle_chunk_order(const int64_t *t2f, int64_t nT, const int64_t *tetids, int64_t a0, int64_t a1,
                       const int64_t *indptr, const int32_t *indices, int64_t N, int32_t *perm, int32_t *tgt,
                       int64_t *splits, int nsplit, int nthreads) {
  set_threads(nthreads);
  const int64_t S = 400 * (a1 - a0);
  int64_t *cnt = (int64_t *)calloc((size_t)(N + 1), sizeof(int64_t));
  int32_t *pos = (int32_t *)malloc((size_t)(S ? S : 1) * sizeof(int32_t));
  int64_t *colof = (int64_t *)malloc((size_t)(S ? S : 1) * sizeof(int64_t));
  if (!cnt || !pos || !colof) {
    free(cnt);
    free(pos);
    free(colof);
    return -2;
  }
  int err = 0;
#pragma omp parallel for schedule(static) reduction(| : err)
  for (int64_t s = 0; s < S; ++s) {
    const int64_t t = tetids[a0 + s / 400];
    const int ii = (int)((s % 400) / 20), jj = (int)(s % 20);
    const int64_t r = t2f[ii * nT + t], c = t2f[jj * nT + t];
    if (c < 0 || c >= N) {
      err |= 1;
      continue;
    }
    int64_t lo = indptr[c], hi = indptr[c + 1];
    while (lo < hi) {  /* first position with row >= r */
      const int64_t m = (lo + hi) / 2;
      if (indices[m] < r) lo = m + 1;
      else hi = m;
    }
    if (lo >= indptr[c + 1] || indices[lo] != r) err |= 1;
    pos[s] = (int32_t)lo;
    colof[s] = c;
  }
  if (err) {
    free(cnt);
    free(pos);
    free(colof);
    return -1;
  }
  for (int64_t s = 0; s < S; ++s) cnt[colof[s] + 1]++;
  for (int64_t c = 0; c < N; ++c) cnt[c + 1] += cnt[c];
  int64_t *cur = (int64_t *)malloc((size_t)(N ? N : 1) * sizeof(int64_t));
  if (!cur) {
    free(cnt);
    free(pos);
    free(colof);
    return -2;
  }
  memcpy(cur, cnt, (size_t)N * sizeof(int64_t));
  for (int64_t s = 0; s < S; ++s) perm[cur[colof[s]]++] = (int32_t)s; /* slots ascending within a column */
  free(cur);
  free(colof);
  /* within a column: by position (= row), then slot; insertion sort, stable */
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t c = 0; c < N; ++c) {
    for (int64_t k = cnt[c] + 1; k < cnt[c + 1]; ++k) {
      const int32_t v = perm[k];
      int64_t j = k - 1;
      while (j >= cnt[c] && pos[perm[j]] > pos[v]) {
        perm[j + 1] = perm[j];
        --j;
      }
      perm[j + 1] = v;
    }
  }
  free(cnt);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < S; ++k) tgt[k] = pos[perm[k]];
  free(pos);
  splits[0] = 0;
  for (int i = 1; i < nsplit; ++i) {
    int64_t k = S * i / nsplit;
    if (k < splits[i - 1]) k = splits[i - 1];
    while (k > 0 && k < S && tgt[k] == tgt[k - 1]) ++k;
    splits[i] = k;
  }
  splits[nsplit] = S;
  return 0;
}

/* data_csc[tgt[k]] += alpha*dataE[perm[k]] + beta*dataB[perm[k]] in k order
 * within each run of one position (scatter_to_csc_c16, csc_cast.py:162-177,
 * on the caller's combination Evec - Bvec*k0^2, assembler.py:494). */
void oracle_chunk_scatter(const cplx *dataE, const cplx *dataB, double alpha_re, double alpha_im, double beta_re,
                          double beta_im, const int32_t *perm, const int32_t *tgt, const int64_t *splits,
                          int nsplit, cplx *data_csc, int nthreads) {
  set_threads(nthreads);
  const cplx alpha = alpha_re + alpha_im * I, beta = beta_re + beta_im * I;
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < nsplit; ++i)
    for (int64_t k = splits[i]; k < splits[i + 1]; ++k) {
      const int32_t s = perm[k];
      data_csc[tgt[k]] += alpha * dataE[s] + beta * dataB[s];
    }
}
