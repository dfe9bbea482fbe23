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
  uint8_t pad;
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

// element kernel launchers, one translation unit per (form, material kind);
// form 0 = reference-faithful FP64, 1 = mixed, 2 = exact closed form
#define EMG_DECLARE_ELEM(F, K) int launch_element_##F##_##K(const ElemArgs &a, int out, cudaStream_t s);
EMG_DECLARE_ELEM(0, 0)
EMG_DECLARE_ELEM(0, 1)
EMG_DECLARE_ELEM(0, 2)
EMG_DECLARE_ELEM(1, 0)
EMG_DECLARE_ELEM(1, 1)
EMG_DECLARE_ELEM(1, 2)
EMG_DECLARE_ELEM(2, 0)
EMG_DECLARE_ELEM(2, 1)
EMG_DECLARE_ELEM(2, 2)

// element values are complex64 for the mixed form, complex128 otherwise
inline bool values_fp32(int precision) { return precision == EMG_MIXED; }

// plan.cu
size_t plan_workspace_bytes(const emg_plan *p);
size_t plan_layout(emg_plan *p);
int plan_build(emg_plan *p, const int32_t *t2e, const int32_t *t2t, const int32_t *tetids, void *d_plan, void *d_ws,
               int32_t *indptr, int64_t *st, cudaStream_t s);
int plan_finish(const emg_plan *p, const int32_t *t2e, const int32_t *t2t, const int32_t *tetids, void *d_plan,
                const int32_t *indptr, int32_t *indices, int64_t *st, cudaStream_t s);
int status_reset(int64_t *st, cudaStream_t s);

// gather.cu
int launch_gather(const emg_plan *p, const void *d_plan, const int32_t *indptr, const void *v1, const void *v2,
                  int precision, double ar, double ai, double br, double bi, void *A, int64_t *st, cudaStream_t s);
int launch_form_sweep(const void *K, const void *M, const void *P, int64_t nnz, const double *coef, int nf,
                      void *out, int64_t stride, cudaStream_t s);

}  // namespace emg
