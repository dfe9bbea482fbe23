// solve.cu -- the reduced system handed to a sparse direct solver on the
// device. The reference solves A[:, solve_ids][solve_ids, :] x = b[solve_ids]
// (solver.py:2071) with SuperLU / Pardiso / MUMPS on the host or cuDSS on the
// GPU (SolverCuDSS, solver.py:1274-1323). cuDSS is not part of this toolkit;
// this entry point passes the device arrays to cuSOLVER's sparse QR
// (cusolverSpZcsrlsvqr). cuSOLVER and cuSPARSE are loaded on first use with
// dlopen, so the rest of the library loads and works without them.
#include "common.cuh"

#include <cusolverSp.h>
#include <cusparse.h>
#include <dlfcn.h>

#include <cstdio>
#include <mutex>

namespace {

struct SpSolverApi {
  decltype(&cusolverSpCreate) create = nullptr;
  decltype(&cusolverSpDestroy) destroy = nullptr;
  decltype(&cusolverSpSetStream) set_stream = nullptr;
  decltype(&cusolverSpZcsrlsvqr) zqr = nullptr;
  decltype(&cusparseCreateMatDescr) descr_create = nullptr;
  decltype(&cusparseDestroyMatDescr) descr_destroy = nullptr;
  decltype(&cusparseSetMatType) set_type = nullptr;
  decltype(&cusparseSetMatIndexBase) set_base = nullptr;
  char err[256] = "";
  bool ok = false;
};

void *open_first(const char *const *names) {
  for (; *names; ++names)
    if (void *h = dlopen(*names, RTLD_NOW | RTLD_GLOBAL)) return h;
  return nullptr;
}

template <typename F>
bool bind(void *lib, const char *name, F &fn) {
  fn = reinterpret_cast<F>(dlsym(lib, name));
  return fn != nullptr;
}

const SpSolverApi &sp_api() {
  static SpSolverApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    const char *solver_names[] = {"libcusolver.so.11", "/usr/local/cuda/lib64/libcusolver.so.11", nullptr};
    const char *sparse_names[] = {"libcusparse.so.12", "/usr/local/cuda/lib64/libcusparse.so.12", nullptr};
    void *hs = open_first(solver_names);
    void *hp = open_first(sparse_names);
    if (!hs || !hp) {
      snprintf(api.err, sizeof(api.err), "cannot load %s", !hs ? "libcusolver.so.11" : "libcusparse.so.12");
      return;
    }
    const bool all = bind(hs, "cusolverSpCreate", api.create) && bind(hs, "cusolverSpDestroy", api.destroy) &&
                     bind(hs, "cusolverSpSetStream", api.set_stream) &&
                     bind(hs, "cusolverSpZcsrlsvqr", api.zqr) &&
                     bind(hp, "cusparseCreateMatDescr", api.descr_create) &&
                     bind(hp, "cusparseDestroyMatDescr", api.descr_destroy) &&
                     bind(hp, "cusparseSetMatType", api.set_type) &&
                     bind(hp, "cusparseSetMatIndexBase", api.set_base);
    if (!all) {
      snprintf(api.err, sizeof(api.err), "a cuSOLVER / cuSPARSE entry point is missing");
      return;
    }
    api.ok = true;
  });
  return api;
}

}  // namespace

using namespace emg;

extern "C" int emg_sparse_solve(int64_t n, int64_t nnz, const int32_t *d_row_ptr, const int32_t *d_col_ind,
                                const void *d_values, const void *d_b, void *d_x, double tol, int reorder,
                                int64_t *h_singularity, emg_stream_t stream) {
  if (!h_singularity) return fail(EMG_EINVAL, "null singularity pointer");
  *h_singularity = -1;
  if (n < 0 || nnz < 0) return fail(EMG_EINVAL, "negative size");
  if (n > INT32_MAX || nnz > INT32_MAX) return fail(EMG_ERANGE, "more than 2^31 - 1 rows or nonzeros");
  if (reorder < 0 || reorder > 3) return fail(EMG_EINVAL, "reorder must be 0 (none), 1 (symrcm), 2 (symamd) or 3 (metis)");
  if (n == 0) return EMG_OK;
  if (!d_row_ptr || !d_values || !d_b || !d_x || (nnz > 0 && !d_col_ind)) return fail(EMG_EINVAL, "null pointer");
  const SpSolverApi &api = sp_api();
  if (!api.ok) return fail(EMG_EDEVICE, "sparse direct solver unavailable: %s", api.err);
  cusolverSpHandle_t h = nullptr;
  if (api.create(&h) != CUSOLVER_STATUS_SUCCESS) return fail(EMG_ECUDA, "cusolverSpCreate failed");
  cusparseMatDescr_t descr = nullptr;
  if (api.descr_create(&descr) != CUSPARSE_STATUS_SUCCESS) {
    api.destroy(h);
    return fail(EMG_ECUDA, "cusparseCreateMatDescr failed");
  }
  api.set_type(descr, CUSPARSE_MATRIX_TYPE_GENERAL);
  api.set_base(descr, CUSPARSE_INDEX_BASE_ZERO);
  int sing = -1;
  cusolverStatus_t s = api.set_stream(h, S(stream));
  if (s == CUSOLVER_STATUS_SUCCESS)
    s = api.zqr(h, (int)n, (int)nnz, descr, static_cast<const cuDoubleComplex *>(d_values), d_row_ptr, d_col_ind,
                static_cast<const cuDoubleComplex *>(d_b), tol, reorder, static_cast<cuDoubleComplex *>(d_x), &sing);
  api.descr_destroy(descr);
  api.destroy(h);
  if (s != CUSOLVER_STATUS_SUCCESS) {
    (void)cudaGetLastError();  // a failed allocation inside cuSOLVER must not surface at a later launch check
    return fail(EMG_ECUDA, "cusolverSpZcsrlsvqr returned status %d%s", (int)s,
                s == CUSOLVER_STATUS_ALLOC_FAILED ? " (out of device memory: the QR factor's fill-in)" : "");
  }
  *h_singularity = sing;
  return EMG_OK;
}
