// noalloc.cu -- emg_assemble_noalloc: the one-call assembly with its element
// value scratch in a file-scope device array instead of a caller workspace.
//
// Who needs it: callers that cannot allocate device memory at the call site,
// e.g. a plugin running inside another framework's pre-reserved device pool,
// or a latency-bound loop that must not call cudaMalloc/cudaFree (cudaFree
// synchronises the whole device). They still pass inputs and outputs.
#include "common.cuh"

namespace emg {
namespace {

// 96 MiB of element-value scratch, held by every GPU that loads the library
// until the process exits: 28,597 assembled tets in FP64/exact form (3520 B
// of element values per tet, the workspace size of either value layout),
// 57,195 in the mixed form (1760 B).
constexpr size_t kStaticValuesBytes = size_t(96) << 20;
static __device__ __align__(256) unsigned char g_static_values[kStaticValuesBytes];

// Device address of g_static_values in the current device's context. Looked
// up on every call: the lookup is a host-side table read once the module is
// loaded, and a cached address would go stale when the caller resets the
// device (cudaDeviceReset unloads the module; the next lookup loads it
// again). The host-side name is only a stand-in, never a device address.
int static_values_address(void **out) {
  void *p = nullptr;
  CUDA_TRY(cudaGetSymbolAddress(&p, g_static_values));
  *out = p;
  return EMG_OK;
}

}  // namespace
}  // namespace emg

using namespace emg;

extern "C" int emg_assemble_noalloc(const emg_plan *p, const void *d_plan, const int32_t *d_indptr,
                                    const double *d_nodes, int64_t n_nodes, const int32_t *d_tets,
                                    const int32_t *d_tetids, const emg_material *mat, int precision, double ar,
                                    double ai, double br, double bi, void *d_A, int64_t *d_status,
                                    emg_stream_t stream) {
  if (!p) return fail(EMG_EINVAL, "null plan");
  const size_t need = emg_assemble_workspace_size(p->n_assy, precision);
  if (p->n_assy > 0 && need == 0) return fail(EMG_EINVAL, "bad precision %d", precision);
  if (need > kStaticValuesBytes)
    return fail(EMG_ERANGE,
                "emg_assemble_noalloc: %lld assembled tets need %zu bytes of element values, the static "
                "scratch holds %zu (at most %zu tets in this precision); use emg_assemble with a workspace",
                (long long)p->n_assy, need, kStaticValuesBytes,
                kStaticValuesBytes / (need / (size_t)(p->n_assy > 0 ? p->n_assy : 1)));
  void *ws = nullptr;
  int rc = static_values_address(&ws);
  if (rc) return rc;
  // the array keeps the previous call's values: clear the range this call
  // uses so a tet the kernel skips (flagged in the status word) reads zeros
  if (need > 0) CUDA_TRY(cudaMemsetAsync(ws, 0, need, S(stream)));
  return emg_assemble(p, d_plan, d_indptr, d_nodes, n_nodes, d_tets, d_tetids, mat, precision, ar, ai, br, bi, ws,
                      need, d_A, d_status, stream);
}
