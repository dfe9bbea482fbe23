// api.cu -- the extern "C" boundary of libemgpu (declared in include/emgpu.h).
#include "common.cuh"

#include <algorithm>
#include <thread>
#include <vector>

namespace emg {

namespace {
thread_local char g_err[512] = "";
}

int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

const char *last_error() { return g_err; }

namespace {
__global__ void k_probe() {}

int launch_element_batch(const ElemArgs *d_jobs, const int64_t *d_cta_start, int n_jobs, int64_t total, int kind,
                         int precision, int layout, cudaStream_t s) {
  switch (precision * 3 + kind) {
    case 0: return launch_element_batch_0_0(d_jobs, d_cta_start, n_jobs, total, layout, s);
    case 1: return launch_element_batch_0_1(d_jobs, d_cta_start, n_jobs, total, layout, s);
    case 2: return launch_element_batch_0_2(d_jobs, d_cta_start, n_jobs, total, layout, s);
    case 3: return launch_element_batch_1_0(d_jobs, d_cta_start, n_jobs, total, layout, s);
    case 4: return launch_element_batch_1_1(d_jobs, d_cta_start, n_jobs, total, layout, s);
    case 5: return launch_element_batch_1_2(d_jobs, d_cta_start, n_jobs, total, layout, s);
    case 6: return launch_element_batch_2_0(d_jobs, d_cta_start, n_jobs, total, layout, s);
    case 7: return launch_element_batch_2_1(d_jobs, d_cta_start, n_jobs, total, layout, s);
    case 8: return launch_element_batch_2_2(d_jobs, d_cta_start, n_jobs, total, layout, s);
  }
  return fail(EMG_EINVAL, "bad precision %d or kind %d", precision, kind);
}

// table layout of emg_assemble_batch: ElemArgs[n] | int64 cta[n+1] | GatherJob[n] | int64 gcta[n+1]
size_t batch_offset(int n, int part) {
  size_t o = 0;
  const size_t sizes[4] = {sizeof(ElemArgs) * (size_t)n, sizeof(int64_t) * (size_t)(n + 1),
                           sizeof(GatherJob) * (size_t)n, sizeof(int64_t) * (size_t)(n + 1)};
  for (int i = 0; i < part; ++i) o = align_up(o + sizes[i], 16);
  return o;
}

int launch_element(const ElemArgs &a, int kind, int precision, int layout, cudaStream_t s) {
  if (kind < EMG_MAT_ISO || kind > EMG_MAT_FULL) return fail(EMG_EINVAL, "bad material kind %d", kind);
  switch (precision * 3 + kind) {
    case 0: return launch_element_0_0(a, layout, s);
    case 1: return launch_element_0_1(a, layout, s);
    case 2: return launch_element_0_2(a, layout, s);
    case 3: return launch_element_1_0(a, layout, s);
    case 4: return launch_element_1_1(a, layout, s);
    case 5: return launch_element_1_2(a, layout, s);
    case 6: return launch_element_2_0(a, layout, s);
    case 7: return launch_element_2_1(a, layout, s);
    case 8: return launch_element_2_2(a, layout, s);
  }
  return fail(EMG_EINVAL, "bad precision %d", precision);
}
}  // namespace

}  // namespace emg

using namespace emg;

#define EMG_VERSION 1

extern "C" {

int emg_version(void) { return EMG_VERSION; }

const char *emg_last_error(void) { return emg::last_error(); }

// One pass over a complex128 [3][3][nT] tensor array on host threads: is any
// off-diagonal entry nonzero (FULL), are the three diagonals equal tet by
// tet (ISO, else DIAG), and is it the identity. Comparisons are numpy's for
// complex values: nonzero when either part is, equal when both parts are
// (a NaN is nonzero and equal to nothing).
int emg_material_classify(const double *h_t, int64_t n_tets, int n_threads, int *h_kind, int *h_identity) {
  if (!h_kind || !h_identity) return fail(EMG_EINVAL, "null output pointer");
  if (n_tets < 0) return fail(EMG_EINVAL, "negative size");
  if (n_tets > 0 && !h_t) return fail(EMG_EINVAL, "null tensor pointer");
  const int64_t nT = n_tets;
  int nth = n_threads > 0 ? n_threads : (int)std::thread::hardware_concurrency();
  nth = (int)std::max<int64_t>(1, std::min<int64_t>(std::max(nth, 1), nT / 65536));
  struct Flags {
    bool off = false, diag_ne = false, not_one = false;
  };
  std::vector<Flags> fl(nth);
  auto work = [&](int w) {
    const int64_t b = nT * w / nth, e = nT * (w + 1) / nth;
    Flags f;
    for (int c = 0; c < 9 && !f.off; ++c) {
      if (c % 4 == 0) continue;  // diagonal component
      const double *p = h_t + 2 * (int64_t)c * nT;
      for (int64_t t = b; t < e; ++t)
        if (p[2 * t] != 0.0 || p[2 * t + 1] != 0.0) {
          f.off = true;
          break;
        }
    }
    const double *d0 = h_t, *d1 = h_t + 2 * 4 * nT, *d2 = h_t + 2 * 8 * nT;
    for (int64_t t = b; t < e; ++t) {
      const double a0 = d0[2 * t], b0 = d0[2 * t + 1], a1 = d1[2 * t], b1 = d1[2 * t + 1];
      const double a2 = d2[2 * t], b2 = d2[2 * t + 1];
      f.diag_ne |= !(a0 == a1 && b0 == b1 && a1 == a2 && b1 == b2);
      f.not_one |= !(a0 == 1.0 && b0 == 0.0 && a1 == 1.0 && b1 == 0.0 && a2 == 1.0 && b2 == 0.0);
    }
    fl[w] = f;
  };
  std::vector<std::thread> pool;
  for (int w = 1; w < nth; ++w) pool.emplace_back(work, w);
  work(0);
  for (auto &th : pool) th.join();
  bool off = false, diag_ne = false, not_one = false;
  for (const Flags &f : fl) {
    off |= f.off;
    diag_ne |= f.diag_ne;
    not_one |= f.not_one;
  }
  *h_kind = off ? EMG_MAT_FULL : (diag_ne ? EMG_MAT_DIAG : EMG_MAT_ISO);
  *h_identity = (!off && !not_one) ? 1 : 0;
  return EMG_OK;
}

int emg_device_check(int device) {
  cudaDeviceProp p;
  CUDA_TRY(cudaGetDeviceProperties(&p, device));
  if (p.major != 10)
    return fail(EMG_EDEVICE, "device %d is sm_%d%d; this build targets sm_100a", device, p.major, p.minor);
  cudaFuncAttributes fa;
  CUDA_TRY(cudaFuncGetAttributes(&fa, k_probe));
  return EMG_OK;
}

int emg_status_reset(int64_t *d_status, emg_stream_t stream) {
  if (!d_status) return fail(EMG_EINVAL, "null status pointer");
  return status_reset(d_status, S(stream));
}

int emg_status_read(const int64_t *d_status, int64_t *h_flags, int64_t *h_first_index, emg_stream_t stream) {
  if (!d_status || !h_flags || !h_first_index) return fail(EMG_EINVAL, "null pointer");
  int64_t h[2];
  CUDA_TRY(cudaMemcpyAsync(h, d_status, sizeof(h), cudaMemcpyDeviceToHost, S(stream)));
  CUDA_TRY(cudaStreamSynchronize(S(stream)));
  *h_flags = h[0];
  *h_first_index = h[1];
  return EMG_OK;
}

int emg_plan_init(int64_t n_tets, int64_t n_assy, int64_t n_edges, int64_t n_tris, emg_plan *p) {
  if (!p) return fail(EMG_EINVAL, "null plan");
  if (n_tets < 0 || n_assy < 0 || n_edges < 0 || n_tris < 0) return fail(EMG_EINVAL, "negative size");
  if (n_assy > n_tets) return fail(EMG_EINVAL, "n_assy (%lld) > n_tets (%lld)", (long long)n_assy, (long long)n_tets);
  if (n_assy > (int64_t)(INT32_MAX / 400) || n_tets > INT32_MAX || 2 * (n_edges + n_tris) >= INT32_MAX ||
      n_assy * 20 > (int64_t)INT32_MAX / 10)
    return fail(EMG_ERANGE, "mesh too large for 32-bit indexing (n_assy=%lld)", (long long)n_assy);
  memset(p, 0, sizeof(*p));
  p->n_tets = n_tets;
  p->n_assy = n_assy;
  p->n_edges = n_edges;
  p->n_tris = n_tris;
  p->n_ent = n_edges + n_tris;
  p->n_items = 10 * n_assy;
  p->N = 2 * (n_edges + n_tris);
  p->record_bytes = 8;
  p->value_layout = EMG_LAYOUT_PACKED;
  plan_layout(p);
  p->workspace_bytes = plan_workspace_bytes(p);
  return EMG_OK;
}

int emg_plan_set_value_layout(emg_plan *p, int layout) {
  if (!p) return fail(EMG_EINVAL, "null plan");
  if (layout != EMG_LAYOUT_PACKED && layout != EMG_LAYOUT_BLOCK)
    return fail(EMG_EINVAL, "value layout must be EMG_LAYOUT_PACKED or EMG_LAYOUT_BLOCK, got %d", layout);
  if (layout == EMG_LAYOUT_BLOCK && !block_record_fits(p->n_assy))
    return fail(EMG_ERANGE, "block records address at most %lld assembled tets", (long long)((1LL << 31) / 55));
  p->value_layout = layout;
  plan_layout(p);
  p->workspace_bytes = plan_workspace_bytes(p);
  return EMG_OK;
}

int emg_plan_set_record_width(emg_plan *p, int bytes) {
  if (!p) return fail(EMG_EINVAL, "null plan");
  if (bytes != 4 && bytes != 8) return fail(EMG_EINVAL, "record width must be 4 or 8 bytes, got %d", bytes);
  if (bytes == 4 && !pidx_compact_fits(p->n_assy))
    return fail(EMG_ERANGE, "4-byte records address at most %lld assembled tets", (long long)((1LL << 31) / 210));
  p->record_bytes = bytes;
  plan_layout(p);
  p->workspace_bytes = plan_workspace_bytes(p);
  return EMG_OK;
}

int emg_plan_build(emg_plan *p, const int32_t *d_tets, const int32_t *d_t2e, const int32_t *d_t2t,
                   const int32_t *d_tetids, void *d_plan, void *d_ws, int32_t *d_indptr, int64_t *d_status,
                   emg_stream_t stream) {
  if (!p || !d_plan || !d_ws || !d_indptr || !d_status) return fail(EMG_EINVAL, "null pointer");
  if (p->n_assy > 0 && (!d_tets || !d_t2e || !d_t2t)) return fail(EMG_EINVAL, "null topology pointer");
  return plan_build(p, d_tets, d_t2e, d_t2t, d_tetids, d_plan, d_ws, d_indptr, d_status, S(stream));
}

int emg_plan_finish(const emg_plan *p, const int32_t *d_t2e, const int32_t *d_t2t, const int32_t *d_tetids,
                    void *d_plan, const int32_t *d_indptr, int32_t *d_indices, int64_t *d_status,
                    emg_stream_t stream) {
  if (!p || !d_plan || !d_indptr || !d_status) return fail(EMG_EINVAL, "null pointer");
  if (p->nnz > 0 && !d_indices) return fail(EMG_EINVAL, "null indices");
  return plan_finish(p, d_t2e, d_t2t, d_tetids, d_plan, d_indptr, d_indices, d_status, S(stream));
}

int emg_element_values(const double *d_nodes, int64_t n_nodes, const int32_t *d_tets, int64_t n_tets,
                       const int32_t *d_tetids, int64_t n_assy, const emg_material *mat, int precision, int out,
                       int layout, double ar, double ai, double br, double bi, void *d_values, int64_t *d_status,
                       emg_stream_t stream) {
  if (!mat || !mat->d_er) return fail(EMG_EINVAL, "material with a null er pointer");
  if (n_assy < 0 || n_tets < 0 || n_nodes < 0) return fail(EMG_EINVAL, "negative size");
  if (n_assy > 0 && (!d_nodes || !d_tets || !d_values)) return fail(EMG_EINVAL, "null pointer");
  if (n_assy > (int64_t)(INT32_MAX / 400)) return fail(EMG_ERANGE, "too many tets (%lld)", (long long)n_assy);
  if (!d_tetids && n_assy > n_tets) return fail(EMG_EINVAL, "n_assy > n_tets without tetids");
  if (out == EMG_OUT_K) {
    ar = 1.0, ai = 0.0, br = 0.0, bi = 0.0;
  } else if (out == EMG_OUT_M) {
    ar = 0.0, ai = 0.0, br = 1.0, bi = 0.0;
  } else if (out != EMG_OUT_LINCOMB) {
    return fail(EMG_EINVAL, "bad output selector %d", out);
  }
  ElemArgs a{d_nodes, n_nodes, d_tets, n_tets, d_tetids, n_assy, mat->d_er, mat->d_ur, ar, ai, br, bi, d_values,
             d_status};
  return launch_element(a, mat->kind, precision, layout, S(stream));
}

int emg_gather(const emg_plan *p, const void *d_plan, const int32_t *d_indptr, const void *d_v1, const void *d_v2,
               int precision, int layout, double ar, double ai, double br, double bi, void *d_A, int64_t *d_status,
               emg_stream_t stream) {
  if (!p || !d_plan || !d_indptr) return fail(EMG_EINVAL, "null pointer");
  if (p->nnz > 0 && (!d_v1 || !d_A)) return fail(EMG_EINVAL, "null value pointer");
  if ((layout == EMG_LAYOUT_PACKED || layout == EMG_LAYOUT_BLOCK) && d_v2)
    return fail(EMG_EINVAL, "the packed and block layouts take one value array");
  if (layout == EMG_LAYOUT_BLOCK && p->value_layout != EMG_LAYOUT_BLOCK)
    return fail(EMG_EINVAL, "a block-layout gather needs a plan built with EMG_LAYOUT_BLOCK");
  if (layout == EMG_LAYOUT_PACKED && p->value_layout != EMG_LAYOUT_PACKED)
    return fail(EMG_EINVAL, "a packed-layout gather needs a plan built with EMG_LAYOUT_PACKED");
  return launch_gather(p, d_plan, d_indptr, d_v1, d_v2, precision, layout, ar, ai, br, bi, d_A, d_status,
                       S(stream));
}

size_t emg_assemble_workspace_size(int64_t n_assy, int precision) {
  if (n_assy < 0) return 0;
  if (precision < EMG_FP64 || precision > EMG_EXACT) return 0;
  return (size_t)n_assy * kBlockValues * (values_fp32(precision) ? 8 : 16);  // either layout (210 or 220 per tet)
}

int emg_assemble(const emg_plan *p, const void *d_plan, const int32_t *d_indptr, const double *d_nodes,
                 int64_t n_nodes, const int32_t *d_tets, const int32_t *d_tetids, const emg_material *mat,
                 int precision, double ar, double ai, double br, double bi, void *d_ws, size_t ws_bytes, void *d_A,
                 int64_t *d_status, emg_stream_t stream) {
  if (!p) return fail(EMG_EINVAL, "null plan");
  if (p->n_assy > 0 && (!d_ws || ws_bytes < emg_assemble_workspace_size(p->n_assy, precision)))
    return fail(EMG_EINVAL, "workspace too small: %zu < %zu", ws_bytes,
                emg_assemble_workspace_size(p->n_assy, precision));
  const int layout = p->value_layout == EMG_LAYOUT_BLOCK ? EMG_LAYOUT_BLOCK : EMG_LAYOUT_PACKED;
  int rc = emg_element_values(d_nodes, n_nodes, d_tets, p->n_tets, d_tetids, p->n_assy, mat, precision,
                              EMG_OUT_LINCOMB, layout, ar, ai, br, bi, d_ws, d_status, stream);
  if (rc) return rc;
  return emg_gather(p, d_plan, d_indptr, d_ws, nullptr, precision, layout, 1.0, 0.0, 0.0, 0.0, d_A, d_status,
                    stream);
}

size_t emg_assemble_batch_table_bytes(int n_jobs) { return n_jobs < 0 ? 0 : batch_offset(n_jobs, 4); }

int emg_assemble_batch(const emg_assembly_job *h_jobs, int n_jobs, int precision, void *h_table, void *d_table,
                       size_t table_bytes, emg_stream_t stream) {
  if (n_jobs < 0 || (n_jobs > 0 && (!h_jobs || !h_table || !d_table))) return fail(EMG_EINVAL, "null pointer");
  if (precision < EMG_FP64 || precision > EMG_EXACT) return fail(EMG_EINVAL, "bad precision %d", precision);
  if (n_jobs == 0) return EMG_OK;
  if (table_bytes < batch_offset(n_jobs, 4)) return fail(EMG_EINVAL, "table too small");
  char *h = static_cast<char *>(h_table);
  ElemArgs *ea = reinterpret_cast<ElemArgs *>(h + batch_offset(n_jobs, 0));
  int64_t *ecta = reinterpret_cast<int64_t *>(h + batch_offset(n_jobs, 1));
  GatherJob *ga = reinterpret_cast<GatherJob *>(h + batch_offset(n_jobs, 2));
  int64_t *gcta = reinterpret_cast<int64_t *>(h + batch_offset(n_jobs, 3));
  const int kind = h_jobs[0].mat.kind;
  const int layout = h_jobs[0].plan ? h_jobs[0].plan->value_layout : EMG_LAYOUT_PACKED;
  ecta[0] = gcta[0] = 0;
  for (int i = 0; i < n_jobs; ++i) {
    const emg_assembly_job &j = h_jobs[i];
    const emg_plan *p = j.plan;
    if (!p || !j.d_plan || !j.d_indptr || !j.mat.d_er) return fail(EMG_EINVAL, "job %d: null pointer", i);
    if (j.mat.kind != kind) return fail(EMG_EINVAL, "job %d: material kind %d differs from %d", i, j.mat.kind, kind);
    if (p->value_layout != layout)
      return fail(EMG_EINVAL, "job %d: value layout %d differs from %d", i, p->value_layout, layout);
    if (p->n_assy > 0 && (!j.d_nodes || !j.d_tets || !j.d_values || !j.d_A))
      return fail(EMG_EINVAL, "job %d: null pointer", i);
    if (p->n_assy < p->n_tets && !j.d_tetids) return fail(EMG_EINVAL, "job %d: tetids required", i);
    ea[i] = ElemArgs{j.d_nodes, j.n_nodes, j.d_tets, p->n_tets, j.d_tetids, p->n_assy, j.mat.d_er, j.mat.d_ur,
                     j.alpha_re, j.alpha_im, j.beta_re, j.beta_im, j.d_values, j.d_status};
    ecta[i + 1] = ecta[i] + (p->n_assy + 127) / 128;
    int rc = gather_job_fill(p, j.d_plan, j.d_indptr, j.d_values, j.d_A, &ga[i]);
    if (rc) return rc;
    gcta[i + 1] = gcta[i] + (p->n_ent > 0 ? ga[i].n_ctas : 0);
  }
  CUDA_TRY(cudaMemcpyAsync(d_table, h_table, batch_offset(n_jobs, 4), cudaMemcpyHostToDevice, S(stream)));
  const char *d = static_cast<const char *>(d_table);
  int rc = launch_element_batch(reinterpret_cast<const ElemArgs *>(d + batch_offset(n_jobs, 0)),
                                reinterpret_cast<const int64_t *>(d + batch_offset(n_jobs, 1)), n_jobs,
                                ecta[n_jobs], kind, precision, layout, S(stream));
  if (rc) return rc;
  return launch_gather_batch(reinterpret_cast<const GatherJob *>(d + batch_offset(n_jobs, 2)),
                             reinterpret_cast<const int64_t *>(d + batch_offset(n_jobs, 3)), n_jobs, gcta[n_jobs],
                             precision, layout, S(stream));
}

int emg_form_sweep(const void *d_K, const void *d_M, const void *d_P, int64_t nnz, const double *h_coef, int nf,
                   void *d_out, int64_t out_stride, emg_stream_t stream) {
  if (!d_K || !d_M || !h_coef || !d_out || nf < 0 || nnz < 0) return fail(EMG_EINVAL, "null pointer or bad size");
  if (out_stride < nnz) return fail(EMG_EINVAL, "out_stride < nnz");
  return launch_form_sweep(d_K, d_M, d_P, nnz, h_coef, nf, d_out, out_stride, S(stream));
}

int emg_plan_order(const emg_plan *p, void *d_plan, const double *d_nodes, int64_t n_nodes, const int32_t *d_tets,
                   const int32_t *d_tetids, void *d_ws, emg_stream_t stream) {
  if (!p || !d_plan || n_nodes < 0 || (p->n_assy > 0 && (!d_nodes || !d_tets || !d_ws)))
    return fail(EMG_EINVAL, "null pointer or bad size");
  if (p->n_assy > 0 && p->n_assy < p->n_tets && !d_tetids)
    return fail(EMG_EINVAL, "tetids required when n_assy < n_tets");
  return plan_order(p, d_plan, d_nodes, n_nodes, d_tets, d_tetids, d_ws, S(stream));
}

int emg_form_batch(const emg_form_item *d_items, const int64_t *d_tile_start, const int32_t *d_n_items, int max_items,
                   emg_stream_t stream) {
  if (!d_items || !d_tile_start || !d_n_items || max_items <= 0) return fail(EMG_EINVAL, "null pointer or max_items");
  return launch_form_batch(d_items, d_tile_start, d_n_items, max_items, S(stream));
}

}  // extern "C"
