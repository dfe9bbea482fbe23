// element_inst.cu -- one (form, material kind) instance of the element kernel
// per object file, selected with -DEMG_FORM=0|1|2 -DEMG_KIND=0|1|2, so the
// nine instances compile in parallel.
#include "element.cuh"

#ifndef EMG_FORM
#error "define EMG_FORM"
#endif
#ifndef EMG_KIND
#error "define EMG_KIND"
#endif

#define EMG_CAT2(a, b, c) a##b##_##c
#define EMG_CAT(a, b, c) EMG_CAT2(a, b, c)

namespace emg {
int EMG_CAT(launch_element_, EMG_FORM, EMG_KIND)(const ElemArgs &a, int layout, cudaStream_t s) {
  return launch_element_k<EMG_FORM, EMG_KIND>(a, layout, s);
}
int EMG_CAT(launch_element_batch_, EMG_FORM, EMG_KIND)(const ElemArgs *d_jobs, const int64_t *d_cta_start,
                                                       int n_jobs, int64_t total_ctas, int layout, cudaStream_t s) {
  if (layout == EMG_LAYOUT_BLOCK)
    return launch_element_batch_t<EMG_FORM, EMG_KIND, 2>(d_jobs, d_cta_start, n_jobs, total_ctas, s);
  if (layout == EMG_LAYOUT_PACKED)
    return launch_element_batch_t<EMG_FORM, EMG_KIND, 1>(d_jobs, d_cta_start, n_jobs, total_ctas, s);
  return fail(EMG_EINVAL, "batched assembly takes the packed or block layout, got %d", layout);
}
}  // namespace emg
