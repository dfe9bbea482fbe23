// element_inst.cu -- one (material kind, precision) instance of the element
// kernel per object file, selected with -DEMG_KIND=0|1|2 -DEMG_PREC=0|1 so the
// six instances compile in parallel.
#include "element.cuh"

#ifndef EMG_KIND
#error "define EMG_KIND"
#endif
#ifndef EMG_PREC
#error "define EMG_PREC"
#endif

#define EMG_CAT2(a, b, c) a##b##_##c
#define EMG_CAT(a, b, c) EMG_CAT2(a, b, c)

namespace emg {
int EMG_CAT(launch_element_, EMG_KIND, EMG_PREC)(const ElemArgs &a, int out, cudaStream_t s) {
#if EMG_PREC == 0
  return launch_element_k<EMG_KIND, double>(a, out, s);
#else
  return launch_element_k<EMG_KIND, float>(a, out, s);
#endif
}
}  // namespace emg
