// fb_fast_inst.cu -- the specialised lengths (compiled once per element type).
//
// Each entry's radix list must equal the planner's radix program for that
// length (fb_plan.cu radix_program); fast_selfcheck() verifies it and the
// planner only uses entries that pass.  T is the number of threads per line.
#include "fb_fast.cuh"

#ifndef FB_R
#error "FB_R and FB_FAST_TABLE must be defined"
#endif

namespace fb {

#define FB_E(L, T, ...)                                                         \
  {L, T, RList<__VA_ARGS__>::n, {__VA_ARGS__},                                 \
   &FastEntry<FB_R, RList<__VA_ARGS__>, T>::launch,                            \
   &FastEntry<FB_R, RList<__VA_ARGS__>, T>::launch_staged,                     \
   (size_t)FastEntry<FB_R, RList<__VA_ARGS__>, T>::LPAD}

static const FastFn kTable[] = {
    FB_E(2, 1, 2),
    FB_E(4, 1, 4),
    FB_E(8, 1, 8),
    FB_E(16, 1, 16),
    FB_E(32, 4, 8, 4),
    FB_E(64, 4, 16, 4),
    FB_E(128, 8, 16, 8),
    FB_E(256, 16, 16, 16),
    FB_E(512, 32, 16, 8, 4),
    FB_E(1024, 64, 16, 16, 4),
    FB_E(2048, 128, 16, 16, 8),
    FB_E(4096, 256, 16, 16, 16),
    FB_E(8192, 512, 16, 16, 8, 4),
#if FB_WIDE_LINES
    FB_E(16384, 512, 16, 16, 16, 4),
#endif
    FB_E(3, 1, 3),
    FB_E(9, 1, 9),
    FB_E(27, 3, 9, 3),
    FB_E(81, 9, 9, 9),
    FB_E(243, 27, 9, 9, 3),
    FB_E(729, 81, 9, 9, 9),
    FB_E(2187, 243, 9, 9, 9, 3),
    FB_E(6561, 512, 9, 9, 9, 9),
    FB_E(1000, 125, 8, 5, 5, 5),
};

const FastFn* FB_FAST_TABLE(int* count) {
  *count = (int)(sizeof(kTable) / sizeof(kTable[0]));
  return kTable;
}

}  // namespace fb
