// fb_fast_inst.cu -- the specialised lengths, one part of the table per
// compilation (the Makefile builds FB_PART = 0..3 for ComplexF32 and F64).
//
// fb_fast_table.inc (generated by gen_fast_table.py) lists each length with
// the planner's radix program for it; the planner only uses an entry whose
// radix list equals its own program for that length.
#include "fb_fast.cuh"

#ifndef FB_R
#error "FB_R, FB_PART and FB_FAST_TABLE must be defined"
#endif

namespace fb {

#define FB_E(L, T, ...)                                                         \
  {L, T, RList<__VA_ARGS__>::n, {__VA_ARGS__},                                 \
   &FastEntry<FB_R, RList<__VA_ARGS__>, T>::launch,                            \
   &FastEntry<FB_R, RList<__VA_ARGS__>, T>::launch_tile,                       \
   (size_t)FastEntry<FB_R, RList<__VA_ARGS__>, T>::LPAD,                       \
   FastEntry<FB_R, RList<__VA_ARGS__>, T>::has_stream                          \
       ? &FastEntry<FB_R, RList<__VA_ARGS__>, T>::launch_stream                \
       : nullptr,                                                              \
   FastEntry<FB_R, RList<__VA_ARGS__>, T>::has_tc                              \
       ? &FastEntry<FB_R, RList<__VA_ARGS__>, T>::launch_tc                    \
       : nullptr,                                                              \
   FastEntry<FB_R, RList<__VA_ARGS__>, T>::has_tile_tc                         \
       ? &FastEntry<FB_R, RList<__VA_ARGS__>, T>::launch_tile_tc               \
       : nullptr,                                                              \
   FastEntry<FB_R, RList<__VA_ARGS__>, T>::TILE_THREADS,                      \
   FastEntry<FB_R, RList<__VA_ARGS__>, T>::has_tma                             \
       ? &FastEntry<FB_R, RList<__VA_ARGS__>, T>::launch_tile_tma              \
       : nullptr,                                                              \
   FastEntry<FB_R, RList<__VA_ARGS__>, T>::has_real                            \
       ? &FastEntry<FB_R, RList<__VA_ARGS__>, T>::launch_real                  \
       : nullptr,                                                              \
   TileThreads<FB_R, T, true>::value}

static const FastFn kTable[] = {
#include "fb_fast_table.inc"
};

const FastFn* FB_FAST_TABLE(int* count) {
  *count = (int)(sizeof(kTable) / sizeof(kTable[0]));
  return kTable;
}

}  // namespace fb
