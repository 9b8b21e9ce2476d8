// fb_line_inst.cu -- one instantiation of the line kernel.  The Makefile
// compiles this file six times (ComplexF32/F64 x 16-value, 32-value and
// big-prime register budgets) so the instantiations build in parallel.
#include "fb_line.cuh"

#ifndef FB_R
#error "FB_R, FB_CAP, FB_BIG and FB_LAUNCH must be defined"
#endif

namespace fb {

cudaError_t FB_LAUNCH(const LineArgs& a, size_t smem, cudaStream_t s) {
  static int set_bytes[64] = {0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (smem > 48 * 1024 && (dev >= 64 || set_bytes[dev] < (int)smem)) {
    e = cudaFuncSetAttribute(line_kernel<FB_R, FB_CAP, FB_BIG>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e != cudaSuccess) return e;
    if (dev < 64) set_bytes[dev] = 227 * 1024;
  }
  const int64_t nblk = (a.nlines + a.G - 1) / a.G;
  if (nblk <= 0) return cudaSuccess;
  dim3 grid((unsigned)nblk), block(a.T, a.G);
  line_kernel<FB_R, FB_CAP, FB_BIG><<<grid, block, smem, s>>>(a);
  return cudaGetLastError();
}

// Launch ndesc descriptors (device arrays) as one grid of `nblocks` blocks of
// `threads` threads with `smem` bytes of dynamic shared memory each.
cudaError_t FB_LAUNCH_DESC(const LineArgs* descs, const int64_t* bstart, int ndesc,
                           int64_t nblocks, int threads, size_t smem, cudaStream_t s) {
  static int set_bytes[64] = {0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (smem > 48 * 1024 && (dev >= 64 || set_bytes[dev] < (int)smem)) {
    e = cudaFuncSetAttribute(line_kernel_desc<FB_R, FB_CAP, FB_BIG>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    if (e != cudaSuccess) return e;
    if (dev < 64) set_bytes[dev] = 220 * 1024;
  }
  if (nblocks <= 0 || ndesc <= 0) return cudaSuccess;
  line_kernel_desc<FB_R, FB_CAP, FB_BIG><<<dim3((unsigned)nblocks), dim3(threads), smem, s>>>(
      descs, bstart, ndesc);
  return cudaGetLastError();
}

}  // namespace fb
