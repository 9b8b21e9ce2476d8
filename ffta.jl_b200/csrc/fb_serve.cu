// fb_serve.cu -- the serving loop's resident kernel: one persistent launch
// driven by a queue of per-transform work descriptors.
//
// FFTA has no serving layer (a batch is a serial loop, src/plan.jl:194-207).
// Here the server (fb_server_* in fb_plan.cu) appends each admitted small
// request of a served length -- contiguous batched lines of 16..4096 (powers
// of two), ComplexF32 or ComplexF64, either direction -- to a descriptor ring
// in mapped pinned host memory and publishes it by advancing the ring's tail.
// One kernel stays resident and serves the ring:
//
//   block 0 (the feeder) polls the host tail, copies new descriptors into a
//     device-memory ring and publishes them with a device tail;
//   every other block (a worker) claims chunks of lines of the current
//     request -- a tagged counter per slot, advanced by compare-and-swap, so a
//     late block can never claim work of a slot's next occupant -- and runs
//     them with the same compile-time stage programs as the specialised
//     direct kernel (fb_fast.cuh), so served results equal a plan's bit for
//     bit; the block that finishes a request's last chunk writes its
//     completion time and status into mapped host memory.
//
// Every wait is bounded.  The feeder ends after `idle_ns` without a new
// descriptor (or when the host asks it to stop), the workers end when the
// feeder has ended and no work is left (or after twice `idle_ns` idle);
// the host relaunches the kernel when a request arrives and none is
// resident.  A descriptor slot that does not hold the request the tail
// promised (a lost or torn write) is waited for at most `desc_wait_ns`;
// then the request is completed with status kPqStatTimeout and skipped.
// No trap, no unbounded spin.
#include <cuda_runtime.h>

#include <atomic>
#include <cstring>
#include <string>
#include <vector>

#include "fb_fast.cuh"
#include "fb_internal.h"

namespace fb {

constexpr int kPqThreads = 256;
constexpr int64_t kPqSlots = int64_t(1) << 16;
constexpr int kPqPrograms = 36;  // (C32, C64) x (forward, backward) x 2^4 .. 2^12
constexpr unsigned long long kPqCountMask = (1ull << 24) - 1;
constexpr int64_t kPqTagMask = (int64_t(1) << 40) - 1;

// A work descriptor: `batch` contiguous lines of the program's length.
struct PDesc {
  const void* in;
  void* out;
  int64_t batch;
  int64_t seq;   // request index + 1: the request this slot holds
  int32_t prog;  // program id (pq_program_id)
  int32_t pad0;
  int64_t pad[3];
};
static_assert(sizeof(PDesc) == 64, "descriptor is 64 bytes");

// A program: its stage twiddle table, the odd-prime table, and the lines per
// block step (G) and per claimed chunk.
struct PProg {
  const void* tw;
  const void* pcs;
  int G, chunk;
  int64_t pad;
};
static_assert(sizeof(PProg) == 32, "program entry is two 16-byte words");

// Host-written control words (mapped pinned memory).
struct PHost {
  int64_t tail;  // descriptors published
  int32_t stop;  // end the kernel once the ring is drained
  int32_t pad;
};

// Device-side state.
struct PShared {
  int64_t dtail;  // descriptors copied into the device ring
  int64_t cur;    // the request whose chunks are being claimed
  int32_t ended;  // the feeder has ended
  int32_t pad;
};

struct PqArgs {
  const PDesc* hring;      // host ring (mapped)
  const PHost* hctl;       // host control (mapped)
  int64_t* hdone;          // per slot: request index + 1 once complete (mapped)
  int64_t* htime;          // per slot: completion time, globaltimer ns (mapped)
  int32_t* hstat;          // per slot: 0, or kPqStat* (mapped)
  PDesc* dring;
  PShared* sh;
  unsigned long long* claim;  // per slot: (request tag << 24) | chunks claimed
  unsigned long long* done;   // per slot: (request tag << 24) | chunks finished
  const PProg* progs;
  uint64_t idle_ns, desc_wait_ns;
};

__device__ __forceinline__ int64_t ld_acquire_sys(const int64_t* p) {
  int64_t v;
  asm volatile("ld.acquire.sys.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ int64_t ld_acquire_gpu(const int64_t* p) {
  int64_t v;
  asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(int64_t* p, int64_t v) {
  asm volatile("st.release.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ int64_t ld_relaxed(const int64_t* p) {
  return *(const volatile int64_t*)p;
}

// Lines [c*chunk, min(batch, (c+1)*chunk)) of a request, G lines per step.
template <typename R, int DIR, class RL, int T>
__device__ __noinline__ void pq_lines(const PDesc& d, const PProg& p, int64_t c,
                                      unsigned char* smraw) {
  typedef cplx<R> C;
  constexpr int L = prog_len<RL>();
  constexpr int LPAD = lpad_of(L);
  constexpr int G = kPqThreads / T;
  const int u = (int)threadIdx.x % T, g = (int)threadIdx.x / T;
  C* buf = (C*)smraw + g * LPAD;
  const int64_t l0 = c * p.chunk;
  const int64_t l1 = l0 + p.chunk < d.batch ? l0 + p.chunk : d.batch;
  for (int64_t l = l0; l < l1; l += G) {
    const int64_t line = l + g;
    const bool ok = line < l1;
    const int64_t li = ok ? line : l0;
    const DirectIn<R> in{(const C*)d.in + li * L, ok};
    const DirectOut<R> out{(C*)d.out + li * L, ok, R(1), true};
    fast_prog<R, DIR, RL, T>(buf, in, out, (const C*)p.tw, (const R*)p.pcs, u);
    __syncthreads();  // the next lines reuse the buffers
  }
}

// Program ids: ((dtype * 2 + backward) * 9 + log2(L) - 4); the radix
// programs are the planner's for these lengths (fb_fast_table.inc).
__device__ __forceinline__ bool pq_run(const PDesc& d, const PProg& p, int64_t c,
                                       unsigned char* sm) {
#define FB_PQ(R, DIR, base)                                                     \
  case base + 0: pq_lines<R, DIR, RList<16>, 1>(d, p, c, sm); return true;       \
  case base + 1: pq_lines<R, DIR, RList<8, 4>, 4>(d, p, c, sm); return true;     \
  case base + 2: pq_lines<R, DIR, RList<16, 4>, 4>(d, p, c, sm); return true;    \
  case base + 3: pq_lines<R, DIR, RList<16, 8>, 8>(d, p, c, sm); return true;    \
  case base + 4: pq_lines<R, DIR, RList<16, 16>, 16>(d, p, c, sm); return true;  \
  case base + 5: pq_lines<R, DIR, RList<16, 8, 4>, 32>(d, p, c, sm); return true; \
  case base + 6: pq_lines<R, DIR, RList<16, 16, 4>, 64>(d, p, c, sm); return true; \
  case base + 7: pq_lines<R, DIR, RList<16, 16, 8>, 128>(d, p, c, sm); return true; \
  case base + 8: pq_lines<R, DIR, RList<16, 16, 16>, 256>(d, p, c, sm); return true;
  switch (d.prog) {
    FB_PQ(float, -1, 0)
    FB_PQ(float, 1, 9)
    FB_PQ(double, -1, 18)
    FB_PQ(double, 1, 27)
    default: return false;
  }
#undef FB_PQ
}

// Claim the next chunk of request r in its slot (tagged counter); false when
// every chunk is taken or the slot has moved on.
__device__ __forceinline__ bool pq_claim(unsigned long long* w_, int64_t r, int64_t nch,
                                         int64_t* c) {
  const unsigned long long tag = (unsigned long long)(r & kPqTagMask);
  unsigned long long w = *(volatile unsigned long long*)w_;
  for (int it = 0; it < 1 << 20; ++it) {
    const unsigned long long wt = w >> 24;
    unsigned long long want;
    if (wt == tag) {
      if ((int64_t)(w & kPqCountMask) >= nch) return false;
      *c = (int64_t)(w & kPqCountMask);
      want = w + 1;
    } else if (wt < tag) {  // the slot's previous occupant: start request r
      *c = 0;
      want = (tag << 24) | 1ull;
    } else {
      return false;
    }
    const unsigned long long old = atomicCAS(w_, w, want);
    if (old == w) return true;
    w = old;
  }
  return false;
}

// Count one finished chunk of request r; returns the chunks finished so far.
__device__ __forceinline__ int64_t pq_count_done(unsigned long long* w_, int64_t r) {
  const unsigned long long tag = (unsigned long long)(r & kPqTagMask);
  unsigned long long w = *(volatile unsigned long long*)w_;
  for (int it = 0; it < 1 << 20; ++it) {
    const unsigned long long want = (w >> 24) == tag ? w + 1 : ((tag << 24) | 1ull);
    const unsigned long long old = atomicCAS(w_, w, want);
    if (old == w) return (int64_t)(want & kPqCountMask);
    w = old;
  }
  return -1;
}

// Completion of request r (slot s) in host memory: time and status first,
// then the done word the host polls.
__device__ __forceinline__ void pq_complete(const PqArgs& a, int64_t s, int64_t r, int32_t st) {
  *(volatile int64_t*)(a.htime + s) = (int64_t)global_ns();
  *(volatile int32_t*)(a.hstat + s) = st;
  __threadfence_system();
  *(volatile int64_t*)(a.hdone + s) = r + 1;
}

__device__ void pq_feeder(const PqArgs& a) {
  __shared__ int64_t s_t;
  __shared__ int s_end;
  const int tid = threadIdx.x;
  int64_t dt = ld_relaxed(&a.sh->dtail);
  uint64_t last = global_ns();
  for (;;) {
    if (tid == 0) {
      const int64_t t = ld_acquire_sys(&a.hctl->tail);
      int end = 0;
      if (t <= dt) {
        if (*(const volatile int32_t*)&a.hctl->stop) end = 1;
        else if (global_ns() - last > a.idle_ns) end = 1;
      }
      s_t = t;
      s_end = end;
    }
    __syncthreads();
    const int64_t t = s_t;
    const int end = s_end;
    if (end) break;
    if (t > dt) {
      for (int64_t r = dt + tid; r < t; r += kPqThreads) {
        const int64_t s = r % kPqSlots;
        const volatile uint4* src = (const volatile uint4*)(a.hring + s);
        uint4* dst = (uint4*)(a.dring + s);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          uint4 v;
          v.x = src[q].x;
          v.y = src[q].y;
          v.z = src[q].z;
          v.w = src[q].w;
          dst[q] = v;
        }
      }
      __threadfence();
      __syncthreads();
      if (tid == 0) st_release_gpu(&a.sh->dtail, t);
      dt = t;
      last = global_ns();
    } else if (tid == 0) {
      __nanosleep(500);
    }
    __syncthreads();
  }
  if (tid == 0) {
    *(volatile int32_t*)&a.sh->ended = 1;
    __threadfence();
  }
}

__device__ void pq_worker(const PqArgs& a, unsigned char* smraw) {
  __shared__ PDesc s_d;
  __shared__ PProg s_p;
  __shared__ int64_t s_r, s_c, s_n;
  __shared__ int s_act;  // 0: nothing, 1: run chunk s_c of s_r, 2: end
  const int tid = threadIdx.x;
  uint64_t idle0 = global_ns();
  for (;;) {
    if (tid == 0) {
      s_act = 0;
      uint64_t desc_t0 = 0;
      int64_t desc_r = -1;
      for (int spin = 0; s_act == 0; ++spin) {
        const int64_t r = ld_relaxed(&a.sh->cur);
        const int64_t t = ld_acquire_gpu(&a.sh->dtail);
        if (r >= t) {
          const bool fed_out = *(const volatile int32_t*)&a.sh->ended != 0;
          if ((fed_out && r >= ld_acquire_gpu(&a.sh->dtail)) ||
              global_ns() - idle0 > 2 * a.idle_ns) {
            s_act = 2;
            break;
          }
          __nanosleep(256);
          continue;
        }
        const int64_t s = r % kPqSlots;
        PDesc d;
        {
          const uint4* src = (const uint4*)(a.dring + s);
          uint4* dst = (uint4*)&d;
#pragma unroll
          for (int q = 0; q < 4; ++q) dst[q] = __ldcg(src + q);
        }
        if (d.seq != r + 1 || d.prog < 0 || d.prog >= kPqPrograms || d.batch < 1) {
          // not the request the tail promised: wait a little, then give up on it
          if (desc_r != r) {
            desc_r = r;
            desc_t0 = global_ns();
          }
          if (global_ns() - desc_t0 > a.desc_wait_ns) {
            if (atomicCAS((unsigned long long*)&a.sh->cur, (unsigned long long)r,
                          (unsigned long long)(r + 1)) == (unsigned long long)r)
              pq_complete(a, s, r, d.seq != r + 1 ? kPqStatTimeout : kPqStatBadProgram);
          }
          continue;
        }
        // the entry is read from L2: the host may have filled it after this
        // block last read the line it shares with other entries
        PProg p;
        ((uint4*)&p)[0] = __ldcg((const uint4*)(a.progs + d.prog));
        ((uint4*)&p)[1] = __ldcg((const uint4*)(a.progs + d.prog) + 1);
        const int64_t nch = (d.batch + p.chunk - 1) / p.chunk;
        int64_t c = 0;
        if (p.tw == nullptr || p.chunk < 1) {
          // no program registered for this id: the request fails, nothing runs
          if (atomicCAS((unsigned long long*)&a.sh->cur, (unsigned long long)r,
                        (unsigned long long)(r + 1)) == (unsigned long long)r)
            pq_complete(a, s, r, kPqStatBadProgram);
          continue;
        }
        if (pq_claim(a.claim + s, r, nch, &c)) {
          s_d = d;
          s_p = p;
          s_r = r;
          s_c = c;
          s_n = nch;
          s_act = 1;
          break;
        }
        atomicCAS((unsigned long long*)&a.sh->cur, (unsigned long long)r,
                  (unsigned long long)(r + 1));
      }
    }
    __syncthreads();
    if (s_act == 2) break;
    const PDesc d = s_d;
    const PProg p = s_p;
    const int64_t r = s_r, c = s_c, nch = s_n;
    pq_run(d, p, c, smraw);
    __syncthreads();
    if (tid == 0) {
      __threadfence();  // this chunk's outputs before its count
      const int64_t s = r % kPqSlots;
      if (pq_count_done(a.done + s, r) == nch) {
        __threadfence_system();
        pq_complete(a, s, r, kPqStatOk);
      }
    }
    idle0 = global_ns();
  }
}

__global__ void __launch_bounds__(kPqThreads, 3) pq_kernel(const PqArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  if (blockIdx.x == 0)
    pq_feeder(a);
  else
    pq_worker(a, smraw);
}

// ------------------------------------------------------------------ host
struct PQueue {
  int device = 0;
  PDesc* hring = nullptr;  // mapped pinned
  PHost* hctl = nullptr;
  int64_t* hdone = nullptr;
  int64_t* htime = nullptr;
  int32_t* hstat = nullptr;
  void* dmem = nullptr;  // device ring, state, counters, programs
  PqArgs args;
  PProg progs[kPqPrograms];
  bool prog_set[kPqPrograms] = {};
  int64_t pushed = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ended = nullptr;
  bool launched = false;
  int nblocks = 0;
  size_t smem = 0;
};

int pq_program_id(int dtype, int dir, int64_t L) {
  int lg = 0;
  while ((int64_t(1) << lg) < L) ++lg;
  if ((int64_t(1) << lg) != L || lg < 4 || lg > 12) return -1;
  if (dtype != 0 && dtype != 1) return -1;
  return (dtype * 2 + (dir > 0 ? 1 : 0)) * 9 + (lg - 4);
}

static int pq_T(int lg) {
  static const int T[9] = {1, 4, 4, 8, 16, 32, 64, 128, 256};
  return T[lg - 4];
}

// Shared memory of the largest program: G lines of lpad_of(L) elements.
static size_t pq_smem_bytes() {
  size_t m = 0;
  for (int lg = 4; lg <= 12; ++lg) {
    const int L = 1 << lg, G = kPqThreads / pq_T(lg);
    m = std::max(m, (size_t)G * lpad_of(L) * 16);
  }
  return m;
}

static cudaError_t pq_fail(const std::string& what, cudaError_t e) {
  set_last_error("persistent queue: " + what + ": " + cudaGetErrorString(e));
  return e;
}

cudaError_t pq_create(PQueue** out, uint64_t idle_ns) {
  *out = nullptr;
  PQueue* q = new PQueue();
  cudaError_t e = cudaGetDevice(&q->device);
  auto host = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaHostAlloc(p, bytes, cudaHostAllocMapped);
    if (e == cudaSuccess) memset(*p, 0, bytes);
  };
  host((void**)&q->hring, sizeof(PDesc) * kPqSlots);
  host((void**)&q->hctl, sizeof(PHost));
  host((void**)&q->hdone, sizeof(int64_t) * kPqSlots);
  host((void**)&q->htime, sizeof(int64_t) * kPqSlots);
  host((void**)&q->hstat, sizeof(int32_t) * kPqSlots);
  const size_t off_sh = sizeof(PDesc) * kPqSlots;
  const size_t off_claim = off_sh + 256;
  const size_t off_done = off_claim + sizeof(unsigned long long) * kPqSlots;
  const size_t off_prog = off_done + sizeof(unsigned long long) * kPqSlots;
  const size_t bytes = off_prog + sizeof(PProg) * kPqPrograms;
  if (e == cudaSuccess) e = cudaMalloc(&q->dmem, bytes);
  if (e == cudaSuccess) e = cudaMemset(q->dmem, 0, bytes);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&q->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&q->ended, cudaEventDisableTiming);
  PqArgs& a = q->args;
  memset(&a, 0, sizeof(a));
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void**)&a.hring, q->hring, 0);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void**)&a.hctl, q->hctl, 0);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void**)&a.hdone, q->hdone, 0);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void**)&a.htime, q->htime, 0);
  if (e == cudaSuccess) e = cudaHostGetDevicePointer((void**)&a.hstat, q->hstat, 0);
  q->smem = pq_smem_bytes();
  int per_sm = 0, nsm = 0;
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(pq_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)q->smem);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pq_kernel, kPqThreads, q->smem);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, q->device);
  if (e == cudaSuccess && per_sm < 1) e = cudaErrorInvalidConfiguration;
  if (e != cudaSuccess) {
    pq_fail("set-up", e);
    cudaGetLastError();
    pq_destroy(q);
    return e;
  }
  char* d = (char*)q->dmem;
  a.dring = (PDesc*)d;
  a.sh = (PShared*)(d + off_sh);
  a.claim = (unsigned long long*)(d + off_claim);
  a.done = (unsigned long long*)(d + off_done);
  a.progs = (const PProg*)(d + off_prog);
  a.idle_ns = idle_ns;
  a.desc_wait_ns = 2000000;  // 2 ms
  // one block per SM: the rest of each SM stays free for the descriptor and
  // plan launches of other requests (two per SM measured 13-15x against
  // 18-19x for one, on the small-request trace)
  q->nblocks = nsm;
  *out = q;
  return cudaSuccess;
}

cudaError_t pq_set_program(PQueue* q, int id, const void* tw, const void* pcs) {
  if (id < 0 || id >= kPqPrograms) return cudaErrorInvalidValue;
  if (q->prog_set[id]) return cudaSuccess;
  const int lg = id % 9 + 4;
  PProg p;
  p.tw = tw;
  p.pcs = pcs;
  p.G = kPqThreads / pq_T(lg);
  // chunks of at least 16384 elements (whole block steps)
  const int steps = std::max(1, 16384 / (p.G << lg));
  p.chunk = p.G * steps;
  q->progs[id] = p;
  cudaError_t e = cudaMemcpy((void*)(q->args.progs + id), &p, sizeof(p), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return pq_fail("program table", e);
  q->prog_set[id] = true;
  return cudaSuccess;
}

bool pq_has_program(const PQueue* q, int id) {
  return id >= 0 && id < kPqPrograms && q->prog_set[id];
}

int64_t pq_slots() { return kPqSlots; }

// Append one request (the caller keeps at most pq_slots() outstanding).
int64_t pq_push(PQueue* q, int prog, const void* in, void* out, int64_t batch, int64_t seq_add) {
  const int64_t r = q->pushed++;
  PDesc& d = q->hring[r % kPqSlots];
  d.in = in;
  d.out = out;
  d.batch = batch;
  d.prog = prog;
  d.seq = r + 1 + seq_add;  // seq_add != 0 only to test a descriptor that never arrives
  return r;
}

// Publish everything pushed so far.
void pq_publish(PQueue* q) {
  std::atomic_thread_fence(std::memory_order_release);
  *(volatile int64_t*)&q->hctl->tail = q->pushed;
}

bool pq_running(PQueue* q) {
  if (!q->launched) return false;
  const cudaError_t e = cudaEventQuery(q->ended);
  if (e == cudaErrorNotReady) return true;
  cudaGetLastError();
  q->launched = false;
  return false;
}

// Make sure a kernel is resident while work is outstanding.
cudaError_t pq_kick(PQueue* q) {
  if (pq_running(q)) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(&q->args.sh->ended, 0, sizeof(int32_t), q->stream);
  if (e != cudaSuccess) return pq_fail("reset", e);
  pq_kernel<<<q->nblocks, kPqThreads, q->smem, q->stream>>>(q->args);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaEventRecord(q->ended, q->stream);
  if (e != cudaSuccess) return pq_fail("launch", e);
  q->launched = true;
  return cudaSuccess;
}

// Completion of request r: 1 (done; *t_ns and *status set), 0 (not yet).
int pq_poll(PQueue* q, int64_t r, int64_t* t_ns, int32_t* status) {
  const int64_t s = r % kPqSlots;
  if (*(volatile int64_t*)(q->hdone + s) != r + 1) return 0;
  std::atomic_thread_fence(std::memory_order_acquire);
  *t_ns = *(volatile int64_t*)(q->htime + s);
  *status = *(volatile int32_t*)(q->hstat + s);
  return 1;
}

void pq_destroy(PQueue* q) {
  if (!q) return;
  if (q->hctl) *(volatile int32_t*)&q->hctl->stop = 1;
  if (q->launched) cudaEventSynchronize(q->ended);  // ends: stop flag, or idle limit
  if (q->ended) cudaEventDestroy(q->ended);
  if (q->stream) cudaStreamDestroy(q->stream);
  if (q->dmem) cudaFree(q->dmem);
  for (void* p : {(void*)q->hring, (void*)q->hctl, (void*)q->hdone, (void*)q->htime,
                  (void*)q->hstat})
    if (p) cudaFreeHost(p);
  delete q;
}

// Device globaltimer now (for the server's clock origin): a one-thread
// kernel writes it into mapped memory on `s`.
__global__ void pq_clock_kernel(int64_t* out) { *(volatile int64_t*)out = (int64_t)global_ns(); }

cudaError_t pq_clock(cudaStream_t s, int64_t* host_mapped_dev, int64_t* host_mapped) {
  *(volatile int64_t*)host_mapped = 0;
  pq_clock_kernel<<<1, 1, 0, s>>>(host_mapped_dev);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  return e;
}

}  // namespace fb
