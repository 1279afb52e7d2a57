// Host emulation of whole CUDA thread blocks for the kernels of
// feram_b200/csrc/fg_kernels.cuh: the threads of a block are user-level
// fibers (ucontext) on one OS thread, switched at __syncthreads() and at
// warp shuffles: a fiber runs until it reaches one of them, a barrier
// releases when every live thread of the block has reached it, a shuffle
// when every live lane of the warp has written its value (and again when
// every lane has read).  __shared__ variables are function statics (one
// block runs at a time), the dynamic shared memory is one aligned buffer per
// launch, blocks run one after another in grid order.  The inline-PTX
// helpers of fg_common.cuh are replaced (FG_HOST_EMU) by their plain
// meaning: copies, loads, no-op waits.  Enough to run a kernel's own index
// arithmetic and data flow on the host against an exact reference, not to
// time anything.
#pragma once
#define FG_HOST_EMU 1
#include <cuda_runtime.h>

#include <atomic>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <cstdio>
#include <functional>
#include <vector>

#include <ucontext.h>

#include <cmath>

#undef __shared__
#define __shared__ static
#ifndef __noinline__
#define __noinline__ __attribute__((noinline))
#endif
#undef __launch_bounds__
#define __launch_bounds__(...)
using std::isfinite;
using std::log;
using std::sqrt;

inline uint3 threadIdx;  // of the fiber running now
inline uint3 blockIdx;
inline dim3 blockDim, gridDim;

namespace emu {
enum Wait : int { RUN = 0, BARRIER, SHFL_W, SHFL_R, DONE };
struct Fiber {
  ucontext_t ctx;
  int wait = RUN;
};
struct Block {
  unsigned nt = 0, cur = 0;
  std::vector<Fiber> f;
  ucontext_t sched;
  std::vector<unsigned long long> xchg;  // one 8-byte slot per thread
};
inline Block* g_block = nullptr;
inline unsigned char* g_dyn = nullptr;
inline std::function<void()> g_body;

// leave the running fiber until the scheduler releases `w`
inline void yield_as(int w) {
  Block& B = *g_block;
  Fiber& F = B.f[B.cur];
  F.wait = w;
  swapcontext(&F.ctx, &B.sched);
}
}  // namespace emu

#define FG_DYN_SMEM(name) unsigned char* name = emu::g_dyn

inline void __syncthreads() { emu::yield_as(emu::BARRIER); }
inline void __threadfence() {}
template <class T>
inline T __ldg(const T* p) { return *p; }
template <class T>
inline T __ldcg(const T* p) { return *p; }
inline unsigned atomicAdd(unsigned* a, unsigned v) {
  const unsigned o = *a;
  *a = o + v;
  return o;
}
inline int atomicCAS(int* a, int cmp, int v) {
  const int o = *a;
  if (o == cmp) *a = v;
  return o;
}
template <class T>
inline T __shfl_down_sync(unsigned, T v, unsigned delta, int = 32) {
  static_assert(sizeof(T) <= 8, "8-byte exchange slots");
  emu::Block& B = *emu::g_block;
  const unsigned t = threadIdx.x, lane = t & 31u;
  std::memcpy(&B.xchg[t], &v, sizeof(T));
  emu::yield_as(emu::SHFL_W);
  T r = v;
  if (lane + delta < 32u) std::memcpy(&r, &B.xchg[t + delta], sizeof(T));
  emu::yield_as(emu::SHFL_R);
  return r;
}

#include "fg_common.cuh"

namespace fg {
template <int BYTES>
inline void cp_async(void* smem, const void* gmem) { std::memcpy(smem, gmem, BYTES); }
inline void cp_async_wait() {}
inline unsigned long long l2_evict_first() { return 0; }
inline void cp_async16_first(void* smem, const void* gmem, unsigned long long) { std::memcpy(smem, gmem, 16); }
inline float2 ld_first(const float2* a, unsigned long long) { return *a; }
inline double2 ld_first(const double2* a, unsigned long long) { return *a; }
inline float4 ld_first(const float4* a, unsigned long long) { return *a; }
inline void cp_async_commit() {}
template <int N>
inline void cp_async_wait_group() {}
inline void pdl_enter() {}
}  // namespace fg

namespace emu {
inline void fiber_entry() {
  g_body();
  g_block->f[g_block->cur].wait = DONE;  // uc_link returns to the scheduler
}

// Run one block: every fiber until it waits, then release what can go on.
inline void run_block(Block& B, char* stacks, size_t stack_bytes) {
  for (unsigned t = 0; t < B.nt; ++t) {
    Fiber& F = B.f[t];
    getcontext(&F.ctx);
    F.ctx.uc_stack.ss_sp = stacks + (size_t)t * stack_bytes;
    F.ctx.uc_stack.ss_size = stack_bytes;
    F.ctx.uc_link = &B.sched;
    makecontext(&F.ctx, fiber_entry, 0);
    F.wait = RUN;
  }
  for (;;) {
    for (unsigned t = 0; t < B.nt; ++t)
      if (B.f[t].wait == RUN) {
        B.cur = t;
        threadIdx = make_uint3(t, 0, 0);
        swapcontext(&B.sched, &B.f[t].ctx);
      }
    // release: warps whose live lanes all reached the same shuffle step,
    // else the block barrier once every live thread waits at it
    bool any = false, all_done = true, all_barrier = true;
    for (unsigned w0 = 0; w0 < B.nt; w0 += 32) {
      const unsigned w1 = std::min(B.nt, w0 + 32);
      int step = -1;
      bool same = true;
      for (unsigned t = w0; t < w1; ++t) {
        const int s = B.f[t].wait;
        if (s == DONE) continue;
        all_done = false;
        if (s != BARRIER) all_barrier = false;
        if (s != SHFL_W && s != SHFL_R) same = false;
        else if (step < 0) step = s;
        else if (step != s) same = false;
      }
      if (same && step >= 0) {
        for (unsigned t = w0; t < w1; ++t)
          if (B.f[t].wait == step) B.f[t].wait = RUN;
        any = true;
      }
    }
    if (all_done) return;
    if (!any && all_barrier) {
      for (unsigned t = 0; t < B.nt; ++t)
        if (B.f[t].wait == BARRIER) B.f[t].wait = RUN;
      any = true;
    }
    if (!any) {
      std::fprintf(stderr, "emulated block (%u,%u,%u): threads wait at different barriers\n", blockIdx.x, blockIdx.y,
                   blockIdx.z);
      std::abort();
    }
  }
}

// kern<<<grid, block, smem>>>(args...), one block at a time in grid order;
// a 1-D block.
template <class... KArgs, class... Args>
void launch(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, Args... args) {
  const unsigned nt = block.x;
  gridDim = grid;
  blockDim = block;
  const size_t bytes = (smem + 127) / 128 * 128 + 128;
  unsigned char* dyn = static_cast<unsigned char*>(std::aligned_alloc(128, bytes));
  std::memset(dyn, 0xff, bytes);  // uninitialised shared memory reads as NaN
  g_dyn = dyn;
  const size_t stack_bytes = 256 * 1024;
  char* stacks = static_cast<char*>(std::malloc(stack_bytes * nt));
  g_body = [&] { kern(args...); };
  Block B;
  B.nt = nt;
  B.f.resize(nt);
  B.xchg.assign(nt, 0);
  g_block = &B;
  for (unsigned bz = 0; bz < grid.z; ++bz)
    for (unsigned by = 0; by < grid.y; ++by)
      for (unsigned bx = 0; bx < grid.x; ++bx) {
        blockIdx = make_uint3(bx, by, bz);
        run_block(B, stacks, stack_bytes);
      }
  g_block = nullptr;
  g_body = nullptr;
  std::free(stacks);
  std::free(dyn);
  g_dyn = nullptr;
}
}  // namespace emu
