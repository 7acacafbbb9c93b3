// A small SIMT emulator for running GPU kernel source as plain C++ on the
// host, so that the oracle's reference harness can execute the reference's
// own SPAI kernels (src/spai_single_dcu.cpp) unmodified.  TEST
// INFRASTRUCTURE ONLY: nothing in the product uses it.
//
// Execution model.  A launch runs its blocks in parallel over the host's
// OpenMP threads; inside a block every thread is a fiber (ucontext) with its
// own stack, and the block's fibers run one at a time.  A scheduler pass
// resumes each live fiber until it reaches __syncthreads() or returns, so one
// pass is one barrier interval: a barrier completes when every thread of the
// block that has not exited has arrived, which is what the reference's
// kernels rely on (warps of one block leave their column loops after
// different numbers of barriers).  Between two barriers the fibers run in
// thread order, which is one of the interleavings the hardware allows.
// __shared__ arrays are thread_local statics: one copy per host thread, shared
// by the fibers of the block that thread is running.  atomicAdd is a plain
// read-modify-write (the fibers of a block never run concurrently, and the
// kernels here only use it on their own column's counter).
#pragma once

#include <ucontext.h>

#include <cstdio>
#include <cstdlib>
#include <functional>
#include <vector>

namespace simt {

struct Dim3 {
  unsigned x = 1, y = 1, z = 1;
};

struct Fiber {
  ucontext_t ctx;
  std::vector<char> stack;
  bool done = true;
};

struct BlockRunner {
  ucontext_t home;
  std::vector<Fiber> fibers;
  int current = 0;
  const std::function<void()>* body = nullptr;
};

inline thread_local Dim3 threadIdx_, blockIdx_, blockDim_, gridDim_;
inline thread_local BlockRunner* runner_ = nullptr;

constexpr size_t kStackBytes = 64 * 1024;

inline void fiber_entry() {
  BlockRunner* r = runner_;
  (*r->body)();
  r->fibers[r->current].done = true;
  // returning switches to uc_link (the scheduler's context)
}

inline void syncthreads() {
  BlockRunner* r = runner_;
  swapcontext(&r->fibers[r->current].ctx, &r->home);
}

// Run body() as grid x block threads (1-D).  blockIdx / threadIdx / blockDim
// / gridDim are set for the body as CUDA would.
inline void launch(unsigned grid, unsigned block, const std::function<void()>& body) {
#pragma omp parallel
  {
    BlockRunner r;
    r.fibers.resize(block);
    for (auto& f : r.fibers) f.stack.resize(kStackBytes);
    r.body = &body;
    runner_ = &r;
    blockDim_.x = block;
    gridDim_.x = grid;
#pragma omp for schedule(dynamic, 1)
    for (long b = 0; b < (long)grid; ++b) {
      blockIdx_.x = (unsigned)b;
      for (unsigned t = 0; t < block; ++t) {
        Fiber& f = r.fibers[t];
        getcontext(&f.ctx);
        f.ctx.uc_stack.ss_sp = f.stack.data();
        f.ctx.uc_stack.ss_size = f.stack.size();
        f.ctx.uc_link = &r.home;
        makecontext(&f.ctx, fiber_entry, 0);
        f.done = false;
      }
      bool live = true;
      while (live) {
        live = false;
        for (unsigned t = 0; t < block; ++t) {
          if (r.fibers[t].done) continue;
          r.current = (int)t;
          threadIdx_.x = t;
          swapcontext(&r.home, &r.fibers[t].ctx);
          live = live || !r.fibers[t].done;
        }
      }
    }
    runner_ = nullptr;
  }
}

}  // namespace simt

// The CUDA/HIP spellings the kernels use.
#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __shared__ static thread_local
#define threadIdx (simt::threadIdx_)
#define blockIdx (simt::blockIdx_)
#define blockDim (simt::blockDim_)
#define gridDim (simt::gridDim_)
#define __syncthreads() simt::syncthreads()

inline int atomicAdd(int* p, int v) {
  int old = *p;
  *p = old + v;
  return old;
}
