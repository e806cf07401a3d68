/*
 * Host emulation of the small part of CUDA C++ that the reference's kernels use, so that
 * their sources compile with g++ and run on the CPU as the oracle's cross-check.
 *
 * TEST INFRASTRUCTURE ONLY (never linked into the product).  Each kernel launch runs every
 * thread of every block on the calling CPU thread: a thread is a ucontext fibre with its
 * own stack, __syncthreads() switches back to the block scheduler, and the scheduler
 * resumes every live fibre once per barrier phase.  That is CUDA's barrier semantics for
 * kernels whose threads all reach the same barriers; warp-synchronous code without
 * barriers is NOT emulated (such kernels are not run through this layer).  __shared__
 * arrays become function-static, which is correct because one block runs at a time.
 */
#pragma once
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <ucontext.h>

#include <functional>
#include <vector>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __shared__ static
#define __constant__

struct uint3 {
  unsigned x, y, z;
};
struct dim3 {
  unsigned x, y, z;
  dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
struct short2 {
  short x, y;
};
struct ushort2 {
  unsigned short x, y;
};
struct char4 {
  signed char x, y, z, w;
};

static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }

namespace emu {

inline uint3 thread_idx{0, 0, 0}, block_idx{0, 0, 0};
inline dim3 block_dim, grid_dim;

struct Fibre {
  ucontext_t ctx;
  std::vector<char> stack;
  uint3 tid;
  bool done = false;
};

inline ucontext_t sched_ctx;
inline Fibre *current = nullptr;
inline const std::function<void()> *body = nullptr;

inline void fibre_entry() {
  (*body)();
  current->done = true;
  swapcontext(&current->ctx, &sched_ctx);
}

inline void barrier() { swapcontext(&current->ctx, &sched_ctx); }

// Runs f() once per CUDA thread of a <<<grid, block>>> launch.
inline void launch(dim3 grid, dim3 block, const std::function<void()> &f, size_t stack_bytes = 1 << 16) {
  grid_dim = grid;
  block_dim = block;
  body = &f;
  const unsigned nthreads = block.x * block.y * block.z;
  std::vector<Fibre> fibres(nthreads);
  for (auto &fb : fibres) fb.stack.resize(stack_bytes);
  for (unsigned bz = 0; bz < grid.z; ++bz)
    for (unsigned by = 0; by < grid.y; ++by)
      for (unsigned bx = 0; bx < grid.x; ++bx) {
        block_idx = {bx, by, bz};
        for (unsigned t = 0; t < nthreads; ++t) {
          Fibre &fb = fibres[t];
          fb.done = false;
          fb.tid = {t % block.x, (t / block.x) % block.y, t / (block.x * block.y)};
          getcontext(&fb.ctx);
          fb.ctx.uc_stack.ss_sp = fb.stack.data();
          fb.ctx.uc_stack.ss_size = fb.stack.size();
          fb.ctx.uc_link = nullptr;
          makecontext(&fb.ctx, fibre_entry, 0);
        }
        for (bool live = true; live;) {  // one pass per barrier phase
          live = false;
          for (auto &fb : fibres) {
            if (fb.done) continue;
            current = &fb;
            thread_idx = fb.tid;
            swapcontext(&sched_ctx, &fb.ctx);
            live |= !fb.done;
          }
        }
      }
  current = nullptr;
}

}  // namespace emu

#define threadIdx (emu::thread_idx)
#define blockIdx (emu::block_idx)
#define blockDim (emu::block_dim)
#define gridDim (emu::grid_dim)
inline void __syncthreads() { emu::barrier(); }

// KLAUNCH(kernel, grid, block, args...) stands for kernel<<<grid, block>>>(args...).
#define KLAUNCH(k, g, b, ...) emu::launch(dim3(g), dim3(b), [&]() { k(__VA_ARGS__); })
