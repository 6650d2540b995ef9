// Host executor for the reference's OpenCL kernels (TEST INFRASTRUCTURE ONLY).
//
// Runs an NDRange the way an OpenCL device defines it: work-groups one after another, and
// inside a group every work-item as a fiber (its own stack) on one host thread.  barrier()
// switches to the next work-item of the group; a work-item runs again only after every
// work-item of the group has reached the same barrier, so __local data written before a
// barrier is complete when any work-item passes it.  A group in which some work-items
// finish while others wait at a barrier (undefined behaviour in OpenCL) is reported as an
// error.  Global sizes that are not multiples of the work-group size are rounded up to
// whole groups (the kernels guard their global ids), which is what an OpenCL 1.x host must
// do; dynamic __local buffers (clSetKernelArg with a NULL pointer) are filled with NaN at
// the start of each group so a read of unwritten local memory shows in the output.
//
// The translation unit includes ONE reference kernel file, rewritten by the Makefile and
// named by CLREF_SOURCE, with its `float` standing for clshim.hpp's contraction-aware type,
// and exports C entry points with the kernels' own argument lists plus the NDRange (global
// and local sizes, and the dynamic local-memory size).
#include "clshim.hpp"

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <functional>
#include <vector>

namespace clref {

thread_local const Item* g_item = nullptr;

// ---- fibers: callee-saved registers + stack pointer switch (System V x86-64) --------
extern "C" void clref_switch(void** save_sp, void* load_sp);
asm(R"(
.text
.globl clref_switch
.type clref_switch,@function
clref_switch:
  pushq %rbp
  pushq %rbx
  pushq %r12
  pushq %r13
  pushq %r14
  pushq %r15
  movq %rsp, (%rdi)
  movq %rsi, %rsp
  popq %r15
  popq %r14
  popq %r13
  popq %r12
  popq %rbx
  popq %rbp
  ret
.size clref_switch, .-clref_switch
)");

struct Fiber {
  void* sp = nullptr;
  char* stack = nullptr;
  bool done = false;
  Item item;
};

struct Group {
  std::vector<Fiber> fibers;
  void* sched_sp = nullptr;
  Fiber* running = nullptr;
  const std::function<void()>* body = nullptr;
};

thread_local Group* g_group = nullptr;
constexpr size_t kStack = 128 * 1024;

static void fiber_entry() {
  Group* g = g_group;
  (*g->body)();
  g->running->done = true;
  clref_switch(&g->running->sp, g->sched_sp);
  abort();  // a finished fiber is never resumed
}

void barrier_yield() {
  Group* g = g_group;
  clref_switch(&g->running->sp, g->sched_sp);
}

static void prepare(Fiber& f) {
  // stack top 16-byte aligned; after the six pops and the `ret` into fiber_entry the stack
  // pointer is top - 8, as at the entry of a called function
  uintptr_t top = ((uintptr_t)(f.stack + kStack)) & ~(uintptr_t)15;
  void** sp = (void**)top;
  *--sp = nullptr;                     // fake return address of fiber_entry
  *--sp = (void*)&fiber_entry;         // `ret` target
  for (int i = 0; i < 6; i++) *--sp = nullptr;  // rbp rbx r12 r13 r14 r15
  f.sp = sp;
  f.done = false;
}

// Runs `body` for every work-item of an NDRange.  `local_mem` (may be null) is filled with
// NaN before each group.  Returns 0, or -1 when a group's work-items diverged on barriers.
static int run_ndrange(size_t g0, size_t g1, size_t l0, size_t l1, float* local_mem, size_t local_floats,
                       const std::function<void()>& body) {
  if (l0 == 0 || l1 == 0) return -2;
  const size_t n0 = (g0 + l0 - 1) / l0, n1 = (g1 + l1 - 1) / l1, L = l0 * l1;
  Group grp;
  grp.fibers.resize(L);
  for (auto& f : grp.fibers) f.stack = (char*)malloc(kStack);
  grp.body = &body;
  Group* saved = g_group;
  g_group = &grp;
  int rc = 0;
  for (size_t b1 = 0; b1 < n1 && rc == 0; b1++)
    for (size_t b0 = 0; b0 < n0 && rc == 0; b0++) {
      if (local_mem)
        for (size_t i = 0; i < local_floats; i++) local_mem[i] = NAN;
      for (size_t i = 0; i < L; i++) {
        Fiber& f = grp.fibers[i];
        prepare(f);
        f.item.lid[0] = i % l0;
        f.item.lid[1] = i / l0;
        f.item.gid[0] = b0;
        f.item.gid[1] = b1;
        f.item.lsz[0] = l0;
        f.item.lsz[1] = l1;
        f.item.ngr[0] = n0;
        f.item.ngr[1] = n1;
      }
      size_t alive = L;
      while (alive) {
        size_t finished = 0, waiting = 0;
        for (auto& f : grp.fibers) {
          if (f.done) continue;
          grp.running = &f;
          g_item = &f.item;
          clref_switch(&grp.sched_sp, f.sp);
          if (f.done)
            finished++;
          else
            waiting++;
        }
        if (finished && waiting) {
          fprintf(stderr, "clref: work-group (%zu,%zu): %zu work-items returned while %zu wait at a barrier\n", b0,
                  b1, finished, waiting);
          rc = -1;
          break;
        }
        alive -= finished;
      }
    }
  g_group = saved;
  g_item = nullptr;
  for (auto& f : grp.fibers) free(f.stack);
  return rc;
}

}  // namespace clref

// the kernel file's `float` is the contraction-aware clf (clshim.hpp)
#define float clf
#include CLREF_SOURCE
#undef float

using clref::run_ndrange;
#define CF(p) reinterpret_cast<const clf*>(p)
#define MF(p) reinterpret_cast<clf*>(p)
#define LF(p) reinterpret_cast<volatile clf*>(p)
static_assert(sizeof(clf) == sizeof(float), "clf must be layout-compatible with float");

#ifdef CLREF_FARNEBACK
// Entry points with the argument lists of src/optical_flow_farneback.cl.  `ig` points to
// the 4 floats of the float4 argument.
extern "C" int clref_polynomialExpansion(const float* src, int srcStep, float* dst, int dstStep, int rows, int cols,
                                         const float* c_g, const float* c_xg, const float* c_xxg, size_t smem_bytes,
                                         const float* ig, size_t g0, size_t g1, size_t l0, size_t l1) {
  std::vector<float> smem(smem_bytes / 4 + 1);
  float4 v;
  v.s0 = ig[0];
  v.s1 = ig[1];
  v.s2 = ig[2];
  v.s3 = ig[3];
  return run_ndrange(g0, g1, l0, l1, smem.data(), smem.size(), [&] {
    polynomialExpansion(CF(src), srcStep, MF(dst), dstStep, rows, cols, CF(c_g), CF(c_xg), CF(c_xxg), LF(smem.data()), v);
  });
}

extern "C" int clref_gaussianBlur(const float* src, int srcStep, float* dst, int dstStep, int rows, int cols,
                                  const float* c_gKer, int ksizeHalf, size_t smem_bytes, size_t g0, size_t g1, size_t l0,
                                  size_t l1) {
  std::vector<float> smem(smem_bytes / 4 + 1);
  return run_ndrange(g0, g1, l0, l1, smem.data(), smem.size(), [&] {
    gaussianBlur(CF(src), srcStep, MF(dst), dstStep, rows, cols, CF(c_gKer), ksizeHalf, LF(smem.data()));
  });
}

extern "C" int clref_gaussianBlur5(const float* src, int srcStep, float* dst, int dstStep, int rows, int cols,
                                   const float* c_gKer, int ksizeHalf, size_t smem_bytes, size_t g0, size_t g1,
                                   size_t l0, size_t l1) {
  std::vector<float> smem(smem_bytes / 4 + 1);
  return run_ndrange(g0, g1, l0, l1, smem.data(), smem.size(), [&] {
    gaussianBlur5(CF(src), srcStep, MF(dst), dstStep, rows, cols, CF(c_gKer), ksizeHalf, LF(smem.data()));
  });
}

extern "C" int clref_boxFilter5(const float* src, int srcStep, float* dst, int dstStep, int rows, int cols,
                                int ksizeHalf, size_t smem_bytes, size_t g0, size_t g1, size_t l0, size_t l1) {
  std::vector<float> smem(smem_bytes / 4 + 1);
  return run_ndrange(g0, g1, l0, l1, smem.data(), smem.size(), [&] {
    boxFilter5(CF(src), srcStep, MF(dst), dstStep, rows, cols, ksizeHalf, LF(smem.data()));
  });
}

extern "C" int clref_updateMatrices(const float* flowx, int xStep, const float* flowy, int yStep, int rows, int cols,
                                    const float* R0, int R0Step, const float* R1, int R1Step, float* M, int mStep,
                                    size_t g0, size_t g1, size_t l0, size_t l1) {
  return run_ndrange(g0, g1, l0, l1, nullptr, 0, [&] {
    updateMatrices(CF(flowx), xStep, CF(flowy), yStep, rows, cols, CF(R0), R0Step, CF(R1), R1Step, MF(M), mStep);
  });
}

extern "C" int clref_updateFlow(const float* M, int mStep, float* flowx, int xStep, float* flowy, int yStep, int rows,
                                int cols, size_t g0, size_t g1, size_t l0, size_t l1) {
  return run_ndrange(g0, g1, l0, l1, nullptr, 0,
                     [&] { updateFlow(CF(M), mStep, MF(flowx), xStep, MF(flowy), yStep, rows, cols); });
}
#endif

#ifdef CLREF_LK
// Entry point with the argument list of lkDense (src/pyrlkDenseLargeW.cl:304-310); the
// two images are single-channel float32 H x W arrays.
extern "C" int clref_lkDense(const float* I, const float* J, int img_h, int img_w, float* u, float* v, uchar* status,
                             float* err, int level, int rows, int cols, int PATCH_X, int PATCH_Y, int c_winSize_x,
                             int c_winSize_y, int aL, int aR, int aT, int aB, int c_iters, int calcErr, size_t g0,
                             size_t g1, size_t l0, size_t l1) {
  clref_image ii = {I, img_w, img_h}, jj = {J, img_w, img_h};
  return run_ndrange(g0, g1, l0, l1, nullptr, 0, [&] {
    lkDense(&ii, &jj, MF(u), MF(v), status, MF(err), level, rows, cols, PATCH_X, PATCH_Y, c_winSize_x, c_winSize_y, aL, aR, aT, aB,
            c_iters, (char)calcErr);
  });
}
#endif
