// OpenCL C -> C++ shim for compiling the reference's OpenCL kernel source on the host CPU.
//
// TEST INFRASTRUCTURE ONLY (part of the oracle).  Together with clexec.cpp it turns the
// reference's own kernel files (src/optical_flow_farneback.cl, src/pyrlkDenseLargeW.cl)
// into host functions, so the C restatement in of_oracle.c can be checked against the
// reference's code instead of against itself.  The kernel files are compiled as they are,
// with this header included first, after three mechanical rewrites done by the Makefile
// (OpenCL vector literals "(float2)(a, b)" become "float2(a, b)"; __local arrays declared
// in a kernel body become static volatile, i.e. shared by the work-items of the group that
// is running; "__local volatile" loses its now repeated qualifier).  Nothing else of the
// source is changed.
//
// What this header supplies:
//  - the address-space and kernel qualifiers (no-ops on the host);
//  - float2 / float4 with the arithmetic and component names the kernels use;
//  - the work-item functions, answered by the executor in clexec.cpp for the fiber that is
//    running; barrier() switches to the next work-item of the group;
//  - mad (fused, fmaf), mad24, convert_int, min/max on int;
//  - image2d_t + read_imagef for a single-channel float image with the one sampler the
//    kernels use (unnormalised coordinates, CLAMP_TO_EDGE, LINEAR).  This is the one
//    piece that is not the reference's code: the OpenCL device filters in hardware with
//    reduced-precision (fixed-point) weights.  Here the texel weights are exact float32
//    values and the four taps are combined in a fixed order (w00*t00, then three fused
//    multiply-adds), the same rule the restatement and the CUDA kernels use.
#pragma once
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>

#define __kernel
#define kernel
#define __global
#define __private
// __local data is volatile here: every access is a load or store of shared memory, so
// values do not travel between statements in registers.  With GCC's contraction (which
// otherwise fuses across statements) this keeps a multiply stored to local memory from
// being fused into a later statement's add: contraction stays within one expression, as
// OpenCL's FP_CONTRACT defines it.
#define __local volatile
#define local volatile
#define __constant const
#define __const const
#define __read_only
#define __write_only
#define CLK_LOCAL_MEM_FENCE 1
#define CLK_GLOBAL_MEM_FENCE 2
#define CLK_NORMALIZED_COORDS_FALSE 0
#define CLK_ADDRESS_CLAMP_TO_EDGE 2
#define CLK_FILTER_LINEAR 16
#define reqd_work_group_size(...) unused

typedef unsigned char uchar;
typedef unsigned short ushort;
typedef unsigned int uint;
typedef int sampler_t;

struct float2 {
  float x, y;
  float2() : x(0.f), y(0.f) {}
  float2(float a, float b) : x(a), y(b) {}
  float2& operator+=(const float2& o) {
    x += o.x;
    y += o.y;
    return *this;
  }
  float2& operator-=(const float2& o) {
    x -= o.x;
    y -= o.y;
    return *this;
  }
};
inline float2 operator+(float2 a, const float2& b) { return a += b; }
inline float2 operator-(float2 a, const float2& b) { return a -= b; }

struct float4 {
  union {
    struct {
      float x, y, z, w;
    };
    struct {
      float s0, s1, s2, s3;
    };
  };
};

// ---- work-item state (clexec.cpp) --------------------------------------------------
namespace clref {
struct Item {
  size_t lid[2], gid[2], lsz[2], ngr[2];
};
extern thread_local const Item* g_item;
void barrier_yield();
}  // namespace clref

inline size_t get_local_id(int d) { return clref::g_item->lid[d]; }
inline size_t get_group_id(int d) { return clref::g_item->gid[d]; }
inline size_t get_local_size(int d) { return clref::g_item->lsz[d]; }
inline size_t get_num_groups(int d) { return clref::g_item->ngr[d]; }
inline size_t get_global_id(int d) { return clref::g_item->gid[d] * clref::g_item->lsz[d] + clref::g_item->lid[d]; }
inline size_t get_global_size(int d) { return clref::g_item->ngr[d] * clref::g_item->lsz[d]; }
inline void barrier(int) { clref::barrier_yield(); }

// ---- built-ins ----------------------------------------------------------------------
inline float mad(float a, float b, float c) { return fmaf(a, b, c); }
inline int mad24(int a, int b, int c) { return a * b + c; }
inline int convert_int(float v) { return (int)v; }
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
// abs(int), floor(float) and fabs(float) are the C++ library's overloads (<math.h>,
// <stdlib.h> in C++ mode), which return the argument's type as OpenCL's do.

// ---- images -------------------------------------------------------------------------
struct clref_image {
  const float* data;
  int width, height;
};
typedef const clref_image* image2d_t;

inline float clref_texel(image2d_t im, int x, int y) {
  x = x < 0 ? 0 : (x > im->width - 1 ? im->width - 1 : x);
  y = y < 0 ? 0 : (y > im->height - 1 ? im->height - 1 : y);
  return im->data[(size_t)y * im->width + x];
}

// Unnormalised coordinates, CLAMP_TO_EDGE, LINEAR (the only sampler the kernels use):
// texel centres at integer + 0.5, exact float32 weights.
inline float4 read_imagef(image2d_t im, sampler_t, float2 c) {
  float xs = c.x - 0.5f, ys = c.y - 0.5f;
  float fx0 = floorf(xs), fy0 = floorf(ys);
  float a = xs - fx0, b = ys - fy0;
  int i0 = (int)fx0, j0 = (int)fy0;
  float t00 = clref_texel(im, i0, j0), t10 = clref_texel(im, i0 + 1, j0);
  float t01 = clref_texel(im, i0, j0 + 1), t11 = clref_texel(im, i0 + 1, j0 + 1);
  float oa = 1.f - a, ob = 1.f - b;
  float w00 = oa * ob, w10 = a * ob, w01 = oa * b, w11 = a * b;
  float r = w00 * t00;
  r = fmaf(w10, t10, r);
  r = fmaf(w01, t01, r);
  r = fmaf(w11, t11, r);
  float4 o;
  o.x = r;
  o.y = 0.f;
  o.z = 0.f;
  o.w = 1.f;
  return o;
}

// ---- per-expression floating-point contraction ---------------------------------------
// OpenCL C contracts a*b+c into one fused multiply-add only within one expression
// (FP_CONTRACT ON, the default); GCC's contraction also fuses across statements, so the
// libraries are compiled with -ffp-contract=off and the kernels' `float` is this type
// instead (clexec.cpp defines `float` as `clf` around the kernel file only).  A product of
// two floats stays unrounded (`prod`) until it is an operand of + or - in the same
// expression, where it fuses (CLREF_CONTRACT=1); anywhere else it rounds.  Operands are
// taken by value so that volatile (__local) operands bind as exact matches.  With two
// products, as in a*b + c*d, the left one fuses and the right one rounds first (the order
// clang-based OpenCL compilers use).  CLREF_CONTRACT=0 rounds every product.
#ifndef CLREF_CONTRACT
#define CLREF_CONTRACT 1
#endif
namespace clref {
struct prod;
struct clf {
  float v;
  clf() = default;
  clf(const clf&) = default;
  clf& operator=(const clf&) = default;
  clf(const volatile clf& o) : v(o.v) {}
  clf& operator=(const volatile clf& o) {
    v = o.v;
    return *this;
  }
  constexpr clf(float x) : v(x) {}
  constexpr clf(int x) : v((float)x) {}
  inline clf(const prod& p);
  operator float() const { return v; }
  operator float() const volatile { return v; }
  void operator=(clf o) volatile { v = o.v; }
  inline clf& operator+=(clf o);
  inline clf& operator-=(clf o);
  inline clf& operator+=(const prod& p);
  inline clf& operator-=(const prod& p);
  clf& operator*=(clf o) {
    v = v * o.v;
    return *this;
  }
  clf& operator/=(clf o) {
    v = v / o.v;
    return *this;
  }
  inline void operator+=(clf o) volatile;
  inline void operator+=(const prod& p) volatile;
};
struct prod {
  float a, b;
  float r() const { return a * b; }
  operator float() const { return a * b; }
};
inline clf::clf(const prod& p) : v(p.r()) {}
inline float fused(const prod& p, float c) { return CLREF_CONTRACT ? fmaf(p.a, p.b, c) : p.r() + c; }
inline clf& clf::operator+=(clf o) {
  v = v + o.v;
  return *this;
}
inline clf& clf::operator-=(clf o) {
  v = v - o.v;
  return *this;
}
inline clf& clf::operator+=(const prod& p) {
  v = fused(p, v);
  return *this;
}
inline clf& clf::operator-=(const prod& p) {
  v = fused(prod{-p.a, p.b}, v);
  return *this;
}
inline void clf::operator+=(clf o) volatile { v = v + o.v; }
inline void clf::operator+=(const prod& p) volatile { v = fused(p, v); }

// products
inline prod operator*(clf a, clf b) { return {a.v, b.v}; }
inline prod operator*(clf a, float b) { return {a.v, b}; }
inline prod operator*(float a, clf b) { return {a, b.v}; }
inline prod operator*(clf a, int b) { return {a.v, (float)b}; }
inline prod operator*(int a, clf b) { return {(float)a, b.v}; }
inline prod operator*(const prod& p, clf b) { return {p.r(), b.v}; }
inline prod operator*(clf a, const prod& q) { return {a.v, q.r()}; }
inline prod operator*(const prod& p, float b) { return {p.r(), b}; }
inline prod operator*(const prod& p, const prod& q) { return {p.r(), q.r()}; }
// sums and differences (a product operand fuses)
#define CLREF_ADDSUB(OP, SGN)                                                                         \
  inline clf operator OP(clf a, clf b) { return clf(a.v OP b.v); }                      \
  inline clf operator OP(clf a, float b) { return clf(a.v OP b); }                             \
  inline clf operator OP(float a, clf b) { return clf(a OP b.v); }                             \
  inline clf operator OP(clf a, int b) { return clf(a.v OP(float) b); }                        \
  inline clf operator OP(int a, clf b) { return clf((float)a OP b.v); }                        \
  inline clf operator OP(const prod& p, clf c) { return clf(fused(p, SGN c.v)); }              \
  inline clf operator OP(const prod& p, float c) { return clf(fused(p, SGN c)); }                     \
  inline clf operator OP(const prod& p, int c) { return clf(fused(p, SGN(float) c)); }                \
  inline clf operator OP(const prod& p, const prod& q) { return clf(fused(p, SGN q.r())); }           \
  inline clf operator OP(clf c, const prod& p) { return clf(fused(prod{SGN p.a, p.b}, c.v)); } \
  inline clf operator OP(float c, const prod& p) { return clf(fused(prod{SGN p.a, p.b}, c)); }
CLREF_ADDSUB(+, +)
CLREF_ADDSUB(-, -)
#undef CLREF_ADDSUB
inline clf operator-(clf a) { return clf(-a.v); }
inline clf operator/(clf a, clf b) { return clf(a.v / b.v); }
inline clf operator/(clf a, float b) { return clf(a.v / b); }
inline clf operator/(float a, clf b) { return clf(a / b.v); }
inline clf operator/(clf a, int b) { return clf(a.v / (float)b); }
inline clf operator/(const prod& p, clf b) { return clf(p.r() / b.v); }
}  // namespace clref
using clref::clf;
