// The Horn-Schunck sweep on a region held in shared memory, shared by the multi-launch pass
// (hs.cu) and the persistent kernels (hsq.cu): src/HornSchunck.py:61-70 (HS_helper), cell
// for cell the arithmetic of hs_sweep_kernel.
#pragma once

#include <type_traits>

#include "common.cuh"

namespace ofb {

constexpr int HQ_THREADS = 256;  // threads per CTA of the region sweeps

// (u, v) as held in shared memory: float64 copies of the float32 values for the bit-exact
// arithmetic (the reference's float64 stencil sums then need no conversion per
// neighbour), float32 for the float32 averaging.
template <bool FAST>
using HqVal = typename std::conditional<FAST, float, double>::type;

// A thread's window row: the values of columns c - 1, c, c + 1 (mirrored on image borders)
// of one region row, for u and v.
template <bool FAST>
struct HqRow {
  HqVal<FAST> ul, um, ur, vl, vm, vr;
};

template <int RW, bool FAST>
__device__ __forceinline__ void hq_load(HqRow<FAST>& R, const HqVal<FAST>* __restrict__ su,
                                        const HqVal<FAST>* __restrict__ sv, int row, int cm, int c, int cp) {
  const int o = row * RW;
  R.ul = su[o + cm];
  R.um = su[o + c];
  R.ur = su[o + cp];
  R.vl = sv[o + cm];
  R.vm = sv[o + c];
  R.vr = sv[o + cp];
}

// The float32 quotient num / den, correctly rounded, from rd = 1 / (double)den rounded to
// float64: RN32(RN64(num * rd)).  RN64(num * rd) lies within 2^-52 (relative) of num / den.
// A quotient of two float32 values is never that close to a midpoint m = M 2^e (M odd, 25
// bits) of two float32 neighbours unless it equals it, which it cannot: den * m would need
// 25 significant bits for num to have 24, and a non-zero num - den * m is a multiple of
// 2^e ulp(den), i.e. at least 2^-49 of m relative; the same bound holds for the midpoints of
// the subnormal range.  So the last rounding falls on the side of num / den (the
// innocuous-double-rounding argument of S. Figueroa, "When is double rounding innocuous?",
// SIGNUM Newsletter 30(3), 1995).  Zeros, infinities and NaNs give IEEE's answers (rd = inf
// for den = 0, 0 for den = inf), and float64's range holds every product.  No branch: the
// rows of a sweep are one basic block the scheduler interleaves.
__device__ __forceinline__ float hq_div(float num, double rd) { return __double2float_rn(__dmul_rn((double)num, rd)); }

// The update of region cell i from its window rows U (above), C and D (below):
// hs_sweep_kernel's arithmetic, the 8 neighbours summed in its order.  RD: the quotient
// from the cell's float64 reciprocal srd[i] of the denominator (hq_div), else __fdiv_rn;
// both are the correctly rounded float32 quotient.
template <bool FAST, bool RD>
__device__ __forceinline__ void hq_cell(const HqRow<FAST>& U, const HqRow<FAST>& C, const HqRow<FAST>& D, int i,
                                        const float* __restrict__ sfx, const float* __restrict__ sfy,
                                        const float* __restrict__ sft, const double* __restrict__ srd, float a2,
                                        HqVal<FAST>& uo, HqVal<FAST>& vo) {
  float ua, va;
  if constexpr (FAST) {  // float32 averaging: corner and edge sums, one multiply-add each
    const float wcf = 1.0f / 12.0f, wef = 1.0f / 6.0f;
    const float cu = __fadd_rn(__fadd_rn(U.ul, U.ur), __fadd_rn(D.ul, D.ur));
    const float eu = __fadd_rn(__fadd_rn(U.um, D.um), __fadd_rn(C.ul, C.ur));
    const float cv = __fadd_rn(__fadd_rn(U.vl, U.vr), __fadd_rn(D.vl, D.vr));
    const float ev = __fadd_rn(__fadd_rn(U.vm, D.vm), __fadd_rn(C.vl, C.vr));
    ua = __fmaf_rn(cu, wcf, __fmul_rn(eu, wef));
    va = __fmaf_rn(cv, wcf, __fmul_rn(ev, wef));
  } else {
    const double wc = (double)(1.0f / 12.0f), we = (double)(1.0f / 6.0f);
    double a = 0.0, b = 0.0;  // float32 values held as float64: no conversions here
    a = __fma_rn(U.ul, wc, a); b = __fma_rn(U.vl, wc, b);
    a = __fma_rn(U.um, we, a); b = __fma_rn(U.vm, we, b);
    a = __fma_rn(U.ur, wc, a); b = __fma_rn(U.vr, wc, b);
    a = __fma_rn(C.ul, we, a); b = __fma_rn(C.vl, we, b);
    a = __fma_rn(C.ur, we, a); b = __fma_rn(C.vr, we, b);
    a = __fma_rn(D.ul, wc, a); b = __fma_rn(D.vl, wc, b);
    a = __fma_rn(D.um, we, a); b = __fma_rn(D.vm, we, b);
    a = __fma_rn(D.ur, wc, a); b = __fma_rn(D.vr, wc, b);
    ua = (float)a;
    va = (float)b;
  }
  const float gxv = sfx[i], gyv = sfy[i];
  const float num = __fadd_rn(__fadd_rn(__fmul_rn(gxv, ua), __fmul_rn(gyv, va)), sft[i]);
  float der;
  if constexpr (RD) {
    der = hq_div(num, srd[i]);
  } else {
    const float den = __fadd_rn(__fadd_rn(a2, __fmul_rn(gxv, gxv)), __fmul_rn(gyv, gyv));
    der = __fdiv_rn(num, den);
  }
  uo = (HqVal<FAST>)__fsub_rn(ua, __fmul_rn(gxv, der));
  vo = (HqVal<FAST>)__fsub_rn(va, __fmul_rn(gyv, der));
}

// The float64 reciprocal of a cell's denominator a2 + fx^2 + fy^2 (float32 operations in
// hs_sweep_kernel's order), for hq_div.
__device__ __forceinline__ double hq_recip_den(float gx, float gy, float a2) {
  const float den = __fadd_rn(__fadd_rn(a2, __fmul_rn(gx, gx)), __fmul_rn(gy, gy));
  return __drcp_rn((double)den);
}

template <bool FAST>
__device__ __forceinline__ void hq_update(const HqRow<FAST>& U, const HqRow<FAST>& C, const HqRow<FAST>& D, int i,
                                          const float* __restrict__ sfx, const float* __restrict__ sfy,
                                          const float* __restrict__ sft, HqVal<FAST>* __restrict__ du,
                                          HqVal<FAST>* __restrict__ dv, float a2) {
  hq_cell<FAST, false>(U, C, D, i, sfx, sfy, sft, nullptr, a2, du[i], dv[i]);
}

// Sweep s of the region: thread t owns column t % RW and walks a band of the rows the sweep
// computes (band t / RW of NT / RW, NT the CTA's threads) with a 3-row register window, so each row it
// visits costs one row of loads.  The input and output buffers are distinct (ping-pong), so
// the pointers are restrict: the loads of the next rows may move ahead of this row's
// stores and the rows' float64 chains overlap.  On image borders the neighbour columns and the window's
// outer rows go through the 'mirror' map; inside the image the mapped row is the row.
template <int RW, int RH, int T, bool EDGE, bool FAST, int NT = HQ_THREADS>
__device__ __forceinline__ void hq_sweep(const float* __restrict__ sfx, const float* __restrict__ sfy,
                                         const float* __restrict__ sft, const HqVal<FAST>* __restrict__ su,
                                         const HqVal<FAST>* __restrict__ sv, HqVal<FAST>* __restrict__ du,
                                         HqVal<FAST>* __restrict__ dv, int s, int x0, int y0, int H, int W,
                                         float a2) {
  static_assert(NT % RW == 0, "a whole number of bands");
  constexpr int NB = NT / RW;
  const int c = (int)threadIdx.x % RW, band = (int)threadIdx.x / RW;
  if (c < 1 + s || c >= RW - 1 - s) return;
  const int gx = x0 - T + c;
  if (EDGE && (gx < 0 || gx >= W)) return;
  int cm = c - 1, cp = c + 1;
  if (EDGE) {
    cm = mirror1(gx - 1, W) - (x0 - T);
    cp = mirror1(gx + 1, W) - (x0 - T);
  }
  int lo = 1 + s, hi = RH - 1 - s;
  if (EDGE) {  // rows in the image only
    lo = max(lo, T - y0);
    hi = min(hi, H + T - y0);
  }
  const int n = hi - lo;
  if (n <= 0) return;
  const int ra = lo + (n * band) / NB, rb = lo + (n * (band + 1)) / NB;
  if (rb <= ra) return;
  auto row_of = [&](int r) { return EDGE ? mirror1(y0 - T + r, H) - (y0 - T) : r; };
  HqRow<FAST> A, B, C;
  hq_load<RW, FAST>(A, su, sv, row_of(ra - 1), cm, c, cp);
  hq_load<RW, FAST>(B, su, sv, ra, cm, c, cp);
#pragma unroll 1
  for (int r = ra; r < rb; r += 3) {
    hq_load<RW, FAST>(C, su, sv, row_of(r + 1), cm, c, cp);
    hq_update<FAST>(A, B, C, r * RW + c, sfx, sfy, sft, du, dv, a2);
    if (r + 1 < rb) {
      hq_load<RW, FAST>(A, su, sv, row_of(r + 2), cm, c, cp);
      hq_update<FAST>(B, C, A, (r + 1) * RW + c, sfx, sfy, sft, du, dv, a2);
    }
    if (r + 2 < rb) {
      hq_load<RW, FAST>(B, su, sv, row_of(r + 3), cm, c, cp);
      hq_update<FAST>(C, A, B, (r + 2) * RW + c, sfx, sfy, sft, du, dv, a2);
    }
  }
}

// K consecutive rows r0 .. r0 + K - 1 of a thread's column in one basic block: rows r0 - 1
// .. r0 + K are loaded, the K cells computed and stored, so the scheduler overlaps the
// rows' float64 chains instead of running them one after another.
template <int RW, int K, bool EDGE, bool FAST, bool RD, class RowOf>
__device__ __forceinline__ void hq_rows(const float* __restrict__ sfx, const float* __restrict__ sfy,
                                        const float* __restrict__ sft, const double* __restrict__ srd,
                                        const HqVal<FAST>* __restrict__ su, const HqVal<FAST>* __restrict__ sv,
                                        HqVal<FAST>* __restrict__ du, HqVal<FAST>* __restrict__ dv, int r0, int cm,
                                        int c, int cp, float a2, const RowOf& row_of) {
  HqRow<FAST> w[K + 2];
#pragma unroll
  for (int j = 0; j < K + 2; j++) hq_load<RW, FAST>(w[j], su, sv, row_of(r0 - 1 + j), cm, c, cp);
#pragma unroll
  for (int j = 0; j < K; j++) {
    const int i = (r0 + j) * RW + c;
    hq_cell<FAST, RD>(w[j], w[j + 1], w[j + 2], i, sfx, sfy, sft, srd, a2, du[i], dv[i]);
  }
}

// Sweep s of the region, the cells and band partition of hq_sweep, with each band walked in
// chunks of up to HQ_CHUNK rows (hq_rows).  A band is a whole number of warps (RW a multiple
// of 32), so the chunk lengths are warp-uniform.  RD as in hq_cell.
constexpr int HQ_CHUNK = 4;

template <int RW, int RH, int T, bool EDGE, bool FAST, int NT, bool RD>
__device__ __forceinline__ void hq_sweep2(const float* __restrict__ sfx, const float* __restrict__ sfy,
                                          const float* __restrict__ sft, const double* __restrict__ srd,
                                          const HqVal<FAST>* __restrict__ su, const HqVal<FAST>* __restrict__ sv,
                                          HqVal<FAST>* __restrict__ du, HqVal<FAST>* __restrict__ dv, int s, int x0,
                                          int y0, int H, int W, float a2) {
  static_assert(NT % RW == 0 && RW % 32 == 0, "whole bands of whole warps");
  constexpr int NB = NT / RW;
  const int c = (int)threadIdx.x % RW, band = (int)threadIdx.x / RW;
  if (c < 1 + s || c >= RW - 1 - s) return;
  const int gx = x0 - T + c;
  if (EDGE && (gx < 0 || gx >= W)) return;
  int cm = c - 1, cp = c + 1;
  if (EDGE) {
    cm = mirror1(gx - 1, W) - (x0 - T);
    cp = mirror1(gx + 1, W) - (x0 - T);
  }
  int lo = 1 + s, hi = RH - 1 - s;
  if (EDGE) {
    lo = max(lo, T - y0);
    hi = min(hi, H + T - y0);
  }
  const int n = hi - lo;
  if (n <= 0) return;
  const int ra = lo + (n * band) / NB, rb = lo + (n * (band + 1)) / NB;
  auto row_of = [&](int r) { return EDGE ? mirror1(y0 - T + r, H) - (y0 - T) : r; };
#pragma unroll 1
  for (int r0 = ra; r0 < rb; r0 += HQ_CHUNK) {
    switch (min(HQ_CHUNK, rb - r0)) {
      case 4: hq_rows<RW, 4, EDGE, FAST, RD>(sfx, sfy, sft, srd, su, sv, du, dv, r0, cm, c, cp, a2, row_of); break;
      case 3: hq_rows<RW, 3, EDGE, FAST, RD>(sfx, sfy, sft, srd, su, sv, du, dv, r0, cm, c, cp, a2, row_of); break;
      case 2: hq_rows<RW, 2, EDGE, FAST, RD>(sfx, sfy, sft, srd, su, sv, du, dv, r0, cm, c, cp, a2, row_of); break;
      default: hq_rows<RW, 1, EDGE, FAST, RD>(sfx, sfy, sft, srd, su, sv, du, dv, r0, cm, c, cp, a2, row_of); break;
    }
  }
}

}  // namespace ofb
