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

// The update of region cell i from its window rows U (above), C and D (below):
// hs_sweep_kernel's arithmetic, the 8 neighbours summed in its order.
template <bool FAST>
__device__ __forceinline__ void hq_update(const HqRow<FAST>& U, const HqRow<FAST>& C, const HqRow<FAST>& D, int i,
                                          const float* __restrict__ sfx, const float* __restrict__ sfy,
                                          const float* __restrict__ sft, HqVal<FAST>* __restrict__ du,
                                          HqVal<FAST>* __restrict__ dv, float a2) {
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
  const float den = __fadd_rn(__fadd_rn(a2, __fmul_rn(gxv, gxv)), __fmul_rn(gyv, gyv));
  const float der = __fdiv_rn(num, den);
  du[i] = (HqVal<FAST>)__fsub_rn(ua, __fmul_rn(gxv, der));
  dv[i] = (HqVal<FAST>)__fsub_rn(va, __fmul_rn(gyv, der));
}

// Sweep s of the region: thread t owns column t % RW and walks a band of the rows the sweep
// computes (band t / RW of HQ_THREADS / RW) with a 3-row register window, so each row it
// visits costs one row of loads.  The input and output buffers are distinct (ping-pong), so
// the pointers are restrict: the loads of the next rows may move ahead of this row's
// stores and the rows' float64 chains overlap.  On image borders the neighbour columns and the window's
// outer rows go through the 'mirror' map; inside the image the mapped row is the row.
template <int RW, int RH, int T, bool EDGE, bool FAST>
__device__ __forceinline__ void hq_sweep(const float* __restrict__ sfx, const float* __restrict__ sfy,
                                         const float* __restrict__ sft, const HqVal<FAST>* __restrict__ su,
                                         const HqVal<FAST>* __restrict__ sv, HqVal<FAST>* __restrict__ du,
                                         HqVal<FAST>* __restrict__ dv, int s, int x0, int y0, int H, int W,
                                         float a2) {
  static_assert(HQ_THREADS % RW == 0, "a whole number of bands");
  constexpr int NB = HQ_THREADS / RW;
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

}  // namespace ofb
