// A10/A11 dense pyramidal Lucas-Kanade (src/pyrlkDenseLargeW.cl:304-669 with
// -DWSX/-DWSY as set by src/denseLucasKanade_PyCL.py:57-71).
//
// The reference runs one 64-work-item group per pixel.  Here one WARP handles one pixel
// and a CTA handles an 8x8 pixel tile whose window data is shared: the intensity patch
// (41x41 with the Scharr border, clamp-to-edge) and its unweighted Scharr gradients
// (39x39) are staged once per CTA in shared memory.  Lane l plays the reference's work
// items l and l+32 (xid = l&7, yid = l>>3 and yid+4), so the first level of the
// reference's 64->1 reduction tree is an in-lane add and the rest are warp shuffles in
// the same pairing: A, b and the error are reduced in exactly the reference's order.
// J is sampled with exact float32 bilinear weights (pixel-centre convention, clamp to
// edge) from a 64x64 region staged per CTA around the tile's mean displaced window, stored
// as (J[y][x], J[y][x+1]) pairs so a bilinear footprint is two 64-bit loads; the gradients
// are stored as (dx, dy) pairs.  A warp whose every footprint of a Newton step lies in the
// region runs the samples without per-sample region tests; others fall back per sample to
// clamped global reads.  Issue bound: ~7e4 FP32 flops per pixel at a 27x27 window and
// 5 Newton steps, about 7 shared-memory reads per sample.
#include <float.h>

#include <type_traits>

#include "common.cuh"

namespace ofb {

constexpr int LK_PT = 8;            // pixel tile edge
constexpr int LK_G = LK_PT + 31;    // gradient positions per axis
constexpr int LK_I = LK_G + 2;      // intensity positions per axis
// Row strides of the staged patches: a warp reads 4 rows of 8 consecutive columns at once,
// so a stride of 8 or 24 (mod 32) banks puts the 4 rows in disjoint banks.
constexpr int LK_IP = 56, LK_GP = 40;  // LK_GP counts float2 (dx, dy) pairs
static_assert(LK_IP >= LK_I && LK_GP >= LK_G && LK_IP % 32 == 24 && LK_GP % 16 == 8, "patch strides");
// J region staged per CTA for the Newton steps: LK_JR x LK_JR texels centred on the tile's
// mean displaced window, row stride LK_JP (72: the 4 rows a warp reads at once fall in
// distinct banks).  Texels hold clamped-coordinate values, so a bilinear footprint inside
// the region reads exactly what the clamped global path reads.
constexpr int LK_JR = 64, LK_JP = 72;  // LK_JP counts float2 texel pairs
static_assert(LK_JP % 16 == 8, "J pair stride");
// dynamic shared memory of the kernel: sJ2 pairs, sD2 pairs, sI
constexpr size_t LK_SMEM = (size_t)LK_JR * LK_JP * 8 + (size_t)LK_G * LK_GP * 8 + (size_t)LK_I * LK_IP * 4;

struct LkParams {
  int ws, hw, aL, aR, aT, aB, niter;
};

// per-axis tile weights of work item `id` (:339-373); base[] feeds the error guards
__device__ __forceinline__ void lk_weights(int id, int ws, int lo, int hi, float w[4], int base[2]) {
  if (ws >= 16) {
    base[0] = 16 + id;
    base[1] = 24 + id;
    w[0] = 1.f;
    w[1] = id == 0 ? (float)(1 - lo) : 1.f;
    w[2] = base[0] < ws - hi ? 1.f : 0.f;
    w[3] = base[1] < ws - hi ? 1.f : 0.f;
  } else {
    base[0] = 8 + id;
    base[1] = 16 + id;
    w[0] = 1.f;
    w[1] = id == 0 ? (float)(1 - lo) : (base[0] < ws - hi ? 1.f : 0.f);
    w[2] = 0.f;
    w[3] = 0.f;
  }
}

__device__ __forceinline__ float lk_bilinear(const float* __restrict__ J, int H, int W, int pitch, float x, float y) {
  float xs = __fsub_rn(x, 0.5f), ys = __fsub_rn(y, 0.5f);
  float fx0 = floorf(xs), fy0 = floorf(ys);
  float a = __fsub_rn(xs, fx0), b = __fsub_rn(ys, fy0);
  int i0 = (int)fx0, j0 = (int)fy0;
  int xa = clampi(i0, 0, W - 1), xb = clampi(i0 + 1, 0, W - 1);
  int ya = clampi(j0, 0, H - 1), yb = clampi(j0 + 1, 0, H - 1);
  float t00 = __ldg(J + (size_t)ya * pitch + xa), t10 = __ldg(J + (size_t)ya * pitch + xb);
  float t01 = __ldg(J + (size_t)yb * pitch + xa), t11 = __ldg(J + (size_t)yb * pitch + xb);
  float oa = __fsub_rn(1.f, a), ob = __fsub_rn(1.f, b);
  float r = __fmul_rn(__fmul_rn(oa, ob), t00);
  r = __fmaf_rn(__fmul_rn(a, ob), t10, r);
  r = __fmaf_rn(__fmul_rn(oa, b), t01, r);
  r = __fmaf_rn(__fmul_rn(a, b), t11, r);
  return r;
}

// The same bilinear sample from the staged region when its 2 x 2 footprint lies inside it
// (rx, ry: footprint origin relative to the region), else from global memory.
__device__ __forceinline__ float lk_bilinear_s(const float2* __restrict__ sJ, const float* __restrict__ J, int H, int W,
                                               int pitch, float x, float y, int ox, int oy) {
  float xs = __fsub_rn(x, 0.5f), ys = __fsub_rn(y, 0.5f);
  float fx0 = floorf(xs), fy0 = floorf(ys);
  float a = __fsub_rn(xs, fx0), b = __fsub_rn(ys, fy0);
  int i0 = (int)fx0, j0 = (int)fy0;
  const int rx = i0 - ox, ry = j0 - oy;
  float t00, t10, t01, t11;
  if ((unsigned)rx <= (unsigned)(LK_JR - 2) && (unsigned)ry <= (unsigned)(LK_JR - 2)) {
    const float2 top = sJ[ry * LK_JP + rx], bot = sJ[(ry + 1) * LK_JP + rx];
    t00 = top.x;
    t10 = top.y;
    t01 = bot.x;
    t11 = bot.y;
  } else {
    int xa = clampi(i0, 0, W - 1), xb = clampi(i0 + 1, 0, W - 1);
    int ya = clampi(j0, 0, H - 1), yb = clampi(j0 + 1, 0, H - 1);
    t00 = __ldg(J + (size_t)ya * pitch + xa);
    t10 = __ldg(J + (size_t)ya * pitch + xb);
    t01 = __ldg(J + (size_t)yb * pitch + xa);
    t11 = __ldg(J + (size_t)yb * pitch + xb);
  }
  float oa = __fsub_rn(1.f, a), ob = __fsub_rn(1.f, b);
  float r = __fmul_rn(__fmul_rn(oa, ob), t00);
  r = __fmaf_rn(__fmul_rn(a, ob), t10, r);
  r = __fmaf_rn(__fmul_rn(oa, b), t01, r);
  r = __fmaf_rn(__fmul_rn(a, b), t11, r);
  return r;
}

// floor(x) for |x| < 2^22, as a float and as an int, on the FMA pipe: x + 1.5 * 2^23 rounded
// toward -inf is floor(x) + 1.5 * 2^23 (that binade's unit is 1), and its low mantissa bits
// hold the integer.
__device__ __forceinline__ float lk_floor(float x, int& i) {
  const float t = __fadd_rd(x, 12582912.0f);
  i = __float_as_int(t) - 0x4B400000;
  return __fsub_rn(t, 12582912.0f);
}

// the reference's reduce tree: (t, t+32) in-lane, then 16, 8, 4, (0+1)+(2+3)
__device__ __forceinline__ float lk_tree(float lo, float hi) {
  float q = __fadd_rn(lo, hi);
  q = __fadd_rn(q, __shfl_down_sync(0xffffffffu, q, 16));
  q = __fadd_rn(q, __shfl_down_sync(0xffffffffu, q, 8));
  q = __fadd_rn(q, __shfl_down_sync(0xffffffffu, q, 4));
  float a = __fadd_rn(q, __shfl_down_sync(0xffffffffu, q, 1));
  float t = __fadd_rn(a, __shfl_down_sync(0xffffffffu, a, 2));
  return __shfl_sync(0xffffffffu, t, 0);
}

// Whether sample (v, ty, tx) of lane (xid, yid) has a non-zero tile weight.
template <bool DEF>
__device__ __forceinline__ bool lk_on(unsigned act, int v, int ty, int tx, int xid, int yid) {
  if (DEF) return (tx < 3 || xid < 3) && (ty < 3 || (v == 0 && yid < 3));
  return (act >> (16 * v + 4 * ty + tx)) & 1u;
}

// DEF: the default window (27 x 27, no asymmetric mask), whose tile-weight pattern is known
// at compile time (and whose registers fit 3 CTAs per SM, 80 per thread): lane (xid, yid)'s 4th column tile is used when xid < 3, its 4th row tile
// of the first half when yid < 3, the 4th row tile of the second half never.
template <bool DEF>
__global__ void __launch_bounds__(256, DEF ? 3 : 2) lk_dense_kernel(const float* __restrict__ I, const float* __restrict__ J,
                                                       float* __restrict__ U, float* __restrict__ V, int H, int W,
                                                       int pitch, LkParams p, uint8_t* __restrict__ status,
                                                       float* __restrict__ err) {
  extern __shared__ float4 lk_dyn[];
  float2* const sJ = reinterpret_cast<float2*>(lk_dyn);  // (J[y][x], J[y][x + 1]) pairs
  float2* const sD = sJ + LK_JR * LK_JP;                 // (dx, dy) pairs
  float* const sI = reinterpret_cast<float*>(sD + LK_G * LK_GP);
  const int i0 = blockIdx.y * LK_PT, j0 = blockIdx.x * LK_PT;
  const int oy = i0 - p.hw - 1, ox = j0 - p.hw - 1;  // image position of sI[0][0]
  for (int t = threadIdx.x; t < LK_I * LK_I; t += blockDim.x) {
    int ly = t / LK_I, lx = t - ly * LK_I;
    sI[ly * LK_IP + lx] = I[(size_t)clampi(oy + ly, 0, H - 1) * pitch + clampi(ox + lx, 0, W - 1)];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < LK_G * LK_G; t += blockDim.x) {
    int gy = t / LK_G, gx = t - gy * LK_G;
    const float* c = sI + (gy + 1) * LK_IP + gx + 1;
#define P(dy, dx) c[(dy) * LK_IP + (dx)]
    float ddx, ddy;
    ddx = __fmaf_rn(__fsub_rn(__fsub_rn(__fadd_rn(P(-1, 1), P(1, 1)), P(-1, -1)), P(1, -1)), 3.0f,
                       __fmul_rn(__fsub_rn(P(0, 1), P(0, -1)), 10.0f));
    ddy = __fmaf_rn(__fsub_rn(__fsub_rn(__fadd_rn(P(1, -1), P(1, 1)), P(-1, -1)), P(-1, 1)), 3.0f,
                       __fmul_rn(__fsub_rn(P(1, 0), P(-1, 0)), 10.0f));
#undef P
    sD[gy * LK_GP + gx] = make_float2(ddx, ddy);
  }
  // J region: centred on the tile centre displaced by the mean initial flow of the tile
  __shared__ float red_u[8], red_v[8];
  {
    float su = 0.f, sv = 0.f;
    if (threadIdx.x < LK_PT * LK_PT) {
      const int yy = min(i0 + (int)(threadIdx.x >> 3), H - 1), xx = min(j0 + (int)(threadIdx.x & 7), W - 1);
      su = U[(size_t)yy * pitch + xx];
      sv = V[(size_t)yy * pitch + xx];
      su = isfinite(su) ? fminf(fmaxf(su, -1e6f), 1e6f) : 0.f;
      sv = isfinite(sv) ? fminf(fmaxf(sv, -1e6f), 1e6f) : 0.f;
    }
    for (int o = 16; o > 0; o >>= 1) {
      su += __shfl_down_sync(0xffffffffu, su, o);
      sv += __shfl_down_sync(0xffffffffu, sv, o);
    }
    if ((threadIdx.x & 31) == 0) {
      red_u[threadIdx.x >> 5] = su;
      red_v[threadIdx.x >> 5] = sv;
    }
  }
  __syncthreads();
  const float mu = (red_u[0] + red_u[1]) * (1.f / 64.f), mv = (red_v[0] + red_v[1]) * (1.f / 64.f);
  const int jox = j0 + LK_PT / 2 + (int)floorf(mu) - LK_JR / 2, joy = i0 + LK_PT / 2 + (int)floorf(mv) - LK_JR / 2;
  for (int t = threadIdx.x; t < LK_JR * LK_JR; t += blockDim.x) {
    const int ly = t / LK_JR, lx = t - ly * LK_JR;
    const float* row = J + (size_t)clampi(joy + ly, 0, H - 1) * pitch;
    sJ[ly * LK_JP + lx] = make_float2(__ldg(row + clampi(jox + lx, 0, W - 1)), __ldg(row + clampi(jox + lx + 1, 0, W - 1)));
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int xid = lane & 7, yid = lane >> 3;
  unsigned act = 0;  // bit 16 v + 4 ty + tx: the sample's tile weight is not 0
  {
    float wx[4], wy0[4], wy1[4];
    int bx[2], by0[2], by1[2];
    lk_weights(xid, p.ws, p.aL, p.aR, wx, bx);
    lk_weights(yid, p.ws, p.aT, p.aB, wy0, by0);
    lk_weights(yid + 4, p.ws, p.aT, p.aB, wy1, by1);
#pragma unroll
    for (int v = 0; v < 2; v++)
#pragma unroll
      for (int ty = 0; ty < 4; ty++)
#pragma unroll
        for (int tx = 0; tx < 4; tx++)
          act |= (unsigned)(__fmul_rn(wx[tx], (v ? wy1 : wy0)[ty]) != 0.f) << (16 * v + 4 * ty + tx);
  }
  const float hw = (float)p.hw;
  const int i = i0 + warp;
  if (i >= H) return;
  for (int c = 0; c < LK_PT; c++) {
    const int j = j0 + c;
    if (j >= W) break;
    const int gyb = warp, gxb = c;  // gradient-tile origin of this pixel's window
    float a11[2] = {0.f, 0.f}, a12[2] = {0.f, 0.f}, a22[2] = {0.f, 0.f};
#pragma unroll
    for (int v = 0; v < 2; v++) {
      const int yy = yid + 4 * v;
#pragma unroll
      for (int ty = 0; ty < 4; ty++)
#pragma unroll
        for (int tx = 0; tx < 4; tx++) {
          if (!lk_on<DEF>(act, v, ty, tx, xid, yid)) continue;  // tile weight 0
          int g = (gyb + ty * 8 + yy) * LK_GP + gxb + tx * 8 + xid;
          // w is 1 here (the tile weights are products of 0 / 1 values and w == 0 is
          // skipped), so the reference's multiplications by w are exact identities
          const float2 d = sD[g];
          const float dx = d.x, dy = d.y;
          a11[v] = __fmaf_rn(dx, dx, a11[v]);
          a12[v] = __fmaf_rn(dx, dy, a12[v]);
          a22[v] = __fmaf_rn(dy, dy, a22[v]);
        }
    }
    float A11 = lk_tree(a11[0], a11[1]), A12 = lk_tree(a12[0], a12[1]), A22 = lk_tree(a22[0], a22[1]);
    const size_t gid = (size_t)i * pitch + j;
    float D = __fmaf_rn(A11, A22, -__fmul_rn(A12, A12));
    if (D < 1.192092896e-07f) {
      if (lane == 0) {
        if (status) status[gid] = 0;
        if (err) err[gid] = 0.f;
      }
      continue;
    }
    A11 = __fdiv_rn(A11, D);
    A12 = __fdiv_rn(A12, D);
    A22 = __fdiv_rn(A22, D);
    float ptx = __fsub_rn(__fadd_rn((float)j, U[gid]), hw), pty = __fsub_rn(__fadd_rn((float)i, V[gid]), hw);
    float lx[4], ly[2][4];
    lx[0] = __fadd_rn(ptx, __fadd_rn((float)xid, 0.5f));
    ly[0][0] = __fadd_rn(pty, __fadd_rn((float)yid, 0.5f));
    ly[1][0] = __fadd_rn(pty, __fadd_rn((float)(yid + 4), 0.5f));
#pragma unroll
    for (int t = 1; t < 4; t++) {
      lx[t] = __fadd_rn(lx[t - 1], 8.0f);
      ly[0][t] = __fadd_rn(ly[0][t - 1], 8.0f);
      ly[1][t] = __fadd_rn(ly[1][t - 1], 8.0f);
    }
    uint8_t st = 1;
    for (int k = 0; k < p.niter; k++) {
      if (ptx < -hw || ptx >= (float)W || pty < -hw || pty >= (float)H) {
        st = 0;
        break;
      }
      // The bilinear sample positions of a Newton step: x parts per column tile, y parts per
      // row tile (the same float32 operations as lk_bilinear_s, computed once per step)
      float xa[4], xoa[4], yb[2][4], yob[2][4];
      int xr[4], yr[2][4];
      unsigned inx = 0, iny = 0;
#pragma unroll
      for (int t = 0; t < 4; t++) {
        // positions here are within a window of the image (the step's range test), so
        // |xs|, |ys| < 2^22 (the ABI caps H, W) and lk_floor is floorf
        int ix;
        const float xs = __fsub_rn(lx[t], 0.5f), fx0 = lk_floor(xs, ix);
        xa[t] = __fsub_rn(xs, fx0);
        xoa[t] = __fsub_rn(1.f, xa[t]);
        xr[t] = ix - jox;
        inx |= ((unsigned)xr[t] <= (unsigned)(LK_JR - 2)) << t;
#pragma unroll
        for (int v = 0; v < 2; v++) {
          int iy;
          const float ys = __fsub_rn(ly[v][t], 0.5f), fy0 = lk_floor(ys, iy);
          yb[v][t] = __fsub_rn(ys, fy0);
          yob[v][t] = __fsub_rn(1.f, yb[v][t]);
          yr[v][t] = iy - joy;
          iny |= ((unsigned)yr[v][t] <= (unsigned)(LK_JR - 2)) << (4 * v + t);
        }
      }
      float b1[2] = {0.f, 0.f}, b2[2] = {0.f, 0.f};
      // The samples of the step; a warp whose every footprint lies inside the staged J
      // region (the common case) runs the variant without the per-sample region test.
      auto samples = [&](auto all_in) {
#pragma unroll
        for (int v = 0; v < 2; v++) {
          const int yy = yid + 4 * v;
#pragma unroll
          for (int ty = 0; ty < 4; ty++)
#pragma unroll
            for (int tx = 0; tx < 4; tx++) {
              if (!lk_on<DEF>(act, v, ty, tx, xid, yid)) continue;  // tile weight 0
              int g = (gyb + ty * 8 + yy) * LK_GP + gxb + tx * 8 + xid;
              float Iv = sI[(gyb + ty * 8 + yy + 1) * LK_IP + gxb + tx * 8 + xid + 1];
              float t00, t10, t01, t11;
              if (decltype(all_in)::value || (((inx >> tx) & (iny >> (4 * v + ty))) & 1u)) {
                const float2* q = sJ + yr[v][ty] * LK_JP + xr[tx];
                const float2 top = q[0], bot = q[LK_JP];
                t00 = top.x;
                t10 = top.y;
                t01 = bot.x;
                t11 = bot.y;
              } else {  // outside the staged region: clamped global reads
                const int i0 = xr[tx] + jox, j0 = yr[v][ty] + joy;
                const int xa0 = clampi(i0, 0, W - 1), xb0 = clampi(i0 + 1, 0, W - 1);
                const int ya0 = clampi(j0, 0, H - 1), yb0 = clampi(j0 + 1, 0, H - 1);
                t00 = __ldg(J + (size_t)ya0 * pitch + xa0);
                t10 = __ldg(J + (size_t)ya0 * pitch + xb0);
                t01 = __ldg(J + (size_t)yb0 * pitch + xa0);
                t11 = __ldg(J + (size_t)yb0 * pitch + xb0);
              }
              float Jv = __fmul_rn(__fmul_rn(xoa[tx], yob[v][ty]), t00);
              Jv = __fmaf_rn(__fmul_rn(xa[tx], yob[v][ty]), t10, Jv);
              Jv = __fmaf_rn(__fmul_rn(xoa[tx], yb[v][ty]), t01, Jv);
              Jv = __fmaf_rn(__fmul_rn(xa[tx], yb[v][ty]), t11, Jv);
              float diff = __fsub_rn(Jv, Iv);  // (Jv - Iv) * w with w == 1
              const float2 d = sD[g];
              b1[v] = __fmaf_rn(diff, d.x, b1[v]);
              b2[v] = __fmaf_rn(diff, d.y, b2[v]);
            }
        }
      };
      if (__all_sync(0xffffffffu, inx == 0xFu && iny == 0xFFu))
        samples(std::true_type());
      else
        samples(std::false_type());
      float B1 = lk_tree(b1[0], b1[1]), B2 = lk_tree(b2[0], b2[1]);
      float dx = __fmul_rn(__fmaf_rn(A12, B2, -__fmul_rn(A22, B1)), 32.0f);
      float dy = __fmul_rn(__fmaf_rn(A12, B1, -__fmul_rn(A11, B2)), 32.0f);
      ptx = __fadd_rn(ptx, dx);
      pty = __fadd_rn(pty, dy);
#pragma unroll
      for (int t = 0; t < 4; t++) {
        lx[t] = __fadd_rn(lx[t], dx);
        ly[0][t] = __fadd_rn(ly[0][t], dy);
        ly[1][t] = __fadd_rn(ly[1][t], dy);
      }
      if (fabsf(dx) < 0.01f && fabsf(dy) < 0.01f) break;
    }
    if (err) {
      // GetError visiting order and guards (:620-653); bits: 1 xBase, 2 yBase, 4 xBase2, 8 yBase2
      const int ord[16] = {0x000, 0x010, 0x100, 0x110, 0x021, 0x121, 0x202, 0x212,
                           0x223, 0x034, 0x134, 0x234, 0x308, 0x318, 0x328, 0x33c};
      float wx[4], wy0[4], wy1[4];  // recomputed here rather than kept live through the steps
      int bx[2], by0[2], by1[2];
      lk_weights(xid, p.ws, p.aL, p.aR, wx, bx);
      lk_weights(yid, p.ws, p.aT, p.aB, wy0, by0);
      lk_weights(yid + 4, p.ws, p.aT, p.aB, wy1, by1);
      float e[2] = {0.f, 0.f};
#pragma unroll
      for (int v = 0; v < 2; v++) {
        const float* wy = v ? wy1 : wy0;
        const int* by = v ? by1 : by0;
        const int yy = yid + 4 * v;
#pragma unroll
        for (int o = 0; o < 16; o++) {
          int ty = ord[o] >> 8, tx = (ord[o] >> 4) & 15, gb = ord[o] & 15;
          if ((gb & 1) && !(bx[0] < p.ws)) continue;
          if ((gb & 2) && !(by[0] < p.ws)) continue;
          if ((gb & 4) && !(bx[1] < p.ws)) continue;
          if ((gb & 8) && !(by[1] < p.ws)) continue;
          float w = __fmul_rn(wx[tx], wy[ty]);
          float Iv = sI[(gyb + ty * 8 + yy + 1) * LK_IP + gxb + tx * 8 + xid + 1];
          float Jv = lk_bilinear_s(sJ, J, H, W, pitch, lx[tx], ly[v][ty], jox, joy);
          float d = __fmul_rn(__fsub_rn(__fdiv_rn(__fmaf_rn(Jv, 16384.f, 256.f), 512.f),
                                        __fdiv_rn(__fmaf_rn(Iv, 16384.f, 256.f), 512.f)),
                              w);
          e[v] = __fadd_rn(e[v], fabsf(d));
        }
      }
      float E = lk_tree(e[0], e[1]);
      if (lane == 0) err[gid] = __fdiv_rn(E, (float)(32 * p.ws * p.ws));
    }
    if (lane == 0) {
      U[gid] = __fsub_rn(__fadd_rn(ptx, hw), (float)j);
      V[gid] = __fsub_rn(__fadd_rn(pty, hw), (float)i);
      if (status) status[gid] = st;
    }
  }
}

}  // namespace ofb

using namespace ofb;

extern "C" int of_lk_dense(const float* I, const float* J, float* U, float* V, int H, int W, int pitch, int half_win,
                           int niter, const int* asym, uint8_t* status, float* err, void* stream) {
  OF_REQUIRE(!bad_plane(I, H, W, pitch) && J && U && V, "of_lk_dense: bad plane");
  OF_REQUIRE(half_win >= 1 && half_win <= 15, "of_lk_dense: half_win must be in 1..15");
  OF_REQUIRE(niter >= 0, "of_lk_dense: niter < 0");
  OF_REQUIRE(H < (1 << 21) && W < (1 << 21), "of_lk_dense: H and W must be below 2^21");
  LkParams p;
  p.ws = 2 * half_win + 1;
  p.hw = (p.ws - 1) >> 1;
  p.aL = asym ? asym[0] : 0;
  p.aR = asym ? asym[1] : 0;
  p.aT = asym ? asym[2] : 0;
  p.aB = asym ? asym[3] : 0;
  // the reference's window masks are 0 / 1 (denseLucasKanade_PyCL.py:75-92); the kernel's
  // tile weights rely on it
  OF_REQUIRE(((p.aL | p.aR | p.aT | p.aB) & ~1) == 0, "of_lk_dense: asym entries must be 0 or 1");
  p.niter = niter;
  dim3 grid((W + LK_PT - 1) / LK_PT, (H + LK_PT - 1) / LK_PT);
  const bool def = p.ws == 27 && !(p.aL | p.aR | p.aT | p.aB);
  cudaError_t e = def ? OF_SMEM_OPT_IN(lk_dense_kernel<true>, LK_SMEM) : OF_SMEM_OPT_IN(lk_dense_kernel<false>, LK_SMEM);
  if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_lk_dense: %s", cudaGetErrorString(e));
  if (def)
    lk_dense_kernel<true><<<grid, 256, LK_SMEM, as_stream(stream)>>>(I, J, U, V, H, W, pitch, p, status, err);
  else
    lk_dense_kernel<false><<<grid, 256, LK_SMEM, as_stream(stream)>>>(I, J, U, V, H, W, pitch, p, status, err);
  return check_launch("of_lk_dense");
}
