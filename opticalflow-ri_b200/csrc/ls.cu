// A8/A9 Liu-Shen physics-based optimiser (src/PhysicsBasedOpticalFlowLiuShen.py:33-158),
// bit-exact with the reference's float32 fields.
//
// Set-up: per-frame maxima (order-preserving atomicMax), normalised frames I1 = im1/max,
// I2 = im2/max and Et = I2 - I1, then the eight per-pixel coefficient planes
// (IIx, IIy, II, Ixt, Iyt and B = A^-1) exactly as the reference's float32 expressions.
// Sweep: the twelve 3x3 stencils of bu / bv (double accumulation over the non-zero
// weights in C order, rounded to float32; 'nearest' borders, 'constant' 0 for H), the
// float32 combination in the reference's order, u <- -(B11 bu + B12 bv), v <- ...,
// and the squared change reduced in double for the convergence test.
// Stop rule (:141): sweep k runs only while err_{k-1} > tol; every sweep kernel reads the
// previous sweep's error from device memory, so the host enqueues maxnum sweeps with no
// synchronisation and the sequence can be captured in a CUDA graph.
// Inside the solver u is the row (y) component and v the column (x) component (:38-39).
#include <stdlib.h>

#include "common.cuh"
#include "tma.cuh"

namespace ofb {

struct LsCtrl {
  unsigned int maxkey[2];
  int K;          // sweeps run (written by the pass that ends the loop)
  int final_buf;  // ping-pong buffer holding the last pass's result
};
// Workspace after LsCtrl: int run[maxnum+1] (run[k] != 0: sweep k runs; run[0] is unused),
// unsigned done[maxnum] (blocks finished per sweep), double ss[maxnum][2] (squared changes).

__device__ __forceinline__ unsigned int f2key(float f) {
  unsigned int b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key2f(unsigned int k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// The largest value of each frame (as order-preserving keys): one CTA per row, rows
// strided over the grid, float4 loads when the rows are 16-byte aligned.  max is exact and
// order-free, so the traversal does not change the result.
__global__ void __launch_bounds__(256) ls_max_kernel(const float* __restrict__ a, const float* __restrict__ b, int H,
                                                     int W, int pitch, int vec, unsigned int* keys) {
  unsigned int ka = 0, kb = 0;
  for (int y = blockIdx.x; y < H; y += gridDim.x) {
    const float* ra = a + (size_t)y * pitch;
    const float* rb = b + (size_t)y * pitch;
    int x = threadIdx.x;
    if (vec) {
      const int W4 = W >> 2;
      for (; x < W4; x += blockDim.x) {
        const float4 va = __ldg(reinterpret_cast<const float4*>(ra) + x);
        const float4 vb = __ldg(reinterpret_cast<const float4*>(rb) + x);
        ka = max(ka, max(max(f2key(va.x), f2key(va.y)), max(f2key(va.z), f2key(va.w))));
        kb = max(kb, max(max(f2key(vb.x), f2key(vb.y)), max(f2key(vb.z), f2key(vb.w))));
      }
      x = 4 * W4 + threadIdx.x;
    }
    for (; x < W; x += blockDim.x) {
      ka = max(ka, f2key(ra[x]));
      kb = max(kb, f2key(rb[x]));
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    ka = max(ka, __shfl_down_sync(0xffffffffu, ka, o));
    kb = max(kb, __shfl_down_sync(0xffffffffu, kb, o));
  }
  __shared__ unsigned int sa[8], sb[8];
  if ((threadIdx.x & 31) == 0) {
    sa[threadIdx.x >> 5] = ka;
    sb[threadIdx.x >> 5] = kb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {  // one atomic per block
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
      ka = max(ka, sa[w]);
      kb = max(kb, sb[w]);
    }
    atomicMax(keys, ka);
    atomicMax(keys + 1, kb);
  }
}

__device__ __forceinline__ double dacc(double a, float v, double w) { return __dadd_rn(a, __dmul_rn((double)v, w)); }
__device__ __forceinline__ double dadd(double a, float v) { return __dadd_rn(a, (double)v); }

// 3x3 neighbourhood with 'nearest' borders, p[r][c] = P[y-1+r][x-1+c]
struct Nb3 {
  float p[3][3];
  __device__ __forceinline__ void load(const float* __restrict__ P, int y, int x, int H, int W, int pitch) {
    int ys[3] = {clampi(y - 1, 0, H - 1), y, clampi(y + 1, 0, H - 1)};
    int xs[3] = {clampi(x - 1, 0, W - 1), x, clampi(x + 1, 0, W - 1)};
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
      for (int c = 0; c < 3; c++) p[r][c] = P[(size_t)ys[r] * pitch + xs[c]];
  }
  __device__ __forceinline__ float dy() const { return (float)dacc(dacc(0.0, p[0][1], -0.5), p[2][1], 0.5); }
  __device__ __forceinline__ float dx() const { return (float)dacc(dacc(0.0, p[1][0], -0.5), p[1][2], 0.5); }
  __device__ __forceinline__ float fy() const { return (float)dadd(dadd(0.0, p[0][1]), p[2][1]); }
  __device__ __forceinline__ float fx() const { return (float)dadd(dadd(0.0, p[1][0]), p[1][2]); }
  __device__ __forceinline__ float m() const {
    return (float)dacc(dacc(dacc(dacc(0.0, p[0][0], 0.25), p[0][2], -0.25), p[2][0], -0.25), p[2][2], 0.25);
  }
  __device__ __forceinline__ float d2y() const {
    return (float)dadd(dacc(dadd(0.0, p[0][1]), p[1][1], -2.0), p[2][1]);
  }
  __device__ __forceinline__ float d2x() const {
    return (float)dadd(dacc(dadd(0.0, p[1][0]), p[1][1], -2.0), p[1][2]);
  }
};

// 8-neighbour sum with constant-0 border, C order
__device__ __forceinline__ float hsum(const float* __restrict__ P, int y, int x, int H, int W, int pitch) {
  double a = 0.0;
#pragma unroll
  for (int dy = -1; dy <= 1; dy++)
#pragma unroll
    for (int dx = -1; dx <= 1; dx++) {
      if (dy == 0 && dx == 0) continue;
      int yy = y + dy, xx = x + dx;
      float v = (yy >= 0 && yy < H && xx >= 0 && xx < W) ? P[(size_t)yy * pitch + xx] : 0.0f;
      a = dadd(a, v);
    }
  return (float)a;
}

// Coefficient planes of pixel (y, x) (pitch-`pitch` index i) from its 3x3 neighbourhoods
// of the normalised frame (n) and the temporal difference (e).
__device__ __forceinline__ void ls_coef_at(const Nb3& n, const Nb3& e, int y, int x, int H, int W, float h,
                                           float* __restrict__ coef, size_t plane, size_t i) {
  float I = n.p[1][1];
  int cnt = 0;
#pragma unroll
  for (int dy = -1; dy <= 1; dy++)
#pragma unroll
    for (int dx = -1; dx <= 1; dx++)
      if (dy || dx) cnt += (y + dy >= 0 && y + dy < H && x + dx >= 0 && x + dx < W);
  float cm = (float)cnt;
  coef[i] = __fmul_rn(I, n.dy());                 // IIx
  coef[plane + i] = __fmul_rn(I, n.dx());         // IIy
  coef[2 * plane + i] = __fmul_rn(I, I);          // II
  coef[3 * plane + i] = __fmul_rn(I, e.dy());     // Ixt
  coef[4 * plane + i] = __fmul_rn(I, e.dx());     // Iyt
  float twoI = __fmul_rn(2.0f, I);
  float hc = __fmul_rn(h, cm);
  float A11 = __fsub_rn(__fmul_rn(I, __fsub_rn(n.d2y(), twoI)), hc);
  float A22 = __fsub_rn(__fmul_rn(I, __fsub_rn(n.d2x(), twoI)), hc);
  float A12 = __fmul_rn(I, n.m());
  float det = __fsub_rn(__fmul_rn(A11, A22), __fmul_rn(A12, A12));
  coef[5 * plane + i] = __fdiv_rn(A22, det);
  coef[6 * plane + i] = __fdiv_rn(-A12, det);
  coef[7 * plane + i] = __fdiv_rn(A11, det);
}

__global__ void ls_coef_kernel(const float* __restrict__ I1, const float* __restrict__ Et, float* __restrict__ coef,
                               size_t plane, int H, int W, int pitch, float h) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  Nb3 n, e;
  n.load(I1, y, x, H, W, pitch);
  e.load(Et, y, x, H, W, pitch);
  ls_coef_at(n, e, y, x, H, W, h, coef, plane, (size_t)y * pitch + x);
}

// The whole set-up of a solve after the frame maxima, in one pass: a 32 x 8 tile of the
// normalised frame I1 = im1 / max1 and of Et = im2 / max2 - I1 is formed in shared memory
// with a 1-pixel halo of clamped ('nearest') coordinates -- exactly the neighbourhoods
// Nb3::load reads -- then each pixel's coefficient planes are computed as in
// ls_coef_kernel, and the initial field (V, U) is copied into ping-pong buffer 0.  The
// normalised planes never reach global memory.
__global__ void __launch_bounds__(256) ls_prep_kernel(const float* __restrict__ a, const float* __restrict__ b,
                                                      int sp, const unsigned int* __restrict__ keys,
                                                      const float* __restrict__ V, const float* __restrict__ U,
                                                      float* __restrict__ coef, size_t plane, float* __restrict__ u0,
                                                      float* __restrict__ v0, int H, int W, int P, float h) {
  __shared__ float t1[10][35], te[10][35];
  const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 8;
  const float ma = key2f(keys[0]), mb = key2f(keys[1]);
  for (int k = threadIdx.x; k < 10 * 34; k += 256) {
    const int ly = k / 34, lx = k - ly * 34;
    const size_t g = (size_t)clampi(y0 - 1 + ly, 0, H - 1) * sp + clampi(x0 - 1 + lx, 0, W - 1);
    const float i1 = __fdiv_rn(a[g], ma), i2 = __fdiv_rn(b[g], mb);
    t1[ly][lx] = i1;
    te[ly][lx] = __fsub_rn(i2, i1);
  }
  __syncthreads();
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int x = x0 + tx, y = y0 + ty;
  if (x >= W || y >= H) return;
  Nb3 n, e;
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) {
      n.p[r][c] = t1[ty + r][tx + c];
      e.p[r][c] = te[ty + r][tx + c];
    }
  const size_t i = (size_t)y * P + x, si = (size_t)y * sp + x;
  ls_coef_at(n, e, y, x, H, W, h, coef, plane, i);
  u0[i] = V[si];
  v0[i] = U[si];
}

__device__ __forceinline__ double ls_err(const double* ss, int k, double inv_n) {
  return (sqrt(ss[2 * k]) + sqrt(ss[2 * k + 1])) * inv_n;
}

// Stencil helpers of the sweep.
//  - 2-term stencils (D, D^T, F, F^T) in float32 as 0 + w0*a + w1*b: with exact operand
//    halves, one float32 rounding of the exact value equals the reference's double
//    accumulation rounded to float32 (including the sign of zero; double rounding through
//    53 bits is innocuous for a sum of two 24-bit values);
//  - M (4 terms) and H (8 terms) keep the reference's double accumulation order; H uses
//    'constant' 0 outside the image (the EDGE variant selects +0.0 there).
// The weights (+-0.5, 1, +-0.25) are powers of two, so every product is exact and an add of
// the product rounds exactly as a fused multiply-add does: each term is one FMA.
// The float32 arithmetic of a lane's two cells runs as packed f32x2 operations (sm_100
// fma / add / mul .rn.f32x2): each half rounds exactly as the scalar operation does.
constexpr long long LS_WAIT_LIMIT = 1ll << 22;

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 f2s(float a) { return make_float2(a, a); }
// Packed f32x2 arithmetic.  The assembler contracts a packed multiply feeding a packed add
// into one fused multiply-add even when both carry .rn (measured on sm_100a with CUDA 12.9;
// scalar .rn operations are left alone), and it sees through literal ones and zeros.  So a
// sum of products is written as fma(product, one, sum) with `one` a kernel argument equal
// to 1.0f: that rounds exactly as product + sum, and a multiplier whose value the assembler
// does not know cannot be folded away or fused with the product.
__device__ __forceinline__ float2 pmul(float2 a, float2 b) {
  float2 d;
  asm("{.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\t"
      "mov.b64 rb, {%4, %5};\n\t"
      "mul.rn.f32x2 rd, ra, rb;\n\t"
      "mov.b64 {%0, %1}, rd;}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 padd(float2 a, float2 b) {
  float2 d;
  asm("{.reg .b64 ra, rb, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\t"
      "mov.b64 rb, {%4, %5};\n\t"
      "add.rn.f32x2 rd, ra, rb;\n\t"
      "mov.b64 {%0, %1}, rd;}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return d;
}
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) {
  float2 d;
  asm("{.reg .b64 ra, rb, rc, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\t"
      "mov.b64 rb, {%4, %5};\n\t"
      "mov.b64 rc, {%6, %7};\n\t"
      "fma.rn.f32x2 rd, ra, rb, rc;\n\t"
      "mov.b64 {%0, %1}, rd;}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return d;
}
__device__ __forceinline__ float2 st2x2(float2 a, float2 b, float wa, float wb) {
  return pfma(b, f2s(wb), pfma(a, f2s(wa), f2s(0.0f)));
}
// M at column j of the lane's 4-column window (j = 1: the even cell, 2: the odd cell)
__device__ __forceinline__ float st_m(const double* U, const double* D, int j) {
  double t = __fma_rn(U[j - 1], 0.25, 0.0);
  t = __fma_rn(U[j + 1], -0.25, t);
  t = __fma_rn(D[j - 1], -0.25, t);
  t = __fma_rn(D[j + 1], 0.25, t);
  return (float)t;
}
// H at column j; on an image border the out-of-image neighbours count as +0.0
template <bool EDGE>
__device__ __forceinline__ float st_h(const double* U, const double* C, const double* D, int j, bool T, bool B,
                                      bool L, bool R) {
  double t = 0.0;
  t = __dadd_rn(t, (EDGE && (T || L)) ? 0.0 : U[j - 1]);
  t = __dadd_rn(t, (EDGE && T) ? 0.0 : U[j]);
  t = __dadd_rn(t, (EDGE && (T || R)) ? 0.0 : U[j + 1]);
  t = __dadd_rn(t, (EDGE && L) ? 0.0 : C[j - 1]);
  t = __dadd_rn(t, (EDGE && R) ? 0.0 : C[j + 1]);
  t = __dadd_rn(t, (EDGE && (B || L)) ? 0.0 : D[j - 1]);
  t = __dadd_rn(t, (EDGE && B) ? 0.0 : D[j]);
  t = __dadd_rn(t, (EDGE && (B || R)) ? 0.0 : D[j + 1]);
  return (float)t;
}

// Temporally blocked sweeps: one pass runs up to LB_T sweeps on a tile held in shared
// memory, so the 8 coefficient planes and (u, v) cross HBM/L2 once per LB_T sweeps.
// Tile: 56 x 23 owned pixels plus a 4-pixel halo = a 64 x 31 region, loaded by one 3-D TMA
// (8 coefficient planes, 62 KB) and two 2-D TMAs (u, v) starting at (x0-4, y0-4): x stays
// 16-byte aligned.  (23 rows: a 1024 x 1024 image is 19 x 45 tiles, 2.9 waves of 2 CTAs
// on 148 SMs.)  Each lane owns a column pair (2 lane, 2 lane + 1) of the region and
// walks it down a band of rows (its warp's share of the sweep's rows), so every float32
// step of the two cells is one packed instruction and the centre pair, the coefficient
// pairs and the results move as 64-bit shared-memory accesses.  Sweep s computes the rows
// at least s + 1 from the region's top and bottom edge (all later sweeps need) and every
// column; a cell's value is exact after sweep s only if it lies at least s + 1 from the
// region's edge, so after LB_T = 4 sweeps exactly the owned 56 x 23 pixels are, and the
// last sweep stores those straight to global memory.  The region's outermost columns use
// their own value as the missing neighbour (inexact, like the rest of the halo).
// Image borders: every neighbour index is clamped into the image ('nearest'), H uses
// 'constant' 0 through the border flags, and out-of-image rows are not computed; the cells
// of out-of-image columns are computed from clamped values but never read.
// The squared change of every sweep is accumulated over owned pixels only, so each pixel is
// counted once per sweep.  The stop rule: the last CTA of a pass finds the first sweep
// whose error is <= tol; if that is not the pass's last sweep, the pass ran too far and the
// next launch (which the stop rule has cancelled as a pass) recomputes it from its
// unchanged input with the right count.
constexpr int LB_T = 4, LB_TW = 56, LB_TH = 23, LB_RW = LB_TW + 2 * LB_T, LB_RH = LB_TH + 2 * LB_T;  // 64 x 31
constexpr int LB_PLANE = LB_RW * LB_RH * 4;                  // 7936 B, a multiple of 128 (TMA destinations)
static_assert(LB_PLANE % 128 == 0, "each staged plane must start 128-byte aligned");
// The sweeps update region rows 1 .. LB_RH - 2 only, so the coefficient planes are staged
// for those rows: LB_CH rows per plane.
constexpr int LB_CH = LB_RH - 2;
constexpr int LB_CPLANE = LB_RW * LB_CH * 4;                 // 7424 B
static_assert(LB_CPLANE % 128 == 0, "the u, v planes after the coefficients must start 128-byte aligned");
constexpr int LB_PL = LB_RW * LB_CH;                         // floats per coefficient plane
constexpr int LB_COEF_BYTES = 8 * LB_CPLANE;
// The float64-sum pass ping-pongs (u, v) between two buffers; the float32 pass updates one
// buffer in place (each warp keeps the old values of its band's boundary rows in registers),
// which brings it to 75.5 KB: 3 CTAs per SM.
constexpr size_t lb_smem(bool fast) { return LB_COEF_BYTES + (fast ? 2 : 4) * LB_PLANE + 128 + 128; }
#ifndef OF_LS_PASS_WARPS
#define OF_LS_PASS_WARPS 6
#endif
constexpr int LB_WARPS = OF_LS_PASS_WARPS;  // warps per CTA, each a band of the region's rows

typedef float LbPlane[LB_RW];

struct LbPass {  // per-launch description of a pass
  int k0;        // first sweep index
  int nsweep;    // sweeps in this pass (<= LB_T)
  int pass;      // pass index
  int last;      // 1: the launch after the last pass, which only rolls that pass back
};

// One window row of a lane: the float32 centre pair and the float64 values of the four
// columns 2 lane - 1 .. 2 lane + 2 (clamped), for u and v.
struct LbRow {
  float2 cu, cv;
  double du[4], dv[4];
};

// Columns of a lane's window: k[0..3] for 2 lane - 1 .. 2 lane + 2.  EDGE tiles clamp all
// four into the image; interior tiles only the two outside the region (lanes 0 and 31).
struct LbCols {
  int k[4];
};

template <bool EDGE>
__device__ __forceinline__ void lb_load(LbRow& R, const LbPlane* su, const LbPlane* sv, int row, const LbCols& c) {
  if (EDGE) {
    R.cu = f2(su[row][c.k[1]], su[row][c.k[2]]);
    R.cv = f2(sv[row][c.k[1]], sv[row][c.k[2]]);
  } else {
    R.cu = *reinterpret_cast<const float2*>(&su[row][c.k[1]]);
    R.cv = *reinterpret_cast<const float2*>(&sv[row][c.k[1]]);
  }
  R.du[0] = (double)su[row][c.k[0]];
  R.du[1] = (double)R.cu.x;
  R.du[2] = (double)R.cu.y;
  R.du[3] = (double)su[row][c.k[3]];
  R.dv[0] = (double)sv[row][c.k[0]];
  R.dv[1] = (double)R.cv.x;
  R.dv[2] = (double)R.cv.y;
  R.dv[3] = (double)sv[row][c.k[3]];
}

struct LbStrip {  // what a lane needs beyond the window rows
  const float* sc;  // coefficient planes
  const LbPlane *su, *sv;  // input buffers of the sweep
  int kl, kr;       // the window's outer columns (clamped 2 lane - 1, 2 lane + 2)
  LbPlane *ou, *ov;  // output buffers of the sweep (null on the last sweep)
  float *gu, *gv;   // global output of the last sweep, at the lane's even column, row 0 of the region
  int pitch;
  int c0;           // the lane's even region column
  int gx0, gy0;     // global x of column c0, global y of the strip's first row
  int H, W;
  float h;
  float one;        // 1.0f, unknown to the assembler (see pfma)
  bool own_col;     // the pair lies in the owned columns
};

// Update of the lane's cell pair in region row `row` from window rows U (above), C, D (below).
template <bool EDGE>
__device__ __forceinline__ void lb_pair(const LbRow& U, const LbRow& C, const LbRow& D, const LbStrip& S, int row,
                                        int gy, bool own_row, double& acc_u, double& acc_v) {
  const bool T = gy == 0, B = gy == S.H - 1;
  const bool L0 = S.gx0 == 0, R0 = S.gx0 == S.W - 1, L1 = S.gx0 + 1 == 0, R1 = S.gx0 + 1 == S.W - 1;
  const int o = (row - 1) * LB_RW + S.c0;  // coefficient rows start at region row 1
  const float* sc = S.sc;
  const float2 a = *reinterpret_cast<const float2*>(sc + o);
  const float2 b = *reinterpret_cast<const float2*>(sc + LB_PL + o);
  const float2 cc = *reinterpret_cast<const float2*>(sc + 2 * LB_PL + o);
  // the outer columns of the centre row again as float32 (cheaper than keeping them live)
  const float2 Lu = f2(S.su[row][S.kl], C.cu.x), Ru = f2(C.cu.y, S.su[row][S.kr]);
  const float2 Lv = f2(S.sv[row][S.kl], C.cv.x), Rv = f2(C.cv.y, S.sv[row][S.kr]);
  const float2 Du = st2x2(U.cu, D.cu, -0.5f, 0.5f), DTu = st2x2(Lu, Ru, -0.5f, 0.5f);
  const float2 Dv = st2x2(U.cv, D.cv, -0.5f, 0.5f), DTv = st2x2(Lv, Rv, -0.5f, 0.5f);
  const float2 Fu = st2x2(U.cu, D.cu, 1.0f, 1.0f), FTv = st2x2(Lv, Rv, 1.0f, 1.0f);
  const float2 Mu = f2(st_m(U.du, D.du, 1), st_m(U.du, D.du, 2));
  const float2 Mv = f2(st_m(U.dv, D.dv, 1), st_m(U.dv, D.dv, 2));
  const float2 Hu = f2(st_h<EDGE>(U.du, C.du, D.du, 1, T, B, L0, R0), st_h<EDGE>(U.du, C.du, D.du, 2, T, B, L1, R1));
  const float2 Hv = f2(st_h<EDGE>(U.dv, C.dv, D.dv, 1, T, B, L0, R0), st_h<EDGE>(U.dv, C.dv, D.dv, 2, T, B, L1, R1));
  const float2 h2 = f2s(S.h), two = f2s(2.0f), one = f2s(S.one);
  // acc + x * y with two roundings: fma(x * y, one, acc)
#define LB_MAC(acc, x, y) pfma(pmul((x), (y)), one, (acc))
  float2 bu = pmul(pmul(two, a), Du);
  bu = LB_MAC(bu, a, DTv);
  bu = LB_MAC(bu, b, Dv);
  bu = LB_MAC(bu, cc, Fu);
  bu = LB_MAC(bu, cc, Mv);
  bu = LB_MAC(bu, h2, Hu);
  bu = padd(bu, *reinterpret_cast<const float2*>(sc + 3 * LB_PL + o));
  float2 bv = pmul(b, Du);
  bv = LB_MAC(bv, a, DTu);
  bv = LB_MAC(bv, pmul(two, b), DTv);
  bv = LB_MAC(bv, cc, Mu);
  bv = LB_MAC(bv, cc, FTv);
  bv = LB_MAC(bv, h2, Hv);
  bv = padd(bv, *reinterpret_cast<const float2*>(sc + 4 * LB_PL + o));
  const float2 B11 = *reinterpret_cast<const float2*>(sc + 5 * LB_PL + o);
  const float2 B12 = *reinterpret_cast<const float2*>(sc + 6 * LB_PL + o);
  const float2 B22 = *reinterpret_cast<const float2*>(sc + 7 * LB_PL + o);
  const float2 m1 = f2s(-S.one);  // exact negation, the sign of zero included
  const float2 nu = pmul(LB_MAC(pmul(B11, bu), B12, bv), m1);
  const float2 nv = pmul(LB_MAC(pmul(B12, bu), B22, bv), m1);
#undef LB_MAC
  const bool in0 = S.gx0 < S.W, in1 = S.gx0 + 1 < S.W;
  if (S.ou) {
    *reinterpret_cast<float2*>(&S.ou[row][S.c0]) = nu;
    *reinterpret_cast<float2*>(&S.ov[row][S.c0]) = nv;
  } else if (own_row && S.own_col) {  // last sweep: owned cells straight to global
    const size_t gi = (size_t)row * S.pitch;
    if (in1) {
      *reinterpret_cast<float2*>(S.gu + gi) = nu;
      *reinterpret_cast<float2*>(S.gv + gi) = nv;
    } else if (in0) {
      S.gu[gi] = nu.x;
      S.gv[gi] = nv.x;
    }
  }
  if (own_row && S.own_col) {
    // float32 change, as the reference's unew - u; squares summed in double
    const float2 eu = pfma(C.cu, m1, nu), ev = pfma(C.cv, m1, nv);
    const float eu0 = in0 ? eu.x : 0.0f, ev0 = in0 ? ev.x : 0.0f;
    const float eu1 = in1 ? eu.y : 0.0f, ev1 = in1 ? ev.y : 0.0f;
    acc_u = __fma_rn((double)eu0, (double)eu0, acc_u);
    acc_u = __fma_rn((double)eu1, (double)eu1, acc_u);
    acc_v = __fma_rn((double)ev0, (double)ev0, acc_v);
    acc_v = __fma_rn((double)ev1, (double)ev1, acc_v);
  }
}

// One sweep of a lane's band: rows [r0, r0 + n) of its column pair.  The three window rows
// rotate through three register sets (3-row steps), so sliding the window costs loads only.
// EDGE tiles clamp the window rows into [rlo, rhi].
template <bool EDGE>
__device__ __forceinline__ void lb_strip(const LbPlane* su, const LbPlane* sv, const LbStrip& S, const LbCols& cols,
                                         int r0, int n, int rlo, int rhi, double& acc_u, double& acc_v) {
  LbRow A, B, C;
#define LB_ROW(r) (EDGE ? clampi((r), rlo, rhi) : (r))
#define LB_OWN(row) ((row) >= LB_T && (row) < LB_T + LB_TH)
  lb_load<EDGE>(A, su, sv, LB_ROW(r0 - 1), cols);
  lb_load<EDGE>(B, su, sv, r0, cols);
#pragma unroll 1
  for (int r = 0; r < n; r += 3) {
    const int row = r0 + r;
    lb_load<EDGE>(C, su, sv, LB_ROW(row + 1), cols);
    lb_pair<EDGE>(A, B, C, S, row, S.gy0 + r, LB_OWN(row), acc_u, acc_v);
    if (r + 1 < n) {
      lb_load<EDGE>(A, su, sv, LB_ROW(row + 2), cols);
      lb_pair<EDGE>(B, C, A, S, row + 1, S.gy0 + r + 1, LB_OWN(row + 1), acc_u, acc_v);
    }
    if (r + 2 < n) {
      lb_load<EDGE>(B, su, sv, LB_ROW(row + 3), cols);
      lb_pair<EDGE>(C, A, B, S, row + 2, S.gy0 + r + 2, LB_OWN(row + 2), acc_u, acc_v);
    }
  }
#undef LB_OWN
#undef LB_ROW
}

// ---- float32 pass (OF_LS_FAST) ----------------------------------------------------------
// The same sweep, tile and stop rule with float32 arithmetic throughout: no float64 stencil
// sums, no conversions, fused multiply-adds.  The stencils share their parts: per field the
// vertical difference vd = down - up and sum vs = up + down of the lane's four columns give
// D (= vd / 2), F (= vs), M (= (vd[c+1] - vd[c-1]) / 4) and, with the centre row's
// neighbours, D^T (= (right - left) / 2), F^T (= left + right) and H (= vs[c-1] + vs[c] +
// vs[c+1] + left + right in the interior); the constant factors are folded into the
// coefficients (exact power-of-two scalings).  Results differ from the reference's float32
// fields by float32 rounding only (<= 1e-3 px of the float64 answer at the configurations).
struct LbRowF {
  float2 cu, cv;           // the lane's cell pair
  float lu, ru, lv, rv;    // the window's outer columns (2 lane - 1, 2 lane + 2)
};

template <bool EDGE>
__device__ __forceinline__ void lbf_load(LbRowF& R, const LbPlane* su, const LbPlane* sv, int row, const LbCols& c) {
  if (EDGE) {
    R.cu = f2(su[row][c.k[1]], su[row][c.k[2]]);
    R.cv = f2(sv[row][c.k[1]], sv[row][c.k[2]]);
  } else {
    R.cu = *reinterpret_cast<const float2*>(&su[row][c.k[1]]);
    R.cv = *reinterpret_cast<const float2*>(&sv[row][c.k[1]]);
  }
  R.lu = su[row][c.k[0]];
  R.ru = su[row][c.k[3]];
  R.lv = sv[row][c.k[0]];
  R.rv = sv[row][c.k[3]];
}

// Packed float32 arithmetic of the float32 pass: sm_100's builtins (the compiler pairs the
// registers itself; contraction is welcome here).  a - b is one fused multiply-add.
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 fmul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }

// 8-neighbour sum of the pair with out-of-image neighbours as 0 (H's 'constant' border)
__device__ __forceinline__ float2 lbf_hsum_edge(const LbRowF& U, const LbRowF& C, const LbRowF& D, bool T, bool B,
                                                bool L0, bool R0, bool L1, bool R1, bool uv) {
  const float2 u = uv ? U.cv : U.cu, c = uv ? C.cv : C.cu, d = uv ? D.cv : D.cu;
  const float ul = uv ? U.lv : U.lu, ur = uv ? U.rv : U.ru, cl = uv ? C.lv : C.lu, cr = uv ? C.rv : C.ru;
  const float dl = uv ? D.lv : D.lu, dr = uv ? D.rv : D.ru;
  float h0 = (T || L0) ? 0.f : ul;
  h0 = __fadd_rn(h0, T ? 0.f : u.x);
  h0 = __fadd_rn(h0, (T || R0) ? 0.f : u.y);
  h0 = __fadd_rn(h0, L0 ? 0.f : cl);
  h0 = __fadd_rn(h0, R0 ? 0.f : c.y);
  h0 = __fadd_rn(h0, (B || L0) ? 0.f : dl);
  h0 = __fadd_rn(h0, B ? 0.f : d.x);
  h0 = __fadd_rn(h0, (B || R0) ? 0.f : d.y);
  float h1 = (T || L1) ? 0.f : u.x;
  h1 = __fadd_rn(h1, T ? 0.f : u.y);
  h1 = __fadd_rn(h1, (T || R1) ? 0.f : ur);
  h1 = __fadd_rn(h1, L1 ? 0.f : c.x);
  h1 = __fadd_rn(h1, R1 ? 0.f : cr);
  h1 = __fadd_rn(h1, (B || L1) ? 0.f : d.x);
  h1 = __fadd_rn(h1, B ? 0.f : d.y);
  h1 = __fadd_rn(h1, (B || R1) ? 0.f : dr);
  return f2(h0, h1);
}

template <bool EDGE>
__device__ __forceinline__ void lbf_pair(const LbRowF& U, const LbRowF& C, const LbRowF& D, const LbStrip& S, int row,
                                         int gy, bool own_row, float& acc_u, float& acc_v) {
  const int o = (row - 1) * LB_RW + S.c0;  // coefficient rows start at region row 1
  const float* sc = S.sc;
  const float2 IIx = *reinterpret_cast<const float2*>(sc + o);
  const float2 IIy = *reinterpret_cast<const float2*>(sc + LB_PL + o);
  const float2 II = *reinterpret_cast<const float2*>(sc + 2 * LB_PL + o);
  // vertical differences and sums at the pair and at the outer columns
  const float2 vdu = fsub2(D.cu, U.cu), vsu = fadd2(U.cu, D.cu);
  const float2 vdv = fsub2(D.cv, U.cv), vsv = fadd2(U.cv, D.cv);
  const float2 vdo_u = fsub2(f2(D.lu, D.ru), f2(U.lu, U.ru));  // (left column, right column)
  const float2 vdo_v = fsub2(f2(D.lv, D.rv), f2(U.lv, U.rv));
  const float2 mdu = fsub2(f2(vdu.y, vdo_u.y), f2(vdo_u.x, vdu.x));  // 4 M
  const float2 mdv = fsub2(f2(vdv.y, vdo_v.y), f2(vdo_v.x, vdv.x));
  // centre-row neighbours of the pair
  const float2 Lu = f2(C.lu, C.cu.x), Ru = f2(C.cu.y, C.ru);
  const float2 Lv = f2(C.lv, C.cv.x), Rv = f2(C.cv.y, C.rv);
  const float2 dtu = fsub2(Ru, Lu), dtv = fsub2(Rv, Lv);  // 2 D^T
  const float2 hsv = fadd2(Lv, Rv);                       // F^T
  float2 Hu, Hv;
  if (EDGE) {
    const bool T = gy == 0, B = gy == S.H - 1;
    const bool L0 = S.gx0 == 0, R0 = S.gx0 == S.W - 1, L1 = S.gx0 + 1 == 0, R1 = S.gx0 + 1 == S.W - 1;
    Hu = lbf_hsum_edge(U, C, D, T, B, L0, R0, L1, R1, false);
    Hv = lbf_hsum_edge(U, C, D, T, B, L0, R0, L1, R1, true);
  } else {
    const float2 vso_u = fadd2(f2(U.lu, U.ru), f2(D.lu, D.ru));
    const float2 vso_v = fadd2(f2(U.lv, U.rv), f2(D.lv, D.rv));
    Hu = fadd2(fadd2(vso_u, f2s(__fadd_rn(vsu.x, vsu.y))), fadd2(Lu, Ru));
    Hv = fadd2(fadd2(vso_v, f2s(__fadd_rn(vsv.x, vsv.y))), hsv);
  }
  const float2 a2 = fmul2(IIx, f2s(0.5f)), a3 = fmul2(IIy, f2s(0.5f)), a5 = fmul2(II, f2s(0.25f));
  const float2 h2 = f2s(S.h);
  // bu = 2 IIx D u + IIx D^T v + IIy D v + II F u + II M v + h H u + Ixt
  float2 bu = *reinterpret_cast<const float2*>(sc + 3 * LB_PL + o);
  bu = ffma2(h2, Hu, bu);
  bu = ffma2(a5, mdv, bu);
  bu = ffma2(II, vsu, bu);
  bu = ffma2(a3, vdv, bu);
  bu = ffma2(a2, dtv, bu);
  bu = ffma2(IIx, vdu, bu);
  // bv = IIy D u + IIx D^T u + 2 IIy D^T v + II M u + II F^T v + h H v + Iyt
  float2 bv = *reinterpret_cast<const float2*>(sc + 4 * LB_PL + o);
  bv = ffma2(h2, Hv, bv);
  bv = ffma2(a5, mdu, bv);
  bv = ffma2(II, hsv, bv);
  bv = ffma2(IIy, dtv, bv);
  bv = ffma2(a2, dtu, bv);
  bv = ffma2(a3, vdu, bv);
  const float2 B11 = *reinterpret_cast<const float2*>(sc + 5 * LB_PL + o);
  const float2 B12 = *reinterpret_cast<const float2*>(sc + 6 * LB_PL + o);
  const float2 B22 = *reinterpret_cast<const float2*>(sc + 7 * LB_PL + o);
  const float2 m1 = f2s(-1.0f);
  const float2 nu = fmul2(ffma2(B11, bu, fmul2(B12, bv)), m1);
  const float2 nv = fmul2(ffma2(B12, bu, fmul2(B22, bv)), m1);
  const bool in0 = S.gx0 < S.W, in1 = S.gx0 + 1 < S.W;
  if (S.ou) {
    __syncwarp();  // in place: every lane has read this row (as its window's next row) already
    *reinterpret_cast<float2*>(&S.ou[row][S.c0]) = nu;
    *reinterpret_cast<float2*>(&S.ov[row][S.c0]) = nv;
  } else if (own_row && S.own_col) {
    const size_t gi = (size_t)row * S.pitch;
    if (in1) {
      *reinterpret_cast<float2*>(S.gu + gi) = nu;
      *reinterpret_cast<float2*>(S.gv + gi) = nv;
    } else if (in0) {
      S.gu[gi] = nu.x;
      S.gv[gi] = nv.x;
    }
  }
  if (own_row && S.own_col) {
    const float2 eu = fsub2(nu, C.cu), ev = fsub2(nv, C.cv);
    const float eu0 = in0 ? eu.x : 0.0f, ev0 = in0 ? ev.x : 0.0f;
    const float eu1 = in1 ? eu.y : 0.0f, ev1 = in1 ? ev.y : 0.0f;
    acc_u = __fmaf_rn(eu0, eu0, __fmaf_rn(eu1, eu1, acc_u));
    acc_v = __fmaf_rn(ev0, ev0, __fmaf_rn(ev1, ev1, acc_v));
  }
}

// The old values a band needs from outside it, read before any warp of the CTA writes the
// sweep's results in place: the row above the band and its first row (the window's start)
// and the row below it.
template <bool EDGE>
__device__ __forceinline__ void lbf_edges(LbRowF& A, LbRowF& B, LbRowF& E, const LbPlane* su, const LbPlane* sv,
                                          const LbCols& cols, int r0, int n, int rlo, int rhi) {
  lbf_load<EDGE>(A, su, sv, EDGE ? clampi(r0 - 1, rlo, rhi) : r0 - 1, cols);
  lbf_load<EDGE>(B, su, sv, r0, cols);
  lbf_load<EDGE>(E, su, sv, EDGE ? clampi(r0 + n, rlo, rhi) : r0 + n, cols);
}

// One float32 sweep of a lane's band, rows [r0, r0 + n), in place: the window starts from
// A, B (lbf_edges) and takes E for the row below the band; every other row is read from
// shared memory before this warp overwrites it (the rows of the band belong to this warp).
template <bool EDGE>
__device__ __forceinline__ void lbf_strip(const LbPlane* su, const LbPlane* sv, const LbStrip& S, const LbCols& cols,
                                          int r0, int n, int rlo, int rhi, LbRowF& A, LbRowF& B, const LbRowF& E,
                                          double& acc_u, double& acc_v) {
  LbRowF C;
  float au = 0.f, av = 0.f;
  const int rend = r0 + n;
#define LB_OWN(row) ((row) >= LB_T && (row) < LB_T + LB_TH)
#define LB_NEXT(X, r)                                                     \
  do {                                                                    \
    if ((r) == rend)                                                      \
      X = E;                                                              \
    else                                                                  \
      lbf_load<EDGE>(X, su, sv, EDGE ? clampi((r), rlo, rhi) : (r), cols); \
  } while (0)
#pragma unroll 1
  for (int r = 0; r < n; r += 3) {
    const int row = r0 + r;
    LB_NEXT(C, row + 1);
    lbf_pair<EDGE>(A, B, C, S, row, S.gy0 + r, LB_OWN(row), au, av);
    if (r + 1 < n) {
      LB_NEXT(A, row + 2);
      lbf_pair<EDGE>(B, C, A, S, row + 1, S.gy0 + r + 1, LB_OWN(row + 1), au, av);
    }
    if (r + 2 < n) {
      LB_NEXT(B, row + 3);
      lbf_pair<EDGE>(C, A, B, S, row + 2, S.gy0 + r + 2, LB_OWN(row + 2), au, av);
    }
  }
#undef LB_NEXT
#undef LB_OWN
  acc_u += (double)au;
  acc_v += (double)av;
}

template <bool FAST, int NW>
__global__ void __launch_bounds__(32 * NW, (FAST && NW == 6) ? 3 : 2) ls_pass_kernel(const __grid_constant__ CUtensorMap tm_coef,
                                                         const __grid_constant__ CUtensorMap tm_u0,
                                                         const __grid_constant__ CUtensorMap tm_v0,
                                                         const __grid_constant__ CUtensorMap tm_u1,
                                                         const __grid_constant__ CUtensorMap tm_v1,
                                                         float* ub0, float* vb0, float* ub1, float* vb1, int H, int W,
                                                         int pitch, float h, LbPass P, LsCtrl* ctrl, double* ss,
                                                         int* run, unsigned int* done, int* redo, double inv_n,
                                                         double tol, int* err_flag, float one) {
  // Passes after the first are launched as programmatic dependents of the previous pass:
  // every CTA lets the next pass be scheduled at once, so its CTAs take the SM slots this
  // pass's tail frees and prefetch their coefficient tile (the coefficients do not change
  // during a solve); griddepcontrol.wait then holds them until the previous pass has
  // completed and its memory (u, v and the stop-rule flags) is visible.  Launched without
  // the attribute, both instructions have no effect.
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  extern __shared__ __align__(128) unsigned char lb_smem_raw[];
  unsigned char* base = lb_smem_raw + ((128 - (smem_u32(lb_smem_raw) & 127)) & 127);
  const float* sc = reinterpret_cast<const float*>(base);
  // ping-pong buffer q: u at base + COEF + 2q planes, v right after it
#define LB_U(q) reinterpret_cast<LbPlane*>(base + LB_COEF_BYTES + (2 * (q)) * LB_PLANE)
#define LB_V(q) reinterpret_cast<LbPlane*>(base + LB_COEF_BYTES + (2 * (q) + 1) * LB_PLANE)
  // the barriers follow the (u, v) buffers: 2 planes in place (float32 pass), else 4
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + LB_COEF_BYTES + (FAST ? 2 : 4) * LB_PLANE);  // coefficients
  uint64_t* bar2 = bar + 1;                                                           // u, v
  const int x0 = blockIdx.x * LB_TW, y0 = blockIdx.y * LB_TH;
  const int lane = threadIdx.x, warp = threadIdx.y;
  const int t = warp * 32 + lane;
  if (t == 0) {
    mbar_init(bar, 1);
    mbar_init(bar2, 1);
  }
  __syncthreads();
  const bool pre = !P.last;  // the launch after the last pass only rolls back: no prefetch
  if (pre && t == 0) {
    mbar_expect_tx(bar, LB_COEF_BYTES);
    tma_load_3d((void*)sc, &tm_coef, x0 - LB_T, y0 - LB_T + 1, 0, bar);
  }
  asm volatile("griddepcontrol.wait;" ::: "memory");
  // Pass p reads ping-pong buffer p & 1 and writes the other.  A pass that the stop rule
  // cancelled (and the launch after the last pass) instead rolls the previous pass back
  // when that pass ran past its stopping sweep: it recomputes it from the same input with
  // the sweep count the stop rule chose (redo[p - 1]) and keeps no error sums.
  int k0 = P.k0, nsw = P.nsweep, pass = P.pass;
  bool rollback = false;
  if (P.last || (k0 > 0 && *(volatile int*)(run + k0) == 0)) {
    const int r = pass > 0 ? *(volatile int*)(redo + pass - 1) : 0;
    if (r == 0) {
      if (pre && !mbar_wait(bar, 0, LS_WAIT_LIMIT) && t == 0) atomicExch(err_flag, 1);  // the prefetch lands
      return;
    }
    rollback = true;
    pass -= 1;
    k0 -= LB_T;
    nsw = r;
  }
  const int in = pass & 1, out = in ^ 1;
  const CUtensorMap* tm_u = in ? &tm_u1 : &tm_u0;
  const CUtensorMap* tm_v = in ? &tm_v1 : &tm_v0;
  float* un = out ? ub1 : ub0;
  float* vn = out ? vb1 : vb0;
  if (t == 0) {
    if (!pre) {
      mbar_expect_tx(bar, LB_COEF_BYTES);
      tma_load_3d((void*)sc, &tm_coef, x0 - LB_T, y0 - LB_T + 1, 0, bar);
    }
    mbar_expect_tx(bar2, 2 * LB_PLANE);
    tma_load_2d(LB_U(0), tm_u, x0 - LB_T, y0 - LB_T, bar2);
    tma_load_2d(LB_V(0), tm_v, x0 - LB_T, y0 - LB_T, bar2);
  }
  const bool ok_c = mbar_wait(bar, 0, LS_WAIT_LIMIT), ok_uv = mbar_wait(bar2, 0, LS_WAIT_LIMIT);
  if (!ok_c || !ok_uv) {
    if (t == 0) atomicExch(err_flag, 1);
    if (!ok_c) mbar_wait(bar, 0, LS_WAIT_LIMIT);  // one more bounded wait for the copies in flight
    if (!ok_uv) mbar_wait(bar2, 0, LS_WAIT_LIMIT);
    nsw = 0;
  }
  // in-image region rows / columns (region row r <-> y0 - 4 + r, column c <-> x0 - 4 + c)
  const int rlo = max(0, LB_T - y0), rhi = min(LB_RH - 1, H - 1 + LB_T - y0);
  const int clo = max(0, LB_T - x0), chi = min(LB_RW - 1, W - 1 + LB_T - x0);
  const bool edge = rlo > 0 || clo > 0 || rhi < LB_RH - 1 || chi < LB_RW - 1;
  const int c0 = 2 * lane;
  LbCols cols;
  if (edge) {
#pragma unroll
    for (int j = 0; j < 4; j++) cols.k[j] = clampi(c0 - 1 + j, clo, chi);
  } else {
    cols.k[0] = max(c0 - 1, 0);
    cols.k[1] = c0;
    cols.k[2] = c0 + 1;
    cols.k[3] = min(c0 + 2, LB_RW - 1);
  }
  LbStrip S;
  S.sc = sc;
  S.kl = cols.k[0];
  S.kr = cols.k[3];
  S.pitch = pitch;
  S.c0 = c0;
  S.gx0 = x0 - LB_T + c0;
  S.H = H;
  S.W = W;
  S.h = h;
  S.one = one;
  S.own_col = c0 >= LB_T && c0 < LB_T + LB_TW;
  __shared__ double red[LB_T][2][NW];
  __syncthreads();
#pragma unroll 1
  for (int s = 0; s < nsw; s++) {
    // the float32 pass updates buffer 0 in place; the float64-sum pass ping-pongs
    const int in = FAST ? 0 : s & 1, out = FAST ? 0 : in ^ 1;
    const bool last = s == nsw - 1;
    double au = 0.0, av = 0.0;
    // sweep s computes the rows at least s + 1 from the region's edge (later sweeps read no
    // others) that lie in the image, split evenly over the warps
    const int lo = max(1 + s, rlo), hi = min(LB_RH - 1 - s, rhi + 1);
    const int n = hi - lo;
    const int ra = lo + (n * warp) / NW, rb = lo + (n * (warp + 1)) / NW;
    LbRowF A, B, E;
    if (FAST) {
      if (rb > ra) {
        if (edge)
          lbf_edges<true>(A, B, E, LB_U(0), LB_V(0), cols, ra, rb - ra, rlo, rhi);
        else
          lbf_edges<false>(A, B, E, LB_U(0), LB_V(0), cols, ra, rb - ra, rlo, rhi);
      }
      if (!last) __syncthreads();  // every band's boundary rows are read before any row is rewritten
    }
    if (rb > ra) {
      S.su = LB_U(in);
      S.sv = LB_V(in);
      S.ou = last ? nullptr : LB_U(out);
      S.ov = last ? nullptr : LB_V(out);
      // global address of (row 0, column c0) of the region; only owned cells are stored
      S.gu = un + ((ptrdiff_t)(y0 - LB_T) * pitch + S.gx0);
      S.gv = vn + ((ptrdiff_t)(y0 - LB_T) * pitch + S.gx0);
      S.gy0 = y0 - LB_T + ra;
      if (FAST) {
        if (edge)
          lbf_strip<true>(LB_U(0), LB_V(0), S, cols, ra, rb - ra, rlo, rhi, A, B, E, au, av);
        else
          lbf_strip<false>(LB_U(0), LB_V(0), S, cols, ra, rb - ra, rlo, rhi, A, B, E, au, av);
      } else {
        if (edge)
          lb_strip<true>(LB_U(in), LB_V(in), S, cols, ra, rb - ra, rlo, rhi, au, av);
        else
          lb_strip<false>(LB_U(in), LB_V(in), S, cols, ra, rb - ra, rlo, rhi, au, av);
      }
    }
    if (!rollback) {
      for (int o = 16; o > 0; o >>= 1) {
        au += __shfl_down_sync(0xffffffffu, au, o);
        av += __shfl_down_sync(0xffffffffu, av, o);
      }
      if (lane == 0) {
        red[s][0][warp] = au;
        red[s][1][warp] = av;
      }
    }
    __syncthreads();
  }
  if (rollback) return;
  // per-sweep squared changes -> ss[k0 + s]; the last CTA applies the stop rule
  if (t == 0) {
    for (int s = 0; s < nsw; s++) {
      double a = 0.0, b = 0.0;
      for (int w = 0; w < NW; w++) {
        a += red[s][0][w];
        b += red[s][1][w];
      }
      atomicAdd(ss + 2 * (k0 + s), a);
      atomicAdd(ss + 2 * (k0 + s) + 1, b);
    }
    __threadfence();
    if (atomicAdd(done + pass, 1u) == gridDim.x * gridDim.y - 1) {
      __threadfence();
      int stop = -1;
      for (int s = 0; s < nsw; s++) {
        double s0 = atomicAdd(ss + 2 * (k0 + s), 0.0), s1 = atomicAdd(ss + 2 * (k0 + s) + 1, 0.0);
        if (!((sqrt(s0) + sqrt(s1)) * inv_n > tol)) {
          stop = s;
          break;
        }
      }
      if (stop < 0) {
        run[k0 + nsw] = 1;
        ctrl->K = k0 + nsw;
      } else {
        run[k0 + nsw] = 0;
        ctrl->K = k0 + stop + 1;
        redo[pass] = (stop < nsw - 1) ? stop + 1 : 0;
      }
      ctrl->final_buf = out;
    }
  }
}

#undef LB_U
#undef LB_V

// Sweeps run (and the last sweep's error); a TMA wait timeout in any pass is reported as
// iters = -1, err = NaN.
__global__ void ls_count_kernel(LsCtrl* ctrl, const double* ss, double inv_n, const int* err_flag, int* iters_out,
                                double* err_out) {
  int K = ctrl->K;
  bool failed = *err_flag != 0;
  if (iters_out) *iters_out = failed ? -1 : K;
  if (err_out) *err_out = failed ? __longlong_as_double(0x7ff8000000000000ll) : (K > 0 ? ls_err(ss, K - 1, inv_n) : 0.0);
}

// Result (ping-pong buffer ctrl->final_buf) -> caller's V (row component) and U.
__global__ void ls_finalize_kernel(const float* __restrict__ u0, const float* __restrict__ v0,
                                   const float* __restrict__ u1, const float* __restrict__ v1, float* __restrict__ V,
                                   float* __restrict__ U, int W, int sp, int dp, const LsCtrl* ctrl) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const bool one = ctrl->final_buf & 1;
  size_t i = (size_t)y * sp + x, o = (size_t)y * dp + x;
  V[o] = one ? u1[i] : u0[i];
  U[o] = one ? v1[i] : v0[i];
}

}  // namespace ofb

using namespace ofb;

static inline int ls_pitch(int W) { return (W + 31) / 32 * 32; }

extern "C" int of_ls_coefficients(const float* I1n, const float* Et, float* coef, int H, int W, int pitch, float h,
                                  void* stream) {
  OF_REQUIRE(!bad_plane(I1n, H, W, pitch) && Et && coef, "of_ls_coefficients: bad plane");
  dim3 blk(32, 8), grd((W + 31) / 32, (H + 7) / 8);
  ls_coef_kernel<<<grd, blk, 0, as_stream(stream)>>>(I1n, Et, coef, (size_t)H * pitch, H, W, pitch, h);
  return check_launch("of_ls_coefficients");
}

extern "C" size_t of_ls_workspace_size(int H, int W, int pitch, int maxnum) {
  Sizer s;
  size_t N = (size_t)H * ls_pitch(W);
  s.take<float>(3 * N);  // reserved (the set-up now forms I1 and Et in shared memory)
  s.take<float>(8 * N);  // coefficient planes
  s.take<float>(4 * N);  // u0, v0, u1, v1
  s.take<LsCtrl>(1);
  s.take<int>((size_t)maxnum + 2);  // run[] and the TMA error flag
  s.take<unsigned int>((size_t)maxnum + 1);  // done[] per pass
  s.take<int>((size_t)maxnum + 1);           // redo[] per pass
  s.take<double>(2 * (size_t)(maxnum > 0 ? maxnum : 1));
  return s.off;
}

extern "C" int of_ls_solve_mode(const float* I0, const float* I1, float* U, float* V, int H, int W, int pitch, float h,
                                int maxnum, double tol, int mode, int* iters_out, double* err_out, void* workspace,
                                size_t workspace_bytes, void* stream) {
  OF_REQUIRE(!bad_plane(I0, H, W, pitch) && I1 && U && V, "of_ls_solve: bad plane");
  OF_REQUIRE(mode == OF_LS_EXACT || mode == OF_LS_FAST, "of_ls_solve: mode must be OF_LS_EXACT or OF_LS_FAST");
  const bool fast = mode == OF_LS_FAST;
  OF_REQUIRE(maxnum >= 0 && maxnum <= 100000, "of_ls_solve: maxnum out of range");
  size_t need = of_ls_workspace_size(H, W, pitch, maxnum);
  if (!workspace || workspace_bytes < need)
    return set_error(OF_ERR_WORKSPACE, "of_ls_solve: workspace too small (%zu < %zu)", workspace_bytes, need);
  cudaStream_t st = as_stream(stream);
  const int P = ls_pitch(W);
  const size_t N = (size_t)H * P;
  Carver c(workspace, workspace_bytes);
  float* nrm = c.take<float>(3 * N);
  float* coef = c.take<float>(8 * N);
  float* uv = c.take<float>(4 * N);
  LsCtrl* ctrl = c.take<LsCtrl>(1);
  int* run = c.take<int>((size_t)maxnum + 2);
  unsigned int* done = c.take<unsigned int>((size_t)maxnum + 1);
  int* redo = c.take<int>((size_t)maxnum + 1);
  double* ss = c.take<double>(2 * (size_t)(maxnum > 0 ? maxnum : 1));
  int* err_flag = run + maxnum + 1;
  (void)nrm;  // normalised frames: formed in shared memory by ls_prep_kernel
  float* ub[2] = {uv, uv + 2 * N};
  float* vb[2] = {uv + N, uv + 3 * N};
  // tensor maps over the whole solve: the 8 coefficient planes (3-D) and the four u / v
  // planes (2-D), all with the 32 x 72 region box of a pass
  CUtensorMap tm_coef, tm_u[2], tm_v[2];
  {
    uint64_t d3[3] = {(uint64_t)W, (uint64_t)H, 8}, s3[2] = {(uint64_t)P * 4, (uint64_t)N * 4};
    uint32_t b3[3] = {LB_RW, LB_CH, 8};  // region rows 1 .. LB_RH - 2
    int rc = tmap_f32(&tm_coef, coef, 3, d3, s3, b3);
    if (rc) return rc;
    uint64_t d2[2] = {(uint64_t)W, (uint64_t)H}, s2[1] = {(uint64_t)P * 4};
    uint32_t b2[2] = {LB_RW, LB_RH};
    for (int q = 0; q < 2; q++) {
      if ((rc = tmap_f32(&tm_u[q], ub[q], 2, d2, s2, b2))) return rc;
      if ((rc = tmap_f32(&tm_v[q], vb[q], 2, d2, s2, b2))) return rc;
    }
  }
  {
    cudaError_t e = OF_SMEM_OPT_IN((ls_pass_kernel<false, LB_WARPS>), lb_smem(false));
    if (e == cudaSuccess) e = OF_SMEM_OPT_IN((ls_pass_kernel<true, 6>), lb_smem(true));
    if (e == cudaSuccess) e = OF_SMEM_OPT_IN((ls_pass_kernel<true, 8>), lb_smem(true));
    if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_ls_solve: %s", cudaGetErrorString(e));
  }
  // control block, flags, counters, redo counts and sums are contiguous: one memset
  cudaMemsetAsync(ctrl, 0, (size_t)((char*)(ss + 2 * (size_t)(maxnum > 0 ? maxnum : 1)) - (char*)ctrl), st);
  {
    const int vec = (pitch % 4) == 0 && ((reinterpret_cast<uintptr_t>(I0) | reinterpret_cast<uintptr_t>(I1)) & 15) == 0;
    ls_max_kernel<<<H < 4 * 148 ? H : 4 * 148, 256, 0, st>>>(I0, I1, H, W, pitch, vec, ctrl->maxkey);
  }
  dim3 rg((W + 255) / 256, H);
  ls_prep_kernel<<<dim3((W + 31) / 32, (H + 7) / 8), 256, 0, st>>>(I0, I1, pitch, ctrl->maxkey, V, U, coef, N,
                                                                 ub[0], vb[0], H, W, P, h);
  double inv_n = 1.0 / ((double)H * (double)W);
  // warps per CTA: 6 for the float64 pass (its registers allow 2 CTAs of 6); 6 for the
  // float32 pass too (96 registers and 75.5 KB of shared memory: 3 CTAs per SM;
  // OFB_LS_FAST_WARPS=8 selects 8 warps, 2 CTAs per SM)
  static const int fast_nw = [] {
    const char* e = getenv("OFB_LS_FAST_WARPS");
    return (e && atoi(e) == 8) ? 8 : 6;
  }();
  const int nw = fast ? fast_nw : LB_WARPS;
  dim3 pgrd((W + LB_TW - 1) / LB_TW, (H + LB_TH - 1) / LB_TH), pblk(32, nw);
  long long nl = 3;
  int p = 0, k0 = 0;
  // pass 0 waits for the set-up in stream order; later passes (and the rollback launch)
  // are programmatic dependents of the pass before them
  cudaLaunchAttribute pdl[1];
  pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  pdl[0].val.programmaticStreamSerializationAllowed = 1;
  auto launch_pass = [&](LbPass PP, bool dependent) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = pgrd;
    cfg.blockDim = pblk;
    cfg.dynamicSmemBytes = lb_smem(fast);
    cfg.stream = st;
    cfg.attrs = dependent ? pdl : nullptr;
    cfg.numAttrs = dependent ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, !fast ? ls_pass_kernel<false, LB_WARPS> : nw == 6 ? ls_pass_kernel<true, 6>
                                                                               : ls_pass_kernel<true, 8>,
                              tm_coef, tm_u[0], tm_v[0],
                              tm_u[1], tm_v[1], ub[0], vb[0], ub[1], vb[1], H, W, P, h, PP, ctrl, ss, run, done, redo,
                              inv_n, tol, err_flag, 1.0f);
  };
  for (; k0 < maxnum; k0 += LB_T, p++) {
    LbPass P0{k0, maxnum - k0 < LB_T ? maxnum - k0 : LB_T, p, 0};
    cudaError_t e = launch_pass(P0, p > 0);
    if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_ls_solve: pass launch: %s", cudaGetErrorString(e));
    nl++;
  }
  if (p > 0) {  // rolls the last pass back if it ran past the stopping sweep
    LbPass PL{k0, 0, p, 1};
    cudaError_t e = launch_pass(PL, true);
    if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_ls_solve: pass launch: %s", cudaGetErrorString(e));
    nl++;
  }
  ls_count_kernel<<<1, 1, 0, st>>>(ctrl, ss, inv_n, err_flag, iters_out, err_out);
  ls_finalize_kernel<<<rg, 256, 0, st>>>(ub[0], vb[0], ub[1], vb[1], V, U, W, P, pitch, ctrl);
  return check_launch("of_ls_solve", nl + 1);
}

extern "C" int of_ls_solve(const float* I0, const float* I1, float* U, float* V, int H, int W, int pitch, float h,
                           int maxnum, double tol, int* iters_out, double* err_out, void* workspace,
                           size_t workspace_bytes, void* stream) {
  return of_ls_solve_mode(I0, I1, U, V, H, W, pitch, h, maxnum, tol, OF_LS_EXACT, iters_out, err_out, workspace,
                          workspace_bytes, stream);
}

// ---------------------------------------------------------------------------------------
// Allocation-free Liu-Shen solve.
//
// Some callers cannot allocate device memory when they run the solver: a host framework
// that owns every allocation through its own pool, a plugin loaded into a process whose
// allocator must not be touched, or a real-time loop where cudaMalloc's implicit device
// synchronisation is not allowed.  This variant needs no workspace argument: its scratch
// is a fixed array compiled into the library (OF_LS_NOALLOC_SCRATCH_BYTES, 4 MiB), which
// every GPU that loads the library holds until the process exits.  That bounds the image:
// of_ls_workspace_size(H, W, pitch, maxnum) must not exceed the array (256 x 256 with the
// reference's 60 sweeps fits).
//
// Host code cannot pass the array's name to a kernel (on the host it only stands for the
// symbol), so the first call on each device looks up its device address with
// cudaGetSymbolAddress while that device is current and caches it; make that first call
// before capturing any stream.  All calls share the one array and it keeps the previous
// call's contents; the solver clears its control words itself.  Calls that overlap on the
// GPU (other streams, other host threads) race on the array.
// ---------------------------------------------------------------------------------------
#include <mutex>

static __device__ __align__(256) unsigned char g_ls_noalloc_scratch[OF_LS_NOALLOC_SCRATCH_BYTES];

static void* ls_noalloc_scratch_ptr(int* rc) {
  static std::mutex mu;
  static void* ptrs[64] = {nullptr};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    *rc = set_error(OF_ERR_CUDA, "of_ls_solve_noalloc: cudaGetDevice failed (%s)", cudaGetErrorString(e));
    return nullptr;
  }
  if (dev < 0 || dev >= 64) {
    *rc = set_error(OF_ERR_UNSUPPORTED, "of_ls_solve_noalloc: device ordinal %d; the address cache covers 0-63", dev);
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!ptrs[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_ls_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      *rc = set_error(OF_ERR_CUDA, "of_ls_solve_noalloc: cudaGetSymbolAddress failed (%s)", cudaGetErrorString(e));
      return nullptr;
    }
    ptrs[dev] = p;
  }
  *rc = OF_OK;
  return ptrs[dev];
}

extern "C" int of_ls_solve_noalloc(const float* I0, const float* I1, float* U, float* V, int H, int W, int pitch,
                                   float h, int maxnum, double tol, int* iters_out, double* err_out, void* stream) {
  OF_REQUIRE(!bad_plane(I0, H, W, pitch) && I1 && U && V, "of_ls_solve_noalloc: bad plane");
  OF_REQUIRE(maxnum >= 0 && maxnum <= 100000, "of_ls_solve_noalloc: maxnum out of range");
  size_t need = of_ls_workspace_size(H, W, pitch, maxnum);
  if (need > (size_t)OF_LS_NOALLOC_SCRATCH_BYTES)
    return set_error(OF_ERR_INVALID,
                     "of_ls_solve_noalloc: a %d x %d solve with %d sweeps needs %zu bytes of scratch, more than the "
                     "library's fixed %d-byte array; use of_ls_solve with a workspace",
                     H, W, maxnum, need, OF_LS_NOALLOC_SCRATCH_BYTES);
  int rc = OF_OK;
  void* scratch = ls_noalloc_scratch_ptr(&rc);
  if (!scratch) return rc;
  return of_ls_solve(I0, I1, U, V, H, W, pitch, h, maxnum, tol, iters_out, err_out, scratch,
                     (size_t)OF_LS_NOALLOC_SCRATCH_BYTES, stream);
}
