// A12-A19 Farneback kernels (src/optical_flow_farneback.cl:72-429).
//
// Arithmetic follows the OpenCL source with its multiply-adds fused the way the CPU
// oracle fixes them (`acc += a*b` -> fmaf(a, b, acc); `a*b + c*d` -> fmaf(a, b, c*d)),
// so GPU and oracle agree bit for bit.  Planar 5-coefficient fields are 5 stacked H x W
// planes sharing one pitch.
//
// Kernels
//  - fb_blur_kernel: separable Gaussian (vertical then horizontal, reflect-101), one plane
//    per blockIdx.z; the input tile with its halo is staged in shared memory once.
//  - fb_polyexp_kernel: 7- (or 5-) tap vertical moments of the clamped neighbourhood into
//    shared memory, then the horizontal combination into the 5 coefficient planes.
//  - fb_iter_kernel: one solver iteration fused — blur5 of M, updateFlow, and
//    updateMatrices into the other M buffer — so M is read once per iteration and the
//    blurred M never leaves the SM.
#include "common.cuh"
#include "tma.cuh"

namespace ofb {

constexpr int FB_MAXKH = 32;
struct FbTaps {
  float g[FB_MAXKH + 1];
};

__host__ __device__ __forceinline__ int fb_low(int y, int last) { return abs(y) % (last + 1); }
__host__ __device__ __forceinline__ int fb_high(int y, int last) { return abs(last - abs(last - y)) % (last + 1); }
// reflect-101 mapping of the gaussianBlur kernels (idx_row_low / idx_row_high / idx_col)
__device__ __forceinline__ int fb_row(int y, int rows) {
  if (y < 0) return fb_low(y, rows - 1);
  if (y > rows - 1) return fb_high(y, rows - 1);
  return y;
}
__device__ __forceinline__ int fb_col(int x, int cols) { return fb_low(fb_high(x, cols - 1), cols - 1); }

constexpr int FBB_TW = 64, FBB_TH = 16;

// Blur of plane blockIdx.z: out = H(V(src)).  smem: input (TH+2kh) x (TW+2kh), vertical
// result TH x (TW+2kh).  KHC > 0: the half width is the compile-time KHC (the Farneback
// levels' frame smoothing uses 1 and 4), so the tile widths are constants and the tap
// loops unroll; KHC = 0: kh at run time.
template <int KHC = 0>
__global__ void __launch_bounds__(256) fb_blur_kernel(const float* __restrict__ src, float* __restrict__ dst, int H,
                                                      int W, int pitch, FbTaps t, int khrt) {
  extern __shared__ float sm[];
  const int kh = KHC > 0 ? KHC : khrt;
  const int iw = FBB_TW + 2 * kh, ih = FBB_TH + 2 * kh;
  float* tin = sm;
  float* tv = sm + ih * iw;
  const size_t plane = (size_t)H * pitch * blockIdx.z;
  const float* s = src + plane;
  const int x0 = blockIdx.x * FBB_TW, y0 = blockIdx.y * FBB_TH;
  // interior tiles (halo inside the image) need no reflect-101 mapping
  const bool inside = x0 >= kh && y0 >= kh && x0 + FBB_TW + kh <= W && y0 + FBB_TH + kh <= H;
  for (int i = threadIdx.x; i < ih * iw; i += blockDim.x) {
    int ly = i / iw, lx = i - ly * iw;
    const int gy = y0 - kh + ly, gx = x0 - kh + lx;
    tin[i] = inside ? s[(size_t)gy * pitch + gx] : s[(size_t)fb_row(gy, H) * pitch + fb_col(gx, W)];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < FBB_TH * iw; i += blockDim.x) {
    int ly = i / iw, lx = i - ly * iw;
    const float* c = tin + (ly + kh) * iw + lx;
    float acc = __fmul_rn(c[0], t.g[0]);
#pragma unroll
    for (int j = 1; j <= (KHC > 0 ? KHC : FB_MAXKH); j++) {
      if (KHC == 0 && j > kh) break;
      acc = __fmaf_rn(__fadd_rn(c[-j * iw], c[j * iw]), t.g[j], acc);
    }
    tv[i] = acc;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < FBB_TH * FBB_TW; i += blockDim.x) {
    int ly = i / FBB_TW, lx = i - ly * FBB_TW;
    int y = y0 + ly, x = x0 + lx;
    if (y >= H || x >= W) continue;
    const float* r = tv + ly * iw + lx + kh;
    float res = __fmul_rn(r[0], t.g[0]);
#pragma unroll
    for (int j = 1; j <= (KHC > 0 ? KHC : FB_MAXKH); j++) {
      if (KHC == 0 && j > kh) break;
      res = __fmaf_rn(__fadd_rn(r[-j], r[j]), t.g[j], res);
    }
    dst[plane + (size_t)y * pitch + x] = res;
  }
}

// boxFilter5 (:350-406): clamped borders, plain sums, one plane per blockIdx.z
__global__ void __launch_bounds__(256) fb_box_kernel(const float* __restrict__ src, float* __restrict__ dst, int H,
                                                     int W, int pitch, int kh, float inv) {
  extern __shared__ float sm[];
  const int iw = FBB_TW + 2 * kh, ih = FBB_TH + 2 * kh;
  float* tin = sm;
  float* tv = sm + ih * iw;
  const size_t plane = (size_t)H * pitch * blockIdx.z;
  const float* s = src + plane;
  const int x0 = blockIdx.x * FBB_TW, y0 = blockIdx.y * FBB_TH;
  for (int i = threadIdx.x; i < ih * iw; i += blockDim.x) {
    int ly = i / iw, lx = i - ly * iw;
    tin[i] = s[(size_t)clampi(y0 - kh + ly, 0, H - 1) * pitch + clampi(x0 - kh + lx, 0, W - 1)];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < FBB_TH * iw; i += blockDim.x) {
    int ly = i / iw, lx = i - ly * iw;
    const float* c = tin + (ly + kh) * iw + lx;
    float acc = c[0];
    for (int j = 1; j <= kh; j++) acc = __fadd_rn(acc, __fadd_rn(c[-j * iw], c[j * iw]));
    tv[i] = acc;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < FBB_TH * FBB_TW; i += blockDim.x) {
    int ly = i / FBB_TW, lx = i - ly * FBB_TW;
    int y = y0 + ly, x = x0 + lx;
    if (y >= H || x >= W) continue;
    const float* r = tv + ly * iw + lx + kh;
    float res = r[0];
    for (int j = 1; j <= kh; j++) res = __fadd_rn(res, __fadd_rn(r[-j], r[j]));
    dst[plane + (size_t)y * pitch + x] = __fmul_rn(res, inv);
  }
}

struct FbPoly {
  float g[8], xg[8], xxg[8], ig[4];
  int n;
};

// polynomialExpansion: one CTA = 1 row segment of 256-2n outputs (the reference's
// (256,1) work-group shape), vertical moments for 256 clamped columns in smem.
constexpr int FBP_T = 256;
__global__ void __launch_bounds__(FBP_T) fb_polyexp_kernel(const float* __restrict__ src, float* __restrict__ dst,
                                                           int H, int W, int pitch, FbPoly P) {
  __shared__ float row[3][FBP_T];
  const int n = P.n;
  const int y = blockIdx.y, tx = threadIdx.x;
  const int x = blockIdx.x * (FBP_T - 2 * n) + tx - n;
  const int xw = clampi(x, 0, W - 1);
  float r0 = __fmul_rn(src[(size_t)y * pitch + xw], P.g[0]), r1 = 0.f, r2 = 0.f;
  for (int k = 1; k <= n; k++) {
    float t0 = src[(size_t)max(y - k, 0) * pitch + xw];
    float t1 = src[(size_t)min(y + k, H - 1) * pitch + xw];
    r0 = __fmaf_rn(P.g[k], __fadd_rn(t0, t1), r0);
    r1 = __fmaf_rn(P.xg[k], __fsub_rn(t1, t0), r1);
    r2 = __fmaf_rn(P.xxg[k], __fadd_rn(t0, t1), r2);
  }
  row[0][tx] = r0;
  row[1][tx] = r1;
  row[2][tx] = r2;
  __syncthreads();
  if (tx >= n && tx + n < FBP_T && x < W) {
    float b1 = __fmul_rn(P.g[0], row[0][tx]), b3 = __fmul_rn(P.g[0], row[1][tx]), b5 = __fmul_rn(P.g[0], row[2][tx]);
    float b2 = 0.f, b4 = 0.f, b6 = 0.f;
    for (int k = 1; k <= n; k++) {
      float sp = __fadd_rn(row[0][tx + k], row[0][tx - k]), sm_ = __fsub_rn(row[0][tx + k], row[0][tx - k]);
      b1 = __fmaf_rn(sp, P.g[k], b1);
      b4 = __fmaf_rn(sp, P.xxg[k], b4);
      b2 = __fmaf_rn(sm_, P.xg[k], b2);
      b3 = __fmaf_rn(__fadd_rn(row[1][tx + k], row[1][tx - k]), P.g[k], b3);
      b6 = __fmaf_rn(__fsub_rn(row[1][tx + k], row[1][tx - k]), P.xg[k], b6);
      b5 = __fmaf_rn(__fadd_rn(row[2][tx + k], row[2][tx - k]), P.g[k], b5);
    }
    const size_t pl = (size_t)H * pitch, i = (size_t)y * pitch + x;
    dst[i] = __fmul_rn(b3, P.ig[0]);
    dst[pl + i] = __fmul_rn(b2, P.ig[0]);
    dst[2 * pl + i] = __fmaf_rn(b1, P.ig[1], __fmul_rn(b5, P.ig[2]));
    dst[3 * pl + i] = __fmaf_rn(b1, P.ig[1], __fmul_rn(b4, P.ig[2]));
    dst[4 * pl + i] = __fmul_rn(b6, P.ig[3]);
  }
}

// Tiled polynomial expansion for a compile-time half width N (polyN 5 and 7, the
// reference's two settings).  The row kernel above loads 2N+1 samples per output from
// global memory; here a CTA covers FBQ_R rows x FBQ_OW columns.  Each thread walks one
// column down the tile with a register window (FBQ_R + 2N loads for FBQ_R outputs) and
// leaves the three vertical moments in shared memory; then each thread takes 8 consecutive
// outputs of one row with a register window along the row.  The arithmetic of every
// output is the row kernel's, in the same order.  The moment rows are padded by one float
// per 8 columns, so the 8-column segments of a warp's lanes fall in distinct banks.
//
// BLUR = true fuses the level's 3-tap frame blur in front (gaussianBlur with kh = 1 and
// reflect-101 borders, :160-253, then the expansion of the blurred frame, as at the
// pyramid's full-size level where no resize lies between them).  The CTA first computes
// the vertical blur V of its rows for the CW + 2 columns around its window into shared
// memory (the storage the moments use later), then each thread forms the blurred samples
// of its column from V and its two reflect-101 neighbours.  Every blurred value is the
// blur kernel's, operation for operation, so the result equals of_fb_blur followed by
// of_fb_polyexp.  Needs H, W >= 3.
constexpr int FBQ_OW = 240, FBQ_R = 8, FBQ_SEG = 8;
__device__ __forceinline__ int fbq_col(int c) { return c + (c >> 3); }
template <int N, bool BLUR>
__global__ void __launch_bounds__(256) fb_polyexp_tile_kernel(const float* __restrict__ src, float* __restrict__ dst,
                                                              int H, int W, int pitch, FbPoly P, int vec, float bg0,
                                                              float bg1) {
  constexpr int CW = FBQ_OW + 2 * N;          // columns that get vertical moments
  constexpr int CWP = CW + (CW >> 3) + 1;     // padded row length
  constexpr int WIN = FBQ_SEG + 2 * N;
  constexpr int NR = FBQ_R + 2 * N;           // rows of the vertical window
  static_assert(CW + 2 <= 256 && NR * 256 <= 3 * FBQ_R * CWP, "blur rows must fit the moment storage");
  __shared__ float mom[3][FBQ_R][CWP];
  const int x0 = blockIdx.x * FBQ_OW, y0 = blockIdx.y * FBQ_R, tx = threadIdx.x;
  float c[NR];
  if (BLUR) {
    // V(y, x) = g1 (src[y-1] + src[y+1]) + g0 src[y] at the window's clamped rows y, for
    // the columns clamp(x0 - N - 1 + j), j <= CW + 1
    float (*vs)[256] = reinterpret_cast<float (*)[256]>(&mom[0][0][0]);
    if (tx < CW + 2) {
      const float* col = src + clampi(x0 - N - 1 + tx, 0, W - 1);
      if (y0 - N - 1 >= 0 && y0 + FBQ_R + N < H) {  // rows y0-N-1 .. y0+R+N, all inside
        float r[NR + 2];
#pragma unroll
        for (int q = 0; q < NR + 2; q++) r[q] = col[(size_t)(y0 - N - 1 + q) * pitch];
#pragma unroll
        for (int q = 0; q < NR; q++) vs[q][tx] = __fmaf_rn(__fadd_rn(r[q], r[q + 2]), bg1, __fmul_rn(r[q + 1], bg0));
      } else {
#pragma unroll
        for (int q = 0; q < NR; q++) {
          const int y = clampi(y0 - N + q, 0, H - 1);
          const float up = col[(size_t)fb_row(y - 1, H) * pitch], mid = col[(size_t)y * pitch],
                      dn = col[(size_t)fb_row(y + 1, H) * pitch];
          vs[q][tx] = __fmaf_rn(__fadd_rn(up, dn), bg1, __fmul_rn(mid, bg0));
        }
      }
    }
    __syncthreads();
    if (tx < CW) {
      // column u = x0 - N + tx, clamped to xw; V's column j holds clamp(x0 - N - 1 + j)
      const int u = x0 - N + tx;
      int jl = tx, jr = tx + 2;  // xw - 1 and xw + 1 inside the image
      if (u <= 0) jl = jr = N + 2 - x0;           // xw = 0: both reflect-101 neighbours are column 1
      else if (u >= W - 1) jl = jr = W - 1 - x0 + N;  // xw = W - 1: both are column W - 2
#pragma unroll
      for (int q = 0; q < NR; q++) c[q] = __fmaf_rn(__fadd_rn(vs[q][jl], vs[q][jr]), bg1, __fmul_rn(vs[q][tx + 1], bg0));
    }
    __syncthreads();  // V is overwritten by the moments below
  }
  if (tx < CW) {
    if (!BLUR) {
      const int xw = clampi(x0 - N + tx, 0, W - 1);
#pragma unroll
      for (int q = 0; q < NR; q++) c[q] = src[(size_t)clampi(y0 - N + q, 0, H - 1) * pitch + xw];
    }
#pragma unroll
    for (int r = 0; r < FBQ_R; r++) {
      float r0 = __fmul_rn(c[r + N], P.g[0]), r1 = 0.f, r2 = 0.f;
#pragma unroll
      for (int k = 1; k <= N; k++) {
        const float t0 = c[r + N - k], t1 = c[r + N + k];
        r0 = __fmaf_rn(P.g[k], __fadd_rn(t0, t1), r0);
        r1 = __fmaf_rn(P.xg[k], __fsub_rn(t1, t0), r1);
        r2 = __fmaf_rn(P.xxg[k], __fadd_rn(t0, t1), r2);
      }
      mom[0][r][fbq_col(tx)] = r0;
      mom[1][r][fbq_col(tx)] = r1;
      mom[2][r][fbq_col(tx)] = r2;
    }
  }
  __syncthreads();
  constexpr int NSEG = FBQ_OW / FBQ_SEG;
  if (tx >= FBQ_R * NSEG) return;
  const int r = tx / NSEG, sg = tx - r * NSEG;
  const int y = y0 + r, xs = x0 + sg * FBQ_SEG;
  if (y >= H || xs >= W) return;
  // output column xs + i is moment column sg*8 + i + N; its window is sg*8 .. sg*8 + 7 + 2N
  float a0[WIN], a1[WIN], a2[WIN];
#pragma unroll
  for (int q = 0; q < WIN; q++) {
    const int cc = sg * (FBQ_SEG + 1) + q + (q >> 3);  // fbq_col(sg * 8 + q)
    a0[q] = mom[0][r][cc];
    a1[q] = mom[1][r][cc];
    a2[q] = mom[2][r][cc];
  }
  const size_t pl = (size_t)H * pitch;
  float o[5][FBQ_SEG];
#pragma unroll
  for (int i = 0; i < FBQ_SEG; i++) {
    const int t = i + N;
    float b1 = __fmul_rn(P.g[0], a0[t]), b3 = __fmul_rn(P.g[0], a1[t]), b5 = __fmul_rn(P.g[0], a2[t]);
    float b2 = 0.f, b4 = 0.f, b6 = 0.f;
#pragma unroll
    for (int k = 1; k <= N; k++) {
      const float sp = __fadd_rn(a0[t + k], a0[t - k]), sm_ = __fsub_rn(a0[t + k], a0[t - k]);
      b1 = __fmaf_rn(sp, P.g[k], b1);
      b4 = __fmaf_rn(sp, P.xxg[k], b4);
      b2 = __fmaf_rn(sm_, P.xg[k], b2);
      b3 = __fmaf_rn(__fadd_rn(a1[t + k], a1[t - k]), P.g[k], b3);
      b6 = __fmaf_rn(__fsub_rn(a1[t + k], a1[t - k]), P.xg[k], b6);
      b5 = __fmaf_rn(__fadd_rn(a2[t + k], a2[t - k]), P.g[k], b5);
    }
    o[0][i] = __fmul_rn(b3, P.ig[0]);
    o[1][i] = __fmul_rn(b2, P.ig[0]);
    o[2][i] = __fmaf_rn(b1, P.ig[1], __fmul_rn(b5, P.ig[2]));
    o[3][i] = __fmaf_rn(b1, P.ig[1], __fmul_rn(b4, P.ig[2]));
    o[4][i] = __fmul_rn(b6, P.ig[3]);
  }
  const size_t i0 = (size_t)y * pitch + xs;
  if (vec && xs + FBQ_SEG <= W) {
#pragma unroll
    for (int p = 0; p < 5; p++) {
      float4* d = reinterpret_cast<float4*>(dst + p * pl + i0);
      d[0] = make_float4(o[p][0], o[p][1], o[p][2], o[p][3]);
      d[1] = make_float4(o[p][4], o[p][5], o[p][6], o[p][7]);
    }
  } else {
#pragma unroll
    for (int i = 0; i < FBQ_SEG; i++)
      if (xs + i < W) {
#pragma unroll
        for (int p = 0; p < 5; p++) dst[p * pl + i0 + i] = o[p][i];
      }
  }
}

__constant__ float c_border[6] = {0.14f, 0.14f, 0.4472f, 0.4472f, 0.4472f, 1.f};

// updateMatrices for pixel (y, x) given its flow; writes the 5 M planes.
__device__ __forceinline__ void fb_matrices_at(int y, int x, float dx, float dy, const float* __restrict__ R0,
                                               const float* __restrict__ R1, float* __restrict__ M, int H, int W,
                                               int pitch) {
  const size_t pl = (size_t)H * pitch, i = (size_t)y * pitch + x;
  float fx = __fadd_rn((float)x, dx), fy = __fadd_rn((float)y, dy);
  float flx = floorf(fx), fly = floorf(fy);
  int x1 = (int)flx, y1 = (int)fly;
  fx = __fsub_rn(fx, (float)x1);
  fy = __fsub_rn(fy, (float)y1);
  float r2, r3, r4, r5, r6;
  if (x1 >= 0 && y1 >= 0 && x1 < W - 1 && y1 < H - 1) {
    float a00 = __fmul_rn(__fsub_rn(1.f, fx), __fsub_rn(1.f, fy)), a01 = __fmul_rn(fx, __fsub_rn(1.f, fy));
    float a10 = __fmul_rn(__fsub_rn(1.f, fx), fy), a11 = __fmul_rn(fx, fy);
    float rr[5];
    const size_t j = (size_t)y1 * pitch + x1;
#pragma unroll
    for (int p = 0; p < 5; p++) {
      const float* R = R1 + p * pl;
      float tt = __fmaf_rn(a00, R[j], __fmul_rn(a01, R[j + 1]));
      tt = __fmaf_rn(a10, R[j + pitch], tt);
      tt = __fmaf_rn(a11, R[j + pitch + 1], tt);
      rr[p] = tt;
    }
    r2 = rr[0];
    r3 = rr[1];
    r4 = __fmul_rn(__fadd_rn(R0[2 * pl + i], rr[2]), 0.5f);
    r5 = __fmul_rn(__fadd_rn(R0[3 * pl + i], rr[3]), 0.5f);
    r6 = __fmul_rn(__fadd_rn(R0[4 * pl + i], rr[4]), 0.25f);
  } else {
    r2 = r3 = 0.f;
    r4 = R0[2 * pl + i];
    r5 = R0[3 * pl + i];
    r6 = __fmul_rn(R0[4 * pl + i], 0.5f);
  }
  r2 = __fmul_rn(__fsub_rn(R0[i], r2), 0.5f);
  r3 = __fmul_rn(__fsub_rn(R0[pl + i], r3), 0.5f);
  r2 = __fadd_rn(r2, __fmaf_rn(r4, dy, __fmul_rn(r6, dx)));
  r3 = __fadd_rn(r3, __fmaf_rn(r6, dy, __fmul_rn(r5, dx)));
  float scale = __fmul_rn(c_border[min(x, 5)], c_border[min(y, 5)]);
  scale = __fmul_rn(scale, c_border[min(W - x - 1, 5)]);
  scale = __fmul_rn(scale, c_border[min(H - y - 1, 5)]);
  r2 = __fmul_rn(r2, scale);
  r3 = __fmul_rn(r3, scale);
  r4 = __fmul_rn(r4, scale);
  r5 = __fmul_rn(r5, scale);
  r6 = __fmul_rn(r6, scale);
  M[i] = __fmaf_rn(r4, r4, __fmul_rn(r6, r6));
  M[pl + i] = __fmul_rn(__fadd_rn(r4, r5), r6);
  M[2 * pl + i] = __fmaf_rn(r5, r5, __fmul_rn(r6, r6));
  M[3 * pl + i] = __fmaf_rn(r4, r2, __fmul_rn(r6, r3));
  M[4 * pl + i] = __fmaf_rn(r6, r2, __fmul_rn(r5, r3));
}

__device__ __forceinline__ void fb_flow_from(float g11, float g12, float g22, float h1, float h2, float* fx,
                                             float* fy) {
  float detInv = __fdiv_rn(1.f, __fadd_rn(__fmaf_rn(g11, g22, -__fmul_rn(g12, g12)), 1e-3f));
  *fx = __fmul_rn(__fmaf_rn(g11, h2, -__fmul_rn(g12, h1)), detInv);
  *fy = __fmul_rn(__fmaf_rn(g22, h1, -__fmul_rn(g12, h2)), detInv);
}

__global__ void fb_update_matrices_kernel(const float* __restrict__ flowx, const float* __restrict__ flowy,
                                          const float* __restrict__ R0, const float* __restrict__ R1,
                                          float* __restrict__ M, int H, int W, int pitch) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  size_t i = (size_t)y * pitch + x;
  fb_matrices_at(y, x, flowx[i], flowy[i], R0, R1, M, H, W, pitch);
}

__global__ void fb_update_flow_kernel(const float* __restrict__ M, float* __restrict__ flowx, float* __restrict__ flowy,
                                      int H, int W, int pitch) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  const size_t pl = (size_t)H * pitch, i = (size_t)y * pitch + x;
  float fx, fy;
  fb_flow_from(M[i], M[pl + i], M[2 * pl + i], M[3 * pl + i], M[4 * pl + i], &fx, &fy);
  flowx[i] = fx;
  flowy[i] = fy;
}

// Fused iteration.  CTA tile: FBI_TW x FBI_TH outputs, all 5 planes.  Per plane the input
// tile (+kh halo) is staged, blurred vertically into tv, horizontally into registers; the
// 5 blurred values of each output pixel then feed updateFlow and updateMatrices.
constexpr int FBI_TW = 32, FBI_TH = 16;
__global__ void __launch_bounds__(256) fb_iter_kernel(const float* __restrict__ Min, float* __restrict__ Mout,
                                                      const float* __restrict__ R0, const float* __restrict__ R1,
                                                      float* __restrict__ flowx, float* __restrict__ flowy, int H,
                                                      int W, int pitch, FbTaps t, int kh, int upd) {
  extern __shared__ float sm[];
  const int iw = FBI_TW + 2 * kh, ih = FBI_TH + 2 * kh;
  float* tin = sm;
  float* tv = sm + ih * iw;
  const size_t pl = (size_t)H * pitch;
  const int x0 = blockIdx.x * FBI_TW, y0 = blockIdx.y * FBI_TH;
  // each thread owns 2 output pixels of the 32x16 tile
  float res[2][5];
#pragma unroll
  for (int p = 0; p < 5; p++) {
    const float* s = Min + p * pl;
    for (int i = threadIdx.x; i < ih * iw; i += blockDim.x) {
      int ly = i / iw, lx = i - ly * iw;
      tin[i] = s[(size_t)fb_row(y0 - kh + ly, H) * pitch + fb_col(x0 - kh + lx, W)];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < FBI_TH * iw; i += blockDim.x) {
      int ly = i / iw, lx = i - ly * iw;
      const float* c = tin + (ly + kh) * iw + lx;
      float acc = __fmul_rn(c[0], t.g[0]);
      for (int j = 1; j <= kh; j++) acc = __fmaf_rn(__fadd_rn(c[-j * iw], c[j * iw]), t.g[j], acc);
      tv[i] = acc;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 2; q++) {
      int o = threadIdx.x + q * 256;
      int ly = o / FBI_TW, lx = o - ly * FBI_TW;
      const float* r = tv + ly * iw + lx + kh;
      float v = __fmul_rn(r[0], t.g[0]);
      for (int j = 1; j <= kh; j++) v = __fmaf_rn(__fadd_rn(r[-j], r[j]), t.g[j], v);
      res[q][p] = v;
    }
    __syncthreads();
  }
#pragma unroll
  for (int q = 0; q < 2; q++) {
    int o = threadIdx.x + q * 256;
    int ly = o / FBI_TW, lx = o - ly * FBI_TW;
    int y = y0 + ly, x = x0 + lx;
    if (y >= H || x >= W) continue;
    float fx, fy;
    fb_flow_from(res[q][0], res[q][1], res[q][2], res[q][3], res[q][4], &fx, &fy);
    size_t i = (size_t)y * pitch + x;
    flowx[i] = fx;
    flowy[i] = fy;
    if (upd) fb_matrices_at(y, x, fx, fy, R0, R1, Mout, H, W, pitch);
  }
}

// Fused iteration for a compile-time half window KH (the default windowSize 33 -> KH 16).
// CTA: 64 x 32 outputs, 256 threads.  Per plane: the (32+2KH) x (64+2KH) input tile is
// staged once; the vertical pass gives each thread 8 consecutive rows of one column
// (8+2KH values read once, 8 outputs), the horizontal pass 8 consecutive columns of one
// row; taps fully unrolled in the reference order.  The thread's 8 pixels x 5 blurred
// planes stay in registers for updateFlow / updateMatrices.
constexpr int FBK_TW = 64, FBK_TH = 32, FBK_R = 8;
constexpr long long FBK_WAIT_LIMIT = 1ll << 22;
template <int KH>
struct FbkGeom {
  static constexpr int IW = FBK_TW + 2 * KH, IH = FBK_TH + 2 * KH;
  static constexpr int STAGE = IW * IH * 4;  // bytes of one staged input plane tile
  static constexpr size_t SMEM = 2 * STAGE + (size_t)FBK_TH * IW * 4 + 128 + 128;
  static_assert(2 * STAGE >= 5 * FBK_TH * FBK_TW * 4, "the epilogue's plane transpose reuses the stages");
};

// reflect-101 fix-up of a staged tile: cells outside the image take their mirror image.
// Only those cells are visited: the out-of-image rows [0, rt) and [rb, IH) in full, and
// the out-of-image columns [0, cl) and [cr, IW) of the rows in between.
template <int KH>
__device__ __forceinline__ void fbk_reflect(float* tin, int x0, int y0, int H, int W) {
  constexpr int IW = FbkGeom<KH>::IW, IH = FbkGeom<KH>::IH;
  const int rt = min(max(KH - y0, 0), IH), rb = max(min(H - (y0 - KH), IH), rt);
  const int cl = min(max(KH - x0, 0), IW), cr = max(min(W - (x0 - KH), IW), cl);
  const int nt = rt * IW, nb = (IH - rb) * IW, side = cl + (IW - cr), n = nt + nb + (rb - rt) * side;
  for (int i = threadIdx.x; i < n; i += 256) {
    int ly, lx;
    if (i < nt) {
      ly = i / IW;
      lx = i - ly * IW;
    } else if (i < nt + nb) {
      const int k = i - nt;
      ly = rb + k / IW;
      lx = k - (ly - rb) * IW;
    } else {
      const int k = i - nt - nb, r = k / side, c = k - r * side;
      ly = rt + r;
      lx = c < cl ? c : cr + (c - cl);
    }
    const int gy = y0 - KH + ly, gx = x0 - KH + lx;
    const int sy = fb_row(gy, H) - (y0 - KH), sx = fb_col(gx, W) - (x0 - KH);
    if (sy < 0 || sy >= IH || sx < 0 || sx >= IW) continue;  // only outside every used window
    tin[ly * IW + lx] = tin[sy * IW + sx];
  }
}

// Fused iteration for a compile-time half window KH (windowSize 33 -> KH 16).
// CTA: 64 x 32 outputs, 256 threads.  The 5 planes' (32+2KH) x (64+2KH) input tiles arrive
// by TMA (a 3-D map over the 5 stacked planes, one plane per box) into two stages, so plane
// p+1 is in flight while plane p is blurred; border tiles get their reflect-101 cells
// filled in shared memory (one reflection: H, W >= KH + 1).  The vertical pass gives each
// thread 8 consecutive rows of one column, the horizontal pass 8 consecutive columns of one
// row; taps fully unrolled in the reference order.  The 8 pixels x 5 blurred planes of a
// thread stay in registers for updateFlow / updateMatrices.
template <int KH>
__global__ void __launch_bounds__(256, 2) fb_iter_fixed_kernel(const __grid_constant__ CUtensorMap tm_m,
                                                               float* __restrict__ Mout, const float* __restrict__ R0,
                                                               const float* __restrict__ R1, float* __restrict__ flowx,
                                                               float* __restrict__ flowy, int H, int W, int pitch,
                                                               FbTaps t, int upd) {
  using G = FbkGeom<KH>;
  constexpr int IW = G::IW;
  extern __shared__ __align__(128) unsigned char fbk_raw[];
  unsigned char* base = fbk_raw + ((128 - (smem_u32(fbk_raw) & 127)) & 127);
  float* stage[2] = {reinterpret_cast<float*>(base), reinterpret_cast<float*>(base + G::STAGE)};
  float* tv = reinterpret_cast<float*>(base + 2 * G::STAGE);  // FBK_TH x IW
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + 2 * G::STAGE + FBK_TH * IW * 4);
  const int x0 = blockIdx.x * FBK_TW, y0 = blockIdx.y * FBK_TH;
  const bool border = x0 < KH || y0 < KH || x0 + FBK_TW + KH > W || y0 + FBK_TH + KH > H;
  const int hx = (threadIdx.x & 7) * FBK_R, hy = threadIdx.x >> 3;  // horizontal-pass assignment
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 0; q < 2; q++) {
      mbar_expect_tx(&bar[q], G::STAGE);
      tma_load_3d(stage[q], &tm_m, x0 - KH, y0 - KH, q, &bar[q]);
    }
  }
  float g[KH + 1];
#pragma unroll
  for (int j = 0; j <= KH; j++) g[j] = t.g[j];
  float res[5][FBK_R];
  bool ok = true;
#pragma unroll
  for (int p = 0; p < 5; p++) {
    float* tin = stage[p & 1];
    if (ok && !mbar_wait(&bar[p & 1], (p >> 1) & 1, FBK_WAIT_LIMIT)) ok = false;
    if (border) {
      fbk_reflect<KH>(tin, x0, y0, H, W);
      __syncthreads();
    }
    // vertical: work item = (column, 8-row group)
    for (int it = threadIdx.x; it < IW * (FBK_TH / FBK_R); it += 256) {
      const int col = it % IW, r0 = (it / IW) * FBK_R;
      float c[FBK_R + 2 * KH];
#pragma unroll
      for (int q = 0; q < FBK_R + 2 * KH; q++) c[q] = tin[(r0 + q) * IW + col];
#pragma unroll
      for (int r = 0; r < FBK_R; r++) {
        float acc = __fmul_rn(c[r + KH], g[0]);
#pragma unroll
        for (int j = 1; j <= KH; j++) acc = __fmaf_rn(__fadd_rn(c[r + KH - j], c[r + KH + j]), g[j], acc);
        tv[(r0 + r) * IW + col] = acc;
      }
    }
    __syncthreads();
    // the stage is free again: bring plane p+2 into it while the horizontal pass runs
    if (threadIdx.x == 0 && p + 2 < 5 && ok) {
      mbar_expect_tx(&bar[p & 1], G::STAGE);
      tma_load_3d(tin, &tm_m, x0 - KH, y0 - KH, p + 2, &bar[p & 1]);
    }
    {
      float c[FBK_R + 2 * KH];
#pragma unroll
      for (int q = 0; q < FBK_R + 2 * KH; q++) c[q] = tv[hy * IW + hx + q];
#pragma unroll
      for (int r = 0; r < FBK_R; r++) {
        float acc = __fmul_rn(c[r + KH], g[0]);
#pragma unroll
        for (int j = 1; j <= KH; j++) acc = __fmaf_rn(__fadd_rn(c[r + KH - j], c[r + KH + j]), g[j], acc);
        res[p][r] = acc;
      }
    }
    __syncthreads();
  }
  // The blurred planes go through shared memory (the staging buffers are free now) so the
  // epilogue runs one pixel per lane: its flow / R0 / M accesses and the R1 gathers of
  // neighbouring lanes fall on neighbouring addresses.
  float* rs = stage[0];  // [plane][FBK_TH][FBK_TW], 40 KB of the two 24 KB stages
#pragma unroll
  for (int p = 0; p < 5; p++) {
    float4* d = reinterpret_cast<float4*>(rs + (p * FBK_TH + hy) * FBK_TW + hx);
    d[0] = make_float4(res[p][0], res[p][1], res[p][2], res[p][3]);
    d[1] = make_float4(res[p][4], res[p][5], res[p][6], res[p][7]);
  }
  __syncthreads();
#pragma unroll 1
  for (int o = threadIdx.x; o < FBK_TH * FBK_TW; o += 256) {
    const int ly = o / FBK_TW, lx = o - ly * FBK_TW;
    const int y = y0 + ly, x = x0 + lx;
    if (y >= H || x >= W) continue;
    const size_t i = (size_t)y * pitch + x;
    if (!ok) {  // a tile copy never arrived: the tile's flow is reported as NaN
      flowx[i] = __int_as_float(0x7fc00000);
      flowy[i] = __int_as_float(0x7fc00000);
      continue;
    }
    const float* q = rs + ly * FBK_TW + lx;
    float fx, fy;
    fb_flow_from(q[0], q[FBK_TH * FBK_TW], q[2 * FBK_TH * FBK_TW], q[3 * FBK_TH * FBK_TW], q[4 * FBK_TH * FBK_TW], &fx,
                 &fy);
    flowx[i] = fx;
    flowy[i] = fy;
    if (upd) fb_matrices_at(y, x, fx, fy, R0, R1, Mout, H, W, pitch);
  }
}

static FbTaps make_taps(const float* gk, int kh) {
  FbTaps t{};
  for (int j = 0; j <= kh; j++) t.g[j] = gk[j];
  return t;
}

}  // namespace ofb

using namespace ofb;

extern "C" int of_fb_blur(const float* src, float* dst, int H, int W, int pitch, int planes, const float* gk, int kh,
                          void* stream) {
  OF_REQUIRE(!bad_plane(src, H, W, pitch) && dst && src != dst, "of_fb_blur: bad plane");
  OF_REQUIRE(gk && kh >= 0 && kh <= FB_MAXKH && planes >= 1 && planes <= 65535, "of_fb_blur: bad kernel");
  size_t smem = sizeof(float) * ((size_t)(FBB_TH + 2 * kh) * (FBB_TW + 2 * kh) + (size_t)FBB_TH * (FBB_TW + 2 * kh));
  if (smem > 48 * 1024) {
    cudaError_t e = OF_SMEM_OPT_IN(fb_blur_kernel<0>, 64 * 1024);
    if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_fb_blur: %s", cudaGetErrorString(e));
  }
  dim3 grid((W + FBB_TW - 1) / FBB_TW, (H + FBB_TH - 1) / FBB_TH, planes);
  const FbTaps tp = make_taps(gk, kh);
  if (kh == 1)
    fb_blur_kernel<1><<<grid, 256, smem, as_stream(stream)>>>(src, dst, H, W, pitch, tp, kh);
  else if (kh == 4)
    fb_blur_kernel<4><<<grid, 256, smem, as_stream(stream)>>>(src, dst, H, W, pitch, tp, kh);
  else
    fb_blur_kernel<0><<<grid, 256, smem, as_stream(stream)>>>(src, dst, H, W, pitch, tp, kh);
  return check_launch("of_fb_blur");
}

extern "C" int of_fb_box5(const float* src, float* dst, int H, int W, int pitch, int kh, void* stream) {
  OF_REQUIRE(!bad_plane(src, H, W, pitch) && dst && src != dst, "of_fb_box5: bad plane");
  OF_REQUIRE(kh >= 0 && kh <= FB_MAXKH, "of_fb_box5: bad kernel");
  size_t smem = sizeof(float) * ((size_t)(FBB_TH + 2 * kh) * (FBB_TW + 2 * kh) + (size_t)FBB_TH * (FBB_TW + 2 * kh));
  if (smem > 48 * 1024) {
    cudaError_t e = OF_SMEM_OPT_IN(fb_box_kernel, 64 * 1024);
    if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_fb_box5: %s", cudaGetErrorString(e));
  }
  dim3 grid((W + FBB_TW - 1) / FBB_TW, (H + FBB_TH - 1) / FBB_TH, 5);
  float inv = 1.f / (float)((1 + 2 * kh) * (1 + 2 * kh));
  fb_box_kernel<<<grid, 256, smem, as_stream(stream)>>>(src, dst, H, W, pitch, kh, inv);
  return check_launch("of_fb_box5");
}

extern "C" int of_fb_polyexp(const float* src, float* dst, int H, int W, int pitch, const of_fb_poly_consts* c,
                             void* stream) {
  OF_REQUIRE(!bad_plane(src, H, W, pitch) && dst && c, "of_fb_polyexp: bad plane");
  OF_REQUIRE(c->polyN >= 1 && c->polyN <= 7, "of_fb_polyexp: polyN must be in 1..7");
  FbPoly P{};
  P.n = c->polyN;
  for (int k = 0; k <= P.n; k++) {
    P.g[k] = c->g[k];
    P.xg[k] = c->xg[k];
    P.xxg[k] = c->xxg[k];
  }
  for (int k = 0; k < 4; k++) P.ig[k] = c->ig[k];
  if (P.n == 5 || P.n == 7) {  // the reference's polyN settings: the tiled kernel
    const int vec = (pitch % 4) == 0 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0;
    dim3 grid((W + FBQ_OW - 1) / FBQ_OW, (H + FBQ_R - 1) / FBQ_R);
    if (P.n == 7)
      fb_polyexp_tile_kernel<7, false><<<grid, 256, 0, as_stream(stream)>>>(src, dst, H, W, pitch, P, vec, 0.f, 0.f);
    else
      fb_polyexp_tile_kernel<5, false><<<grid, 256, 0, as_stream(stream)>>>(src, dst, H, W, pitch, P, vec, 0.f, 0.f);
    return check_launch("of_fb_polyexp");
  }
  dim3 grid((W + (FBP_T - 2 * P.n) - 1) / (FBP_T - 2 * P.n), H);
  fb_polyexp_kernel<<<grid, FBP_T, 0, as_stream(stream)>>>(src, dst, H, W, pitch, P);
  return check_launch("of_fb_polyexp");
}

extern "C" int of_fb_polyexp_blurred(const float* src, float* dst, int H, int W, int pitch, const float* gk,
                                     const of_fb_poly_consts* c, void* stream) {
  OF_REQUIRE(!bad_plane(src, H, W, pitch) && dst && c && gk, "of_fb_polyexp_blurred: bad plane");
  OF_REQUIRE(c->polyN == 5 || c->polyN == 7, "of_fb_polyexp_blurred: polyN must be 5 or 7");
  OF_REQUIRE(H >= 3 && W >= 3, "of_fb_polyexp_blurred: the frame must be at least 3 x 3");
  FbPoly P{};
  P.n = c->polyN;
  for (int k = 0; k <= P.n; k++) {
    P.g[k] = c->g[k];
    P.xg[k] = c->xg[k];
    P.xxg[k] = c->xxg[k];
  }
  for (int k = 0; k < 4; k++) P.ig[k] = c->ig[k];
  const int vec = (pitch % 4) == 0 && (reinterpret_cast<uintptr_t>(dst) & 15) == 0;
  dim3 grid((W + FBQ_OW - 1) / FBQ_OW, (H + FBQ_R - 1) / FBQ_R);
  if (P.n == 7)
    fb_polyexp_tile_kernel<7, true><<<grid, 256, 0, as_stream(stream)>>>(src, dst, H, W, pitch, P, vec, gk[0], gk[1]);
  else
    fb_polyexp_tile_kernel<5, true><<<grid, 256, 0, as_stream(stream)>>>(src, dst, H, W, pitch, P, vec, gk[0], gk[1]);
  return check_launch("of_fb_polyexp_blurred");
}

extern "C" int of_fb_update_matrices(const float* flowx, const float* flowy, const float* R0, const float* R1, float* M,
                                     int H, int W, int pitch, void* stream) {
  OF_REQUIRE(!bad_plane(flowx, H, W, pitch) && flowy && R0 && R1 && M, "of_fb_update_matrices: bad plane");
  dim3 blk(32, 8), grd((W + 31) / 32, (H + 7) / 8);
  fb_update_matrices_kernel<<<grd, blk, 0, as_stream(stream)>>>(flowx, flowy, R0, R1, M, H, W, pitch);
  return check_launch("of_fb_update_matrices");
}

extern "C" int of_fb_update_flow(const float* M, float* flowx, float* flowy, int H, int W, int pitch, void* stream) {
  OF_REQUIRE(!bad_plane(M, H, W, pitch) && flowx && flowy, "of_fb_update_flow: bad plane");
  dim3 blk(32, 8), grd((W + 31) / 32, (H + 7) / 8);
  fb_update_flow_kernel<<<grd, blk, 0, as_stream(stream)>>>(M, flowx, flowy, H, W, pitch);
  return check_launch("of_fb_update_flow");
}

extern "C" int of_fb_iteration(const float* M_in, float* M_out, const float* R0, const float* R1, float* flowx,
                               float* flowy, int H, int W, int pitch, const float* wk, int kh, int update_matrices,
                               void* stream) {
  OF_REQUIRE(!bad_plane(M_in, H, W, pitch) && R0 && R1 && flowx && flowy, "of_fb_iteration: bad plane");
  OF_REQUIRE(!update_matrices || (M_out && M_out != M_in), "of_fb_iteration: M_out missing or aliases M_in");
  OF_REQUIRE(wk && kh >= 0 && kh <= FB_MAXKH, "of_fb_iteration: bad kernel");
  // windowSize 33 (the reference default) on images with a single reflect-101 border and
  // TMA-compatible strides: the unrolled, TMA-staged kernel
  if (kh == 16 && H > 16 && W > 16 && (pitch % 4) == 0 && (reinterpret_cast<uintptr_t>(M_in) & 15) == 0) {
    constexpr int KH = 16;
    using G = FbkGeom<KH>;
    CUtensorMap tm;
    uint64_t dims[3] = {(uint64_t)W, (uint64_t)H, 5}, strides[2] = {(uint64_t)pitch * 4, (uint64_t)H * pitch * 4};
    uint32_t box[3] = {G::IW, G::IH, 1};
    int rc = tmap_f32(&tm, M_in, 3, dims, strides, box);
    if (rc) return rc;
    cudaError_t e = OF_SMEM_OPT_IN(fb_iter_fixed_kernel<KH>, G::SMEM);
    if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_fb_iteration: %s", cudaGetErrorString(e));
    dim3 grid((W + FBK_TW - 1) / FBK_TW, (H + FBK_TH - 1) / FBK_TH);
    fb_iter_fixed_kernel<KH><<<grid, 256, G::SMEM, as_stream(stream)>>>(tm, M_out, R0, R1, flowx, flowy, H, W, pitch,
                                                                        make_taps(wk, kh), update_matrices);
    return check_launch("of_fb_iteration");
  }
  size_t smem = sizeof(float) * ((size_t)(FBI_TH + 2 * kh) * (FBI_TW + 2 * kh) + (size_t)FBI_TH * (FBI_TW + 2 * kh));
  dim3 grid((W + FBI_TW - 1) / FBI_TW, (H + FBI_TH - 1) / FBI_TH);
  fb_iter_kernel<<<grid, 256, smem, as_stream(stream)>>>(M_in, M_out, R0, R1, flowx, flowy, H, W, pitch,
                                                         make_taps(wk, kh), kh, update_matrices);
  return check_launch("of_fb_iteration");
}
