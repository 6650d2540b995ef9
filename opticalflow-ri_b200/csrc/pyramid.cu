// Level-transition kernels of the pyramid driver (src/GenericPyramidalOpticalFlow.py).
//
//  A2 of_resize: Pillow's antialiased two-pass resample of a float32 image.  The
//     per-output-coordinate kernels (bounds + normalised double weights) are built on the
//     device by one thread per output coordinate with the same double operations as the
//     published algorithm; the horizontal pass writes a float32 intermediate, the vertical
//     pass reads it; both accumulate in double.  Bit-exact with Pillow.
//  A3 of_spline_upsample: not-a-knot cubic interpolant (the s=0 RectBivariateSpline),
//     separable: moments along y per coarse column, evaluation at the fine rows, moments
//     along x per fine row, evaluation at the fine columns; double throughout.
//  A4 of_warp_pair_bilinear: doBiLinearWarping's round-half-even base, float64 weights.
//  of_warp_liushen_*: the optical-flow-equation warp (biLinear=False): a last-writer-wins
//     integer scatter (atomicMax of the source's row-major position per destination, then
//     a gather) and the float32 optical-flow-equation correction.
#include <climits>

#include "common.cuh"

namespace ofb {

// ----------------------------------------------------------------------------- resize
__device__ __forceinline__ double filt(double x, int bicubic) {
  if (x < 0.0) x = -x;
  if (!bicubic) return x < 1.0 ? __dadd_rn(1.0, -x) : 0.0;
  const double a = -0.5;
  if (x < 1.0) return __dadd_rn(__dmul_rn(__dmul_rn(__dadd_rn(__dmul_rn(a + 2.0, x), -(a + 3.0)), x), x), 1.0);
  if (x < 2.0) {
    double t = __dmul_rn(__dadd_rn(x, -5.0), x);
    t = __dmul_rn(__dadd_rn(t, 8.0), x);
    return __dmul_rn(__dadd_rn(t, -4.0), a);
  }
  return 0.0;
}

__host__ __device__ inline void resize_geom(int inSize, int outSize, int bicubic, double* scale, double* fscale,
                                            double* support, int* ksize) {
  double s = (double)((float)inSize - 0.0f) / outSize;
  double fs = s < 1.0 ? 1.0 : s;
  double sup = (bicubic ? 2.0 : 1.0) * fs;
  *scale = s;
  *fscale = fs;
  *support = sup;
  *ksize = (int)ceil(sup) * 2 + 1;
}

// Weights and source window of output index xx along one axis: window [*pmin, *pmin + *pcnt),
// k[j * kstride] for j < ksize (zero past the window).
__device__ __forceinline__ void resize_coeff_at(int inSize, int outSize, int bicubic, int ksize, int xx, int* pmin,
                                                int* pcnt, double* k, int kstride) {
  double scale, fscale, support;
  int ks;
  resize_geom(inSize, outSize, bicubic, &scale, &fscale, &support, &ks);
  double center = __dadd_rn(0.0, __dmul_rn(__dadd_rn((double)xx, 0.5), scale));
  double ww = 0.0, ss = __ddiv_rn(1.0, fscale);
  int xmin = (int)__dadd_rn(__dadd_rn(center, -support), 0.5);
  if (xmin < 0) xmin = 0;
  int xmax = (int)__dadd_rn(__dadd_rn(center, support), 0.5);
  if (xmax > inSize) xmax = inSize;
  xmax -= xmin;
  int x;
  for (x = 0; x < xmax; x++) {
    double w = filt(__dmul_rn(__dadd_rn(__dadd_rn((double)(x + xmin), -center), 0.5), ss), bicubic);
    k[x * kstride] = w;
    ww = __dadd_rn(ww, w);
  }
  for (x = 0; x < xmax; x++)
    if (ww != 0.0) k[x * kstride] = __ddiv_rn(k[x * kstride], ww);
  for (; x < ksize; x++) k[x * kstride] = 0.0;
  *pmin = xmin;
  *pcnt = xmax;
}

// sum over j < n of (double)a(j) * w(j), accumulated in the order j = 0, 1, ... (Pillow's);
// the loads go in groups of 8 ahead of the group's adds, so a thread waits on one memory
// latency per 8 taps instead of one per tap.
template <class A, class Wt>
__device__ __forceinline__ double rz_dot(int n, const A& a, const Wt& w) {
  double ss = 0.0;
  int j = 0;
  for (; j + 8 <= n; j += 8) {
    float v[8];
    double k[8];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      v[q] = a(j + q);
      k[q] = w(j + q);
    }
#pragma unroll
    for (int q = 0; q < 8; q++) ss = __dadd_rn(ss, __dmul_rn((double)v[q], k[q]));
  }
  for (; j < n; j++) ss = __dadd_rn(ss, __dmul_rn((double)a(j), w(j)));
  return ss;
}

__global__ void resize_coeff_kernel(int inSize, int outSize, int bicubic, int ksize, int* bounds, double* kk) {
  int xx = blockIdx.x * blockDim.x + threadIdx.x;
  if (xx >= outSize) return;
  resize_coeff_at(inSize, outSize, bicubic, ksize, xx, &bounds[2 * xx], &bounds[2 * xx + 1], kk + (size_t)xx * ksize,
                  1);
}

// The same weights tap-major (kk[tap * outSize + xx]), the layout of the caller-kept tables:
// the outputs of a warp read consecutive words of one tap.
__global__ void resize_coeff_t_kernel(int inSize, int outSize, int bicubic, int ksize, int* bounds, double* kk) {
  int xx = blockIdx.x * blockDim.x + threadIdx.x;
  if (xx >= outSize) return;
  resize_coeff_at(inSize, outSize, bicubic, ksize, xx, &bounds[2 * xx], &bounds[2 * xx + 1], kk + xx, outSize);
}

// Horizontal pass from a tap-major table: a CTA takes 128 output columns of `rb` rows; per
// row it stages the source span those columns read into shared memory with coalesced loads
// (index i stored at i + i / 32, so outputs 8 samples apart, as at a downscale by 8, fall in
// distinct banks), then each thread sums its taps from there.  Same sums as resize_h_kernel.
__device__ __forceinline__ int rz_pad(int i) { return i + (i >> 5); }
__global__ void __launch_bounds__(128) resize_ht_kernel(const float* __restrict__ src, int sp, float* __restrict__ dst,
                                                        int dp, int Hs, int Wd, const int* __restrict__ bounds,
                                                        const double* __restrict__ kk, int rb) {
  extern __shared__ float seg[];
  const int xb = blockIdx.x * 128, xl = min(Wd, xb + 128) - 1;
  const int lo = bounds[2 * xb], n = bounds[2 * xl] + bounds[2 * xl + 1] - lo;  // window ends never decrease
  const int xx = xb + (int)threadIdx.x;
  const bool act = xx < Wd;
  const int xmin = act ? bounds[2 * xx] - lo : 0, cnt = act ? bounds[2 * xx + 1] : 0;
  const double* k = kk + xx;
  const int y1 = min(Hs, (int)(blockIdx.y + 1) * rb);
  for (int y = blockIdx.y * rb; y < y1; y++) {
    const float* row = src + (size_t)y * sp + lo;
    __syncthreads();  // the previous row's span is no longer read
    for (int i = threadIdx.x; i < n; i += 128) seg[rz_pad(i)] = row[i];
    __syncthreads();
    if (act) {
      const double ss = rz_dot(cnt, [&](int x) { return seg[rz_pad(xmin + x)]; },
                               [&](int x) { return k[(size_t)x * Wd]; });
      dst[(size_t)y * dp + xx] = (float)ss;
    }
  }
}

// The horizontal pass from a tap-major table with the source read from global memory (one
// row per CTA), for spans too long to stage.
__global__ void __launch_bounds__(128) resize_htg_kernel(const float* __restrict__ src, int sp, float* __restrict__ dst,
                                                         int dp, int Wd, const int* __restrict__ bounds,
                                                         const double* __restrict__ kk) {
  const int xx = blockIdx.x * 128 + threadIdx.x, y = blockIdx.y;
  if (xx >= Wd) return;
  const float* row = src + (size_t)y * sp + bounds[2 * xx];
  const double* k = kk + xx;
  const double ss = rz_dot(bounds[2 * xx + 1], [&](int x) { return row[x]; }, [&](int x) { return k[(size_t)x * Wd]; });
  dst[(size_t)y * dp + xx] = (float)ss;
}

// Vertical pass from a tap-major table: a thread sums its column for `rb` output rows
// (the row's weights are read by every thread at once).
__global__ void __launch_bounds__(128) resize_vt_kernel(const float* __restrict__ src, int sp, float* __restrict__ dst,
                                                        int dp, int Hd, int Wd, const int* __restrict__ bounds,
                                                        const double* __restrict__ kk, int rb) {
  const int x = blockIdx.x * 128 + threadIdx.x;
  if (x >= Wd) return;
  const int y1 = min(Hd, (int)(blockIdx.y + 1) * rb);
  for (int yy = blockIdx.y * rb; yy < y1; yy++) {
    const int ymin = bounds[2 * yy], ymax = bounds[2 * yy + 1];
    const float* col = src + (size_t)ymin * sp + x;
    const double ss = rz_dot(ymax, [&](int y) { return col[(size_t)y * sp]; },
                             [&](int y) { return kk[(size_t)y * Hd + yy]; });
    dst[(size_t)yy * dp + x] = (float)ss;
  }
}

// Fused passes for kernels of up to RZ_MAXK taps: a CTA computes the weights it needs into
// shared memory (the horizontal pass: its 128 output columns; the vertical pass: its
// `rb` output rows) and applies them to a band of rb <= RZ_RB rows, so a resize is two
// launches, not four.  Same weights and sums as the table path.  RZ_MAXK = 40 covers
// Pillow's bicubic support up to a factor of 9.5 (33 taps at 8x: 1024 -> 128) and its
// bilinear support up to 19x.  The band height is picked per launch (rz_band) so that
// small outputs still spread over the SMs.
constexpr int RZ_MAXK = 40, RZ_RB = 16;
__global__ void __launch_bounds__(128) resize_hf_kernel(const float* __restrict__ src, int sp, float* __restrict__ dst,
                                                        int dp, int Hs, int Ws, int Wd, int bicubic, int ksize,
                                                        int rb) {
  __shared__ double kk[RZ_MAXK * 128];
  const int xx = blockIdx.x * 128 + threadIdx.x;
  if (xx >= Wd) return;  // no barrier below: every thread uses only its own column's weights
  int xmin, xcnt;
  resize_coeff_at(Ws, Wd, bicubic, ksize, xx, &xmin, &xcnt, kk + threadIdx.x, 128);
  const double* k = kk + threadIdx.x;
  const int y1 = min(Hs, (blockIdx.y + 1) * rb);
  for (int y = blockIdx.y * rb; y < y1; y++) {
    const float* row = src + (size_t)y * sp + xmin;
    const double ss = rz_dot(xcnt, [&](int x) { return row[x]; }, [&](int x) { return k[x * 128]; });
    dst[(size_t)y * dp + xx] = (float)ss;
  }
}

__global__ void __launch_bounds__(128) resize_vf_kernel(const float* __restrict__ src, int sp, float* __restrict__ dst,
                                                        int dp, int Hs, int Hd, int Wd, int bicubic, int ksize,
                                                        int rb) {
  __shared__ double kk[RZ_RB * RZ_MAXK];
  __shared__ int bnd[RZ_RB][2];
  const int yy0 = blockIdx.y * rb;
  if (threadIdx.x < rb && yy0 + threadIdx.x < Hd)
    resize_coeff_at(Hs, Hd, bicubic, ksize, yy0 + threadIdx.x, &bnd[threadIdx.x][0], &bnd[threadIdx.x][1],
                    kk + threadIdx.x * RZ_MAXK, 1);
  __syncthreads();
  const int x = blockIdx.x * 128 + threadIdx.x;
  if (x >= Wd) return;
  const int n = min(rb, Hd - yy0);
  for (int r = 0; r < n; r++) {
    const int ymin = bnd[r][0], ymax = bnd[r][1];
    const double* k = kk + r * RZ_MAXK;
    const float* col = src + (size_t)ymin * sp + x;
    const double ss = rz_dot(ymax, [&](int y) { return col[(size_t)y * sp]; }, [&](int y) { return k[y]; });
    dst[(size_t)(yy0 + r) * dp + x] = (float)ss;
  }
}

// Rows per CTA of a fused pass: RZ_RB, halved while the grid would cover fewer than two
// CTAs per SM of a 148-SM part (a 128 x 128 output has one column block).
static int rz_band(int col_blocks, int rows) {
  int rb = RZ_RB;
  while (rb > 1 && (long long)col_blocks * ((rows + rb - 1) / rb) < 2 * 148) rb >>= 1;
  return rb;
}

__global__ void resize_h_kernel(const float* __restrict__ src, int sp, float* __restrict__ dst, int dp, int Hs, int Wd,
                                const int* __restrict__ bounds, const double* __restrict__ kk, int ksize) {
  int xx = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (xx >= Wd) return;
  int xmin = bounds[2 * xx], xmax = bounds[2 * xx + 1];
  const double* k = kk + (size_t)xx * ksize;
  const float* row = src + (size_t)y * sp + xmin;
  const double ss = rz_dot(xmax, [&](int x) { return row[x]; }, [&](int x) { return k[x]; });
  dst[(size_t)y * dp + xx] = (float)ss;
}

__global__ void resize_v_kernel(const float* __restrict__ src, int sp, float* __restrict__ dst, int dp, int Wd,
                                const int* __restrict__ bounds, const double* __restrict__ kk, int ksize) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, yy = blockIdx.y;
  if (x >= Wd) return;
  int ymin = bounds[2 * yy], ymax = bounds[2 * yy + 1];
  const double* k = kk + (size_t)yy * ksize;
  const float* col = src + (size_t)ymin * sp + x;
  const double ss = rz_dot(ymax, [&](int y) { return col[(size_t)y * sp]; }, [&](int y) { return k[y]; });
  dst[(size_t)yy * dp + x] = (float)ss;
}

__global__ void copy_plane_kernel(const float* __restrict__ src, int sp, float* __restrict__ dst, int dp, int W) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x < W) dst[(size_t)y * dp + x] = src[(size_t)y * sp + x];
}

static int ksize_of(int in, int out, int bicubic) {
  double a, b, c;
  int k;
  resize_geom(in, out, bicubic, &a, &b, &c, &k);
  return k;
}

// ----------------------------------------------------------------------------- spline
// Reciprocal pivots of the constant (1, 4, 1) tridiagonal elimination, shared by every
// line: c[0] = 1/4, c[r] = 1/(4 - c[r-1]) until the fixed point (2 - sqrt 3) repeats in
// double.  One thread runs the short division chain (about 20 steps); the block fills the
// constant tail.
__global__ void spline_recip_kernel(double* c, int m) {
  __shared__ double tail;
  __shared__ int rc;
  if (threadIdx.x == 0) {
    int r = 0;
    double v = 0.0;
    if (m > 0) {
      v = __ddiv_rn(1.0, 4.0);
      c[0] = v;
      for (r = 1; r < m; r++) {
        double nv = __ddiv_rn(1.0, __dadd_rn(4.0, -v));
        c[r] = nv;
        if (nv == v) break;
        v = nv;
      }
    }
    tail = v;
    rc = r;
  }
  __syncthreads();
  for (int r = rc + 1 + threadIdx.x; r < m; r += blockDim.x) c[r] = tail;
}

// Thomas-algorithm moments of the not-a-knot spline through n >= 4 samples with unit
// spacing; sample i of a line is y[i*ys] (float or double), moment and scratch i are
// M[i*ls] and dp[i*ls] (double).  The elimination multiplies by the shared pivots, so a
// step is one add and one multiply.
//
// Each line is one thread and the recurrence is serial, with few lines in flight (one warp
// per scheduler), so every instruction on a line's thread costs close to its full latency.
// The work of a step that does not depend on the previous step -- its right-hand side
// 6 (y[r+3] - 2 y[r+2] + y[r+1]), with the end corrections of the first and last step --
// is done first by a fully parallel kernel (nak_rhs, one thread per line and step) into
// the scratch array; the serial kernel (nak_solve) then reads it back a chunk ahead and
// does only the add, the multiply and the store of each step, overwriting the right-hand
// side with the eliminated value.  The arithmetic is the same, in the same order.
#define NAK_CH 32
#define NAK_SPIV 4096  // pivots staged in shared memory (32 KB)
template <typename TY>
__device__ __forceinline__ double nak_m1(const TY* __restrict__ y, size_t ys) {
  return __dadd_rn(__dadd_rn((double)y[2 * ys], -__dmul_rn(2.0, (double)y[ys])), (double)y[0]);
}
template <typename TY>
__device__ __forceinline__ double nak_ml(const TY* __restrict__ y, size_t ys, int n) {
  return __dadd_rn(__dadd_rn((double)y[(size_t)(n - 1) * ys], -__dmul_rn(2.0, (double)y[(size_t)(n - 2) * ys])),
                   (double)y[(size_t)(n - 3) * ys]);
}
// right-hand side of step r (0 <= r < m = n - 4) of one line into dp[r*ls]
template <typename TY>
__device__ __forceinline__ void nak_rhs(const TY* __restrict__ y, size_t ys, double* __restrict__ dp, size_t ls,
                                        int r, int n) {
  const int m = n - 4;
  const double yp = (double)y[(size_t)(r + 3) * ys], y0 = (double)y[(size_t)(r + 2) * ys];
  const double ym = (double)y[(size_t)(r + 1) * ys];
  double v = __dmul_rn(6.0, __dadd_rn(__dadd_rn(yp, -__dmul_rn(2.0, y0)), ym));
  if (r == 0) v = __dadd_rn(v, -nak_m1<TY>(y, ys));
  if (r == m - 1) v = __dadd_rn(v, -nak_ml<TY>(y, ys, n));
  dp[(size_t)r * ls] = v;
}
template <typename TY>
__device__ void nak_solve(const TY* __restrict__ y, size_t ys, size_t ls, double* __restrict__ M,
                          const double* __restrict__ cp, const double* sp, int nsp, double* __restrict__ dp, int n) {
#define MV(i) M[(size_t)(i) * ls]
#define PIV(r) ((r) < nsp ? sp[r] : cp[r])
  const double M1 = nak_m1<TY>(y, ys), Ml = nak_ml<TY>(y, ys, n);
  MV(1) = M1;
  MV(n - 2) = Ml;
  double M2 = Ml, M3 = Ml;  // M[2], M[n-3] for the end conditions
  const int m = n - 4;
  if (m > 0) {
    double dprev = 0.0;
    double rb[NAK_CH];
#pragma unroll
    for (int j = 0; j < NAK_CH; j++) rb[j] = j < m ? dp[(size_t)j * ls] : 0.0;
#pragma unroll 1
    for (int r0 = 0; r0 < m; r0 += NAK_CH) {
      double rn[NAK_CH], cb[NAK_CH];
#pragma unroll
      for (int j = 0; j < NAK_CH; j++) {
        const int r = r0 + NAK_CH + j;
        rn[j] = r < m ? dp[(size_t)r * ls] : 0.0;  // the next chunk, in flight during this one
        cb[j] = r0 + j < m ? PIV(r0 + j) : 0.0;
      }
      if (r0 + NAK_CH <= m) {  // a whole chunk: the chain alone
#pragma unroll
        for (int j = 0; j < NAK_CH; j++) {
          const double d = (r0 + j == 0) ? __dmul_rn(rb[j], cb[j]) : __dmul_rn(__dadd_rn(rb[j], -dprev), cb[j]);
          dp[(size_t)(r0 + j) * ls] = d;
          dprev = d;
        }
      } else {
#pragma unroll
        for (int j = 0; j < NAK_CH; j++) {
          if (r0 + j < m) {
            const double d = (r0 + j == 0) ? __dmul_rn(rb[j], cb[j]) : __dmul_rn(__dadd_rn(rb[j], -dprev), cb[j]);
            dp[(size_t)(r0 + j) * ls] = d;
            dprev = d;
          }
        }
      }
#pragma unroll
      for (int j = 0; j < NAK_CH; j++) rb[j] = rn[j];
    }
    double next = dprev;
    MV(m + 1) = next;
    M3 = next;  // M[n-3] = M[m+1]
    // back substitution, r = m-2 .. 0, in chunks loaded one ahead
    double db[NAK_CH];
#pragma unroll
    for (int j = 0; j < NAK_CH; j++) db[j] = m - 2 - j >= 0 ? dp[(size_t)(m - 2 - j) * ls] : 0.0;
#pragma unroll 1
    for (int r1 = m - 2; r1 >= 0; r1 -= NAK_CH) {
      double dn[NAK_CH], cb[NAK_CH];
#pragma unroll
      for (int j = 0; j < NAK_CH; j++) {
        const int r = r1 - NAK_CH - j;
        dn[j] = r >= 0 ? dp[(size_t)r * ls] : 0.0;
        cb[j] = r1 - j >= 0 ? PIV(r1 - j) : 0.0;
      }
      if (r1 - NAK_CH + 1 >= 0) {
#pragma unroll
        for (int j = 0; j < NAK_CH; j++) {
          next = __dadd_rn(db[j], -__dmul_rn(cb[j], next));
          MV(r1 - j + 2) = next;
        }
      } else {
#pragma unroll
        for (int j = 0; j < NAK_CH; j++) {
          if (r1 - j >= 0) {
            next = __dadd_rn(db[j], -__dmul_rn(cb[j], next));
            MV(r1 - j + 2) = next;
          }
        }
      }
#pragma unroll
      for (int j = 0; j < NAK_CH; j++) db[j] = dn[j];
    }
    M2 = next;  // M[2]
  } else {
    M2 = Ml;  // n == 4: M[2] = M[n-2], M[n-3] = M[1]
    M3 = M1;
  }
  MV(0) = __dadd_rn(__dmul_rn(2.0, M1), -M2);
  MV(n - 1) = __dadd_rn(__dmul_rn(2.0, Ml), -M3);
#undef PIV
#undef MV
}

// The first min(m, NAK_SPIV) pivots into shared memory (before any thread leaves).
__device__ __forceinline__ int nak_stage_pivots(double* sp, const double* __restrict__ cp, int m) {
  const int nsp = m < NAK_SPIV ? (m > 0 ? m : 0) : NAK_SPIV;
  for (int i = threadIdx.x; i < nsp; i += blockDim.x) sp[i] = cp[i];
  __syncthreads();
  return nsp;
}

__device__ __forceinline__ double nak_eval(double yi, double yi1, double Mi, double Mi1, double t) {
  double u = __dadd_rn(1.0, -t);
  double a = __dadd_rn(__dmul_rn(u, yi), __dmul_rn(t, yi1));
  double cu = __dadd_rn(__dmul_rn(__dmul_rn(u, u), u), -u);
  double ct = __dadd_rn(__dmul_rn(__dmul_rn(t, t), t), -t);
  double b = __dadd_rn(__dmul_rn(cu, Mi), __dmul_rn(ct, Mi1));
  return __dadd_rn(a, __ddiv_rn(b, 6.0));
}

__device__ __forceinline__ void fine_index(int j, int N, int n, int* i, double* t) {
  double s = __dmul_rn(__ddiv_rn((double)j, (double)N), (double)n);
  if (s < 0.0) s = 0.0;
  if (s > n - 1) s = n - 1;
  int k = (int)floor(s);
  if (k > n - 2) k = n - 2;
  *i = k;
  *t = __dadd_rn(s, -(double)k);
}

// One or two planes (blockIdx of the plane dimension) upsampled by the same launches; plane
// p's workspace arrays sit `pstride` doubles after plane 0's, and both use plane 0's pivots.
struct SplinePlanes {
  const float* src[2];
  float* dst[2];
  float scale[2];
  size_t pstride;
};

// right-hand sides along y: one thread per coarse column x and step r (grid.y = steps,
// grid.z = plane)
__global__ void __launch_bounds__(128) spline_ry_kernel(SplinePlanes P, int sp, int h, int w, double* S) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y, q = blockIdx.z;
  if (x >= w) return;
  nak_rhs<float>((q ? P.src[1] : P.src[0]) + x, (size_t)sp, S + q * P.pstride + x, (size_t)w, r, h);
}

// moments along y for each coarse column x, read straight from the float field (pitch sp)
__global__ void __launch_bounds__(128) spline_my_kernel(SplinePlanes P, int sp, int h, int w, double* M, double* S,
                                                        const double* __restrict__ cp) {
  extern __shared__ double s_piv[];
  const int nsp = nak_stage_pivots(s_piv, cp, h - 4);
  int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= w) return;
  const int q = blockIdx.y;
  // moments and scratch are laid out [i][x] with stride w
  nak_solve<float>((q ? P.src[1] : P.src[0]) + x, (size_t)sp, (size_t)w, M + q * P.pstride + x, cp, s_piv, nsp,
                   S + q * P.pstride + x, h);
}

// Tt[x][Y] = column spline of coarse column x at fine row Y.  A 32x32 tile goes through
// shared memory so the reads (along x) and the transposed writes (along Y) both coalesce.
__global__ void __launch_bounds__(256) spline_ey_kernel(SplinePlanes P, int sp, const double* __restrict__ M,
                                                        double* __restrict__ Tt, int h, int w, int H) {
  __shared__ double tile[32][33];
  const float* __restrict__ src = blockIdx.z ? P.src[1] : P.src[0];
  M += blockIdx.z * P.pstride;
  Tt += blockIdx.z * P.pstride;
  int x0 = blockIdx.x * 32, Y0 = blockIdx.y * 32;
  int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int k = ty; k < 32; k += 8) {
    int Y = Y0 + k, x = x0 + tx;
    if (Y < H && x < w) {
      int i;
      double t;
      fine_index(Y, H, h, &i, &t);
      tile[k][tx] = nak_eval((double)src[(size_t)i * sp + x], (double)src[(size_t)(i + 1) * sp + x],
                             M[(size_t)i * w + x], M[(size_t)(i + 1) * w + x], t);
    }
  }
  __syncthreads();
  for (int k = ty; k < 32; k += 8) {
    int x = x0 + k, Y = Y0 + tx;
    if (x < w && Y < H) Tt[(size_t)x * H + Y] = tile[tx][k];
  }
}

// moments along x for each fine row Y of Tt (layout [k][Y], stride H)
// right-hand sides along x for each fine row Y: one thread per Y and step r
__global__ void __launch_bounds__(128) spline_rx_kernel(const double* __restrict__ Tt, int w, int H, double* dp,
                                                        size_t pstride) {
  const int Y = blockIdx.x * blockDim.x + threadIdx.x, r = blockIdx.y;
  if (Y >= H) return;
  const size_t o = blockIdx.z * pstride;
  nak_rhs<double>(Tt + o + Y, (size_t)H, dp + o + Y, (size_t)H, r, w);
}

__global__ void __launch_bounds__(128) spline_mx_kernel(const double* __restrict__ Tt, int w, int H, double* M,
                                                        const double* __restrict__ cp, double* dp, size_t pstride) {
  extern __shared__ double s_piv[];
  const int nsp = nak_stage_pivots(s_piv, cp, w - 4);
  int Y = blockIdx.x * blockDim.x + threadIdx.x;
  if (Y >= H) return;
  const size_t o = blockIdx.y * pstride;
  nak_solve<double>(Tt + o + Y, (size_t)H, (size_t)H, M + o + Y, cp, s_piv, nsp, dp + o + Y, w);
}

// dst[Y][X] = row spline of fine row Y at fine column X (times scale).  The coarse
// samples and moments a 32x32 output tile needs (columns i..i+1 of Tt/M for each X, all
// along Y) are staged through shared memory with loads that coalesce along Y.
#define EX_SPAN 40
__global__ void __launch_bounds__(256) spline_ex_kernel(const double* __restrict__ Tt, const double* __restrict__ M,
                                                        SplinePlanes P, int dpitch, int w, int H, int W) {
  __shared__ double sT[EX_SPAN][33], sM[EX_SPAN][33];
  Tt += blockIdx.z * P.pstride;
  M += blockIdx.z * P.pstride;
  float* __restrict__ dst = blockIdx.z ? P.dst[1] : P.dst[0];
  const float scale = blockIdx.z ? P.scale[1] : P.scale[0];
  int X0 = blockIdx.x * 32, Y0 = blockIdx.y * 32;
  int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  int Xl = min(X0 + 31, W - 1);
  int ilo, ihi;
  double tt;
  fine_index(X0, W, w, &ilo, &tt);
  fine_index(Xl, W, w, &ihi, &tt);
  ihi += 1;  // the interval's right sample
  bool staged = ihi - ilo + 1 <= EX_SPAN;  // false only for strong downsampling
  if (staged) {
    for (int k = ty; k <= ihi - ilo; k += 8) {
      int Y = Y0 + tx;
      if (Y < H) {
        sT[k][tx] = Tt[(size_t)(ilo + k) * H + Y];
        sM[k][tx] = M[(size_t)(ilo + k) * H + Y];
      }
    }
  }
  __syncthreads();
  int X = X0 + tx;
  if (X >= W) return;
  int i;
  double t;
  fine_index(X, W, w, &i, &t);
  for (int k = ty; k < 32; k += 8) {
    int Y = Y0 + k;
    if (Y >= H) break;
    double v;
    if (staged) {
      v = nak_eval(sT[i - ilo][k], sT[i - ilo + 1][k], sM[i - ilo][k], sM[i - ilo + 1][k], t);
    } else {
      v = nak_eval(Tt[(size_t)i * H + Y], Tt[(size_t)(i + 1) * H + Y], M[(size_t)i * H + Y],
                   M[(size_t)(i + 1) * H + Y], t);
    }
    dst[(size_t)Y * dpitch + X] = __fmul_rn((float)v, scale);
  }
}

// ----------------------------------------------------------------------------- Liu-Shen warp
__global__ void lsw_init_kernel(int* owner, int n, int* bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) owner[i] = -1;
  if (i < 2) bad[i] = INT_MAX;
}

// numpy: usSwap = int32(xsMesh + floor(usNew + 0.5)) (float32 add and floor, exact
// integer sum); dUsNew = usNew - floor(usNew + float32(0.5)).
__global__ void lsw_owner_kernel(const float* __restrict__ u, const float* __restrict__ v, int H, int W, int pitch,
                                 int* __restrict__ owner, float* __restrict__ du, float* __restrict__ dv,
                                 int* __restrict__ bad) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  size_t i = (size_t)y * pitch + x;
  const float fu = floorf(__fadd_rn(u[i], 0.5f)), fv = floorf(__fadd_rn(v[i], 0.5f));
  du[i] = __fsub_rn(u[i], fu);
  dv[i] = __fsub_rn(v[i], fv);
  const int p = y * W + x;
  // destinations beyond +-2^30 (or non-finite shifts) are out of range for any image
  const bool okv = fv > -1073741824.0f && fv < 1073741824.0f, oku = fu > -1073741824.0f && fu < 1073741824.0f;
  const int ty = okv ? y + (int)fv : INT_MIN, tx = oku ? x + (int)fu : INT_MIN;
  const bool inv = okv && ty >= -H && ty < H, inu = oku && tx >= -W && tx < W;
  if (!inv) atomicMin(&bad[0], p);
  if (!inu) atomicMin(&bad[1], p);
  if (inv && inu) atomicMax(&owner[(ty < 0 ? ty + H : ty) * W + (tx < 0 ? tx + W : tx)], p);
}

__global__ void lsw_gather_kernel(const float* __restrict__ I, const int* __restrict__ owner, float* __restrict__ out,
                                  int H, int W, int pitch) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const int o = owner[y * W + x];
  out[(size_t)y * pitch + x] = o >= 0 ? I[(size_t)(o / W) * pitch + (o % W)] : I[(size_t)y * pitch + x];
}

__global__ void lsw_ofe_kernel(const float* __restrict__ I, const float* __restrict__ du, const float* __restrict__ dv,
                               float* __restrict__ out, int H, int W, int pitch) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  size_t i = (size_t)y * pitch + x;
  if (y == H - 1 || x == W - 1) {
    out[i] = I[i];
    return;
  }
  const float c = __fmul_rn(I[i], du[i]), cy = __fmul_rn(I[i], dv[i]);
  const float tdx = __fsub_rn(__fmul_rn(I[i + 1], du[i + 1]), c);
  const float tdy = __fsub_rn(__fmul_rn(I[i + pitch], dv[i + pitch]), cy);
  out[i] = __fsub_rn(I[i], __fadd_rn(tdx, tdy));
}

// ----------------------------------------------------------------------------- warp
__device__ __forceinline__ float warp_sample(const float* __restrict__ img, int H, int W, int pitch, float cy,
                                             float cx) {
  int iy = (int)rintf(cy), ix = (int)rintf(cx);
  double dy = __dadd_rn((double)cy, -(double)iy), dx = __dadd_rn((double)cx, -(double)ix);
  int ny = dy < 0 ? iy - 1 : iy + 1, nx = dx < 0 ? ix - 1 : ix + 1;
  dy = fabs(dy);
  dx = fabs(dx);
  iy = clampi(iy, 0, H - 1);
  ny = clampi(ny, 0, H - 1);
  ix = clampi(ix, 0, W - 1);
  nx = clampi(nx, 0, W - 1);
  double oy = __dadd_rn(1.0, -dy), ox = __dadd_rn(1.0, -dx);
  double a = __dmul_rn(__dmul_rn(oy, ox), (double)img[(size_t)iy * pitch + ix]);
  a = __dadd_rn(a, __dmul_rn(__dmul_rn(oy, dx), (double)img[(size_t)iy * pitch + nx]));
  a = __dadd_rn(a, __dmul_rn(__dmul_rn(dy, ox), (double)img[(size_t)ny * pitch + ix]));
  a = __dadd_rn(a, __dmul_rn(__dmul_rn(dy, dx), (double)img[(size_t)ny * pitch + nx]));
  return (float)a;
}

__global__ void warp_pair_kernel(const float* __restrict__ I0, const float* __restrict__ I1,
                                 const float* __restrict__ U, const float* __restrict__ V, float* __restrict__ O0,
                                 float* __restrict__ O1, int H, int W, int pitch) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  size_t i = (size_t)y * pitch + x;
  float hv = __fdiv_rn(V[i], 2.0f), hu = __fdiv_rn(U[i], 2.0f);
  float cy0 = (float)__dadd_rn((double)y, -(double)hv), cx0 = (float)__dadd_rn((double)x, -(double)hu);
  float cy1 = (float)__dadd_rn((double)y, (double)hv), cx1 = (float)__dadd_rn((double)x, (double)hu);
  O0[i] = warp_sample(I0, H, W, pitch, cy0, cx0);
  O1[i] = warp_sample(I1, H, W, pitch, cy1, cx1);
}

__global__ void warp_coords_kernel(const float* __restrict__ img, const float* __restrict__ cy,
                                   const float* __restrict__ cx, float* __restrict__ out, int H, int W, int pitch) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  size_t i = (size_t)y * pitch + x;
  out[i] = warp_sample(img, H, W, pitch, cy[i], cx[i]);
}

}  // namespace ofb

using namespace ofb;

extern "C" int of_warp_bilinear_coords(const float* img, const float* coordsY, const float* coordsX, float* out, int H,
                                       int W, int pitch, void* stream) {
  OF_REQUIRE(!bad_plane(img, H, W, pitch) && coordsY && coordsX && out, "of_warp_bilinear_coords: bad plane");
  warp_coords_kernel<<<dim3((W + 255) / 256, H), 256, 0, as_stream(stream)>>>(img, coordsY, coordsX, out, H, W, pitch);
  return check_launch("of_warp_bilinear_coords");
}

extern "C" size_t of_resize_workspace_size(int Hs, int Ws, int Hd, int Wd, int filter) {
  Sizer s;
  int bic = filter == OF_FILTER_BICUBIC;
  s.take<int>(2 * (size_t)(Wd > 0 ? Wd : 1));
  s.take<double>((size_t)ksize_of(Ws, Wd > 0 ? Wd : 1, bic) * (Wd > 0 ? Wd : 1));
  s.take<int>(2 * (size_t)(Hd > 0 ? Hd : 1));
  s.take<double>((size_t)ksize_of(Hs, Hd > 0 ? Hd : 1, bic) * (Hd > 0 ? Hd : 1));
  s.take<float>((size_t)Hs * (Wd > 0 ? Wd : 1));
  return s.off;
}

extern "C" int of_resize(const float* src, int Hs, int Ws, int src_pitch, float* dst, int Hd, int Wd, int dst_pitch,
                         int filter, void* workspace, size_t workspace_bytes, void* stream) {
  OF_REQUIRE(!bad_plane(src, Hs, Ws, src_pitch) && !bad_plane(dst, Hd, Wd, dst_pitch), "of_resize: bad plane");
  OF_REQUIRE(filter == OF_FILTER_BILINEAR || filter == OF_FILTER_BICUBIC, "of_resize: unknown filter");
  cudaStream_t st = as_stream(stream);
  if (Hs == Hd && Ws == Wd) {
    copy_plane_kernel<<<dim3((Wd + 255) / 256, Hd), 256, 0, st>>>(src, src_pitch, dst, dst_pitch, Wd);
    return check_launch("of_resize");
  }
  size_t need = of_resize_workspace_size(Hs, Ws, Hd, Wd, filter);
  if (!workspace || workspace_bytes < need)
    return set_error(OF_ERR_WORKSPACE, "of_resize: workspace too small (%zu < %zu)", workspace_bytes, need);
  int bic = filter == OF_FILTER_BICUBIC;
  int kh = ksize_of(Ws, Wd, bic), kv = ksize_of(Hs, Hd, bic);
  Carver c(workspace, workspace_bytes);
  int* bh = c.take<int>(2 * (size_t)Wd);
  double* kkh = c.take<double>((size_t)kh * Wd);
  int* bv = c.take<int>(2 * (size_t)Hd);
  double* kkv = c.take<double>((size_t)kv * Hd);
  float* tmp = c.take<float>((size_t)Hs * Wd);
  bool need_h = Wd != Ws, need_v = Hd != Hs;
  if (kh <= RZ_MAXK && kv <= RZ_MAXK) {  // the fused passes
    float* mid = need_v ? tmp : dst;
    const int mp = need_v ? Wd : dst_pitch;
    const int cb = (Wd + 127) / 128;
    if (need_h) {
      const int rb = rz_band(cb, Hs);
      resize_hf_kernel<<<dim3(cb, (Hs + rb - 1) / rb), 128, 0, st>>>(src, src_pitch, mid, mp, Hs, Ws, Wd, bic, kh, rb);
    }
    if (need_v) {
      const int rb = rz_band(cb, Hd);
      resize_vf_kernel<<<dim3(cb, (Hd + rb - 1) / rb), 128, 0, st>>>(need_h ? tmp : src, need_h ? Wd : src_pitch, dst,
                                                                     dst_pitch, Hs, Hd, Wd, bic, kv, rb);
    }
    return check_launch("of_resize", (int)need_h + (int)need_v);
  }
  const float* cur = src;
  int cur_pitch = src_pitch;
  if (need_h) {
    resize_coeff_kernel<<<(Wd + 127) / 128, 128, 0, st>>>(Ws, Wd, bic, kh, bh, kkh);
    float* out = need_v ? tmp : dst;
    int op = need_v ? Wd : dst_pitch;
    resize_h_kernel<<<dim3((Wd + 127) / 128, Hs), 128, 0, st>>>(src, src_pitch, out, op, Hs, Wd, bh, kkh, kh);
    cur = out;
    cur_pitch = op;
  }
  if (need_v) {
    resize_coeff_kernel<<<(Hd + 127) / 128, 128, 0, st>>>(Hs, Hd, bic, kv, bv, kkv);
    resize_v_kernel<<<dim3((Wd + 127) / 128, Hd), 128, 0, st>>>(cur, cur_pitch, dst, dst_pitch, Wd, bv, kkv, kv);
  }
  return check_launch("of_resize", 2 * (int)need_h + 2 * (int)need_v);
}

// Weight tables of one axis, computed once and kept by the caller (a downscale by 8 has 33
// bicubic taps per output, whose weights cost more than the resize's sums when every CTA of
// a fused pass recomputes them).  Layout: int bounds[2 * out], then (256-byte aligned)
// double weights[out][ksize], as the table path of of_resize builds them.
extern "C" size_t of_resize_table_size(int in, int out, int filter) {
  if (in <= 0 || out <= 0) return 0;
  Sizer s;
  s.take<int>(2 * (size_t)out);
  s.take<double>((size_t)ksize_of(in, out, filter == OF_FILTER_BICUBIC) * out);
  return s.off;
}

extern "C" int of_resize_table(int in, int out, int filter, void* table, size_t table_bytes, void* stream) {
  OF_REQUIRE(in > 0 && out > 0 && table, "of_resize_table: bad arguments");
  OF_REQUIRE(filter == OF_FILTER_BILINEAR || filter == OF_FILTER_BICUBIC, "of_resize_table: unknown filter");
  const size_t need = of_resize_table_size(in, out, filter);
  if (table_bytes < need)
    return set_error(OF_ERR_WORKSPACE, "of_resize_table: table too small (%zu < %zu)", table_bytes, need);
  const int bic = filter == OF_FILTER_BICUBIC, k = ksize_of(in, out, bic);
  Carver c(table, table_bytes);
  int* b = c.take<int>(2 * (size_t)out);
  double* kk = c.take<double>((size_t)k * out);
  resize_coeff_t_kernel<<<(out + 127) / 128, 128, 0, as_stream(stream)>>>(in, out, bic, k, b, kk);
  return check_launch("of_resize_table");
}

extern "C" int of_resize_tabled(const float* src, int Hs, int Ws, int src_pitch, float* dst, int Hd, int Wd,
                                int dst_pitch, int filter, const void* table_h, const void* table_v, void* workspace,
                                size_t workspace_bytes, void* stream) {
  OF_REQUIRE(!bad_plane(src, Hs, Ws, src_pitch) && !bad_plane(dst, Hd, Wd, dst_pitch), "of_resize_tabled: bad plane");
  OF_REQUIRE(filter == OF_FILTER_BILINEAR || filter == OF_FILTER_BICUBIC, "of_resize_tabled: unknown filter");
  cudaStream_t st = as_stream(stream);
  if (Hs == Hd && Ws == Wd) {
    copy_plane_kernel<<<dim3((Wd + 255) / 256, Hd), 256, 0, st>>>(src, src_pitch, dst, dst_pitch, Wd);
    return check_launch("of_resize_tabled");
  }
  const bool need_h = Wd != Ws, need_v = Hd != Hs;
  OF_REQUIRE((!need_h || table_h) && (!need_v || table_v), "of_resize_tabled: missing weight table");
  const int bic = filter == OF_FILTER_BICUBIC;
  const int kh = need_h ? ksize_of(Ws, Wd, bic) : 0, kv = need_v ? ksize_of(Hs, Hd, bic) : 0;
  float* tmp = nullptr;
  if (need_h && need_v) {
    if (!workspace || workspace_bytes < (size_t)Hs * Wd * sizeof(float))
      return set_error(OF_ERR_WORKSPACE, "of_resize_tabled: workspace too small (%zu < %zu)", workspace_bytes,
                       (size_t)Hs * Wd * sizeof(float));
    tmp = static_cast<float*>(workspace);
  }
  const float* cur = src;
  int cur_pitch = src_pitch;
  if (need_h) {
    Carver c(const_cast<void*>(table_h), of_resize_table_size(Ws, Wd, filter));
    const int* bh = c.take<int>(2 * (size_t)Wd);
    const double* kkh = c.take<double>((size_t)kh * Wd);
    float* out = need_v ? tmp : dst;
    const int op = need_v ? Wd : dst_pitch;
    // a CTA's source span: its 128 columns' windows (at most 128 input steps plus one window)
    const long long span = (long long)ceil(128.0 * Ws / Wd) + kh + 2;
    const int cb = (Wd + 127) / 128;
    if (span <= 8192) {
      const size_t smem = sizeof(float) * (size_t)(span + (span >> 5) + 1);
      const int rb = rz_band(cb, Hs);
      resize_ht_kernel<<<dim3(cb, (Hs + rb - 1) / rb), 128, smem, st>>>(src, src_pitch, out, op, Hs, Wd, bh, kkh, rb);
    } else {  // very strong downscales: the span does not fit a CTA's default shared memory
      resize_htg_kernel<<<dim3(cb, Hs), 128, 0, st>>>(src, src_pitch, out, op, Wd, bh, kkh);
    }
    cur = out;
    cur_pitch = op;
  }
  if (need_v) {
    Carver c(const_cast<void*>(table_v), of_resize_table_size(Hs, Hd, filter));
    const int* bv = c.take<int>(2 * (size_t)Hd);
    const double* kkv = c.take<double>((size_t)kv * Hd);
    const int cb = (Wd + 127) / 128, rb = rz_band(cb, Hd);
    resize_vt_kernel<<<dim3(cb, (Hd + rb - 1) / rb), 128, 0, st>>>(cur, cur_pitch, dst, dst_pitch, Hd, Wd, bv, kkv, rb);
  }
  return check_launch("of_resize_tabled", (int)need_h + (int)need_v);
}

extern "C" size_t of_spline_workspace_size(int h, int w, int H, int W) {
  Sizer s;
  size_t a = (size_t)h * w, b = (size_t)H * w;
  s.take<double>(a);      // moments along y
  s.take<double>(a);      // Thomas scratch along y
  s.take<double>((size_t)(h > w ? h : w));  // shared reciprocal pivots
  s.take<double>(b);      // column splines at the fine rows, layout [x][Y]
  s.take<double>(b);      // moments along x
  s.take<double>(b);      // Thomas scratch along x
  (void)W;
  return s.off;
}

static int spline_run(const SplinePlanes& P0, int np, int h, int w, int src_pitch, int H, int W, int dst_pitch,
                      void* workspace, size_t single, cudaStream_t st) {
  size_t a = (size_t)h * w, b = (size_t)H * w;
  Carver c(workspace, single);
  double* My = c.take<double>(a);
  double* Sy = c.take<double>(a);
  double* piv = c.take<double>((size_t)(h > w ? h : w));
  double* Tt = c.take<double>(b);
  double* Mx = c.take<double>(b);
  double* Sx = c.take<double>(b);
  SplinePlanes P = P0;
  P.pstride = single / sizeof(double);
  spline_recip_kernel<<<1, 256, 0, st>>>(piv, (h > w ? h : w) - 4);
  auto piv_smem = [](int m) { return sizeof(double) * (size_t)(m < NAK_SPIV ? (m > 0 ? m : 0) : NAK_SPIV); };
  if (h > 4) spline_ry_kernel<<<dim3((w + 127) / 128, h - 4, np), 128, 0, st>>>(P, src_pitch, h, w, Sy);
  spline_my_kernel<<<dim3((w + 127) / 128, np), 128, piv_smem(h - 4), st>>>(P, src_pitch, h, w, My, Sy, piv);
  spline_ey_kernel<<<dim3((w + 31) / 32, (H + 31) / 32, np), dim3(32, 8), 0, st>>>(P, src_pitch, My, Tt, h, w, H);
  if (w > 4) spline_rx_kernel<<<dim3((H + 127) / 128, w - 4, np), 128, 0, st>>>(Tt, w, H, Sx, P.pstride);
  spline_mx_kernel<<<dim3((H + 127) / 128, np), 128, piv_smem(w - 4), st>>>(Tt, w, H, Mx, piv, Sx, P.pstride);
  spline_ex_kernel<<<dim3((W + 31) / 32, (H + 31) / 32, np), dim3(32, 8), 0, st>>>(Tt, Mx, P, dst_pitch, w, H, W);
  return check_launch("of_spline_upsample", 5 + (h > 4) + (w > 4));
}

extern "C" int of_spline_upsample(const float* src, int h, int w, int src_pitch, float* dst, int H, int W,
                                  int dst_pitch, float scale, void* workspace, size_t workspace_bytes, void* stream) {
  OF_REQUIRE(!bad_plane(src, h, w, src_pitch) && !bad_plane(dst, H, W, dst_pitch), "of_spline_upsample: bad plane");
  OF_REQUIRE(h >= 4 && w >= 4, "of_spline_upsample: the coarse field needs at least 4x4 samples");
  size_t need = of_spline_workspace_size(h, w, H, W);
  if (!workspace || workspace_bytes < need)
    return set_error(OF_ERR_WORKSPACE, "of_spline_upsample: workspace too small (%zu < %zu)", workspace_bytes, need);
  SplinePlanes P{{src, src}, {dst, dst}, {scale, scale}, 0};
  return spline_run(P, 1, h, w, src_pitch, H, W, dst_pitch, workspace, need, as_stream(stream));
}

extern "C" int of_spline_upsample_pair(const float* src_u, const float* src_v, int h, int w, int src_pitch,
                                       float* dst_u, float* dst_v, int H, int W, int dst_pitch, float scale_u,
                                       float scale_v, void* workspace, size_t workspace_bytes, void* stream) {
  OF_REQUIRE(!bad_plane(src_u, h, w, src_pitch) && !bad_plane(src_v, h, w, src_pitch) &&
                 !bad_plane(dst_u, H, W, dst_pitch) && !bad_plane(dst_v, H, W, dst_pitch),
             "of_spline_upsample_pair: bad plane");
  OF_REQUIRE(dst_u != dst_v, "of_spline_upsample_pair: the two outputs alias");
  OF_REQUIRE(h >= 4 && w >= 4, "of_spline_upsample_pair: the coarse field needs at least 4x4 samples");
  size_t single = of_spline_workspace_size(h, w, H, W);
  if (!workspace || workspace_bytes < 2 * single)
    return set_error(OF_ERR_WORKSPACE, "of_spline_upsample_pair: workspace too small (%zu < %zu)", workspace_bytes,
                     2 * single);
  SplinePlanes P{{src_u, src_v}, {dst_u, dst_v}, {scale_u, scale_v}, 0};
  return spline_run(P, 2, h, w, src_pitch, H, W, dst_pitch, workspace, single, as_stream(stream));
}

extern "C" int of_warp_pair_bilinear(const float* I0, const float* I1, const float* U, const float* V, float* O0,
                                     float* O1, int H, int W, int pitch, void* stream) {
  OF_REQUIRE(!bad_plane(I0, H, W, pitch) && I1 && U && V && O0 && O1, "of_warp_pair_bilinear: bad plane");
  warp_pair_kernel<<<dim3((W + 255) / 256, H), 256, 0, as_stream(stream)>>>(I0, I1, U, V, O0, O1, H, W, pitch);
  return check_launch("of_warp_pair_bilinear");
}

extern "C" size_t of_warp_liushen_workspace_size(int H, int W) {
  Sizer s;
  s.take<int>((size_t)H * W);  // owner of each destination
  return s.off;
}

extern "C" int of_warp_liushen_scatter(const float* I, const float* u, const float* v, float* out, float* du, float* dv,
                                       int H, int W, int pitch, int* bad, void* workspace, size_t workspace_bytes,
                                       void* stream) {
  OF_REQUIRE(!bad_plane(I, H, W, pitch) && u && v && out && du && dv && bad, "of_warp_liushen_scatter: bad arguments");
  OF_REQUIRE(out != I, "of_warp_liushen_scatter: out and I alias");
  OF_REQUIRE((long long)H * W < INT_MAX, "of_warp_liushen_scatter: image too large");
  size_t need = of_warp_liushen_workspace_size(H, W);
  if (!workspace || workspace_bytes < need)
    return set_error(OF_ERR_WORKSPACE, "of_warp_liushen_scatter: workspace too small (%zu < %zu)", workspace_bytes,
                     need);
  cudaStream_t st = as_stream(stream);
  int* owner = Carver(workspace, workspace_bytes).take<int>((size_t)H * W);
  const int n = H * W;
  lsw_init_kernel<<<(n + 255) / 256, 256, 0, st>>>(owner, n, bad);
  dim3 g((W + 127) / 128, H);
  lsw_owner_kernel<<<g, 128, 0, st>>>(u, v, H, W, pitch, owner, du, dv, bad);
  lsw_gather_kernel<<<g, 128, 0, st>>>(I, owner, out, H, W, pitch);
  return check_launch("of_warp_liushen_scatter", 3);
}

extern "C" int of_warp_liushen_ofe(const float* I, const float* du, const float* dv, float* out, int H, int W,
                                   int pitch, void* stream) {
  OF_REQUIRE(!bad_plane(I, H, W, pitch) && du && dv && out && out != I, "of_warp_liushen_ofe: bad arguments");
  dim3 g((W + 127) / 128, H);
  lsw_ofe_kernel<<<g, 128, 0, as_stream(stream)>>>(I, du, dv, out, H, W, pitch);
  return check_launch("of_warp_liushen_ofe");
}
