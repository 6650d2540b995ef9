/*
 * CPU oracle for the dense pyramidal optical-flow hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the arithmetic of
 * the reference implementation (OpticalFlow-RI) so that the CUDA kernels can be
 * checked against it.  Only tests/, __graft_entry__.smoke() and the CPU-baseline
 * leg of bench.py load it.  The product library never links or calls it.
 *
 * Parity anchors (reference file:line):
 *   prefilter          src/gaussian_filter.py:24-94
 *   Horn-Schunck       src/HornSchunck.py:51-126
 *   Liu-Shen           src/PhysicsBasedOpticalFlowLiuShen.py:47-158
 *   bilinear warp      src/GenericPyramidalOpticalFlow.py:69-115,197-200
 *   PIL resize         src/GenericPyramidalOpticalFlow.py:66-67, src/Farneback_PyCL.py:61-62
 *                      (third-party: Pillow Image.resize, restated from its published algorithm)
 *   spline upsample    src/GenericPyramidalOpticalFlow.py:151-161
 *                      (third-party: scipy RectBivariateSpline, s=0 cubic interpolation)
 *   Farneback kernels  src/optical_flow_farneback.cl:72-429
 *   dense LK           src/pyrlkDenseLargeW.cl:49-669, src/denseLucasKanade_PyCL.py:113-169
 *
 * Numeric conventions (pinned by tests/golden against the reference's own outputs):
 *   - scipy.ndimage.convolve stencils: the correlation weights (float32 values
 *     promoted to double) that are non-zero are visited in C order of the flipped
 *     weight array; each term input*weight is added to a double accumulator that
 *     starts at 0.0; the result is rounded once to float32.
 *   - numpy / numba float32 elementwise expressions: every * and + rounded to
 *     float32, left to right, no fused multiply-add.
 *   - OpenCL kernels (LK, Farneback): `mad(a,b,c)` and `acc += a*b` are taken as a
 *     fused multiply-add (fmaf); `a*b + c*d` as fmaf(a, b, c*d).  The reference's
 *     OpenCL compilers contract these by default; this restatement fixes one
 *     contraction per expression so that the CUDA kernels can match it bit for bit.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off, no -ffast-math).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define EXPORT __attribute__((visibility("default")))

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* scipy.ndimage 'mirror' (reflect without repeating the edge: d c b | a b c d | c b a) */
static inline int mirror_idx(int i, int n) {
  if (n == 1) return 0;
  int period = 2 * n - 2;
  i %= period;
  if (i < 0) i += period;
  return i < n ? i : period - i;
}

/* ------------------------------------------------------------------------------------------
 * A1 prefilter: src/gaussian_filter.py:54-85 (convolveSeparableFilter / convolveDirect).
 * Row pass then column pass, in place.  Per line of length n with K = 2h+1 taps:
 *   t[h+i] = line[i]; t[h-1-j] = line[j]; t[n+K-2-j] = line[n-1-j]   (j < h)
 *   out[x] = sum_{j=0..K-1} k[j] * t[x+2h-j]   (float32 products and adds, j ascending)
 * ------------------------------------------------------------------------------------------ */
static void prefilter_line(const float* in, int n, int stride, const float* k, int K, float* t, float* out) {
  int h = K / 2;
  for (int i = 0; i < n; i++) t[h + i] = in[(size_t)i * stride];
  for (int j = 0; j < h; j++) {
    t[h - 1 - j] = in[(size_t)j * stride];
    t[n + K - 2 - j] = in[(size_t)(n - 1 - j) * stride];
  }
  for (int x = 0; x < n; x++) {
    float acc = 0.0f;
    for (int j = 0; j < K; j++) {
      float p = t[x + 2 * h - j] * k[j];
      acc = acc + p;
    }
    out[x] = acc;
  }
}

EXPORT void ofo_prefilter(float* img, int H, int W, const float* k, int K) {
  int n = H > W ? H : W;
  float* t = (float*)malloc(sizeof(float) * (size_t)(n + K));
  float* out = (float*)malloc(sizeof(float) * (size_t)n);
  for (int y = 0; y < H; y++) {
    prefilter_line(img + (size_t)y * W, W, 1, k, K, t, out);
    memcpy(img + (size_t)y * W, out, sizeof(float) * (size_t)W);
  }
  for (int x = 0; x < W; x++) {
    prefilter_line(img + x, H, W, k, K, t, out);
    for (int y = 0; y < H; y++) img[(size_t)y * W + x] = out[y];
  }
  free(t);
  free(out);
}

/* ------------------------------------------------------------------------------------------
 * A6 Horn-Schunck derivatives: src/HornSchunck.py:106-126 called as
 * computeDerivatives(frame1, frame0) (HS(im2, im1,...) swaps, :36,:72,:83).
 * 2x2 correlation weights after scipy's flip, origin -1: offsets (0,0),(0,1),(1,0),(1,1).
 * ------------------------------------------------------------------------------------------ */
static float corr2x2_mirror(const float* I, int H, int W, int y, int x, const double w[4]) {
  int y1 = mirror_idx(y + 1, H), x1 = mirror_idx(x + 1, W);
  double acc = 0.0;
  acc += (double)I[(size_t)y * W + x] * w[0];
  acc += (double)I[(size_t)y * W + x1] * w[1];
  acc += (double)I[(size_t)y1 * W + x] * w[2];
  acc += (double)I[(size_t)y1 * W + x1] * w[3];
  return (float)acc;
}

EXPORT void ofo_hs_derivatives(const float* f0, const float* f1, float* fx, float* fy, float* ft, int H, int W) {
  static const double wx[4] = {0.25, -0.25, 0.25, -0.25};
  static const double wy[4] = {0.25, 0.25, -0.25, -0.25};
  static const double wt[4] = {0.25, 0.25, 0.25, 0.25};
  static const double wtn[4] = {-0.25, -0.25, -0.25, -0.25};
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      size_t i = (size_t)y * W + x;
      fx[i] = corr2x2_mirror(f1, H, W, y, x, wx) + corr2x2_mirror(f0, H, W, y, x, wx);
      fy[i] = corr2x2_mirror(f1, H, W, y, x, wy) + corr2x2_mirror(f0, H, W, y, x, wy);
      ft[i] = corr2x2_mirror(f0, H, W, y, x, wt) + corr2x2_mirror(f1, H, W, y, x, wtn);
    }
}

/* A7 one HS Jacobi sweep: src/HornSchunck.py:51-70.  Averaging kernel
 * [[1/12,1/6,1/12],[1/6,0,1/6],[1/12,1/6,1/12]] in float32, mode 'mirror'. */
static void hs_sweep(const float* fx, const float* fy, const float* ft, const float* U, const float* V, float* Un,
                     float* Vn, int H, int W, float alpha) {
  const double wc = (double)(float)(1.0 / 12.0), we = (double)(float)(1.0 / 6.0);
  const double w[8] = {wc, we, wc, we, we, wc, we, wc};
  const int dy[8] = {-1, -1, -1, 0, 0, 1, 1, 1}, dx[8] = {-1, 0, 1, -1, 1, -1, 0, 1};
  float a2 = alpha * alpha;
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      double su = 0.0, sv = 0.0;
      for (int t = 0; t < 8; t++) {
        size_t j = (size_t)mirror_idx(y + dy[t], H) * W + mirror_idx(x + dx[t], W);
        su += (double)U[j] * w[t];
        sv += (double)V[j] * w[t];
      }
      float ua = (float)su, va = (float)sv;
      size_t i = (size_t)y * W + x;
      float gx = fx[i], gy = fy[i];
      float num = (gx * ua + gy * va) + ft[i];
      float den = (a2 + gx * gx) + gy * gy;
      float der = num / den;
      Un[i] = ua - gx * der;
      Vn[i] = va - gy * der;
    }
}

/* HS(): src/HornSchunck.py:72-104.  f0 = frame at t0, f1 = frame at t1 (adapter order).
 * U,V in/out.  err = (||Unew-U0||_F + ||Vnew-V0||_F)/(H*W) in double. */
EXPORT void ofo_hs_solve(const float* f0, const float* f1, float* U, float* V, int H, int W, float alpha, int niter,
                         double* err) {
  size_t N = (size_t)H * W;
  float *fx = malloc(4 * N), *fy = malloc(4 * N), *ft = malloc(4 * N);
  float *U0 = malloc(4 * N), *V0 = malloc(4 * N), *Ua = malloc(4 * N), *Va = malloc(4 * N);
  ofo_hs_derivatives(f0, f1, fx, fy, ft, H, W);
  memcpy(U0, U, 4 * N);
  memcpy(V0, V, 4 * N);
  memcpy(Ua, U, 4 * N);
  memcpy(Va, V, 4 * N);
  float *cu = Ua, *cv = Va, *nu = U, *nv = V;
  for (int k = 0; k < niter; k++) {
    hs_sweep(fx, fy, ft, cu, cv, nu, nv, H, W, alpha);
    float* t = cu; cu = nu; nu = t;
    t = cv; cv = nv; nv = t;
  }
  if (cu != U) {
    memcpy(U, cu, 4 * N);
    memcpy(V, cv, 4 * N);
  }
  double su = 0, sv = 0;
  for (size_t i = 0; i < N; i++) {
    double a = (double)U[i] - U0[i], b = (double)V[i] - V0[i];
    su += a * a;
    sv += b * b;
  }
  if (err) *err = (sqrt(su) + sqrt(sv)) / (double)N;
  free(fx); free(fy); free(ft); free(U0); free(V0); free(Ua); free(Va);
}

/* ------------------------------------------------------------------------------------------
 * A8/A9 Liu-Shen: src/PhysicsBasedOpticalFlowLiuShen.py:47-158.
 * Inside the solver "u" is the row (y) component; the adapter (:37-39) swaps.
 * Borders: 'nearest' (clamp) except H (8-neighbour sum) which is 'constant' 0.
 * ------------------------------------------------------------------------------------------ */
#define AT(P, y, x) (P)[(size_t)clampi((y), 0, H - 1) * W + clampi((x), 0, W - 1)]

static inline float st_dy(const float* P, int H, int W, int y, int x) {  /* D, rows */
  double a = 0.0;
  a += (double)AT(P, y - 1, x) * -0.5;
  a += (double)AT(P, y + 1, x) * 0.5;
  return (float)a;
}
static inline float st_dx(const float* P, int H, int W, int y, int x) {  /* D^T, columns */
  double a = 0.0;
  a += (double)AT(P, y, x - 1) * -0.5;
  a += (double)AT(P, y, x + 1) * 0.5;
  return (float)a;
}
static inline float st_fy(const float* P, int H, int W, int y, int x) {  /* F, rows */
  double a = 0.0;
  a += (double)AT(P, y - 1, x);
  a += (double)AT(P, y + 1, x);
  return (float)a;
}
static inline float st_fx(const float* P, int H, int W, int y, int x) {  /* F^T, columns */
  double a = 0.0;
  a += (double)AT(P, y, x - 1);
  a += (double)AT(P, y, x + 1);
  return (float)a;
}
static inline float st_m(const float* P, int H, int W, int y, int x) {  /* M, mixed */
  double a = 0.0;
  a += (double)AT(P, y - 1, x - 1) * 0.25;
  a += (double)AT(P, y - 1, x + 1) * -0.25;
  a += (double)AT(P, y + 1, x - 1) * -0.25;
  a += (double)AT(P, y + 1, x + 1) * 0.25;
  return (float)a;
}
static inline float st_d2y(const float* P, int H, int W, int y, int x) {
  double a = 0.0;
  a += (double)AT(P, y - 1, x);
  a += (double)AT(P, y, x) * -2.0;
  a += (double)AT(P, y + 1, x);
  return (float)a;
}
static inline float st_d2x(const float* P, int H, int W, int y, int x) {
  double a = 0.0;
  a += (double)AT(P, y, x - 1);
  a += (double)AT(P, y, x) * -2.0;
  a += (double)AT(P, y, x + 1);
  return (float)a;
}
static inline float st_h(const float* P, int H, int W, int y, int x) {  /* 8-neighbour sum, constant 0 */
  double a = 0.0;
  for (int dy = -1; dy <= 1; dy++)
    for (int dx = -1; dx <= 1; dx++) {
      if (!dy && !dx) continue;
      int yy = y + dy, xx = x + dx;
      double v = (yy >= 0 && yy < H && xx >= 0 && xx < W) ? (double)P[(size_t)yy * W + xx] : 0.0;
      a += v;
    }
  return (float)a;
}
static inline float count_nb(int H, int W, int y, int x) {
  int c = 0;
  for (int dy = -1; dy <= 1; dy++)
    for (int dx = -1; dx <= 1; dx++) {
      if (!dy && !dx) continue;
      int yy = y + dy, xx = x + dx;
      c += (yy >= 0 && yy < H && xx >= 0 && xx < W);
    }
  return (float)c;
}

static float max_f32(const float* P, size_t N) {
  float m = P[0];
  for (size_t i = 1; i < N; i++)
    if (P[i] > m || P[i] != P[i]) m = P[i];
  return m;
}

/* Builds the 8 per-pixel coefficient planes of the LS solver from the raw frames:
 * c[0..7] = IIx, IIy, II, Ixt, Iyt, B11, B12, B22 (the exact float32 expressions of :96-128, :47-73). */
EXPORT void ofo_ls_coeffs(const float* im1, const float* im2, int H, int W, float h, float* coef) {
  size_t N = (size_t)H * W;
  float *I1 = malloc(4 * N), *I2 = malloc(4 * N), *Et = malloc(4 * N);
  float m1 = max_f32(im1, N), m2 = max_f32(im2, N);
  for (size_t i = 0; i < N; i++) {
    I1[i] = im1[i] / m1;
    I2[i] = im2[i] / m2;
    Et[i] = I2[i] - I1[i];
  }
  float *IIx = coef, *IIy = coef + N, *II = coef + 2 * N, *Ixt = coef + 3 * N, *Iyt = coef + 4 * N;
  float *B11 = coef + 5 * N, *B12 = coef + 6 * N, *B22 = coef + 7 * N;
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      size_t i = (size_t)y * W + x;
      float I = I1[i];
      IIx[i] = I * st_dy(I1, H, W, y, x);
      IIy[i] = I * st_dx(I1, H, W, y, x);
      II[i] = I * I;
      Ixt[i] = I * st_dy(Et, H, W, y, x);
      Iyt[i] = I * st_dx(Et, H, W, y, x);
      float cm = count_nb(H, W, y, x);
      float twoI = 2.0f * I;
      float A11 = I * (st_d2y(I1, H, W, y, x) - twoI) - h * cm;
      float A22 = I * (st_d2x(I1, H, W, y, x) - twoI) - h * cm;
      float A12 = I * st_m(I1, H, W, y, x);
      float det = A11 * A22 - A12 * A12;
      B11[i] = A22 / det;
      B12[i] = (-A12) / det;
      B22[i] = A11 / det;
    }
  free(I1); free(I2); free(Et);
}

/* One LS sweep (:142-150).  Returns sum of squared changes in ss[0] (u) and ss[1] (v). */
EXPORT void ofo_ls_sweep(const float* coef, const float* u, const float* v, float* un, float* vn, int H, int W,
                         float h, double* ss) {
  size_t N = (size_t)H * W;
  const float *IIx = coef, *IIy = coef + N, *II = coef + 2 * N, *Ixt = coef + 3 * N, *Iyt = coef + 4 * N;
  const float *B11 = coef + 5 * N, *B12 = coef + 6 * N, *B22 = coef + 7 * N;
  double su = 0, sv = 0;
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      size_t i = (size_t)y * W + x;
      float Du = st_dy(u, H, W, y, x), DTu = st_dx(u, H, W, y, x);
      float Dv = st_dy(v, H, W, y, x), DTv = st_dx(v, H, W, y, x);
      float Fu = st_fy(u, H, W, y, x), FTv = st_fx(v, H, W, y, x);
      float Mu = st_m(u, H, W, y, x), Mv = st_m(v, H, W, y, x);
      float Hu = st_h(u, H, W, y, x), Hv = st_h(v, H, W, y, x);
      float a = IIx[i], b = IIy[i], c = II[i];
      float bu = (2.0f * a) * Du;
      bu = bu + a * DTv;
      bu = bu + b * Dv;
      bu = bu + c * Fu;
      bu = bu + c * Mv;
      bu = bu + h * Hu;
      bu = bu + Ixt[i];
      float bv = b * Du;
      bv = bv + a * DTu;
      bv = bv + (2.0f * b) * DTv;
      bv = bv + c * Mu;
      bv = bv + c * FTv;
      bv = bv + h * Hv;
      bv = bv + Iyt[i];
      float nu = -(B11[i] * bu + B12[i] * bv);
      float nv = -(B12[i] * bu + B22[i] * bv);
      /* float32 change as the reference's unew - u (:79); squares summed in double */
      double du = (double)(float)(nu - u[i]), dv = (double)(float)(nv - v[i]);
      su += du * du;
      sv += dv * dv;
      un[i] = nu;
      vn[i] = nv;
    }
  ss[0] = su;
  ss[1] = sv;
}

/* Adapter-level LS: compute(im1, im2, U, V) -> (U, V, error) with U = x (column) flow.
 * Loop rule (:88-89,:141): while err > tol and k < maxnum. */
EXPORT void ofo_ls_solve(const float* im1, const float* im2, float* U, float* V, int H, int W, float h, int maxnum,
                         double tol, int* iters, double* err) {
  size_t N = (size_t)H * W;
  float* coef = malloc(4 * N * 8);
  ofo_ls_coeffs(im1, im2, H, W, h, coef);
  float *u = malloc(4 * N), *v = malloc(4 * N), *un = malloc(4 * N), *vn = malloc(4 * N);
  memcpy(u, V, 4 * N); /* row component */
  memcpy(v, U, 4 * N); /* column component */
  double total = 1e8, e = 0.0;
  int k = 0;
  while (total > tol && k < maxnum) {
    double ss[2];
    ofo_ls_sweep(coef, u, v, un, vn, H, W, h, ss);
    total = (sqrt(ss[0]) + sqrt(ss[1])) / (double)N;
    float* t = u; u = un; un = t;
    t = v; v = vn; vn = t;
    e = total;
    k++;
  }
  memcpy(V, u, 4 * N);
  memcpy(U, v, 4 * N);
  if (iters) *iters = k;
  if (err) *err = e;
  free(coef); free(u); free(v); free(un); free(vn);
}
#undef AT

/* ------------------------------------------------------------------------------------------
 * A4 bilinear warp: src/GenericPyramidalOpticalFlow.py:69-115 with coordinates
 * y -+ v/2, x -+ u/2 rounded to float32 (:197-200).  numpy promotes float32 - int32 to
 * float64, so the fractional weights and the blend are double; the result is float32.
 * ------------------------------------------------------------------------------------------ */
static float round_half_even_f(float c) { return nearbyintf(c); }

static float warp_sample(const float* img, int H, int W, float cy, float cx) {
  int iy = (int)round_half_even_f(cy), ix = (int)round_half_even_f(cx);
  double dyv = (double)cy - (double)iy, dxv = (double)cx - (double)ix;
  int ny = dyv < 0 ? iy - 1 : iy + 1, nx = dxv < 0 ? ix - 1 : ix + 1;
  dyv = fabs(dyv);
  dxv = fabs(dxv);
  iy = clampi(iy, 0, H - 1);
  ny = clampi(ny, 0, H - 1);
  ix = clampi(ix, 0, W - 1);
  nx = clampi(nx, 0, W - 1);
  double a = (1.0 - dyv) * (1.0 - dxv) * (double)img[(size_t)iy * W + ix];
  a = a + (1.0 - dyv) * dxv * (double)img[(size_t)iy * W + nx];
  a = a + dyv * (1.0 - dxv) * (double)img[(size_t)ny * W + ix];
  a = a + dyv * dxv * (double)img[(size_t)ny * W + nx];
  return (float)a;
}

EXPORT void ofo_warp_pair(const float* I0, const float* I1, const float* U, const float* V, float* O0, float* O1,
                          int H, int W) {
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      size_t i = (size_t)y * W + x;
      float hv = V[i] / 2.0f, hu = U[i] / 2.0f;
      float cy0 = (float)((double)y - (double)hv), cx0 = (float)((double)x - (double)hu);
      float cy1 = (float)((double)y + (double)hv), cx1 = (float)((double)x + (double)hu);
      O0[i] = warp_sample(I0, H, W, cy0, cx0);
      O1[i] = warp_sample(I1, H, W, cy1, cx1);
    }
}

/* ------------------------------------------------------------------------------------------
 * A2 antialiased resize of a float32 image (Pillow Image.resize, mode 'F').
 * Restated from Pillow's published two-pass algorithm: per output coordinate a
 * normalised kernel in double over [xmin, xmin+xmax); horizontal pass first into a
 * float32 intermediate, then the vertical pass; double accumulation.
 * filter: 0 = bilinear (support 1), 1 = bicubic a=-0.5 (support 2).
 * ------------------------------------------------------------------------------------------ */
static double filt_bilinear(double x) {
  if (x < 0.0) x = -x;
  if (x < 1.0) return 1.0 - x;
  return 0.0;
}
static double filt_bicubic(double x) {
  const double a = -0.5;
  if (x < 0.0) x = -x;
  if (x < 1.0) return ((a + 2.0) * x - (a + 3.0)) * x * x + 1;
  if (x < 2.0) return (((x - 5) * x + 8) * x - 4) * a;
  return 0.0;
}

EXPORT int ofo_resize_coeffs(int inSize, int outSize, int filter, int* bounds, double* kk, int ksize_cap) {
  double support, scale, filterscale;
  double (*f)(double) = filter ? filt_bicubic : filt_bilinear;
  double fsupport = filter ? 2.0 : 1.0;
  filterscale = scale = (double)((float)inSize - 0.0f) / outSize;
  if (filterscale < 1.0) filterscale = 1.0;
  support = fsupport * filterscale;
  int ksize = (int)ceil(support) * 2 + 1;
  if (!kk) return ksize;
  if (ksize > ksize_cap) return -1;
  for (int xx = 0; xx < outSize; xx++) {
    double center = 0.0 + (xx + 0.5) * scale;
    double ww = 0.0, ss = 1.0 / filterscale;
    int xmin = (int)(center - support + 0.5);
    if (xmin < 0) xmin = 0;
    int xmax = (int)(center + support + 0.5);
    if (xmax > inSize) xmax = inSize;
    xmax -= xmin;
    double* k = &kk[(size_t)xx * ksize];
    int x;
    for (x = 0; x < xmax; x++) {
      double w = f((x + xmin - center + 0.5) * ss);
      k[x] = w;
      ww += w;
    }
    for (x = 0; x < xmax; x++)
      if (ww != 0.0) k[x] /= ww;
    for (; x < ksize; x++) k[x] = 0;
    bounds[xx * 2 + 0] = xmin;
    bounds[xx * 2 + 1] = xmax;
  }
  return ksize;
}

EXPORT void ofo_resize(const float* src, int Hs, int Ws, float* dst, int Hd, int Wd, int filter) {
  if (Hs == Hd && Ws == Wd) {
    memcpy(dst, src, sizeof(float) * (size_t)Hs * Ws);
    return;
  }
  int need_h = Wd != Ws, need_v = Hd != Hs;
  const float* cur = src;
  float* tmp = NULL;
  if (need_h) {
    int ks = ofo_resize_coeffs(Ws, Wd, filter, NULL, NULL, 0);
    int* b = malloc(sizeof(int) * 2 * Wd);
    double* kk = malloc(sizeof(double) * (size_t)ks * Wd);
    ofo_resize_coeffs(Ws, Wd, filter, b, kk, ks);
    float* out = need_v ? (tmp = malloc(sizeof(float) * (size_t)Hs * Wd)) : dst;
    for (int y = 0; y < Hs; y++)
      for (int xx = 0; xx < Wd; xx++) {
        double ss = 0.0;
        const double* k = &kk[(size_t)xx * ks];
        for (int x = 0; x < b[2 * xx + 1]; x++) ss += (double)src[(size_t)y * Ws + x + b[2 * xx]] * k[x];
        out[(size_t)y * Wd + xx] = (float)ss;
      }
    free(b);
    free(kk);
    cur = out;
  }
  if (need_v) {
    int ks = ofo_resize_coeffs(Hs, Hd, filter, NULL, NULL, 0);
    int* b = malloc(sizeof(int) * 2 * Hd);
    double* kk = malloc(sizeof(double) * (size_t)ks * Hd);
    ofo_resize_coeffs(Hs, Hd, filter, b, kk, ks);
    for (int yy = 0; yy < Hd; yy++)
      for (int x = 0; x < Wd; x++) {
        double ss = 0.0;
        const double* k = &kk[(size_t)yy * ks];
        for (int y = 0; y < b[2 * yy + 1]; y++) ss += (double)cur[(size_t)(y + b[2 * yy]) * Wd + x] * k[y];
        dst[(size_t)yy * Wd + x] = (float)ss;
      }
    free(b);
    free(kk);
  }
  free(tmp);
}

/* ------------------------------------------------------------------------------------------
 * A3 flow upsample: src/GenericPyramidalOpticalFlow.py:151-161.
 * RectBivariateSpline(kx=ky=3, s=0) on x_i = i/n is the not-a-knot cubic interpolant
 * (FITPACK places interior knots at x_2..x_{n-3}); it is evaluated at j/N with points
 * beyond the last sample clamped to the domain.  Restated with second-derivative
 * (moment) form on unit spacing, in double, rows then columns; result rounded to f32.
 * ------------------------------------------------------------------------------------------ */
/* moments of the not-a-knot spline through y[0..n-1] (n >= 4), unit spacing */
/* Reciprocal pivots of the constant (1, 4, 1) tridiagonal elimination:
 * c[0] = 1/4, c[r] = 1/(4 - c[r-1]); the sequence reaches its fixed point (2 - sqrt 3) in
 * double after a few tens of steps, after which every entry repeats it. */
static void nak_recip(double* c, int m) {
  if (m <= 0) return;
  c[0] = 1.0 / 4.0;
  int r = 1;
  for (; r < m; r++) {
    c[r] = 1.0 / (4.0 - c[r - 1]);
    if (c[r] == c[r - 1]) break;
  }
  for (; r < m; r++) c[r] = c[r - 1];
}

static void nak_moments(const double* y, int n, double* M, double* cp, double* dp) {
  /* M1 = d1, M_{n-2} = d_{n-2}; interior rows i=2..n-3: M_{i-1}+4M_i+M_{i+1} = 6 d_i,
   * eliminated with the pivots of nak_recip (cp) as multiplications */
  double d1 = y[2] - 2.0 * y[1] + y[0];
  double dl = y[n - 1] - 2.0 * y[n - 2] + y[n - 3];
  M[1] = d1;
  M[n - 2] = dl;
  int m = n - 4; /* unknowns M_2 .. M_{n-3} */
  if (m > 0) {
    nak_recip(cp, m);
    for (int r = 0; r < m; r++) {
      int i = r + 2;
      double rhs = 6.0 * (y[i + 1] - 2.0 * y[i] + y[i - 1]);
      if (r == 0) rhs -= M[1];
      if (r == m - 1) rhs -= M[n - 2];
      if (r == 0)
        dp[r] = rhs * cp[r];
      else
        dp[r] = (rhs - dp[r - 1]) * cp[r];
    }
    M[m + 1] = dp[m - 1];
    for (int r = m - 2; r >= 0; r--) M[r + 2] = dp[r] - cp[r] * M[r + 3];
  }
  M[0] = 2.0 * M[1] - M[2];
  M[n - 1] = 2.0 * M[n - 2] - M[n - 3];
}

static double nak_eval(const double* y, const double* M, int n, double s) {
  if (s < 0.0) s = 0.0;
  if (s > n - 1) s = n - 1;
  int i = (int)floor(s);
  if (i > n - 2) i = n - 2;
  double t = s - i, u = 1.0 - t;
  return u * y[i] + t * y[i + 1] + ((u * u * u - u) * M[i] + (t * t * t - t) * M[i + 1]) / 6.0;
}

/* position of fine sample j of N on the coarse index axis of n samples: (j/N)*n */
static double fine_pos(int j, int N, int n) { return ((double)j / (double)N) * (double)n; }

EXPORT void ofo_spline_upsample(const float* src, int h, int w, float* dst, int H, int W) {
  int nmax = (h > w ? h : w) + 4;
  double *line = malloc(8 * nmax), *M = malloc(8 * nmax), *cp = malloc(8 * nmax), *dp = malloc(8 * nmax);
  double* T = malloc(8 * (size_t)H * w); /* columns interpolated to fine rows */
  for (int x = 0; x < w; x++) {
    for (int i = 0; i < h; i++) line[i] = src[(size_t)i * w + x];
    nak_moments(line, h, M, cp, dp);
    for (int Y = 0; Y < H; Y++) T[(size_t)Y * w + x] = nak_eval(line, M, h, fine_pos(Y, H, h));
  }
  for (int Y = 0; Y < H; Y++) {
    const double* row = &T[(size_t)Y * w];
    nak_moments(row, w, M, cp, dp);
    for (int X = 0; X < W; X++) dst[(size_t)Y * W + X] = (float)nak_eval(row, M, w, fine_pos(X, W, w));
  }
  free(line); free(M); free(cp); free(dp); free(T);
}

/* ------------------------------------------------------------------------------------------
 * Farneback kernels: src/optical_flow_farneback.cl.  Planes are stacked: plane p of an
 * H x W field lives at [p*H*W].
 * ------------------------------------------------------------------------------------------ */
/* polynomialExpansion :72-133; g/xg/xxg hold polyN+1 taps (the centre and one side). */
EXPORT void ofo_fb_polyexp(const float* src, float* dst, int H, int W, int polyN, const float* g, const float* xg,
                           const float* xxg, const float* ig) {
  size_t N = (size_t)H * W;
  float* rows = malloc(sizeof(float) * 3 * (size_t)W);
  for (int y = 0; y < H; y++) {
    for (int x = 0; x < W; x++) {
      float r0 = src[(size_t)y * W + x] * g[0], r1 = 0.f, r2 = 0.f;
      for (int k = 1; k <= polyN; k++) {
        float t0 = src[(size_t)(y - k < 0 ? 0 : y - k) * W + x];
        float t1 = src[(size_t)(y + k > H - 1 ? H - 1 : y + k) * W + x];
        r0 = fmaf(g[k], t0 + t1, r0);
        r1 = fmaf(xg[k], t1 - t0, r1);
        r2 = fmaf(xxg[k], t0 + t1, r2);
      }
      rows[x] = r0;
      rows[W + x] = r1;
      rows[2 * W + x] = r2;
    }
#define RW(p, xx) rows[(p) * W + clampi((xx), 0, W - 1)]
    for (int x = 0; x < W; x++) {
      float b1 = g[0] * RW(0, x), b3 = g[0] * RW(1, x), b5 = g[0] * RW(2, x);
      float b2 = 0, b4 = 0, b6 = 0;
      for (int k = 1; k <= polyN; k++) {
        float sp = RW(0, x + k) + RW(0, x - k), sm = RW(0, x + k) - RW(0, x - k);
        b1 = fmaf(sp, g[k], b1);
        b4 = fmaf(sp, xxg[k], b4);
        b2 = fmaf(sm, xg[k], b2);
        b3 = fmaf(RW(1, x + k) + RW(1, x - k), g[k], b3);
        b6 = fmaf(RW(1, x + k) - RW(1, x - k), xg[k], b6);
        b5 = fmaf(RW(2, x + k) + RW(2, x - k), g[k], b5);
      }
      size_t i = (size_t)y * W + x;
      dst[i] = b3 * ig[0];
      dst[N + i] = b2 * ig[0];
      dst[2 * N + i] = fmaf(b1, ig[1], b5 * ig[2]);
      dst[3 * N + i] = fmaf(b1, ig[1], b4 * ig[2]);
      dst[4 * N + i] = b6 * ig[3];
    }
#undef RW
  }
  free(rows);
}

static inline int fb_row_low(int y, int last) { return abs(y) % (last + 1); }
static inline int fb_row_high(int y, int last) { return abs(last - abs(last - y)) % (last + 1); }
static inline int fb_col(int x, int last) { return fb_row_low(fb_row_high(x, last), last); }

/* gaussianBlur :160-196 on `planes` stacked planes (gaussianBlur5 :198-253 when planes=5). */
EXPORT void ofo_fb_blur(const float* src, float* dst, int H, int W, int planes, const float* gk, int kh) {
  size_t N = (size_t)H * W;
  float* row = malloc(sizeof(float) * (size_t)(W + 2 * kh));
  for (int p = 0; p < planes; p++) {
    const float* s = src + p * N;
    for (int y = 0; y < H; y++) {
      for (int i = 0; i < W + 2 * kh; i++) {
        int xe = fb_col(i - kh, W - 1);
        float acc = s[(size_t)y * W + xe] * gk[0];
        for (int j = 1; j <= kh; j++)
          acc = fmaf(s[(size_t)fb_row_low(y - j, H - 1) * W + xe] + s[(size_t)fb_row_high(y + j, H - 1) * W + xe],
                     gk[j], acc);
        row[i] = acc;
      }
      for (int x = 0; x < W; x++) {
        const float* r = row + x + kh;
        float res = r[0] * gk[0];
        for (int i = 1; i <= kh; i++) res = fmaf(r[-i] + r[i], gk[i], res);
        dst[p * N + (size_t)y * W + x] = res;
      }
    }
  }
  free(row);
}

/* boxFilter5 :350-406 (clamped borders). */
EXPORT void ofo_fb_box5(const float* src, float* dst, int H, int W, int kh) {
  size_t N = (size_t)H * W;
  float inv = 1.f / (float)((1 + 2 * kh) * (1 + 2 * kh));
  float* row = malloc(sizeof(float) * (size_t)(W + 2 * kh));
  for (int p = 0; p < 5; p++) {
    const float* s = src + p * N;
    for (int y = 0; y < H; y++) {
      for (int i = 0; i < W + 2 * kh; i++) {
        int xe = clampi(i - kh, 0, W - 1);
        float acc = s[(size_t)y * W + xe];
        for (int j = 1; j <= kh; j++)
          acc = acc + (s[(size_t)clampi(y - j, 0, H - 1) * W + xe] + s[(size_t)clampi(y + j, 0, H - 1) * W + xe]);
        row[i] = acc;
      }
      for (int x = 0; x < W; x++) {
        const float* r = row + x + kh;
        float res = r[0];
        for (int i = 1; i <= kh; i++) res = res + (r[-i] + r[i]);
        dst[p * N + (size_t)y * W + x] = res * inv;
      }
    }
  }
  free(row);
}

/* updateMatrices :254-348 */
EXPORT void ofo_fb_update_matrices(const float* flowx, const float* flowy, const float* R0, const float* R1,
                                   float* M, int H, int W) {
  static const float c_border[6] = {0.14f, 0.14f, 0.4472f, 0.4472f, 0.4472f, 1.f};
  size_t N = (size_t)H * W;
  for (int y = 0; y < H; y++)
    for (int x = 0; x < W; x++) {
      size_t i = (size_t)y * W + x;
      float dx = flowx[i], dy = flowy[i];
      float fx = (float)x + dx, fy = (float)y + dy;
      int x1 = (int)floorf(fx), y1 = (int)floorf(fy);
      fx -= (float)x1;
      fy -= (float)y1;
      float r2, r3, r4, r5, r6;
      if (x1 >= 0 && y1 >= 0 && x1 < W - 1 && y1 < H - 1) {
        float a00 = (1.f - fx) * (1.f - fy), a01 = fx * (1.f - fy);
        float a10 = (1.f - fx) * fy, a11 = fx * fy;
        float rr[5];
        for (int p = 0; p < 5; p++) {
          const float* R = R1 + p * N;
          size_t j = (size_t)y1 * W + x1;
          float t = fmaf(a00, R[j], a01 * R[j + 1]);
          t = fmaf(a10, R[j + W], t);
          t = fmaf(a11, R[j + W + 1], t);
          rr[p] = t;
        }
        r2 = rr[0];
        r3 = rr[1];
        r4 = (R0[2 * N + i] + rr[2]) * 0.5f;
        r5 = (R0[3 * N + i] + rr[3]) * 0.5f;
        r6 = (R0[4 * N + i] + rr[4]) * 0.25f;
      } else {
        r2 = r3 = 0.f;
        r4 = R0[2 * N + i];
        r5 = R0[3 * N + i];
        r6 = R0[4 * N + i] * 0.5f;
      }
      r2 = (R0[i] - r2) * 0.5f;
      r3 = (R0[N + i] - r3) * 0.5f;
      r2 = r2 + fmaf(r4, dy, r6 * dx);
      r3 = r3 + fmaf(r6, dy, r5 * dx);
      float scale = c_border[x < 5 ? x : 5] * c_border[y < 5 ? y : 5];
      scale = scale * c_border[W - x - 1 < 5 ? W - x - 1 : 5];
      scale = scale * c_border[H - y - 1 < 5 ? H - y - 1 : 5];
      r2 *= scale;
      r3 *= scale;
      r4 *= scale;
      r5 *= scale;
      r6 *= scale;
      M[i] = fmaf(r4, r4, r6 * r6);
      M[N + i] = (r4 + r5) * r6;
      M[2 * N + i] = fmaf(r5, r5, r6 * r6);
      M[3 * N + i] = fmaf(r4, r2, r6 * r3);
      M[4 * N + i] = fmaf(r6, r2, r5 * r3);
    }
}

/* updateFlow :408-429 */
EXPORT void ofo_fb_update_flow(const float* M, float* flowx, float* flowy, int H, int W) {
  size_t N = (size_t)H * W;
  for (size_t i = 0; i < N; i++) {
    float g11 = M[i], g12 = M[N + i], g22 = M[2 * N + i], h1 = M[3 * N + i], h2 = M[4 * N + i];
    float detInv = 1.f / (fmaf(g11, g22, -(g12 * g12)) + 1e-3f);
    flowx[i] = fmaf(g11, h2, -(g12 * h1)) * detInv;
    flowy[i] = fmaf(g22, h1, -(g12 * h2)) * detInv;
  }
}

/* ------------------------------------------------------------------------------------------
 * A10/A11 dense Lucas-Kanade: src/pyrlkDenseLargeW.cl:236-669 (non-CPU build path), one
 * 8x8 work-group per pixel restated as 64 virtual threads; per-thread sums over 16 tiles
 * in the kernel's order, then the 64->1 tree of reduce1/2/3 (:111-224).
 * Image reads use CLAMP_TO_EDGE; J is sampled with exact float32 bilinear weights at
 * (x-0.5, y-0.5) (the reference's sampler uses reduced-precision hardware weights).
 * ------------------------------------------------------------------------------------------ */
static inline float img_at(const float* I, int H, int W, int y, int x) {
  return I[(size_t)clampi(y, 0, H - 1) * W + clampi(x, 0, W - 1)];
}

static inline float bilinear_cl(const float* J, int H, int W, float x, float y) {
  float xs = x - 0.5f, ys = y - 0.5f;
  float fx0 = floorf(xs), fy0 = floorf(ys);
  float a = xs - fx0, b = ys - fy0;
  int i0 = (int)fx0, j0 = (int)fy0;
  float t00 = img_at(J, H, W, j0, i0), t10 = img_at(J, H, W, j0, i0 + 1);
  float t01 = img_at(J, H, W, j0 + 1, i0), t11 = img_at(J, H, W, j0 + 1, i0 + 1);
  float w00 = (1.f - a) * (1.f - b), w10 = a * (1.f - b), w01 = (1.f - a) * b, w11 = a * b;
  float r = w00 * t00;
  r = fmaf(w10, t10, r);
  r = fmaf(w01, t01, r);
  r = fmaf(w11, t11, r);
  return r;
}

/* tree of reduce3/reduce2/reduce1: 64 -> 32 -> 16 -> 8 -> 4 -> (s0+s1)+(s2+s3) */
static float tree64(float* s) {
  for (int t = 0; t < 32; t++) s[t] += s[t + 32];
  for (int t = 0; t < 16; t++) s[t] += s[t + 16];
  for (int t = 0; t < 8; t++) s[t] += s[t + 8];
  for (int t = 0; t < 4; t++) s[t] += s[t + 4];
  return (s[0] + s[1]) + (s[2] + s[3]);
}

/* tile weights of one virtual thread (xid, yid) along one axis, :339-373 */
static void lk_axis_weights(int id, int ws, int asym_lo, int asym_hi, float w[4], int base[2]) {
  if (ws >= 16) {
    w[0] = 1.f;
    w[1] = 1.f;
    base[0] = 16 + id;
    base[1] = 24 + id;
    w[2] = (base[0] < ws - asym_hi) ? 1.f : 0.f;
    w[3] = (base[1] < ws - asym_hi) ? 1.f : 0.f;
    if (id == 0) w[1] = (float)(1 - asym_lo);
  } else {
    base[0] = 8 + id;
    base[1] = 16 + id;
    w[0] = 1.f;
    w[1] = (base[0] < ws - asym_hi) ? 1.f : 0.f;
    if (id == 0) w[1] = (float)(1 - asym_lo);
    w[2] = 0.f;
    w[3] = 0.f;
  }
}

EXPORT void ofo_lk_dense(const float* I, const float* J, float* U, float* V, int H, int W, int halfWin, int niter,
                         const int* asym, unsigned char* status, float* err) {
  const int ws = 2 * halfWin + 1;
  const float hw = (float)((ws - 1) >> 1);
  int aL = asym ? asym[0] : 0, aR = asym ? asym[1] : 0, aT = asym ? asym[2] : 0, aB = asym ? asym[3] : 0;
  float Ip[64][16], Dx[64][16], Dy[64][16], wt[64][16];
  float s1[64], s2[64], s3[64];
  for (int i = 0; i < H; i++)
    for (int j = 0; j < W; j++) {
      size_t gid = (size_t)i * W + j;
      if (status) status[gid] = 1;
      float px = (float)j - hw, py = (float)i - hw;
      /* A matrix */
      for (int tid = 0; tid < 64; tid++) {
        int xid = tid & 7, yid = tid >> 3;
        float wx[4], wy[4];
        int bx[2], by[2];
        lk_axis_weights(xid, ws, aL, aR, wx, bx);
        lk_axis_weights(yid, ws, aT, aB, wy, by);
        float A11 = 0, A12 = 0, A22 = 0;
        for (int ty = 0; ty < 4; ty++)
          for (int tx = 0; tx < 4; tx++) {
            float w = wx[tx] * wy[ty]; /* wx[0] = wy[0] = 1, so this is the kernel's per-tile weight */
            /* window position -> image position (patch read at Point - 1 with +1 offset) */
            int yy = (int)py + ty * 8 + yid, xx = (int)px + tx * 8 + xid;
#define P(dy, dx) img_at(I, H, W, yy + (dy), xx + (dx))
            float dxv = fmaf(((P(-1, 1) + P(1, 1)) - P(-1, -1)) - P(1, -1), 3.0f, (P(0, 1) - P(0, -1)) * 10.0f) * w;
            float dyv = fmaf(((P(1, -1) + P(1, 1)) - P(-1, -1)) - P(-1, 1), 3.0f, (P(1, 0) - P(-1, 0)) * 10.0f) * w;
            Ip[tid][ty * 4 + tx] = P(0, 0);
#undef P
            Dx[tid][ty * 4 + tx] = dxv;
            Dy[tid][ty * 4 + tx] = dyv;
            wt[tid][ty * 4 + tx] = w;
            A11 = fmaf(dxv, dxv, A11);
            A12 = fmaf(dxv, dyv, A12);
            A22 = fmaf(dyv, dyv, A22);
          }
        s1[tid] = A11;
        s2[tid] = A12;
        s3[tid] = A22;
      }
      float A11 = tree64(s1), A12 = tree64(s2), A22 = tree64(s3);
      float D = fmaf(A11, A22, -(A12 * A12));
      if (D < 1.192092896e-07f) {
        if (status) status[gid] = 0;
        if (err) err[gid] = 0.f;
        continue;
      }
      A11 /= D;
      A12 /= D;
      A22 /= D;
      float ptx = ((float)j + U[gid]) - hw, pty = ((float)i + V[gid]) - hw;
      float lx[4][64], ly[4][64]; /* loc0..loc3 per virtual thread */
      for (int tid = 0; tid < 64; tid++) {
        int xid = tid & 7, yid = tid >> 3;
        lx[0][tid] = ptx + ((float)xid + 0.5f);
        ly[0][tid] = pty + ((float)yid + 0.5f);
        for (int t = 1; t < 4; t++) {
          lx[t][tid] = lx[t - 1][tid] + 8.0f;
          ly[t][tid] = ly[t - 1][tid] + 8.0f;
        }
      }
      for (int k = 0; k < niter; k++) {
        if (ptx < -hw || ptx >= (float)W || pty < -hw || pty >= (float)H) {
          if (status) status[gid] = 0;
          break;
        }
        for (int tid = 0; tid < 64; tid++) {
          float b1 = 0, b2 = 0;
          for (int ty = 0; ty < 4; ty++)
            for (int tx = 0; tx < 4; tx++) {
              int q = ty * 4 + tx;
              float diff = (bilinear_cl(J, H, W, lx[tx][tid], ly[ty][tid]) - Ip[tid][q]) * wt[tid][q];
              b1 = fmaf(diff, Dx[tid][q], b1);
              b2 = fmaf(diff, Dy[tid][q], b2);
            }
          s1[tid] = b1;
          s2[tid] = b2;
        }
        float b1 = tree64(s1), b2 = tree64(s2);
        float dx = fmaf(A12, b2, -(A22 * b1)) * 32.0f;
        float dy = fmaf(A12, b1, -(A11 * b2)) * 32.0f;
        ptx += dx;
        pty += dy;
        for (int tid = 0; tid < 64; tid++)
          for (int t = 0; t < 4; t++) {
            lx[t][tid] += dx;
            ly[t][tid] += dy;
          }
        if (fabsf(dx) < 0.01f && fabsf(dy) < 0.01f) break;
      }
      if (err) {
        for (int tid = 0; tid < 64; tid++) {
          int xid = tid & 7, yid = tid >> 3;
          float wx[4], wy[4];
          int bx[2], by[2];
          lk_axis_weights(xid, ws, aL, aR, wx, bx);
          lk_axis_weights(yid, ws, aT, aB, wy, by);
          float e = 0.f;
          /* GetError visiting order and guards, :620-653.  guard bits: 1 xBase, 2 yBase, 4 xBase2, 8 yBase2 */
          static const int order[16][3] = {{0, 0, 0}, {0, 1, 0}, {1, 0, 0}, {1, 1, 0}, {0, 2, 1}, {1, 2, 1},
                                           {2, 0, 2}, {2, 1, 2}, {2, 2, 3}, {0, 3, 4}, {1, 3, 4}, {2, 3, 4},
                                           {3, 0, 8}, {3, 1, 8}, {3, 2, 8}, {3, 3, 12}};
          for (int o = 0; o < 16; o++) {
            int ty = order[o][0], tx = order[o][1], gbits = order[o][2];
            if ((gbits & 1) && !(bx[0] < ws)) continue;
            if ((gbits & 2) && !(by[0] < ws)) continue;
            if ((gbits & 4) && !(bx[1] < ws)) continue;
            if ((gbits & 8) && !(by[1] < ws)) continue;
            int q = ty * 4 + tx;
            float Jv = bilinear_cl(J, H, W, lx[tx][tid], ly[ty][tid]);
            float d = (fmaf(Jv, 16384.f, 256.f) / 512.f - fmaf(Ip[tid][q], 16384.f, 256.f) / 512.f) * wt[tid][q];
            e += fabsf(d);
          }
          s1[tid] = e;
        }
        err[gid] = tree64(s1) / (float)(32 * ws * ws);
      }
      U[gid] = (ptx + hw) - (float)j;
      V[gid] = (pty + hw) - (float)i;
    }
}
