// A6/A7 Horn-Schunck (src/HornSchunck.py:28-126), bit-exact with the reference.
//
// Derivatives: the 2x2 correlations of computeDerivatives(frame1, frame0) with scipy's
// 'mirror' border, each accumulated in double over the non-zero weights in C order and
// rounded to float32.  Sweep: the 3x3 averaging kernel (weights float32(1/12),
// float32(1/6)) accumulated the same way, then HS_helper2's float32 update.
// Layout: U, V, fx, fy, ft are H x W float32 planes with a shared pitch.  A sweep reads
// 3 coefficient planes and the two 3x3 neighbourhoods (served by L1) and writes U, V:
// 28 B per pixel of HBM/L2 traffic.
#include "common.cuh"
#include "hsweep.cuh"

namespace ofb {

__device__ __forceinline__ double dacc(double a, float v, double w) { return __dadd_rn(a, __dmul_rn((double)v, w)); }

__global__ void hs_deriv_kernel(const float* __restrict__ f0, const float* __restrict__ f1, float* __restrict__ fx,
                                float* __restrict__ fy, float* __restrict__ ft, int H, int W, int pitch) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  int y1 = mirror1(y + 1, H), x1 = mirror1(x + 1, W);
  size_t i00 = (size_t)y * pitch + x, i01 = (size_t)y * pitch + x1, i10 = (size_t)y1 * pitch + x, i11 = (size_t)y1 * pitch + x1;
  float a00 = f1[i00], a01 = f1[i01], a10 = f1[i10], a11 = f1[i11];  // frame t1
  float b00 = f0[i00], b01 = f0[i01], b10 = f0[i10], b11 = f0[i11];  // frame t0
  // kernelX flipped: +.25 -.25 / +.25 -.25 ; kernelY flipped: +.25 +.25 / -.25 -.25
  double t;
  t = dacc(dacc(dacc(dacc(0.0, a00, 0.25), a01, -0.25), a10, 0.25), a11, -0.25);
  float gx1 = (float)t;
  t = dacc(dacc(dacc(dacc(0.0, b00, 0.25), b01, -0.25), b10, 0.25), b11, -0.25);
  float gx0 = (float)t;
  t = dacc(dacc(dacc(dacc(0.0, a00, 0.25), a01, 0.25), a10, -0.25), a11, -0.25);
  float gy1 = (float)t;
  t = dacc(dacc(dacc(dacc(0.0, b00, 0.25), b01, 0.25), b10, -0.25), b11, -0.25);
  float gy0 = (float)t;
  t = dacc(dacc(dacc(dacc(0.0, b00, 0.25), b01, 0.25), b10, 0.25), b11, 0.25);
  float gt0 = (float)t;
  t = dacc(dacc(dacc(dacc(0.0, a00, -0.25), a01, -0.25), a10, -0.25), a11, -0.25);
  float gt1 = (float)t;
  fx[i00] = __fadd_rn(gx1, gx0);
  fy[i00] = __fadd_rn(gy1, gy0);
  ft[i00] = __fadd_rn(gt0, gt1);
}

__global__ void hs_sweep_kernel(const float* __restrict__ fx, const float* __restrict__ fy,
                                const float* __restrict__ ft, const float* __restrict__ U, const float* __restrict__ V,
                                float* __restrict__ Un, float* __restrict__ Vn, int H, int W, int pitch, float a2) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  const double wc = (double)(1.0f / 12.0f), we = (double)(1.0f / 6.0f);
  int ym = mirror1(y - 1, H), yp = mirror1(y + 1, H), xm = mirror1(x - 1, W), xp = mirror1(x + 1, W);
  const size_t rm = (size_t)ym * pitch, r0 = (size_t)y * pitch, rp = (size_t)yp * pitch;
  double su = 0.0, sv = 0.0;
  su = dacc(su, U[rm + xm], wc); sv = dacc(sv, V[rm + xm], wc);
  su = dacc(su, U[rm + x], we);  sv = dacc(sv, V[rm + x], we);
  su = dacc(su, U[rm + xp], wc); sv = dacc(sv, V[rm + xp], wc);
  su = dacc(su, U[r0 + xm], we); sv = dacc(sv, V[r0 + xm], we);
  su = dacc(su, U[r0 + xp], we); sv = dacc(sv, V[r0 + xp], we);
  su = dacc(su, U[rp + xm], wc); sv = dacc(sv, V[rp + xm], wc);
  su = dacc(su, U[rp + x], we);  sv = dacc(sv, V[rp + x], we);
  su = dacc(su, U[rp + xp], wc); sv = dacc(sv, V[rp + xp], wc);
  float ua = (float)su, va = (float)sv;
  size_t i = r0 + x;
  float gx = fx[i], gy = fy[i];
  float num = __fadd_rn(__fadd_rn(__fmul_rn(gx, ua), __fmul_rn(gy, va)), ft[i]);
  float den = __fadd_rn(__fadd_rn(a2, __fmul_rn(gx, gx)), __fmul_rn(gy, gy));
  float der = __fdiv_rn(num, den);
  Un[i] = __fsub_rn(ua, __fmul_rn(gx, der));
  Vn[i] = __fsub_rn(va, __fmul_rn(gy, der));
}

// Temporally blocked sweeps: one pass runs up to HB_T sweeps on a tile held in shared
// memory, so the three derivative planes and (U, V) cross HBM/L2 once per HB_T sweeps
// instead of once per sweep.  A CTA owns 56 x 32 pixels and stages a 64 x 40 region (halo
// HB_T): sweep s computes the cells at least s + 1 from the region's edge, which after
// HB_T sweeps leaves exactly the owned pixels exact; they are written back.  On image
// borders every neighbour index goes through the same 'mirror' map as hs_sweep_kernel
// (mapped neighbours stay within one row / column of their cell, so inside the region),
// and out-of-image cells are neither computed nor read.  Each cell's arithmetic is
// hs_sweep_kernel's: the averaging weights are float32 values (24-bit mantissas), so every
// product with a float32 sample is exact in double and fma(v, w, acc) rounds exactly as
// the separate multiply and add.  U and V sit in shared memory as float64 copies of their
// float32 values, so the float64 sums read their operands without a conversion each.
constexpr int HB_T = 4, HB_TW = 56, HB_TH = 32, HB_RW = HB_TW + 2 * HB_T, HB_RH = HB_TH + 2 * HB_T;  // 64 x 40
constexpr int HB_PL = HB_RW * HB_RH;
constexpr size_t HB_SMEM = 3 * (size_t)HB_PL * sizeof(float) + 4 * (size_t)HB_PL * sizeof(double);  // 110 KB

__global__ void __launch_bounds__(HQ_THREADS, 2) hs_pass_kernel(const float* __restrict__ fx, const float* __restrict__ fy,
                                                      const float* __restrict__ ft, const float* __restrict__ U,
                                                      const float* __restrict__ V, float* __restrict__ Un,
                                                      float* __restrict__ Vn, int H, int W, int pitch, float a2,
                                                      int nsw) {
  extern __shared__ float hb_sm[];
  float* sfx = hb_sm;
  float* sfy = sfx + HB_PL;
  float* sft = sfy + HB_PL;
  // ping-pong buffer q (float64): u at plane 2q after the float planes, v right after it
  double* const hb_uv = reinterpret_cast<double*>(sft + HB_PL);
#define HB_U(q) (hb_uv + (2 * (q)) * HB_PL)
#define HB_V(q) (hb_uv + (1 + 2 * (q)) * HB_PL)
  const int x0 = blockIdx.x * HB_TW, y0 = blockIdx.y * HB_TH;
  for (int k = threadIdx.x; k < HB_PL; k += HQ_THREADS) {
    const int r = k / HB_RW, c = k - r * HB_RW;
    const int gy = y0 - HB_T + r, gx = x0 - HB_T + c;
    if (gy < 0 || gy >= H || gx < 0 || gx >= W) continue;  // never read
    const size_t i = (size_t)gy * pitch + gx;
    sfx[k] = fx[i];
    sfy[k] = fy[i];
    sft[k] = ft[i];
    HB_U(0)[k] = U[i];
    HB_V(0)[k] = V[i];
  }
  __syncthreads();
  const bool edge = x0 < HB_T || y0 < HB_T || x0 + HB_TW + HB_T > W || y0 + HB_TH + HB_T > H;
#pragma unroll 1
  for (int s = 0; s < nsw; s++) {
    const int q = s & 1;
    if (edge)
      hq_sweep2<HB_RW, HB_RH, HB_T, true, false, HQ_THREADS, false>(sfx, sfy, sft, nullptr, HB_U(q), HB_V(q),
                                                                   HB_U(q ^ 1), HB_V(q ^ 1), s, x0, y0, H, W, a2);
    else
      hq_sweep2<HB_RW, HB_RH, HB_T, false, false, HQ_THREADS, false>(sfx, sfy, sft, nullptr, HB_U(q), HB_V(q),
                                                                    HB_U(q ^ 1), HB_V(q ^ 1), s, x0, y0, H, W, a2);
    __syncthreads();
  }
  const double* fu = HB_U(nsw & 1);
  const double* fv = HB_V(nsw & 1);
  for (int k = threadIdx.x; k < HB_TW * HB_TH; k += HQ_THREADS) {
    const int r = k / HB_TW, c = k - r * HB_TW;
    const int y = y0 + r, x = x0 + c;
    if (y >= H || x >= W) continue;
    const int o = (r + HB_T) * HB_RW + c + HB_T;
    Un[(size_t)y * pitch + x] = (float)fu[o];
    Vn[(size_t)y * pitch + x] = (float)fv[o];
  }
#undef HB_U
#undef HB_V
}

__global__ void copy2_kernel(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ ao,
                             float* __restrict__ bo, int W, int pitch) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x < W) {
    size_t i = (size_t)y * pitch + x;
    ao[i] = a[i];
    bo[i] = b[i];
  }
}

// sum of squared differences of two plane pairs into acc[0], acc[1] (double atomics)
__global__ void sqdiff2_kernel(const float* __restrict__ a, const float* __restrict__ a0, const float* __restrict__ b,
                               const float* __restrict__ b0, int H, int W, int pitch, double* acc) {
  double sa = 0.0, sb = 0.0;
  for (int y = blockIdx.y; y < H; y += gridDim.y)
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x) {
      size_t i = (size_t)y * pitch + x;
      double da = (double)a[i] - (double)a0[i], db = (double)b[i] - (double)b0[i];
      sa += da * da;
      sb += db * db;
    }
  for (int o = 16; o > 0; o >>= 1) {
    sa += __shfl_down_sync(0xffffffffu, sa, o);
    sb += __shfl_down_sync(0xffffffffu, sb, o);
  }
  __shared__ double ra[32], rb[32];
  int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { ra[w] = sa; rb[w] = sb; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); k++) { sa += ra[k]; sb += rb[k]; }
    atomicAdd(acc, sa);
    atomicAdd(acc + 1, sb);
  }
}

// status (optional): a persistent solve's status word; a solve whose bounded waits gave up
// reports a NaN error
__global__ void hs_err_kernel(const double* acc, double n, double* err_out, const int* status) {
  const bool failed = status && (*status & OF_ST_WAIT_TIMEOUT);
  *err_out = failed ? __longlong_as_double(0x7ff8000000000000ll) : (sqrt(acc[0]) + sqrt(acc[1])) / n;
}

}  // namespace ofb

using namespace ofb;

extern "C" int of_hs_derivatives(const float* I0, const float* I1, float* fx, float* fy, float* ft, int H, int W,
                                 int pitch, void* stream) {
  OF_REQUIRE(!bad_plane(I0, H, W, pitch) && I1 && fx && fy && ft, "of_hs_derivatives: bad plane");
  dim3 blk(32, 8), grd((W + 31) / 32, (H + 7) / 8);
  hs_deriv_kernel<<<grd, blk, 0, as_stream(stream)>>>(I0, I1, fx, fy, ft, H, W, pitch);
  return check_launch("of_hs_derivatives");
}

// of_hs_solve_persistent: one pair through the persistent kernels of hsq.cu (of_hs_batch,
// automatic schedule: the resident schedule when all the launch's CTAs run at once, else the
// device work queue, whose items only wait for items of running CTAs, so it is correct
// beside any other work on the GPU, if slower there).
constexpr int kHsSolveShape = 3;  // of_hs_batch tile shape for one pair: 32 x 32 regions, 8 sweeps per pass

static size_t hs_persistent_ws(int H, int W, int pitch) {
  OfHsBatchPair q = {nullptr, nullptr, nullptr, nullptr, H, W, pitch, 0.f, 1};
  return of_hs_batch_workspace_size(&q, 1);
}

// Covers both of_hs_solve and of_hs_solve_persistent.
extern "C" size_t of_hs_workspace_size(int H, int W, int pitch) {
  size_t N = (size_t)H * pitch;
  Sizer s;  // of_hs_solve
  for (int i = 0; i < 7; i++) s.take<float>(N);
  s.take<double>(2);
  Sizer q;  // of_hs_solve_persistent: initial flow (for the error), sums, status, batch workspace
  q.take<float>(2 * N);
  q.take<double>(2);
  q.take<int>(1);
  q.take<unsigned char>(hs_persistent_ws(H, W, pitch));
  return s.off > q.off ? s.off : q.off;
}

extern "C" int of_hs_solve(const float* I0, const float* I1, float* U, float* V, int H, int W, int pitch, float alpha,
                           int niter, double* err_out, void* workspace, size_t workspace_bytes, void* stream) {
  OF_REQUIRE(!bad_plane(I0, H, W, pitch) && I1 && U && V, "of_hs_solve: bad plane");
  OF_REQUIRE(niter >= 0, "of_hs_solve: niter < 0");
  if (!workspace || workspace_bytes < of_hs_workspace_size(H, W, pitch))
    return set_error(OF_ERR_WORKSPACE, "of_hs_solve: workspace too small (%zu < %zu)", workspace_bytes,
                     of_hs_workspace_size(H, W, pitch));
  cudaStream_t st = as_stream(stream);
  size_t N = (size_t)H * pitch;
  Carver c(workspace, workspace_bytes);
  float *fx = c.take<float>(N), *fy = c.take<float>(N), *ft = c.take<float>(N);
  float *U0 = c.take<float>(N), *V0 = c.take<float>(N), *Ub = c.take<float>(N), *Vb = c.take<float>(N);
  double* acc = c.take<double>(2);
  dim3 blk(32, 8), grd((W + 31) / 32, (H + 7) / 8);
  dim3 rgrid((W + 255) / 256, H);
  hs_deriv_kernel<<<grd, blk, 0, st>>>(I0, I1, fx, fy, ft, H, W, pitch);
  copy2_kernel<<<rgrid, 256, 0, st>>>(U, V, U0, V0, W, pitch);
  float a2 = alpha * alpha;
  if (H >= 16 && W >= 16 && niter > 0) {  // temporally blocked: HB_T sweeps per launch
    cudaError_t e = OF_SMEM_OPT_IN(hs_pass_kernel, HB_SMEM);
    if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_hs_solve: %s", cudaGetErrorString(e));
    const int np = (niter + HB_T - 1) / HB_T;
    dim3 pg((W + HB_TW - 1) / HB_TW, (H + HB_TH - 1) / HB_TH);
    for (int p = 0; p < np; p++) {
      // the last pass writes U, V; earlier ones alternate with Ub, Vb; the first reads U0, V0
      const bool to_uv = ((np - 1 - p) & 1) == 0;
      const float* su = p == 0 ? U0 : (to_uv ? Ub : U);
      const float* sv = p == 0 ? V0 : (to_uv ? Vb : V);
      const int nsw = niter - p * HB_T < HB_T ? niter - p * HB_T : HB_T;
      hs_pass_kernel<<<pg, HQ_THREADS, HB_SMEM, st>>>(fx, fy, ft, su, sv, to_uv ? U : Ub, to_uv ? V : Vb, H, W, pitch, a2,
                                              nsw);
    }
    long long n = 2 + np;
    if (err_out) {
      cudaMemsetAsync(acc, 0, 2 * sizeof(double), st);
      dim3 g2((W + 255) / 256 < 4 ? (W + 255) / 256 : 4, H < 256 ? H : 256);
      sqdiff2_kernel<<<g2, 256, 0, st>>>(U, U0, V, V0, H, W, pitch, acc);
      hs_err_kernel<<<1, 1, 0, st>>>(acc, (double)H * (double)W, err_out, nullptr);
      n += 2;
    }
    return check_launch("of_hs_solve", n);
  }
  for (int k = 0; k < niter; k++) {
    const float *su, *sv;
    float *du, *dv;
    if (k == 0) { su = U0; sv = V0; du = U; dv = V; }
    else if (k & 1) { su = U; sv = V; du = Ub; dv = Vb; }
    else { su = Ub; sv = Vb; du = U; dv = V; }
    hs_sweep_kernel<<<grd, blk, 0, st>>>(fx, fy, ft, su, sv, du, dv, H, W, pitch, a2);
  }
  long long n = 2 + niter;
  if (niter > 0 && ((niter - 1) & 1)) {
    copy2_kernel<<<rgrid, 256, 0, st>>>(Ub, Vb, U, V, W, pitch);
    n += 1;
  }
  if (err_out) {
    cudaMemsetAsync(acc, 0, 2 * sizeof(double), st);
    dim3 g2((W + 255) / 256 < 4 ? (W + 255) / 256 : 4, H < 256 ? H : 256);
    sqdiff2_kernel<<<g2, 256, 0, st>>>(U, U0, V, V0, H, W, pitch, acc);
    hs_err_kernel<<<1, 1, 0, st>>>(acc, (double)H * (double)W, err_out, nullptr);
    n += 2;
  }
  return check_launch("of_hs_solve", n);
}

extern "C" int of_hs_solve_persistent(const float* I0, const float* I1, float* U, float* V, int H, int W, int pitch,
                                      float alpha, int niter, double* err_out, void* workspace, size_t workspace_bytes,
                                      void* stream) {
  OF_REQUIRE(!bad_plane(I0, H, W, pitch) && I1 && U && V, "of_hs_solve_persistent: bad plane");
  OF_REQUIRE(niter >= 0, "of_hs_solve_persistent: niter < 0");
  if (!workspace || workspace_bytes < of_hs_workspace_size(H, W, pitch))
    return set_error(OF_ERR_WORKSPACE, "of_hs_solve_persistent: workspace too small (%zu < %zu)", workspace_bytes,
                     of_hs_workspace_size(H, W, pitch));
  cudaStream_t st = as_stream(stream);
  const size_t N = (size_t)H * pitch;
  Carver c(workspace, workspace_bytes);
  float* U0 = c.take<float>(2 * N);
  float* V0 = U0 + N;
  double* acc = c.take<double>(2);
  int* status = c.take<int>(1);
  const size_t bws = hs_persistent_ws(H, W, pitch);
  void* bw = c.take<unsigned char>(bws);
  long long n = 0;
  if (err_out) {
    copy2_kernel<<<dim3((W + 255) / 256, H), 256, 0, st>>>(U, V, U0, V0, W, pitch);
    n++;
  }
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int), st);
  if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_hs_solve_persistent: %s", cudaGetErrorString(e));
  OfHsBatchPair q = {I0, I1, U, V, H, W, pitch, alpha, niter};
  OfTuning tun = {kHsSolveShape, 0, OF_HS_EXACT, OF_HS_SCHED_AUTO};
  const int rc = of_hs_batch(&q, 1, &tun, status, 1ll << 20, bw, bws, stream);
  if (rc != OF_OK) return rc;
  if (err_out) {
    cudaMemsetAsync(acc, 0, 2 * sizeof(double), st);
    dim3 g2((W + 255) / 256 < 4 ? (W + 255) / 256 : 4, H < 256 ? H : 256);
    sqdiff2_kernel<<<g2, 256, 0, st>>>(U, U0, V, V0, H, W, pitch, acc);
    hs_err_kernel<<<1, 1, 0, st>>>(acc, (double)H * (double)W, err_out, status);
    n += 2;
  }
  return check_launch("of_hs_solve_persistent", n);
}
