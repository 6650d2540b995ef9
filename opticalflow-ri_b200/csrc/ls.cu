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
#include "common.cuh"

namespace ofb {

struct LsCtrl {
  unsigned int maxkey[2];
  int K;  // sweeps run, written by ls_count_kernel
  int pad;
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

__global__ void ls_max_kernel(const float* __restrict__ a, const float* __restrict__ b, int H, int W, int pitch,
                              unsigned int* keys) {
  unsigned int ka = 0, kb = 0;
  for (int y = blockIdx.y; y < H; y += gridDim.y)
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x) {
      size_t i = (size_t)y * pitch + x;
      ka = max(ka, f2key(a[i]));
      kb = max(kb, f2key(b[i]));
    }
  for (int o = 16; o > 0; o >>= 1) {
    ka = max(ka, __shfl_down_sync(0xffffffffu, ka, o));
    kb = max(kb, __shfl_down_sync(0xffffffffu, kb, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(keys, ka);
    atomicMax(keys + 1, kb);
  }
}

__global__ void ls_normalize_kernel(const float* __restrict__ a, const float* __restrict__ b,
                                    const unsigned int* __restrict__ keys, float* __restrict__ I1,
                                    float* __restrict__ I2, float* __restrict__ Et, int W, int pitch) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  float ma = key2f(keys[0]), mb = key2f(keys[1]);
  size_t i = (size_t)y * pitch + x;
  float i1 = __fdiv_rn(a[i], ma), i2 = __fdiv_rn(b[i], mb);
  I1[i] = i1;
  I2[i] = i2;
  Et[i] = __fsub_rn(i2, i1);
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

__global__ void ls_coef_kernel(const float* __restrict__ I1, const float* __restrict__ Et, float* __restrict__ coef,
                               size_t plane, int H, int W, int pitch, float h) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= W || y >= H) return;
  Nb3 n, e;
  n.load(I1, y, x, H, W, pitch);
  e.load(Et, y, x, H, W, pitch);
  size_t i = (size_t)y * pitch + x;
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

__device__ __forceinline__ double ls_err(const double* ss, int k, double inv_n) {
  return (sqrt(ss[2 * k]) + sqrt(ss[2 * k + 1])) * inv_n;
}

__global__ void __launch_bounds__(256) ls_sweep_kernel(const float* __restrict__ coef, size_t plane,
                                                       const float* __restrict__ u, const float* __restrict__ v,
                                                       float* __restrict__ un, float* __restrict__ vn, int H, int W,
                                                       int pitch, float h, double* ss, int* run,
                                                       unsigned int* done, int k, double inv_n, double tol) {
  if (k > 0 && *(volatile int*)(run + k) == 0) return;  // the stop rule ended the loop earlier
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  double du2 = 0.0, dv2 = 0.0;
  if (x < W && y < H) {
    Nb3 U, V;
    U.load(u, y, x, H, W, pitch);
    V.load(v, y, x, H, W, pitch);
    size_t i = (size_t)y * pitch + x;
    float a = coef[i], b = coef[plane + i], c = coef[2 * plane + i];
    float Du = U.dy(), DTu = U.dx(), Dv = V.dy(), DTv = V.dx();
    float Fu = U.fy(), FTv = V.fx(), Mu = U.m(), Mv = V.m();
    float Hu = hsum(u, y, x, H, W, pitch), Hv = hsum(v, y, x, H, W, pitch);
    float bu = __fmul_rn(__fmul_rn(2.0f, a), Du);
    bu = __fadd_rn(bu, __fmul_rn(a, DTv));
    bu = __fadd_rn(bu, __fmul_rn(b, Dv));
    bu = __fadd_rn(bu, __fmul_rn(c, Fu));
    bu = __fadd_rn(bu, __fmul_rn(c, Mv));
    bu = __fadd_rn(bu, __fmul_rn(h, Hu));
    bu = __fadd_rn(bu, coef[3 * plane + i]);
    float bv = __fmul_rn(b, Du);
    bv = __fadd_rn(bv, __fmul_rn(a, DTu));
    bv = __fadd_rn(bv, __fmul_rn(__fmul_rn(2.0f, b), DTv));
    bv = __fadd_rn(bv, __fmul_rn(c, Mu));
    bv = __fadd_rn(bv, __fmul_rn(c, FTv));
    bv = __fadd_rn(bv, __fmul_rn(h, Hv));
    bv = __fadd_rn(bv, coef[4 * plane + i]);
    float B11 = coef[5 * plane + i], B12 = coef[6 * plane + i], B22 = coef[7 * plane + i];
    float nu = -__fadd_rn(__fmul_rn(B11, bu), __fmul_rn(B12, bv));
    float nv = -__fadd_rn(__fmul_rn(B12, bu), __fmul_rn(B22, bv));
    un[i] = nu;
    vn[i] = nv;
    double a1 = (double)nu - (double)U.p[1][1], a2 = (double)nv - (double)V.p[1][1];
    du2 = a1 * a1;
    dv2 = a2 * a2;
  }
  for (int o = 16; o > 0; o >>= 1) {
    du2 += __shfl_down_sync(0xffffffffu, du2, o);
    dv2 += __shfl_down_sync(0xffffffffu, dv2, o);
  }
  __shared__ double ru[8], rv[8];
  int t = threadIdx.y * blockDim.x + threadIdx.x;
  if ((t & 31) == 0) {
    ru[t >> 5] = du2;
    rv[t >> 5] = dv2;
  }
  __syncthreads();
  if (t == 0) {
    for (int w = 1; w < 8; w++) {
      du2 += ru[w];
      dv2 += rv[w];
    }
    atomicAdd(ss + 2 * k, du2);
    atomicAdd(ss + 2 * k + 1, dv2);
    __threadfence();
    unsigned int nblk = gridDim.x * gridDim.y;
    if (atomicAdd(done + k, 1u) == nblk - 1) {  // last block of this sweep decides the next one
      __threadfence();
      double s0 = atomicAdd(ss + 2 * k, 0.0), s1 = atomicAdd(ss + 2 * k + 1, 0.0);
      double e = (sqrt(s0) + sqrt(s1)) * inv_n;
      run[k + 1] = (e > tol) ? 1 : 0;
    }
  }
}

__global__ void ls_count_kernel(LsCtrl* ctrl, const int* run, const double* ss, int maxnum, double inv_n,
                                int* iters_out, double* err_out) {
  int K = maxnum;
  for (int k = 1; k < maxnum; k++)
    if (!run[k]) {
      K = k;
      break;
    }
  ctrl->K = K;
  if (iters_out) *iters_out = K;
  if (err_out) *err_out = K > 0 ? ls_err(ss, K - 1, inv_n) : 0.0;
}

// The last sweep wrote the ping-pong buffers when the sweep count is odd.
__global__ void ls_finalize_kernel(const float* __restrict__ bu, const float* __restrict__ bv, float* __restrict__ V,
                                   float* __restrict__ U, int W, int pitch, const LsCtrl* ctrl) {
  if (!(ctrl->K & 1)) return;
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x < W) {
    size_t i = (size_t)y * pitch + x;
    V[i] = bu[i];
    U[i] = bv[i];
  }
}

}  // namespace ofb

using namespace ofb;

extern "C" int of_ls_coefficients(const float* I1n, const float* Et, float* coef, int H, int W, int pitch, float h,
                                  void* stream) {
  OF_REQUIRE(!bad_plane(I1n, H, W, pitch) && Et && coef, "of_ls_coefficients: bad plane");
  dim3 blk(32, 8), grd((W + 31) / 32, (H + 7) / 8);
  ls_coef_kernel<<<grd, blk, 0, as_stream(stream)>>>(I1n, Et, coef, (size_t)H * pitch, H, W, pitch, h);
  return check_launch("of_ls_coefficients");
}

extern "C" size_t of_ls_workspace_size(int H, int W, int pitch, int maxnum) {
  Sizer s;
  size_t N = (size_t)H * pitch;
  s.take<float>(3 * N);  // I1, I2, Et
  s.take<float>(8 * N);  // coefficient planes
  s.take<float>(2 * N);  // ping-pong u, v
  s.take<LsCtrl>(1);
  s.take<int>((size_t)maxnum + 1);
  s.take<unsigned int>((size_t)maxnum + 1);
  s.take<double>(2 * (size_t)(maxnum > 0 ? maxnum : 1));
  return s.off;
}

extern "C" int of_ls_solve(const float* I0, const float* I1, float* U, float* V, int H, int W, int pitch, float h,
                           int maxnum, double tol, int* iters_out, double* err_out, void* workspace,
                           size_t workspace_bytes, void* stream) {
  OF_REQUIRE(!bad_plane(I0, H, W, pitch) && I1 && U && V, "of_ls_solve: bad plane");
  OF_REQUIRE(maxnum >= 0 && maxnum <= 100000, "of_ls_solve: maxnum out of range");
  size_t need = of_ls_workspace_size(H, W, pitch, maxnum);
  if (!workspace || workspace_bytes < need)
    return set_error(OF_ERR_WORKSPACE, "of_ls_solve: workspace too small (%zu < %zu)", workspace_bytes, need);
  cudaStream_t st = as_stream(stream);
  size_t N = (size_t)H * pitch;
  Carver c(workspace, workspace_bytes);
  float* nrm = c.take<float>(3 * N);
  float* coef = c.take<float>(8 * N);
  float* pp = c.take<float>(2 * N);
  LsCtrl* ctrl = c.take<LsCtrl>(1);
  int* run = c.take<int>((size_t)maxnum + 1);
  unsigned int* done = c.take<unsigned int>((size_t)maxnum + 1);
  double* ss = c.take<double>(2 * (size_t)(maxnum > 0 ? maxnum : 1));
  float *n1 = nrm, *n2 = nrm + N, *et = nrm + 2 * N, *bu = pp, *bv = pp + N;
  // control block, flags, counters and sums are contiguous: one memset clears them
  cudaMemsetAsync(ctrl, 0, (size_t)((char*)(ss + 2 * (size_t)(maxnum > 0 ? maxnum : 1)) - (char*)ctrl), st);
  dim3 mg((W + 255) / 256 < 8 ? (W + 255) / 256 : 8, H < 512 ? H : 512);
  ls_max_kernel<<<mg, 256, 0, st>>>(I0, I1, H, W, pitch, ctrl->maxkey);
  dim3 rg((W + 255) / 256, H);
  ls_normalize_kernel<<<rg, 256, 0, st>>>(I0, I1, ctrl->maxkey, n1, n2, et, W, pitch);
  dim3 blk(32, 8), grd((W + 31) / 32, (H + 7) / 8);
  ls_coef_kernel<<<grd, blk, 0, st>>>(n1, et, coef, N, H, W, pitch, h);
  double inv_n = 1.0 / ((double)H * (double)W);
  for (int k = 0; k < maxnum; k++) {
    const float *su = (k & 1) ? bu : V, *sv = (k & 1) ? bv : U;
    float *du = (k & 1) ? V : bu, *dv = (k & 1) ? U : bv;
    ls_sweep_kernel<<<grd, blk, 0, st>>>(coef, N, su, sv, du, dv, H, W, pitch, h, ss, run, done, k, inv_n, tol);
  }
  ls_count_kernel<<<1, 1, 0, st>>>(ctrl, run, ss, maxnum, inv_n, iters_out, err_out);
  ls_finalize_kernel<<<rg, 256, 0, st>>>(bu, bv, V, U, W, pitch, ctrl);
  return check_launch("of_ls_solve", 5 + (long long)maxnum);
}
