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
  __shared__ unsigned int ra[8], rb[8];
  if ((threadIdx.x & 31) == 0) {
    ra[threadIdx.x >> 5] = ka;
    rb[threadIdx.x >> 5] = kb;
  }
  __syncthreads();
  if (threadIdx.x == 0) {  // one atomic per block
    for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
      ka = max(ka, ra[w]);
      kb = max(kb, rb[w]);
    }
    atomicMax(keys, ka);
    atomicMax(keys + 1, kb);
  }
}

__global__ void ls_normalize_kernel(const float* __restrict__ a, const float* __restrict__ b,
                                    const unsigned int* __restrict__ keys, float* __restrict__ I1,
                                    float* __restrict__ I2, float* __restrict__ Et, int W, int sp, int dp) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  float ma = key2f(keys[0]), mb = key2f(keys[1]);
  size_t i = (size_t)y * sp + x, o = (size_t)y * dp + x;
  float i1 = __fdiv_rn(a[i], ma), i2 = __fdiv_rn(b[i], mb);
  I1[o] = i1;
  I2[o] = i2;
  Et[o] = __fsub_rn(i2, i1);
}

// (a, b) -> (ao, bo) plane copy between pitches
__global__ void ls_copy2_kernel(const float* __restrict__ a, const float* __restrict__ b, float* __restrict__ ao,
                                float* __restrict__ bo, int W, int sp, int dp, const int* __restrict__ gate) {
  if (gate && !(*gate & 1)) return;
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  size_t i = (size_t)y * sp + x, o = (size_t)y * dp + x;
  ao[o] = a[i];
  bo[o] = b[i];
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

// Stencil helpers of the sweep.
//  - 2-term stencils (D, D^T, F, F^T) in float32 as 0 + w0*a + w1*b: with exact operand
//    halves, one float32 rounding of the exact value equals the reference's double
//    accumulation rounded to float32 (including the sign of zero; double rounding through
//    53 bits is innocuous for a sum of two 24-bit values);
//  - M (4 terms) and H (8 terms) keep the reference's double accumulation order; H uses
//    'constant' 0 outside the image (the EDGE variant selects +0.0 there).
constexpr long long LS_WAIT_LIMIT = 1ll << 22;

// The weights (+-0.5, 1, +-0.25) are powers of two, so every product is exact and an add of
// the product rounds exactly as a fused multiply-add does: each term is one FMA.
__device__ __forceinline__ float st2(float a, float b, float wa, float wb) {
  return __fmaf_rn(b, wb, __fmaf_rn(a, wa, 0.0f));
}
__device__ __forceinline__ float st_m(const double d[3][3]) {
  double t = __fma_rn(d[0][0], 0.25, 0.0);
  t = __fma_rn(d[0][2], -0.25, t);
  t = __fma_rn(d[2][0], -0.25, t);
  t = __fma_rn(d[2][2], 0.25, t);
  return (float)t;
}
template <bool EDGE>
__device__ __forceinline__ float st_h(const double d[3][3], bool T, bool B, bool L, bool R) {
  double t = 0.0;
  t = __dadd_rn(t, (EDGE && (T || L)) ? 0.0 : d[0][0]);
  t = __dadd_rn(t, (EDGE && T) ? 0.0 : d[0][1]);
  t = __dadd_rn(t, (EDGE && (T || R)) ? 0.0 : d[0][2]);
  t = __dadd_rn(t, (EDGE && L) ? 0.0 : d[1][0]);
  t = __dadd_rn(t, (EDGE && R) ? 0.0 : d[1][2]);
  t = __dadd_rn(t, (EDGE && (B || L)) ? 0.0 : d[2][0]);
  t = __dadd_rn(t, (EDGE && B) ? 0.0 : d[2][1]);
  t = __dadd_rn(t, (EDGE && (B || R)) ? 0.0 : d[2][2]);
  return (float)t;
}

// Temporally blocked sweeps: one pass runs up to LB_T sweeps on a tile held in shared
// memory, so the 8 coefficient planes and (u, v) cross HBM/L2 once per LB_T sweeps.
// Tile: 24 x 64 owned pixels plus a 4-pixel halo = a 32 x 72 region, loaded by one 3-D TMA
// (8 coefficient planes, 72 KB) and two 2-D TMAs (u, v) starting at (x0-4, y0-4): x stays
// 16-byte aligned.  Each sweep computes every cell of the region that has its full 3x3
// neighbourhood in the tile; after sweep s only the cells at least s+1 from the region's
// edge are exact, so after LB_T = 4 sweeps exactly the owned 24 x 64 pixels are, and those
// are written back.  Out-of-image cells hold their clamped ('nearest') neighbour and are
// refreshed after every sweep; H uses 'constant' 0 through the border flags.
// The squared change of every sweep is accumulated over owned pixels only, so each pixel is
// counted once per sweep.  The stop rule: the last CTA of a pass finds the first sweep
// whose error is <= tol; if that is not the pass's last sweep, the pass ran too far and the
// rollback launch recomputes the pass from its (unchanged) input with the right count.
constexpr int LB_T = 4, LB_TW = 24, LB_TH = 64, LB_RW = LB_TW + 2 * LB_T, LB_RH = LB_TH + 2 * LB_T;  // 32 x 72
constexpr int LB_PLANE = LB_RW * LB_RH * 4;                  // 9216 B, a multiple of 128
constexpr int LB_COEF_BYTES = 8 * LB_PLANE;
constexpr size_t LB_SMEM = LB_COEF_BYTES + 4 * LB_PLANE + 128 + 128;  // coef + 2 x (u, v) + barrier + slack
constexpr int LB_ROWS = (LB_RH + 7) / 8;                       // rows per thread (9)

typedef float LbPlane[LB_RW];

struct LbPass {  // per-launch description of a pass
  int k0;        // first sweep index
  int nsweep;    // sweeps in this pass (<= LB_T)
  int pass;      // pass index
  int redo;      // 1: rollback launch (sweep count read from redo[pass])
};

__device__ __forceinline__ void lb_refresh(LbPlane* u, LbPlane* v, int x0, int y0, int H, int W, int t) {
  for (int e = t; e < LB_RH * LB_RW; e += 256) {
    int r = e / LB_RW, c = e - r * LB_RW;
    int gy = y0 - LB_T + r, gx = x0 - LB_T + c;
    if (gy >= 0 && gy < H && gx >= 0 && gx < W) continue;
    int sy = clampi(gy, 0, H - 1) - (y0 - LB_T), sx = clampi(gx, 0, W - 1) - (x0 - LB_T);
    if (sy < 0 || sy >= LB_RH || sx < 0 || sx >= LB_RW) continue;
    u[r][c] = u[sy][sx];
    v[r][c] = v[sy][sx];
  }
}

// One row of a thread's 3x3 window: the three u, v values as float32 and float64.
struct LbRow {
  float fu[3], fv[3];
  double du[3], dv[3];
};

__device__ __forceinline__ void lb_load(LbRow& R, const LbPlane* su, const LbPlane* sv, int row, int c) {
#pragma unroll
  for (int j = 0; j < 3; j++) {
    R.fu[j] = su[row][c - 1 + j];
    R.fv[j] = sv[row][c - 1 + j];
    R.du[j] = (double)R.fu[j];
    R.dv[j] = (double)R.fv[j];
  }
}

// Update of the cell (row, c) from its window rows U (above), C (centre), D (below).
template <bool EDGE>
__device__ __forceinline__ void lb_cell(const LbRow& U, const LbRow& C, const LbRow& D, LbPlane* du_, LbPlane* dv_,
                                        const float* sc, int row, int c, int gx, int gy, int H, int W, float h,
                                        bool own, double& acc_u, double& acc_v) {
  if (EDGE && (gy < 0 || gy >= H || gx < 0 || gx >= W)) return;  // refreshed from its clamp source
  const bool T = gy == 0, B = gy == H - 1, L = gx == 0, R = gx == W - 1;
  const double du[3][3] = {{U.du[0], U.du[1], U.du[2]}, {C.du[0], C.du[1], C.du[2]}, {D.du[0], D.du[1], D.du[2]}};
  const double dv[3][3] = {{U.dv[0], U.dv[1], U.dv[2]}, {C.dv[0], C.dv[1], C.dv[2]}, {D.dv[0], D.dv[1], D.dv[2]}};
  const int o = row * LB_RW + c;
  const int PL = LB_RW * LB_RH;
  const float a = sc[o], b = sc[PL + o], cc = sc[2 * PL + o];
  float Du = st2(U.fu[1], D.fu[1], -0.5f, 0.5f), DTu = st2(C.fu[0], C.fu[2], -0.5f, 0.5f);
  float Dv = st2(U.fv[1], D.fv[1], -0.5f, 0.5f), DTv = st2(C.fv[0], C.fv[2], -0.5f, 0.5f);
  float Fu = st2(U.fu[1], D.fu[1], 1.0f, 1.0f), FTv = st2(C.fv[0], C.fv[2], 1.0f, 1.0f);
  float Mu = st_m(du), Mv = st_m(dv);
  float Hu = st_h<EDGE>(du, T, B, L, R), Hv = st_h<EDGE>(dv, T, B, L, R);
  float bu = __fmul_rn(__fmul_rn(2.0f, a), Du);
  bu = __fadd_rn(bu, __fmul_rn(a, DTv));
  bu = __fadd_rn(bu, __fmul_rn(b, Dv));
  bu = __fadd_rn(bu, __fmul_rn(cc, Fu));
  bu = __fadd_rn(bu, __fmul_rn(cc, Mv));
  bu = __fadd_rn(bu, __fmul_rn(h, Hu));
  bu = __fadd_rn(bu, sc[3 * PL + o]);
  float bv = __fmul_rn(b, Du);
  bv = __fadd_rn(bv, __fmul_rn(a, DTu));
  bv = __fadd_rn(bv, __fmul_rn(__fmul_rn(2.0f, b), DTv));
  bv = __fadd_rn(bv, __fmul_rn(cc, Mu));
  bv = __fadd_rn(bv, __fmul_rn(cc, FTv));
  bv = __fadd_rn(bv, __fmul_rn(h, Hv));
  bv = __fadd_rn(bv, sc[4 * PL + o]);
  const float B11 = sc[5 * PL + o], B12 = sc[6 * PL + o], B22 = sc[7 * PL + o];
  float nu = -__fadd_rn(__fmul_rn(B11, bu), __fmul_rn(B12, bv));
  float nv = -__fadd_rn(__fmul_rn(B12, bu), __fmul_rn(B22, bv));
  du_[row][c] = nu;
  dv_[row][c] = nv;
  if (own) {
    double eu = __dadd_rn((double)nu, -C.du[1]), ev = __dadd_rn((double)nv, -C.dv[1]);
    acc_u = __fma_rn(eu, eu, acc_u);
    acc_v = __fma_rn(ev, ev, acc_v);
  }
}

// One sweep of one thread's column strip: rows [r0, r0+n) of column c (1 <= c <= RW-2).
// The three window rows rotate through three register sets (3-row steps), so sliding the
// window costs loads only.
template <bool EDGE>
__device__ __forceinline__ void lb_strip(const LbPlane* su, const LbPlane* sv, LbPlane* du_, LbPlane* dv_,
                                         const float* sc, int c, int r0, int n, int gx, int gy0, int H, int W, float h,
                                         bool own_col, double& acc_u, double& acc_v) {
  LbRow A, B, C;
  lb_load(A, su, sv, r0 - 1, c);
  lb_load(B, su, sv, r0, c);
#define LB_OWN(row) (own_col && (row) >= LB_T && (row) < LB_T + LB_TH)
#pragma unroll 1
  for (int r = 0; r < n; r += 3) {
    const int row = r0 + r;
    lb_load(C, su, sv, row + 1, c);
    lb_cell<EDGE>(A, B, C, du_, dv_, sc, row, c, gx, gy0 + r, H, W, h, LB_OWN(row), acc_u, acc_v);
    if (r + 1 < n) {
      lb_load(A, su, sv, row + 2, c);
      lb_cell<EDGE>(B, C, A, du_, dv_, sc, row + 1, c, gx, gy0 + r + 1, H, W, h, LB_OWN(row + 1), acc_u, acc_v);
    }
    if (r + 2 < n) {
      lb_load(B, su, sv, row + 3, c);
      lb_cell<EDGE>(C, A, B, du_, dv_, sc, row + 2, c, gx, gy0 + r + 2, H, W, h, LB_OWN(row + 2), acc_u, acc_v);
    }
  }
#undef LB_OWN
}

__global__ void __launch_bounds__(256, 2) ls_pass_kernel(const __grid_constant__ CUtensorMap tm_coef,
                                                         const __grid_constant__ CUtensorMap tm_u,
                                                         const __grid_constant__ CUtensorMap tm_v,
                                                         float* __restrict__ un, float* __restrict__ vn, int H, int W,
                                                         int pitch, float h, LbPass P, LsCtrl* ctrl, double* ss,
                                                         int* run, unsigned int* done, int* redo, double inv_n,
                                                         double tol, int* err_flag, int final_buf) {
  int nsw = P.nsweep;
  if (P.redo) {
    nsw = *(volatile int*)(redo + P.pass);
    if (nsw == 0) return;
  } else if (P.k0 > 0 && *(volatile int*)(run + P.k0) == 0) {
    return;  // the stop rule ended the loop in an earlier pass
  }
  extern __shared__ __align__(128) unsigned char lb_smem_raw[];
  unsigned char* base = lb_smem_raw + ((128 - (smem_u32(lb_smem_raw) & 127)) & 127);
  const float* sc = reinterpret_cast<const float*>(base);
  // ping-pong buffer q: u at base + COEF + 2q planes, v right after it
#define LB_U(q) reinterpret_cast<LbPlane*>(base + LB_COEF_BYTES + (2 * (q)) * LB_PLANE)
#define LB_V(q) reinterpret_cast<LbPlane*>(base + LB_COEF_BYTES + (2 * (q) + 1) * LB_PLANE)
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + LB_COEF_BYTES + 4 * LB_PLANE);
  const int x0 = blockIdx.x * LB_TW, y0 = blockIdx.y * LB_TH;
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  if (t == 0) mbar_init(bar, 1);
  __syncthreads();
  if (t == 0) {
    mbar_expect_tx(bar, LB_COEF_BYTES + 2 * LB_PLANE);
    tma_load_3d((void*)sc, &tm_coef, x0 - LB_T, y0 - LB_T, 0, bar);
    tma_load_2d(LB_U(0), &tm_u, x0 - LB_T, y0 - LB_T, bar);
    tma_load_2d(LB_V(0), &tm_v, x0 - LB_T, y0 - LB_T, bar);
  }
  if (!mbar_wait(bar, 0, LS_WAIT_LIMIT)) {
    if (t == 0) atomicExch(err_flag, 1);
    mbar_wait(bar, 0, LS_WAIT_LIMIT);  // one more bounded wait for the copies in flight
    nsw = 0;
  }
  const bool edge = x0 < LB_T || y0 < LB_T || x0 + LB_TW + LB_T > W || y0 + LB_TH + LB_T > H;
  if (edge) {
    __syncthreads();
    lb_refresh(LB_U(0), LB_V(0), x0, y0, H, W, t);
  }
  __syncthreads();
  const int c = threadIdx.x;  // region column
  const int gx = x0 - LB_T + c;
  const bool own_col = c >= LB_T && c < LB_T + LB_TW;
  int r0 = threadIdx.y * LB_ROWS, r1 = r0 + LB_ROWS;
  if (r0 < 1) r0 = 1;
  if (r1 > LB_RH - 1) r1 = LB_RH - 1;
  __shared__ double red[LB_T][2][8];
#pragma unroll 1
  for (int s = 0; s < nsw; s++) {
    const int in = s & 1, out = in ^ 1;
    double au = 0.0, av = 0.0;
    // sweep s only needs the rows at least s + 1 from the region's edge (later sweeps
    // read no others)
    const int ra = r0 > 1 + s ? r0 : 1 + s, rb = r1 < LB_RH - 1 - s ? r1 : LB_RH - 1 - s;
    if (c >= 1 && c <= LB_RW - 2 && rb > ra) {
      if (edge)
        lb_strip<true>(LB_U(in), LB_V(in), LB_U(out), LB_V(out), sc, c, ra, rb - ra, gx, y0 - LB_T + ra, H, W, h,
                       own_col, au, av);
      else
        lb_strip<false>(LB_U(in), LB_V(in), LB_U(out), LB_V(out), sc, c, ra, rb - ra, gx, y0 - LB_T + ra, H, W,
                        h, own_col, au, av);
    }
    if (!P.redo) {
      for (int o = 16; o > 0; o >>= 1) {
        au += __shfl_down_sync(0xffffffffu, au, o);
        av += __shfl_down_sync(0xffffffffu, av, o);
      }
      if ((t & 31) == 0) {
        red[s][0][t >> 5] = au;
        red[s][1][t >> 5] = av;
      }
    }
    __syncthreads();
    if (edge) {
      lb_refresh(LB_U(out), LB_V(out), x0, y0, H, W, t);
      __syncthreads();
    }
  }
  // owned pixels of the last sweep -> global
  if (nsw > 0) {
    const LbPlane* fu = LB_U(nsw & 1);
    const LbPlane* fv = LB_V(nsw & 1);
    for (int e = t; e < LB_TW * LB_TH; e += 256) {
      int r = e / LB_TW, cl = e - r * LB_TW;
      int y = y0 + r, x = x0 + cl;
      if (y < H && x < W) {
        size_t i = (size_t)y * pitch + x;
        un[i] = fu[r + LB_T][cl + LB_T];
        vn[i] = fv[r + LB_T][cl + LB_T];
      }
    }
  }
  if (P.redo) return;
  // per-sweep squared changes -> ss[k0 + s]; the last CTA applies the stop rule
  if (t == 0) {
    for (int s = 0; s < nsw; s++) {
      double a = 0.0, b = 0.0;
      for (int w = 0; w < 8; w++) {
        a += red[s][0][w];
        b += red[s][1][w];
      }
      atomicAdd(ss + 2 * (P.k0 + s), a);
      atomicAdd(ss + 2 * (P.k0 + s) + 1, b);
    }
    __threadfence();
    if (atomicAdd(done + P.pass, 1u) == gridDim.x * gridDim.y - 1) {
      __threadfence();
      int stop = -1;
      for (int s = 0; s < nsw; s++) {
        double s0 = atomicAdd(ss + 2 * (P.k0 + s), 0.0), s1 = atomicAdd(ss + 2 * (P.k0 + s) + 1, 0.0);
        if (!((sqrt(s0) + sqrt(s1)) * inv_n > tol)) {
          stop = s;
          break;
        }
      }
      if (stop < 0) {
        run[P.k0 + nsw] = 1;
        ctrl->K = P.k0 + nsw;
      } else {
        run[P.k0 + nsw] = 0;
        ctrl->K = P.k0 + stop + 1;
        redo[P.pass] = (stop < nsw - 1) ? stop + 1 : 0;
      }
      ctrl->final_buf = final_buf;
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
  s.take<float>(3 * N);  // I1, I2, Et
  s.take<float>(8 * N);  // coefficient planes
  s.take<float>(4 * N);  // u0, v0, u1, v1
  s.take<LsCtrl>(1);
  s.take<int>((size_t)maxnum + 2);  // run[] and the TMA error flag
  s.take<unsigned int>((size_t)maxnum + 1);  // done[] per pass
  s.take<int>((size_t)maxnum + 1);           // redo[] per pass
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
  float *n1 = nrm, *n2 = nrm + N, *et = nrm + 2 * N;
  float* ub[2] = {uv, uv + 2 * N};
  float* vb[2] = {uv + N, uv + 3 * N};
  // tensor maps over the whole solve: the 8 coefficient planes (3-D) and the four u / v
  // planes (2-D), all with the 32 x 72 region box of a pass
  CUtensorMap tm_coef, tm_u[2], tm_v[2];
  {
    uint64_t d3[3] = {(uint64_t)W, (uint64_t)H, 8}, s3[2] = {(uint64_t)P * 4, (uint64_t)N * 4};
    uint32_t b3[3] = {LB_RW, LB_RH, 8};
    int rc = tmap_f32(&tm_coef, coef, 3, d3, s3, b3);
    if (rc) return rc;
    uint64_t d2[2] = {(uint64_t)W, (uint64_t)H}, s2[1] = {(uint64_t)P * 4};
    uint32_t b2[2] = {LB_RW, LB_RH};
    for (int q = 0; q < 2; q++) {
      if ((rc = tmap_f32(&tm_u[q], ub[q], 2, d2, s2, b2))) return rc;
      if ((rc = tmap_f32(&tm_v[q], vb[q], 2, d2, s2, b2))) return rc;
    }
  }
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(ls_pass_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LB_SMEM);
    attr = true;
  }
  // control block, flags, counters, redo counts and sums are contiguous: one memset
  cudaMemsetAsync(ctrl, 0, (size_t)((char*)(ss + 2 * (size_t)(maxnum > 0 ? maxnum : 1)) - (char*)ctrl), st);
  dim3 mg((W + 255) / 256 < 2 ? (W + 255) / 256 : 2, H < 148 ? H : 148);
  ls_max_kernel<<<mg, 256, 0, st>>>(I0, I1, H, W, pitch, ctrl->maxkey);
  dim3 rg((W + 255) / 256, H);
  ls_normalize_kernel<<<rg, 256, 0, st>>>(I0, I1, ctrl->maxkey, n1, n2, et, W, pitch, P);
  dim3 blk(32, 8), grd((W + 31) / 32, (H + 7) / 8);
  ls_coef_kernel<<<grd, blk, 0, st>>>(n1, et, coef, N, H, W, P, h);
  ls_copy2_kernel<<<rg, 256, 0, st>>>(V, U, ub[0], vb[0], W, pitch, P, nullptr);
  double inv_n = 1.0 / ((double)H * (double)W);
  dim3 pgrd((W + LB_TW - 1) / LB_TW, (H + LB_TH - 1) / LB_TH), pblk(32, 8);
  long long nl = 5;
  for (int k0 = 0, p = 0; k0 < maxnum; k0 += LB_T, p++) {
    const int in = p & 1, out = in ^ 1;
    LbPass P0{k0, maxnum - k0 < LB_T ? maxnum - k0 : LB_T, p, 0};
    ls_pass_kernel<<<pgrd, pblk, LB_SMEM, st>>>(tm_coef, tm_u[in], tm_v[in], ub[out], vb[out], H, W, P, h, P0, ctrl, ss,
                                               run, done, redo, inv_n, tol, err_flag, out);
    LbPass P1 = P0;
    P1.redo = 1;  // rollback: recompute this pass with the sweep count the stop rule chose
    ls_pass_kernel<<<pgrd, pblk, LB_SMEM, st>>>(tm_coef, tm_u[in], tm_v[in], ub[out], vb[out], H, W, P, h, P1, ctrl, ss,
                                               run, done, redo, inv_n, tol, err_flag, out);
    nl += 2;
  }
  ls_count_kernel<<<1, 1, 0, st>>>(ctrl, ss, inv_n, err_flag, iters_out, err_out);
  ls_finalize_kernel<<<rg, 256, 0, st>>>(ub[0], vb[0], ub[1], vb[1], V, U, W, P, pitch, ctrl);
  return check_launch("of_ls_solve", nl + 1);
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
  if (e != cudaSuccess || dev < 0 || dev >= 64) {
    *rc = set_error(OF_ERR_CUDA, "of_ls_solve_noalloc: cudaGetDevice failed (%s)", cudaGetErrorString(e));
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
