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

// Sweep kernel.  CTA tile: 32 columns x 64 rows, 32x8 threads, each thread an 8-row strip
// of one column with a sliding 3x3 window (float32 and double copies), so every u, v value
// is read from shared memory and converted to double once per thread.
// Data movement (one mbarrier, one elected thread): a 3-D TMA copy brings the 8 coefficient
// planes of the tile (32 x 64 x 8 floats = 64 KB) and two 2-D TMA copies the u, v tiles
// with their 1-pixel halo (40 x 66 floats each, x starting 4 floats left of the tile so the
// copy stays 16-byte aligned).  Out-of-image cells (zero-filled by TMA) are replaced by
// their clamped neighbours ('nearest') on tiles that touch the border.
// Arithmetic:
//  - 2-term stencils (D, D^T, F, F^T) in float32 as 0 + w0*a + w1*b: with exact operand
//    halves, one float32 rounding of the exact value equals the reference's double
//    accumulation rounded to float32 (including the sign of zero);
//  - M (4 terms) and H (8 terms) keep the reference's double accumulation order; H uses
//    'constant' 0 outside the image (selected on border tiles).
constexpr int LS_TW = 32, LS_TH = 64, LS_TY = 16, LS_RPT = LS_TH / LS_TY, LS_THREADS = LS_TW * LS_TY;
constexpr int LS_UW = LS_TW + 8, LS_UH = LS_TH + 2;  // u/v tile: x from x0-4, y from y0-1
constexpr int LS_COEF_BYTES = 8 * LS_TW * LS_TH * 4, LS_UV_BYTES = LS_UW * LS_UH * 4;
constexpr int LS_UV_STRIDE = (LS_UV_BYTES + 127) / 128 * 128;  // keeps every TMA destination 128-byte aligned
constexpr int LS_STAGE = LS_COEF_BYTES + 2 * LS_UV_STRIDE;               // one tile: coefficients + u + v
constexpr size_t LS_SMEM = 2 * LS_STAGE + 128 + 128;  // two stages + barriers + alignment slack
constexpr long long LS_WAIT_LIMIT = 1ll << 22;

__device__ __forceinline__ float st2(float a, float b, float wa, float wb) {
  return __fadd_rn(__fadd_rn(0.0f, __fmul_rn(a, wa)), __fmul_rn(b, wb));
}
__device__ __forceinline__ float st_m(const double d[3][3]) {
  double t = __dadd_rn(0.0, __dmul_rn(d[0][0], 0.25));
  t = __dadd_rn(t, __dmul_rn(d[0][2], -0.25));
  t = __dadd_rn(t, __dmul_rn(d[2][0], -0.25));
  t = __dadd_rn(t, __dmul_rn(d[2][2], 0.25));
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

template <bool EDGE>
__device__ __forceinline__ void ls_strip(const float (*su)[LS_UW], const float (*sv)[LS_UW],
                                         const float (*sc)[LS_TH][LS_TW], float* __restrict__ un,
                                         float* __restrict__ vn, int H, int W, int pitch, float h, int x, int y0,
                                         int r0, int tx, double& du2, double& dv2) {
  const int c = tx + 4;  // tile column of x
  float fu[3][3], fv[3][3];
  double du[3][3], dv[3][3];
#pragma unroll
  for (int r = 0; r < 2; r++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      fu[r + 1][j] = su[r0 + r][c - 1 + j];
      fv[r + 1][j] = sv[r0 + r][c - 1 + j];
      du[r + 1][j] = (double)fu[r + 1][j];
      dv[r + 1][j] = (double)fv[r + 1][j];
    }
#pragma unroll
  for (int r = 0; r < LS_RPT; r++) {
#pragma unroll
    for (int j = 0; j < 3; j++) {
      fu[0][j] = fu[1][j]; fu[1][j] = fu[2][j];
      fv[0][j] = fv[1][j]; fv[1][j] = fv[2][j];
      du[0][j] = du[1][j]; du[1][j] = du[2][j];
      dv[0][j] = dv[1][j]; dv[1][j] = dv[2][j];
      fu[2][j] = su[r0 + r + 2][c - 1 + j];
      fv[2][j] = sv[r0 + r + 2][c - 1 + j];
      du[2][j] = (double)fu[2][j];
      dv[2][j] = (double)fv[2][j];
    }
    const int y = y0 + r;
    if (y >= H || x >= W) continue;
    const int ly = r0 + r;
    const bool T = y == 0, B = y == H - 1, L = x == 0, R = x == W - 1;
    const float a = sc[0][ly][tx], b = sc[1][ly][tx], cc = sc[2][ly][tx];
    float Du = st2(fu[0][1], fu[2][1], -0.5f, 0.5f), DTu = st2(fu[1][0], fu[1][2], -0.5f, 0.5f);
    float Dv = st2(fv[0][1], fv[2][1], -0.5f, 0.5f), DTv = st2(fv[1][0], fv[1][2], -0.5f, 0.5f);
    float Fu = st2(fu[0][1], fu[2][1], 1.0f, 1.0f), FTv = st2(fv[1][0], fv[1][2], 1.0f, 1.0f);
    float Mu = st_m(du), Mv = st_m(dv);
    float Hu = st_h<EDGE>(du, T, B, L, R), Hv = st_h<EDGE>(dv, T, B, L, R);
    float bu = __fmul_rn(__fmul_rn(2.0f, a), Du);
    bu = __fadd_rn(bu, __fmul_rn(a, DTv));
    bu = __fadd_rn(bu, __fmul_rn(b, Dv));
    bu = __fadd_rn(bu, __fmul_rn(cc, Fu));
    bu = __fadd_rn(bu, __fmul_rn(cc, Mv));
    bu = __fadd_rn(bu, __fmul_rn(h, Hu));
    bu = __fadd_rn(bu, sc[3][ly][tx]);
    float bv = __fmul_rn(b, Du);
    bv = __fadd_rn(bv, __fmul_rn(a, DTu));
    bv = __fadd_rn(bv, __fmul_rn(__fmul_rn(2.0f, b), DTv));
    bv = __fadd_rn(bv, __fmul_rn(cc, Mu));
    bv = __fadd_rn(bv, __fmul_rn(cc, FTv));
    bv = __fadd_rn(bv, __fmul_rn(h, Hv));
    bv = __fadd_rn(bv, sc[4][ly][tx]);
    const float B11 = sc[5][ly][tx], B12 = sc[6][ly][tx], B22 = sc[7][ly][tx];
    float nu = -__fadd_rn(__fmul_rn(B11, bu), __fmul_rn(B12, bv));
    float nv = -__fadd_rn(__fmul_rn(B12, bu), __fmul_rn(B22, bv));
    const size_t i = (size_t)y * pitch + x;
    un[i] = nu;
    vn[i] = nv;
    // squared change for the stop rule, in double
    double eu = __dadd_rn((double)nu, -du[1][1]), ev = __dadd_rn((double)nv, -dv[1][1]);
    du2 = __fma_rn(eu, eu, du2);
    dv2 = __fma_rn(ev, ev, dv2);
  }
}

// One sweep, persistent: gridDim.x CTAs (one per SM) walk the tiles with a two-stage TMA
// pipeline - while a tile is computed the next one is already in flight into the other
// stage.  `err_flag` receives 1 if a TMA wait times out (the CTA then stops early).
struct LsStage {
  float (*sc)[LS_TH][LS_TW];
  float (*su)[LS_UW];
  float (*sv)[LS_UW];
};

__device__ __forceinline__ LsStage ls_stage(unsigned char* base, int s) {
  unsigned char* p = base + s * LS_STAGE;
  return {reinterpret_cast<float(*)[LS_TH][LS_TW]>(p), reinterpret_cast<float(*)[LS_UW]>(p + LS_COEF_BYTES),
          reinterpret_cast<float(*)[LS_UW]>(p + LS_COEF_BYTES + LS_UV_STRIDE)};
}

__device__ __forceinline__ void ls_issue(const LsStage& S, uint64_t* bar, const CUtensorMap* tc, const CUtensorMap* tu,
                                         const CUtensorMap* tv, int x0, int y0) {
  mbar_expect_tx(bar, LS_COEF_BYTES + 2 * LS_UV_BYTES);
  tma_load_3d(S.sc, tc, x0, y0, 0, bar);
  tma_load_2d(S.su, tu, x0 - 4, y0 - 1, bar);
  tma_load_2d(S.sv, tv, x0 - 4, y0 - 1, bar);
}

__global__ void __launch_bounds__(LS_THREADS, 1) ls_sweep_kernel(const __grid_constant__ CUtensorMap tm_coef,
                                                                 const __grid_constant__ CUtensorMap tm_u,
                                                                 const __grid_constant__ CUtensorMap tm_v,
                                                                 float* __restrict__ un, float* __restrict__ vn, int H,
                                                                 int W, int pitch, float h, double* ss, int* run,
                                                                 unsigned int* done, int k, double inv_n, double tol,
                                                                 int* err_flag) {
  if (k > 0 && *(volatile int*)(run + k) == 0) return;  // the stop rule ended the loop earlier
  extern __shared__ __align__(128) unsigned char ls_smem_raw[];
  unsigned char* base = ls_smem_raw + ((128 - (smem_u32(ls_smem_raw) & 127)) & 127);
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + 2 * LS_STAGE);
  const int tilesx = (W + LS_TW - 1) / LS_TW, ntiles = tilesx * ((H + LS_TH - 1) / LS_TH);
  const int t = threadIdx.y * blockDim.x + threadIdx.x;
  if (t == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
  }
  __syncthreads();
  int tile = blockIdx.x;
  if (t == 0 && tile < ntiles) ls_issue(ls_stage(base, 0), &bar[0], &tm_coef, &tm_u, &tm_v, (tile % tilesx) * LS_TW,
                                        (tile / tilesx) * LS_TH);
  double du2 = 0.0, dv2 = 0.0;
  for (int i = 0; tile < ntiles; i++, tile += gridDim.x) {
    const int s = i & 1;
    const int next = tile + gridDim.x;
    if (t == 0 && next < ntiles)  // the other stage was released by the barrier that ended iteration i-1
      ls_issue(ls_stage(base, s ^ 1), &bar[s ^ 1], &tm_coef, &tm_u, &tm_v, (next % tilesx) * LS_TW,
               (next / tilesx) * LS_TH);
    const LsStage S = ls_stage(base, s);
    if (!mbar_wait(&bar[s], (i >> 1) & 1, LS_WAIT_LIMIT)) {
      if (t == 0) atomicExch(err_flag, 1);
      mbar_wait(&bar[s], (i >> 1) & 1, LS_WAIT_LIMIT);  // one more bounded wait for the copies in flight
      if (next < ntiles) mbar_wait(&bar[s ^ 1], ((i + 1) >> 1) & 1, LS_WAIT_LIMIT);
      break;
    }
    const int x0 = (tile % tilesx) * LS_TW, y0 = (tile / tilesx) * LS_TH;
    const bool edge = x0 == 0 || y0 == 0 || x0 + LS_TW >= W || y0 + LS_TH >= H;
    if (edge) {
      // out-of-image cells of the u/v halo tiles take their clamped ('nearest') value
      for (int e = t; e < LS_UH * LS_UW; e += LS_THREADS) {
        int r = e / LS_UW, cl = e - r * LS_UW;
        int gy = y0 - 1 + r, gx = x0 - 4 + cl;
        if (gy >= 0 && gy < H && gx >= 0 && gx < W) continue;
        int cy = clampi(gy, 0, H - 1) - (y0 - 1), cx = clampi(gx, 0, W - 1) - (x0 - 4);
        if (cy < 0 || cy >= LS_UH || cx < 0 || cx >= LS_UW) continue;  // cell outside every stencil
        S.su[r][cl] = S.su[cy][cx];
        S.sv[r][cl] = S.sv[cy][cx];
      }
      __syncthreads();
    }
    const int x = x0 + threadIdx.x, r0 = threadIdx.y * LS_RPT, ys = y0 + r0;
    if (edge)
      ls_strip<true>(S.su, S.sv, S.sc, un, vn, H, W, pitch, h, x, ys, r0, threadIdx.x, du2, dv2);
    else
      ls_strip<false>(S.su, S.sv, S.sc, un, vn, H, W, pitch, h, x, ys, r0, threadIdx.x, du2, dv2);
    __syncthreads();  // stage s is free for the load issued at iteration i+1
  }
  for (int o = 16; o > 0; o >>= 1) {
    du2 += __shfl_down_sync(0xffffffffu, du2, o);
    dv2 += __shfl_down_sync(0xffffffffu, dv2, o);
  }
  __shared__ double ru[LS_THREADS / 32], rv[LS_THREADS / 32];
  if ((t & 31) == 0) {
    ru[t >> 5] = du2;
    rv[t >> 5] = dv2;
  }
  __syncthreads();
  if (t == 0) {
    for (int w = 1; w < LS_THREADS / 32; w++) {
      du2 += ru[w];
      dv2 += rv[w];
    }
    atomicAdd(ss + 2 * k, du2);
    atomicAdd(ss + 2 * k + 1, dv2);
    __threadfence();
    if (atomicAdd(done + k, 1u) == gridDim.x - 1) {  // last CTA of this sweep decides the next one
      __threadfence();
      double s0 = atomicAdd(ss + 2 * k, 0.0), s1 = atomicAdd(ss + 2 * k + 1, 0.0);
      double e = (sqrt(s0) + sqrt(s1)) * inv_n;
      run[k + 1] = (e > tol) ? 1 : 0;
    }
  }
}

__global__ void ls_count_kernel(LsCtrl* ctrl, const int* run, const double* ss, int maxnum, double inv_n,
                                const int* err_flag, int* iters_out, double* err_out) {
  int K = maxnum;
  for (int k = 1; k < maxnum; k++)
    if (!run[k]) {
      K = k;
      break;
    }
  ctrl->K = K;
  bool failed = *err_flag != 0;
  if (iters_out) *iters_out = failed ? -1 : K;
  if (err_out) *err_out = failed ? __longlong_as_double(0x7ff8000000000000ll) : (K > 0 ? ls_err(ss, K - 1, inv_n) : 0.0);
}

// Result of the last sweep (buffer K mod 2) -> caller's V (row component) and U.
__global__ void ls_finalize_kernel(const float* __restrict__ u0, const float* __restrict__ v0,
                                   const float* __restrict__ u1, const float* __restrict__ v1, float* __restrict__ V,
                                   float* __restrict__ U, int W, int sp, int dp, const LsCtrl* ctrl) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W) return;
  const bool odd = ctrl->K & 1;
  size_t i = (size_t)y * sp + x, o = (size_t)y * dp + x;
  V[o] = odd ? u1[i] : u0[i];
  U[o] = odd ? v1[i] : v0[i];
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
  const int P = ls_pitch(W);
  const size_t N = (size_t)H * P;
  Carver c(workspace, workspace_bytes);
  float* nrm = c.take<float>(3 * N);
  float* coef = c.take<float>(8 * N);
  float* uv = c.take<float>(4 * N);
  LsCtrl* ctrl = c.take<LsCtrl>(1);
  int* run = c.take<int>((size_t)maxnum + 2);
  unsigned int* done = c.take<unsigned int>((size_t)maxnum + 1);
  double* ss = c.take<double>(2 * (size_t)(maxnum > 0 ? maxnum : 1));
  int* err_flag = run + maxnum + 1;
  float *n1 = nrm, *n2 = nrm + N, *et = nrm + 2 * N;
  float* ub[2] = {uv, uv + 2 * N};
  float* vb[2] = {uv + N, uv + 3 * N};
  // tensor maps: 8 coefficient planes (3-D) and the four u / v planes (2-D)
  CUtensorMap tm_coef, tm_u[2], tm_v[2];
  {
    uint64_t d3[3] = {(uint64_t)W, (uint64_t)H, 8}, s3[2] = {(uint64_t)P * 4, (uint64_t)N * 4};
    uint32_t b3[3] = {LS_TW, LS_TH, 8};
    int rc = tmap_f32(&tm_coef, coef, 3, d3, s3, b3);
    if (rc) return rc;
    uint64_t d2[2] = {(uint64_t)W, (uint64_t)H}, s2[1] = {(uint64_t)P * 4};
    uint32_t b2[2] = {LS_UW, LS_UH};
    for (int q = 0; q < 2; q++) {
      if ((rc = tmap_f32(&tm_u[q], ub[q], 2, d2, s2, b2))) return rc;
      if ((rc = tmap_f32(&tm_v[q], vb[q], 2, d2, s2, b2))) return rc;
    }
  }
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(ls_sweep_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LS_SMEM);
    attr = true;
  }
  // control block, flags, counters and sums are contiguous: one memset clears them
  cudaMemsetAsync(ctrl, 0, (size_t)((char*)(ss + 2 * (size_t)(maxnum > 0 ? maxnum : 1)) - (char*)ctrl), st);
  dim3 mg((W + 255) / 256 < 8 ? (W + 255) / 256 : 8, H < 512 ? H : 512);
  ls_max_kernel<<<mg, 256, 0, st>>>(I0, I1, H, W, pitch, ctrl->maxkey);
  dim3 rg((W + 255) / 256, H);
  ls_normalize_kernel<<<rg, 256, 0, st>>>(I0, I1, ctrl->maxkey, n1, n2, et, W, pitch, P);
  dim3 blk(32, 8), grd((W + 31) / 32, (H + 7) / 8);
  ls_coef_kernel<<<grd, blk, 0, st>>>(n1, et, coef, N, H, W, P, h);
  ls_copy2_kernel<<<rg, 256, 0, st>>>(V, U, ub[0], vb[0], W, pitch, P, nullptr);
  double inv_n = 1.0 / ((double)H * (double)W);
  int ntiles = ((W + LS_TW - 1) / LS_TW) * ((H + LS_TH - 1) / LS_TH);
  int sgrd = ntiles < kNumSMs ? ntiles : kNumSMs;
  dim3 sblk(LS_TW, LS_TY);
  for (int k = 0; k < maxnum; k++) {
    int s = k & 1;
    ls_sweep_kernel<<<sgrd, sblk, LS_SMEM, st>>>(tm_coef, tm_u[s], tm_v[s], ub[s ^ 1], vb[s ^ 1], H, W, P, h, ss, run,
                                                done, k, inv_n, tol, err_flag);
  }
  ls_count_kernel<<<1, 1, 0, st>>>(ctrl, run, ss, maxnum, inv_n, err_flag, iters_out, err_out);
  ls_finalize_kernel<<<rg, 256, 0, st>>>(ub[0], vb[0], ub[1], vb[1], V, U, W, P, pitch, ctrl);
  return check_launch("of_ls_solve", 6 + (long long)maxnum);
}
