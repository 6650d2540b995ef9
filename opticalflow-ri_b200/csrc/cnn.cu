// Kernels of the learned warm start for Liu-Shen: a small encoder-decoder CNN over
// bfloat16 NHWC activations with float32 accumulation.
//
//  of_cnn_conv3x3   3x3 convolution, zero padding, as an implicit GEMM on the 5th-gen
//                   tensor cores: M = 128 output pixels (a bh x bw patch of one image, or
//                   nb whole images when an image has fewer than 128 pixels),
//                   N = output channels (<= 256 per CTA), K = 9 taps x input channels.
//                   Warp 0 streams A (the input patch shifted by the tap; TMA fills the
//                   zero padding) and B (the tap's weights) into a 4-stage shared-memory
//                   ring; one thread of warp 1 issues tcgen05.mma into a TMEM accumulator;
//                   warps 2-5 read TMEM back (one pixel per thread) and apply bias, ReLU
//                   and the bf16 / f32 store, into a channel slice of a wider tensor when
//                   the output feeds a concatenation.  The same kernel computes the input
//                   gradient (transposed, flipped weights).
//  of_cnn_conv3x3_wgrad  weight gradient (CUDA cores, f32 FMA over bf16 operands).
//  pooling, nearest upsampling, ReLU masks, loss, Adam and weight packing: elementwise.
//
// Every wait on an mbarrier is bounded by time (about one second); a CTA that gives up
// sets a bit in the caller's error word, waits (bounded) for its copies in flight and
// for its MMAs, frees its TMEM and exits.
#include <cuda_bf16.h>

#include "common.cuh"
#include "tma.cuh"

namespace ofb {

typedef __nv_bfloat16 bf16;

constexpr int CV_M = 128;
constexpr int CV_STAGES = 4;
constexpr int CV_THREADS = 192;
constexpr unsigned long long CV_WAIT_NS = 1000000000ull;

enum { CV_RELU = 1, CV_F32 = 2 };

struct ConvParams {
  int n, H, W, ck, nchunks;
  int bw, bh, nb, tiles_x, tiles_per_group;  // a tile: nb images x bh rows x bw columns = 128 pixels
  int bn, cout_store, flags;
  const float* bias;
  void* y;
  int y_ctot, y_coff;
  unsigned* err;
  uint32_t a_bytes, b_bytes, stage_bytes, tmem_cols;
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for phase `parity`; gives up after CV_WAIT_NS or when *abort becomes nonzero.
__device__ bool cv_wait(uint64_t* bar, uint32_t parity, volatile int* abort) {
  unsigned long long t0 = globaltimer_ns();
  while (!mbar_try(bar, parity)) {
    if (abort && *abort) return false;
    if (globaltimer_ns() - t0 > CV_WAIT_NS) return false;
  }
  return true;
}

// Shared-memory matrix descriptor (sm_100 UMMA), K-major operand with a 32/64/128-byte
// swizzle: rows of `swz` bytes, 8-row core groups `8 * swz` bytes apart.
__device__ __forceinline__ uint64_t umma_desc_k(uint32_t saddr, int swz) {
  uint64_t layout = swz == 128 ? 2ull : (swz == 64 ? 4ull : 6ull);
  uint64_t sbo = (uint64_t)(8 * swz) >> 4;
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | (sbo << 32) | (1ull << 46) | (layout << 61);
}

// Instruction descriptor: kind::f16 with bf16 A and B (both K-major), f32 accumulator.
__host__ __device__ inline uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
          tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// TMEM accumulator row (this thread's pixel) -> bias, ReLU, bf16 / f32 store of the N tile
// starting at channel n0.  taddr: the warp's TMEM lane quarter, column 0.
__device__ __forceinline__ void cv_epilogue(const ConvParams& p, uint32_t taddr, size_t pix, int n0) {
  for (int c = 0; c < p.bn; c += 16) {
    uint32_t r[16];
    tmem_ld16(taddr + (uint32_t)c, r);
    const int co = n0 + c;
    if (co >= p.cout_store) continue;
    float v[16];
#pragma unroll
    for (int j = 0; j < 16; j++) {
      float a = __uint_as_float(r[j]);
      if (p.bias && co + j < p.cout_store) a = __fadd_rn(a, p.bias[co + j]);
      if (p.flags & CV_RELU) a = fmaxf(a, 0.f);
      v[j] = a;
    }
    const int nvalid = p.cout_store - co < 16 ? p.cout_store - co : 16;
    if (p.flags & CV_F32) {
      float* yo = static_cast<float*>(p.y) + pix * p.y_ctot + p.y_coff + co;
#pragma unroll
      for (int j = 0; j < 16; j++)
        if (j < nvalid) yo[j] = v[j];
    } else {
      bf16* yo = static_cast<bf16*>(p.y) + pix * p.y_ctot + p.y_coff + co;
      if (nvalid == 16) {
        uint32_t w[8];
#pragma unroll
        for (int j = 0; j < 8; j++) {
          __nv_bfloat162 h2 = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
          w[j] = *reinterpret_cast<uint32_t*>(&h2);
        }
        reinterpret_cast<uint4*>(yo)[0] = make_uint4(w[0], w[1], w[2], w[3]);
        reinterpret_cast<uint4*>(yo)[1] = make_uint4(w[4], w[5], w[6], w[7]);
      } else {
#pragma unroll
        for (int j = 0; j < 16; j++)
          if (j < nvalid) yo[j] = __float2bfloat16_rn(v[j]);
      }
    }
  }
}

__global__ void __launch_bounds__(CV_THREADS, 1)
    conv3x3_tc_kernel(const __grid_constant__ CUtensorMap tm_x, const __grid_constant__ CUtensorMap tm_w,
                      const ConvParams p) {
  extern __shared__ uint8_t cv_smem_raw[];
  __shared__ __align__(8) uint64_t full[CV_STAGES], empty[CV_STAGES], accf;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(cv_smem_raw) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int grp = blockIdx.x / p.tiles_per_group, t_in = blockIdx.x - grp * p.tiles_per_group;
  const int tyi = t_in / p.tiles_x, txi = t_in - tyi * p.tiles_x, img0 = grp * p.nb;
  const int x0 = txi * p.bw, y0 = tyi * p.bh, n0 = blockIdx.y * p.bn;
  const int kiters = 9 * p.nchunks;

  if (threadIdx.x == 0) {
    for (int s = 0; s < CV_STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&accf, 1);
    // once any CTA has given up, the rest skip their work instead of timing out in turn
    abort_flag = *reinterpret_cast<volatile unsigned*>(p.err) != 0u;
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(p.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int issued = 0;
      for (int it = 0; it < kiters && !abort_flag; it++) {
        const int s = it % CV_STAGES;
        const uint32_t ph = (uint32_t)(it / CV_STAGES) & 1u;
        if (!cv_wait(&empty[s], ph ^ 1u, &abort_flag)) {
          atomicOr(p.err, 1u);
          abort_flag = 1;
          break;
        }
        const int tap = it / p.nchunks, ch = it - tap * p.nchunks;
        const int dy = tap / 3 - 1, dx = tap % 3 - 1;
        uint8_t* a = smem + (size_t)s * p.stage_bytes;
        mbar_expect_tx(&full[s], p.a_bytes + p.b_bytes);
        tma_load_4d(a, &tm_x, ch * p.ck, x0 + dx, y0 + dy, img0, &full[s]);
        tma_load_3d(a + p.a_bytes, &tm_w, ch * p.ck, n0, tap, &full[s]);
        issued = it + 1;
      }
      // the copies of the last stages must land before the CTA's shared memory is released
      for (int it = issued > CV_STAGES ? issued - CV_STAGES : 0; it < issued; it++) {
        const int s = it % CV_STAGES;
        if (!cv_wait(&full[s], (uint32_t)(it / CV_STAGES) & 1u, nullptr)) atomicOr(p.err, 2u);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = umma_idesc_bf16(CV_M, p.bn);
      const int swz = p.ck * 2, ksteps = p.ck / 16;
      for (int it = 0; it < kiters; it++) {
        const int s = it % CV_STAGES;
        if (!cv_wait(&full[s], (uint32_t)(it / CV_STAGES) & 1u, &abort_flag)) {
          atomicOr(p.err, 4u);
          abort_flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t a = smem_u32(smem + (size_t)s * p.stage_bytes), b = a + p.a_bytes;
        const uint64_t ad = umma_desc_k(a, swz), bd = umma_desc_k(b, swz);
        for (int kk = 0; kk < ksteps; kk++)  // +32 bytes of K per step (descriptor address unit: 16 B)
          umma_bf16(tmem, ad + 2ull * kk, bd + 2ull * kk, idesc, (it | kk) != 0);
        umma_commit(&empty[s]);
      }
      umma_commit(&accf);  // arrives once every MMA issued above has completed
    }
    __syncwarp();
  } else {
    const int q = warp & 3;  // a warp reads the TMEM lanes 32 * (warp % 4) ...
    const int m = q * 32 + lane;
    const int mi = m / (p.bh * p.bw), mr = m - mi * (p.bh * p.bw);
    const int img = img0 + mi, py = y0 + mr / p.bw, px = x0 + mr % p.bw;
    const bool ok = cv_wait(&accf, 0u, nullptr);
    if (!ok) atomicOr(p.err, 8u);
    tc_fence_after();
    if (ok && !abort_flag) cv_epilogue(p, tmem + ((uint32_t)(q * 32) << 16), ((size_t)img * p.H + py) * p.W + px, n0);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(p.tmem_cols) : "memory");
  }
}

// ----------------------------------------------------------------------------- wgrad, tensor cores
// dW[tap] = sum over pixels of dY[p] (x) X[p + tap]: per tap a GEMM whose K is the pixel
// count.  NHWC keeps the channels contiguous, so both operands are MN-major: a TMA box of
// 64 channels x 64 pixels lands as 64 rows of 128 B (128-byte swizzle), which is the
// canonical MN-major layout (8-row groups 1024 B apart, 64-channel atoms 8 KB apart).
// A is the wider channel side (M = 128, channels past its end are zero-filled by TMA and
// their rows ignored), B the narrower (N <= 256).  X is shifted by the tap through the box
// coordinates (zero padding from TMA's out-of-bounds fill).  CTAs split the pixel range;
// each adds its 128 x N partial sums into dW with atomics.
constexpr int WT_KP = 64;  // pixels per K chunk
constexpr int WT_STAGES = 4;

struct WgParams {
  int n, H, W, bw, bh, nb, tiles_x, tiles_per_group, nchunk;  // pixel chunk geometry
  int chunks_per_cta, mtiles, ntiles;
  int a_is_dy, a_ch, b_ch;   // channel counts of the A and B sides
  int nmma, batoms;          // MMA N and 64-channel atoms loaded for B
  int cin, cout;
  float* dw;
  unsigned* err;
  uint32_t a_bytes, b_bytes, stage_bytes, tmem_cols;
};

// Shared-memory descriptor of a MN-major operand with the 128-byte swizzle: 64-element atoms
// `lbo` bytes apart along M/N, 8-row K groups 1024 bytes apart.
__device__ __forceinline__ uint64_t umma_desc_mn128(uint32_t saddr, uint32_t lbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) | ((uint64_t)(1024 >> 4) << 32) |
         (1ull << 46) | (2ull << 61);
}

__host__ __device__ inline uint32_t umma_idesc_bf16_mn(int m, int n) {
  return umma_idesc_bf16(m, n) | (1u << 15) | (1u << 16);  // A and B MN-major
}

__global__ void __launch_bounds__(CV_THREADS, 1)
    wgrad_tc_kernel(const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_b,
                    const WgParams p) {
  extern __shared__ uint8_t wg_smem_raw[];
  __shared__ __align__(8) uint64_t full[WT_STAGES], empty[WT_STAGES], accf;
  __shared__ uint32_t tmem_slot;
  __shared__ volatile int abort_flag;
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(wg_smem_raw) + 1023) & ~(uintptr_t)1023);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tap = blockIdx.z, mt = blockIdx.y / p.ntiles, nt = blockIdx.y - mt * p.ntiles;
  const int m0 = mt * 128, n0 = nt * 256;
  const int c0 = blockIdx.x * p.chunks_per_cta;
  const int c1 = c0 + p.chunks_per_cta < p.nchunk ? c0 + p.chunks_per_cta : p.nchunk;
  const int kiters = c1 > c0 ? c1 - c0 : 0;
  const int dy = tap / 3 - 1, dx = tap % 3 - 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < WT_STAGES; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&accf, 1);
    abort_flag = *reinterpret_cast<volatile unsigned*>(p.err) != 0u;
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(p.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      int issued = 0;
      for (int it = 0; it < kiters && !abort_flag; it++) {
        const int s = it % WT_STAGES;
        if (!cv_wait(&empty[s], ((uint32_t)(it / WT_STAGES) & 1u) ^ 1u, &abort_flag)) {
          atomicOr(p.err, 1u);
          abort_flag = 1;
          break;
        }
        const int ch = c0 + it, grp = ch / p.tiles_per_group, t_in = ch - grp * p.tiles_per_group;
        const int ty = t_in / p.tiles_x, tx = t_in - ty * p.tiles_x;
        const int x0 = tx * p.bw, y0 = ty * p.bh, img0 = grp * p.nb;
        // the A side is dY (unshifted) or X (shifted), the B side the other
        const int ax = p.a_is_dy ? x0 : x0 + dx, ay = p.a_is_dy ? y0 : y0 + dy;
        const int bx = p.a_is_dy ? x0 + dx : x0, by = p.a_is_dy ? y0 + dy : y0;
        uint8_t* a = smem + (size_t)s * p.stage_bytes;
        mbar_expect_tx(&full[s], p.a_bytes + p.b_bytes);
        tma_load_4d(a, &tm_a, m0, ax, ay, img0, &full[s]);
        tma_load_4d(a + 8192, &tm_a, m0 + 64, ax, ay, img0, &full[s]);
        for (int j = 0; j < p.batoms; j++)
          tma_load_4d(a + p.a_bytes + j * 8192, &tm_b, n0 + 64 * j, bx, by, img0, &full[s]);
        issued = it + 1;
      }
      for (int it = issued > WT_STAGES ? issued - WT_STAGES : 0; it < issued; it++)
        if (!cv_wait(&full[it % WT_STAGES], (uint32_t)(it / WT_STAGES) & 1u, nullptr)) atomicOr(p.err, 2u);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = umma_idesc_bf16_mn(128, p.nmma);
      for (int it = 0; it < kiters; it++) {
        const int s = it % WT_STAGES;
        if (!cv_wait(&full[s], (uint32_t)(it / WT_STAGES) & 1u, &abort_flag)) {
          atomicOr(p.err, 4u);
          abort_flag = 1;
          break;
        }
        tc_fence_after();
        const uint32_t a = smem_u32(smem + (size_t)s * p.stage_bytes), b = a + p.a_bytes;
        const uint64_t ad = umma_desc_mn128(a, 8192), bd = umma_desc_mn128(b, 8192);
        for (int kk = 0; kk < WT_KP / 16; kk++)  // 16 pixels = two 8-row groups: +2048 B (128 descriptor units)
          umma_bf16(tmem, ad + 128ull * kk, bd + 128ull * kk, idesc, (it | kk) != 0);
        umma_commit(&empty[s]);
      }
      umma_commit(&accf);
    }
    __syncwarp();
  } else {
    const int q = warp & 3;
    const int m = q * 32 + lane;
    const bool ok = cv_wait(&accf, 0u, nullptr);
    if (!ok) atomicOr(p.err, 8u);
    tc_fence_after();
    const int am = m0 + m;  // this thread's A-side channel
    if (ok && !abort_flag && kiters > 0) {
      for (int c = 0; c < p.nmma; c += 16) {
        uint32_t r[16];
        tmem_ld16(tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)c, r);
        if (am >= p.a_ch) continue;
#pragma unroll
        for (int j = 0; j < 16; j++) {
          const int bn = n0 + c + j;
          if (bn >= p.b_ch) break;
          const int co = p.a_is_dy ? am : bn, ci = p.a_is_dy ? bn : am;
          atomicAdd(&p.dw[((size_t)tap * p.cout + co) * p.cin + ci], __uint_as_float(r[j]));
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(p.tmem_cols) : "memory");
  }
}

// ----------------------------------------------------------------------------- wgrad
// dW[tap][co][ci] += sum over pixels p of dY[p][co] * X[p + tap][ci]  (zero outside the
// image).  A CTA owns a 32 (co) x 32 (ci) block of all 9 taps and walks 64-pixel row
// segments; each thread keeps 9 x 4 accumulators (one co, four ci).
constexpr int WG_SEG = 64;

__global__ void __launch_bounds__(256) conv3x3_wgrad_kernel(const bf16* __restrict__ X, int xct, int xco,
                                                            const bf16* __restrict__ dY, int dct, int dco, int n,
                                                            int H, int W, int cin, int cout, float* __restrict__ dW) {
  __shared__ __align__(16) float sx[3][WG_SEG + 2][32];
  __shared__ float sg[WG_SEG][33];
  const int t = threadIdx.x, col = t >> 3, cg = (t & 7) * 4;
  const int ci0 = blockIdx.y * 32, co0 = blockIdx.z * 32;
  const int segs = (W + WG_SEG - 1) / WG_SEG;
  const long long units = (long long)n * H * segs;
  float acc[9][4];
#pragma unroll
  for (int k = 0; k < 9; k++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[k][j] = 0.f;
  for (long long u = blockIdx.x; u < units; u += gridDim.x) {
    const int sgi = (int)(u % segs);
    const long long rowi = u / segs;
    const int y = (int)(rowi % H), img = (int)(rowi / H), xs = sgi * WG_SEG;
    __syncthreads();
    for (int e = t; e < 3 * (WG_SEG + 2) * 32; e += 256) {
      int c = e & 31, rest = e >> 5, xx = rest % (WG_SEG + 2), ky = rest / (WG_SEG + 2);
      int gy = y + ky - 1, gx = xs + xx - 1, ci = ci0 + c;
      float v = 0.f;
      if (gy >= 0 && gy < H && gx >= 0 && gx < W && ci < cin)
        v = __bfloat162float(X[(((size_t)img * H + gy) * W + gx) * xct + xco + ci]);
      sx[ky][xx][c] = v;
    }
    for (int e = t; e < WG_SEG * 32; e += 256) {
      int c = e & 31, xx = e >> 5, gx = xs + xx, co = co0 + c;
      float v = 0.f;
      if (gx < W && co < cout) v = __bfloat162float(dY[(((size_t)img * H + y) * W + gx) * dct + dco + co]);
      sg[xx][c] = v;
    }
    __syncthreads();
#pragma unroll 4
    for (int xx = 0; xx < WG_SEG; xx++) {
      const float g = sg[xx][col];
#pragma unroll
      for (int ky = 0; ky < 3; ky++)
#pragma unroll
        for (int kx = 0; kx < 3; kx++) {
          const float4 xv = *reinterpret_cast<const float4*>(&sx[ky][xx + kx][cg]);
          float* a = acc[ky * 3 + kx];
          a[0] = __fmaf_rn(g, xv.x, a[0]);
          a[1] = __fmaf_rn(g, xv.y, a[1]);
          a[2] = __fmaf_rn(g, xv.z, a[2]);
          a[3] = __fmaf_rn(g, xv.w, a[3]);
        }
    }
  }
  const int co = co0 + col;
  if (co >= cout) return;
#pragma unroll
  for (int k = 0; k < 9; k++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int ci = ci0 + cg + j;
      if (ci < cin) atomicAdd(&dW[((size_t)k * cout + co) * cin + ci], acc[k][j]);
    }
}

// db[co] += sum over pixels of dY[p][co]
__global__ void bias_grad_kernel(const bf16* __restrict__ dY, int dct, int dco, long long P, int cout,
                                 float* __restrict__ db) {
  const int c = threadIdx.x;  // blockDim.x >= cout
  float s = 0.f;
  if (c < cout)
    for (long long p = blockIdx.x; p < P; p += gridDim.x) s = __fadd_rn(s, __bfloat162float(dY[p * dct + dco + c]));
  if (c < cout) atomicAdd(&db[c], s);
}

// ----------------------------------------------------------------------------- elementwise
// out[img][y][x][0..cpad) = (I0 / max I0, I1 / max I1, 0, ...)  in bf16; max over the frame
__global__ void frame_max_kernel(const float* __restrict__ I, int H, int W, int pitch, unsigned* __restrict__ mx) {
  float m = 0.f;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < (long long)H * W;
       e += (long long)gridDim.x * blockDim.x) {
    int y = (int)(e / W), x = (int)(e - (long long)y * W);
    m = fmaxf(m, I[(size_t)y * pitch + x]);
  }
  for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(mx, __float_as_uint(m));  // non-negative floats order as integers
}

// One pixel of the network input: (a, b, 0, ...) over cpad channels; 16-byte stores when
// cpad is a multiple of 8 and the pixel's channels start 16-byte aligned.
__device__ __forceinline__ void pack_store(bf16* o, int cpad, float a, float b) {
  if ((cpad & 7) == 0 && (reinterpret_cast<uintptr_t>(o) & 15) == 0) {
    const __nv_bfloat162 ab = __floats2bfloat162_rn(a, b);
    uint4 v = make_uint4(*reinterpret_cast<const unsigned int*>(&ab), 0u, 0u, 0u);
    reinterpret_cast<uint4*>(o)[0] = v;
    v.x = 0u;
    for (int c = 8; c < cpad; c += 8) reinterpret_cast<uint4*>(o + c)[0] = v;
    return;
  }
  o[0] = __float2bfloat16_rn(a);
  o[1] = __float2bfloat16_rn(b);
  for (int c = 2; c < cpad; c++) o[c] = __float2bfloat16_rn(0.f);
}

__global__ void pack_pair_kernel(const float* __restrict__ I0, const float* __restrict__ I1, int H, int W, int pitch,
                                 const unsigned* __restrict__ mx, bf16* __restrict__ out, int cpad) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)H * W) return;
  int y = (int)(e / W), x = (int)(e - (long long)y * W);
  float m0 = __uint_as_float(mx[0]), m1 = __uint_as_float(mx[1]);
  float a = m0 > 0.f ? __fdiv_rn(I0[(size_t)y * pitch + x], m0) : 0.f;
  float b = m1 > 0.f ? __fdiv_rn(I1[(size_t)y * pitch + x], m1) : 0.f;
  pack_store(out + (size_t)e * cpad, cpad, a, b);
}

// Both maxima and the packing in one CTA, for the small frames the network runs on (up to
// 64 K pixels): the maxima are the same (max is exact and order-free, NaN-free through
// fmaxf as in frame_max_kernel) and the packing is pack_pair_kernel's per pixel.
constexpr int PK1_THREADS = 1024;
__global__ void __launch_bounds__(PK1_THREADS) pack_pair_one_kernel(const float* __restrict__ I0,
                                                                     const float* __restrict__ I1, int H, int W,
                                                                     int pitch, unsigned* __restrict__ mx,
                                                                     bf16* __restrict__ out, int cpad) {
  __shared__ float r0[32], r1[32];
  const int n = H * W;
  float m0 = 0.f, m1 = 0.f;
  for (int e = threadIdx.x; e < n; e += PK1_THREADS) {
    const int y = e / W, x = e - y * W;
    m0 = fmaxf(m0, I0[(size_t)y * pitch + x]);
    m1 = fmaxf(m1, I1[(size_t)y * pitch + x]);
  }
  for (int o = 16; o; o >>= 1) {
    m0 = fmaxf(m0, __shfl_xor_sync(0xffffffffu, m0, o));
    m1 = fmaxf(m1, __shfl_xor_sync(0xffffffffu, m1, o));
  }
  if ((threadIdx.x & 31) == 0) {
    r0[threadIdx.x >> 5] = m0;
    r1[threadIdx.x >> 5] = m1;
  }
  __syncthreads();
  m0 = r0[0];
  m1 = r1[0];
  for (int w = 1; w < PK1_THREADS / 32; w++) {
    m0 = fmaxf(m0, r0[w]);
    m1 = fmaxf(m1, r1[w]);
  }
  if (threadIdx.x == 0) {
    mx[0] = __float_as_uint(m0);
    mx[1] = __float_as_uint(m1);
  }
  for (int e = threadIdx.x; e < n; e += PK1_THREADS) {
    const int y = e / W, x = e - y * W;
    const float a = m0 > 0.f ? __fdiv_rn(I0[(size_t)y * pitch + x], m0) : 0.f;
    const float b = m1 > 0.f ? __fdiv_rn(I1[(size_t)y * pitch + x], m1) : 0.f;
    pack_store(out + (size_t)e * cpad, cpad, a, b);
  }
}

__global__ void avgpool2_kernel(const bf16* __restrict__ x, int xct, int xco, int n, int H, int W, int C,
                                bf16* __restrict__ y, int yct, int yco) {
  const int h = H / 2, w = W / 2;
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * h * w * C) return;
  int c = (int)(e % C);
  long long q = e / C;
  int ox = (int)(q % w), oy = (int)((q / w) % h), img = (int)(q / ((long long)w * h));
  const bf16* b = x + (((size_t)img * H + 2 * oy) * W + 2 * ox) * xct + xco + c;
  float s = __fadd_rn(__fadd_rn(__bfloat162float(b[0]), __bfloat162float(b[xct])),
                      __fadd_rn(__bfloat162float(b[(size_t)W * xct]), __bfloat162float(b[(size_t)W * xct + xct])));
  y[(((size_t)img * h + oy) * w + ox) * yct + yco + c] = __float2bfloat16_rn(__fmul_rn(s, 0.25f));
}

// The same two kernels on 8 channels (16 bytes) per thread, one output row per blockIdx.y
// (image * rows + row) and 32-bit index arithmetic: used when the channel counts, channel
// offsets and row strides are multiples of 8 and the bases 16-byte aligned (every layer of
// the network).  Per channel the arithmetic is the scalar kernels'.
__device__ __forceinline__ float2 bf2f(unsigned int u) {
  return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
}
__device__ __forceinline__ unsigned int f2bf(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const unsigned int*>(&h);
}

__global__ void avgpool2_v8_kernel(const bf16* __restrict__ x, int xct, int xco, int H, int W, int C,
                                   bf16* __restrict__ y, int yct, int yco) {
  const int h = H / 2, w = W / 2, c8 = C / 8;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= w * c8) return;
  const int ox = t / c8, c = 8 * (t - ox * c8);
  const int img = blockIdx.y / h, oy = blockIdx.y - img * h;
  const bf16* b = x + (((size_t)img * H + 2 * oy) * W + 2 * ox) * xct + xco + c;
  const uint4 p0 = *reinterpret_cast<const uint4*>(b), p1 = *reinterpret_cast<const uint4*>(b + xct);
  const uint4 p2 = *reinterpret_cast<const uint4*>(b + (size_t)W * xct);
  const uint4 p3 = *reinterpret_cast<const uint4*>(b + (size_t)W * xct + xct);
  const unsigned int a0[4] = {p0.x, p0.y, p0.z, p0.w}, a1[4] = {p1.x, p1.y, p1.z, p1.w};
  const unsigned int a2[4] = {p2.x, p2.y, p2.z, p2.w}, a3[4] = {p3.x, p3.y, p3.z, p3.w};
  unsigned int o[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const float2 v0 = bf2f(a0[k]), v1 = bf2f(a1[k]), v2 = bf2f(a2[k]), v3 = bf2f(a3[k]);
    const float sx = __fadd_rn(__fadd_rn(v0.x, v1.x), __fadd_rn(v2.x, v3.x));
    const float sy = __fadd_rn(__fadd_rn(v0.y, v1.y), __fadd_rn(v2.y, v3.y));
    o[k] = f2bf(__fmul_rn(sx, 0.25f), __fmul_rn(sy, 0.25f));
  }
  *reinterpret_cast<uint4*>(y + (((size_t)img * h + oy) * w + ox) * yct + yco + c) = make_uint4(o[0], o[1], o[2], o[3]);
}

__global__ void upsample2_v8_kernel(const bf16* __restrict__ x, int xct, int xco, int h, int w, int C,
                                    bf16* __restrict__ y, int yct, int yco) {
  const int H = 2 * h, W = 2 * w, c8 = C / 8;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= W * c8) return;
  const int xx = t / c8, c = 8 * (t - xx * c8);
  const int img = blockIdx.y / H, yy = blockIdx.y - img * H;
  *reinterpret_cast<uint4*>(y + (((size_t)img * H + yy) * W + xx) * yct + yco + c) =
      *reinterpret_cast<const uint4*>(x + (((size_t)img * h + yy / 2) * w + xx / 2) * xct + xco + c);
}

static bool v8_ok(const void* x, int xct, int xco, const void* y, int yct, int yco, int C) {
  return C % 8 == 0 && xct % 8 == 0 && xco % 8 == 0 && yct % 8 == 0 && yco % 8 == 0 &&
         ((reinterpret_cast<uintptr_t>(x) | reinterpret_cast<uintptr_t>(y)) & 15) == 0;
}

// dx (fine) = dy (coarse parent) / 4, added to dx when accumulate
__global__ void avgpool2_bwd_kernel(const bf16* __restrict__ dy, int dct, int dco, int n, int H, int W, int C,
                                    bf16* __restrict__ dx, int xct, int xco, int accumulate) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * H * W * C) return;
  int c = (int)(e % C);
  long long q = e / C;
  int xx = (int)(q % W), yy = (int)((q / W) % H), img = (int)(q / ((long long)W * H));
  const int h = H / 2, w = W / 2;
  float g = __fmul_rn(__bfloat162float(dy[(((size_t)img * h + yy / 2) * w + xx / 2) * dct + dco + c]), 0.25f);
  bf16* o = dx + (((size_t)img * H + yy) * W + xx) * xct + xco + c;
  if (accumulate) g = __fadd_rn(g, __bfloat162float(*o));
  *o = __float2bfloat16_rn(g);
}

// nearest 2x upsampling of x (n, h, w, C) into a channel slice of y (n, 2h, 2w, yct)
__global__ void upsample2_kernel(const bf16* __restrict__ x, int xct, int xco, int n, int h, int w, int C,
                                 bf16* __restrict__ y, int yct, int yco) {
  const int H = 2 * h, W = 2 * w;
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * H * W * C) return;
  int c = (int)(e % C);
  long long q = e / C;
  int xx = (int)(q % W), yy = (int)((q / W) % H), img = (int)(q / ((long long)W * H));
  y[(((size_t)img * H + yy) * W + xx) * yct + yco + c] = x[(((size_t)img * h + yy / 2) * w + xx / 2) * xct + xco + c];
}

__global__ void upsample2_bwd_kernel(const bf16* __restrict__ dy, int dct, int dco, int n, int h, int w, int C,
                                     bf16* __restrict__ dx, int xct, int xco) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)n * h * w * C) return;
  int c = (int)(e % C);
  long long q = e / C;
  int ox = (int)(q % w), oy = (int)((q / w) % h), img = (int)(q / ((long long)w * h));
  const int W = 2 * w, H = 2 * h;
  const bf16* b = dy + (((size_t)img * H + 2 * oy) * W + 2 * ox) * dct + dco + c;
  float s = __fadd_rn(__fadd_rn(__bfloat162float(b[0]), __bfloat162float(b[dct])),
                      __fadd_rn(__bfloat162float(b[(size_t)W * dct]), __bfloat162float(b[(size_t)W * dct + dct])));
  dx[(((size_t)img * h + oy) * w + ox) * xct + xco + c] = __float2bfloat16_rn(s);
}

// g = g * (y > 0) over a channel slice (the ReLU derivative from the layer's output)
__global__ void relu_bwd_kernel(bf16* __restrict__ g, int gct, int gco, const bf16* __restrict__ y, int yct, int yco,
                                long long P, int C) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= P * C) return;
  long long p = e / C;
  int c = (int)(e - p * C);
  if (!(__bfloat162float(y[p * yct + yco + c]) > 0.f)) g[p * gct + gco + c] = __float2bfloat16_rn(0.f);
}

// mean squared flow error: loss += sum (pred - label)^2 / (2 P);  dpred = (pred - label) / P
// (bf16, padded to gct channels, the padding zeroed)
__global__ void flow_mse_kernel(const float* __restrict__ pred, const float* __restrict__ label, long long P,
                                bf16* __restrict__ dpred, int gct, double* __restrict__ loss) {
  long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (p < P) {
    const float inv = __frcp_rn((float)P);
    float du = __fadd_rn(pred[2 * p], -label[2 * p]), dv = __fadd_rn(pred[2 * p + 1], -label[2 * p + 1]);
    l = __fadd_rn(__fmul_rn(du, du), __fmul_rn(dv, dv));
    if (dpred) {
      bf16* o = dpred + p * gct;
      o[0] = __float2bfloat16_rn(__fmul_rn(du, inv));
      o[1] = __float2bfloat16_rn(__fmul_rn(dv, inv));
      for (int c = 2; c < gct; c++) o[c] = __float2bfloat16_rn(0.f);
    }
  }
  for (int o = 16; o; o >>= 1) l = __fadd_rn(l, __shfl_xor_sync(0xffffffffu, l, o));
  if ((threadIdx.x & 31) == 0 && p - (threadIdx.x & 31) < P) atomicAdd(loss, (double)l / (2.0 * (double)P));
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float bc1,
                            float bc2) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = g[i];
  float mi = __fadd_rn(__fmul_rn(b1, m[i]), __fmul_rn(__fadd_rn(1.f, -b1), gi));
  float vi = __fadd_rn(__fmul_rn(b2, v[i]), __fmul_rn(__fadd_rn(1.f, -b2), __fmul_rn(gi, gi)));
  m[i] = mi;
  v[i] = vi;
  float mh = __fdiv_rn(mi, bc1), vh = __fdiv_rn(vi, bc2);
  w[i] = __fadd_rn(w[i], -__fdiv_rn(__fmul_rn(lr, mh), __fadd_rn(__fsqrt_rn(vh), eps)));
}

// master weights w[tap][co][ci] (f32, the wgrad layout) -> bf16 B operands:
//   forward:  out[tap][co][ci]                     (cout_pad x cin_pad rows per tap)
//   backward: out[tap'][ci][co] = w[co][ci][8-tap'] (cin_pad x cout_pad rows per tap)
__global__ void pack_weights_kernel(const float* __restrict__ w, int cout, int cin, int cout_pad, int cin_pad,
                                    int transpose_flip, bf16* __restrict__ out) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long total = 9LL * cout_pad * cin_pad;
  if (e >= total) return;
  int tap = (int)(e / ((long long)cout_pad * cin_pad));
  int r = (int)(e - (long long)tap * cout_pad * cin_pad);
  int cols = transpose_flip ? cout_pad : cin_pad;
  int row = r / cols, colm = r - row * cols;
  int co = transpose_flip ? colm : row, ci = transpose_flip ? row : colm;
  int k = transpose_flip ? 8 - tap : tap;
  float v = (co < cout && ci < cin) ? w[((size_t)k * cout + co) * cin + ci] : 0.f;
  out[e] = __float2bfloat16_rn(v);
}

// (h, w, 2) interleaved f32 flow -> two planes with row pitch `pitch`
__global__ void split_flow_kernel(const float* __restrict__ f, int h, int w, float* __restrict__ u,
                                  float* __restrict__ v, int pitch) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long long)h * w) return;
  int y = (int)(e / w), x = (int)(e - (long long)y * w);
  u[(size_t)y * pitch + x] = f[2 * e];
  v[(size_t)y * pitch + x] = f[2 * e + 1];
}

// (h, w, 2) interleaved f32 flow -> U, V planes at (f h, f w), bilinear with pixel-centre
// alignment (fine pixel X samples coarse position (X + 0.5) / f - 0.5, clamped) and the
// displacement scaled by `scale`.
__global__ void flow_up_kernel(const float* __restrict__ fl, int h, int w, int f, float* __restrict__ U,
                               float* __restrict__ V, int pitch, float scale) {
  const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y;
  if (X >= f * w) return;
  const float inv = __frcp_rn((float)f);
  const float sx = fmaxf(__fsub_rn(__fmul_rn(__fadd_rn((float)X, 0.5f), inv), 0.5f), 0.f);
  const float sy = fmaxf(__fsub_rn(__fmul_rn(__fadd_rn((float)Y, 0.5f), inv), 0.5f), 0.f);
  int x0 = (int)sx, y0 = (int)sy;
  x0 = x0 < w - 1 ? x0 : w - 1;
  y0 = y0 < h - 1 ? y0 : h - 1;
  const int x1 = x0 + 1 < w ? x0 + 1 : w - 1, y1 = y0 + 1 < h ? y0 + 1 : h - 1;
  const float ax = __fsub_rn(sx, (float)x0), ay = __fsub_rn(sy, (float)y0);
#pragma unroll
  for (int c = 0; c < 2; c++) {
    const float a = fl[((size_t)y0 * w + x0) * 2 + c], b = fl[((size_t)y0 * w + x1) * 2 + c];
    const float d = fl[((size_t)y1 * w + x0) * 2 + c], e = fl[((size_t)y1 * w + x1) * 2 + c];
    const float top = __fmaf_rn(ax, __fsub_rn(b, a), a), bot = __fmaf_rn(ax, __fsub_rn(e, d), d);
    const float v = __fmul_rn(__fmaf_rn(ay, __fsub_rn(bot, top), top), scale);
    (c == 0 ? U : V)[(size_t)Y * pitch + X] = v;
  }
}

static int blocks_for(long long n, int t = 256) { return (int)((n + t - 1) / t); }

}  // namespace ofb

using namespace ofb;

extern "C" int of_cnn_conv3x3(const void* x, int n, int H, int W, int cin, int x_ctot, int x_coff, const void* w,
                              int cout, const float* bias, int flags, void* y, int y_ctot, int y_coff, int cout_store,
                              unsigned* err, void* stream) {
  OF_REQUIRE(x && w && y && err && n > 0 && H > 0 && W > 0, "of_cnn_conv3x3: bad arguments");
  int ck = cin % 64 == 0 ? 64 : (cin % 32 == 0 ? 32 : (cin == 16 ? 16 : 0));
  OF_REQUIRE(ck, "of_cnn_conv3x3: input channels %d (need 16, a multiple of 32)", cin);
  OF_REQUIRE(cout % 16 == 0 && cout <= 512 && cout > 0, "of_cnn_conv3x3: output channels %d (need 16..512, /16)", cout);
  int ntile = (cout + 255) / 256, bn = cout / ntile;
  OF_REQUIRE(bn * ntile == cout && bn % 16 == 0, "of_cnn_conv3x3: output channels %d do not split into N tiles", cout);
  int bw = W < CV_M ? W : CV_M;
  OF_REQUIRE(CV_M % bw == 0 && W % bw == 0, "of_cnn_conv3x3: width %d (need a divisor of 128 or a multiple)", W);
  int bh = CV_M / bw < H ? CV_M / bw : H;
  OF_REQUIRE(H % bh == 0 && (CV_M / bw) % bh == 0, "of_cnn_conv3x3: height %d does not tile by %d", H, bh);
  int nb = CV_M / (bw * bh);  // small images: one tile spans nb whole images
  OF_REQUIRE(n % nb == 0, "of_cnn_conv3x3: %d images of %d x %d do not fill 128-pixel tiles", n, H, W);
  OF_REQUIRE(x_ctot % 8 == 0 && x_coff % 8 == 0 && x_coff + cin <= x_ctot, "of_cnn_conv3x3: input channel slice");
  // bf16 stores go out 16 bytes at a time; f32 stores are scalar
  const bool f32 = (flags & CV_F32) != 0;
  OF_REQUIRE((f32 || (y_ctot % 8 == 0 && y_coff % 8 == 0)) && cout_store <= cout && cout_store > 0 &&
                 y_coff + cout_store <= y_ctot,
             "of_cnn_conv3x3: output channel slice");
  OF_REQUIRE(f32 || ((uintptr_t)y & 15) == 0, "of_cnn_conv3x3: output not 16-byte aligned");
  CUtensorMap tmx, tmw;
  {
    uint64_t dims[4] = {(uint64_t)cin, (uint64_t)W, (uint64_t)H, (uint64_t)n};
    uint64_t st[3] = {(uint64_t)x_ctot * 2, (uint64_t)W * x_ctot * 2, (uint64_t)H * W * x_ctot * 2};
    uint32_t box[4] = {(uint32_t)ck, (uint32_t)bw, (uint32_t)bh, (uint32_t)nb};
    int rc = tmap_bf16(&tmx, static_cast<const bf16*>(x) + x_coff, 4, dims, st, box, ck * 2);
    if (rc) return rc;
  }
  {
    uint64_t dims[3] = {(uint64_t)cin, (uint64_t)cout, 9};
    uint64_t st[2] = {(uint64_t)cin * 2, (uint64_t)cout * cin * 2};
    uint32_t box[3] = {(uint32_t)ck, (uint32_t)bn, 1};
    int rc = tmap_bf16(&tmw, w, 3, dims, st, box, ck * 2);
    if (rc) return rc;
  }
  ConvParams p;
  p.n = n;
  p.H = H;
  p.W = W;
  p.ck = ck;
  p.nchunks = cin / ck;
  p.bw = bw;
  p.bh = bh;
  p.nb = nb;
  p.tiles_x = W / bw;
  p.tiles_per_group = (W / bw) * (H / bh);
  p.bn = bn;
  p.cout_store = cout_store;
  p.flags = flags;
  p.bias = bias;
  p.y = y;
  p.y_ctot = y_ctot;
  p.y_coff = y_coff;
  p.err = err;
  p.a_bytes = (uint32_t)(CV_M * ck * 2);
  p.b_bytes = (uint32_t)(bn * ck * 2);
  p.stage_bytes = (uint32_t)align_up(p.a_bytes + p.b_bytes, 1024);
  p.tmem_cols = bn <= 32 ? 32 : (bn <= 64 ? 64 : (bn <= 128 ? 128 : 256));
  // shared memory in proportion to the TMEM columns held, so the CTAs resident on an SM
  // never ask for more than its 512 columns
  size_t smem = 1024 + (size_t)CV_STAGES * p.stage_bytes;
  size_t floor_smem = (size_t)p.tmem_cols * 456 + 1024;
  if (smem < floor_smem) smem = floor_smem;
  {
    cudaError_t e = OF_SMEM_OPT_IN(conv3x3_tc_kernel, smem);
    if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_cnn_conv3x3: %zu B of shared memory: %s", smem,
                                           cudaGetErrorString(e));
  }
  dim3 grid((n / nb) * p.tiles_per_group, ntile);
  conv3x3_tc_kernel<<<grid, CV_THREADS, smem, as_stream(stream)>>>(tmx, tmw, p);
  return check_launch("of_cnn_conv3x3");
}

extern "C" int of_cnn_conv3x3_wgrad(const void* x, int x_ctot, int x_coff, const void* dy, int dy_ctot, int dy_coff,
                                    int n, int H, int W, int cin, int cout, float* dw, void* stream) {
  OF_REQUIRE(x && dy && dw && n > 0 && H > 0 && W > 0 && cin > 0 && cout > 0, "of_cnn_conv3x3_wgrad: bad arguments");
  long long units = (long long)n * H * ((W + WG_SEG - 1) / WG_SEG);
  int gx = (int)(units < 4LL * kNumSMs ? units : 4LL * kNumSMs);
  dim3 grid(gx, (cin + 31) / 32, (cout + 31) / 32);
  conv3x3_wgrad_kernel<<<grid, 256, 0, as_stream(stream)>>>(static_cast<const bf16*>(x), x_ctot, x_coff,
                                                             static_cast<const bf16*>(dy), dy_ctot, dy_coff, n, H, W,
                                                             cin, cout, dw);
  return check_launch("of_cnn_conv3x3_wgrad");
}

extern "C" int of_cnn_bias_grad(const void* dy, int dy_ctot, int dy_coff, long long P, int cout, float* db,
                                void* stream) {
  OF_REQUIRE(dy && db && P > 0 && cout > 0 && cout <= 1024, "of_cnn_bias_grad: bad arguments");
  int t = (cout + 31) / 32 * 32;
  int g = (int)(P < 2LL * kNumSMs * 8 ? P : 2LL * kNumSMs * 8);
  bias_grad_kernel<<<g, t, 0, as_stream(stream)>>>(static_cast<const bf16*>(dy), dy_ctot, dy_coff, P, cout, db);
  return check_launch("of_cnn_bias_grad");
}

extern "C" int of_cnn_pack_pair(const float* I0, const float* I1, int H, int W, int pitch, unsigned* max2, void* out,
                                int cpad, void* stream) {
  OF_REQUIRE(I0 && I1 && max2 && out && H > 0 && W > 0 && pitch >= W && cpad >= 2, "of_cnn_pack_pair: bad arguments");
  cudaStream_t st = as_stream(stream);
  if ((long long)H * W <= 65536) {
    pack_pair_one_kernel<<<1, PK1_THREADS, 0, st>>>(I0, I1, H, W, pitch, max2, static_cast<bf16*>(out), cpad);
    return check_launch("of_cnn_pack_pair");
  }
  cudaMemsetAsync(max2, 0, 2 * sizeof(unsigned), st);
  int g = blocks_for((long long)H * W);
  int gm = g < 4 * kNumSMs ? g : 4 * kNumSMs;
  frame_max_kernel<<<gm, 256, 0, st>>>(I0, H, W, pitch, max2);
  frame_max_kernel<<<gm, 256, 0, st>>>(I1, H, W, pitch, max2 + 1);
  pack_pair_kernel<<<g, 256, 0, st>>>(I0, I1, H, W, pitch, max2, static_cast<bf16*>(out), cpad);
  return check_launch("of_cnn_pack_pair", 3);
}

extern "C" int of_cnn_avgpool2(const void* x, int x_ctot, int x_coff, int n, int H, int W, int C, void* y, int y_ctot,
                               int y_coff, void* stream) {
  OF_REQUIRE(x && y && H % 2 == 0 && W % 2 == 0 && C > 0, "of_cnn_avgpool2: bad arguments");
  if (v8_ok(x, x_ctot, x_coff, y, y_ctot, y_coff, C) && (long long)n * (H / 2) <= 65535) {
    avgpool2_v8_kernel<<<dim3(blocks_for((long long)(W / 2) * (C / 8)), n * (H / 2)), 256, 0, as_stream(stream)>>>(
        static_cast<const bf16*>(x), x_ctot, x_coff, H, W, C, static_cast<bf16*>(y), y_ctot, y_coff);
    return check_launch("of_cnn_avgpool2");
  }
  long long tot = (long long)n * (H / 2) * (W / 2) * C;
  avgpool2_kernel<<<blocks_for(tot), 256, 0, as_stream(stream)>>>(static_cast<const bf16*>(x), x_ctot, x_coff, n, H,
                                                                   W, C, static_cast<bf16*>(y), y_ctot, y_coff);
  return check_launch("of_cnn_avgpool2");
}

extern "C" int of_cnn_avgpool2_bwd(const void* dy, int dy_ctot, int dy_coff, int n, int H, int W, int C, void* dx,
                                   int dx_ctot, int dx_coff, int accumulate, void* stream) {
  OF_REQUIRE(dy && dx && H % 2 == 0 && W % 2 == 0 && C > 0, "of_cnn_avgpool2_bwd: bad arguments");
  long long tot = (long long)n * H * W * C;
  avgpool2_bwd_kernel<<<blocks_for(tot), 256, 0, as_stream(stream)>>>(
      static_cast<const bf16*>(dy), dy_ctot, dy_coff, n, H, W, C, static_cast<bf16*>(dx), dx_ctot, dx_coff, accumulate);
  return check_launch("of_cnn_avgpool2_bwd");
}

extern "C" int of_cnn_upsample2(const void* x, int x_ctot, int x_coff, int n, int h, int w, int C, void* y, int y_ctot,
                                int y_coff, void* stream) {
  OF_REQUIRE(x && y && h > 0 && w > 0 && C > 0, "of_cnn_upsample2: bad arguments");
  if (v8_ok(x, x_ctot, x_coff, y, y_ctot, y_coff, C) && (long long)n * 2 * h <= 65535) {
    upsample2_v8_kernel<<<dim3(blocks_for((long long)(2 * w) * (C / 8)), n * 2 * h), 256, 0, as_stream(stream)>>>(
        static_cast<const bf16*>(x), x_ctot, x_coff, h, w, C, static_cast<bf16*>(y), y_ctot, y_coff);
    return check_launch("of_cnn_upsample2");
  }
  long long tot = (long long)n * 4 * h * w * C;
  upsample2_kernel<<<blocks_for(tot), 256, 0, as_stream(stream)>>>(static_cast<const bf16*>(x), x_ctot, x_coff, n, h,
                                                                    w, C, static_cast<bf16*>(y), y_ctot, y_coff);
  return check_launch("of_cnn_upsample2");
}

extern "C" int of_cnn_upsample2_bwd(const void* dy, int dy_ctot, int dy_coff, int n, int h, int w, int C, void* dx,
                                    int dx_ctot, int dx_coff, void* stream) {
  OF_REQUIRE(dy && dx && h > 0 && w > 0 && C > 0, "of_cnn_upsample2_bwd: bad arguments");
  long long tot = (long long)n * h * w * C;
  upsample2_bwd_kernel<<<blocks_for(tot), 256, 0, as_stream(stream)>>>(
      static_cast<const bf16*>(dy), dy_ctot, dy_coff, n, h, w, C, static_cast<bf16*>(dx), dx_ctot, dx_coff);
  return check_launch("of_cnn_upsample2_bwd");
}

extern "C" int of_cnn_relu_bwd(void* g, int g_ctot, int g_coff, const void* y, int y_ctot, int y_coff, long long P,
                               int C, void* stream) {
  OF_REQUIRE(g && y && P > 0 && C > 0, "of_cnn_relu_bwd: bad arguments");
  relu_bwd_kernel<<<blocks_for(P * C), 256, 0, as_stream(stream)>>>(static_cast<bf16*>(g), g_ctot, g_coff,
                                                                     static_cast<const bf16*>(y), y_ctot, y_coff, P, C);
  return check_launch("of_cnn_relu_bwd");
}

extern "C" int of_cnn_flow_mse(const float* pred, const float* label, long long P, void* dpred, int g_ctot,
                               double* loss, void* stream) {
  OF_REQUIRE(pred && label && loss && P > 0 && (!dpred || g_ctot >= 2), "of_cnn_flow_mse: bad arguments");
  flow_mse_kernel<<<blocks_for(P), 256, 0, as_stream(stream)>>>(pred, label, P, static_cast<bf16*>(dpred), g_ctot,
                                                                 loss);
  return check_launch("of_cnn_flow_mse");
}

extern "C" int of_cnn_adam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2,
                           float eps, int step, void* stream) {
  OF_REQUIRE(w && g && m && v && n > 0 && step >= 1, "of_cnn_adam: bad arguments");
  float bc1 = (float)(1.0 - pow((double)b1, step)), bc2 = (float)(1.0 - pow((double)b2, step));
  adam_kernel<<<blocks_for(n), 256, 0, as_stream(stream)>>>(w, g, m, v, n, lr, b1, b2, eps, bc1, bc2);
  return check_launch("of_cnn_adam");
}

extern "C" int of_cnn_pack_weights(const float* w, int cout, int cin, int cout_pad, int cin_pad, int transpose_flip,
                                   void* out, void* stream) {
  OF_REQUIRE(w && out && cout > 0 && cin > 0 && cout_pad >= cout && cin_pad >= cin, "of_cnn_pack_weights: bad arguments");
  long long tot = 9LL * cout_pad * cin_pad;
  pack_weights_kernel<<<blocks_for(tot), 256, 0, as_stream(stream)>>>(w, cout, cin, cout_pad, cin_pad, transpose_flip,
                                                                       static_cast<bf16*>(out));
  return check_launch("of_cnn_pack_weights");
}

extern "C" int of_cnn_split_flow(const float* flow, int h, int w, float* u, float* v, int pitch, void* stream) {
  OF_REQUIRE(flow && u && v && h > 0 && w > 0 && pitch >= w, "of_cnn_split_flow: bad arguments");
  split_flow_kernel<<<blocks_for((long long)h * w), 256, 0, as_stream(stream)>>>(flow, h, w, u, v, pitch);
  return check_launch("of_cnn_split_flow");
}

extern "C" int of_cnn_conv3x3_wgrad_tc(const void* x, int x_ctot, int x_coff, const void* dy, int dy_ctot, int dy_coff,
                                       int n, int H, int W, int cin, int cout, float* dw, unsigned* err, void* stream) {
  OF_REQUIRE(x && dy && dw && err && n > 0 && H > 0 && W > 0 && cin > 0 && cout > 0 && cin <= 512 && cout <= 512,
             "of_cnn_conv3x3_wgrad_tc: bad arguments");
  OF_REQUIRE(x_ctot % 8 == 0 && x_coff % 8 == 0 && dy_ctot % 8 == 0 && dy_coff % 8 == 0 && x_coff + cin <= x_ctot &&
                 dy_coff + cout <= dy_ctot,
             "of_cnn_conv3x3_wgrad_tc: channel slices");
  int bw = W < WT_KP ? W : WT_KP;
  OF_REQUIRE(WT_KP % bw == 0 && W % bw == 0, "of_cnn_conv3x3_wgrad_tc: width %d", W);
  int bh = WT_KP / bw < H ? WT_KP / bw : H;
  OF_REQUIRE(H % bh == 0 && (WT_KP / bw) % bh == 0, "of_cnn_conv3x3_wgrad_tc: height %d", H);
  int nb = WT_KP / (bw * bh);
  OF_REQUIRE(n % nb == 0, "of_cnn_conv3x3_wgrad_tc: %d images of %d x %d", n, H, W);
  WgParams p;
  p.n = n;
  p.H = H;
  p.W = W;
  p.bw = bw;
  p.bh = bh;
  p.nb = nb;
  p.tiles_x = W / bw;
  p.tiles_per_group = (W / bw) * (H / bh);
  p.nchunk = (n / nb) * p.tiles_per_group;
  p.a_is_dy = cout >= cin;
  p.a_ch = p.a_is_dy ? cout : cin;
  p.b_ch = p.a_is_dy ? cin : cout;
  p.mtiles = (p.a_ch + 127) / 128;
  p.ntiles = (p.b_ch + 255) / 256;
  int nb_last = p.b_ch - (p.ntiles - 1) * 256;  // every N tile uses the same MMA N: the largest needed
  int nmax = p.ntiles > 1 ? 256 : nb_last;
  p.nmma = (nmax + 15) / 16 * 16;
  p.batoms = (p.nmma + 63) / 64;
  p.cin = cin;
  p.cout = cout;
  p.dw = dw;
  p.err = err;
  p.a_bytes = 2 * 8192;
  p.b_bytes = (uint32_t)p.batoms * 8192;
  p.stage_bytes = p.a_bytes + p.b_bytes;
  p.tmem_cols = p.nmma <= 32 ? 32 : (p.nmma <= 64 ? 64 : (p.nmma <= 128 ? 128 : 256));
  // split the pixel chunks so that about 4 CTAs per SM run, at least 8 chunks each
  const long long tiles = 9LL * p.mtiles * p.ntiles;
  long long ks = (4LL * kNumSMs + tiles - 1) / tiles;
  if (ks > p.nchunk / 8) ks = p.nchunk / 8;
  if (ks < 1) ks = 1;
  p.chunks_per_cta = (int)((p.nchunk + ks - 1) / ks);
  ks = (p.nchunk + p.chunks_per_cta - 1) / p.chunks_per_cta;
  CUtensorMap tma, tmb;
  {
    const void* ap = p.a_is_dy ? dy : x;
    int act = p.a_is_dy ? dy_ctot : x_ctot, aco = p.a_is_dy ? dy_coff : x_coff;
    uint64_t dims[4] = {(uint64_t)p.a_ch, (uint64_t)W, (uint64_t)H, (uint64_t)n};
    uint64_t st[3] = {(uint64_t)act * 2, (uint64_t)W * act * 2, (uint64_t)H * W * act * 2};
    uint32_t box[4] = {64, (uint32_t)bw, (uint32_t)bh, (uint32_t)nb};
    int rc = tmap_bf16(&tma, static_cast<const bf16*>(ap) + aco, 4, dims, st, box, 128);
    if (rc) return rc;
  }
  {
    const void* bp = p.a_is_dy ? x : dy;
    int bct = p.a_is_dy ? x_ctot : dy_ctot, bco = p.a_is_dy ? x_coff : dy_coff;
    uint64_t dims[4] = {(uint64_t)p.b_ch, (uint64_t)W, (uint64_t)H, (uint64_t)n};
    uint64_t st[3] = {(uint64_t)bct * 2, (uint64_t)W * bct * 2, (uint64_t)H * W * bct * 2};
    uint32_t box[4] = {64, (uint32_t)bw, (uint32_t)bh, (uint32_t)nb};
    int rc = tmap_bf16(&tmb, static_cast<const bf16*>(bp) + bco, 4, dims, st, box, 128);
    if (rc) return rc;
  }
  size_t smem = 1024 + (size_t)WT_STAGES * p.stage_bytes;
  size_t floor_smem = (size_t)p.tmem_cols * 456 + 1024;  // resident CTAs never exceed 512 TMEM columns
  if (smem < floor_smem) smem = floor_smem;
  {
    cudaError_t e = OF_SMEM_OPT_IN(wgrad_tc_kernel, smem);
    if (e != cudaSuccess)
      return set_error(OF_ERR_CUDA, "of_cnn_conv3x3_wgrad_tc: %zu B of shared memory: %s", smem, cudaGetErrorString(e));
  }
  dim3 grid((unsigned)ks, p.mtiles * p.ntiles, 9);
  wgrad_tc_kernel<<<grid, CV_THREADS, smem, as_stream(stream)>>>(tma, tmb, p);
  return check_launch("of_cnn_conv3x3_wgrad_tc");
}

extern "C" int of_cnn_flow_up(const float* flow, int h, int w, int factor, float* U, float* V, int pitch, float scale,
                              void* stream) {
  OF_REQUIRE(flow && U && V && h > 0 && w > 0 && factor >= 1 && factor <= 16 && pitch >= factor * w,
             "of_cnn_flow_up: bad arguments");
  dim3 g((factor * w + 255) / 256, factor * h);
  flow_up_kernel<<<g, 256, 0, as_stream(stream)>>>(flow, h, w, factor, U, V, pitch, scale);
  return check_launch("of_cnn_flow_up");
}
