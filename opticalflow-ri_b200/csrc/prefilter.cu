// A1 Gaussian prefilter (src/gaussian_filter.py:24-94), bit-exact.
//
// One CTA filters a 64x32 output tile.  The input tile (with a K/2 halo, the
// reference's border mapping applied per axis) is staged in shared memory, the row
// pass runs over every staged row (halo rows included, because the column pass of the
// reference reads row-filtered values), then the column pass writes the tile.
// Arithmetic is float32 multiply then add, taps j = 0..K-1 against t[x+2h-j]: the exact
// order of convolveDirect.  HBM traffic: one read of the frame (uint8 or float32) and
// one float32 write.
#include "common.cuh"

namespace ofb {

constexpr int PF_TW = 64, PF_TH = 32, PF_MAXK = 15;  // the pyramid's prefilters (3 and 5 taps)
constexpr int PF_MAXK_LARGE = 81;                     // the Liu-Shen warp's 73-tap smoothing

struct PfTaps {
  float k[PF_MAXK_LARGE];
};

// Border of convolveSeparableFilter (:62-66): coordinate c of a line of length n with
// half width h maps to line[-1-c] left of the line and line[c-h] right of it.
__device__ __forceinline__ int pf_map(int c, int n, int h) {
  if (c < 0) c = -1 - c;
  else if (c >= n) c = c - h;
  return clampi(c, 0, n - 1);  // only reached for outputs outside the image
}

// KC > 0: the tap count is the compile-time KC (the pyramid's 3- and 5-tap prefilters), so
// the tile widths are constants (no integer division per staged element) and the tap loops
// carry no bound test; KC = 0: K taps at run time, up to MAXK.
template <typename Tin, int MAXK, int KC = 0>
__global__ void __launch_bounds__(256) prefilter_kernel(const Tin* __restrict__ src, int sp, float* __restrict__ dst,
                                                        int dp, int H, int W, const PfTaps taps, int Krt) {
  extern __shared__ float sm[];
  const int K = KC > 0 ? KC : Krt;
  const int h = K >> 1;
  const int iw = PF_TW + 2 * h, ih = PF_TH + 2 * h;
  float* tin = sm;             // ih x iw
  float* trow = sm + ih * iw;  // ih x PF_TW
  const int x0 = blockIdx.x * PF_TW, y0 = blockIdx.y * PF_TH;
  const int tid = threadIdx.x;
  for (int i = tid; i < ih * iw; i += blockDim.x) {
    int ly = i / iw, lx = i - ly * iw;
    int gy = pf_map(y0 - h + ly, H, h), gx = pf_map(x0 - h + lx, W, h);
    tin[i] = (float)src[(size_t)gy * sp + gx];
  }
  __syncthreads();
  // row pass: out[x] = sum_j k[j] * P(x + h - j), P(c) = tin[.][c - (x0 - h)]
  for (int i = tid; i < ih * PF_TW; i += blockDim.x) {
    int ly = i / PF_TW, lx = i - ly * PF_TW;
    const float* t = tin + ly * iw + lx + 2 * h;
    float acc = 0.0f;
#pragma unroll(MAXK <= PF_MAXK ? MAXK : 8)
    for (int j = 0; j < MAXK; j++)
      if (KC > 0 || j < K) acc = __fadd_rn(acc, __fmul_rn(t[-j], taps.k[j]));
    trow[i] = acc;
  }
  __syncthreads();
  for (int i = tid; i < PF_TH * PF_TW; i += blockDim.x) {
    int ly = i / PF_TW, lx = i - ly * PF_TW;
    int y = y0 + ly, x = x0 + lx;
    if (y >= H || x >= W) continue;
    const float* t = trow + (ly + 2 * h) * PF_TW + lx;
    float acc = 0.0f;
#pragma unroll(MAXK <= PF_MAXK ? MAXK : 8)
    for (int j = 0; j < MAXK; j++)
      if (KC > 0 || j < K) acc = __fadd_rn(acc, __fmul_rn(t[-j * PF_TW], taps.k[j]));
    dst[(size_t)y * dp + x] = acc;
  }
}

template <typename Tin>
static int launch_prefilter(const Tin* src, int sp, float* dst, int dp, int H, int W, const float* taps, int K,
                            void* stream, const char* name) {
  OF_REQUIRE(!bad_plane(src, H, W, sp) && !bad_plane(dst, H, W, dp), "%s: bad plane", name);
  OF_REQUIRE(taps && K >= 1 && K <= PF_MAXK_LARGE && (K & 1), "%s: K must be odd and <= %d", name, PF_MAXK_LARGE);
  OF_REQUIRE(H >= K / 2 && W >= K / 2, "%s: image smaller than the half kernel", name);
  OF_REQUIRE((const void*)src != (const void*)dst, "%s: src and dst alias", name);
  PfTaps t{};
  for (int j = 0; j < K; j++) t.k[j] = taps[j];
  int h = K / 2;
  size_t smem = sizeof(float) * ((size_t)(PF_TH + 2 * h) * (PF_TW + 2 * h) + (size_t)(PF_TH + 2 * h) * PF_TW);
  dim3 grid((W + PF_TW - 1) / PF_TW, (H + PF_TH - 1) / PF_TH);
  if (K <= PF_MAXK) {
    if (K == 5)
      prefilter_kernel<Tin, 5, 5><<<grid, 256, smem, as_stream(stream)>>>(src, sp, dst, dp, H, W, t, K);
    else if (K == 3)
      prefilter_kernel<Tin, 3, 3><<<grid, 256, smem, as_stream(stream)>>>(src, sp, dst, dp, H, W, t, K);
    else
      prefilter_kernel<Tin, PF_MAXK><<<grid, 256, smem, as_stream(stream)>>>(src, sp, dst, dp, H, W, t, K);
  } else {
    // up to 83 KB of staged tile for 81 taps
    cudaError_t e = OF_SMEM_OPT_IN((prefilter_kernel<Tin, PF_MAXK_LARGE>), 96 * 1024);
    if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "%s: %s", name, cudaGetErrorString(e));
    prefilter_kernel<Tin, PF_MAXK_LARGE><<<grid, 256, smem, as_stream(stream)>>>(src, sp, dst, dp, H, W, t, K);
  }
  return check_launch(name);
}

}  // namespace ofb

using namespace ofb;

extern "C" int of_prefilter_f32(const float* src, int src_pitch, float* dst, int dst_pitch, int H, int W,
                                const float* taps, int K, void* stream) {
  return launch_prefilter<float>(src, src_pitch, dst, dst_pitch, H, W, taps, K, stream, "of_prefilter_f32");
}

extern "C" int of_prefilter_u8(const uint8_t* src, int src_pitch, float* dst, int dst_pitch, int H, int W,
                               const float* taps, int K, void* stream) {
  return launch_prefilter<uint8_t>(src, src_pitch, dst, dst_pitch, H, W, taps, K, stream, "of_prefilter_u8");
}
