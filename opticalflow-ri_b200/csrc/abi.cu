// Error reporting, version and the small elementwise entry points of the C ABI.
#include <string.h>

#include <atomic>

#include "common.cuh"
#include "tma.cuh"

namespace ofb {

static thread_local char g_err[1024] = "";
static std::atomic<unsigned long long> g_launches{0};

int set_error(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int tmap_encode(CUtensorMap* map, CUtensorMapDataType dtype, const void* base, int rank, const uint64_t* dims,
                       const uint64_t* strides_bytes, const uint32_t* box, CUtensorMapSwizzle swz) {
  static EncodeTiledFn encode = nullptr;
  if (!encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn)
      return set_error(OF_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    encode = reinterpret_cast<EncodeTiledFn>(fn);
  }
  if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) return set_error(OF_ERR_INVALID, "tensor base not 16-byte aligned");
  if (rank < 1 || rank > 5) return set_error(OF_ERR_INVALID, "tensor map rank %d", rank);
  cuuint64_t d[5], s[4];
  cuuint32_t b[5], e[5] = {1, 1, 1, 1, 1};
  for (int i = 0; i < rank; i++) {
    d[i] = dims[i];
    b[i] = box[i];
  }
  for (int i = 0; i + 1 < rank; i++) {
    if (strides_bytes[i] % 16) return set_error(OF_ERR_INVALID, "tensor stride not a multiple of 16 bytes");
    s[i] = strides_bytes[i];
  }
  CUresult r = encode(map, dtype, (cuuint32_t)rank, const_cast<void*>(base), d, s, b, e, CU_TENSOR_MAP_INTERLEAVE_NONE,
                      swz, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(OF_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return OF_OK;
}

int tmap_f32(CUtensorMap* map, const void* base, int rank, const uint64_t* dims, const uint64_t* strides_bytes,
             const uint32_t* box) {
  if (rank > 3) return set_error(OF_ERR_INVALID, "tmap_f32: rank %d", rank);
  return tmap_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, base, rank, dims, strides_bytes, box,
                     CU_TENSOR_MAP_SWIZZLE_NONE);
}

int tmap_bf16(CUtensorMap* map, const void* base, int rank, const uint64_t* dims, const uint64_t* strides_bytes,
              const uint32_t* box, int swizzle_bytes) {
  CUtensorMapSwizzle swz;
  switch (swizzle_bytes) {
    case 0: swz = CU_TENSOR_MAP_SWIZZLE_NONE; break;
    case 32: swz = CU_TENSOR_MAP_SWIZZLE_32B; break;
    case 64: swz = CU_TENSOR_MAP_SWIZZLE_64B; break;
    case 128: swz = CU_TENSOR_MAP_SWIZZLE_128B; break;
    default: return set_error(OF_ERR_INVALID, "tmap_bf16: swizzle %d", swizzle_bytes);
  }
  if (swizzle_bytes && box[0] * 2u != (uint32_t)swizzle_bytes)
    return set_error(OF_ERR_INVALID, "tmap_bf16: inner box of %u B does not match the %d B swizzle", box[0] * 2u,
                     swizzle_bytes);
  return tmap_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, base, rank, dims, strides_bytes, box, swz);
}

int check_launch(const char* what, long long nlaunch) {
  g_launches.fetch_add((unsigned long long)nlaunch, std::memory_order_relaxed);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return OF_OK;
}

template <typename T>
__global__ void to_f32_kernel(const T* __restrict__ src, int sp, float* __restrict__ dst, int dp, int H, int W) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x < W) dst[(size_t)y * dp + x] = (float)src[(size_t)y * sp + x];
}

__global__ void accumulate_kernel(float* __restrict__ dst, const float* __restrict__ src, int pitch, int W) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x < W) {
    size_t i = (size_t)y * pitch + x;
    dst[i] = __fadd_rn(dst[i], src[i]);
  }
}

__global__ void scale_kernel(const float* __restrict__ src, float* __restrict__ dst, float s, int pitch, int W) {
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x < W) {
    size_t i = (size_t)y * pitch + x;
    dst[i] = __fmul_rn(src[i], s);
  }
}

}  // namespace ofb

using namespace ofb;

extern "C" int of_version(void) { return 100; }

extern "C" unsigned long long of_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

extern "C" int of_last_error(char* buf, size_t n) {
  size_t len = strlen(g_err);
  if (buf && n) {
    size_t c = len < n - 1 ? len : n - 1;
    memcpy(buf, g_err, c);
    buf[c] = 0;
  }
  return (int)len;
}

extern "C" int of_u8_to_f32(const uint8_t* src, int src_pitch, float* dst, int dst_pitch, int H, int W,
                            void* stream) {
  OF_REQUIRE(!bad_plane(src, H, W, src_pitch) && !bad_plane(dst, H, W, dst_pitch), "of_u8_to_f32: bad plane");
  dim3 grid((W + 255) / 256, H);
  to_f32_kernel<uint8_t><<<grid, 256, 0, as_stream(stream)>>>(src, src_pitch, dst, dst_pitch, H, W);
  return check_launch("of_u8_to_f32");
}

extern "C" int of_u16_to_f32(const uint16_t* src, int src_pitch, float* dst, int dst_pitch, int H, int W,
                             void* stream) {
  OF_REQUIRE(!bad_plane(src, H, W, src_pitch) && !bad_plane(dst, H, W, dst_pitch), "of_u16_to_f32: bad plane");
  dim3 grid((W + 255) / 256, H);
  to_f32_kernel<uint16_t><<<grid, 256, 0, as_stream(stream)>>>(src, src_pitch, dst, dst_pitch, H, W);
  return check_launch("of_u16_to_f32");
}

extern "C" int of_accumulate(float* dst, const float* src, int H, int W, int pitch, void* stream) {
  OF_REQUIRE(!bad_plane(dst, H, W, pitch) && src, "of_accumulate: bad plane");
  dim3 grid((W + 255) / 256, H);
  accumulate_kernel<<<grid, 256, 0, as_stream(stream)>>>(dst, src, pitch, W);
  return check_launch("of_accumulate");
}

extern "C" int of_scale(const float* src, float* dst, float s, int H, int W, int pitch, void* stream) {
  OF_REQUIRE(!bad_plane(dst, H, W, pitch) && src, "of_scale: bad plane");
  dim3 grid((W + 255) / 256, H);
  scale_kernel<<<grid, 256, 0, as_stream(stream)>>>(src, dst, s, pitch, W);
  return check_launch("of_scale");
}

namespace ofb {
// ORs `bit` into *status when any sample of the plane is NaN or Inf (one atomic per block).
__global__ void check_finite_kernel(const float* __restrict__ p, int H, int W, int pitch, int* status, int bit) {
  int bad = 0;
  for (int y = blockIdx.y; y < H; y += gridDim.y)
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x)
      bad |= !isfinite(p[(size_t)y * pitch + x]);
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(status, bit);
}

// Liu-Shen convergence: OF_ST_NOT_CONVERGED when the solve ran all `maxnum` sweeps and its
// last error is still above `tol`, or when it failed (iters < 0).
__global__ void ls_status_kernel(const int* iters, const double* err, int maxnum, double tol, int* status) {
  const int k = *iters;
  if (k < 0 || (k >= maxnum && !(*err <= tol))) atomicOr(status, OF_ST_NOT_CONVERGED);
}
__global__ void status_or_kernel(const int* src, int* dst) { atomicOr(dst, *src); }

int status_or(const int* src, int* dst, cudaStream_t stream) {
  status_or_kernel<<<1, 1, 0, stream>>>(src, dst);
  return check_launch("status_or");
}
}  // namespace ofb

extern "C" int of_check_finite(const float* p, int H, int W, int pitch, int* status, int bit, void* stream) {
  OF_REQUIRE(!bad_plane(p, H, W, pitch) && status, "of_check_finite: bad plane");
  dim3 grid((W + 255) / 256 < 4 ? (W + 255) / 256 : 4, H < 64 ? H : 64);
  check_finite_kernel<<<grid, 256, 0, as_stream(stream)>>>(p, H, W, pitch, status, bit);
  return check_launch("of_check_finite");
}

extern "C" int of_ls_status(const int* iters, const double* err, int maxnum, double tol, int* status, void* stream) {
  OF_REQUIRE(iters && err && status, "of_ls_status: null pointer");
  ls_status_kernel<<<1, 1, 0, as_stream(stream)>>>(iters, err, maxnum, tol, status);
  return check_launch("of_ls_status");
}
