/*
 * ofb200 — C ABI of the B200 (sm_100a) dense pyramidal optical-flow kernels.
 *
 * Conventions
 *  - Every entry point returns an int status: OF_OK (0) or a negative OF_ERR_* code;
 *    of_last_error() returns the message of the calling thread's last failure.
 *  - All image / flow buffers are DEVICE pointers to row-major float32 planes of H rows
 *    and W columns with a row pitch of `pitch` elements (pitch >= W).  U is the +x
 *    (column) displacement, V the +y (row) displacement.
 *  - `stream` is a cudaStream_t (NULL = legacy default stream).  Calls only enqueue work:
 *    results are ready when the stream is synchronised.  Values reported "to device"
 *    (iteration counts, errors) are written to device memory for the same reason.
 *  - Entry points that need scratch memory take a caller-provided device workspace of at
 *    least the size returned by the matching *_workspace_size() call; they never
 *    allocate.  Distinct streams need distinct workspaces.
 *  - No C++ exception crosses this boundary.  The library holds no state besides the
 *    per-thread error message, a launch counter and the fixed scratch array of
 *    of_ls_solve_noalloc.
 *
 * Each declaration names the reference interface it replaces (OpticalFlow-RI,
 * file:line).
 */
#ifndef OFB200_H
#define OFB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OF_OK 0
#define OF_ERR_INVALID (-1)   /* bad argument (size, pointer, pitch, parameter) */
#define OF_ERR_CUDA (-2)      /* a CUDA launch or runtime call failed */
#define OF_ERR_WORKSPACE (-3) /* workspace missing or smaller than required */
#define OF_ERR_UNSUPPORTED (-4)

#define OF_FILTER_BILINEAR 0
#define OF_FILTER_BICUBIC 1

/* Library version (major*10000 + minor*100 + patch). */
int of_version(void);

/* Number of CUDA kernels this library has launched in the process (all threads); lets a
 * caller count the launches of a timed region. */
unsigned long long of_launch_count(void);

/* Copies the calling thread's last error message into buf (always NUL-terminated);
 * returns its full length. */
int of_last_error(char* buf, size_t n);

/* Host memcpy of `bytes` between two non-overlapping HOST buffers, split over a small
 * persistent pool of threads when it is 1 MiB or more (the staging copies of host-buffer
 * calls: numpy frame -> pinned upload buffer, pinned download buffer -> numpy result).
 * Blocking; one pooled copy runs at a time; a forked child copies on its own thread. */
int of_host_copy(void* dst, const void* src, size_t bytes);

/* ---------------------------------------------------------------------------------
 * A1 Gaussian prefilter — replaces gaussian_filterPx / convolveSeparableFilter
 * (src/gaussian_filter.py:54-94).  Separable K-tap FIR (K odd, 1..81; H, W >= K/2), row pass then
 * column pass, with the reference's border (left mirrored, right copied in order) and
 * float32 arithmetic order; bit-exact with the reference.  `taps` is a HOST array of K
 * floats (e.g. prepareGaussianKernel(sigma, K), src/gaussian_filter.py:47-52).
 * src and dst may not alias.  of_prefilter_u8 reads uint8 frames (fused cast).
 * ------------------------------------------------------------------------------- */
int of_prefilter_f32(const float* src, int src_pitch, float* dst, int dst_pitch, int H, int W,
                     const float* taps, int K, void* stream);
int of_prefilter_u8(const uint8_t* src, int src_pitch, float* dst, int dst_pitch, int H, int W,
                    const float* taps, int K, void* stream);

/* uint8 / uint16 -> float32 plane conversion (the examples' imread(...).astype(np.float32);
 * 10- and 12-bit PIV frames arrive in 16-bit containers). */
int of_u8_to_f32(const uint8_t* src, int src_pitch, float* dst, int dst_pitch, int H, int W, void* stream);
int of_u16_to_f32(const uint16_t* src, int src_pitch, float* dst, int dst_pitch, int H, int W, void* stream);

/* ---------------------------------------------------------------------------------
 * A2 antialiased resize — replaces imresize (src/GenericPyramidalOpticalFlow.py:66-67,
 * PIL BICUBIC) and the Farneback imresize (src/Farneback_PyCL.py:61-62, PIL BILINEAR):
 * Pillow Image.resize on a mode 'F' image (horizontal pass into a float32 intermediate,
 * then vertical pass; double accumulation).  Same size is a copy.
 * ------------------------------------------------------------------------------- */
size_t of_resize_workspace_size(int Hs, int Ws, int Hd, int Wd, int filter);
int of_resize(const float* src, int Hs, int Ws, int src_pitch, float* dst, int Hd, int Wd, int dst_pitch, int filter,
              void* workspace, size_t workspace_bytes, void* stream);
/* The same resize from weight tables the caller computed once per (size, filter) and keeps
 * (same results bit for bit): of_resize_table fills one axis's table (in -> out samples,
 * of_resize_table_size bytes, DEVICE memory); of_resize_tabled takes the horizontal
 * (Ws -> Wd) and vertical (Hs -> Hd) tables (either may be NULL when that axis keeps its
 * size) and, when both axes change, a workspace of Hs * Wd floats.  Each table must be
 * the one built for that axis's (in, out, filter): the kernels trust its contents.  Worth
 * it for strong downscales, whose many taps per output make the weights the dominant cost. */
size_t of_resize_table_size(int in, int out, int filter);
int of_resize_table(int in, int out, int filter, void* table, size_t table_bytes, void* stream);
int of_resize_tabled(const float* src, int Hs, int Ws, int src_pitch, float* dst, int Hd, int Wd, int dst_pitch,
                     int filter, const void* table_h, const void* table_v, void* workspace, size_t workspace_bytes,
                     void* stream);

/* ---------------------------------------------------------------------------------
 * A3 flow upsample — replaces the RectBivariateSpline branch of updateNextPyramidalLevel
 * (src/GenericPyramidalOpticalFlow.py:151-171): cubic interpolating (not-a-knot) spline
 * of the h x w field on x_i = i/w, y_i = i/h evaluated at X/W, Y/H (clamped to the
 * last sample), rounded to float32, then multiplied by `scale` (float32) — pass 1.0f
 * when the level does not scale.  h, w >= 4.
 * ------------------------------------------------------------------------------- */
size_t of_spline_workspace_size(int h, int w, int H, int W);
int of_spline_upsample(const float* src, int h, int w, int src_pitch, float* dst, int H, int W, int dst_pitch,
                       float scale, void* workspace, size_t workspace_bytes, void* stream);
/* Both flow components of one level transition in the same launches (twice the lines in
 * flight for the serial spline recurrences): results equal two of_spline_upsample calls.
 * Workspace: 2 * of_spline_workspace_size(h, w, H, W) bytes. */
int of_spline_upsample_pair(const float* src_u, const float* src_v, int h, int w, int src_pitch, float* dst_u,
                            float* dst_v, int H, int W, int dst_pitch, float scale_u, float scale_v, void* workspace,
                            size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------------------
 * A4 symmetric bilinear warp — replaces doBiLinearWarping as called at
 * src/GenericPyramidalOpticalFlow.py:197-200: O0 = I0 sampled at (y - V/2, x - U/2),
 * O1 = I1 sampled at (y + V/2, x + U/2); round-half-even base, replicate borders.
 * ------------------------------------------------------------------------------- */
int of_warp_pair_bilinear(const float* I0, const float* I1, const float* U, const float* V, float* O0, float* O1,
                          int H, int W, int pitch, void* stream);
/* doBiLinearWarping(img, coordsY, coordsX) itself (src/GenericPyramidalOpticalFlow.py:69-115)
 * for arbitrary float32 coordinate planes. */
int of_warp_bilinear_coords(const float* img, const float* coordsY, const float* coordsX, float* out, int H, int W,
                            int pitch, void* stream);

/* dst = dst + src (the driver's Uaccum += U, src/GenericPyramidalOpticalFlow.py:412-413),
 * and dst = src * s (float32). */
int of_accumulate(float* dst, const float* src, int H, int W, int pitch, void* stream);
int of_scale(const float* src, float* dst, float s, int H, int W, int pitch, void* stream);

/* ---------------------------------------------------------------------------------
 * A6/A7 Horn-Schunck — replaces HSOpticalFlowAlgoAdapter.compute / HS
 * (src/HornSchunck.py:28-104): 2x2-cube derivatives, `niter` Jacobi sweeps with the
 * 3x3 averaging kernel (mirror borders), bit-exact with the reference.  I0 = frame at t0,
 * I1 = frame at t1.  U, V: initial flow in, result out.  err_out (device, optional):
 * (||U-U0||_F + ||V-V0||_F) / (H*W) as float64.
 * ------------------------------------------------------------------------------- */
size_t of_hs_workspace_size(int H, int W, int pitch);
/* computeDerivatives (src/HornSchunck.py:106-126) as HS calls it: fx, fy, ft of the pair
 * (I0 = frame t0, I1 = frame t1). */
int of_hs_derivatives(const float* I0, const float* I1, float* fx, float* fy, float* ft, int H, int W, int pitch,
                      void* stream);
int of_hs_solve(const float* I0, const float* I1, float* U, float* V, int H, int W, int pitch, float alpha,
                int niter, double* err_out, void* workspace, size_t workspace_bytes, void* stream);
/* The same solve in one persistent launch (of_hs_batch with one pair, device work queue):
 * the same results bit for bit, for callers that solve one pair at a time (its latency is
 * a chain of passes rather than a chain of launches).  Beside other launches on other
 * streams it stays correct but gains nothing: there of_hs_solve, whose short launches
 * interleave with the other streams' work, is the faster choice.  The workspace is
 * of_hs_workspace_size's.  A bounded wait that gave up (OF_ST_WAIT_TIMEOUT) makes err_out NaN. */
int of_hs_solve_persistent(const float* I0, const float* I1, float* U, float* V, int H, int W, int pitch,
                           float alpha, int niter, double* err_out, void* workspace, size_t workspace_bytes,
                           void* stream);

/* ---------------------------------------------------------------------------------
 * Batches of frame pairs (the batched workload of uneven pairs).  Per-pair status words:
 * bits ORed into a caller's DEVICE int array (zero it before the first call).
 * ------------------------------------------------------------------------------- */
#define OF_ST_NONFINITE_INPUT 0x1  /* a frame holds NaN or Inf */
#define OF_ST_WAIT_TIMEOUT 0x2     /* a bounded device wait gave up; the pair's result is invalid */
#define OF_ST_NOT_CONVERGED 0x4    /* an iterative solve used all its sweeps above its tolerance */
#define OF_ST_SINGULAR 0x8         /* singular per-pixel systems (LK det < eps, LS det == 0) */
#define OF_ST_NONFINITE_OUTPUT 0x10 /* the result holds NaN or Inf */

/* Tuning of a batched launch: tile_shape indexes the kernel's table of (region width,
 * region height, sweeps per pass) shapes, listed by of_hs_batch_shape(). */
typedef struct OfTuning {
  int tile_shape;
  int streams;   /* host-side concurrency of callers that use streams; unused by the kernels */
  int hs_arithmetic; /* OF_HS_EXACT (bit-exact with the reference) or OF_HS_FAST (float32 averaging) */
  int hs_schedule;   /* OF_HS_SCHED_*: how the persistent Horn-Schunck launch hands out its tiles */
} OfTuning;
#define OF_HS_EXACT 0
#define OF_HS_FAST 1
/* AUTO: when the device can hold one CTA per tile, a launch of one CTA per tile that runs
 * the RESIDENT schedule if all its CTAs get an SM at once and the QUEUE otherwise (the CTAs
 * decide at their start, within a bounded poll: other work holding SMs only costs speed);
 * else QUEUE.  of_hs_batch_schedule reports which one ran.
 * QUEUE: (pass, pair, tile) items from a device ticket counter.
 * RESIDENT: one CTA per tile for the whole solve, its derivative planes and flow kept in
 * shared memory, only the halo ring exchanged through global memory (OF_ERR_INVALID when
 * the tiles outnumber the resident CTAs).
 * CLUSTER: one pair of at most 16 tiles of 64 x 64 (256 x 256 and smaller) on one
 * thread-block cluster, the halo exchanged through distributed shared memory with one
 * cluster barrier per sweep (OF_ERR_INVALID for other batches, OF_ERR_UNSUPPORTED where
 * the device cannot hold the cluster).  At 256 x 256 its per-sweep cluster barrier makes
 * it slower than RESIDENT; AUTO does not pick it.
 * The schedules give identical results. */
#define OF_HS_SCHED_AUTO 0
#define OF_HS_SCHED_QUEUE 1
#define OF_HS_SCHED_RESIDENT 2
#define OF_HS_SCHED_CLUSTER 3

/* One Horn-Schunck pair of a batch: DEVICE planes of H x W float32 with row pitch `pitch`;
 * U, V hold the initial flow and receive the result. */
typedef struct OfHsBatchPair {
  const float* I0;
  const float* I1;
  float* U;
  float* V;
  int H, W, pitch;
  float alpha;
  int niter;
} OfHsBatchPair;

/* Horn-Schunck of n pairs (any sizes) in ONE persistent launch — replaces n calls of
 * HSOpticalFlowAlgoAdapter.compute / HS (src/HornSchunck.py:34-104), bit-exact like
 * of_hs_solve.  Work items (pass, pair, tile) come from a device queue; a pass of a pair
 * waits for its previous pass with a bounded poll of at most `wait_limit` iterations, after
 * which the pair gets OF_ST_WAIT_TIMEOUT and is skipped (the launch still ends).  The
 * derivative pass sets OF_ST_NONFINITE_INPUT for frames with NaN / Inf, the last sweep pass
 * OF_ST_NONFINITE_OUTPUT.  status: DEVICE int[n].  The HS error value is not computed.
 * tuning->hs_arithmetic OF_HS_FAST averages in float32 (corner and edge sums, two
 * multiply-adds) instead of the reference's float64 sum: within float32 rounding. */
int of_hs_batch_shape(int index, int* region_w, int* region_h, int* sweeps_per_pass);
/* Status helpers for batches (no counterpart in the reference, which lets NaN propagate):
 * of_check_finite ORs `bit` into *status (DEVICE int) when the plane holds NaN or Inf;
 * of_ls_status ORs OF_ST_NOT_CONVERGED when a Liu-Shen solve's DEVICE sweep count reached
 * maxnum with its last error above tol (or the solve failed). */
int of_check_finite(const float* p, int H, int W, int pitch, int* status, int bit, void* stream);
int of_ls_status(const int* iters, const double* err, int maxnum, double tol, int* status, void* stream);
size_t of_hs_batch_workspace_size(const OfHsBatchPair* pairs, int n);
int of_hs_batch(const OfHsBatchPair* pairs, int n, const OfTuning* tuning, int* status, long long wait_limit,
                void* workspace, size_t workspace_bytes, void* stream);
/* The schedule the last AUTO launch of of_hs_batch over this pair list and workspace ran:
 * OF_HS_SCHED_RESIDENT or OF_HS_SCHED_QUEUE into *schedule (OF_HS_SCHED_AUTO when that launch
 * chose statically: an explicit schedule, or tiles beyond one CTA each).  Waits for `stream`. */
int of_hs_batch_schedule(const OfHsBatchPair* pairs, int n, const void* workspace, size_t workspace_bytes,
                         int* schedule, void* stream);

/* ---------------------------------------------------------------------------------
 * A8/A9 Liu-Shen physics-based optimiser — replaces LiuShenOpticalFlowAlgoAdapter.compute /
 * physicsBasedOpticalFlowLiuShen (src/PhysicsBasedOpticalFlowLiuShen.py:33-158).
 * Frames are normalised by their maxima; sweeps run while err > tol and k < maxnum
 * (reference: tol 1e-8, maxnum 60); bit-exact with the reference's float32 fields.
 * U, V: initial flow in, result out.  iters_out / err_out: DEVICE int / double
 * (optional): sweeps run and the last sweep's error.
 * ------------------------------------------------------------------------------- */
size_t of_ls_workspace_size(int H, int W, int pitch, int maxnum);
/* The eight per-pixel coefficient planes of the solver (IIx, IIy, II, Ixt, Iyt and
 * B11, B12, B22 of generate_invmatrix, src/PhysicsBasedOpticalFlowLiuShen.py:47-73,124-128)
 * from a normalised frame I1n and Et = I2n - I1n; coef holds 8 stacked H x W planes. */
int of_ls_coefficients(const float* I1n, const float* Et, float* coef, int H, int W, int pitch, float h, void* stream);
int of_ls_solve(const float* I0, const float* I1, float* U, float* V, int H, int W, int pitch, float h, int maxnum,
                double tol, int* iters_out, double* err_out, void* workspace, size_t workspace_bytes, void* stream);
/* The same solve (same reference interface, same workspace) with a choice of arithmetic:
 * OF_LS_EXACT is of_ls_solve (bit-exact with the reference's float32 fields: its stencils
 * are float64 sums in the reference's order); OF_LS_FAST computes the sweep in float32
 * with fused multiply-adds (fields within float32 rounding of the reference's, <= 1e-3 px
 * of the algorithm's float64 answer; the stop rule is evaluated on its own float32 changes). */
#define OF_LS_EXACT 0
#define OF_LS_FAST 1
int of_ls_solve_mode(const float* I0, const float* I1, float* U, float* V, int H, int W, int pitch, float h,
                     int maxnum, double tol, int mode, int* iters_out, double* err_out, void* workspace,
                     size_t workspace_bytes, void* stream);

/* The same Liu-Shen solve for callers that cannot allocate device memory at call time
 * (a framework that owns all allocations, a plugin that must not touch the process's
 * allocator, a real-time loop that cannot afford cudaMalloc's synchronisation).  It has no
 * counterpart in the reference.  Its scratch is a fixed OF_LS_NOALLOC_SCRATCH_BYTES array
 * inside the library (held by every GPU that loads it), so it takes no workspace and
 * rejects, with OF_ERR_INVALID, any size whose of_ls_workspace_size exceeds that array
 * (256 x 256 with 60 sweeps fits).  The first call on each device looks up the array's
 * device address; make it before any stream capture.  All calls share the array: calls
 * that overlap on the GPU race.  Results equal of_ls_solve's. */
#define OF_LS_NOALLOC_SCRATCH_BYTES (4 * 1024 * 1024)
int of_ls_solve_noalloc(const float* I0, const float* I1, float* U, float* V, int H, int W, int pitch, float h,
                        int maxnum, double tol, int* iters_out, double* err_out, void* stream);

/* ---------------------------------------------------------------------------------
 * A10/A11 dense Lucas-Kanade — replaces denseLucasKanade_PyCl.compute
 * (src/denseLucasKanade_PyCL.py:113-169) and the lkDense kernel
 * (src/pyrlkDenseLargeW.cl:304-669): per pixel, Scharr gradients over a
 * (2*half_win+1)^2 window (half_win <= 15), <= niter Newton steps on a bilinear J
 * (float32 weights), stop at |delta| < 0.01.  asym: {left,right,top,bottom} window
 * masks (HOST array of 0 / 1 values, may be NULL = all 0).  status (uint8, optional): 1 = tracked,
 * 0 = singular / left the image.  err (float, optional): the kernel's mean |J-I|.
 * Pixels with a singular gradient matrix keep their input U, V.
 * ------------------------------------------------------------------------------- */
int of_lk_dense(const float* I, const float* J, float* U, float* V, int H, int W, int pitch, int half_win, int niter,
                const int* asym, uint8_t* status, float* err, void* stream);

/* ---------------------------------------------------------------------------------
 * A12-A19 Farneback — replaces Farneback_PyCL.compute (src/Farneback_PyCL.py:461-603)
 * and its kernels (src/optical_flow_farneback.cl:72-429).  The planar 5-coefficient
 * fields (RA, RB, M) are 5*H x W stacks with row pitch `pitch`.
 * ------------------------------------------------------------------------------- */
typedef struct {
  int polyN;           /* 5 or 7 */
  float g[8], xg[8], xxg[8]; /* polyN+1 taps (centre first), FarnebackPrepareGaussian */
  float ig[4];         /* invG[1,1], invG[0,3], invG[3,3], invG[5,5] as float32 */
} of_fb_poly_consts;

/* gaussianBlur / gaussianBlur5 (:160-253): `planes` stacked planes, reflect-101 borders,
 * half kernel gk[0..kh] (centre first, HOST array, kh <= 32). */
int of_fb_blur(const float* src, float* dst, int H, int W, int pitch, int planes, const float* gk, int kh,
               void* stream);
/* boxFilter5 (:350-406), clamped borders. */
int of_fb_box5(const float* src, float* dst, int H, int W, int pitch, int kh, void* stream);
/* polynomialExpansion (:72-133): src H x W -> dst 5H x W. consts: HOST struct. */
int of_fb_polyexp(const float* src, float* dst, int H, int W, int pitch, const of_fb_poly_consts* consts,
                  void* stream);
/* gaussianBlur with a 3-tap kernel (kh = 1, reflect-101) followed by polynomialExpansion
 * (:160-253 then :72-133), as the full-size level of Farneback_PyCL.compute runs them
 * (src/Farneback_PyCL.py:562-583, no resize between): one launch, the blurred frame never
 * stored.  Equals of_fb_blur(src, tmp, ..., 1, gk, 1) then of_fb_polyexp(tmp, dst, ...)
 * bit for bit.  gk: HOST array of 2 taps (centre first); polyN 5 or 7; H, W >= 3. */
int of_fb_polyexp_blurred(const float* src, float* dst, int H, int W, int pitch, const float* gk,
                          const of_fb_poly_consts* consts, void* stream);
/* updateMatrices (:256-348): M from the flow and the two expansions. */
int of_fb_update_matrices(const float* flowx, const float* flowy, const float* R0, const float* R1, float* M, int H,
                          int W, int pitch, void* stream);
/* updateFlow (:408-429). */
int of_fb_update_flow(const float* M, float* flowx, float* flowy, int H, int W, int pitch, void* stream);
/* One Farneback iteration fused (updateFlowGaussianBlur, src/Farneback_PyCL.py:441-456):
 * blur5(M_in) with the half kernel wk[0..kh] (HOST array) -> updateFlow -> (if
 * update_matrices) updateMatrices into M_out.  Same result as the three kernels above.
 * M_in and M_out must not alias (the blur reads a (2kh+1)^2 neighbourhood). */
int of_fb_iteration(const float* M_in, float* M_out, const float* R0, const float* R1, float* flowx, float* flowy,
                    int H, int W, int pitch, const float* wk, int kh, int update_matrices, void* stream);

/* ---------------------------------------------------------------------------------
 * The Liu-Shen optical-flow-equation warp of the pyramid's level transition
 * (updateNextPyramidalLevel with biLinear=False, src/GenericPyramidalOpticalFlow.py:
 * 184-218).  Step 1 (of_warp_liushen_scatter): the integer shift
 * out[y + floor(v + 0.5)][x + floor(u + 0.5)] = I[y][x] with numpy's rules (negative
 * destinations wrap once; when several sources land on one pixel the last in row-major
 * order wins; pixels nobody lands on keep I), and the sub-pixel parts du = u - floor(u +
 * 0.5), dv likewise.  bad[0] / bad[1] (device ints) receive the row-major position of the
 * first source whose destination row / column lies outside [-H, H) / [-W, W), or INT_MAX:
 * the reference raises IndexError there.  Step 2: du, dv are smoothed with the reference's
 * 73-tap gaussian_filter (of_prefilter_f32, prepareGaussianKernel(0.6 * 3, 73)).  Step 3
 * (of_warp_liushen_ofe): out[y][x] = I - ((I[y][x+1] du[y][x+1] - I du) + (I[y+1][x]
 * dv[y+1][x] - I dv)) for y < H-1, x < W-1 (float32, the reference's order); the last row
 * and column are copied.  I is step 1's output.
 * ------------------------------------------------------------------------------- */
size_t of_warp_liushen_workspace_size(int H, int W);
int of_warp_liushen_scatter(const float* I, const float* u, const float* v, float* out, float* du, float* dv, int H,
                            int W, int pitch, int* bad, void* workspace, size_t workspace_bytes, void* stream);
int of_warp_liushen_ofe(const float* I, const float* du, const float* dv, float* out, int H, int W, int pitch,
                        void* stream);

/* ---------------------------------------------------------------------------------
 * Learned warm start for Liu-Shen (no reference counterpart: the reference has no
 * learned component).  An encoder-decoder CNN over bfloat16 NHWC activations
 * ([image][y][x][channel], a tensor may be a channel slice [coff, coff + C) of a wider
 * one with ctot channels per pixel; for bf16 tensors ctot and coff multiples of 8), f32
 * accumulation.
 * `err` is a device word; the conv kernel ORs a nonzero code into it when one of its
 * bounded waits gives up (its output is then incomplete).
 * ------------------------------------------------------------------------------- */
#define OF_CNN_RELU 1 /* apply max(0, .) after the bias */
#define OF_CNN_F32 2  /* store float32 instead of bfloat16 */
/* y = conv3x3(x, w) + bias, zero padding, tensor cores (tcgen05, TMEM accumulator).
 * x: n x H x W x cin slice (cin 16 or a multiple of 32); w: bf16 [9][cout][cin] (tap =
 * 3 * (dy + 1) + (dx + 1)); cout a multiple of 16, <= 512; W a divisor or a multiple of
 * 128, H a multiple of 128 / min(W, 128) or a divisor of it, and then n a multiple of
 * 128 / (W * H).  Channels [0, cout_store) are written. */
int of_cnn_conv3x3(const void* x, int n, int H, int W, int cin, int x_ctot, int x_coff, const void* w, int cout,
                   const float* bias, int flags, void* y, int y_ctot, int y_coff, int cout_store, unsigned* err,
                   void* stream);
/* dw[tap][co][ci] += sum_p dy[p][co] * x[p + tap][ci] on the tensor cores (tcgen05, both
 * operands MN-major from NHWC, f32 accumulate, split over pixel ranges and added with
 * atomics).  W a divisor or a multiple of 64, H likewise for 64 / min(W, 64); cin, cout <= 512. */
int of_cnn_conv3x3_wgrad_tc(const void* x, int x_ctot, int x_coff, const void* dy, int dy_ctot, int dy_coff, int n,
                            int H, int W, int cin, int cout, float* dw, unsigned* err, void* stream);
/* dw[tap][co][ci] += sum_p dy[p][co] * x[p + tap][ci]   (f32, CUDA cores). */
int of_cnn_conv3x3_wgrad(const void* x, int x_ctot, int x_coff, const void* dy, int dy_ctot, int dy_coff, int n,
                         int H, int W, int cin, int cout, float* dw, void* stream);
/* db[c] += sum_p dy[p][c] over P pixels. */
int of_cnn_bias_grad(const void* dy, int dy_ctot, int dy_coff, long long P, int cout, float* db, void* stream);
/* out[y][x] = (I0 / max I0, I1 / max I1, 0 ...) over cpad channels; max2: 2 device words. */
int of_cnn_pack_pair(const float* I0, const float* I1, int H, int W, int pitch, unsigned* max2, void* out, int cpad,
                     void* stream);
int of_cnn_avgpool2(const void* x, int x_ctot, int x_coff, int n, int H, int W, int C, void* y, int y_ctot,
                    int y_coff, void* stream);
int of_cnn_avgpool2_bwd(const void* dy, int dy_ctot, int dy_coff, int n, int H, int W, int C, void* dx, int dx_ctot,
                        int dx_coff, int accumulate, void* stream);
int of_cnn_upsample2(const void* x, int x_ctot, int x_coff, int n, int h, int w, int C, void* y, int y_ctot,
                     int y_coff, void* stream);
int of_cnn_upsample2_bwd(const void* dy, int dy_ctot, int dy_coff, int n, int h, int w, int C, void* dx, int dx_ctot,
                         int dx_coff, void* stream);
/* g *= (y > 0) over P pixels x C channels. */
int of_cnn_relu_bwd(void* g, int g_ctot, int g_coff, const void* y, int y_ctot, int y_coff, long long P, int C,
                    void* stream);
/* loss += sum |pred - label|^2 / (2P) over P two-channel f32 pixels; dpred (bf16, g_ctot
 * channels, padding zeroed; may be NULL) = (pred - label) / P. */
int of_cnn_flow_mse(const float* pred, const float* label, long long P, void* dpred, int g_ctot, double* loss,
                    void* stream);
int of_cnn_adam(float* w, const float* g, float* m, float* v, long long n, float lr, float b1, float b2, float eps,
                int step, void* stream);
/* master w[tap][co][ci] (f32) -> bf16 [9][cout_pad][cin_pad], or with transpose_flip
 * the input-gradient operand [9][cin_pad][cout_pad] with the taps mirrored. */
int of_cnn_pack_weights(const float* w, int cout, int cin, int cout_pad, int cin_pad, int transpose_flip, void* out,
                        void* stream);
/* (h, w, 2) interleaved f32 flow -> U, V planes at (factor h, factor w) (row pitch
 * `pitch`): bilinear, pixel-centre aligned, edges clamped, displacements times `scale`. */
int of_cnn_flow_up(const float* flow, int h, int w, int factor, float* U, float* V, int pitch, float scale,
                   void* stream);
/* (h, w, 2) interleaved f32 flow -> u, v planes (row pitch `pitch`). */
int of_cnn_split_flow(const float* flow, int h, int w, float* u, float* v, int pitch, void* stream);

/* ---------------------------------------------------------------------------------
 * Batches through the whole pyramid — of_batch_run replaces genericPyramidalOpticalFlow
 * (src/GenericPyramidalOpticalFlow.py:237-415) called once per pair with the HS, LK or
 * Farneback adapter (+ the optional Liu-Shen refine), bilinear warp and kLevels = 1; the
 * same kernels run with the same arguments as the Python drop-in, so results are equal.
 * Host constants the reference computes in Python come with the descriptor: the prefilter
 * taps (prepareGaussianKernel, src/gaussian_filter.py:47-52) and the Farneback kernels and
 * polynomial constants (src/Farneback_PyCL.py:123-208).  Pairs run in stream order on
 * `stream`; single-level Horn-Schunck pairs are gathered into one persistent launch
 * (of_hs_batch, with tuning->tile_shape).  status (DEVICE int[n], optional): the OF_ST_*
 * words of each pair (cleared by the call).
 * ------------------------------------------------------------------------------- */
#define OF_METHOD_HS 0
#define OF_METHOD_LK 1
#define OF_METHOD_FB 2
#define OF_FB_MAX_LEVELS 8

/* Farneback_PyCL(windowSize, Niters, polyN, polySigma, useGaussian, pyrScale, pyramidalLevels) */
typedef struct OfFbParams {
  int window_size, niters, use_gaussian, levels;
  double pyr_scale;
  of_fb_poly_consts poly;
  const float* window_taps; /* half kernel (centre first) of getGaussianKernelBitExact(windowSize, windowSize/2*0.3) */
  int window_kh;
  const float* level_taps[OF_FB_MAX_LEVELS]; /* per internal level k (0 = full size): the frame blur's half kernel */
  int level_kh[OF_FB_MAX_LEVELS];
} OfFbParams;

typedef struct OfPairDesc {
  int method;                  /* OF_METHOD_* */
  int frame_u8;                /* 1: I0, I1 are uint8 planes, 0: float32 */
  const void* I0;              /* DEVICE frames H x W, row pitch in_pitch elements */
  const void* I1;
  int in_pitch;
  float* U;                    /* DEVICE result (float32 H x W, row pitch out_pitch) */
  float* V;
  int out_pitch;
  int H, W;
  float filter;                /* FILTER; > 1e-3 prefilters with filter_taps (3 taps, HOST) */
  const float* filter_taps;
  int levels;                  /* pyramidalLevels */
  int refine_ls;               /* the Liu-Shen refine (optionalOFlowAlgoAdapter) */
  float filter_opt;            /* FILTER_OPT; > 1e-3 prefilters the refine's frames (5 taps, HOST) */
  const float* filter_opt_taps;
  float ls_h;                  /* LiuShenOpticalFlowAlgoAdapter(alpha) */
  int ls_arithmetic;           /* OF_LS_EXACT or OF_LS_FAST */
  int warping, intermediate_scaling, scaling;  /* -1: the main adapter's pyramid defaults */
  float hs_alphas[8];          /* HSOpticalFlowAlgoAdapter(alphas, Niter): popped from the end */
  int hs_nalphas, hs_niter;
  int lk_half_win, lk_niter;   /* denseLucasKanade_PyCl(Niter, halfWindow) */
  const OfFbParams* fb;        /* HOST, for OF_METHOD_FB */
} OfPairDesc;

size_t of_batch_workspace_size(const OfPairDesc* descs, int n, const OfTuning* tuning);
int of_batch_run(const OfPairDesc* descs, int n, const OfTuning* tuning, int* status, void* workspace,
                 size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* OFB200_H */
