// Horn-Schunck for one or many frame pairs in ONE persistent launch over a device work
// queue (src/HornSchunck.py:51-126, bit-exact like hs.cu).
//
// Work items are (pass, pair, tile), handed out in that order by an atomic ticket
// counter to CTAs that stay resident for the whole launch.  Pass 0 of a pair computes its
// derivative planes (computeDerivatives, :106-126) and copies the initial U, V for a tile;
// pass p >= 1 runs up to HQ_T Jacobi sweeps (HS_helper, :61-70) on the tile with a halo of
// HQ_T cells staged in shared memory (temporal blocking), reading
// the previous pass's fields and writing the next buffer of a ping-pong pair.  An item of
// pass p waits only for its own tile and its (up to) 8 neighbouring tiles to have finished
// pass p - 1 (a counter of finished passes per tile): the halo of T cells lies inside those
// tiles, and since the neighbourhood is symmetric the same wait also guarantees that no
// neighbour still reads (at pass p - 1) the buffer this item overwrites.  Passes therefore
// overlap as a wavefront instead of meeting at a per-pass barrier.  The ticket order makes
// this free of deadlock: an item only waits for items with smaller tickets, which were
// handed out earlier to CTAs that are running and never wait for later ones.  The wait is
// bounded: after `wait_limit` polls the item gives up, sets OF_ST_WAIT_TIMEOUT in its pair's
// status word and the launch's error flag, and every later item of that pair is skipped
// (still counted, so nothing waits on it).
// Cross-CTA data goes through L2 only (ld.global.cg / st.global.cg), published by
// __syncthreads + __threadfence + atomicAdd and consumed after the counter is observed.
#include <cooperative_groups.h>

#include "common.cuh"
#include "hsweep.cuh"

namespace ofb {

struct HsqPair {
  const float* I0;   // frame at t0
  const float* I1;   // frame at t1
  float* U;          // initial flow in, result out
  float* V;
  float* fx;         // workspace planes (pitch `pitch`)
  float* fy;
  float* ft;
  float* U0;         // the initial flow (kept for the reference's error)
  float* V0;
  float* Ub;         // ping-pong partner of U / V
  float* Vb;
  int H, W, pitch;
  float a2;          // alpha^2
  int niter;
  int passes;        // 1 + ceil(niter / T): the derivative pass and the sweep passes
  int tx, tiles;     // tiles per row, tiles per pass
  unsigned int tile0;  // sum of tiles of the earlier pairs
};

__device__ __forceinline__ double hq_acc(double a, float v, double w) { return __fma_rn((double)v, w, a); }

// Derivatives of one pixel (hs_deriv_kernel's arithmetic).  Returns false when a frame
// sample of the pixel is not finite.
__device__ __forceinline__ bool hq_deriv(const HsqPair& P, int y, int x, float& fx, float& fy, float& ft) {
  const int H = P.H, W = P.W, pitch = P.pitch;
  int y1 = mirror1(y + 1, H), x1 = mirror1(x + 1, W);
  size_t i00 = (size_t)y * pitch + x, i01 = (size_t)y * pitch + x1, i10 = (size_t)y1 * pitch + x,
         i11 = (size_t)y1 * pitch + x1;
  const float* f1 = P.I1;
  const float* f0 = P.I0;
  float a00 = f1[i00], a01 = f1[i01], a10 = f1[i10], a11 = f1[i11];
  float b00 = f0[i00], b01 = f0[i01], b10 = f0[i10], b11 = f0[i11];
  double t;
  t = hq_acc(hq_acc(hq_acc(hq_acc(0.0, a00, 0.25), a01, -0.25), a10, 0.25), a11, -0.25);
  float gx1 = (float)t;
  t = hq_acc(hq_acc(hq_acc(hq_acc(0.0, b00, 0.25), b01, -0.25), b10, 0.25), b11, -0.25);
  float gx0 = (float)t;
  t = hq_acc(hq_acc(hq_acc(hq_acc(0.0, a00, 0.25), a01, 0.25), a10, -0.25), a11, -0.25);
  float gy1 = (float)t;
  t = hq_acc(hq_acc(hq_acc(hq_acc(0.0, b00, 0.25), b01, 0.25), b10, -0.25), b11, -0.25);
  float gy0 = (float)t;
  t = hq_acc(hq_acc(hq_acc(hq_acc(0.0, b00, 0.25), b01, 0.25), b10, 0.25), b11, 0.25);
  float gt0 = (float)t;
  t = hq_acc(hq_acc(hq_acc(hq_acc(0.0, a00, -0.25), a01, -0.25), a10, -0.25), a11, -0.25);
  float gt1 = (float)t;
  fx = __fadd_rn(gx1, gx0);
  fy = __fadd_rn(gy1, gy0);
  ft = __fadd_rn(gt0, gt1);
  return isfinite(a00) && isfinite(b00);
}

// The derivative planes of one pixel into the workspace, and the copy of its initial flow.
__device__ __forceinline__ bool hq_deriv_px(const HsqPair& P, int y, int x) {
  float fx, fy, ft;
  const bool ok = hq_deriv(P, y, x, fx, fy, ft);
  const size_t i00 = (size_t)y * P.pitch + x;
  __stcg(P.fx + i00, fx);
  __stcg(P.fy + i00, fy);
  __stcg(P.ft + i00, ft);
  __stcg(P.U0 + i00, __ldcg(P.U + i00));
  __stcg(P.V0 + i00, __ldcg(P.V + i00));
  return ok;
}

// Called by all of warp 0: lanes 0-8 poll, in parallel, the finished-stage counters of the
// tile and its (up to) 8 neighbours until each reaches `need`; lane 9 reads the pair's status
// word.  Every poll gives up after `wait_limit` rounds, which marks the pair
// (OF_ST_WAIT_TIMEOUT) and the launch's error flag.  Returns 1 when the item may run: no
// wait gave up and the pair had not failed before.  Lane 0 issues the acquire fence.
__device__ __forceinline__ unsigned int hq_ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int hq_wait(const unsigned int* done, unsigned int tile0, int tile, int ntx, int nty,
                                       unsigned int need, long long wait_limit, int* status_i, int* err_flag) {
  const int lane = threadIdx.x & 31;
  bool gave_up = false, failed_before = false;
  if (lane < 9) {
    const int ty = tile / ntx, tx = tile - ty * ntx;
    const int yy = ty + lane / 3 - 1, xx = tx + lane % 3 - 1;
    if (need > 0 && yy >= 0 && yy < nty && xx >= 0 && xx < ntx) {
      const unsigned int* c = done + tile0 + yy * ntx + xx;
      long long k = 0;
      while (hq_ld_acquire(c) < need) {
        if (++k > wait_limit) {
          gave_up = true;
          break;
        }
        __nanosleep(32);
      }
    }
  } else if (lane == 9) {
    failed_before = (*(volatile int*)status_i & OF_ST_WAIT_TIMEOUT) != 0;
  }
  const bool timeout = __any_sync(0xffffffffu, gave_up);
  const bool before = __any_sync(0xffffffffu, failed_before);
  if (lane == 0 && timeout && !before) {
    atomicOr(status_i, OF_ST_WAIT_TIMEOUT);
    atomicExch(err_flag, 1);
  }
  // the polls are acquire loads: the neighbours' stores released before their counters are
  // visible to this CTA after the barrier that follows
  return !(timeout || before);
}

// Up to T sweeps on one tile: region RW x RH = (TW + 2T) x (TH + 2T) in shared memory.
// Sweep s computes the cells at least s + 1 from the region's edge, which after T sweeps
// leaves exactly the owned cells exact.  On image borders every neighbour index goes
// through hs_sweep_kernel's 'mirror' map (mapped neighbours stay within one row / column of
// their cell, so inside the region), and out-of-image cells are neither computed nor read.
// Each cell's arithmetic is hs_sweep_kernel's: the averaging weights are float32 values
// (24-bit mantissas), so every product with a float32 sample is exact in double and
// fma(v, w, acc) rounds exactly as the separate multiply and add.
// Shared memory: the derivative planes as float32 and two (u, v) buffers, float64 for the
// bit-exact arithmetic (the values are float32 results, held exactly, so the reference's
// float64 stencil sums need no conversion per neighbour) and float32 for OF_HS_FAST.
// RD: after the (u, v) buffers, each cell's float64 reciprocal of its denominator (hq_div,
// the branch-free quotient); left out of the largest region, whose two CTAs per SM it
// would not leave room for (that shape divides with __fdiv_rn).
template <int RW, int RH, int T>
struct HqTile {
  static constexpr int TW = RW - 2 * T, TH = RH - 2 * T, PL = RW * RH;
  static constexpr bool RD = PL <= 2048;
  static_assert(PL % 2 == 0, "the float64 planes stay 8-byte aligned");
  static constexpr size_t smem(bool fast) {
    return 3 * (size_t)PL * 4 + 4 * (size_t)PL * (fast ? 4 : 8) + (RD ? (size_t)PL * 8 : 0);
  }
};

// The sweeps of one pass on the region (nsw <= T of them), ping-pong from buffer 0, so an
// even count leaves the result in buffer 0.
template <int RW, int RH, int T, bool FAST, int NT>
__device__ __forceinline__ void hq_sweeps(const float* sfx, const float* sfy, const float* sft, const double* srd,
                                          HqVal<FAST>* bu0, HqVal<FAST>* bv0, HqVal<FAST>* bu1, HqVal<FAST>* bv1,
                                          int nsw, bool edge, int x0, int y0, int H, int W, float a2) {
#pragma unroll 1
  for (int s = 0; s < nsw; s++) {
    const bool q = s & 1;
    HqVal<FAST>* iu = q ? bu1 : bu0;
    HqVal<FAST>* iv = q ? bv1 : bv0;
    HqVal<FAST>* ou = q ? bu0 : bu1;
    HqVal<FAST>* ov = q ? bv0 : bv1;
    constexpr bool RD = HqTile<RW, RH, T>::RD;
    if (edge)
      hq_sweep2<RW, RH, T, true, FAST, NT, RD>(sfx, sfy, sft, srd, iu, iv, ou, ov, s, x0, y0, H, W, a2);
    else
      hq_sweep2<RW, RH, T, false, FAST, NT, RD>(sfx, sfy, sft, srd, iu, iv, ou, ov, s, x0, y0, H, W, a2);
    __syncthreads();
  }
}

// Returns false when a result of the last pass is not finite.
template <int RW, int RH, int T, bool FAST, int NT>
__device__ bool hq_sweep_item(const HsqPair& P, int pass, int tile, float* sm) {
  using G = HqTile<RW, RH, T>;
  const int ty = tile / P.tx, tx = tile - ty * P.tx;
  const int x0 = tx * G::TW, y0 = ty * G::TH;
  const int H = P.H, W = P.W, pitch = P.pitch;
  const int np = P.passes - 1;   // sweep passes
  const int p = pass - 1;        // this sweep pass
  // pass p reads the initial flow (p == 0) or the previous pass's buffer and writes U, V when
  // an even number of passes remain after it (so the last pass writes U, V)
  const bool to_uv = ((np - 1 - p) & 1) == 0;
  const float* srcu = p == 0 ? P.U0 : (to_uv ? P.Ub : P.U);
  const float* srcv = p == 0 ? P.V0 : (to_uv ? P.Vb : P.V);
  float* dstu = to_uv ? P.U : P.Ub;
  float* dstv = to_uv ? P.V : P.Vb;
  const int nsw = min(T, P.niter - p * T);
  float* sfx = sm;
  float* sfy = sfx + G::PL;
  float* sft = sfy + G::PL;
  using V = HqVal<FAST>;
  V* const bu0 = reinterpret_cast<V*>(sft + G::PL);  // 3 PL floats: 8-byte aligned for even PL
  V* const bv0 = bu0 + G::PL;
  V* const bu1 = bu0 + 2 * G::PL;
  V* const bv1 = bu0 + 3 * G::PL;
  double* const srd = reinterpret_cast<double*>(bu0 + 4 * G::PL);
  for (int k = threadIdx.x; k < G::PL; k += NT) {
    const int r = k / RW, c = k - r * RW;
    const int gy = y0 - T + r, gx = x0 - T + c;
    if (gy < 0 || gy >= H || gx < 0 || gx >= W) continue;  // never read
    const size_t i = (size_t)gy * pitch + gx;
    const float gxv = __ldcg(P.fx + i), gyv = __ldcg(P.fy + i);
    sfx[k] = gxv;
    sfy[k] = gyv;
    sft[k] = __ldcg(P.ft + i);
    if (G::RD) srd[k] = hq_recip_den(gxv, gyv, P.a2);
    bu0[k] = __ldcg(srcu + i);
    bv0[k] = __ldcg(srcv + i);
  }
  __syncthreads();
  const bool edge = x0 < T || y0 < T || x0 + G::TW + T > W || y0 + G::TH + T > H;
  hq_sweeps<RW, RH, T, FAST, NT>(sfx, sfy, sft, srd, bu0, bv0, bu1, bv1, nsw, edge, x0, y0, H, W, P.a2);
  const V* fu = (nsw & 1) ? bu1 : bu0;
  const V* fv = (nsw & 1) ? bv1 : bv0;
  bool finite = true;
  for (int k = threadIdx.x; k < G::TW * G::TH; k += NT) {
    const int r = k / G::TW, c = k - r * G::TW;
    const int y = y0 + r, x = x0 + c;
    if (y >= H || x >= W) continue;
    const int o = (r + T) * RW + c + T;
    __stcg(dstu + (size_t)y * pitch + x, (float)fu[o]);
    __stcg(dstv + (size_t)y * pitch + x, (float)fv[o]);
    finite = finite && isfinite(fu[o]) && isfinite(fv[o]);
  }
  return finite || p != np - 1;
}

// The pair whose tiles hold global tile index r (tile0 ascending).
__device__ __forceinline__ int hq_pair_of(const HsqPair* __restrict__ pairs, int npairs, unsigned int r) {
  int lo = 0, hi = npairs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (pairs[mid].tile0 <= r) lo = mid; else hi = mid - 1;
  }
  return lo;
}

template <int RW, int RH, int T, bool FAST, int NT>
__device__ __forceinline__ void hsq_body(const HsqPair* __restrict__ pairs, int npairs, unsigned int tiles_total,
                                         int max_passes, unsigned long long* ticket, unsigned int* done, int* status,
                                         long long wait_limit, int* err_flag) {
  extern __shared__ float hq_sm[];
  __shared__ unsigned long long s_item;
  __shared__ int s_run, s_pair;
  const unsigned long long nitems = (unsigned long long)tiles_total * (unsigned long long)max_passes;
  using G = HqTile<RW, RH, T>;
  // thread 0 holds the next ticket while the current item runs (its atomic's latency is
  // hidden); an item still only waits for items with smaller tickets
  unsigned long long next = 0;
  if (threadIdx.x == 0) next = atomicAdd(ticket, 1ull);
  for (;;) {
    if (threadIdx.x == 0) {
      s_item = next;
      if (next < nitems) next = atomicAdd(ticket, 1ull);
    }
    __syncthreads();
    const unsigned long long n = s_item;
    if (n >= nitems) break;
    const int pass = (int)(n / tiles_total);
    const unsigned int r = (unsigned int)(n - (unsigned long long)pass * tiles_total);
    if (threadIdx.x == 0) s_pair = hq_pair_of(pairs, npairs, r);
    __syncthreads();
    const int i = s_pair;
    const HsqPair& P = pairs[i];
    const int tile = (int)(r - P.tile0);
    if (threadIdx.x < 32) {
      // this tile and its neighbours must have finished pass - 1 (counters of passes done)
      int run = pass < P.passes;
      if (run) run = hq_wait(done, P.tile0, tile, P.tx, P.tiles / P.tx, (unsigned int)pass, wait_limit, status + i,
                             err_flag);
      if (threadIdx.x == 0) s_run = run;
    }
    __syncthreads();
    bool ok = true;
    if (s_run) {
      if (pass == 0) {
        const int ty = tile / P.tx, tx = tile - ty * P.tx;
        for (int k = threadIdx.x; k < G::TW * G::TH; k += NT) {
          const int rr = k / G::TW, cc = k - rr * G::TW;
          const int y = ty * G::TH + rr, x = tx * G::TW + cc;
          if (y < P.H && x < P.W) ok = hq_deriv_px(P, y, x) && ok;
        }
      } else {
        ok = hq_sweep_item<RW, RH, T, FAST, NT>(P, pass, tile, hq_sm);
      }
    }
    const int bad = __syncthreads_or(!ok);  // also: every store of the item is issued
    if (threadIdx.x == 0 && bad) atomicOr(status + i, pass == 0 ? OF_ST_NONFINITE_INPUT : OF_ST_NONFINITE_OUTPUT);
    if (threadIdx.x == 0 && pass < P.passes) {
      __threadfence();  // release
      atomicAdd(done + P.tile0 + tile, 1u);
    }
  }
}

// Cell k of a region's halo ring (the region minus its owned tile): the top T rows, the
// bottom T rows, then the T columns left and right of the tile in each tile row.
template <int RW, int RH, int T>
__device__ __forceinline__ void hq_ring_cell(int k, int& r, int& c) {
  constexpr int TW = RW - 2 * T, BAND = T * RW;
  if (k < BAND) {
    r = k / RW;
    c = k - r * RW;
  } else if (k < 2 * BAND) {
    const int q = k - BAND;
    r = RH - T + q / RW;
    c = q - (q / RW) * RW;
  } else {
    const int m = k - 2 * BAND, cc = m % (2 * T);
    r = T + m / (2 * T);
    c = cc < T ? cc : cc + TW;
  }
}

// Each warp publishes its own part of a stage: its stores (or reads) are ordered before its
// increment of the tile's counter, so a stage of a tile is complete when the counter has
// grown by the CTA's warp count; no CTA barrier sits between the last store and the release.
__device__ __forceinline__ void hq_release_warp(unsigned int* counter) {
  __syncwarp();
  __threadfence();
  if ((threadIdx.x & 31) == 0) atomicAdd(counter, 1u);
}

// The resident schedule, for launches where every tile gets a CTA of its own (all CTAs
// resident): CTA b owns global tile b for the whole solve and keeps its region on chip.
// Stage 0 computes the derivative planes of the WHOLE region (owned tile and halo: they
// depend on the frames only) and loads the region's initial flow; both stay in shared
// memory.  Stage s >= 1 runs up to T sweeps as a queue item of pass s does, but only the
// halo ring comes from global memory (the neighbours' results of stage s - 1); the owned
// part is already in shared memory, where the previous stage's T (even) sweeps left it.
// The owned tile is published every stage.  Waits are the queue kernel's, the counters
// count warps: a stage waits for its own and its neighbours' counters to reach s x (NT /
// 32), which also orders every overwrite of a ping-pong buffer (or of the initial U, V at
// stage 1) after the neighbours' reads of it.  The halo ring of a stage is gathered with
// every thread's loads in flight at once (one L2 round trip), then written to shared memory.
template <int RW, int RH, int T, bool FAST, int NT>
__device__ __forceinline__ void hsr_body(const HsqPair* __restrict__ pairs, int npairs, unsigned int* done,
                                         int* status, long long wait_limit, int* err_flag) {
  static_assert(T % 2 == 0, "a full stage must leave its result in the first buffer");
  extern __shared__ float hq_sm[];
  __shared__ int s_pair, s_run;
  using G = HqTile<RW, RH, T>;
  const unsigned int gtile = blockIdx.x;
  if (threadIdx.x == 0) s_pair = hq_pair_of(pairs, npairs, gtile);
  __syncthreads();
  const int i = s_pair;
  const HsqPair& P = pairs[i];
  const int tile = (int)(gtile - P.tile0);
  const int ty = tile / P.tx, tx = tile - ty * P.tx;
  const int x0 = tx * G::TW, y0 = ty * G::TH;
  const int H = P.H, W = P.W, pitch = P.pitch, np = P.passes - 1, nty = P.tiles / P.tx;
  float* sfx = hq_sm;
  float* sfy = sfx + G::PL;
  float* sft = sfy + G::PL;
  using V = HqVal<FAST>;
  V* const bu0 = reinterpret_cast<V*>(sft + G::PL);  // 3 PL floats: 8-byte aligned for even PL
  V* const bv0 = bu0 + G::PL;
  V* const bu1 = bu0 + 2 * G::PL;
  V* const bv1 = bu0 + 3 * G::PL;
  double* const srd = reinterpret_cast<double*>(bu0 + 4 * G::PL);
  const bool edge = x0 < T || y0 < T || x0 + G::TW + T > W || y0 + G::TH + T > H;
  // stage 0
  bool ok = true;
  for (int k = threadIdx.x; k < G::PL; k += NT) {
    const int r = k / RW, c = k - r * RW;
    const int gy = y0 - T + r, gx = x0 - T + c;
    if (gy < 0 || gy >= H || gx < 0 || gx >= W) continue;  // never read
    float fx, fy, ft;
    const bool f = hq_deriv(P, gy, gx, fx, fy, ft);
    sfx[k] = fx;
    sfy[k] = fy;
    sft[k] = ft;
    if (G::RD) srd[k] = hq_recip_den(fx, fy, P.a2);
    const size_t gi = (size_t)gy * pitch + gx;
    bu0[k] = __ldcg(P.U + gi);
    bv0[k] = __ldcg(P.V + gi);
    if (r >= T && r < T + G::TH && c >= T && c < T + G::TW) ok = ok && f;  // each pixel checked once
  }
  const int bad0 = __syncthreads_or(!ok);
  if (threadIdx.x == 0 && bad0) atomicOr(status + i, OF_ST_NONFINITE_INPUT);
  hq_release_warp(done + gtile);  // this warp's reads of the initial U, V are done
  for (int p = 0; p < np; p++) {
    const int stage = p + 1;
    if (threadIdx.x < 32) {
      const int run = hq_wait(done, P.tile0, tile, P.tx, nty, (unsigned int)(stage * (NT / 32)), wait_limit,
                              status + i, err_flag);
      if (threadIdx.x == 0) s_run = run;
    }
    __syncthreads();
    ok = true;
    if (s_run) {
      const bool to_uv = ((np - 1 - p) & 1) == 0;  // the last stage writes U, V
      float* dstu = to_uv ? P.U : P.Ub;
      float* dstv = to_uv ? P.V : P.Vb;
      if (p > 0) {  // halo ring: the neighbours' results of the previous stage
        const float* srcu = to_uv ? P.Ub : P.U;
        const float* srcv = to_uv ? P.Vb : P.V;
        constexpr int RING = G::PL - G::TW * G::TH, NK = (RING + NT - 1) / NT;
        float hu[NK], hv[NK];
        int ho[NK];
#pragma unroll
        for (int j = 0; j < NK; j++) {
          int r, c;
          hq_ring_cell<RW, RH, T>((int)threadIdx.x + j * NT, r, c);
          const int gy = y0 - T + r, gx = x0 - T + c;
          ho[j] = -1;
          if ((int)threadIdx.x + j * NT < RING && gy >= 0 && gy < H && gx >= 0 && gx < W) {
            const size_t gi = (size_t)gy * pitch + gx;
            hu[j] = __ldcg(srcu + gi);
            hv[j] = __ldcg(srcv + gi);
            ho[j] = r * RW + c;
          }
        }
#pragma unroll
        for (int j = 0; j < NK; j++) {
          if (ho[j] >= 0) {
            bu0[ho[j]] = hu[j];
            bv0[ho[j]] = hv[j];
          }
        }
        __syncthreads();
      }
      const int nsw = min(T, P.niter - p * T);
      hq_sweeps<RW, RH, T, FAST, NT>(sfx, sfy, sft, srd, bu0, bv0, bu1, bv1, nsw, edge, x0, y0, H, W, P.a2);
      const V* fu = (nsw & 1) ? bu1 : bu0;
      const V* fv = (nsw & 1) ? bv1 : bv0;
      for (int k = threadIdx.x; k < G::TW * G::TH; k += NT) {
        const int r = k / G::TW, c = k - r * G::TW;
        const int y = y0 + r, x = x0 + c;
        if (y >= H || x >= W) continue;
        const int o = (r + T) * RW + c + T;
        __stcg(dstu + (size_t)y * pitch + x, (float)fu[o]);
        __stcg(dstv + (size_t)y * pitch + x, (float)fv[o]);
        if (p == np - 1) ok = ok && isfinite(fu[o]) && isfinite(fv[o]);
      }
    }
    if (p == np - 1) {
      const int bad = __syncthreads_or(!ok);
      if (threadIdx.x == 0 && bad) atomicOr(status + i, OF_ST_NONFINITE_OUTPUT);
    }
    hq_release_warp(done + gtile);  // this warp's stores of the stage
  }
}

template <int RW, int RH, int T, bool FAST, int NT>
__global__ void __launch_bounds__(NT, NT >= 512 ? 1 : 2)
    hsq_kernel(const HsqPair* __restrict__ pairs, int npairs, unsigned int tiles_total, int max_passes,
               unsigned long long* ticket, unsigned int* done, int* status, long long wait_limit, int* err_flag) {
  hsq_body<RW, RH, T, FAST, NT>(pairs, npairs, tiles_total, max_passes, ticket, done, status, wait_limit, err_flag);
}

template <int RW, int RH, int T, bool FAST, int NT>
__global__ void __launch_bounds__(NT, NT >= 512 ? 1 : 2)
    hsr_kernel(const HsqPair* __restrict__ pairs, int npairs, unsigned int* done, int* status, long long wait_limit,
               int* err_flag) {
  hsr_body<RW, RH, T, FAST, NT>(pairs, npairs, done, status, wait_limit, err_flag);
}

// The adaptive schedule (one CTA per tile launched): the resident schedule when every CTA of
// the launch runs at once, the queue otherwise, decided by the CTAs themselves at the start.
// Each CTA counts itself into `arrived` and polls; the first to see all gridDim.x CTAs
// arrived (all are running, and a running CTA runs to its end) sets the mode word to
// RESIDENT, the first to give up after HQ_ARRIVE_POLLS polls (CTAs still waiting for an SM
// that other work holds) sets it to QUEUE; the word is set once (compare-and-swap) and every
// CTA follows it.  The queue is correct with any number of CTAs running, so neither outcome
// waits on a CTA that may never start.
constexpr int HQ_MODE_UNDECIDED = OF_HS_SCHED_AUTO, HQ_MODE_RESIDENT = OF_HS_SCHED_RESIDENT,
              HQ_MODE_QUEUE = OF_HS_SCHED_QUEUE;
constexpr int HQ_ARRIVE_POLLS = 256;

__device__ __forceinline__ int hq_ld_acquire_i(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int hq_decide_mode(unsigned int* arrived, int* mode) {
  __shared__ int s_mode;
  if (threadIdx.x == 0) {
    atomicAdd(arrived, 1u);
    int m;
    for (int k = 0;; k++) {  // at most HQ_ARRIVE_POLLS + 2 rounds: a give-up sets the word
      m = hq_ld_acquire_i(mode);
      if (m != HQ_MODE_UNDECIDED) break;
      if (hq_ld_acquire(arrived) >= gridDim.x)
        atomicCAS(mode, HQ_MODE_UNDECIDED, HQ_MODE_RESIDENT);
      else if (k >= HQ_ARRIVE_POLLS)
        atomicCAS(mode, HQ_MODE_UNDECIDED, HQ_MODE_QUEUE);
      else
        __nanosleep(128);
    }
    s_mode = m;
  }
  __syncthreads();
  return s_mode;
}

template <int RW, int RH, int T, bool FAST, int NT>
__global__ void __launch_bounds__(NT, NT >= 512 ? 1 : 2)
    hsa_kernel(const HsqPair* __restrict__ pairs, int npairs, unsigned int tiles_total, int max_passes,
               unsigned long long* ticket, unsigned int* done, int* status, long long wait_limit, int* err_flag,
               unsigned int* arrived, int* mode) {
  if (hq_decide_mode(arrived, mode) == HQ_MODE_RESIDENT)
    hsr_body<RW, RH, T, FAST, NT>(pairs, npairs, done, status, wait_limit, err_flag);
  else
    hsq_body<RW, RH, T, FAST, NT>(pairs, npairs, tiles_total, max_passes, ticket, done, status, wait_limit,
                                  err_flag);
}

// ---- One pair on one thread-block cluster ------------------------------------------------
// For images that one cluster of at most 16 CTAs covers with tiles of at most HC_T x HC_T
// cells (256 x 256 and smaller).  CTA (cx, cy) owns a tile and holds the tile plus a
// one-cell halo ring of (u, v) in shared memory, in two buffers, with the tile's derivative
// planes.  A sweep reads its input buffer (all local), writes the owned cells of the output
// buffer, and every cell that a halo ring shows (a neighbouring tile's ring, or a mirrored
// position on the image border) is also stored there, in that CTA's shared memory
// (distributed shared memory).  One cluster barrier per sweep publishes the sweep: no
// global memory and no polling between sweeps.  Each halo position has exactly one source
// cell, so no position is written twice; a CTA only reads its input buffer while its
// neighbours write its output buffer.  Cell arithmetic: hq_update, bit for bit.
constexpr int HC_T = 64;              // largest tile edge
constexpr int HC_RS = HC_T + 2;       // region row stride: tile + halo ring
constexpr int HC_PL = HC_RS * HC_RS;  // cells per region plane
constexpr int HC_THREADS = 512;
constexpr int HC_MAX_CTAS = 16;
static_assert((3 * HC_PL * 4) % 8 == 0, "the float64 planes after the float planes stay 8-byte aligned");

template <bool FAST>
constexpr size_t hc_smem() {
  return 3 * (size_t)HC_PL * sizeof(float) + 4 * (size_t)HC_PL * sizeof(HqVal<FAST>);
}

struct HcGeom {
  int CX, CY;  // tiles per row / column (the cluster's shape)
  int TW, TH;  // tile size (the last column / row of tiles may be smaller)
};

// Tiles of one axis whose region (tile plus the halo ring) contains position p (-1 .. n):
// the tile p lies in (or the nearest one, for -1 and n) and, on a tile edge, its neighbour.
__device__ __forceinline__ int hc_tiles_of(int p, int n, int T, int ntiles, int t[3]) {
  const int own = clampi(p < 0 ? 0 : p / T, 0, ntiles - 1);
  const int lo = own * T, hi = min(lo + T, n) - 1;  // the tile's cells
  int k = 0;
  t[k++] = own;
  if (p == lo && own > 0) t[k++] = own - 1;          // the previous tile's last halo row
  if (p == hi && own < ntiles - 1) t[k++] = own + 1;  // the next tile's first halo row
  return k;
}

// The other positions a halo ring shows cell (gy, gx) at, as (CTA rank << 16 | region
// offset) entries: mirror images on the image border (index -1 shows 1, H shows H - 2) and
// the neighbouring tiles' rings.  Returns the count (at most HC_MAX_TARGETS).
constexpr int HC_MAX_TARGETS = 8;
__device__ __forceinline__ int hc_targets(int gy, int gx, int H, int W, const HcGeom& g, int cx, int cy,
                                          int* tgt) {
  int ys[2], xs[2], ny = 1, nx = 1, n = 0;
  ys[0] = gy;
  xs[0] = gx;
  if (gy == 1) ys[ny++] = -1;
  else if (gy == H - 2) ys[ny++] = H;
  if (gx == 1) xs[nx++] = -1;
  else if (gx == W - 2) xs[nx++] = W;
  for (int a = 0; a < ny; a++) {
    int ty[3];
    const int nty = hc_tiles_of(ys[a], H, g.TH, g.CY, ty);
    for (int b = 0; b < nx; b++) {
      int tx[3];
      const int ntx = hc_tiles_of(xs[b], W, g.TW, g.CX, tx);
      for (int i = 0; i < nty; i++)
        for (int j = 0; j < ntx; j++) {
          if (a == 0 && b == 0 && ty[i] == cy && tx[j] == cx) continue;  // the cell itself
          if (n == HC_MAX_TARGETS) return n;
          const int o = (ys[a] - ty[i] * g.TH + 1) * HC_RS + (xs[b] - tx[j] * g.TW + 1);
          tgt[n++] = ((tx[j] + ty[i] * g.CX) << 16) | o;  // rank, region offset (< 2^16)
        }
    }
  }
  return n;
}

template <bool FAST>
__global__ void __launch_bounds__(HC_THREADS, 1) hsc_kernel(const HsqPair P, const HcGeom g, int* status) {
  namespace cg = cooperative_groups;
  cg::cluster_group cl = cg::this_cluster();
  extern __shared__ __align__(16) float hc_sm[];
  using V = HqVal<FAST>;
  float* const sfx = hc_sm;
  float* const sfy = sfx + HC_PL;
  float* const sft = sfy + HC_PL;
  V* const bu0 = reinterpret_cast<V*>(sft + HC_PL);
  V* const bv0 = bu0 + HC_PL;
  V* const bu1 = bu0 + 2 * HC_PL;
  V* const bv1 = bu0 + 3 * HC_PL;
  const int cx = blockIdx.x, cy = blockIdx.y;
  const int H = P.H, W = P.W, pitch = P.pitch;
  const int x0 = cx * g.TW, y0 = cy * g.TH;
  const int tw = min(g.TW, W - x0), th = min(g.TH, H - y0);
  // region cell (ry, rx) <-> image cell (y0 - 1 + ry, x0 - 1 + rx); the ring mirrors the
  // image border like the stencil's neighbour map
  bool ok = true;
  for (int k = threadIdx.x; k < (th + 2) * (tw + 2); k += HC_THREADS) {
    const int ry = k / (tw + 2), rx = k - ry * (tw + 2);
    const int o = ry * HC_RS + rx;
    const size_t gi = (size_t)mirror1(y0 - 1 + ry, H) * pitch + mirror1(x0 - 1 + rx, W);
    bu0[o] = (V)P.U[gi];
    bv0[o] = (V)P.V[gi];
    if (ry >= 1 && ry <= th && rx >= 1 && rx <= tw) {
      float fx, fy, ft;
      ok = hq_deriv(P, y0 - 1 + ry, x0 - 1 + rx, fx, fy, ft) && ok;
      sfx[o] = fx;
      sfy[o] = fy;
      sft[o] = ft;
    }
  }
  if (__syncthreads_or(!ok) && threadIdx.x == 0) atomicOr(status, OF_ST_NONFINITE_INPUT);
  cl.sync();  // every CTA of the cluster runs and holds its initial region
  // the thread's halo source: candidate t among the tile's edge rows and columns and the
  // rows / columns the image border mirrors (4 rows x tw + 4 columns x th <= HC_THREADS),
  // with the positions it is copied to after each sweep
  int hsrc = -1, ntg = 0, tgt[HC_MAX_TARGETS];
  {
    const int t = threadIdx.x;
    const int rset[4] = {1, th, 2 - y0, H - 1 - y0};  // region rows of gy = y0, y0 + th - 1, 1, H - 2
    const int cset[4] = {1, tw, 2 - x0, W - 1 - x0};
    auto in_rset = [&](int r, int upto) {
      for (int j = 0; j < upto; j++)
        if (rset[j] == r) return true;
      return false;
    };
    int r = -1, cc = -1;
    bool valid = false;
    if (t < 4 * tw) {
      const int k = t / tw;
      r = rset[k];
      cc = t - k * tw + 1;
      valid = r >= 1 && r <= th && !in_rset(r, k);
    } else if (t < 4 * tw + 4 * th) {
      const int u = t - 4 * tw, k = u / th;
      cc = cset[k];
      r = u - k * th + 1;
      bool dup = false;
      for (int j = 0; j < k; j++) dup = dup || cset[j] == cc;
      for (int j = 0; j < 4; j++) dup = dup || (rset[j] == r && rset[j] >= 1 && rset[j] <= th);
      valid = cc >= 1 && cc <= tw && !dup;
    }
    if (valid) {
      ntg = hc_targets(y0 - 1 + r, x0 - 1 + cc, H, W, g, cx, cy, tgt);
      if (ntg > 0) hsrc = r * HC_RS + cc;
    }
  }
  // compute: owned column c of the tile, a band of its rows
  constexpr int NB = HC_THREADS / HC_T;
  const int c = (int)threadIdx.x % HC_T, band = (int)threadIdx.x / HC_T;
  const int ra = 1 + (th * band) / NB, rb = 1 + (th * (band + 1)) / NB;  // region rows
  const int rc = c + 1;                                                // region column
  const bool on = c < tw && rb > ra;
  for (int s = 0; s < P.niter; s++) {
    const bool q = s & 1;
    const V* su = q ? bu1 : bu0;
    const V* sv = q ? bv1 : bv0;
    V* du = q ? bu0 : bu1;
    V* dv = q ? bv0 : bv1;
    if (on) {
      HqRow<FAST> A, B, C;
      hq_load<HC_RS, FAST>(A, su, sv, ra - 1, rc - 1, rc, rc + 1);
      hq_load<HC_RS, FAST>(B, su, sv, ra, rc - 1, rc, rc + 1);
#pragma unroll 1
      for (int r = ra; r < rb; r += 3) {
        hq_load<HC_RS, FAST>(C, su, sv, r + 1, rc - 1, rc, rc + 1);
        hq_update<FAST>(A, B, C, r * HC_RS + rc, sfx, sfy, sft, du, dv, P.a2);
        if (r + 1 < rb) {
          hq_load<HC_RS, FAST>(A, su, sv, r + 2, rc - 1, rc, rc + 1);
          hq_update<FAST>(B, C, A, (r + 1) * HC_RS + rc, sfx, sfy, sft, du, dv, P.a2);
        }
        if (r + 2 < rb) {
          hq_load<HC_RS, FAST>(B, su, sv, r + 3, rc - 1, rc, rc + 1);
          hq_update<FAST>(C, A, B, (r + 2) * HC_RS + rc, sfx, sfy, sft, du, dv, P.a2);
        }
      }
    }
    __syncthreads();  // the tile's cells of this sweep are in shared memory
    if (hsrc >= 0) {  // copies on the halo rings (this CTA's and its neighbours')
      const V u = du[hsrc], v = dv[hsrc];
#pragma unroll
      for (int k = 0; k < HC_MAX_TARGETS; k++)
        if (k < ntg) {
          const unsigned int rank = (unsigned int)tgt[k] >> 16;
          const int o = tgt[k] & 0xffff;
          *cl.map_shared_rank(du + o, rank) = u;
          *cl.map_shared_rank(dv + o, rank) = v;
        }
    }
    cl.sync();  // the sweep, rings included, is visible cluster-wide
  }
  const V* fu = (P.niter & 1) ? bu1 : bu0;
  const V* fv = (P.niter & 1) ? bv1 : bv0;
  ok = true;
  for (int k = threadIdx.x; k < th * tw; k += HC_THREADS) {
    const int r = k / tw, cc = k - r * tw;
    const int o = (r + 1) * HC_RS + cc + 1;
    const size_t gi = (size_t)(y0 + r) * pitch + x0 + cc;
    P.U[gi] = (float)fu[o];
    P.V[gi] = (float)fv[o];
    ok = ok && isfinite(fu[o]) && isfinite(fv[o]);
  }
  if (__syncthreads_or(!ok) && threadIdx.x == 0 && P.niter > 0) atomicOr(status, OF_ST_NONFINITE_OUTPUT);
}

// Pair descriptors travel as kernel parameters (captured by value in a CUDA graph), up to
// HQ_DESC_CHUNK per launch of this copy kernel.
constexpr int HQ_DESC_CHUNK = 24;  // 24 x 128 B, within the classic 4 KB of parameters
struct HsqDescChunk {
  HsqPair p[HQ_DESC_CHUNK];
};
__global__ void hsq_desc_kernel(const __grid_constant__ HsqDescChunk chunk, int n, HsqPair* dst) {
  const int i = threadIdx.x;
  if (i < n) dst[i] = chunk.p[i];
}

}  // namespace ofb

using namespace ofb;

namespace {
// tile shapes (region width x height, sweeps per pass, threads per CTA) the persistent
// kernels are built for; hsq_with_shape maps an index to the same shape at compile time
struct HsqShape {
  int rw, rh, t, nt;
};
constexpr HsqShape kHsqShapes[] = {{64, 40, 4, 256}, {32, 24, 4, 256}, {64, 24, 4, 256}, {32, 32, 8, 256},
                                   {32, 48, 8, 512}};
constexpr int kHsqNumShapes = sizeof(kHsqShapes) / sizeof(kHsqShapes[0]);

template <int RW_, int RH_, int T_, int NT_>
struct HsqShapeT {
  static constexpr int RW = RW_, RH = RH_, T = T_, NT = NT_;
};

template <class F>
cudaError_t hsq_with_shape(int shape, F&& f) {
  switch (shape) {
    case 0: return f(HsqShapeT<64, 40, 4, 256>{});
    case 1: return f(HsqShapeT<32, 24, 4, 256>{});
    case 2: return f(HsqShapeT<64, 24, 4, 256>{});
    case 3: return f(HsqShapeT<32, 32, 8, 256>{});
    case 4: return f(HsqShapeT<32, 48, 8, 512>{});
    default: return cudaErrorInvalidValue;
  }
}

// which persistent kernel a launch uses
enum HqKind { HQ_QUEUE, HQ_RESIDENT, HQ_ADAPTIVE };

template <class S, bool FAST>
const void* hsq_kernel_ptr(HqKind kind) {
  constexpr int RW = S::RW, RH = S::RH, T = S::T, NT = S::NT;
  return kind == HQ_RESIDENT ? (const void*)hsr_kernel<RW, RH, T, FAST, NT>
         : kind == HQ_QUEUE  ? (const void*)hsq_kernel<RW, RH, T, FAST, NT>
                             : (const void*)hsa_kernel<RW, RH, T, FAST, NT>;
}

// Opts the chosen kernel into its shared memory and reports how many of its CTAs fit on an SM.
template <class S>
cudaError_t hsq_resident(bool fast, HqKind kind, int* per_sm) {
  constexpr int RW = S::RW, RH = S::RH, T = S::T, NT = S::NT;
  using G = HqTile<RW, RH, T>;
  cudaError_t e;
  if (kind == HQ_RESIDENT)
    e = fast ? OF_SMEM_OPT_IN((hsr_kernel<RW, RH, T, true, NT>), G::smem(true))
             : OF_SMEM_OPT_IN((hsr_kernel<RW, RH, T, false, NT>), G::smem(false));
  else if (kind == HQ_QUEUE)
    e = fast ? OF_SMEM_OPT_IN((hsq_kernel<RW, RH, T, true, NT>), G::smem(true))
             : OF_SMEM_OPT_IN((hsq_kernel<RW, RH, T, false, NT>), G::smem(false));
  else
    e = fast ? OF_SMEM_OPT_IN((hsa_kernel<RW, RH, T, true, NT>), G::smem(true))
             : OF_SMEM_OPT_IN((hsa_kernel<RW, RH, T, false, NT>), G::smem(false));
  if (e != cudaSuccess) return e;
  const void* k = fast ? hsq_kernel_ptr<S, true>(kind) : hsq_kernel_ptr<S, false>(kind);
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k, NT, G::smem(fast));
}

template <class S, bool FAST>
void hsq_launch_as(HqKind kind, int grid, const HsqPair* pairs, int n, unsigned int tiles_total, int max_passes,
                   unsigned long long* ticket, unsigned int* done, int* status, long long wait_limit, int* err_flag,
                   unsigned int* arrived, int* mode, cudaStream_t st) {
  constexpr int RW = S::RW, RH = S::RH, T = S::T, NT = S::NT;
  const size_t smem = HqTile<RW, RH, T>::smem(FAST);
  if (kind == HQ_RESIDENT)
    hsr_kernel<RW, RH, T, FAST, NT><<<grid, NT, smem, st>>>(pairs, n, done, status, wait_limit, err_flag);
  else if (kind == HQ_QUEUE)
    hsq_kernel<RW, RH, T, FAST, NT><<<grid, NT, smem, st>>>(pairs, n, tiles_total, max_passes, ticket, done, status,
                                                           wait_limit, err_flag);
  else
    hsa_kernel<RW, RH, T, FAST, NT><<<grid, NT, smem, st>>>(pairs, n, tiles_total, max_passes, ticket, done, status,
                                                           wait_limit, err_flag, arrived, mode);
}
}  // namespace

// The cluster schedule's geometry for an H x W image: at most HC_MAX_CTAS tiles of at most
// HC_T x HC_T cells.
static bool hc_geometry(int H, int W, HcGeom* g) {
  if (H < 16 || W < 16) return false;
  g->CX = (W + HC_T - 1) / HC_T;
  g->CY = (H + HC_T - 1) / HC_T;
  if (g->CX * g->CY > HC_MAX_CTAS) return false;
  g->TW = (W + g->CX - 1) / g->CX;
  g->TH = (H + g->CY - 1) / g->CY;
  return true;
}

template <bool FAST>
static cudaError_t hsc_config(const HcGeom& g, cudaStream_t st, cudaLaunchConfig_t* cfg, cudaLaunchAttribute* attr) {
  cudaError_t e = cudaFuncSetAttribute(hsc_kernel<FAST>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e == cudaSuccess) e = OF_SMEM_OPT_IN(hsc_kernel<FAST>, hc_smem<FAST>());
  *cfg = cudaLaunchConfig_t{};
  cfg->gridDim = dim3(g.CX, g.CY, 1);
  cfg->blockDim = dim3(HC_THREADS, 1, 1);
  cfg->dynamicSmemBytes = hc_smem<FAST>();
  cfg->stream = st;
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = g.CX;
  attr[0].val.clusterDim.y = g.CY;
  attr[0].val.clusterDim.z = 1;
  cfg->attrs = attr;
  cfg->numAttrs = 1;
  return e;
}

// Whether the device can hold a cluster of this shape (all its CTAs at once).
static bool hsc_schedulable(bool fast, const HcGeom& g) {
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute attr[1];
  int n = 0;
  cudaError_t e;
  if (fast) {
    e = hsc_config<true>(g, nullptr, &cfg, attr);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters(&n, hsc_kernel<true>, &cfg);
  } else {
    e = hsc_config<false>(g, nullptr, &cfg, attr);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters(&n, hsc_kernel<false>, &cfg);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();  // clear: a refused shape only means the other schedules run
    return false;
  }
  return n >= 1;
}

static cudaError_t hsc_launch(bool fast, const HsqPair& P, const HcGeom& g, int* status, cudaStream_t st) {
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute attr[1];
  cudaError_t e;
  if (fast) {
    e = hsc_config<true>(g, st, &cfg, attr);
    if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg, hsc_kernel<true>, P, g, status);
  } else {
    e = hsc_config<false>(g, st, &cfg, attr);
    if (e == cudaSuccess) e = cudaLaunchKernelEx(&cfg, hsc_kernel<false>, P, g, status);
  }
  return e;
}

// tiles of a pair under the tile shape that cuts it finest (sizes the per-tile counters)
static size_t hsq_max_tiles(const OfHsBatchPair* pairs, int n) {
  size_t total = 0;
  for (int i = 0; i < n; i++) {
    size_t best = 0;
    for (int k = 0; k < kHsqNumShapes; k++) {
      const int TW = kHsqShapes[k].rw - 2 * kHsqShapes[k].t, TH = kHsqShapes[k].rh - 2 * kHsqShapes[k].t;
      const size_t t = (size_t)((pairs[i].W + TW - 1) / TW) * (size_t)((pairs[i].H + TH - 1) / TH);
      if (t > best) best = t;
    }
    total += best;
  }
  return total;
}

// The launch-control part at the start of the workspace: descriptors, ticket, per-tile
// counters, error flag, the adaptive schedule's arrival count and mode word.
struct HsqControl {
  HsqPair* dpairs;
  unsigned long long* ticket;
  unsigned int* done;  // passes (queue) or warp stages (resident) finished, per tile
  int* err_flag;
  unsigned int* arrived;
  int* mode;
};

static HsqControl hsq_carve_control(Carver& c, const OfHsBatchPair* pairs, int n) {
  HsqControl k;
  k.dpairs = c.take<HsqPair>((size_t)n);
  k.ticket = c.take<unsigned long long>(1);
  k.done = c.take<unsigned int>(hsq_max_tiles(pairs, n));
  k.err_flag = c.take<int>(1);
  k.arrived = c.take<unsigned int>(1);
  k.mode = c.take<int>(1);
  return k;
}

extern "C" int of_hs_batch_schedule(const OfHsBatchPair* pairs, int n, const void* workspace, size_t workspace_bytes,
                                    int* schedule, void* stream) {
  OF_REQUIRE(pairs && n > 0 && n <= (1 << 20) && schedule, "of_hs_batch_schedule: bad arguments");
  Carver c(const_cast<void*>(workspace), workspace_bytes);
  const HsqControl ctl = hsq_carve_control(c, pairs, n);
  OF_REQUIRE(workspace && c.ok(), "of_hs_batch_schedule: workspace too small");
  cudaStream_t st = as_stream(stream);
  int m = 0;
  cudaError_t e = cudaMemcpyAsync(&m, ctl.mode, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_hs_batch_schedule: %s", cudaGetErrorString(e));
  *schedule = m;
  return OF_OK;
}

extern "C" size_t of_hs_batch_workspace_size(const OfHsBatchPair* pairs, int n) {
  if (!pairs || n <= 0) return 0;
  Sizer s;
  s.take<HsqPair>((size_t)n);
  s.take<unsigned long long>(1);
  s.take<unsigned int>(hsq_max_tiles(pairs, n));
  s.take<int>(1);
  s.take<unsigned int>(1);
  s.take<int>(1);
  for (int i = 0; i < n; i++) {
    size_t N = (size_t)pairs[i].H * (size_t)pairs[i].pitch;
    for (int k = 0; k < 7; k++) s.take<float>(N);
  }
  return s.off;
}

extern "C" int of_hs_batch(const OfHsBatchPair* pairs, int n, const OfTuning* tuning, int* status,
                           long long wait_limit, void* workspace, size_t workspace_bytes, void* stream) {
  OF_REQUIRE(pairs && n > 0 && n <= (1 << 20), "of_hs_batch: bad pair list");
  OF_REQUIRE(status, "of_hs_batch: status (a device array of n ints) is required");
  OF_REQUIRE(wait_limit > 0, "of_hs_batch: wait_limit must be positive");
  int shape = tuning ? tuning->tile_shape : 0;
  const int arith = tuning ? tuning->hs_arithmetic : OF_HS_EXACT;
  OF_REQUIRE(arith == OF_HS_EXACT || arith == OF_HS_FAST, "of_hs_batch: hs_arithmetic must be OF_HS_EXACT or OF_HS_FAST");
  const bool fast = arith == OF_HS_FAST;
  const int sched = tuning ? tuning->hs_schedule : OF_HS_SCHED_AUTO;
  OF_REQUIRE(sched == OF_HS_SCHED_AUTO || sched == OF_HS_SCHED_QUEUE || sched == OF_HS_SCHED_RESIDENT ||
                 sched == OF_HS_SCHED_CLUSTER,
             "of_hs_batch: hs_schedule must be OF_HS_SCHED_AUTO, _QUEUE, _RESIDENT or _CLUSTER");
  OF_REQUIRE(shape >= 0 && shape < kHsqNumShapes, "of_hs_batch: tile_shape must be in 0..%d", kHsqNumShapes - 1);
  const HsqShape sh = kHsqShapes[shape];
  const int TW = sh.rw - 2 * sh.t, TH = sh.rh - 2 * sh.t;
  size_t need = of_hs_batch_workspace_size(pairs, n);
  if (!workspace || workspace_bytes < need)
    return set_error(OF_ERR_WORKSPACE, "of_hs_batch: workspace too small (%zu < %zu)", workspace_bytes, need);
  cudaStream_t st = as_stream(stream);
  Carver c(workspace, workspace_bytes);
  const HsqControl ctl = hsq_carve_control(c, pairs, n);
  HsqPair* dpairs = ctl.dpairs;
  unsigned long long* ticket = ctl.ticket;
  unsigned int* done = ctl.done;
  int* err_flag = ctl.err_flag;
  unsigned int* arrived = ctl.arrived;
  int* mode = ctl.mode;
  // descriptors are built on the host and written to the workspace by kernels that take
  // them as parameters (no host buffer outlives this call, and a graph capture holds copies)
  HsqPair* hp = new HsqPair[n];
  unsigned int tiles_total = 0;
  int max_passes = 0;
  for (int i = 0; i < n; i++) {
    const OfHsBatchPair& q = pairs[i];
    if (bad_plane(q.I0, q.H, q.W, q.pitch) || !q.I1 || !q.U || !q.V || q.niter < 0) {
      delete[] hp;
      return set_error(OF_ERR_INVALID, "of_hs_batch: pair %d: bad plane or niter", i);
    }
    HsqPair& P = hp[i];
    P.I0 = q.I0;
    P.I1 = q.I1;
    P.U = q.U;
    P.V = q.V;
    size_t N = (size_t)q.H * q.pitch;
    P.fx = c.take<float>(N);
    P.fy = c.take<float>(N);
    P.ft = c.take<float>(N);
    P.U0 = c.take<float>(N);
    P.V0 = c.take<float>(N);
    P.Ub = c.take<float>(N);
    P.Vb = c.take<float>(N);
    P.H = q.H;
    P.W = q.W;
    P.pitch = q.pitch;
    P.a2 = q.alpha * q.alpha;
    P.niter = q.niter;
    P.passes = 1 + (q.niter + sh.t - 1) / sh.t;
    P.tx = (q.W + TW - 1) / TW;
    P.tiles = P.tx * ((q.H + TH - 1) / TH);
    P.tile0 = tiles_total;
    tiles_total += (unsigned int)P.tiles;
    if (P.passes > max_passes) max_passes = P.passes;
  }
  // the cluster schedule (one pair that one cluster covers); it needs neither the
  // descriptors in memory nor the counters
  if (sched == OF_HS_SCHED_CLUSTER) {
    HcGeom hg;
    const bool fits = n == 1 && hc_geometry(pairs[0].H, pairs[0].W, &hg);
    const HsqPair P = hp[0];
    delete[] hp;
    if (!fits)
      return set_error(OF_ERR_INVALID, "of_hs_batch: the cluster schedule takes one pair of at most %d tiles of %d x %d",
                       HC_MAX_CTAS, HC_T, HC_T);
    if (!hsc_schedulable(fast, hg))
      return set_error(OF_ERR_UNSUPPORTED, "of_hs_batch: the device cannot hold a %d x %d cluster of this kernel",
                       hg.CX, hg.CY);
    cudaError_t e = cudaMemsetAsync(mode, 0, sizeof(int), st);  // no adaptive decision
    if (e == cudaSuccess) e = hsc_launch(fast, P, hg, status, st);
    if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_hs_batch: cluster launch: %s", cudaGetErrorString(e));
    return check_launch("of_hs_batch", 1);
  }
  long long nl = 0;
  for (int b = 0; b < n; b += HQ_DESC_CHUNK) {
    HsqDescChunk chunk;
    const int m = n - b < HQ_DESC_CHUNK ? n - b : HQ_DESC_CHUNK;
    for (int k = 0; k < m; k++) chunk.p[k] = hp[b + k];
    hsq_desc_kernel<<<1, HQ_DESC_CHUNK, 0, st>>>(chunk, m, dpairs + b);
    nl++;
  }
  delete[] hp;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_hs_batch: descriptor kernel: %s", cudaGetErrorString(e));
  // ticket, counters, error flag, arrival count and mode word are contiguous
  e = cudaMemsetAsync(ticket, 0, (size_t)((char*)(mode + 1) - (char*)ticket), st);
  if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_hs_batch: %s", cudaGetErrorString(e));
  int dev = 0, sms = kNumSMs;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // every CTA must be resident (items wait for items of running CTAs)
  auto capacity = [&](HqKind kind, long long* cap) {
    int per_sm = 0;
    const cudaError_t rc =
        hsq_with_shape(shape, [&](auto S) { return hsq_resident<decltype(S)>(fast, kind, &per_sm); });
    *cap = (long long)sms * per_sm;
    return rc == cudaSuccess && per_sm >= 1;
  };
  // RESIDENT: one CTA per tile, all of them running at once (refused when the device cannot
  // hold them); AUTO: the adaptive kernel with one CTA per tile when the device can hold them
  // (it falls back to the queue itself when they do not all get an SM), else the queue
  HqKind kind = HQ_QUEUE;
  long long cap = 0;
  if (sched == OF_HS_SCHED_RESIDENT || sched == OF_HS_SCHED_AUTO) {
    const HqKind k = sched == OF_HS_SCHED_RESIDENT ? HQ_RESIDENT : HQ_ADAPTIVE;
    if (!capacity(k, &cap)) return set_error(OF_ERR_CUDA, "of_hs_batch: occupancy query failed");
    if ((long long)tiles_total <= cap)
      kind = k;
    else if (sched == OF_HS_SCHED_RESIDENT)
      return set_error(OF_ERR_INVALID, "of_hs_batch: %u tiles exceed the %lld resident CTAs of the resident schedule",
                       tiles_total, cap);
  }
  long long grid = tiles_total;  // resident and adaptive: one CTA per tile
  if (kind == HQ_QUEUE) {
    if (!capacity(HQ_QUEUE, &cap)) return set_error(OF_ERR_CUDA, "of_hs_batch: occupancy query failed");
    grid = cap < (long long)tiles_total ? cap : (long long)tiles_total;  // no more CTAs than items of a pass
  }
  if (grid < 1) grid = 1;
  e = hsq_with_shape(shape, [&](auto S) {
    using Sh = decltype(S);
    if (fast)
      hsq_launch_as<Sh, true>(kind, (int)grid, dpairs, n, tiles_total, max_passes, ticket, done, status, wait_limit,
                              err_flag, arrived, mode, st);
    else
      hsq_launch_as<Sh, false>(kind, (int)grid, dpairs, n, tiles_total, max_passes, ticket, done, status, wait_limit,
                               err_flag, arrived, mode, st);
    return cudaGetLastError();
  });
  if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_hs_batch: launch: %s", cudaGetErrorString(e));
  return check_launch("of_hs_batch", nl + 1);
}

extern "C" int of_hs_batch_shape(int index, int* region_w, int* region_h, int* sweeps_per_pass) {
  if (index < 0 || index >= kHsqNumShapes) return OF_ERR_INVALID;
  if (region_w) *region_w = kHsqShapes[index].rw;
  if (region_h) *region_h = kHsqShapes[index].rh;
  if (sweeps_per_pass) *sweeps_per_pass = kHsqShapes[index].t;
  return OF_OK;
}
