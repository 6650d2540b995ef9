// of_batch_run: the pyramid driver genericPyramidalOpticalFlow
// (src/GenericPyramidalOpticalFlow.py:237-415) in C++ over this library's entry points,
// for callers outside Python that run many frame pairs (the batched workload of uneven
// pairs, HS / LK / Farneback mains, optional Liu-Shen refine).  Its results equal the
// Python drop-in's bit for bit: the same kernels are called with the same arguments in the
// same order.  Host constants that the reference computes in Python (prefilter taps, the
// Farneback kernels and polynomial constants) come with each pair's descriptor.
//
// Pairs run one after another in stream order and share one scratch arena (its size is
// the largest pair's).  The Horn-Schunck solves of single-level pairs are not run one by
// one: after every pair's set-up, all of them run in one persistent launch (of_hs_batch).
#include <math.h>
#include <string.h>

#include <vector>

#include "common.cuh"

namespace {

using namespace ofb;

// Scratch carving with a sizing mode: the driver runs once without launching anything to
// measure the arena, then for real.
struct Arena {
  bool sizing;
  char* base;
  size_t cap, off;
  template <class T>
  T* take(size_t n) {
    off = align_up(off, 256);
    T* p = sizing ? nullptr : reinterpret_cast<T*>(base + off);
    off += n * sizeof(T);
    return p;
  }
};

struct Plane {
  float* p;
  int H, W, pitch;
};

Plane new_plane(Arena& A, int H, int W, int planes = 1) {
  const int P = (W + 31) / 32 * 32;
  return Plane{A.take<float>((size_t)planes * H * P), H, W, P};
}

#define CALL(expr)                          \
  do {                                      \
    if (!A.sizing) {                        \
      int rc_ = (expr);                     \
      if (rc_ != OF_OK) return rc_;         \
    }                                       \
  } while (0)

#define CUDA_CALL(expr)                                                                        \
  do {                                                                                         \
    if (!A.sizing) {                                                                           \
      cudaError_t e_ = (expr);                                                                 \
      if (e_ != cudaSuccess) return set_error(OF_ERR_CUDA, "of_batch_run: %s", cudaGetErrorString(e_)); \
    }                                                                                          \
  } while (0)

int rint_i(double v) { return (int)nearbyint(v); }  // numpy's round (half to even)

int zero(Arena& A, const Plane& p, cudaStream_t st) {
  CUDA_CALL(cudaMemsetAsync(p.p, 0, sizeof(float) * (size_t)p.H * p.pitch, st));
  return OF_OK;
}

int copy_plane(Arena& A, const float* src, int src_pitch, float* dst, int dst_pitch, int H, int W, cudaStream_t st) {
  CUDA_CALL(cudaMemcpy2DAsync(dst, sizeof(float) * dst_pitch, src, sizeof(float) * src_pitch, sizeof(float) * W, H,
                              cudaMemcpyDeviceToDevice, st));
  return OF_OK;
}

int resize_to(Arena& A, const Plane& src, const Plane& dst, int filter, cudaStream_t st) {
  const size_t wn = of_resize_workspace_size(src.H, src.W, dst.H, dst.W, filter);
  void* ws = A.take<char>(wn);
  CALL(of_resize(src.p, src.H, src.W, src.pitch, dst.p, dst.H, dst.W, dst.pitch, filter, ws, wn, st));
  return OF_OK;
}

int prefilter_to(Arena& A, const Plane& src, Plane& dst, const float* taps, int K, cudaStream_t st) {
  dst = new_plane(A, src.H, src.W);
  CALL(of_prefilter_f32(src.p, src.pitch, dst.p, dst.pitch, src.H, src.W, taps, K, st));
  return OF_OK;
}

// Farneback_PyCL.compute (src/Farneback_PyCL.py:461-603) on one pyramid level's frames;
// U, V: the initial flow, replaced by the result.
int farneback(Arena& A, const OfFbParams& fb, const Plane& im1, const Plane& im2, Plane& U, Plane& V,
              cudaStream_t st) {
  const int Hs = im1.H, Ws = im1.W;
  int nlev = 0;
  double scale = 1.0;
  while (nlev < fb.levels - 1) {
    scale *= fb.pyr_scale;
    if (Ws * scale < 32 || Hs * scale < 32) break;
    nlev++;
  }
  Plane cx{}, cy{};
  bool have_prev = false;
  for (int k = nlev; k >= 0; k--) {
    double sc = 1.0;
    for (int i = 0; i < k; i++) sc *= fb.pyr_scale;
    const double sigma = (1.0 / sc - 1.0) * 0.5;
    int smooth = (int)nearbyint(sigma * 5.0) | 1;
    if (smooth < 3) smooth = 3;
    if (k >= OF_FB_MAX_LEVELS || !fb.level_taps[k] || fb.level_kh[k] != smooth / 2)
      return set_error(OF_ERR_INVALID, "of_batch_run: Farneback level %d needs its %d-tap frame blur", k, smooth);
    const int w = rint_i(Ws * sc), h = rint_i(Hs * sc);
    Plane nx = new_plane(A, h, w), ny = new_plane(A, h, w);
    const Plane& sx = have_prev ? cx : U;
    const Plane& sy = have_prev ? cy : V;
    const float s = have_prev ? (float)(1.0 / fb.pyr_scale) : (float)sc;
    Plane rx = new_plane(A, h, w), ry = new_plane(A, h, w);
    if (resize_to(A, sx, rx, OF_FILTER_BILINEAR, st) || resize_to(A, sy, ry, OF_FILTER_BILINEAR, st))
      return OF_ERR_CUDA;
    if (s != 1.0f) {  // x * 1 is x: the full-size level keeps the resized copies
      CALL(of_scale(rx.p, nx.p, s, h, w, nx.pitch, st));
      CALL(of_scale(ry.p, ny.p, s, h, w, ny.pitch, st));
      cx = nx;
      cy = ny;
    } else {
      cx = rx;
      cy = ry;
    }
    Plane RA = new_plane(A, 5 * h, w), RB = new_plane(A, 5 * h, w);
    RA.H = RB.H = h;
    const bool fused = h == Hs && w == Ws && fb.level_kh[k] == 1 && (fb.poly.polyN == 5 || fb.poly.polyN == 7) &&
                       h >= 3 && w >= 3 && im1.pitch == RA.pitch && im2.pitch == RA.pitch;
    for (int f = 0; f < 2; f++) {
      const Plane& src = f ? im2 : im1;
      if (fused) {  // blur and expansion in one launch at the full-size level
        CALL(of_fb_polyexp_blurred(src.p, (f ? RB : RA).p, h, w, RA.pitch, fb.level_taps[k], &fb.poly, st));
        continue;
      }
      Plane bl = new_plane(A, Hs, Ws);
      CALL(of_fb_blur(src.p, bl.p, Hs, Ws, bl.pitch, 1, fb.level_taps[k], fb.level_kh[k], st));
      Plane lv = bl;
      if (h != Hs || w != Ws) {
        lv = new_plane(A, h, w);
        if (resize_to(A, bl, lv, OF_FILTER_BILINEAR, st)) return OF_ERR_CUDA;
      }
      const Plane& R = f ? RB : RA;
      if (lv.pitch != R.pitch) return set_error(OF_ERR_INVALID, "of_batch_run: pitch mismatch");
      CALL(of_fb_polyexp(lv.p, R.p, h, w, R.pitch, &fb.poly, st));
    }
    Plane M = new_plane(A, 5 * h, w), Mb = new_plane(A, 5 * h, w);
    CALL(of_fb_update_matrices(cx.p, cy.p, RA.p, RB.p, M.p, h, w, M.pitch, st));
    if (fb.use_gaussian) {
      for (int i = 0; i < fb.niters; i++) {
        const int upd = i < fb.niters - 1;
        CALL(of_fb_iteration(M.p, Mb.p, RA.p, RB.p, cx.p, cy.p, h, w, M.pitch, fb.window_taps, fb.window_kh, upd,
                             st));
        if (upd) {
          Plane t = M;
          M = Mb;
          Mb = t;
        }
      }
    } else {
      const int kh = fb.window_size / 2;
      for (int i = 0; i < fb.niters; i++) {
        CALL(of_fb_box5(M.p, Mb.p, h, w, M.pitch, kh, st));
        CALL(of_fb_update_flow(Mb.p, cx.p, cy.p, h, w, M.pitch, st));
        if (i < fb.niters - 1) CALL(of_fb_update_matrices(cx.p, cy.p, RA.p, RB.p, M.p, h, w, M.pitch, st));
      }
    }
    have_prev = true;
  }
  U = cx;
  V = cy;
  return OF_OK;
}

struct Deferred {  // a single-level Horn-Schunck solve gathered for one persistent launch
  OfHsBatchPair p;
  int pair;
  Plane U, V;      // the solve's fields (U, V in place)
  Plane Ua, Va;    // the accumulators receiving them
};

// One pair.  `defer` non-null: a single-level Horn-Schunck main is not solved here; its
// inputs are recorded for the persistent launch and the caller finishes the pair.
int run_pair(Arena& A, const OfPairDesc& d, int index, int* status, std::vector<Deferred>* defer, cudaStream_t st) {
  const int H = d.H, W = d.W;
  // the adapters' pyramid defaults (getGenericPyramidalDefaults) unless the caller overrides
  int warping = 1, inter = 1, last = 0;
  if (d.method == OF_METHOD_HS) warping = 1, last = 1;
  else if (d.method == OF_METHOD_LK) warping = 0, inter = 1, last = 0;
  else warping = 0, last = 1;  // Farneback
  if (d.warping >= 0) warping = d.warping;
  if (d.intermediate_scaling >= 0) inter = d.intermediate_scaling;
  if (d.scaling >= 0) last = d.scaling;
  Plane I1, I2;
  if (d.frame_u8) {
    I1 = new_plane(A, H, W);
    I2 = new_plane(A, H, W);
    CALL(of_u8_to_f32((const uint8_t*)d.I0, d.in_pitch, I1.p, I1.pitch, H, W, st));
    CALL(of_u8_to_f32((const uint8_t*)d.I1, d.in_pitch, I2.p, I2.pitch, H, W, st));
  } else {
    I1 = Plane{(float*)d.I0, H, W, d.in_pitch};
    I2 = Plane{(float*)d.I1, H, W, d.in_pitch};
  }
  const int L = d.levels;
  double scale = 1.0 / pow(2.0, L - 1);
  Plane U{}, V{}, Ua{}, Va{};
  int ph = 0, pw = 0;  // previous level's working size
  int calls = 0;       // main-adapter calls so far (Horn-Schunck pops one alpha per call)
  for (int level = 1; level <= L; level++) {
    const int lscale = level == L ? last : inter;
    Plane n1 = I1, n2 = I2;
    if (scale < 1.0 && level != L) {
      const int w = rint_i(I1.W * scale), h = rint_i(I1.H * scale);
      n1 = new_plane(A, h, w);
      n2 = new_plane(A, h, w);
      if (resize_to(A, I1, n1, OF_FILTER_BICUBIC, st) || resize_to(A, I2, n2, OF_FILTER_BICUBIC, st))
        return OF_ERR_CUDA;
    }
    const int h = n1.H, w = n1.W;
    Plane w1 = n1, w2 = n2;
    if (level > 1) {
      const float sx = lscale ? (float)w / (float)pw : 1.0f, sy = lscale ? (float)h / (float)ph : 1.0f;
      Plane us = new_plane(A, h, w), vs = new_plane(A, h, w);
      if (ph != h || pw != w) {
        const size_t wn = 2 * of_spline_workspace_size(ph, pw, h, w);
        void* ws = A.take<char>(wn);
        CALL(of_spline_upsample_pair(Ua.p, Va.p, ph, pw, Ua.pitch, us.p, vs.p, h, w, us.pitch, sx, sy, ws, wn, st));
      } else if (lscale) {
        CALL(of_scale(Ua.p, us.p, sx, h, w, us.pitch, st));
        CALL(of_scale(Va.p, vs.p, sy, h, w, vs.pitch, st));
      } else {  // a copy: the mains update their initial field in place
        if (copy_plane(A, Ua.p, Ua.pitch, us.p, us.pitch, h, w, st) ||
            copy_plane(A, Va.p, Va.pitch, vs.p, vs.pitch, h, w, st))
          return OF_ERR_CUDA;
      }
      U = new_plane(A, h, w);
      V = new_plane(A, h, w);
      if (warping) {
        // with the bilinear warp (biLinear=False is not offered here)
        Plane o1 = new_plane(A, h, w), o2 = new_plane(A, h, w);
        if (n1.pitch != o1.pitch) {
          Plane c1 = new_plane(A, h, w), c2 = new_plane(A, h, w);
          if (copy_plane(A, n1.p, n1.pitch, c1.p, c1.pitch, h, w, st) ||
              copy_plane(A, n2.p, n2.pitch, c2.p, c2.pitch, h, w, st))
            return OF_ERR_CUDA;
          n1 = c1;
          n2 = c2;
        }
        CALL(of_warp_pair_bilinear(n1.p, n2.p, us.p, vs.p, o1.p, o2.p, h, w, o1.pitch, st));
        w1 = o1;
        w2 = o2;
        Ua = us;
        Va = vs;
        if (zero(A, U, st) || zero(A, V, st)) return OF_ERR_CUDA;
      } else {
        Ua = new_plane(A, h, w);
        Va = new_plane(A, h, w);
        if (zero(A, Ua, st) || zero(A, Va, st)) return OF_ERR_CUDA;
        U = us;
        V = vs;
      }
    } else {
      U = new_plane(A, h, w);
      V = new_plane(A, h, w);
      Ua = new_plane(A, h, w);
      Va = new_plane(A, h, w);
      if (zero(A, U, st) || zero(A, V, st) || zero(A, Ua, st) || zero(A, Va, st)) return OF_ERR_CUDA;
    }
    Plane k1 = w1, k2 = w2;
    if (d.filter > 1e-3f) {
      if (prefilter_to(A, w1, k1, d.filter_taps, 3, st) || prefilter_to(A, w2, k2, d.filter_taps, 3, st))
        return OF_ERR_CUDA;
    }
    Plane o1 = n1, o2 = n2;
    if (d.refine_ls && d.filter_opt > 1e-3f) {
      if (prefilter_to(A, n1, o1, d.filter_opt_taps, 5, st) || prefilter_to(A, n2, o2, d.filter_opt_taps, 5, st))
        return OF_ERR_CUDA;
    }
    // the main adapter (k1, k2 share one pitch with U, V: every plane here is 32-aligned)
    if (k1.pitch != U.pitch) {
      Plane c1 = new_plane(A, h, w), c2 = new_plane(A, h, w);
      if (copy_plane(A, k1.p, k1.pitch, c1.p, c1.pitch, h, w, st) ||
          copy_plane(A, k2.p, k2.pitch, c2.p, c2.pitch, h, w, st))
        return OF_ERR_CUDA;
      k1 = c1;
      k2 = c2;
    }
    if (d.method == OF_METHOD_HS) {
      if (calls >= d.hs_nalphas) return set_error(OF_ERR_INVALID, "of_batch_run: pair %d: too few alphas", index);
      const float alpha = d.hs_alphas[d.hs_nalphas - 1 - calls];
      if (defer && L == 1 && !d.refine_ls) {
        Deferred q;
        q.p = OfHsBatchPair{k1.p, k2.p, U.p, V.p, h, w, U.pitch, alpha, d.hs_niter};
        q.pair = index;
        q.U = U;
        q.V = V;
        q.Ua = Ua;
        q.Va = Va;
        if (!A.sizing) defer->push_back(q);
        calls++;
        scale *= 2;
        continue;
      }
      const size_t wn = of_hs_workspace_size(h, w, U.pitch);
      void* ws = A.take<char>(wn);
      CALL(of_hs_solve(k1.p, k2.p, U.p, V.p, h, w, U.pitch, alpha, d.hs_niter, nullptr, ws, wn, st));
    } else if (d.method == OF_METHOD_LK) {
      CALL(of_lk_dense(k1.p, k2.p, U.p, V.p, h, w, U.pitch, d.lk_half_win, d.lk_niter, nullptr, nullptr, nullptr, st));
    } else if (d.method == OF_METHOD_FB) {
      if (!d.fb) return set_error(OF_ERR_INVALID, "of_batch_run: pair %d: Farneback parameters missing", index);
      if (farneback(A, *d.fb, k1, k2, U, V, st)) return OF_ERR_CUDA;
    } else {
      return set_error(OF_ERR_INVALID, "of_batch_run: pair %d: unknown method %d", index, d.method);
    }
    calls++;
    if (d.refine_ls) {
      // Liu-Shen refine on the FILTER_OPT-prefiltered, unwarped frames (:379-385, 408-410)
      if (o1.pitch != U.pitch) {
        Plane c1 = new_plane(A, h, w), c2 = new_plane(A, h, w);
        if (copy_plane(A, o1.p, o1.pitch, c1.p, c1.pitch, h, w, st) ||
            copy_plane(A, o2.p, o2.pitch, c2.p, c2.pitch, h, w, st))
          return OF_ERR_CUDA;
        o1 = c1;
        o2 = c2;
      }
      Plane u2 = new_plane(A, h, w), v2 = new_plane(A, h, w);
      if (copy_plane(A, U.p, U.pitch, u2.p, u2.pitch, h, w, st) || copy_plane(A, V.p, V.pitch, v2.p, v2.pitch, h, w, st))
        return OF_ERR_CUDA;
      const size_t wn = of_ls_workspace_size(h, w, u2.pitch, 60);
      void* ws = A.take<char>(wn);
      int* iters = A.take<int>(1);
      double* err = A.take<double>(1);
      CALL(of_ls_solve_mode(o1.p, o2.p, u2.p, v2.p, h, w, u2.pitch, d.ls_h, 60, 1e-8, d.ls_arithmetic, iters, err,
                            ws, wn, st));
      if (status && level == L) CALL(of_ls_status(iters, err, 60, 1e-8, status + index, st));
      U = u2;
      V = v2;
    }
    CALL(of_accumulate(Ua.p, U.p, h, w, Ua.pitch, st));
    CALL(of_accumulate(Va.p, V.p, h, w, Va.pitch, st));
    ph = h;
    pw = w;
    scale *= 2;
  }
  if (!(defer && d.method == OF_METHOD_HS && L == 1 && !d.refine_ls)) {
    if (copy_plane(A, Ua.p, Ua.pitch, d.U, d.out_pitch, H, W, st) ||
        copy_plane(A, Va.p, Va.pitch, d.V, d.out_pitch, H, W, st))
      return OF_ERR_CUDA;
    if (status) {
      CALL(of_check_finite(d.U, H, W, d.out_pitch, status + index, OF_ST_NONFINITE_OUTPUT, st));
      CALL(of_check_finite(d.V, H, W, d.out_pitch, status + index, OF_ST_NONFINITE_OUTPUT, st));
    }
  }
  return OF_OK;
}

int validate(const OfPairDesc& d, int i) {
  if (!d.I0 || !d.I1 || !d.U || !d.V || d.H < 4 || d.W < 4 || d.in_pitch < d.W || d.out_pitch < d.W)
    return set_error(OF_ERR_INVALID, "of_batch_run: pair %d: bad planes", i);
  if (d.levels < 1 || d.levels > 8) return set_error(OF_ERR_INVALID, "of_batch_run: pair %d: levels in 1..8", i);
  if (d.filter > 1e-3f && !d.filter_taps) return set_error(OF_ERR_INVALID, "of_batch_run: pair %d: filter taps", i);
  if (d.refine_ls && d.filter_opt > 1e-3f && !d.filter_opt_taps)
    return set_error(OF_ERR_INVALID, "of_batch_run: pair %d: filter_opt taps", i);
  return OF_OK;
}

}  // namespace

static size_t pair_arena(const OfPairDesc& d, int i) {
  Arena A{true, nullptr, 0, 0};
  std::vector<Deferred> defer;
  if (run_pair(A, d, i, nullptr, &defer, nullptr) != OF_OK) return 0;
  return A.off;
}

extern "C" size_t of_batch_workspace_size(const OfPairDesc* descs, int n, const OfTuning* tuning) {
  (void)tuning;
  if (!descs || n <= 0) return 0;
  // one arena per pair slot: a deferred Horn-Schunck pair keeps its planes until the
  // persistent launch, so the arenas are laid out one after another
  Sizer s;
  for (int i = 0; i < n; i++) {
    if (validate(descs[i], i) != OF_OK) return 0;
    s.take<char>(pair_arena(descs[i], i));
  }
  std::vector<OfHsBatchPair> hs;
  for (int i = 0; i < n; i++)
    if (descs[i].method == OF_METHOD_HS && descs[i].levels == 1 && !descs[i].refine_ls) {
      const int P = (descs[i].W + 31) / 32 * 32;
      hs.push_back(OfHsBatchPair{nullptr, nullptr, nullptr, nullptr, descs[i].H, descs[i].W, P, 0.f, 0});
    }
  if (!hs.empty()) {
    s.take<char>(of_hs_batch_workspace_size(hs.data(), (int)hs.size()));
    s.take<int>(hs.size());  // the persistent launch's status words
  }
  return s.off;
}

extern "C" int of_batch_run(const OfPairDesc* descs, int n, const OfTuning* tuning, int* status, void* workspace,
                            size_t workspace_bytes, void* stream) {
  OF_REQUIRE(descs && n > 0, "of_batch_run: empty batch");
  for (int i = 0; i < n; i++)
    if (validate(descs[i], i) != OF_OK) return OF_ERR_INVALID;
  const size_t need = of_batch_workspace_size(descs, n, tuning);
  if (!workspace || workspace_bytes < need)
    return set_error(OF_ERR_WORKSPACE, "of_batch_run: workspace too small (%zu < %zu)", workspace_bytes, need);
  cudaStream_t st = as_stream(stream);
  if (status) {
    cudaError_t e = cudaMemsetAsync(status, 0, sizeof(int) * (size_t)n, st);
    if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_batch_run: %s", cudaGetErrorString(e));
  }
  Carver c(workspace, workspace_bytes);
  std::vector<Deferred> defer;
  for (int i = 0; i < n; i++) {
    const size_t bytes = pair_arena(descs[i], i);
    char* base = c.take<char>(bytes);
    Arena A{false, base, bytes, 0};
    if (status && descs[i].frame_u8 == 0) {
      int rc = of_check_finite((const float*)descs[i].I0, descs[i].H, descs[i].W, descs[i].in_pitch, status + i,
                               OF_ST_NONFINITE_INPUT, stream);
      if (!rc)
        rc = of_check_finite((const float*)descs[i].I1, descs[i].H, descs[i].W, descs[i].in_pitch, status + i,
                             OF_ST_NONFINITE_INPUT, stream);
      if (rc) return rc;
    }
    int rc = run_pair(A, descs[i], i, status, &defer, st);
    if (rc != OF_OK) return rc;
  }
  if (!defer.empty()) {
    std::vector<OfHsBatchPair> hp;
    for (auto& q : defer) hp.push_back(q.p);
    const size_t wn = of_hs_batch_workspace_size(hp.data(), (int)hp.size());
    void* ws = c.take<char>(wn);
    // the persistent launch's status words (contiguous), ORed into the pairs' afterwards
    int* hs_status = c.take<int>(hp.size());
    if (!c.ok()) return set_error(OF_ERR_WORKSPACE, "of_batch_run: workspace too small");
    int* hst = status;
    cudaError_t e = cudaMemsetAsync(hs_status, 0, sizeof(int) * hp.size(), st);
    if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_batch_run: %s", cudaGetErrorString(e));
    OfTuning tun{};
    if (tuning) tun = *tuning;
    int rc = of_hs_batch(hp.data(), (int)hp.size(), &tun, hs_status, 1ll << 20, ws, wn, stream);
    if (rc != OF_OK) return rc;
    for (size_t k = 0; k < defer.size(); k++) {
      const Deferred& q = defer[k];
      const OfPairDesc& d = descs[q.pair];
      if ((rc = of_accumulate(q.Ua.p, q.U.p, q.U.H, q.U.W, q.Ua.pitch, stream)) ||
          (rc = of_accumulate(q.Va.p, q.V.p, q.V.H, q.V.W, q.Va.pitch, stream)))
        return rc;
      e = cudaMemcpy2DAsync(d.U, sizeof(float) * d.out_pitch, q.Ua.p, sizeof(float) * q.Ua.pitch,
                            sizeof(float) * d.W, d.H, cudaMemcpyDeviceToDevice, st);
      if (e == cudaSuccess)
        e = cudaMemcpy2DAsync(d.V, sizeof(float) * d.out_pitch, q.Va.p, sizeof(float) * q.Va.pitch,
                              sizeof(float) * d.W, d.H, cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) return set_error(OF_ERR_CUDA, "of_batch_run: %s", cudaGetErrorString(e));
      if (hst) {
        if ((rc = status_or(hs_status + k, hst + q.pair, st))) return rc;
        if ((rc = of_check_finite(d.U, d.H, d.W, d.out_pitch, hst + q.pair, OF_ST_NONFINITE_OUTPUT, stream)) ||
            (rc = of_check_finite(d.V, d.H, d.W, d.out_pitch, hst + q.pair, OF_ST_NONFINITE_OUTPUT, stream)))
          return rc;
      }
    }
  }
  return check_launch("of_batch_run", 0);
}
