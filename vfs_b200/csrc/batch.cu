// Host schedule of the fused path: the reference's coarse-to-fine schedule
// (stereotgv.cu:389-515 / 256-387) for a batch of pairs, with one batched launch
// per step and pyramid level, and the reference's pointer swaps applied to every
// pair.  Pairs may differ in size and pyramid depth; a pair joins the schedule at
// its own coarsest level.
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "fused.cuh"
#include "stereo_tgv.cuh"

namespace vfs {

namespace {

template <class ArgsT>
void set_tiles(ArgsT& A, int k, int w, int h) {
  A.pr[k].tiles_x = tiles_x_of(w);
  A.pr[k].tile0 = A.ntiles;
  A.ntiles += tiles_of(w, h);
}

void set_iter_tiles(IterArgs& A, int k, int w, int h, int rows) {
  A.pr[k].tiles_x = iter_tiles_x_of(w);
  A.pr[k].tile0 = A.ntiles;
  A.ntiles += iter_tiles_of(w, h, rows);
}

}  // namespace

// level_variant[l]: tile variant of the iteration kernel at level l; -1 = time the
// variants on this level's data before its first iteration (only when can_tune) and
// store the fastest there.
// concurrency: one-pair solves running at the same time on other streams (the batch's
// concurrent mode); the tuner's cost of a variant is its time per iteration times the larger
// of the share of the GPU its launches occupy and 1 / concurrency, so that with several pairs
// in flight it weighs the GPU time a variant takes from the others, and alone its latency.
// part: 0 the whole solve; 1 the calibration warp, the pyramid and the levels above full
// resolution (ending with the upscale to it); 2 the full-resolution level alone.  Running part 1
// then part 2 enqueues exactly what part 0 does.
void fused_solve_direct(std::vector<StereoTgvImpl*>& pairs, bool masked, bool half, cudaStream_t st,
                        std::vector<int>& level_variant, bool can_tune, int concurrency, int part) {
  const int n = (int)pairs.size();
  if (n == 0) return;
  if (n > kMaxPairs) throw ArgError{"batch larger than " + std::to_string(kMaxPairs) + " pairs"};
  const SolverParams& P0 = pairs[0]->P;
  int maxL = 0;
  for (auto* s : pairs) {
    if (!s->initialized()) throw ArgError{"fused solve: pair not initialized"};
    if (s->P.nWarpIters != P0.nWarpIters || s->P.nSolverIters != P0.nSolverIters ||
        s->P.timestep_lambda != P0.timestep_lambda)
      throw ArgError{"fused solve: pairs of one batch need equal warp / iteration counts and timestep_lambda"};
    s->ensureFused();
    maxL = std::max(maxL, s->levels());
  }
  StereoTgvImpl* prof = pairs[0];
  // first level of each pair: its coarsest, or the level a warm start begins at
  std::vector<int> top(n);
  for (int k = 0; k < n; k++) top[k] = pairs[k]->topLevel();
  auto top_of = [&](const StereoTgvImpl* s) {
    for (int k = 0; k < n; k++)
      if (pairs[k] == s) return top[k];
    return s->levels() - 1;
  };
  // ---- calibration warp, state reset, image pyramid (stereotgv.cu:392-405) ---------
  if (part != 2) {
  for (int k = 0; k < n; k++) {
    StereoTgvImpl* s = pairs[k];
    launch_warp_image(s->tex1(s->pI1[0], 0), s->d_cv, s->d_i1calibrated, s->geomAt(0), st);
    std::swap(s->pI1[0], s->d_i1calibrated);
    s->startState(top[k], st);
  }
  for (int l = 1; l < maxL; l++) {
    DownArgs D{};
    int k = 0;
    for (auto* s : pairs) {
      if (l >= s->levels()) continue;
      DownPair& d = D.pr[k];
      d.texI0 = s->tex1(s->pI0[l - 1], l - 1);
      d.texI1 = s->tex1(s->pI1[l - 1], l - 1);
      d.I0 = s->pI0[l];
      d.I1 = s->pI1[l];
      d.w = s->pW[l];
      d.h = s->pH[l];
      d.s = s->pS[l];
      set_tiles(D, k, d.w, d.h);
      k++;
    }
    D.npairs = k;
    launch_downscale_batched(D, st);
  }
  }  // part != 2
  // ---- levels -------------------------------------------------------------------------
  for (int level = maxL - 1; level >= 0; level--) {
    if ((part == 1 && level == 0) || (part == 2 && level > 0)) continue;
    TraceRange trace(level_range_name(level));
    std::vector<StereoTgvImpl*> act;
    for (int k = 0; k < n; k++)
      if (level <= top[k]) act.push_back(pairs[k]);
    if (act.empty()) continue;
    const int na = (int)act.size();
    long long px_level = 0;
    for (auto* s : act) px_level += (long long)s->pW[level] * s->pH[level];
    {
      LevelArgs L{};
      for (int k = 0; k < na; k++) {
        StereoTgvImpl* s = act[k];
        LevelPair& d = L.pr[k];
        d.texI0 = s->tex1(s->pI0[level], level);
        d.texSmooth = s->tex1(s->d_i0smooth, level);
        d.mask = masked ? s->pMask[level] : nullptr;
        d.i0smooth = s->d_i0smooth;
        d.a = s->d_a;
        d.b = s->d_b;
        d.c = s->d_c;
        d.warpUV = s->d_warpUV;
        d.u = s->d_u;
        d.tv = s->pTvF[level];
        d.init_flow = level == top_of(s);
        d.w = s->pW[level];
        d.h = s->pH[level];
        d.s = s->pS[level];
        int xcov = ((d.h + s->blockWidth - 1) / s->blockWidth) * s->blockWidth;  // calcTensor.cu:81,227
        d.xmax = std::min(d.w, xcov);
        d.beta = s->P.beta;
        d.gamma = s->P.gamma;
        d.cuda_math = s->tensor_cuda_math;
        d.abce = half ? s->f_abce : nullptr;
        d.rv = half ? s->f_rv : nullptr;
        d.alpha0 = s->P.alpha0;
        d.alpha1 = s->P.alpha1;
        set_tiles(L, k, d.w, d.h);
      }
      L.npairs = na;
      launch_level_gaussian(L, st);
      launch_level_tensor(L, st);
    }
    // the per-warp prologue's arguments (the current v-bar buffer is the one the iterations
    // left current, so the same call serves a warp's start and the previous warp's epilogue)
    auto warp_start_args = [&]() {
      WarpStartArgs W{};
      for (int k = 0; k < na; k++) {
        StereoTgvImpl* s = act[k];
        WarpStartPair& d = W.pr[k];
        d.texI1 = s->tex1(s->pI1[level], level);
        d.texTv = s->tex2(s->pTvF[level], level);
        d.warpUV = s->d_warpUV;
        d.tv2 = s->d_tv2;
        d.i1warp = s->d_i1warp;
        d.p = s->f_p;
        d.q = s->f_q;
        d.v_ = half ? s->f_vh : (void*)s->d_v_;
        d.w = s->pW[level];
        d.h = s->pH[level];
        d.s = s->pS[level];
        set_tiles(W, k, d.w, d.h);
      }
      W.npairs = na;
      return W;
    };
    for (int warpIter = 0; warpIter < P0.nWarpIters; warpIter++) {
      prof->profBeginPx(kProfPrologue, px_level, 1, st);
      // later warps' prologues run in the previous warp's epilogue launch
      if (warpIter == 0) launch_warp_start(warp_start_args(), half, st);
      {
        DerivArgs Dv{};
        for (int k = 0; k < na; k++) {
          StereoTgvImpl* s = act[k];
          DerivPair& d = Dv.pr[k];
          d.texI0 = s->tex1(s->pI0[level], level);
          d.texI1w = half ? s->tex1h(s->d_i1warp, level) : s->tex1(s->d_i1warp, level);
          d.tv = s->pTvF[level];
          d.Iu = s->d_Iu;
          d.Iz = s->d_Iz;
          d.u = s->d_u;
          d.u_last = s->d_u_last;
          d.w = s->pW[level];
          d.h = s->pH[level];
          d.s = s->pS[level];
          set_tiles(Dv, k, d.w, d.h);
        }
        Dv.npairs = na;
        launch_derivatives_batched(Dv, st);
      }
      prof->profEnd(st);
      auto iter_args = [&](int variant, float sigma_, float tau_, float mu_, int write_tp) {
        IterArgs A{};
        A.sigma = sigma_;
        A.tau = tau_;
        A.mu = mu_;
        A.write_tp = write_tp;
        for (int k = 0; k < na; k++) {
          StereoTgvImpl* s = act[k];
          IterPair& d = A.pr[k];
          d.code = masked ? s->code_masked[level] : s->code_plain[level];
          d.u_ = s->d_u_;
          d.u = s->d_u;
          d.v_ = half ? s->f_vh : (const void*)s->d_v_;
          d.p = s->f_p;
          d.q = s->f_q;
          d.Tp = s->d_Tp;
          d.a = s->d_a;
          d.b = s->d_b;
          d.c = s->d_c;
          d.Iu = s->d_Iu;
          d.Iz = s->d_Iz;
          d.abce = half ? s->f_abce : nullptr;
          d.rv = half ? s->f_rv : nullptr;
          d.us = s->d_us;
          d.u_s = s->d_u_s;
          d.v_s = half ? s->f_vhs : (void*)s->d_v_s;
          d.w = s->pW[level];
          d.h = s->pH[level];
          d.s = s->pS[level];
          d.alpha0 = s->P.alpha0;
          d.alpha1 = s->P.alpha1;
          d.lambda = s->P.lambda;
          // updateDualVariables.cu:174-176, 217: uniform per launch, evaluated here in float
          A.sp[k] = s->P.alpha1 * sigma_ / 3.0f;
          A.sq[k] = s->P.alpha0 * sigma_ / 2.0f;
          set_iter_tiles(A, k, d.w, d.h, kIterVariantRows[variant]);
        }
        A.npairs = na;
        A.span_rows = 0;
        // the TMA variant has the 8-row tiles of variant 1, and its tile spans
        const int sv = variant == kIterTmaVariant ? 1 : iter_span_slot(variant);
        if (na == 1 && masked && sv >= 0) {
          const StereoTgvImpl* s = act[0];
          if (level < (int)s->span_lo[sv].size()) {
            const std::vector<uint16_t>& lo = s->span_lo[sv][level];
            const std::vector<uint16_t>& hi = s->span_hi[sv][level];
            if (!lo.empty() && (int)lo.size() <= kMaxSpanRows) {
              A.span_rows = (int)lo.size();
              A.span_max = 0;
              const std::vector<uint16_t>& ilo = s->inner_lo[sv][level];
              const std::vector<uint16_t>& ihi = s->inner_hi[sv][level];
              const bool have_inner = ilo.size() == lo.size() && ihi.size() == lo.size();
              for (size_t r = 0; r < lo.size(); r++) {
                A.span_lo[r] = lo[r];
                A.span_hi[r] = hi[r];
                A.in_lo[r] = have_inner ? ilo[r] : 1;
                A.in_hi[r] = have_inner ? ihi[r] : 0;
                if (hi[r] >= lo[r]) A.span_max = std::max(A.span_max, (int)hi[r] - (int)lo[r] + 1);
              }
            }
          }
        }
        return A;
      };
      // the K-iterations-per-launch kernel: one pair per launch, and exact at this level
      const bool tb_here = na == 1 && (!masked || (level < (int)act[0]->tb_ok.size() && act[0]->tb_ok[level]));
      const bool tma_here = na == 1 && (!masked || (level < (int)act[0]->tma_ok.size() && act[0]->tma_ok[level]));
      auto tb_args = [&](float sigma_, float tau_, int iter0, int k) {
        IterTBArgs T{};
        T.P = iter_args(kIterDefaultVariant, sigma_, tau_, 1.0f, 0).pr[0];
        for (int j = 0; j < k; j++) {
          float mu_;
          if (sigma_ < 1000.0f) mu_ = 1.0f / std::sqrt(1 + 0.7f * tau_ * P0.timestep_lambda);
          else mu_ = 1;
          T.sp[j] = act[0]->P.alpha1 * sigma_ / 3.0f;
          T.sq[j] = act[0]->P.alpha0 * sigma_ / 2.0f;
          T.tau[j] = tau_;
          T.mu[j] = mu_;
          sigma_ = sigma_ / mu_;
          tau_ = tau_ * mu_;
        }
        T.parity = iter0 & 1;
        T.write_tp = 0;
        return T;
      };
      // the cluster-resident kernel: the same schedule for k (up to kCLMaxIters) iterations
      auto cl_args = [&](int variant_, float sigma_, float tau_, int iter0, int k) {
        IterCLArgs C{};
        C.P = iter_args(kIterDefaultVariant, sigma_, tau_, 1.0f, 0).pr[0];
        for (int j = 0; j < k; j++) {
          float mu_;
          if (sigma_ < 1000.0f) mu_ = 1.0f / std::sqrt(1 + 0.7f * tau_ * P0.timestep_lambda);
          else mu_ = 1;
          C.sp[j] = act[0]->P.alpha1 * sigma_ / 3.0f;
          C.sq[j] = act[0]->P.alpha0 * sigma_ / 2.0f;
          C.tau[j] = tau_;
          C.mu[j] = mu_;
          sigma_ = sigma_ / mu_;
          tau_ = tau_ * mu_;
        }
        C.n = k;
        C.parity = iter0 & 1;
        C.write_tp = 0;
        C.rows = cluster_rows(variant_, C.P.h);
        C.ctas = cluster_ctas(variant_);
        return C;
      };
      const int lw = act[0]->pW[level], lh = act[0]->pH[level];
      if (level_variant[level] < 0) {
        if (can_tune && warpIter == 0 && P0.nSolverIters > 0) {
          // Time every tile variant on this level's data.  These launches read the same
          // inputs as the first iteration below and write only what it overwrites (the
          // other p / q plane, us, u_s, v_s at in-mask pixels; T p is left alone), so they
          // do not change any result.
          double best = 1e30;
          int best_v = kIterDefaultVariant;
          const double floor_share = 1.0 / (double)std::max(1, concurrency);
          float mu0 = 1.0f / std::sqrt(1 + 0.7f * 1.0f * P0.timestep_lambda);
          cudaEvent_t e0, e1;
          VFS_CUDA(cudaEventCreate(&e0));
          VFS_CUDA(cudaEventCreate(&e1));
          // two passes over the candidates, each keeping its faster pass, so that one
          // disturbed measurement (other pairs' work on the GPU) does not decide the level
          std::vector<float> best_ms(kIterVariants, 1e30f);
          for (int pass = 0; pass < 2; pass++)
          for (int v = 0; v < kIterVariants; v++) {
            if (!iter_variant_valid(v)) continue;
            const int kv = tb_iterations(v);
            if (kv > 1 && (!tb_here || kv > P0.nSolverIters)) continue;
            // Several iterations per launch recompute the tile halos, which pays only for a pair
            // alone: in the 8-pair 848x800 batch they cost 6-12 % of the step at 212 x 200.
            if (kv > 1 && concurrency > 1) continue;
            // Nor do the other tile heights of the one-iteration kernel: in the 8-pair batch none
            // beat variant 1 by more than the run-to-run spread at any level (15 rows: 0-2 %
            // slower at 848 x 800; 16 rows: 5 % slower; 4 rows: equal at 212 x 200), while the
            // tuner's timings amid the other pairs' work picked them by mistake (a 2 % loss).
            if (concurrency > 1 && iter_variant_tiled(v) && v != kIterDefaultVariant) continue;
            if (iter_variant_single_pair(v) && na != 1) continue;
            // The TMA-staged kernel has no interior-warp path and is slower than variant 1;
            // per-launch timings amid other pairs' work still picked it at 424 x 400, where it
            // cost 2 % of the 8-pair step.  It runs when forced.
            if (v == kIterTmaVariant) continue;
            const bool clv = iter_variant_cluster(v);
            if (clv && (!tb_here || !cluster_fits(v, masked, half, lw, lh))) continue;
            // With other pairs in flight, a cluster whose threads each hold several pixels takes
            // that many times longer per iteration while it holds a whole cluster of SMs: on
            // B200 the 8-pair 848x800 batch ran 4.5 % slower with it at 212 x 200 (3 pixels per
            // thread) than with one-iteration launches there, which per-launch timings taken
            // amid the other pairs' work did not show.  It stays a candidate for a pair alone.
            if (clv && concurrency > 1 && cluster_pixels_per_thread(v, half, lw, lh) > 1) continue;
            // the cluster-resident kernel is timed over an odd number of iterations, so that it
            // writes the other ping-pong buffers, which the first iteration below overwrites
            const int kc = clv ? ((std::min(P0.nSolverIters, kCLMaxIters) - 1) | 1) : 1;
            IterArgs T = iter_args((kv > 1 || clv) ? kIterDefaultVariant : v, 1.0f, 1.0f, mu0, 0);
            IterTBArgs TB = tb_args(1.0f, 1.0f, 0, kv);
            IterCLArgs CL{};
            if (clv) CL = cl_args(v, 1.0f, 1.0f, 0, kc);
            auto once = [&] {
              if (clv) launch_fused_iteration_cluster(CL, masked, half, st, v);
              else if (kv > 1) launch_fused_iteration_tb(TB, masked, half, st, v);
              else if (v == kIterTmaVariant) launch_fused_iteration_tma(T, masked, half, st, 0);
              else launch_fused_iteration(T, masked, half, st, 0, v);
            };
            once();  // warm the caches / the instruction path
            VFS_CUDA(cudaEventRecord(e0, st));
            for (int r = 0; r < 3; r++) once();
            VFS_CUDA(cudaEventRecord(e1, st));
            VFS_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            VFS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            ms /= (float)(clv ? kc : kv);  // per iteration
            best_ms[v] = std::min(best_ms[v], ms);
            if (pass == 0) continue;
            ms = best_ms[v];
            double share = 1.0;
            if (na == 1) share = iteration_gpu_share(v, masked, half, lw, lh);
            double cost = (double)ms * std::max(share, floor_share);
            // the default keeps its place unless another variant is clearly (5 %) cheaper
            if (v == kIterDefaultVariant) cost *= 0.95;
            if (cost < best) {
              best = cost;
              best_v = v;
            }
          }
          cudaEventDestroy(e0);
          cudaEventDestroy(e1);
          level_variant[level] = best_v;
        } else if (!can_tune) {
          level_variant[level] = kIterDefaultVariant;
        }
      }
      const int variant = level_variant[level] < 0 ? kIterDefaultVariant : level_variant[level];
      // K iterations per launch where the variant is a multi-iteration one and it applies
      // here; the remaining iterations (and the fallback) use the default one-iteration form
      // (the cluster-resident kernel: all iterations, in launches of up to kCLMaxIters)
      const bool cl_here = tb_here && iter_variant_cluster(variant) && cluster_fits(variant, masked, half, lw, lh);
      const int K = cl_here ? kCLMaxIters : tb_here ? tb_iterations(variant) : 1;
      const int v1 = (tb_iterations(variant) > 1 || iter_variant_cluster(variant) ||
                      (iter_variant_single_pair(variant) && na != 1) ||
                      (variant == kIterTmaVariant && !tma_here))
                         ? kIterDefaultVariant
                         : variant;
      float tau = 1.0f;
      float sigma = 1.0f / tau;
      const int n_it = P0.nSolverIters;
      prof->profBeginPx(kProfFused, px_level, n_it, st,
                        cl_here ? (n_it + K - 1) / K : K > 1 ? n_it / K + n_it % K : n_it);
      for (int iter = 0; iter < n_it;) {
        const int k = cl_here ? std::min(K, n_it - iter) : (K > 1 && iter + K <= n_it) ? K : 1;
        if (cl_here) {
          IterCLArgs C = cl_args(variant, sigma, tau, iter, k);
          C.write_tp = iter + k == n_it;
          launch_fused_iteration_cluster(C, masked, half, st, variant);
          for (int j = 0; j < k; j++) {
            sigma = sigma / C.mu[j];
            tau = tau * C.mu[j];
          }
        } else if (k > 1) {
          IterTBArgs T = tb_args(sigma, tau, iter, k);
          T.write_tp = iter + k == n_it;
          launch_fused_iteration_tb(T, masked, half, st, variant);
          for (int j = 0; j < k; j++) {
            sigma = sigma / T.mu[j];
            tau = tau * T.mu[j];
          }
        } else {
          float mu;
          if (sigma < 1000.0f) mu = 1.0f / std::sqrt(1 + 0.7f * tau * P0.timestep_lambda);
          else mu = 1;
          IterArgs A = iter_args(v1, sigma, tau, mu, iter == n_it - 1);
          if (v1 == kIterTmaVariant) launch_fused_iteration_tma(A, masked, half, st, iter & 1);
          else launch_fused_iteration(A, masked, half, st, iter & 1, v1);
          sigma = sigma / mu;
          tau = tau * mu;
        }
        for (int it = iter; it < iter + k; it++) {
          for (auto* s : act) {
            std::swap(s->d_u, s->d_us);
            std::swap(s->d_u_, s->d_u_s);
            if (half) std::swap(s->f_vh, s->f_vhs);
            else std::swap(s->d_v_, s->d_v_s);
            s->f_parity = (it & 1) ? 0 : 1;
          }
        }
        iter += k;
      }
      prof->profEnd(st);
      prof->profBeginPx(kProfEpilogue, px_level, 1, st);
      {
        EpiArgs E{};
        E.median = masked ? 1 : 0;
        for (int k = 0; k < na; k++) {
          StereoTgvImpl* s = act[k];
          EpiPair& d = E.pr[k];
          d.u_in = s->d_u;
          d.u_out = masked ? s->d_us : s->d_u;
          d.u_bar = s->d_u_;
          d.u_last = s->d_u_last;
          d.tv2 = s->d_tv2;
          d.warpUV = s->d_warpUV;
          d.w = s->pW[level];
          d.h = s->pH[level];
          d.s = s->pS[level];
          d.limitRange = s->P.limitRange;
          set_tiles(E, k, d.w, d.h);
        }
        E.npairs = na;
        if (warpIter + 1 < P0.nWarpIters) launch_epilogue_warp_start(E, warp_start_args(), half, st);
        else launch_warp_epilogue_batched(E, st);
        if (masked)
          for (auto* s : act) std::swap(s->d_u, s->d_us);
      }
      prof->profEnd(st);
    }
    if (level > 0) {
      UpArgs U{};
      int k = 0;
      std::vector<StereoTgvImpl*> up;
      for (auto* s : act) {
        UpPair& d = U.pr[k];
        d.texU = s->tex1(s->d_u, level);
        d.texUbar = s->tex1(s->d_u_, level);
        d.texWarp = s->tex2(s->d_warpUV, level);
        d.u_out = s->d_us;
        d.ubar_out = s->d_u_s;
        d.warp_out = s->d_warpUVs;
        d.w = s->pW[level - 1];
        d.h = s->pH[level - 1];
        d.s = s->pS[level - 1];
        d.scale = s->P.fScale;
        set_tiles(U, k, d.w, d.h);
        k++;
      }
      U.npairs = k;
      launch_upscale_batched(U, st);
      for (auto* s : act) {
        std::swap(s->d_u, s->d_us);
        std::swap(s->d_u_, s->d_u_s);
        std::swap(s->d_warpUV, s->d_warpUVs);
      }
    }
  }
}

// ---- CUDA graph of a whole batched solve ---------------------------------------------
// The launch sequence of a solve depends only on the batch composition and on which
// physical buffer currently plays each ping-pong role, so a captured graph is reused
// whenever the pairs are in the same pointer state; the state after the graph is
// recorded at capture and applied after each replay.
PairPtrs get_ptrs(StereoTgvImpl* s) {
  return PairPtrs{s->pI1[0], s->d_i1calibrated, s->d_u, s->d_us, s->d_u_, s->d_u_s,
                  s->d_v_, s->d_v_s, s->d_warpUV, s->d_warpUVs, s->f_vh, s->f_vhs};
}
void set_ptrs(StereoTgvImpl* s, const PairPtrs& p) {
  s->pI1[0] = p.pI1_0;
  s->d_i1calibrated = p.i1cal;
  s->d_u = p.u;
  s->d_us = p.us;
  s->d_u_ = p.u_;
  s->d_u_s = p.u_s;
  s->d_v_ = p.v_;
  s->d_v_s = p.v_s;
  s->d_warpUV = p.warpUV;
  s->d_warpUVs = p.warpUVs;
  s->f_vh = p.vh;
  s->f_vhs = p.vhs;
}

// Tuned choices shared by every engine of the process, keyed like FusedEngine::tuned_.
std::map<std::vector<int>, std::vector<int>>& shared_tuned() {
  static std::map<std::vector<int>, std::vector<int>> m;
  return m;
}
// Tuned choices of one-pair solves per level: form, storage, alone or with other pairs in
// flight, and the level's width and height.  A one-pair engine (each pair of a concurrent
// batch, each request of the server) takes a level's choice from here when that level was
// tuned before in the same setting, whatever the rest of the batch, so a new batch
// composition does not stop the stream to time every variant again.
std::map<std::array<int, 5>, int>& shared_level_tuned() {
  static std::map<std::array<int, 5>, int> m;
  return m;
}
std::atomic<long long>& tuning_solves() {
  static std::atomic<long long> n{0};
  return n;
}
long long tuning_solve_count() { return tuning_solves().load(std::memory_order_relaxed); }
std::mutex& shared_tuned_mutex() {
  static std::mutex m;
  return m;
}

FusedEngine::~FusedEngine() { clear(); }

void FusedEngine::note_variants(const std::vector<int>& v, int part) {
  if (part == 0) {
    last_variants = v;
    return;
  }
  last_variants.resize(v.size(), -1);
  for (size_t l = 0; l < v.size(); l++)
    if ((part == 1 && l > 0) || (part == 2 && l == 0)) last_variants[l] = v[l];
}

void FusedEngine::clear() {
  for (auto& kv : cache_) {
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    for (auto e : kv.second.events) cudaEventDestroy(e);
  }
  cache_.clear();
}

// An executable still in flight is freed when it completes (cudaGraphExecDestroy), and so are
// recorded events (cudaEventDestroy).
void FusedEngine::drop(std::map<std::vector<uintptr_t>, Entry>::iterator it) {
  if (it->second.exec) cudaGraphExecDestroy(it->second.exec);
  for (auto e : it->second.events) cudaEventDestroy(e);
  cache_.erase(it);
}

void FusedEngine::evict(const std::vector<StereoTgvImpl*>& pairs) {
  for (auto it = cache_.begin(); it != cache_.end();) {
    bool stale = false;
    for (const auto& o : it->second.owners)
      for (const auto* s : pairs)
        if (o.first == s && o.second != s->generation) stale = true;
    if (stale) {
      auto next = std::next(it);
      drop(it);
      it = next;
    } else {
      ++it;
    }
  }
  while (cache_.size() >= kMaxGraphs) {
    auto lru = cache_.begin();
    for (auto it = cache_.begin(); it != cache_.end(); ++it)
      if (it->second.last_use < lru->second.last_use) lru = it;
    drop(lru);
  }
}

void FusedEngine::prepare(std::vector<StereoTgvImpl*>& pairs, bool masked) {
  for (auto* s : pairs) {
    if (!s->initialized()) throw ArgError{"fused solve: pair not initialized"};
    s->ensureFused();
    if (masked && !s->codes_valid) {
      for (int l = 0; l < s->levels(); l++)
        launch_edge_codes(s->pMask[l], s->code_masked[l], s->pW[l], s->pH[l], s->pS[l], s->stream());
      // a level without row padding reads the previous row's last pixel west of column 0;
      // the multi-iteration kernel cannot follow that pixel, so it is used there only when
      // no pixel of column 0 is on
      s->tb_ok.assign(s->levels(), 1);
      s->tma_ok.assign(s->levels(), 1);
      for (int v = 0; v < kIterSpanSlots; v++) {
        s->span_lo[v].assign(s->levels(), {});
        s->span_hi[v].assign(s->levels(), {});
        s->inner_lo[v].assign(s->levels(), {});
        s->inner_hi[v].assign(s->levels(), {});
      }
      for (int l = 0; l < s->levels(); l++) {
        const int w = s->pW[l], h = s->pH[l];
        std::vector<uint8_t> code((size_t)w * h);
        VFS_CUDA(cudaMemcpy2DAsync(code.data(), w, s->code_masked[l], s->pS[l], w, h, cudaMemcpyDeviceToHost,
                                   s->stream()));
        VFS_CUDA(cudaStreamSynchronize(s->stream()));
        for (int y = 0; y < h; y++)
          if (code[(size_t)y * w] & kOn) {
            s->tma_ok[l] = 0;
            if (w == s->pS[l]) s->tb_ok[l] = 0;
          }
        // first and last on column of every image row
        std::vector<int> xmin(h, w), xmax(h, -1);
        for (int y = 0; y < h; y++)
          for (int x = 0; x < w; x++)
            if (code[(size_t)y * w + x] & kOn) {
              xmin[y] = std::min(xmin[y], x);
              xmax[y] = std::max(xmax[y], x);
            }
        const int tiles_x = iter_tiles_x_of(w);
        // per row, the number of pixels left of x that are not interior (edge code 0x1F: on,
        // with the four neighbours in the image and on)
        const uint8_t kInterior = kOn | kR | kL | kD | kU;
        std::vector<int> notin((size_t)h * (w + 1), 0);
        for (int y = 0; y < h; y++)
          for (int x = 0; x < w; x++)
            notin[(size_t)y * (w + 1) + x + 1] = notin[(size_t)y * (w + 1) + x] + (code[(size_t)y * w + x] != kInterior);
        for (int v = 0; v < kIterVariants; v++) {
          const int slot = iter_span_slot(v);
          if (slot < 0 || !iter_variant_tiled(v)) continue;
          const int TH = kIterVariantRows[v];
          const int rows = (h + TH - 1) / TH;
          std::vector<uint16_t> lo(rows), hi(rows);
          for (int r = 0; r < rows; r++) {
            // tile row r covers image rows TH r - 1 (north halo) .. TH r + TH - 1; a column x
            // lies in tile x / 31 and, when x % 31 == 30, in the west halo of the next tile
            int a = w, b = -1;
            for (int y = std::max(0, TH * r - 1); y <= std::min(h - 1, TH * r + TH - 1); y++) {
              a = std::min(a, xmin[y]);
              b = std::max(b, xmax[y]);
            }
            if (b < 0) {
              lo[r] = 1;
              hi[r] = 0;
              continue;
            }
            lo[r] = (uint16_t)(a / 31);
            hi[r] = (uint16_t)std::min(tiles_x - 1, b / 31 + (b % 31 == 30 ? 1 : 0));
          }
          s->span_lo[slot][l] = lo;
          s->span_hi[slot][l] = hi;
          // the longest run of tiles whose region (rows TH r - 1 .. TH r + TH - 1, columns
          // 31 tx - 1 .. 31 tx + 30) lies in the image and holds interior pixels only
          std::vector<uint16_t> ilo(rows, 1), ihi(rows, 0);
          for (int r = 0; r < rows; r++) {
            const int y_lo = TH * r - 1, y_hi = TH * r + TH - 1;
            if (y_lo < 0 || y_hi >= h) continue;
            int run0 = -1, best_len = 0;
            for (int tx = 0; tx <= tiles_x; tx++) {
              bool ok = false;
              const int x_lo = 31 * tx - 1, x_hi = 31 * tx + 30;
              if (tx < tiles_x && x_lo >= 0 && x_hi < w) {
                ok = true;
                for (int y = y_lo; ok && y <= y_hi; y++)
                  ok = notin[(size_t)y * (w + 1) + x_hi + 1] == notin[(size_t)y * (w + 1) + x_lo];
              }
              if (ok && run0 < 0) run0 = tx;
              if (!ok && run0 >= 0) {
                if (tx - run0 > best_len) {
                  best_len = tx - run0;
                  ilo[r] = (uint16_t)run0;
                  ihi[r] = (uint16_t)(tx - 1);
                }
                run0 = -1;
              }
            }
          }
          s->inner_lo[slot][l] = ilo;
          s->inner_hi[slot][l] = ihi;
        }
      }
      s->codes_valid = true;
      s->generation = next_generation();  // graphs captured under the old mask are not reused
    }
  }
}

void FusedEngine::solve(std::vector<StereoTgvImpl*>& pairs, bool masked, bool half, cudaStream_t st, int part) {
  solve_parts(pairs, masked, half, st, part);
  for (auto* s : pairs) s->i1warp_half = half;
  if (part != 1)
    for (auto* s : pairs) s->have_prev = true;  // the frame's disparity is in d_u (warm starts)
}

void FusedEngine::solve_parts(std::vector<StereoTgvImpl*>& pairs, bool masked, bool half, cudaStream_t st,
                              int part) {
  if (pairs.empty()) return;
  prepare(pairs, masked);
  // tile variants per level for this batch composition (tuned on its first solve)
  // key: form, storage and the multiset of pair geometries (order does not change the work)
  std::vector<std::array<int, 3>> geo;
  int maxL = 0;
  for (auto* s : pairs) {
    geo.push_back({s->width, s->height, s->levels()});
    maxL = std::max(maxL, s->levels());
  }
  std::sort(geo.begin(), geo.end());
  std::vector<int> comp{(int)masked, (int)half, concurrency};
  for (auto& g : geo) comp.insert(comp.end(), g.begin(), g.end());
  auto tit = tuned_.find(comp);
  const bool forced = forced_variant >= 0 || !forced_levels.empty();
  if (tit == tuned_.end())
    tit = tuned_.emplace(comp, std::vector<int>(maxL, (autotune && !forced) ? -1 : kIterDefaultVariant)).first;
  // levels a warm start skips are not run (and not tuned) in this solve
  int max_top = 0;
  for (auto* s : pairs) max_top = std::max(max_top, s->topLevel());
  auto in_part = [&](int l) { return !((part == 1 && l == 0) || (part == 2 && l > 0)) && l <= max_top; };
  bool need_tune = false;
  const bool one_pair = pairs.size() == 1;
  auto level_key = [&](int l) {
    return std::array<int, 5>{(int)masked, (int)half, concurrency > 1 ? 2 : 1, pairs[0]->pW[l], pairs[0]->pH[l]};
  };
  if (autotune && !forced) {
    // a composition tuned before (by any engine of the process) is reused, so that every
    // pair of a batch runs the same choice and only the first tunes; a one-pair solve also
    // reuses any level tuned before in the same setting
    std::lock_guard<std::mutex> lk(shared_tuned_mutex());
    auto& shared = shared_tuned();
    auto sit = shared.find(comp);
    for (int l = 0; l < maxL; l++) {
      if (!in_part(l) || tit->second[l] >= 0) continue;
      if (sit != shared.end() && l < (int)sit->second.size() && sit->second[l] >= 0) {
        tit->second[l] = sit->second[l];
        continue;
      }
      if (one_pair && l < pairs[0]->levels()) {
        // the same setting first; else the choice made for this level size in the other
        // setting (alone / with other pairs in flight), so that a level size is timed once
        // and a server never stops a stream for a setting it has not met before
        auto key = level_key(l);
        auto lit = shared_level_tuned().find(key);
        if (lit == shared_level_tuned().end()) {
          key[2] = key[2] == 1 ? 2 : 1;
          lit = shared_level_tuned().find(key);
        }
        if (lit != shared_level_tuned().end()) {
          tit->second[l] = lit->second;
          continue;
        }
      }
      need_tune = true;
    }
  }
  if (need_tune) {
    // first solve of this composition (and part): run it directly and tune while it runs
    tuning_solves().fetch_add(1, std::memory_order_relaxed);
    std::vector<int> lv = tit->second;
    fused_solve_direct(pairs, masked, half, st, lv, true, concurrency, part);
    tit->second = lv;
    {
      std::lock_guard<std::mutex> lk(shared_tuned_mutex());
      std::vector<int>& sv = shared_tuned()[comp];
      sv.resize(maxL, -1);
      for (int l = 0; l < maxL; l++)
        if (in_part(l) && lv[l] >= 0) {
          sv[l] = lv[l];
          if (one_pair && l < pairs[0]->levels()) shared_level_tuned().emplace(level_key(l), lv[l]);
        }
    }
    note_variants(lv, part);
    return;
  }
  std::vector<int> variants = tit->second;
  if (forced_variant >= 0) variants.assign(maxL, forced_variant);
  if (!forced_levels.empty()) {
    variants.assign(maxL, kIterDefaultVariant);
    for (int l = 0; l < maxL && l < (int)forced_levels.size(); l++) variants[l] = forced_levels[l];
  }
  note_variants(variants, part);
  if (!use_graph) {
    fused_solve_direct(pairs, masked, half, st, variants, false, concurrency, part);
    return;
  }
  StereoTgvImpl* prof = pairs[0];
  std::vector<uintptr_t> key{(uintptr_t)masked, (uintptr_t)half, (uintptr_t)prof->profiling, (uintptr_t)part,
                             (uintptr_t)(intptr_t)launch_priority()};
  for (int v : variants) key.push_back((uintptr_t)v);
  std::vector<PairPtrs> before;
  for (auto* s : pairs) {
    PairPtrs p = get_ptrs(s);
    before.push_back(p);
    const uintptr_t* w = reinterpret_cast<const uintptr_t*>(&p);
    key.push_back((uintptr_t)s);
    key.push_back((uintptr_t)s->generation);
    key.push_back((uintptr_t)s->topLevel());
    key.push_back((uintptr_t)s->warmStart());  // a warm start from the coarsest level has the cold top
    key.insert(key.end(), w, w + sizeof(PairPtrs) / sizeof(uintptr_t));
    uint32_t lr;
    std::memcpy(&lr, &s->P.limitRange, 4);
    key.push_back(lr);
  }
  auto it = cache_.find(key);
  if (it == cache_.end()) {
    evict(pairs);
    Entry e;
    for (auto* s : pairs) e.owners.emplace_back(s, s->generation);
    std::vector<ProfRec> saved = prof->profRecords();
    prof->profReset();
    prof->capture_events = &e.events;
    cudaGraph_t g = nullptr;
    long long launches0 = launch_counter().load();
    VFS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
    try {
      fused_solve_direct(pairs, masked, half, st, variants, false, concurrency, part);
    } catch (...) {
      prof->capture_events = nullptr;
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(st, &junk);
      if (junk) cudaGraphDestroy(junk);
      for (auto ev : e.events) cudaEventDestroy(ev);
      for (size_t k = 0; k < pairs.size(); k++) set_ptrs(pairs[k], before[k]);
      throw;
    }
    prof->capture_events = nullptr;
    e.kernels = launch_counter().load() - launches0;
    launch_counter().fetch_sub(e.kernels);  // captured, not launched: counted when replayed
    VFS_CUDA(cudaStreamEndCapture(st, &g));
    cudaError_t ie = cudaGraphInstantiate(&e.exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) throw CudaError{ie, "cudaGraphInstantiate", __FILE__, __LINE__};
    for (auto* s : pairs) e.after.push_back(get_ptrs(s));
    e.prof = prof->profRecords();
    prof->setProfRecords(saved);
    for (size_t k = 0; k < pairs.size(); k++) set_ptrs(pairs[k], before[k]);
    it = cache_.emplace(key, std::move(e)).first;
  }
  it->second.last_use = ++use_clock_;
  VFS_CUDA(cudaGraphLaunch(it->second.exec, st));
  launch_counter().fetch_add(it->second.kernels);
  for (size_t k = 0; k < pairs.size(); k++) set_ptrs(pairs[k], it->second.after[k]);
  if (prof->profiling) {
    // the full-resolution part continues the frame whose coarse part ran just before
    std::vector<ProfRec> recs = part == 2 ? prof->profRecords() : std::vector<ProfRec>{};
    recs.insert(recs.end(), it->second.prof.begin(), it->second.prof.end());
    prof->setProfRecords(recs);
  }
}

}  // namespace vfs
