// Host part of the DFT planner (plain C++, no CUDA calls): channel blocks, the
// quadratic log-frequency fits, channels per thread, tile shape and shared
// memory.  Compiled by the host compiler so that it can be tested on any CPU.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "dft_plan.h"

namespace obit {

bool valid_K(int K) { return K == 1 || K == 2 || K == 4 || K == 8 || K == 16 || K == 32; }

bool kernel_exists(int flavor, int K) {
  if (flavor == kFlavorRecur) return K == 2 || K == 4 || K == 8 || K == 16 || K == 32;
  if (flavor == kFlavorPlain) return K == 1 || K == 2 || K == 4 || K == 8 || K == 16;
  return false;
}

int comp_stride(const ModelDesc& m) { return (m.lcomp + 3) & ~3; }

namespace {

// Split a double into a float pair hi + lo with |lo| <= ulp(hi)/2.
void split_ds(double x, float* hi, float* lo) {
  *hi = (float)x;
  *lo = (float)(x - (double)*hi);
}

// Quadratic a0 + a1 k + a2 k^2 interpolating f on k in [0, n] at the three
// Chebyshev nodes x_i = n/2 (1 + cos((2i+1) pi/6)), which keeps the maximum
// interpolation error near the minimax value (|f'''| n^3 / 192).
template <class Fn>
void quad_fit(Fn f, double n, float out[3]) {
  if (n <= 0.0) {
    out[0] = (float)f(0.0);
    out[1] = out[2] = 0.f;
    return;
  }
  const double h = 0.5 * n, c = std::sqrt(3.0) / 2.0;
  const double x0 = h * (1.0 - c), x1 = h, x2 = h * (1.0 + c);
  const double y0 = f(x0), y1 = f(x1), y2 = f(x2);
  // Newton form y0 + d1 (k - x0) + d2 (k - x0)(k - x1), expanded in powers of k
  const double d1 = (y1 - y0) / (x1 - x0);
  const double d2 = ((y2 - y1) / (x2 - x1) - d1) / (x2 - x0);
  out[0] = (float)(y0 - d1 * x0 + d2 * x0 * x1);
  out[1] = (float)(d1 - d2 * (x0 + x1));
  out[2] = (float)d2;
}

}  // namespace

int plan_layout(const LayoutDesc& L, const ModelDesc& M, const ApplyDesc& A, const TuneDesc& T,
                Plan* plan, std::string* err) {
  *plan = Plan();
  plan->tune = T;
  plan->model = M;
  if (M.kind < kPoint || M.kind > kGaussTSpec) {
    *err = "unsupported model type " + std::to_string(M.kind);
    return 3;
  }
  if (M.nterm < 0 || M.nterm > kMaxNTerm) {
    *err = "nterm " + std::to_string(M.nterm) + " outside 0.." + std::to_string(kMaxNTerm);
    return 3;
  }
  if (T.K != 0 && !kernel_exists(T.flavor, T.K)) {
    *err = "no kernel for flavor " + std::to_string(T.flavor) + " K " + std::to_string(T.K);
    return 3;
  }
  if (T.ct < 0 || T.ct > 1024) {
    *err = "components per tile must be in 1..1024 (0: planner's choice)";
    return 3;
  }
  const int nfreq = L.nchan * L.nif;
  if ((int)L.fscale.size() < nfreq) {
    *err = "frequency table shorter than nchan*nif";
    return 3;
  }
  const bool tspec = (M.kind == kPointTSpec || M.kind == kGaussTSpec);
  const bool spec = (M.kind == kPointSpec || M.kind == kGaussSpec);
  if ((spec || tspec) && (int)L.lnspec.size() < nfreq) {
    *err = "spectral models need a log-frequency table";
    return 3;
  }
  if (tspec && (int)L.specIndex.size() < nfreq) {
    *err = "tabulated-spectrum models need a plane index table";
    return 3;
  }
  const int npol = L.stoke - L.stokb + 1;
  if (npol < 1 || npol > kMaxPol || L.stokb < 0 || L.stoke >= L.nstok) {
    *err = "polarization selection out of range";
    return 3;
  }
  if (L.chanb < 0 || L.chane >= L.nchan || L.chanb > L.chane || L.ifb < 0 || L.ife >= L.nif ||
      L.ifb > L.ife) {
    *err = "channel/IF selection out of range";
    return 3;
  }

  // ---- channel blocks --------------------------------------------------
  std::vector<double> dfs;
  auto df_class = [&](double d) -> int {
    for (size_t i = 0; i < dfs.size(); i++)
      // increments that differ only by the rounding of the FP64 frequency
      // table share a class (one step phasor per class and row-component):
      // 1e-12 of df changes a step by < 1e-9 turns at 3e6-turn phases
      if (std::fabs(dfs[i] - d) <= 1e-12 * std::fabs(d)) return (int)i;
    dfs.push_back(d);
    return (int)dfs.size() - 1;
  };
  int K = T.K;
  if (K == 0) {
    // Default channels per thread: 32 (two packed chains of 8 steps, for the
    // phasor and for a Gaussian taper alike), 16 when several spectral terms
    // need the tighter log-frequency fit of shorter blocks; never longer than
    // the selected channel run.  (On the 50,000-component Gaussian+spectrum
    // workload 32 channels per thread run 15 % faster than 16.)
    K = (T.flavor == kFlavorRecur) ? ((M.nterm > 1) ? 16 : 32) : 8;
    const int run = L.chane - L.chanb + 1;
    while (K > 2 && K / 2 >= run) K /= 2;
  }
  // Frequencies that do not advance uniformly within an IF cannot use long
  // recurrences: such plans use one-channel blocks and the shortest kernel.
  bool uniform = true;
  for (int iIF = L.ifb; iIF <= L.ife && uniform; iIF++) {
    const int i0 = L.chanb * L.kincf + iIF * L.kincif;
    if (L.chane <= L.chanb + 1) continue;
    const double f0 = L.fscale[i0], d = L.fscale[i0 + L.kincf] - f0;
    for (int ch = L.chanb + 2; ch <= L.chane; ch++) {
      const double f = L.fscale[ch * L.kincf + iIF * L.kincif];
      if (std::fabs(f - (f0 + (ch - L.chanb) * d)) > 1e-13 * std::fabs(f0)) {
        uniform = false;
        break;
      }
    }
  }
  if (!uniform) K = (T.flavor == kFlavorRecur) ? 2 : 1;
  for (int iIF = L.ifb; iIF <= L.ife; iIF++) {
    int ch = L.chanb;
    while (ch <= L.chane) {
      // run of channels sharing a plane (and a block key)
      int end = ch;
      const int plane = tspec ? L.specIndex[ch * L.kincf + iIF * L.kincif] : 0;
      const bool keyed = (int)L.blockKey.size() >= nfreq;
      const int key = keyed ? L.blockKey[ch * L.kincf + iIF * L.kincif] : 0;
      while (end + 1 <= L.chane &&
             (!tspec || L.specIndex[(end + 1) * L.kincf + iIF * L.kincif] == plane) &&
             (!keyed || L.blockKey[(end + 1) * L.kincf + iIF * L.kincif] == key))
        end++;
      for (int c0 = ch; c0 <= end; c0 += K) {
        int len = std::min(K, end - c0 + 1);
        const int ifq0 = c0 * L.kincf + iIF * L.kincif;
        const double f0 = L.fscale[ifq0];
        double df = 0.0;  // mean increment over the block
        if (len > 1) df = (L.fscale[ifq0 + (len - 1) * L.kincf] - f0) / (len - 1);
        // a block is usable only if its frequencies advance uniformly
        double dev = 0.0;
        for (int k = 2; k < len; k++)
          dev = std::max(dev, std::fabs(L.fscale[ifq0 + k * L.kincf] - (f0 + k * df)));
        plan->maxNonLin = std::max(plan->maxNonLin, dev);
        if (!uniform || dev > 1e-13 * std::fabs(f0)) {
          plan->linear = false;
          len = 1;  // fall back to one-channel blocks here
        }
        BlockDesc b{};
        split_ds(f0, &b.f0_hi, &b.f0_lo);
        b.df = (float)df;
        b.off0 = L.nrparm + iIF * L.incif + c0 * L.incf;
        b.len = len;
        b.dfc = (len > 1) ? df_class(df) : 0;
        b.plane = plane;
        b.ifq0 = ifq0;
        const int nt = tspec ? 1 : (spec ? M.nterm : 0);
        if (nt > 0) {
          // log ratio as a function of fractional channel x within the block
          const double Lr0 = L.lnspec[ifq0];
          // ln(f(x) * r) = ln(f(x)) + (Lr0 - ln f0)
          const double shift = Lr0 - std::log(f0);
          auto Lx = [&](double x) { return std::log(f0 + x * df) + shift; };
          const double n = (double)(len - 1);
          for (int t = 0; t < nt; t++) {
            auto P = [&](double x) { return std::pow(Lx(x), t + 1); };
            quad_fit(P, n, b.l[t]);
          }
        }
        plan->blocks.push_back(b);
        if (len < std::min(K, end - c0 + 1)) c0 += len - K;  // advance by len only
      }
      ch = end + 1;
    }
  }
  if (dfs.empty()) dfs.push_back(0.0);
  if ((int)dfs.size() > kMaxDf) {
    *err = "more than " + std::to_string(kMaxDf) + " distinct channel increments";
    return 3;
  }
  const int nblocks = (int)plan->blocks.size();

  // ---- tile shape --------------------------------------------------------
  KParams& kp = plan->kp;
  kp.lrec = L.lrec;
  kp.ilocu = L.ilocu;
  kp.ilocv = L.ilocv;
  kp.ilocw = L.ilocw;
  kp.incs = L.incs;
  kp.incf = L.incf;
  kp.pol0 = L.stokb;
  kp.npol = npol;
  kp.op = A.op;
  kp.flipMask = A.flipMask;
  kp.cumulative = A.cumulative;
  kp.stokFactor = A.stokFactor;
  for (int i = 0; i < kMaxPol; i++) kp.polFact[i] = A.polFact[i];
  kp.nblocks = nblocks;
  // Tile shape R x Bt = threads (128 or 256), R a power of two >= 8 (warp lanes
  // are rows): the fewest idle blocks, then the most blocks sharing each row's
  // phase work.
  auto pick_bt = [&](int threads) {
    int bestBt = 1;
    long best = 0;
    bool have = false;
    for (int bt = 1; bt <= kMaxBt && threads / bt >= 8; bt *= 2) {
      if (T.Bt > 0 && bt != T.Bt) continue;
      const long tiles = (nblocks + bt - 1) / bt;
      const long waste = tiles * bt - nblocks;
      const long score = waste * 64 - (bt <= 16 ? bt : 16);
      if (!have || score < best) {
        have = true;
        best = score;
        bestBt = bt;
      }
    }
    return bestBt;
  };
  int threads = (T.threads == 128) ? 128 : kThreads;
  kp.Bt = pick_bt(threads);
  // Rows with at most two channel blocks: a 256-thread tile would span 128 rows,
  // and its per-(row, component) shared arrays would cut the component tile;
  // two 128-thread CTAs per SM keep the tile and overlap each other's barriers.
  if (T.threads == 0 && T.flavor == kFlavorRecur && threads / kp.Bt >= 128) {
    threads = 128;
    kp.Bt = pick_bt(threads);
  }
  kp.R = threads / kp.Bt;
  plan->threads = threads;
  kp.nBlockTiles = (nblocks + kp.Bt - 1) / kp.Bt;
  kp.ndf = (int)dfs.size();
  for (int i = 0; i < kp.ndf; i++) split_ds(dfs[i], &kp.df_hi[i], &kp.df_lo[i]);
  kp.cstride = comp_stride(M);
  kp.waitPolls = kDefaultWaitPolls;
  kp.nterm = M.nterm;
  kp.nspec = M.nspec;
  const bool gauss = (M.kind == kGauss || M.kind == kGaussSpec || M.kind == kGaussTSpec);
  // spectral amplitude table: point families with a spectrum (Gaussian
  // families fold the spectrum into their per-row amplitude recurrence)
  const bool table = (M.kind == kPointSpec || M.kind == kPointTSpec);
  // spectral-factored form: point families with one spectral index whose
  // component order (M.specIndex) is known
  bool fspec = (T.flavor == kFlavorRecur) && T.specFactor && spec_factorable(M.kind, K) &&
               (M.kind == kPointTSpec || M.nterm == 1) && M.specIndex != nullptr && M.ncomp > 0;
  // mixed Gaussian models: the point sub-table in the spectral-factored form,
  // then the Gaussian components in the chain form (one launch)
  const int ptKind = (M.kind == kGaussTSpec) ? kPointTSpec : kPointSpec;
  bool mixed = (T.flavor == kFlavorRecur) && T.specFactor && M.ncompPt > 0 &&
               M.specIndex != nullptr && (M.kind == kGaussTSpec || (M.kind == kGaussSpec && M.nterm == 1)) &&
               spec_factorable(ptKind, K);
  if (M.ncompPt > 0 && !mixed) {  // e.g. short blocks (non-uniform frequencies)
    *err = "a table split into point and Gaussian parts needs the mixed recurrence";
    return 4;
  }
  const int nIndexed = mixed ? M.ncompPt : M.ncomp;
  // shrink the component tile until the CTAs that the register budget lets
  // share an SM also fit its shared memory (32-channel recurrences run one
  // 256-thread CTA per SM)
  const bool oneCta = (T.flavor == kFlavorRecur && K >= 32);
  // (one 256-thread or two 128-thread CTAs per SM: 228 KB of shared memory,
  // less 1 KB reserved per CTA)
  const size_t budget = oneCta ? (threads == 128 ? 110 * 1024 : 200 * 1024)
                               : (threads == 128 ? 52 * 1024 : 110 * 1024);
  auto need = [&](int c) {
    const bool factored = (T.flavor == kFlavorRecur) && (point_factored(M.kind, K) || fspec || mixed);
    size_t mainf = (T.flavor == kFlavorRecur)
                       ? smem_floats_main(kp.R, kp.Bt, K, c, kp.cstride, kp.ndf, gauss, table, factored,
                                          fspec || mixed)
                       : (size_t)c * kp.cstride + (size_t)((kp.R * 3 + 3) & ~3) + 4 * (size_t)c;
    return 4 * std::max(mainf + 4, smem_floats_stage(kp.R, kp.Bt, K));
  };
  auto fit_from = [&](int start) {
    int c = (start + 1) & ~1;  // even: the recurrence kernel takes components in pairs
    while (c > 8 && need(c) > budget) c /= 2;
    return c;
  };
  // candidate tiles, preferred first: a requested tile shrunk to fit, or the
  // planner's choice (160 components where shared memory holds them as they
  // are: 1 % faster than 128 at configs 2 and 4; else 128 shrunk to fit)
  auto candidates = [&]() {
    std::vector<int> c;
    if (T.ct > 0) {
      c.push_back(fit_from(T.ct));
    } else {
      if (need(160) <= budget) c.push_back(160);
      c.push_back(fit_from(128));
    }
    return c;
  };
  std::vector<int> cands = candidates();
  int ct = cands[0];
  if (fspec || mixed) {
    // residual bound: the kernel's tile reference index is the midpoint of the
    // tile's first and last index (as floats, as the kernel forms it)
    double quad = 0.0;  // max over blocks of |l2| n^2 / 8
    for (const BlockDesc& b : plan->blocks) {
      const double n = (double)(b.len - 1);
      quad = std::max(quad, std::fabs((double)b.l[0][2]) * n * n / 8.0);
    }
    auto bound_ok = [&](int tile) {
      double spread = 0.0;
      for (int c0 = 0; c0 < nIndexed; c0 += tile) {
        const int nc = std::min(tile, nIndexed - c0);
        const float at = 0.5f * (M.specIndex[c0] + M.specIndex[c0 + nc - 1]);
        for (int c = c0; c < c0 + nc; c++)
          spread = std::max(spread, std::fabs((double)M.specIndex[c] - (double)at));
      }
      return spread * quad <= kSpecResidualTol;
    };
    bool ok = false;
    for (int c : cands) {  // the first candidate tile whose index spread meets the bound
      if (bound_ok(c)) {
        ct = c;
        ok = true;
        break;
      }
    }
    if (!ok) {
      if (mixed) {  // the caller rebuilds the plan from the unsplit table
        *err = "point sub-table fails the spectral-factored residual bound";
        return 4;
      }
      fspec = false;
      ct = candidates()[0];
    }
  }
  plan->specFactored = fspec;
  plan->mixed = mixed;
  plan->model.specIndex = nullptr;  // valid during planning only
  kp.ct = ct;
  plan->smemBytes = need(ct);
  if (plan->smemBytes > 220 * 1024) {
    *err = "tile does not fit in shared memory";
    return 3;
  }

  plan->tune.K = K;
  return 0;
}

}  // namespace obit
