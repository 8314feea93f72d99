// Planner and launcher for the DFT kernels (see dft_kernels.cuh).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "dft_plan.h"

namespace obit {

bool valid_K(int K) { return K == 1 || K == 2 || K == 4 || K == 8 || K == 16 || K == 32; }

int comp_stride(const ModelDesc& m) { return (m.lcomp + 3) & ~3; }

namespace {

using KernelFn = void (*)(const KParams);

template <int K>
KernelFn pick_recur(int mode) {
  switch (mode) {
    case kPoint: return dft_recur_kernel<K, kPoint>;
    case kPointSpec: return dft_recur_kernel<K, kPointSpec>;
    case kPointTSpec: return dft_recur_kernel<K, kPointTSpec>;
    case kGauss: return dft_recur_kernel<K, kGauss>;
    case kGaussSpec: return dft_recur_kernel<K, kGaussSpec>;
    case kGaussTSpec: return dft_recur_kernel<K, kGaussTSpec>;
  }
  return nullptr;
}

template <int K>
KernelFn pick_plain(int mode) {
  switch (mode) {
    case kPoint: return dft_plain_kernel<K, kPoint>;
    case kPointSpec: return dft_plain_kernel<K, kPointSpec>;
    case kPointTSpec: return dft_plain_kernel<K, kPointTSpec>;
    case kGauss: return dft_plain_kernel<K, kGauss>;
    case kGaussSpec: return dft_plain_kernel<K, kGaussSpec>;
    case kGaussTSpec: return dft_plain_kernel<K, kGaussTSpec>;
  }
  return nullptr;
}

KernelFn pick_kernel(int flavor, int K, int mode) {
  if (flavor == kFlavorRecur) {
    switch (K) {
      case 2: return pick_recur<2>(mode);
      case 4: return pick_recur<4>(mode);
      case 8: return pick_recur<8>(mode);
      case 16: return pick_recur<16>(mode);
      case 32: return pick_recur<32>(mode);
    }
  } else if (flavor == kFlavorPlain) {
    switch (K) {
      case 1: return pick_plain<1>(mode);
      case 2: return pick_plain<2>(mode);
      case 4: return pick_plain<4>(mode);
      case 8: return pick_plain<8>(mode);
      case 16: return pick_plain<16>(mode);
    }
  }
  return nullptr;
}

// Split a double into a float pair hi + lo with |lo| <= ulp(hi)/2.
void split_ds(double x, float* hi, float* lo) {
  *hi = (float)x;
  *lo = (float)(x - (double)*hi);
}

// Quadratic a0 + a1 k + a2 k^2 through (0, y0), (m, ym), (n, yn) with m = n/2.
void quad_fit(double y0, double ym, double yn, double n, float out[3]) {
  if (n <= 0.0) {
    out[0] = (float)y0;
    out[1] = out[2] = 0.f;
    return;
  }
  const double m = 0.5 * n;
  // Newton form: y0 + d1 k + d2 k (k - m)
  const double d1 = (ym - y0) / m;
  const double d12 = (yn - ym) / (n - m);
  const double d2 = (d12 - d1) / n;
  out[0] = (float)y0;
  out[1] = (float)(d1 - d2 * m);
  out[2] = (float)d2;
}

}  // namespace

int build_plan(const LayoutDesc& L, const ModelDesc& M, const ApplyDesc& A, const TuneDesc& T,
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
  if (T.K != 0 && (!valid_K(T.K) || !pick_kernel(T.flavor, T.K, M.kind))) {
    *err = "no kernel for flavor " + std::to_string(T.flavor) + " K " + std::to_string(T.K);
    return 3;
  }
  if (T.ct < 1 || T.ct > 1024) {
    *err = "components per tile must be in 1..1024";
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
      if (std::fabs(dfs[i] - d) <= 1e-15 * std::fabs(d)) return (int)i;
    dfs.push_back(d);
    return (int)dfs.size() - 1;
  };
  int K = T.K;
  if (K == 0) {
    // Default channels per thread: 32 (two packed chains of 8 steps) for
    // constant or tabulated amplitudes, 16 when a per-row Gaussian taper adds
    // registers; never longer than the selected channel run.
    const bool g = (M.kind == kGauss || M.kind == kGaussSpec || M.kind == kGaussTSpec);
    K = (T.flavor == kFlavorRecur) ? (g ? 16 : 32) : 8;
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
      // run of channels sharing a plane
      int end = ch;
      const int plane = tspec ? L.specIndex[ch * L.kincf + iIF * L.kincif] : 0;
      while (end + 1 <= L.chane &&
             (!tspec || L.specIndex[(end + 1) * L.kincf + iIF * L.kincif] == plane))
        end++;
      for (int c0 = ch; c0 <= end; c0 += K) {
        int len = std::min(K, end - c0 + 1);
        const int ifq0 = c0 * L.kincf + iIF * L.kincif;
        const double f0 = L.fscale[ifq0];
        double df = 0.0;
        if (len > 1) df = L.fscale[ifq0 + L.kincf] - f0;
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
            quad_fit(P(0.0), P(0.5 * n), P(n), n, b.l[t]);
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
  const int threads = (T.threads == 128) ? 128 : kThreads;
  {
    int bestBt = 1;
    long best = -1;
    for (int bt = 1; bt <= kMaxBt && threads / bt >= 8; bt *= 2) {
      if (T.Bt > 0 && bt != T.Bt) continue;
      const long tiles = (nblocks + bt - 1) / bt;
      const long waste = tiles * bt - nblocks;
      const long score = waste * 64 - (bt <= 16 ? bt : 16);
      if (best < 0 || score < best) {
        best = score;
        bestBt = bt;
      }
    }
    kp.Bt = bestBt;
  }
  kp.R = threads / kp.Bt;
  plan->threads = threads;
  kp.nBlockTiles = (nblocks + kp.Bt - 1) / kp.Bt;
  kp.ndf = (int)dfs.size();
  for (int i = 0; i < kp.ndf; i++) split_ds(dfs[i], &kp.df_hi[i], &kp.df_lo[i]);
  kp.cstride = comp_stride(M);
  kp.nterm = M.nterm;
  kp.nspec = M.nspec;
  const bool gauss = (M.kind == kGauss || M.kind == kGaussSpec || M.kind == kGaussTSpec);
  const bool table = (M.kind == kPointSpec || M.kind == kGaussSpec || M.kind == kPointTSpec ||
                      M.kind == kGaussTSpec);
  // shrink the component tile until two CTAs fit per SM
  int ct = (T.ct + 1) & ~1;  // even: the recurrence kernel takes components in pairs
  const size_t budget = (threads == 128) ? 52 * 1024 : 110 * 1024;
  auto need = [&](int c) {
    size_t mainf = (T.flavor == kFlavorRecur)
                       ? smem_floats_main(kp.R, kp.Bt, K, c, kp.cstride, kp.ndf, gauss, table)
                       : (size_t)c * kp.cstride + (size_t)kp.R * 3;
    return 4 * std::max(mainf + 4, smem_floats_stage(kp.R, kp.Bt, K));
  };
  while (ct > 8 && need(ct) > budget) ct /= 2;
  kp.ct = ct;
  plan->smemBytes = need(ct);
  if (plan->smemBytes > 220 * 1024) {
    *err = "tile does not fit in shared memory";
    return 3;
  }

  KernelFn fn = pick_kernel(T.flavor, K, M.kind);
  plan->tune.K = K;
  cudaError_t ce =
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)plan->smemBytes);
  if (ce != cudaSuccess) {
    *err = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(ce);
    return 2;
  }
  int perSM = 0, dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, threads, plan->smemBytes);
  if (ce != cudaSuccess || perSM < 1) {
    *err = std::string("kernel cannot be resident: ") + cudaGetErrorString(ce);
    return 2;
  }
  plan->gridCap = perSM * nsm;

  ce = cudaMalloc(&plan->d_blocks, sizeof(BlockDesc) * (size_t)std::max(1, nblocks));
  if (ce != cudaSuccess) {
    *err = std::string("cudaMalloc blocks: ") + cudaGetErrorString(ce);
    return 2;
  }
  if (nblocks)
    ce = cudaMemcpy(plan->d_blocks, plan->blocks.data(), sizeof(BlockDesc) * nblocks,
                    cudaMemcpyHostToDevice);
  if (ce != cudaSuccess) {
    *err = std::string("cudaMemcpy blocks: ") + cudaGetErrorString(ce);
    return 2;
  }
  kp.blocks = plan->d_blocks;
  return 0;
}

void free_plan(Plan* plan) {
  if (plan->d_blocks) cudaFree(plan->d_blocks);
  plan->d_blocks = nullptr;
  plan->blocks.clear();
}

int launch_plan(const Plan& plan, float* d_vis, int rowBase, int nvis, const float* d_comps,
                int* d_err, cudaStream_t stream, std::string* err) {
  // An empty model leaves the data untouched for every operation, as the
  // reference CPU DFT does (ObitSkyModel.c:2405, "if (ncomp<=0) goto finish").
  if (nvis <= 0 || plan.kp.nblocks <= 0 || plan.model.ncomp <= 0) return 0;
  KParams kp = plan.kp;
  kp.vis = d_vis;
  kp.rowBase = rowBase;
  kp.nvis = nvis;
  kp.comps = d_comps;
  kp.ncomp = plan.model.ncomp;
  kp.errFlag = d_err;
  const long long nItems = (long long)((nvis + kp.R - 1) / kp.R) * kp.nBlockTiles;
  const int grid = (int)std::min<long long>(nItems, (long long)plan.gridCap);
  KernelFn fn = pick_kernel(plan.tune.flavor, plan.tune.K, plan.model.kind);
  fn<<<grid, plan.threads, plan.smemBytes, stream>>>(kp);
  cudaError_t ce = cudaGetLastError();
  if (ce != cudaSuccess) {
    *err = std::string("kernel launch: ") + cudaGetErrorString(ce);
    return 2;
  }
  return 0;
}

}  // namespace obit
