// Test harness for the host-side DFT planner (obit_b200/csrc/dft_planner.cpp).
// Reads one layout from stdin and prints the plan as JSON.  Input format
// (whitespace separated):
//   lrec nrparm nchan nif nstok incs incf incif kincf kincif
//   chanb chane ifb ife stokb stoke
//   kind nterm lcomp ncomp nspec
//   flavor K ct Bt threads
//   nfreq, then nfreq fscale values, nfreq lnspec values, nfreq specIndex values
//   optionally: nidx, then nidx per-component spectral indices in table order
//   (the component count becomes nidx), then optionally ngauss: the table is
//   a mixed one, nidx point rows followed by ngauss Gaussian rows
#include <cstdio>
#include <iostream>
#include <string>
#include <vector>

#include "dft_plan.h"

using namespace obit;

int main() {
  LayoutDesc L;
  ModelDesc M;
  ApplyDesc A;
  TuneDesc T;
  std::cin >> L.lrec >> L.nrparm >> L.nchan >> L.nif >> L.nstok >> L.incs >> L.incf >> L.incif >>
      L.kincf >> L.kincif;
  std::cin >> L.chanb >> L.chane >> L.ifb >> L.ife >> L.stokb >> L.stoke;
  std::cin >> M.kind >> M.nterm >> M.lcomp >> M.ncomp >> M.nspec;
  std::cin >> T.flavor >> T.K >> T.ct >> T.Bt >> T.threads;
  int nfreq = 0;
  std::cin >> nfreq;
  L.fscale.resize(nfreq);
  L.lnspec.resize(nfreq);
  L.specIndex.resize(nfreq);
  for (auto& v : L.fscale) std::cin >> v;
  for (auto& v : L.lnspec) std::cin >> v;
  for (auto& v : L.specIndex) std::cin >> v;
  int nidx = 0;
  std::vector<float> idx;
  if (std::cin >> nidx && nidx > 0) {
    idx.resize(nidx);
    for (auto& v : idx) std::cin >> v;
    M.ncomp = nidx;
    M.specIndex = idx.data();
    int ngauss = 0;
    if (std::cin >> ngauss && ngauss > 0) {
      M.ncompPt = nidx;
      M.ncomp = ngauss;
    }
  }
  Plan P;
  std::string err;
  const int rc = plan_layout(L, M, A, T, &P, &err);
  printf("{\"rc\": %d, \"err\": \"%s\"", rc, err.c_str());
  if (rc == 0) {
    const KParams& k = P.kp;
    printf(", \"K\": %d, \"Bt\": %d, \"R\": %d, \"ct\": %d, \"threads\": %d, \"nblocks\": %d, "
           "\"ndf\": %d, \"smem\": %zu, \"linear\": %d, \"nBlockTiles\": %d, \"specFactored\": %d, "
           "\"mixed\": %d, \"df\": [",
           P.tune.K, k.Bt, k.R, k.ct, P.threads, k.nblocks, k.ndf, P.smemBytes, (int)P.linear,
           k.nBlockTiles, (int)P.specFactored, (int)P.mixed);
    for (int i = 0; i < k.ndf; i++) printf("%s%.17g", i ? ", " : "", (double)k.df_hi[i] + (double)k.df_lo[i]);
    printf("], \"blocks\": [");
    for (size_t i = 0; i < P.blocks.size(); i++) {
      const BlockDesc& b = P.blocks[i];
      printf("%s{\"f0\": %.17g, \"df\": %.9g, \"off0\": %d, \"len\": %d, \"dfc\": %d, \"plane\": %d, "
             "\"ifq0\": %d, \"l\": [",
             i ? ", " : "", (double)b.f0_hi + (double)b.f0_lo, b.df, b.off0, b.len, b.dfc, b.plane,
             b.ifq0);
      for (int t = 0; t < kMaxNTerm; t++)
        printf("%s[%.9g, %.9g, %.9g]", t ? ", " : "", b.l[t][0], b.l[t][1], b.l[t][2]);
      printf("]}");
    }
    printf("]");
  }
  printf("}\n");
  return 0;
}
