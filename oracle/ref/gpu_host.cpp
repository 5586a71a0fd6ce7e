// The reference's own host driving libccdgpu through the C ABI (boundary test).
//
// Links the unmodified reference objects (everything except main.cpp; parse.cpp for its argp
// front end) and follows main.cpp:25-455 for one MPI rank: argp options, the SPBasis
// subclass, E_ref and normal ordering, channel dimensions, the 1-rank ffdBalance order,
// channel maps, the V chains (loadVnn_*) and the eight loadMaps tables.  The CCD loop of
// main.cpp:491-682 is then replaced by the patch INTEGRATION.md gives: the reference's own
// arrays (chanDims, chanModDims, chanMaps, chanModMaps, threeBodyChanDims, Chain<T>::get
// blocks, ChainIndex maps) go to ccdgpu_create as they are, ccdgpu_solve runs the loop, and
// the amplitudes come back into t2_pphh.  The result is printed as main.cpp:692-702 does.
//
// Usage: gpu_host <ccd.exe options>   (CCD_GPU_PRECISION=mixed_bf16 for the mixed mode)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <omp.h>
#include <mpi.h>
#include "parse.hpp"
#include "load.hpp"
#include "Chain.hpp"
#include "SPBasis.hpp"
#include "balance.hpp"

#include "ccdgpu.h"

// Per-channel block pointers of a Chain (NULL for empty blocks), as ccdgpu_problem expects.
template <typename T>
static std::vector<const T *> blocks(Chain<T> *c, std::size_t n) {
  std::vector<const T *> v(n);
  for (std::size_t ch = 0; ch < n; ch++) v[ch] = c->get(ch);
  return v;
}

int main(int argc, char *argv[]) {
  MPI_Init(0, 0);
  SPBasis *basis;
  double tolerance = 1.e-8;
  int saveMemory = 0, verbose = 0;
  char *timeFile = NULL, timeMode, *modelFile = NULL;
  char *parseMem = parse(argc, argv, &basis, &tolerance, &saveMemory, &timeFile, &timeMode,
                         &modelFile, &verbose, 0);
  const double totalTimeTic = omp_get_wtime();

  // main.cpp:64-136
  const double Eref = basis->referenceEnergy();
  basis->rotateSpEnergiesToNormalOrdered();
  basis->setUpChannelValues();
  basis->setUpChannelDims();
  const std::size_t nch = basis->nChannels, nsp = basis->nSpstates, np = basis->nParticles;
  std::vector<double> costs(nch);
  for (std::size_t c = 0; c < nch; c++) {  // main.cpp:94-112
    const double pp = basis->chanDims[c].ppDim, hh = basis->chanDims[c].hhDim;
    const double ph = basis->chanDims[c].phDim, hp = basis->chanDims[c].hpDim;
    costs[c] = hh * hh + hh * hp + hh * pp + hp * ph + hp * pp + pp * pp + hp * ph + hp * hp;
  }
  std::size_t sc[1], ec[1], smc[1], emc[1], spc[1], epc[1], shc[1], ehc[1];
  ffdBalance(1, nch, costs.data(), basis->channelIndices, sc, ec);
  ffdBalance(1, nch, costs.data(), basis->modChannelIndices, smc, emc);
  clownBalance(1, nsp - np, basis->spChannelIndices, spc, epc);
  clownBalance(1, np, basis->spChannelIndices, shc, ehc);
  basis->setUpInverseChannelIndicesAndPermuteDims();
  basis->setUpChannelMaps();

  // main.cpp:142-455: dimensions, the chains the loop fills, V and the remap tables.
  std::vector<std::size_t> ppD(nch), hhD(nch), phM(nch), hpM(nch), hppD(np), phhD(nsp - np),
      one(nsp, 1);
  for (std::size_t c = 0; c < nch; c++) {
    ppD[c] = basis->chanDims[c].ppDim; hhD[c] = basis->chanDims[c].hhDim;
    phM[c] = basis->chanModDims[c].phDim; hpM[c] = basis->chanModDims[c].hpDim;
  }
  for (std::size_t i = 0; i < np; i++) hppD[i] = basis->threeBodyChanDims[i].hppDim;
  for (std::size_t a = np; a < nsp; a++) phhD[a - np] = basis->threeBodyChanDims[a].phhDim;
  Chain<double> t2_pphh(0, nch, nch, ppD.data(), hhD.data());
  t2_pphh.zero();
  Chain<ChainIndex> map_pphh_iab_j_hpp_h(0, nch, nch, ppD.data(), hhD.data());
  Chain<ChainIndex> map_pphh_jab_i_hpp_h(0, nch, nch, ppD.data(), hhD.data());
  Chain<ChainIndex> map_pphh_a_bij_p_phh(0, nch, nch, ppD.data(), hhD.data());
  Chain<ChainIndex> map_pphh_b_aij_p_phh(0, nch, nch, ppD.data(), hhD.data());
  Chain<ChainIndex> map_pphh_ai_jb_phhp(0, nch, nch, ppD.data(), hhD.data());
  Chain<ChainIndex> map_pphh_aj_ib_phhp(0, nch, nch, ppD.data(), hhD.data());
  Chain<ChainIndex> map_pphh_bi_ja_phhp(0, nch, nch, ppD.data(), hhD.data());
  Chain<ChainIndex> map_pphh_bj_ia_phhp(0, nch, nch, ppD.data(), hhD.data());
  Chain<double> *vnn_hhhh = new Chain<double>(0, nch, nch, hhD.data(), hhD.data());
  Chain<double> *vnn_hhpp = new Chain<double>(0, nch, nch, hhD.data(), ppD.data());
  Chain<double> *vnn_pppp = new Chain<double>(0, nch, nch, ppD.data(), ppD.data());
  Chain<double> *vnn_phh_p = new Chain<double>(0, nsp - np, nsp - np, phhD.data(), one.data());
  Chain<double> *vnn_h_hpp = new Chain<double>(0, np, np, one.data(), hppD.data());
  Chain<double> *vnn_hhpp_hpph_mod = new Chain<double>(0, nch, nch, hpM.data(), phM.data());
  Chain<double> *vnn_hpph_hphp_mod = new Chain<double>(0, nch, nch, hpM.data(), hpM.data());
  loadVnn_hhhh(0, nch, vnn_hhhh, basis);
  loadVnn_hhpp(0, nch, vnn_hhpp, basis);
  loadVnn_pppp(0, nch, vnn_pppp, basis);
  loadVnn_phh_p(0, nsp - np, vnn_phh_p, basis);
  loadVnn_h_hpp(0, np, vnn_h_hpp, basis);
  loadVnn_hhpp_hpph_mod(0, nch, vnn_hhpp_hpph_mod, basis);
  loadVnn_hpph_hphp_mod(0, nch, vnn_hpph_hphp_mod, basis);
  loadMaps(0, nch, map_pphh_iab_j_hpp_h, map_pphh_jab_i_hpp_h, map_pphh_a_bij_p_phh,
           map_pphh_b_aij_p_phh, map_pphh_ai_jb_phhp, map_pphh_aj_ib_phhp, map_pphh_bi_ja_phhp,
           map_pphh_bj_ia_phhp, basis);

  // ---- the INTEGRATION.md patch (replaces main.cpp:491-682) ----
  auto hhhh = blocks(vnn_hhhh, nch), hhpp = blocks(vnn_hhpp, nch), pppp = blocks(vnn_pppp, nch);
  auto hpph = blocks(vnn_hhpp_hpph_mod, nch), hphp = blocks(vnn_hpph_hphp_mod, nch);
  auto hhpp3 = blocks(vnn_h_hpp, np), phh3 = blocks(vnn_phh_p, nsp - np);
  Chain<ChainIndex> *maps[8] = {&map_pphh_iab_j_hpp_h, &map_pphh_jab_i_hpp_h,
                                &map_pphh_a_bij_p_phh, &map_pphh_b_aij_p_phh,
                                &map_pphh_ai_jb_phhp, &map_pphh_aj_ib_phhp,
                                &map_pphh_bi_ja_phhp, &map_pphh_bj_ia_phhp};
  std::vector<const ChainIndex *> mb[8];
  for (int k = 0; k < 8; k++) mb[k] = blocks(maps[k], nch);

  ccdgpu_problem p = {};
  p.n_sp = nsp; p.n_particles = np; p.n_channels = nch;
  p.sp_energy = basis->spEnergy;  // already normal-ordered
  p.chan_dims = (const ccdgpu_channel_dims *)basis->chanDims;
  p.chan_mod_dims = (const ccdgpu_channel_dims *)basis->chanModDims;
  p.chan_maps = (const ccdgpu_channel_maps *)basis->chanMaps;
  p.chan_mod_maps = (const ccdgpu_channel_maps *)basis->chanModMaps;
  p.three_body_dims = (const ccdgpu_three_body_dims *)basis->threeBodyChanDims;
  p.v_hhhh = hhhh.data(); p.v_hhpp = hhpp.data(); p.v_pppp = pppp.data();
  p.v_hpph_mod = hpph.data(); p.v_hphp_mod = hphp.data();
  p.v_h_hpp = hhpp3.data(); p.v_phh_p = phh3.data();
  for (int k = 0; k < 8; k++) p.maps[k] = (const ccdgpu_chain_index *const *)mb[k].data();

  ccdgpu_options opt;
  ccdgpu_default_options(&opt);  // FP64, fused path, CUDA graph
  const char *prec = getenv("CCD_GPU_PRECISION");
  if (prec && !strcmp(prec, "mixed_bf16")) opt.precision = CCDGPU_PREC_MIXED_BF16;
  ccdgpu_handle *h = nullptr;
  int rc = ccdgpu_create(&p, &opt, &h);  // deep copy; host chains may be freed now
  if (rc) { fprintf(stderr, "ccdgpu: %s\n", ccdgpu_strerror(rc)); exit(1); }
  const double cc_time_0 = omp_get_wtime();
  ccdgpu_result res;
  rc = ccdgpu_solve(h, tolerance, /*max_iters=*/100, /*mixing=*/0.5, &res);  // main.cpp:508-519
  if (rc) { fprintf(stderr, "ccdgpu: %s\n", ccdgpu_strerror(rc)); exit(1); }
  const double cc_time_1 = omp_get_wtime();
  // Amplitudes back into t2_pphh, in its own data order (channel blocks, pp x hh row-major).
  std::vector<double> t2(ccdgpu_t2_size(h));
  ccdgpu_get_t2(h, t2.data(), t2.size());
  for (std::size_t ch = 0, off = 0; ch < nch; ch++) {
    std::size_t n = basis->chanDims[ch].ppDim * basis->chanDims[ch].hhDim;
    if (n) std::memcpy(t2_pphh.get(ch), t2.data() + off, n * sizeof(double));
    off += n;
  }
  const double corrCCD = res.e_corr;
  const unsigned long iterations = res.iterations;
  ccdgpu_destroy(h);
  // ---- end of the patch ----

  // The printout of main.cpp:692-702, plus a checksum of t2_pphh as the host now holds it.
  double sumsq = 0.0;
  for (std::size_t ch = 0; ch < nch; ch++)
    for (std::size_t k = 0; k < ppD[ch] * hhD[ch]; k++) sumsq += t2_pphh.get(ch)[k] * t2_pphh.get(ch)[k];
  printf("iterations: %lu\n", iterations);
  printf("CCDCorr: %.17g\n", corrCCD);
  printf("CCDCorr/A: %.17g\n", corrCCD / np);
  printf("E_CCD: %.17g\n", (Eref + corrCCD));
  printf("E_CCD/A: %.17g\n", (Eref + corrCCD) / np);
  printf("Final time: %g s\n", omp_get_wtime() - totalTimeTic);
  printf("cc_diagrams_time: %f\n", cc_time_1 - cc_time_0);
  printf("t2_sumsq: %.17g\n", sumsq);

  delete vnn_hhhh; delete vnn_hhpp; delete vnn_pppp; delete vnn_phh_p; delete vnn_h_hpp;
  delete vnn_hhpp_hpph_mod; delete vnn_hpph_hphp_mod;
  basis->deallocate();
  basis->deallocate_sp_basis();
  parseFree(parseMem);
  MPI_Finalize();
  return 0;
}
