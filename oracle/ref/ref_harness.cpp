// Golden-vector harness around the reference CCD library (test infrastructure only).
//
// Links the unmodified reference objects (everything except main.cpp; parse.cpp is used for
// its argp front end) and drives one single-rank CCD solve the way main.cpp:25-682 does in
// stored-V mode, then writes what the parity tests need to a sectioned binary file:
//   basis/channel structure after the 1-rank ffdBalance permutation (SPBasis.cpp:80-819,
//   balance.cpp:91-144), the normal-ordered single-particle energies, E_ref, E_MBPT2, the
//   correlation energy after every iteration, the converged t2_pphh data, the 8 remap tables
//   of loadMaps (load.cpp:389-532), and FNV-1a hashes of every V chain (full V blocks too
//   when CCD_DUMP_V=1).
//
// Usage: CCD_DUMP=out.bin [CCD_DUMP_V=1] ref_harness <ccd.exe options>
//        CCD_BENCH=steps,iterations,tol ref_harness <ccd.exe options>   (timing only)
// The dump format is read by oracle/refdump.py.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdint>
#include <cmath>
#include <string>
#include <vector>
#include <omp.h>
#include <mpi.h>
#include "parse.hpp"
#include "load.hpp"
#include "calc.hpp"
#include "Chain.hpp"
#include "SPBasis.hpp"
#include "MBPT2Corr.hpp"
#include "balance.hpp"

namespace {

FILE *g_dump = nullptr;

// Section layout: u32 name_len, name bytes, u32 dtype code, u64 element count, raw data.
// dtype codes: 1 = f64, 2 = u64, 3 = i64.
void put_section(const char *name, uint32_t dtype, const void *data, uint64_t count,
                 size_t elem_size) {
  if (!g_dump) return;
  uint32_t n = (uint32_t)strlen(name);
  fwrite(&n, 4, 1, g_dump);
  fwrite(name, 1, n, g_dump);
  fwrite(&dtype, 4, 1, g_dump);
  fwrite(&count, 8, 1, g_dump);
  if (count) fwrite(data, elem_size, count, g_dump);
}
void put_f64(const char *name, const std::vector<double> &v) {
  put_section(name, 1, v.data(), v.size(), 8);
}
void put_u64(const char *name, const std::vector<uint64_t> &v) {
  put_section(name, 2, v.data(), v.size(), 8);
}

uint64_t fnv1a(uint64_t h, const void *data, size_t n) {
  const unsigned char *p = (const unsigned char *)data;
  for (size_t i = 0; i < n; i++) {
    h ^= p[i];
    h *= 1099511628211ULL;
  }
  return h;
}
const uint64_t kFnvSeed = 1469598103934665603ULL;

// Hash of a V chain over the channels whose rows and columns are both non-empty, in
// channel order; optionally appends the raw values to `raw`.
uint64_t hash_chain(Chain<double> *c, size_t start, size_t end, std::vector<double> *raw) {
  uint64_t h = kFnvSeed;
  for (size_t ch = start; ch < end; ch++) {
    size_t n = c->nRows(ch) * c->nColumns(ch);
    if (!n) continue;
    double *b = c->get(ch);
    h = fnv1a(h, b, n * sizeof(double));
    if (raw) raw->insert(raw->end(), b, b + n);
  }
  return h;
}

void dump_map(const char *name, Chain<ChainIndex> &m, size_t nch) {
  std::vector<uint64_t> v;
  for (size_t ch = 0; ch < nch; ch++) {
    for (size_t r = 0; r < m.nRows(ch); r++)
      for (size_t c = 0; c < m.nColumns(ch); c++) {
        ChainIndex x = m.get(ch, r, c);
        v.push_back(x.channel);
        v.push_back(x.row);
        v.push_back(x.column);
      }
  }
  put_u64(name, v);
}

}  // namespace

int main(int argc, char *argv[]) {
  MPI_Init(0, 0);
  const char *dump_path = getenv("CCD_DUMP");
  const bool dump_v = getenv("CCD_DUMP_V") && atoi(getenv("CCD_DUMP_V"));
  if (dump_path) g_dump = fopen(dump_path, "wb");

  SPBasis *basis;
  double tolerance = 1.e-8;
  int saveMemory = 0, verbose = 0;
  char *timeFile = NULL, timeMode, *modelFile = NULL;
  char *parseMem = parse(argc, argv, &basis, &tolerance, &saveMemory, &timeFile, &timeMode,
                         &modelFile, &verbose, 0);

  double t_setup0 = omp_get_wtime();
  double Eref = basis->referenceEnergy();
  basis->rotateSpEnergiesToNormalOrdered();
  basis->setUpChannelValues();
  basis->setUpChannelDims();

  const size_t nch = basis->nChannels, nsp = basis->nSpstates, np = basis->nParticles;
  std::vector<double> costs(nch);
  for (size_t c = 0; c < nch; c++) {  // cost model of main.cpp:94-112
    double pp = basis->chanDims[c].ppDim, hh = basis->chanDims[c].hhDim;
    double ph = basis->chanDims[c].phDim, hp = basis->chanDims[c].hpDim;
    double phm = basis->chanModDims[c].phDim, hpm = basis->chanModDims[c].hpDim;
    (void)phm; (void)hpm;
    costs[c] = 0;
    costs[c] += hh * hh; costs[c] += hh * hp; costs[c] += hh * pp; costs[c] += hp * ph;
    costs[c] += hp * pp; costs[c] += pp * pp; costs[c] += hp * ph; costs[c] += hp * hp;
  }
  size_t sc[1], ec[1], smc[1], emc[1], spc[1], epc[1], shc[1], ehc[1];
  ffdBalance(1, nch, costs.data(), basis->channelIndices, sc, ec);
  ffdBalance(1, nch, costs.data(), basis->modChannelIndices, smc, emc);
  clownBalance(1, nsp - np, basis->spChannelIndices, spc, epc);
  clownBalance(1, np, basis->spChannelIndices, shc, ehc);
  basis->setUpInverseChannelIndicesAndPermuteDims();
  basis->setUpChannelMaps();

  std::vector<size_t> ppD(nch), hhD(nch), phD(nch), hpD(nch), phM(nch), hpM(nch);
  std::vector<size_t> hppD(np), phhD(nsp - np), one(nsp, 1);
  for (size_t c = 0; c < nch; c++) {
    ppD[c] = basis->chanDims[c].ppDim; hhD[c] = basis->chanDims[c].hhDim;
    phD[c] = basis->chanDims[c].phDim; hpD[c] = basis->chanDims[c].hpDim;
    phM[c] = basis->chanModDims[c].phDim; hpM[c] = basis->chanModDims[c].hpDim;
  }
  for (size_t i = 0; i < np; i++) hppD[i] = basis->threeBodyChanDims[i].hppDim;
  for (size_t a = np; a < nsp; a++) phhD[a - np] = basis->threeBodyChanDims[a].phhDim;
  double t_setup1 = omp_get_wtime();

  Chain<double> t2(0, nch, nch, ppD.data(), hhD.data());
  Chain<double> t2Diff(0, nch, nch, ppD.data(), hhD.data());
  Chain<double> t2Diff_phhp(0, nch, nch, phM.data(), hpM.data());
  Chain<double> t2Diff_p2_p1hh(0, nsp - np, nsp - np, one.data(), phhD.data());
  Chain<double> t2Diff_h2pp_h1(0, np, np, hppD.data(), one.data());
  Chain<double> t2Old(0, nch, nch, ppD.data(), hhD.data());
  Chain<double> t2Old_phhp(0, nch, nch, phM.data(), hpM.data());
  Chain<double> t2Old_p1_p2hh(0, nsp - np, nsp - np, one.data(), phhD.data());
  Chain<double> t2Old_p2_p1hh(0, nsp - np, nsp - np, one.data(), phhD.data());
  Chain<double> t2Old_h1pp_h2(0, np, np, hppD.data(), one.data());
  Chain<double> t2Old_h2pp_h1(0, np, np, hppD.data(), one.data());
  Chain<ChainIndex> m_iab_j(0, nch, nch, ppD.data(), hhD.data());
  Chain<ChainIndex> m_jab_i(0, nch, nch, ppD.data(), hhD.data());
  Chain<ChainIndex> m_a_bij(0, nch, nch, ppD.data(), hhD.data());
  Chain<ChainIndex> m_b_aij(0, nch, nch, ppD.data(), hhD.data());
  Chain<ChainIndex> m_ai_jb(0, nch, nch, ppD.data(), hhD.data());
  Chain<ChainIndex> m_aj_ib(0, nch, nch, ppD.data(), hhD.data());
  Chain<ChainIndex> m_bi_ja(0, nch, nch, ppD.data(), hhD.data());
  Chain<ChainIndex> m_bj_ia(0, nch, nch, ppD.data(), hhD.data());
  Chain<double> d_iab_j(0, nch, nch, ppD.data(), hhD.data());
  Chain<double> d_jab_i(0, nch, nch, ppD.data(), hhD.data());
  Chain<double> d_a_bij(0, nch, nch, ppD.data(), hhD.data());
  Chain<double> d_b_aij(0, nch, nch, ppD.data(), hhD.data());
  Chain<double> d_ai_jb(0, nch, nch, ppD.data(), hhD.data());
  Chain<double> d_aj_ib(0, nch, nch, ppD.data(), hhD.data());
  Chain<double> d_bi_ja(0, nch, nch, ppD.data(), hhD.data());
  Chain<double> d_bj_ia(0, nch, nch, ppD.data(), hhD.data());

  Chain<double> *v_hhhh = new Chain<double>(0, nch, nch, hhD.data(), hhD.data());
  Chain<double> *v_hhpp = new Chain<double>(0, nch, nch, hhD.data(), ppD.data());
  Chain<double> *v_pppp = new Chain<double>(0, nch, nch, ppD.data(), ppD.data());
  Chain<double> *v_phh_p = new Chain<double>(0, nsp - np, nsp - np, phhD.data(), one.data());
  Chain<double> *v_h_hpp = new Chain<double>(0, np, np, one.data(), hppD.data());
  Chain<double> *v_hpph_mod = new Chain<double>(0, nch, nch, hpM.data(), phM.data());
  Chain<double> *v_hphp_mod = new Chain<double>(0, nch, nch, hpM.data(), hpM.data());
  loadVnn_hhhh(0, nch, v_hhhh, basis);
  loadVnn_hhpp(0, nch, v_hhpp, basis);
  loadVnn_pppp(0, nch, v_pppp, basis);
  loadVnn_phh_p(0, nsp - np, v_phh_p, basis);
  loadVnn_h_hpp(0, np, v_h_hpp, basis);
  loadVnn_hhpp_hpph_mod(0, nch, v_hpph_mod, basis);
  loadVnn_hpph_hphp_mod(0, nch, v_hphp_mod, basis);
  loadMaps(0, nch, m_iab_j, m_jab_i, m_a_bij, m_b_aij, m_ai_jb, m_aj_ib, m_bi_ja, m_bj_ia, basis);
  size_t s0[1] = {0}, e_ch[1] = {nch}, e_h[1] = {np}, e_p[1] = {nsp - np};
  MapDistributedData *f_ai_jb = m_ai_jb.mapFromDistributedCreate(0, nch, s0, e_ch, MPI_COMM_WORLD);
  MapDistributedData *f_aj_ib = m_aj_ib.mapFromDistributedCreate(0, nch, s0, e_ch, MPI_COMM_WORLD);
  MapDistributedData *f_bi_ja = m_bi_ja.mapFromDistributedCreate(0, nch, s0, e_ch, MPI_COMM_WORLD);
  MapDistributedData *f_bj_ia = m_bj_ia.mapFromDistributedCreate(0, nch, s0, e_ch, MPI_COMM_WORLD);
  MapDistributedData *f_iab_j = m_iab_j.mapFromDistributedCreate(0, nch, s0, e_h, MPI_COMM_WORLD);
  MapDistributedData *f_jab_i = m_jab_i.mapFromDistributedCreate(0, nch, s0, e_h, MPI_COMM_WORLD);
  MapDistributedData *f_a_bij = m_a_bij.mapFromDistributedCreate(0, nch, s0, e_p, MPI_COMM_WORLD);
  MapDistributedData *f_b_aij = m_b_aij.mapFromDistributedCreate(0, nch, s0, e_p, MPI_COMM_WORLD);
  MapDistributedData *t_iab_j = m_iab_j.mapToDistributedCreate(0, nch, s0, e_h, MPI_COMM_WORLD);
  MapDistributedData *t_jab_i = m_jab_i.mapToDistributedCreate(0, nch, s0, e_h, MPI_COMM_WORLD);
  MapDistributedData *t_a_bij = m_a_bij.mapToDistributedCreate(0, nch, s0, e_p, MPI_COMM_WORLD);
  MapDistributedData *t_b_aij = m_b_aij.mapToDistributedCreate(0, nch, s0, e_p, MPI_COMM_WORLD);
  MapDistributedData *t_ai_jb = m_ai_jb.mapToDistributedCreate(0, nch, s0, e_ch, MPI_COMM_WORLD);
  double t_load1 = omp_get_wtime();

  // Bench mode (CCD_BENCH="steps,iterations,tol"): after the one set-up above, `steps`
  // solves from T2 = 0, each a bounded sample of at most `iterations` iterations of the loop
  // below (stopping earlier at |dE| <= tol), timed like cc_diagrams_time; one line per step.
  const char *bench = getenv("CCD_BENCH");
  long bench_steps = 0, bench_iters = 0;
  double bench_tol = 0;
  if (bench && sscanf(bench, "%ld,%ld,%lf", &bench_steps, &bench_iters, &bench_tol) != 3) {
    fprintf(stderr, "CCD_BENCH must be steps,iterations,tol\n");
    return 2;
  }
  double mbpt2 = bench ? 0.0 : MBPT2Corr(0, nch, v_hhpp, basis);

  // Iteration loop: same stop rule, cap and mixing as main.cpp:491-519.
  double energyDiff = 1.0, corrCCD = 100.0, corrPrev = 100.0, mixing = 0.5;
  unsigned long iterations = 0;
  int max_iters = 100;
  std::vector<double> energies;
  auto solve = [&](double tol, unsigned long cap) {
    t2.zero(); t2Old.zero(); t2Old_h2pp_h1.zero(); t2Old_h1pp_h2.zero();
    t2Old_p1_p2hh.zero(); t2Old_p2_p1hh.zero(); t2Old_phhp.zero();
    energyDiff = 1.0; corrCCD = 100.0; corrPrev = 100.0;
    iterations = 0;
    energies.clear();
    while (std::abs(energyDiff) > tol) {
      if (iterations > (unsigned long)max_iters || iterations >= cap) break;
      calcT2Diff_p2_p1hh(0, nsp - np, v_phh_p, t2Old_p1_p2hh, t2Old_p2_p1hh, t2Diff_p2_p1hh, basis);
      calcT2Diff_h2pp_h1(0, np, v_h_hpp, t2Old_h1pp_h2, t2Old_h2pp_h1, t2Diff_h2pp_h1, basis);
      calcT2Diff_phhp(0, nch, v_hpph_mod, v_hphp_mod, t2Old_phhp, t2Diff_phhp, basis);
      calcT2Diff_pphh(0, nch, v_hhhh, v_hhpp, v_pppp, t2Old, t2Diff, basis);
      d_iab_j.mapFromDistributed(&t2Diff_h2pp_h1, f_iab_j);
      d_jab_i.mapFromDistributed(&t2Diff_h2pp_h1, f_jab_i);
      d_a_bij.mapFromDistributed(&t2Diff_p2_p1hh, f_a_bij);
      d_b_aij.mapFromDistributed(&t2Diff_p2_p1hh, f_b_aij);
      d_ai_jb.mapFromDistributed(&t2Diff_phhp, f_ai_jb);
      d_aj_ib.mapFromDistributed(&t2Diff_phhp, f_aj_ib);
      d_bi_ja.mapFromDistributed(&t2Diff_phhp, f_bi_ja);
      d_bj_ia.mapFromDistributed(&t2Diff_phhp, f_bj_ia);
      double corr = calcT2_pphh(0, nch, v_hhpp, t2, t2Diff, t2Old, d_iab_j, d_jab_i, d_a_bij,
                                d_b_aij, d_ai_jb, d_aj_ib, d_bi_ja, d_bj_ia, basis, mixing);
      t2Old.set(&t2);
      t2.mapToDistributed(&t2Old_h2pp_h1, t_jab_i);
      t2.mapToDistributed(&t2Old_h1pp_h2, t_iab_j);
      t2.mapToDistributed(&t2Old_p1_p2hh, t_a_bij);
      t2.mapToDistributed(&t2Old_p2_p1hh, t_b_aij);
      t2.mapToDistributed(&t2Old_phhp, t_ai_jb);
      corrCCD = corr;
      energyDiff = corrCCD - corrPrev;
      corrPrev = corrCCD;
      energies.push_back(corrCCD);
      iterations++;
    }
  };
  if (bench) {
    printf("setup_time: %f\nload_time: %f\n", t_setup1 - t_setup0, t_load1 - t_setup1);
    for (long k = 0; k < bench_steps; k++) {
      double b0 = omp_get_wtime();
      solve(bench_tol, (unsigned long)bench_iters);
      double b1 = omp_get_wtime();
      printf("bench_step: %lu %.9f %.17g\n", iterations, b1 - b0, corrCCD);
      fflush(stdout);
    }
    parseFree(parseMem);
    MPI_Finalize();
    return 0;
  }
  double cc0 = omp_get_wtime();
  solve(tolerance, ~0ul);
  double cc1 = omp_get_wtime();

  printf("iterations: %lu\n", iterations);
  printf("Reference Energy: %.17g\n", Eref);
  printf("MBPT2Corr: %.17g\n", mbpt2);
  printf("CCDCorr: %.17g\n", corrCCD);
  printf("CCDCorr/A: %.17g\n", corrCCD / np);
  printf("E_CCD/A: %.17g\n", (Eref + corrCCD) / np);
  printf("setup_time: %f\nload_time: %f\ncc_diagrams_time: %f\n", t_setup1 - t_setup0,
         t_load1 - t_setup1, cc1 - cc0);

  if (g_dump) {
    std::vector<uint64_t> hdr = {nsp, np, nch, iterations};
    put_u64("header", hdr);
    put_f64("sp_energy", std::vector<double>(basis->spEnergy, basis->spEnergy + nsp));
    put_f64("scalars", {Eref, mbpt2, corrCCD, tolerance});
    put_f64("energies", energies);
    std::vector<uint64_t> dims, mdims, tdims, pp, hh, phm, hpm, hpp, phh;
    for (size_t c = 0; c < nch; c++) {
      dims.insert(dims.end(), {ppD[c], hhD[c], hpD[c], phD[c]});
      mdims.insert(mdims.end(), {basis->chanModDims[c].ppDim, basis->chanModDims[c].hhDim,
                                 hpM[c], phM[c]});
      for (size_t k = 0; k < ppD[c]; k++)
        pp.insert(pp.end(), {basis->chanMaps[c].ppMap[k].p, basis->chanMaps[c].ppMap[k].q});
      for (size_t k = 0; k < hhD[c]; k++)
        hh.insert(hh.end(), {basis->chanMaps[c].hhMap[k].p, basis->chanMaps[c].hhMap[k].q});
      for (size_t k = 0; k < phM[c]; k++)
        phm.insert(phm.end(), {basis->chanModMaps[c].phMap[k].p, basis->chanModMaps[c].phMap[k].q});
      for (size_t k = 0; k < hpM[c]; k++)
        hpm.insert(hpm.end(), {basis->chanModMaps[c].hpMap[k].p, basis->chanModMaps[c].hpMap[k].q});
    }
    for (size_t i = 0; i < nsp; i++)
      tdims.insert(tdims.end(), {basis->threeBodyChanDims[i].phhDim, basis->threeBodyChanDims[i].hppDim});
    for (size_t i = 0; i < np; i++)
      for (size_t k = 0; k < hppD[i]; k++) {
        PQRBundle b = basis->threeBodyChanMaps[i].hppMap[k];
        hpp.insert(hpp.end(), {b.p, b.q, b.r});
      }
    for (size_t a = np; a < nsp; a++)
      for (size_t k = 0; k < phhD[a - np]; k++) {
        PQRBundle b = basis->threeBodyChanMaps[a].phhMap[k];
        phh.insert(phh.end(), {b.p, b.q, b.r});
      }
    put_u64("chan_dims", dims);
    put_u64("chan_mod_dims", mdims);
    put_u64("three_body_dims", tdims);
    put_u64("pp_map", pp);
    put_u64("hh_map", hh);
    put_u64("ph_mod_map", phm);
    put_u64("hp_mod_map", hpm);
    put_u64("hpp_map", hpp);
    put_u64("phh_map", phh);
    std::vector<double> t2data;
    for (size_t c = 0; c < nch; c++) {
      size_t n = ppD[c] * hhD[c];
      if (n) t2data.insert(t2data.end(), t2.get(c), t2.get(c) + n);
    }
    put_f64("t2", t2data);
    dump_map("map_iab_j", m_iab_j, nch);
    dump_map("map_jab_i", m_jab_i, nch);
    dump_map("map_a_bij", m_a_bij, nch);
    dump_map("map_b_aij", m_b_aij, nch);
    dump_map("map_ai_jb", m_ai_jb, nch);
    dump_map("map_aj_ib", m_aj_ib, nch);
    dump_map("map_bi_ja", m_bi_ja, nch);
    dump_map("map_bj_ia", m_bj_ia, nch);
    // V hashes over the channels the solver uses (T-carrying channels only).
    std::vector<double> raw[7];
    std::vector<double> *rp[7];
    for (int k = 0; k < 7; k++) rp[k] = dump_v ? &raw[k] : nullptr;
    std::vector<uint64_t> hashes;
    Chain<double> *vs[7] = {v_hhhh, v_hhpp, v_pppp, v_hpph_mod, v_hphp_mod, v_h_hpp, v_phh_p};
    const char *vn[7] = {"v_hhhh", "v_hhpp", "v_pppp", "v_hpph_mod", "v_hphp_mod", "v_h_hpp", "v_phh_p"};
    for (int k = 0; k < 7; k++) {
      size_t end = (k == 5) ? np : (k == 6) ? nsp - np : nch;
      uint64_t h = kFnvSeed;
      std::vector<double> tmp;
      for (size_t ch = 0; ch < end; ch++) {
        bool active;
        if (k <= 2) active = ppD[ch] && hhD[ch];
        else if (k <= 4) active = phM[ch] && hpM[ch];
        else active = true;
        if (!active) continue;
        size_t n = vs[k]->nRows(ch) * vs[k]->nColumns(ch);
        if (!n) continue;
        h = fnv1a(h, vs[k]->get(ch), n * 8);
        if (rp[k]) rp[k]->insert(rp[k]->end(), vs[k]->get(ch), vs[k]->get(ch) + n);
      }
      hashes.push_back(h);
      if (dump_v) put_f64(vn[k], raw[k]);
    }
    put_u64("v_hashes", hashes);
    fclose(g_dump);
  }
  (void)hash_chain;
  parseFree(parseMem);
  MPI_Finalize();
  return 0;
}
