/* CPU oracle for the CCD T2 iteration — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's stored-V CCD step, used only by tests/, the smoke
 * check and bench.py's cpu_baseline leg as the checker; the product never calls it.
 * Parity is pinned: tests compare this oracle's per-iteration energies and converged T2
 * against golden dumps of the reference itself (oracle/ref/ref_harness.cpp, fixtures in
 * tests/golden/).
 *
 * It follows the reference function by function on a ccdgpu_problem (include/ccdgpu.h):
 *   oracle_calc_t2diff_p2_p1hh   calc.cpp:9-43    (argument order of main.cpp:591-597)
 *   oracle_calc_t2diff_h2pp_h1   calc.cpp:73-107  (main.cpp:601-607 passes t2Old_h1pp_h2 as
 *                                                  the function's t2Old_h2pp_h1 and vice versa)
 *   oracle_calc_t2diff_phhp      calc.cpp:264-339
 *   oracle_calc_t2diff_pphh      calc.cpp:132-231
 *   oracle_map_from_distributed  main.cpp:632-639 via Chain::mapFromDistributed, Chain.hpp:710-755
 *   oracle_calc_t2_pphh          calc.cpp:368-459
 *   oracle_map_to_distributed    main.cpp:660-665 via Chain::set / mapToDistributed, Chain.hpp:503-527,757-802
 *   oracle_solve                 main.cpp:491-519,681 (E_prev = 100, stop on |dE| <= tol,
 *                                                  break once iterations > max_iters)
 * GEMMs are written out as loops (C = alpha*A*B + beta*C, row-major, no transposes, the
 * cblas_dgemm calls of calc.cpp:146,167,188,277,298).  Channels are processed in parallel,
 * each by one thread, and the energy is summed over channels in channel order, so results do
 * not depend on the thread count.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "ccdgpu.h"

typedef struct oracle_state {
  const ccdgpu_problem *p;
  uint64_t nch, nsp, np, npart;
  uint64_t *o_t, *o_m, *o_h, *o_p; /* slab offsets: pphh, phhp, hpp (per hole), phh (per particle) */
  uint64_t n_t, n_m, n_h, n_p;
  double *t2, *t2_old, *diff_pphh, *diff_phhp, *old_phhp;
  double *old_h1pp_h2, *old_h2pp_h1, *diff_h2pp_h1;
  double *old_p1_p2hh, *old_p2_p1hh, *diff_p2_p1hh;
  double *gath[8];       /* gathered pphh chains, ccdgpu_map_id order */
  uint64_t *flat[8];     /* tables as flat offsets into the source slab */
} oracle_state;

static void gemm(uint64_t M, uint64_t N, uint64_t K, double alpha, const double *A,
                 const double *B, double beta, double *C) {
  for (uint64_t m = 0; m < M; m++)
    for (uint64_t n = 0; n < N; n++) {
      double acc = 0.0;
      for (uint64_t k = 0; k < K; k++) acc += A[m * K + k] * B[k * N + n];
      C[m * N + n] = alpha * acc + beta * C[m * N + n];
    }
}

void oracle_free(oracle_state *s);

oracle_state *oracle_create(const ccdgpu_problem *p) {
  oracle_state *s = (oracle_state *)calloc(1, sizeof(oracle_state));
  if (!s) return NULL;
  s->p = p;
  s->nch = p->n_channels;
  s->nsp = p->n_sp;
  s->np = p->n_particles;
  s->npart = s->nsp - s->np;
  s->o_t = (uint64_t *)calloc(s->nch + 1, 8);
  s->o_m = (uint64_t *)calloc(s->nch + 1, 8);
  s->o_h = (uint64_t *)calloc(s->np + 1, 8);
  s->o_p = (uint64_t *)calloc(s->npart + 1, 8);
  for (uint64_t c = 0; c < s->nch; c++) {
    s->o_t[c + 1] = s->o_t[c] + p->chan_dims[c].pp * p->chan_dims[c].hh;
    s->o_m[c + 1] = s->o_m[c] + p->chan_mod_dims[c].ph * p->chan_mod_dims[c].hp;
  }
  for (uint64_t k = 0; k < s->np; k++) s->o_h[k + 1] = s->o_h[k] + p->three_body_dims[k].hpp;
  for (uint64_t a = 0; a < s->npart; a++)
    s->o_p[a + 1] = s->o_p[a] + p->three_body_dims[a + s->np].phh;
  s->n_t = s->o_t[s->nch];
  s->n_m = s->o_m[s->nch];
  s->n_h = s->o_h[s->np];
  s->n_p = s->o_p[s->npart];
  double **bufs[] = {&s->t2, &s->t2_old, &s->diff_pphh};
  for (int i = 0; i < 3; i++) *bufs[i] = (double *)calloc(s->n_t + 1, 8);
  s->diff_phhp = (double *)calloc(s->n_m + 1, 8);
  s->old_phhp = (double *)calloc(s->n_m + 1, 8);
  s->old_h1pp_h2 = (double *)calloc(s->n_h + 1, 8);
  s->old_h2pp_h1 = (double *)calloc(s->n_h + 1, 8);
  s->diff_h2pp_h1 = (double *)calloc(s->n_h + 1, 8);
  s->old_p1_p2hh = (double *)calloc(s->n_p + 1, 8);
  s->old_p2_p1hh = (double *)calloc(s->n_p + 1, 8);
  s->diff_p2_p1hh = (double *)calloc(s->n_p + 1, 8);
  for (int k = 0; k < 8; k++) {
    s->gath[k] = (double *)calloc(s->n_t + 1, 8);
    s->flat[k] = (uint64_t *)calloc(s->n_t + 1, 8);
    if (!s->gath[k] || !s->flat[k]) { oracle_free(s); return NULL; }
  }
  /* ChainIndex -> flat offset into the target chain's data (Chain<T>::get(ChainIndex)). */
  for (uint64_t c = 0; c < s->nch; c++) {
    uint64_t n = p->chan_dims[c].pp * p->chan_dims[c].hh;
    for (int k = 0; k < 8; k++) {
      const ccdgpu_chain_index *m = p->maps[k][c];
      for (uint64_t e = 0; e < n; e++) {
        uint64_t f;
        if (k <= 1) f = s->o_h[m[e].channel] + m[e].row;
        else if (k <= 3) f = s->o_p[m[e].channel] + m[e].column;
        else f = s->o_m[m[e].channel] + m[e].row * p->chan_mod_dims[m[e].channel].hp + m[e].column;
        s->flat[k][s->o_t[c] + e] = f;
      }
    }
  }
  return s;
}

void oracle_free(oracle_state *s) {
  if (!s) return;
  free(s->o_t); free(s->o_m); free(s->o_h); free(s->o_p);
  free(s->t2); free(s->t2_old); free(s->diff_pphh); free(s->diff_phhp); free(s->old_phhp);
  free(s->old_h1pp_h2); free(s->old_h2pp_h1); free(s->diff_h2pp_h1);
  free(s->old_p1_p2hh); free(s->old_p2_p1hh); free(s->diff_p2_p1hh);
  for (int k = 0; k < 8; k++) { free(s->gath[k]); free(s->flat[k]); }
  free(s);
}

uint64_t oracle_t2_size(const oracle_state *s) { return s->n_t; }

/* calc.cpp:9-43: y_a = sum_{(b,i,j)} t2Old_p1_p2hh * v;  diff = -0.5 * y_a * t2Old_p2_p1hh. */
void oracle_calc_t2diff_p2_p1hh(oracle_state *s) {
#pragma omp parallel for schedule(dynamic)
  for (int64_t a = 0; a < (int64_t)s->npart; a++) {
    const double *v = s->p->v_phh_p[a];
    uint64_t n = s->o_p[a + 1] - s->o_p[a];
    const double *t1 = s->old_p1_p2hh + s->o_p[a], *t2 = s->old_p2_p1hh + s->o_p[a];
    double *d = s->diff_p2_p1hh + s->o_p[a];
    double value = 0.;
    for (uint64_t k = 0; k < n; k++) value += t1[k] * v[k];
    for (uint64_t k = 0; k < n; k++) d[k] = -0.5 * value * t2[k];
  }
}

/* calc.cpp:73-107 with main.cpp:601-607's argument order: the dot product runs over
 * main's t2Old_h2pp_h1 and the scale uses main's t2Old_h1pp_h2. */
void oracle_calc_t2diff_h2pp_h1(oracle_state *s) {
#pragma omp parallel for schedule(dynamic)
  for (int64_t k = 0; k < (int64_t)s->np; k++) {
    const double *v = s->p->v_h_hpp[k];
    uint64_t n = s->o_h[k + 1] - s->o_h[k];
    const double *dotsrc = s->old_h2pp_h1 + s->o_h[k], *scalesrc = s->old_h1pp_h2 + s->o_h[k];
    double *d = s->diff_h2pp_h1 + s->o_h[k];
    double value = 0.;
    for (uint64_t t = 0; t < n; t++) value += v[t] * dotsrc[t];
    for (uint64_t t = 0; t < n; t++) d[t] = 0.5 * value * scalesrc[t];
  }
}

/* calc.cpp:264-339: Y = V_hphp + 0.5 V_hpph T_phhp;  R = T_phhp Y. */
void oracle_calc_t2diff_phhp(oracle_state *s) {
#pragma omp parallel for schedule(dynamic)
  for (int64_t ci = 0; ci < (int64_t)s->nch; ci++) {
    uint64_t c = (uint64_t)ci;
    uint64_t ph = s->p->chan_mod_dims[c].ph, hp = s->p->chan_mod_dims[c].hp;
    if (!ph || !hp) continue;
    double *y = (double *)malloc(hp * hp * 8);
    memcpy(y, s->p->v_hphp_mod[c], hp * hp * 8);
    const double *t = s->old_phhp + s->o_m[c];
    gemm(hp, hp, ph, 0.5, s->p->v_hpph_mod[c], t, 1.0, y);
    gemm(ph, hp, hp, 1.0, t, y, 0.0, s->diff_phhp + s->o_m[c]);
    free(y);
  }
}

/* calc.cpp:132-231: X = V_hhhh + 0.5 V_hhpp T;  D = 0.5 T X;  D += 0.5 V_pppp T. */
void oracle_calc_t2diff_pphh(oracle_state *s) {
#pragma omp parallel for schedule(dynamic)
  for (int64_t ci = 0; ci < (int64_t)s->nch; ci++) {
    uint64_t c = (uint64_t)ci;
    uint64_t pp = s->p->chan_dims[c].pp, hh = s->p->chan_dims[c].hh;
    if (!pp || !hh) continue;
    double *x = (double *)malloc(hh * hh * 8);
    memcpy(x, s->p->v_hhhh[c], hh * hh * 8);
    const double *t = s->t2_old + s->o_t[c];
    double *d = s->diff_pphh + s->o_t[c];
    gemm(hh, hh, pp, 0.5, s->p->v_hhpp[c], t, 1.0, x);
    gemm(pp, hh, hh, 0.5, t, x, 0.0, d);
    gemm(pp, hh, pp, 0.5, s->p->v_pppp[c], t, 1.0, d);
    free(x);
  }
}

/* The eight gathers of main.cpp:632-639: out[e] = source[table[e]]. */
void oracle_map_from_distributed(oracle_state *s) {
  const double *src[8] = {s->diff_h2pp_h1, s->diff_h2pp_h1, s->diff_p2_p1hh, s->diff_p2_p1hh,
                          s->diff_phhp, s->diff_phhp, s->diff_phhp, s->diff_phhp};
  for (int k = 0; k < 8; k++) {
#pragma omp parallel for
    for (int64_t e = 0; e < (int64_t)s->n_t; e++) s->gath[k][e] = src[k][s->flat[k][e]];
  }
}

/* calc.cpp:368-459: combine, divide by the denominator, mix, energy. */
double oracle_calc_t2_pphh(oracle_state *s, double mixing) {
  double *corr_c = (double *)calloc(s->nch + 1, 8);
  const double *eps = s->p->sp_energy;
#pragma omp parallel for schedule(dynamic)
  for (int64_t ci = 0; ci < (int64_t)s->nch; ci++) {
    uint64_t c = (uint64_t)ci;
    uint64_t pp = s->p->chan_dims[c].pp, hh = s->p->chan_dims[c].hh;
    if (!pp || !hh) continue;
    const double *v = s->p->v_hhpp[c];
    const ccdgpu_pair *P = s->p->chan_maps[c].pp, *H = s->p->chan_maps[c].hh;
    double corr = 0.;
    for (uint64_t AB = 0; AB < pp; AB++)
      for (uint64_t IJ = 0; IJ < hh; IJ++) {
        uint64_t e = s->o_t[c] + AB * hh + IJ;
        uint64_t a = P[AB].p, b = P[AB].q, i = H[IJ].p, j = H[IJ].q;
        double value = v[IJ * pp + AB];
        value += s->diff_pphh[e];
        value += s->gath[CCDGPU_MAP_AI_JB][e];
        value -= s->gath[CCDGPU_MAP_AJ_IB][e];
        value -= s->gath[CCDGPU_MAP_BI_JA][e];
        value += s->gath[CCDGPU_MAP_BJ_IA][e];
        value += s->gath[CCDGPU_MAP_JAB_I][e];
        value -= s->gath[CCDGPU_MAP_IAB_J][e];
        value += s->gath[CCDGPU_MAP_B_AIJ][e];
        value -= s->gath[CCDGPU_MAP_A_BIJ][e];
        value = value / (eps[i] + eps[j] - eps[a] - eps[b]);
        value = mixing * value + (1. - mixing) * s->t2_old[e];
        s->t2[e] = value;
        corr += v[IJ * pp + AB] * s->t2[e];
      }
    corr_c[c] = 0.25 * corr;
  }
  double corr = 0.;
  for (uint64_t c = 0; c < s->nch; c++) corr += corr_c[c];
  free(corr_c);
  return corr;
}

/* Chain::set (t2Old <- t2) and the five scatters of main.cpp:660-665. */
void oracle_map_to_distributed(oracle_state *s) {
  memcpy(s->t2_old, s->t2, s->n_t * 8);
  double *dst[5] = {s->old_h2pp_h1, s->old_h1pp_h2, s->old_p1_p2hh, s->old_p2_p1hh, s->old_phhp};
  const int tab[5] = {CCDGPU_MAP_JAB_I, CCDGPU_MAP_IAB_J, CCDGPU_MAP_A_BIJ, CCDGPU_MAP_B_AIJ,
                      CCDGPU_MAP_AI_JB};
  for (int k = 0; k < 5; k++) {
#pragma omp parallel for
    for (int64_t e = 0; e < (int64_t)s->n_t; e++) dst[k][s->flat[tab[k]][e]] = s->t2[e];
  }
}

double oracle_step(oracle_state *s, double mixing) {
  oracle_calc_t2diff_p2_p1hh(s);
  oracle_calc_t2diff_h2pp_h1(s);
  oracle_calc_t2diff_phhp(s);
  oracle_calc_t2diff_pphh(s);
  oracle_map_from_distributed(s);
  double corr = oracle_calc_t2_pphh(s, mixing);
  oracle_map_to_distributed(s);
  return corr;
}

void oracle_reset(oracle_state *s) {
  memset(s->t2, 0, s->n_t * 8);
  memset(s->t2_old, 0, s->n_t * 8);
  memset(s->old_phhp, 0, s->n_m * 8);
  memset(s->old_h1pp_h2, 0, s->n_h * 8);
  memset(s->old_h2pp_h1, 0, s->n_h * 8);
  memset(s->old_p1_p2hh, 0, s->n_p * 8);
  memset(s->old_p2_p1hh, 0, s->n_p * 8);
}

/* Loads T2 as if it had just been produced by calcT2_pphh (then set + scatters). */
void oracle_set_t2(oracle_state *s, const double *t2) {
  memcpy(s->t2, t2, s->n_t * 8);
  oracle_map_to_distributed(s);
}

void oracle_get_t2(const oracle_state *s, double *out) { memcpy(out, s->t2, s->n_t * 8); }

/* Returns the iteration count; energies[k] = corrCCD after iteration k (capacity max_iters+2). */
int64_t oracle_solve(oracle_state *s, double tol, int64_t max_iters, double mixing,
                     double *energies, double *e_corr) {
  double diff = 1.0, corr = 100.0, prev = 100.0;
  int64_t it = 0;
  while (fabs(diff) > tol) {
    if (it > max_iters) break;
    corr = oracle_step(s, mixing);
    diff = corr - prev;
    prev = corr;
    if (energies) energies[it] = corr;
    it++;
  }
  if (e_corr) *e_corr = corr;
  return it;
}

/* Reads one chain (ccdgpu_chain_id numbering); returns its length. */
uint64_t oracle_read_chain(const oracle_state *s, int chain, double *out) {
  const double *src = NULL;
  uint64_t n = 0;
  switch (chain) {
    case CCDGPU_CHAIN_T2: src = s->t2; n = s->n_t; break;
    case CCDGPU_CHAIN_T2_OLD: src = s->t2_old; n = s->n_t; break;
    case CCDGPU_CHAIN_DIFF_PPHH: src = s->diff_pphh; n = s->n_t; break;
    case CCDGPU_CHAIN_DIFF_PHHP: src = s->diff_phhp; n = s->n_m; break;
    case CCDGPU_CHAIN_OLD_PHHP: src = s->old_phhp; n = s->n_m; break;
    case CCDGPU_CHAIN_DIFF_H2PP_H1: src = s->diff_h2pp_h1; n = s->n_h; break;
    case CCDGPU_CHAIN_DIFF_P2_P1HH: src = s->diff_p2_p1hh; n = s->n_p; break;
    default:
      if (chain >= CCDGPU_CHAIN_GATHERED0 && chain < CCDGPU_CHAIN_GATHERED0 + 8) {
        src = s->gath[chain - CCDGPU_CHAIN_GATHERED0];
        n = s->n_t;
      }
  }
  if (src && out) memcpy(out, src, n * 8);
  return n;
}

/* FNV-1a 64-bit over raw bytes: the hash the golden dumps carry for V blocks. */
uint64_t oracle_fnv1a(const void *data, uint64_t n) {
  const unsigned char *p = (const unsigned char *)data;
  uint64_t h = 1469598103934665603ULL;
  for (uint64_t i = 0; i < n; i++) {
    h ^= p[i];
    h *= 1099511628211ULL;
  }
  return h;
}
