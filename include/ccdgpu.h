/* ccdgpu — B200-native Coupled-Cluster-Doubles T2 iteration behind a C ABI.
 *
 * Drop-in for the CCD fixed-point loop that the reference driver runs in main.cpp:491-682:
 * the four calc.cpp stages (calcT2Diff_p2_p1hh, calcT2Diff_h2pp_h1, calcT2Diff_phhp,
 * calcT2Diff_pphh), the eight Chain::mapFromDistributed gathers, calcT2_pphh (denominator,
 * mixing, energy) and the Chain::set + five Chain::mapToDistributed scatters.  The host keeps
 * the basis, channel construction, V loaders and loadMaps; it hands their outputs to
 * ccdgpu_create() through plain pointers, in the reference's own memory layouts:
 *
 *   ccdgpu_pair            == PQBundle              (SPBasis.hpp:32-44)
 *   ccdgpu_triple          == PQRBundle             (SPBasis.hpp:46-63)
 *   ccdgpu_channel_dims    == ChannelDims           (SPBasis.hpp:69-74)
 *   ccdgpu_channel_maps    == ChannelMaps           (SPBasis.hpp:80-86)
 *   ccdgpu_three_body_dims == ThreeBodyChannelDims  (SPBasis.hpp:88-91)
 *   ccdgpu_chain_index     == ChainIndex            (Chain.hpp:7-11)
 *   V and map blocks       == Chain<T>::get(channel) block pointers (Chain.hpp:108-120),
 *                             dense row-major, NULL for empty blocks.
 *
 * Every entry point returns CCDGPU_OK (0) or a negative ccdgpu_status; none exits, traps or
 * prints.  A handle owns one CUDA stream and its device memory; it is not thread-safe.
 * All sizes are 64-bit.  T2 on the host is in the reference's t2_pphh data order: channel
 * blocks in channel order, each pp x hh row-major, empty channels contributing nothing.
 */
#ifndef CCDGPU_H
#define CCDGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ccdgpu_pair { uint64_t p, q; } ccdgpu_pair;
typedef struct ccdgpu_triple { uint64_t p, q, r; } ccdgpu_triple;
typedef struct ccdgpu_channel_dims { uint64_t pp, hh, hp, ph; } ccdgpu_channel_dims;
typedef struct ccdgpu_channel_maps {
  const ccdgpu_pair *pp, *hh, *hp, *ph;
} ccdgpu_channel_maps;
typedef struct ccdgpu_three_body_dims { uint64_t phh, hpp; } ccdgpu_three_body_dims;
typedef struct ccdgpu_chain_index { uint64_t channel, row, column; } ccdgpu_chain_index;

/* Order of the eight remap tables of loadMaps (load.cpp:391-398, main.cpp:236-243). */
enum ccdgpu_map_id {
  CCDGPU_MAP_IAB_J = 0, /* map_pphh_iab_j_hpp_h */
  CCDGPU_MAP_JAB_I = 1, /* map_pphh_jab_i_hpp_h */
  CCDGPU_MAP_A_BIJ = 2, /* map_pphh_a_bij_p_phh */
  CCDGPU_MAP_B_AIJ = 3, /* map_pphh_b_aij_p_phh */
  CCDGPU_MAP_AI_JB = 4, /* map_pphh_ai_jb_phhp  */
  CCDGPU_MAP_AJ_IB = 5, /* map_pphh_aj_ib_phhp  */
  CCDGPU_MAP_BI_JA = 6, /* map_pphh_bi_ja_phhp  */
  CCDGPU_MAP_BJ_IA = 7  /* map_pphh_bj_ia_phhp  */
};

/* Interaction model, for generating V_pppp blocks on the device instead of uploading them
 * (the reference's saveMemory mode regenerates blocks through SPBasis::calcTBME,
 * calc.cpp:233-262, load.cpp:220-239). */
enum ccdgpu_model_kind {
  CCDGPU_MODEL_NONE = 0,
  CCDGPU_MODEL_PAIRING = 1,       /* PairingSPBasis::calcTBME, PairingSPBasis.cpp:127-141 */
  CCDGPU_MODEL_INF_MATTER = 2,    /* Minnesota, InfMatterSPBasis.cpp:361-437 */
  CCDGPU_MODEL_ELECTRON_GAS = 3   /* Coulomb, ElectronGasSPBasis.cpp:424-471 */
};
typedef struct ccdgpu_model {
  int32_t kind;                 /* ccdgpu_model_kind */
  int32_t qn_stride;            /* ints per orbital in qn (5 for plane waves, 2 for pairing) */
  const int32_t *qn;            /* [n_sp * qn_stride]: SPBasis::indexMap rows */
  double params[8];             /* EG: {L, e_sq}; PNM: {L}; pairing: {g} */
} ccdgpu_model;

/* Channel numbering of a basis (the inputs of SPBasis::setUpChannelDims / setUpChannelMaps,
 * SPBasis.cpp:80-441): orbital quantum numbers and the channel index rule of the model. */
typedef struct ccdgpu_channel_rule {
  int32_t kind;                 /* ccdgpu_model_kind */
  int32_t qn_stride;            /* ints per orbital in qn (5 for plane waves, 2 for pairing) */
  const int32_t *qn;            /* [n_sp * qn_stride]: SPBasis::indexMap rows */
  uint64_t n_sp, n_particles;   /* orbitals; the first n_particles are holes */
  uint64_t n_channels;          /* channel slots (SPBasis::nChannels) */
  int32_t nmax;                 /* largest |n_x|, |n_y|, |n_z| of the basis (plane waves) */
  int32_t chan_tz_max;          /* T_z rule of regular channels (-2: one T_z, 2: three) */
  int32_t mod_chan_tz_max;      /* T_z rule of modified channels (0: one T_z, 2: three) */
  int32_t device;               /* CUDA device, < 0: the calling thread's current device */
} ccdgpu_channel_rule;

typedef struct ccdgpu_problem {
  uint64_t n_sp;                /* SPBasis::nSpstates; orbitals < n_particles are holes */
  uint64_t n_particles;         /* SPBasis::nParticles */
  uint64_t n_channels;          /* SPBasis::nChannels (regular and modified channel slots) */
  const double *sp_energy;      /* [n_sp] normal-ordered energies (after rotateSpEnergiesToNormalOrdered) */
  const ccdgpu_channel_dims *chan_dims;        /* [n_channels] regular channels, permuted order */
  const ccdgpu_channel_dims *chan_mod_dims;    /* [n_channels] modified (ph') channels */
  const ccdgpu_channel_maps *chan_maps;        /* [n_channels] pp and hh maps are read */
  const ccdgpu_channel_maps *chan_mod_maps;    /* [n_channels] ph and hp maps are read */
  const ccdgpu_three_body_dims *three_body_dims; /* [n_sp] hpp for holes, phh for particles */
  /* V blocks.  v_hhhh, v_hhpp, v_hpph_mod and v_hphp_mod may be NULL together when a model is
   * given: ccdgpu_create then generates them on the device (load.cpp:112-318 elements). */
  const double *const *v_hhhh;      /* [n_channels] hh x hh  (vnn_hhhh) */
  const double *const *v_hhpp;      /* [n_channels] hh x pp  (vnn_hhpp) */
  const double *const *v_pppp;      /* [n_channels] pp x pp  (vnn_pppp); may be NULL if model given */
  const double *const *v_hpph_mod;  /* [n_channels] hp' x ph' (vnn_hhpp_hpph_mod) */
  const double *const *v_hphp_mod;  /* [n_channels] hp' x hp' (vnn_hpph_hphp_mod) */
  const double *const *v_h_hpp;     /* [n_particles] 1 x hpp  (vnn_h_hpp); NULL allowed (fused path) */
  const double *const *v_phh_p;     /* [n_sp - n_particles] phh x 1 (vnn_phh_p); NULL allowed */
  const ccdgpu_chain_index *const *maps[8]; /* [n_channels] pp x hh blocks, ccdgpu_map_id order
                                               (loadMaps, load.cpp:389-532); all eight NULL:
                                               derived on the device from chan_maps (pp, hh),
                                               chan_mod_maps (ph, hp) and three_body_dims */
  const ccdgpu_model *model;        /* optional, required for CCDGPU_V_ON_THE_FLY */
} ccdgpu_problem;

enum ccdgpu_status {
  CCDGPU_OK = 0,
  CCDGPU_ERR_INVALID_ARGUMENT = -1,
  CCDGPU_ERR_CUDA = -2,
  CCDGPU_ERR_OUT_OF_MEMORY = -3,
  CCDGPU_ERR_BAD_TABLE = -4,       /* a remap table entry is out of range or not a bijection */
  CCDGPU_ERR_NONFINITE = -5,       /* NaN/Inf in the amplitudes or the energy */
  CCDGPU_ERR_NO_DEVICE = -6,
  CCDGPU_ERR_UNSUPPORTED = -7,
  CCDGPU_ERR_NOT_CONVERGED = -8,   /* only from ccdgpu_solve when require_convergence is set */
  CCDGPU_ERR_TIMEOUT = -9          /* a bounded device-side wait (an mbarrier of a pipelined
                                      kernel) ran out (1 s of %globaltimer); the kernel stopped
                                      cleanly and the handle stays usable */
};

enum ccdgpu_precision {
  CCDGPU_PREC_FP64 = 0,        /* FP64 throughout: FP64 tensor-core MMA (mma.sync f64) for
                                  the mid/wide pp-ladder classes, the hh ladder and the ring,
                                  FP64 FMA for the thinnest pp-ladder channels */
  CCDGPU_PREC_MIXED_BF16 = 1,  /* pp ladder on tensor cores with 2-term bf16 split operands,
                                  FP32 accumulation; FP64 polish iterations at the end */
  CCDGPU_PREC_MIXED_BF16X3 = 2 /* the same with 3-term bf16 split operands */
};
enum ccdgpu_v_mode {
  CCDGPU_V_STORED = 0,         /* V_pppp uploaded from the host blocks */
  CCDGPU_V_ON_THE_FLY = 1,     /* V_pppp generated on the device from the model
                                  (ccdgpu_problem.model) instead of uploaded: once, at create,
                                  into the FP64 ladder tiles and bf16 images */
  CCDGPU_V_IN_LADDER = 2       /* as CCDGPU_V_ON_THE_FLY, and for the electron gas with a mixed
                                  precision the tensor-core ladder regenerates its V operand
                                  every iteration instead of reading bf16 images (less device
                                  memory; slower than streaming the images on B200) */
};
enum ccdgpu_path {
  CCDGPU_PATH_FUSED = 0,       /* fused kernels: one-body terms from the ladder intermediates,
                                  remaps folded into the assembly kernel */
  CCDGPU_PATH_TABLES = 1       /* stage by stage exactly as main.cpp:591-665: 8 gathers and
                                  5 scatters through the loadMaps tables */
};

typedef struct ccdgpu_options {
  int32_t device;              /* CUDA device ordinal */
  int32_t precision;           /* ccdgpu_precision */
  int32_t v_mode;              /* ccdgpu_v_mode */
  int32_t path;                /* ccdgpu_path */
  double polish_threshold;     /* mixed: switch to FP64 iterations once |dE| <= max(tol,
                                  polish_threshold * |E|) or |dE| stops decreasing */
  int32_t use_graph;           /* capture one iteration as a CUDA graph (fused path) */
  int32_t device_loop;         /* with use_graph: run the whole solve loop on the device (graph
                                  WHILE nodes, default 1); 0 replays per-iteration graphs in
                                  batches (profilers cannot see kernels inside WHILE nodes) */
  int32_t reserved[6];
} ccdgpu_options;

typedef struct ccdgpu_result {
  double e_corr;               /* correlation energy after the last iteration (corrCCD) */
  double e_diff;               /* last energy change (energyDiff) */
  int64_t iterations;          /* iterations performed, counted as main.cpp:681 does */
  int32_t converged;           /* 1 when |e_diff| <= tolerance, 0 when the cap was hit */
  int32_t polish_iterations;   /* mixed precision: iterations run in FP64 polish */
  double seconds;              /* wall time of the loop (cc_diagrams_time counterpart) */
} ccdgpu_result;

typedef struct ccdgpu_handle ccdgpu_handle;

/* Defaults: device 0, FP64, stored V, fused path, graph capture on, polish 1e-6. */
void ccdgpu_default_options(ccdgpu_options *opt);

/* Deep-copies the problem to the device and validates every remap table (range and
 * bijection).  Replaces main.cpp:222-455 allocation/loading as far as the device is
 * concerned; the host data may be freed afterwards.  T2 starts at zero (main.cpp:497-503). */
int ccdgpu_create(const ccdgpu_problem *prob, const ccdgpu_options *opt, ccdgpu_handle **out);
void ccdgpu_destroy(ccdgpu_handle *h);
/* Device memory of destroyed handles stays in a process-wide cache (at most 16 GiB) and is
 * reused by later handles on the same device, so that repeated create/destroy cycles do not
 * call cudaMalloc/cudaFree.  This returns the cached memory to the device. */
void ccdgpu_release_cached_memory(void);
const char *ccdgpu_strerror(int status);

/* Zero every amplitude chain (main.cpp:497-503). */
int ccdgpu_reset(ccdgpu_handle *h);
/* Load / read T2 in t2_pphh order (n = sum of pp*hh).  Loading also refreshes t2Old and
 * the scattered layouts, as main.cpp:660-665 would after an iteration. */
int ccdgpu_set_t2(ccdgpu_handle *h, const double *t2_pphh, uint64_t n);
int ccdgpu_get_t2(ccdgpu_handle *h, double *t2_pphh, uint64_t n);
/* Second-order energy on the device, the reference's MBPT2 (MBPT2Corr.cpp:6-38):
 * E_MBPT2 = 1/4 sum_{abij} |<ij|v|ab>|^2 / (e_i + e_j - e_a - e_b) from the handle's V_hhpp and
 * single-particle energies (deterministic compensated sum).  init_t2 != 0 also makes the
 * first-order amplitudes t_ab,ij = <ab|v|ij> / (e_i + e_j - e_a - e_b) the current T2 (an
 * alternative start to the reference's T2 = 0, main.cpp:497-503). */
int ccdgpu_mbpt2(ccdgpu_handle *h, int32_t init_t2, double *e_mbpt2);
/* Reference energy and normal ordering on the device (SPBasis.cpp:7-40, referenceEnergy and
 * rotateSpEnergiesToNormalOrdered, called at main.cpp:64-67): from the bare single-particle
 * energies sp_energy_bare[n_sp] and the problem's interaction model,
 *   E_ref = sum_{i,j<A} 1/2 <ij|v|ij> + sum_{i<A} e_i,   e'_p = e_p + sum_{j<A} <pj|v|pj>,
 * each summed in the reference's order.  Writes E_ref to *e_ref and, when sp_energy_normal is
 * not NULL, the n_sp normal-ordered energies.  Needs ccdgpu_problem.model at create
 * (CCDGPU_ERR_UNSUPPORTED without it); the handle's own energies are not changed. */
int ccdgpu_reference_energy(ccdgpu_handle *h, const double *sp_energy_bare, double *e_ref,
                            double *sp_energy_normal);
/* Channel construction on the device (SPBasis.cpp:80-441 with the one-rank ffdBalance order of
 * main.cpp:94-115 and balance.cpp:91-144): the regular and modified channel dimensions in
 * permuted order and their pair lists, each sorted by (p, q), for every ordered orbital pair.
 * lists[k] / mod_lists[k] hold kind k = pp, hh, hp, ph for all channels one after another in
 * permuted order: npart^2, A^2, A*npart and npart*A pairs (A = n_particles, npart = n_sp - A).
 * chan / mod_chan / pos / mod_pos (optional, n_sp^2 each, index p * n_sp + q) receive the
 * permuted channel of every pair and its index inside its channel's list.  Returns
 * CCDGPU_ERR_UNSUPPORTED when one channel holds more than 8192 pairs of one kind or n_sp^2
 * does not fit 32 bits. */
int ccdgpu_build_channels(const ccdgpu_channel_rule *rule, ccdgpu_channel_dims *dims,
                          ccdgpu_channel_dims *mod_dims, ccdgpu_pair *const lists[4],
                          ccdgpu_pair *const mod_lists[4], uint32_t *chan, uint32_t *mod_chan,
                          uint32_t *pos, uint32_t *mod_pos);
uint64_t ccdgpu_t2_size(const ccdgpu_handle *h);

/* One CCD iteration (main.cpp:589-670) with the path and precision chosen at create time.
 * Writes the new correlation energy (corrCCD) to *e_corr. */
int ccdgpu_step(ccdgpu_handle *h, double mixing, double *e_corr);

/* Iterate from the current T2 until |E - E_prev| <= tol or iterations exceed max_iters,
 * with E_prev starting at 100 (main.cpp:491-519).  max_iters = 100 reproduces the
 * reference's cap (at most 101 iterations). */
int ccdgpu_solve(ccdgpu_handle *h, double tol, int64_t max_iters, double mixing,
                 ccdgpu_result *res);

/* No counterpart in the reference (its runs are one system per process).  Solves n
 * independent systems together: each handle's iteration loop runs on its own device streams
 * and all of them are in flight at once, so the kernels of small systems share the GPU.  Same
 * stop rule and results as n calls of ccdgpu_solve; res[i] is handle i's result, filled also
 * for a handle whose solve failed (e_corr non-finite for a diverging iteration).  Handles must
 * be distinct; returns the first error, after finishing the solves that started. */
int ccdgpu_solve_batch(ccdgpu_handle *const *handles, int32_t n, double tol, int64_t max_iters,
                       double mixing, ccdgpu_result *res);

/* corrCCD after each iteration of the last ccdgpu_solve (first 128 iterations); *n_out gets
 * the number of iterations stored.  The per-iteration printout of main.cpp:672-680. */
int ccdgpu_energy_history(ccdgpu_handle *h, double *out, int64_t cap, int64_t *n_out);

/* Stage entry points with the reference's names, for stage-level parity tests and for a
 * host that keeps the reference loop structure.  They act on the handle's device chains.  The
 * one-body stages need the three-body V blocks (v_h_hpp, v_phh_p): given by the problem, or
 * generated on the device for a handle of the table path; otherwise they return
 * CCDGPU_ERR_UNSUPPORTED. */
int ccdgpu_calc_t2diff_p2_p1hh(ccdgpu_handle *h);   /* calc.cpp:27-43 */
int ccdgpu_calc_t2diff_h2pp_h1(ccdgpu_handle *h);   /* calc.cpp:91-107 */
int ccdgpu_calc_t2diff_phhp(ccdgpu_handle *h);      /* calc.cpp:315-339 */
int ccdgpu_calc_t2diff_pphh(ccdgpu_handle *h);      /* calc.cpp:205-231 */
int ccdgpu_map_from_distributed(ccdgpu_handle *h);  /* the 8 gathers, main.cpp:632-639 */
int ccdgpu_calc_t2_pphh(ccdgpu_handle *h, double mixing, double *corr); /* calc.cpp:423-459 */
int ccdgpu_map_to_distributed(ccdgpu_handle *h);    /* Chain::set + 5 scatters, main.cpp:660-665 */

/* Chain identifiers for ccdgpu_read_chain (device intermediates, copied to the host). */
enum ccdgpu_chain_id {
  CCDGPU_CHAIN_T2 = 0,          /* t2_pphh          (pp x hh) */
  CCDGPU_CHAIN_T2_OLD = 1,      /* t2Old_pphh       (pp x hh) */
  CCDGPU_CHAIN_DIFF_PPHH = 2,   /* t2Diff_pphh      (pp x hh) */
  CCDGPU_CHAIN_DIFF_PHHP = 3,   /* t2Diff_phhp      (ph' x hp') */
  CCDGPU_CHAIN_OLD_PHHP = 4,    /* t2Old_phhp       (ph' x hp') */
  CCDGPU_CHAIN_DIFF_H2PP_H1 = 5,/* t2Diff_h2pp_h1   (hpp x 1, per hole) */
  CCDGPU_CHAIN_DIFF_P2_P1HH = 6,/* t2Diff_p2_p1hh   (1 x phh, per particle) */
  CCDGPU_CHAIN_GATHERED0 = 8    /* + k: the k-th gathered pphh chain, ccdgpu_map_id order */
};
/* Copies a device chain into out (n doubles); returns its length through *n_out when out is
 * NULL. */
int ccdgpu_read_chain(ccdgpu_handle *h, int32_t chain, double *out, uint64_t n, uint64_t *n_out);

/* Device timing of the last ccdgpu_solve / ccdgpu_step, per kernel family, in
 * milliseconds summed over the iterations, and launch counts. */
typedef struct ccdgpu_profile {
  double ms_ladder;      /* pp ladder + T X GEMM (calc.cpp:162-202) */
  double ms_hh_ladder;   /* hh ladder intermediate X (calc.cpp:141-160) */
  double ms_ring;        /* ring GEMMs (calc.cpp:264-313), on the second stream */
  double ms_onebody;     /* one-body terms (calc.cpp:9-25, 73-89) */
  double ms_assemble;    /* assembly + remaps + energy (calc.cpp:368-421, Chain.hpp:710-802) */
  double ms_total;       /* whole iterations */
  int64_t launches;      /* kernels launched by this library since create */
  int64_t iterations;    /* iterations covered by the ms_* sums */
  /* Host wall time of ccdgpu_create by phase: [0] per-channel metadata and work lists on the
   * host, [1] device allocation and uploads, [2] device set-up kernels (tables, V, operand
   * images) from their launch until they finish, [3] kernel attributes, ladder schedules and
   * the device-loop graph's capture, host work done while the set-up kernels run (so [3] is
   * part of [2]), [4] the whole call. */
  double ms_create[5];
  double ms_loop_graph;  /* host time of building the device solve loop's graph (capture and
                            instantiation; in ccdgpu_create, or on the first device-loop solve
                            after a schedule change) */
} ccdgpu_profile;
int ccdgpu_get_profile(ccdgpu_handle *h, ccdgpu_profile *prof);
/* When on, ccdgpu_solve runs the fused iteration without graph capture and brackets each
 * kernel family with CUDA events on the handle's streams (one host sync per iteration). */
int ccdgpu_enable_profiling(ccdgpu_handle *h, int32_t on);
/* The handle's main CUDA stream (cudaStream_t), for callers that time or order work on it. */
void *ccdgpu_stream(ccdgpu_handle *h);

/* Failure-path test hook; no counterpart in the reference.  Arms a fault for the next
 * ccdgpu_step only: in that iteration the first CTA of every FP64 pp-ladder class withholds
 * its first shared-memory stage, so its bounded mbarrier waits run out after 1 s; the kernel
 * stops cleanly and ccdgpu_step returns CCDGPU_ERR_TIMEOUT.  The handle stays usable (the
 * error is reported once), but that iteration's amplitudes are incomplete: call ccdgpu_reset
 * or ccdgpu_set_t2 before iterating on.  Affects only iterations that run the FP64 ladder. */
int ccdgpu_inject_wait_timeout(ccdgpu_handle *h);

/* Work of one iteration for roofline reporting: *flops = reference GEMM flops (sum over
 * channels of 2 pp^2 hh + 4 pp hh^2 + 4 ph' hp'^2); *ladder_bytes = bytes one pp-ladder launch
 * moves (antisymmetry-packed V_pppp, the T and X operands, D) at the handle's precision (FP64
 * operands, or the bf16 terms of a mixed handle); *ladder_flops = the pp-ladder share of the
 * reference flops (2 pp^2 hh). */
int ccdgpu_work_per_iteration(const ccdgpu_handle *h, double *flops, double *ladder_bytes,
                              double *ladder_flops);

/* pp-ladder schedule (no counterpart in the reference): how far the K dimension of each
 * channel block is split into deterministic partial sums, as a target of tiles per SM for the
 * FP64 thin class (hh <= 8), the FP64 mid/wide classes, and the tensor-core ladder. */
typedef struct ccdgpu_schedule {
  int32_t thin_split_mul;      /* default 1 */
  int32_t wide_split_mul;      /* default 3: FP64 wide class (nb > 32; also mid when mid is 0) */
  int32_t tc_split_mul;        /* default 2 */
  int32_t mid_split_mul;       /* default 0 = as wide_split_mul: FP64 mid class (nb 16..32) */
  int32_t reserved[4];
} ccdgpu_schedule;
int ccdgpu_set_schedule(ccdgpu_handle *h, const ccdgpu_schedule *sch);
int ccdgpu_get_schedule(const ccdgpu_handle *h, ccdgpu_schedule *sch);
/* Autotuner: times `reps` launches of the pp ladders for every candidate schedule on this GPU
 * and this problem (CUDA events), keeps the fastest and returns it with its times (ms per
 * ladder launch, FP64 and tensor-core).  Amplitudes are not changed. */
int ccdgpu_autotune(ccdgpu_handle *h, int32_t reps, ccdgpu_schedule *chosen, double *ms_fp64,
                    double *ms_tc);

/* Each pp-ladder class launched alone, reps times (CUDA events): ms, executed flops (packed:
 * rows a<=b, K over c<d and hh) and algorithmic bytes per launch, indexed FP64 thin (hh <= 8),
 * FP64 mid (nb 16..32), FP64 wide (nb 40..72, the largest channels), tensor-core ladder
 * (mixed handles).  Amplitudes are not changed.  No counterpart in the reference. */
int ccdgpu_ladder_profile(ccdgpu_handle *h, int32_t reps, double ms[4], double flops[4],
                          double bytes[4]);

/* The other kernels of an iteration, each class launched alone `reps` times on the handle's
 * stream (after one warm-up launch): average ms per launch, FP64 flops and algorithmic bytes
 * per launch, indexed ring small (ph', hp' <= 16; with the phhp gather that precedes the ring
 * on the fused path), ring mid (<= 32), ring large, hh ladder
 * small (hh <= 16), hh ladder rest, one-body sums, hh-ladder slice reduction.  Amplitudes are
 * not changed (the kernels write only intermediates).  No counterpart in the reference. */
int ccdgpu_kernel_profile(ccdgpu_handle *h, int32_t reps, double ms[7], double flops[7],
                          double bytes[7]);

/* Kernel start-time trace (diagnostics; no counterpart in the reference).  Arm with the index
 * of an iteration of the next solve (-1 disarms); every kernel of that iteration then records
 * the %globaltimer time (ns) at which its first and its last CTA started.  Kernel ids, in this
 * order: ring small, ring mid, ring large, hh ladder small, hh ladder tiled, one-body, pp
 * ladder thin, mid, wide, tensor-core pp ladder, assembly, loop control, energy, FP64 tile
 * refresh, split-K reduction, hh-ladder reduction, phhp gather (17). */
int ccdgpu_trace_arm(ccdgpu_handle *h, int64_t iteration);
int ccdgpu_trace_read(ccdgpu_handle *h, uint64_t *first, uint64_t *last, int32_t n);
/* The same trace: when the last CTA of each kernel finished (%globaltimer ns; 0 for kernels
 * that do not record it: the loop control, energy and FP64 tile refresh kernels). */
int ccdgpu_trace_read_end(ccdgpu_handle *h, uint64_t *end, int32_t n);

/* No counterpart in the reference.  The ladder term of one regular channel,
 *   D = 0.5 T X + 0.5 V_pppp T   with   X = V_hhhh + 0.5 V_hhpp T,
 * for callers that cannot allocate device memory, such as a host that owns all device memory
 * through its own pool or budget.  Nothing is allocated: every argument is a caller-provided
 * device buffer (row-major: v_pppp pp x pp, v_hhpp hh x pp, v_hhhh hh x hh, t2 pp x hh,
 * d pp x hh), and the intermediate X with its split-K partial sums lives in a fixed 2 MiB
 * scratch array built into the library (one per GPU that loads it, kept until the process
 * exits).  Limits: hh <= 72 and 32 + (ceil(pp/64) + 1) * hh^2 <= 262144 doubles; larger sizes
 * return CCDGPU_ERR_UNSUPPORTED without launching anything.  Work is enqueued on `stream`
 * (a cudaStream_t; NULL = legacy default stream) for the current device.  The first call on a
 * device looks up the scratch address (cudaGetSymbolAddress) and sets a kernel attribute; make
 * that first call before any stream capture.  Both are remembered for the life of the process,
 * so cudaDeviceReset after the first call is not supported.  Every call shares the one scratch
 * array, which keeps the last call's contents: calls whose work overlaps on the GPU (different
 * streams without ordering) race and must not be issued. */
int ccdgpu_calc_channel_t2diff_pphh_noalloc(const double *v_pppp, const double *v_hhpp,
                                            const double *v_hhhh, const double *t2, double *d,
                                            int64_t pp, int64_t hh, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CCDGPU_H */
