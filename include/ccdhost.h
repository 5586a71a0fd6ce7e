/* ccdhost — host-side CCD problem builder that produces a ccdgpu_problem.
 *
 * This is the input side of the drop-in boundary: the reference keeps its own host
 * (SPBasis subclasses, channel construction, loadVnn_*, loadMaps) and fills a
 * ccdgpu_problem from it.  Where the reference is not present (tests, benchmarks, the GPU
 * box), this library builds the same problem from the reference's model parameters, with
 * the same orbital order, the same 1-rank ffdBalance channel permutation, the same sorted
 * channel maps and remap tables (bit-exact), and the same matrix-element arithmetic:
 *
 *   orbitals / energies   ElectronGasSPBasis.cpp:14-210, InfMatterSPBasis.cpp:13-184,
 *                         PairingSPBasis.cpp:14-58
 *   E_ref, normal order   SPBasis.cpp:7-40
 *   channels, maps        SPBasis.cpp:80-819, balance.cpp:91-144, main.cpp:94-136
 *   V blocks              load.cpp:112-318 with the models' calcTBME
 *   remap tables          load.cpp:389-532
 *   MBPT2                 MBPT2Corr.cpp:6-38
 *
 * Only channels that carry amplitudes get V blocks (pp*hh > 0 for regular channels,
 * ph'*hp' > 0 for modified ones); other block pointers are NULL.  Returns 0 or a negative
 * ccdgpu_status.
 */
#ifndef CCDHOST_H
#define CCDHOST_H

#include "ccdgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ccdhost_system ccdhost_system;

/* Build flags (the last int32 argument of the ccdhost_build_* functions). */
enum ccdhost_flags {
  CCDHOST_LOAD_V_PPPP = 1, /* build and pass V_pppp (off: the solver generates it, saveMemory) */
  CCDHOST_NO_TABLES = 2,   /* build no loadMaps remap tables: ccdgpu_problem.maps[] are NULL
                              and ccdgpu_create derives the tables on the device */
  CCDHOST_NO_V = 4,        /* build no V blocks at all (CCDHOST_LOAD_V_PPPP is ignored): every
                              ccdgpu_problem.v_* is NULL and ccdgpu_create generates them on
                              the device from the model (V_pppp needs CCDGPU_V_ON_THE_FLY;
                              without the three-body V only the fused path runs) */
  CCDHOST_DEVICE_CHANNELS = 8 /* channel dimensions and maps built on the current CUDA device
                              (ccdgpu_build_channels) instead of on the host */
};

/* --pairing -l n_pair_states -n n_particles -x xi -g g  (parse.cpp:232-234) */
int ccdhost_build_pairing(double xi, double g, uint64_t n_pair_states, uint64_t n_particles,
                          int32_t flags, ccdhost_system **out);
/* --infMatter -d density -z tz_max -s n_shells -p n_particle_shells  (parse.cpp:235-237) */
int ccdhost_build_inf_matter(double density, int32_t tz_max, uint64_t n_shells,
                             uint64_t n_particle_shells, int32_t flags,
                             ccdhost_system **out);
/* --electronGas -r r_s -s n_shells -p n_particle_shells  (parse.cpp:238-240) */
int ccdhost_build_electron_gas(double r_s, uint64_t n_shells, uint64_t n_particle_shells,
                               int32_t flags, ccdhost_system **out);
void ccdhost_free(ccdhost_system *s);

const ccdgpu_problem *ccdhost_problem(const ccdhost_system *s);
double ccdhost_reference_energy(const ccdhost_system *s); /* SPBasis::referenceEnergy */
double ccdhost_mbpt2(const ccdhost_system *s);            /* MBPT2Corr over all channels */

/* Named flat arrays for tests: "chan_dims", "chan_mod_dims", "three_body_dims", "pp_map",
 * "hh_map", "ph_mod_map", "hp_mod_map", "hpp_map", "phh_map" (u64), "map_<name>" (u64
 * channel,row,column triples in pphh order, <name> as in ccdgpu_map_id), "v_<kind>" (f64, the
 * active-channel blocks concatenated), "sp_energy" (f64, normal ordered), "sp_energy_bare" (f64,
 * before normal ordering), "qn" (i32 SPBasis::indexMap rows).  dtype: 1 = f64, 2 = u64, 4 = i32. */
int ccdhost_array(const ccdhost_system *s, const char *name, const void **data,
                  uint64_t *count, int32_t *dtype);

#ifdef __cplusplus
}
#endif

#endif /* CCDHOST_H */
