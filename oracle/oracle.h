/*
 * CPU oracle: plain-C restatement of the reference's checkerboard SU(2) sweep
 * (fezquerro/QCD_2d_GPU, functions/*.h).  TEST INFRASTRUCTURE ONLY: the
 * tests, the smoke check and the CPU-baseline leg of the benchmark call it as
 * the checker; the product never links or calls it.
 *
 * Layout is the reference's AoS FP64 field (kernel.cu:58, lattice_setup.h:24-37).
 * Random numbers come from one of two sources:
 *   TAPE  draws recorded on the GPU from cuRAND's MRG32k3a streams
 *         (curand_init(seed, id, 0), lattice_setup.h:15-21), with the CUDA
 *         float values of logf / cospif / sincospif of each draw; replaying
 *         them gives the reference's arithmetic bit for bit without
 *         re-implementing cuRAND (pinned against the reference's own outputs
 *         in tests/golden/).
 *   OWN   L'Ecuyer's MRG32k3a with the published 1999 parameters and
 *         2^127-spaced streams (L'Ecuyer, Simard, Chen, Kelton 2002), host
 *         libm for the transcendentals: statistically equivalent, used for the
 *         timed CPU baseline; it is not cuRAND's seeding.
 */
#ifndef QCD_ORACLE_H
#define QCD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_tape_record { /* same layout as qcd_tape_record */
  double ud;
  float uf, log_uf, cospi_2uf, sc_sin, sc_cos;
  unsigned int same_step;
} ora_tape_record;

typedef struct ora_params {
  int lt, lx, ly;
  float beta, epsilon;
  int upd;
  int algo;     /* 0 Metropolis, 1 heat-bath (kernel.cu:11-12) */
  int boundary; /* 0 periodic, 1 PCC, 2 PMC (kernel.cu:28) */
  unsigned long long seed;
} ora_params;

enum { ORA_OK = 0, ORA_ERR_INVALID = -1, ORA_ERR_TAPE = -2, ORA_ERR_NOMEM = -3 };

typedef struct ora_lattice ora_lattice;

/* tape == NULL selects the OWN generator */
ora_lattice* ora_create(const ora_params* p, const ora_tape_record* tape, int tape_streams,
                        int tape_draws);
void ora_destroy(ora_lattice* h);

int ora_init_cold(ora_lattice* h);
int ora_init_hot(ora_lattice* h);
int ora_load(ora_lattice* h, const double* aos);
/* kind: 0 Metropolis, 1 heat-bath, 2 over-relaxation; phase k = 2*mu + parity */
int ora_phase(ora_lattice* h, int k, int kind);
int ora_sweep(ora_lattice* h, int n);
int ora_overrelax(ora_lattice* h, int n);
int ora_normalize(ora_lattice* h);
int ora_measure(ora_lattice* h, double* energy, double* plaquette);
/* One phase of the library's FP32 path (float links, FP64 fix-ups), the
   checker of its FP32 kernels: kind as for ora_phase; draws from Philox4x32-10
   with counter (site id, block, phase lo, phase hi) and key (key lo, key hi);
   renorm re-projects each updated link.  With hb_tries (V ints, reference
   site order) the heat-bath stores the rejection-loop trips of each site. */
/* one Philox4x32-10 block of the FP32 restatement (for pinning it) */
void ora_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
int ora_phase32(ora_lattice* h, int k, int kind, unsigned long long key, unsigned long long phase, int renorm,
                int* hb_tries);
const double* ora_field(const ora_lattice* h);
const int* ora_accept(const ora_lattice* h);
long long ora_volume(const ora_lattice* h);
/* largest number of draws any stream has consumed */
long long ora_max_draws(const ora_lattice* h);
int ora_set_threads(int n);
int ora_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
