/*
 * CPU restatement of the MDACP Lennard-Jones timestep (kohnakagawa/mdacp) for
 * ONE domain covering the whole periodic box.  TEST INFRASTRUCTURE ONLY: it is
 * the oracle that tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
 * leg compare the CUDA product against; nothing in the product links it.
 *
 * It follows the reference step by step, in the same order and with the same
 * floating-point expression trees (compiled with -ffp-contract=off), so that
 * it is bit-identical to the reference's plain (non-SIMD) build:
 *   migration + wrap       src/mdunit.cc:93-138, src/variables.cc:63-84
 *   ghost shell            src/mdunit.cc:140-208, src/mdmanager.cc:387-489, src/mdrect.cc:23-47
 *   cell mesh              src/meshlist.cc:40-65 (ChangeScale), :175-228 (MakeMesh)
 *   pair search            src/meshlist.cc:242-292 (SearchMesh), :555-583 (RegisterPair)
 *   CSR                    src/meshlist.cc:67-104 (MakeList)
 *   skin bookkeeping       src/pairlist.cc:10-121
 *   force kick             src/fcalculator.cc:228-290 (CalculateForceNext)
 *   half drift             src/fcalculator.cc:17-30
 *   thermostats            src/fcalculator.cc:979-1017, src/mdmanager.cc:254-315
 *   observers              src/observer.cc:4-79, src/mdmanager.cc:520-570
 * Parity is pinned against the reference itself, compiled from its sources by
 * oracle/ref/build_ref.sh and driven by oracle/ref/ref_harness.cc (fixtures in
 * tests/golden/).  The one deliberate difference: Langevin noise comes from a
 * counter-based Philox4x32-10 stream (shared with the CUDA path) instead of
 * the reference's per-thread std::mt19937 (src/fcalculator.cc:1003), so that
 * noise is reproducible independently of thread layout.
 */
#ifndef LJ_ORACLE_H
#define LJ_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { LJO_NVE = 0, LJO_NOSE_HOOVER = 1, LJO_LANGEVIN = 2 };

typedef struct {
  double L[3];            /* box lengths (SimulationInfo::L) */
  double rc;              /* CUTOFF_LENGTH */
  double buffer_length;   /* SimulationInfo::BufferLength = 0.3 */
  double dt;              /* TimeStep */
  int check_list_length;  /* CheckListLength, default 500 */
  int thermostat;         /* LJO_NVE / LJO_NOSE_HOOVER / LJO_LANGEVIN */
  double aimed_temperature;
  double heatbath_tau;
  double heatbath_gamma;
  uint64_t seed;          /* Langevin noise key */
} ljo_params;

typedef struct ljo_system ljo_system;

/* Creates a single-domain system holding n real atoms (q, v: n x 3, id: n). */
ljo_system *ljo_create(const ljo_params *prm, int n, const double *q, const double *v,
                       const int32_t *id);
void ljo_destroy(ljo_system *s);

/* MDManager::MakePairList for one unit: migrate + wrap, ghosts, PairList::Init, MakeList. */
int ljo_make_pairlist(ljo_system *s);
/* MDManager::Calculate, nsteps times.  Returns 0, or -1 on a reference exit(1) condition. */
int ljo_step(ljo_system *s, int nsteps);

int ljo_particle_number(const ljo_system *s);
int ljo_total_particle_number(const ljo_system *s);
int64_t ljo_pair_number(const ljo_system *s);
int ljo_constructions(const ljo_system *s);
double ljo_zeta(const ljo_system *s);

/* Real-atom state in the current (reference) index order. */
void ljo_get_state(const ljo_system *s, double *q, double *v, int32_t *id);
/* Directed pairs seen from real atoms, as ids: a real-real pair gives both
   directions, a real-ghost pair gives (real, source of ghost).  Returns count;
   writes at most cap entries. */
int64_t ljo_get_pairs(const ljo_system *s, int32_t *key_id, int32_t *partner_id, int64_t cap);
/* One CalculateForceNext kick on zeroed momenta with dt = 1 (p == F), real atoms,
   current index order.  State is left unchanged. */
void ljo_forces(ljo_system *s, double *f);
/* Sums as the observers return them: KE = sum 1/2 p^2, PE, virial = sum(...)/3. */
void ljo_observe(const ljo_system *s, double *ke, double *pe, double *virial);
/* The same sums with compensated summation (the checker for very long sums). */
void ljo_observe_compensated(const ljo_system *s, double *ke, double *pe, double *virial);

/* Executors the reference's projects run after each Calculate() (real atoms,
   momenta = velocities): kind 1 GravityImposer (src/phaseflow.cc:58-73),
   2 MyPiston (src/rankine.cc:55-97), 3 ShellForce (src/burst.cc:67-99).
   Piston: after the pass the position moves by -velocity, as Rankine::Run
   moves it (src/rankine.cc:117-121); returns the pass's impulse (0 for the
   other kinds). */
typedef struct ljo_external {
  int kind;
  int axis;          /* gravity */
  double strength;   /* gravity: acceleration */
  double time_step;  /* the dt the executor multiplies by */
  double position;   /* piston */
  double velocity;   /* piston: displacement per pass */
  double center[3];  /* shell */
  double radius;     /* shell: radius of the wall surface */
} ljo_external;
double ljo_apply_external(ljo_system *s, ljo_external *e);

/* Philox4x32-10 block (Salmon et al., SC'11), exported for the noise tests. */
void ljo_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* The three standard normals used for atom `id` at Langevin step `step`. */
void ljo_langevin_normals(uint64_t seed, uint32_t id, uint64_t step, double z[3]);

#ifdef __cplusplus
}
#endif
#endif
