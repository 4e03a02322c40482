/*
 * mdacp_b200 -- C ABI of the B200-native Lennard-Jones timestep.
 *
 * One handle owns one periodic single-domain system resident in the GPU's
 * HBM: cell-sorted positions and velocities, the Verlet pairlist, the skin
 * bookkeeping and the step graph.  Plain pointers and sizes only; host
 * arrays use the reference's padded AoS layout (x, y, z, pad per atom, as
 * double q[N][D] / p[N][D] with D = 4, include/mdconfig.h:9, include/variables.h:19-28).
 *
 * Each entry point names the reference interface it replaces
 * (kohnakagawa/mdacp, path:line).  Every call returns an mdg_status; 0 is
 * success, negative values are errors whose text mdg_last_error() returns.
 * The reference reports the same conditions with show_error + exit(1)
 * (include/mdconfig.h:37); the drop-in C++ classes map a negative status
 * back onto that behaviour.
 *
 * A handle is not thread-safe.  Separate handles are independent.  All work
 * is issued on the handle's stream; calls that return host data synchronise
 * that stream.
 */
#ifndef MDACP_B200_H
#define MDACP_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mdg_handle mdg_handle;
typedef int mdg_status;

enum {
  MDG_OK = 0,
  MDG_ERR_INVALID_ARGUMENT = -1,
  MDG_ERR_CUDA = -2,
  MDG_ERR_CAPACITY = -3,         /* atom or neighbour capacity exceeded */
  MDG_ERR_TOO_FAST = -4,         /* 2 vmax dt > BufferLength (src/pairlist.cc:59-63) */
  MDG_ERR_INVALID_POSITION = -5, /* atom outside [0,L] after wrap (src/variables.cc:75-83) */
  MDG_ERR_NONFINITE = -6,        /* NaN / Inf in the state */
  MDG_ERR_BOX_TOO_SMALL = -7,    /* fewer than 3 cells along an axis */
  MDG_ERR_TIMEOUT = -8,          /* a bounded device wait gave up */
  MDG_ERR_STATE = -9,            /* call out of order (e.g. no state uploaded) */
  MDG_ERR_NO_DEVICE = -10,
  MDG_ERR_IO = -11               /* a file could not be read or written, or is not a checkpoint */
};

enum { MDG_FP64 = 0, MDG_FP32_MIXED = 1 };
enum { MDG_OBSERVE_CURRENT = 0, MDG_OBSERVE_GHOST_LAG = 1 };
enum { MDG_NVE = 0, MDG_NOSE_HOOVER = 1, MDG_LANGEVIN = 2 };

/* Run parameters; the reference's SimulationInfo public fields
   (include/simulationinfo.h:20-33, src/simulationinfo.cc:5-51) plus the
   compile-time CUTOFF_LENGTH (include/mdconfig.h:31), which is a runtime
   value here. */
typedef struct {
  int capacity;             /* maximum number of atoms (reference: N, mdconfig.h:11) */
  double L[3];              /* box lengths (SimulationInfo::L) */
  double cutoff;            /* CUTOFF_LENGTH */
  double buffer_length;     /* BufferLength (0.3); SearchLength = cutoff + buffer_length */
  double time_step;         /* TimeStep */
  int precision;            /* MDG_FP64 (drop-in) or MDG_FP32_MIXED */
  int thermostat;           /* MDG_NVE, MDG_NOSE_HOOVER, MDG_LANGEVIN */
  double aimed_temperature; /* AimedTemperature */
  double heatbath_tau;      /* HeatbathTau */
  double heatbath_gamma;    /* HeatbathGamma */
  uint64_t seed;            /* Langevin noise key (Philox4x32-10) */
  int check_list_length;    /* CheckListLength (500) */
  int max_neighbors;        /* neighbour-row capacity; 0 = derived from density */
  int device;               /* CUDA device ordinal */
  void *stream;             /* cudaStream_t to issue work on; NULL = handle-owned stream */
  int stage_atoms;          /* FP32-mixed: partner positions staged in shared memory per
                               128-atom block, at most this many atoms; 0 (default) = off,
                               partners gathered from global memory; -1 = 2304 atoms.
                               Steps with the staged pass run as graphs (step_mode). */
  int threads_per_atom;     /* FP32-mixed force pass: lanes per atom, 1, 2 or 4; every
                               choice gives bit-identical forces (fixed summation tree).
                               0 (default) = chosen by timing the three once per device
                               and problem shape, at the first step */
  int build_block;          /* list build: threads per block, 64, 128 or 256; 0
                               (default) = chosen by timing, as threads_per_atom */
  int build_threads_per_atom; /* list build: lanes per atom, 1, 2, 4 or 8 (the rows are the
                               same for every choice); 0 (default) = chosen by timing
                               together with build_block */
  int step_mode;            /* how mdg_calculate runs FP32-mixed NVE steps:
                               MDG_STEPS_AUTO (default): persistent when every atom's lanes
                               fit in one wave of co-resident blocks, else graphs;
                               MDG_STEPS_GRAPHS: CUDA graphs with conditional rebuild nodes;
                               MDG_STEPS_PERSISTENT: cooperative launches run the steps
                               back to back, displacement checks included (one lane per
                               atom from 16,384 atoms, 2 or 4 below); each stops at a step
                               that needs a rebuild, which a queued graph takes, and the
                               next launch follows without a host wait.  Same results. */
  long long stage_wait_cycles; /* staged FP32-mixed pass (stage_atoms != 0): clock cycles a
                               block waits for its stage copy before it reports
                               MDG_ERR_TIMEOUT; it then still waits up to about a second
                               for the copy to land before it exits.  0 (default): about a
                               second.  A short limit tests the error path. */
} mdg_params;

enum { MDG_STEPS_AUTO = 0, MDG_STEPS_GRAPHS = 1, MDG_STEPS_PERSISTENT = 2 };

/* Fills p with the reference defaults (SimulationInfo ctor, src/simulationinfo.cc:5-51). */
void mdg_default_params(mdg_params *p);

/* Replaces: MDUnit ctor allocation of Variables/MeshList/PairList and the
   CUDA buffers (src/mdunit.cc:8-39, include/cuda_ptr.h:13-152,
   src/meshlist.cu:21-33). */
mdg_status mdg_create(const mdg_params *params, mdg_handle **out);
mdg_status mdg_destroy(mdg_handle *h);

/* Replaces: Variables::AddParticle for a whole array (src/variables.cc:35-47)
   plus the per-step host-to-device copy (src/fcalculator.cu:5-13).  q4, v4 are
   n x 4 doubles (pad ignored), type is n ints (may be NULL).  The list is
   marked stale: the next step rebuilds it.  Atom slots are renumbered at every
   rebuild (cell order); mdg_get_ids gives each slot's upload index. */
mdg_status mdg_set_state(mdg_handle *h, const double *q4, const double *v4, const int *type,
                         int n);
/* Replaces: the device-to-host copy of p (src/fcalculator.cu:15-22) and reads
   of Variables::q/p/type.  Arrays are in the current slot order. */
mdg_status mdg_get_state(mdg_handle *h, double *q4, double *v4, int *type, int n);
mdg_status mdg_get_ids(mdg_handle *h, int *ids, int n);
/* Replaces: an Executor's writes to Variables::p between steps
   (MDManager::ExecuteAll, src/mdmanager.cc:586-592; e.g. GravityImposer,
   src/phaseflow.cc:58-73, MyPiston, src/rankine.cc:55-97): new velocities,
   n x 4 doubles in the current slot order (the order mdg_get_state returns),
   positions untouched.  Unlike mdg_set_state it keeps the list, the skin
   budget and the observers' ghost age, as the reference's executors leave
   its PairList and ghost copies alone; the |v| maximum of the next skin test
   is taken from the new velocities (IsPairListExpired reads the momenta
   after the executor). */
mdg_status mdg_set_velocities(mdg_handle *h, const double *v4, int n);
mdg_status mdg_particle_number(mdg_handle *h, int *n);

/* Replaces: MDManager::MakePairList (src/mdmanager.cc:387-417): wrap into
   [0,L] (Variables::AdjustPeriodicBoundary, src/variables.cc:63-84), cell
   counting sort (MeshList::MakeMesh, src/meshlist.cc:175-228), Verlet list
   within SearchLength (MeshList::MakeList/SearchMesh, src/meshlist.cc:67-104,
   242-292) and PairList::Init (src/pairlist.cc:10-23). */
mdg_status mdg_make_pairlist(mdg_handle *h);

/* Replaces: PairList::IsPairListExpired (src/pairlist.cc:25-45). */
mdg_status mdg_check_expired(mdg_handle *h, int *expired);

/* Replaces: ForceCalculator::UpdatePositionHalf (src/fcalculator.cc:17-30). */
mdg_status mdg_update_position_half(mdg_handle *h);

/* Replaces: ForceCalculator::CalculateForce (src/fcalculator.cc:32-50 and the
   GPU offload src/fcalculator.cu:38-73): the kick p += F(q) * TimeStep. */
mdg_status mdg_calculate_force(mdg_handle *h);

/* Replaces: ForceCalculator::HeatbathZeta / HeatbathMomenta / Langevin
   (src/fcalculator.cc:979-1017, src/fcalculator.cu:75-88). */
mdg_status mdg_heatbath_zeta(mdg_handle *h, double current_temperature);
mdg_status mdg_heatbath_momenta(mdg_handle *h);
mdg_status mdg_langevin(mdg_handle *h);
mdg_status mdg_get_zeta(mdg_handle *h, double *zeta);
mdg_status mdg_set_zeta(mdg_handle *h, double zeta);
/* Replaces: MDManager::SetControlTemperature / SetAimedTemperature
   (include/mdmanager.h:78-79) and the HeatbathType/HeatbathTau/HeatbathGamma
   fields of SimulationInfo: switches the thermostat of later steps. */
mdg_status mdg_set_control(mdg_handle *h, int thermostat, double aimed_temperature,
                           double heatbath_tau, double heatbath_gamma);

/* Replaces: MDManager::Calculate (src/mdmanager.cc:153-186) called nsteps
   times: expiry check, conditional rebuild, half drift, force kick (NVE,
   Nose-Hoover or Langevin branch, src/mdmanager.cc:226-315), half drift.
   Runs as CUDA graphs with device-side conditional rebuild nodes; nothing is
   copied to the host. */
mdg_status mdg_calculate(mdg_handle *h, int nsteps);

/* Forces only, no kick (parity): f4 is n x 4, F = -dV/dq of the smoothed LJ
   potential (the reference's kick with TimeStep = 1). */
mdg_status mdg_forces(mdg_handle *h, double *f4);

/* Replaces: KineticEnergyObserver, PotentialEnergyObserver, VirialObserver
   (src/observer.cc:4-79) summed over the system as MDManager::ObserveDouble
   does (src/mdmanager.cc:520-528): ke = sum 1/2 p^2, pe = sum of pair
   energies, virial = sum(...)/3.  FP64 device reductions. */
mdg_status mdg_observe(mdg_handle *h, double *ke, double *pe, double *virial);

/* Which positions mdg_observe pairs an atom with across the periodic
   boundary.  MDG_OBSERVE_CURRENT (default): every atom at its current
   position.  MDG_OBSERVE_GHOST_LAG: what the reference's observers see after
   MDManager::Calculate in the NVE and Nose-Hoover branches -- its ghost
   copies were refreshed after the first half drift (src/mdmanager.cc:165-167),
   so a partner reached through the boundary sits half a step back,
   q - v dt/2.  The drop-in classes use GHOST_LAG so that projects print what
   the reference prints. */
mdg_status mdg_set_observer_mode(mdg_handle *h, int mode);

/* Directed list entries within the cut-off (pair terms one force
   evaluation computes; unordered pairs = within_cutoff / 2) and all list
   entries, at the current positions. */
mdg_status mdg_pair_counts(mdg_handle *h, int64_t *within_cutoff, int64_t *list_entries);

/* Pairlist readout for parity (MeshList::GetPairNumber, GetKeyPointer,
   GetPartnerNumber, GetSortedList, include/meshlist.h:70-91).  Directed
   (key, partner) pairs, expressed as upload indices, one per atom that has
   the partner within SearchLength; *count returns the total, at most cap
   entries are written. */
mdg_status mdg_get_pairs(mdg_handle *h, int *key, int *partner, int64_t cap, int64_t *count);

/* The full Verlet list in the current slot order (the order mdg_get_state
   returns): row_len[i] partners of slot i, concatenated in `partners`
   (slot indices).  *count returns the total; at most cap entries are
   written.  A half list with key < partner is the reference's
   key_partner_pairs / sorted_list (src/meshlist.cc:67-104, 555-583). */
mdg_status mdg_get_list(mdg_handle *h, int *row_len, int *partners, int64_t cap, int64_t *count);

typedef struct {
  int n;                  /* atoms */
  int ncell[3];           /* cells per axis */
  int max_neighbors;      /* neighbour-row capacity */
  int max_row;            /* longest row of the last build */
  int64_t list_entries;   /* entries of the last build (full list) */
  int64_t steps;          /* MD steps taken */
  int64_t rebuilds;       /* pairlist constructions (MeshList::GetNumberOfConstructions) */
  int64_t displacement_checks;
  double simulation_time;
  double buffer_left;     /* skin budget (PairList::buffer_length) */
  int threads_per_atom;   /* lanes per atom of the FP32-mixed force pass (0: not chosen yet) */
  int build_block;        /* threads per block of the list build (0: not chosen yet) */
  int build_threads_per_atom; /* lanes per atom of the list build (0: not chosen yet) */
  int64_t persistent_steps;   /* steps taken by the persistent pass (step_mode) */
} mdg_info;
mdg_status mdg_get_info(mdg_handle *h, mdg_info *info);

/* Device pointer of the handle's stream (cudaStream_t) and the handle's
   internal timers: each call to mdg_calculate records CUDA events around
   every force kernel when timing is on; mdg_kernel_time returns the summed
   milliseconds and launch count of the force kernel since the last reset. */
void *mdg_stream(mdg_handle *h);
/* use_graphs = 1 (default): mdg_calculate runs batches of steps as CUDA
   graphs with conditional rebuild nodes.  0: every kernel is launched
   directly from the host, with the skin decision read back each step --
   the same kernels and results, for profilers that cannot look inside
   graphs holding conditional nodes. */
mdg_status mdg_set_graph_mode(mdg_handle *h, int use_graphs);
mdg_status mdg_set_kernel_timing(mdg_handle *h, int on);
mdg_status mdg_kernel_time(mdg_handle *h, double *force_ms, int64_t *force_launches,
                           int64_t *kernel_launches);

/* No counterpart in the reference.  mdg_observe for callers that cannot
   allocate device memory (they own all of it, or must avoid the implicit
   synchronisation of cudaMalloc/cudaFree): no handle, all arrays are the
   caller's DEVICE pointers -- q4, v4 (n x 4 doubles), a CSR full list
   row_start (n + 1 ints) / partners (row_start[n] ints, indices into q4),
   out (3 doubles: KE, PE, virial as mdg_observe returns them).  L and cutoff
   are host values.  Work is queued on `stream` (cudaStream_t, NULL = legacy
   default stream); out is ready when the stream is.  Scratch is a static
   device array of 196,608 bytes held by every GPU that loads the library, so
   n is limited to 2,097,152 (MDG_ERR_CAPACITY above).  A call outside a
   stream capture looks the array's address up with its device current; a
   call during a capture uses the address found by the last uncaptured call
   on that device (MDG_ERR_STATE if there was none), so make one call per
   device before capturing.  Calls that overlap on the GPU race on the
   shared scratch.  A partner index outside [0, n) is never read: the pair
   is skipped and the returned PE is NaN.  A CUDA error already pending from
   the caller's earlier work is left pending and reported as MDG_ERR_CUDA
   with nothing launched. */
mdg_status mdg_observe_static(const double *q4, const double *v4, int n, const int *row_start,
                              const int *partners, const double L[3], double cutoff, double *out,
                              void *stream);

/* ---------------------------------------------------------------- ensembles
   Many independent periodic systems (replicas) of different size, density
   and temperature advanced together; no counterpart in the reference, which
   runs one system per MPI job.  Every kernel of a step covers all replicas
   in one launch (per-replica cell grids and offset tables); each replica
   keeps its own skin budget and rebuilds only its own list, with the
   single-system arithmetic, so a replica evolves bit-identically to the
   same system in its own handle.  NVE only.  Arrays are the replicas'
   atoms concatenated in replica order, n x 4 doubles. */
typedef struct mdg_ensemble mdg_ensemble;
typedef struct {
  int n;          /* atoms */
  double L[3];    /* box; every length must exceed 2 x SearchLength */
  double buffer_length; /* > 0: this replica's BufferLength (its SearchLength is
                           cutoff + this, its skin budget starts at this); 0: the
                           common buffer_length.  A replica evolves as a single
                           system with the same buffer_length. */
} mdg_replica;
/* common: cutoff, buffer_length, time_step, precision, check_list_length,
   device (capacity, thermostat and stream are not used). */
mdg_status mdg_ensemble_create(const mdg_params *common, int nrep, const mdg_replica *replicas,
                               mdg_ensemble **out);
mdg_status mdg_ensemble_destroy(mdg_ensemble *e);
mdg_status mdg_ensemble_set_state(mdg_ensemble *e, const double *q4, const double *v4);
/* Current slot order; ids (may be NULL) = upload index within the replica. */
mdg_status mdg_ensemble_get_state(mdg_ensemble *e, double *q4, double *v4, int *ids);
mdg_status mdg_ensemble_calculate(mdg_ensemble *e, int nsteps);
/* Per-replica sums (arrays of nrep), as mdg_observe returns them. */
mdg_status mdg_ensemble_observe(mdg_ensemble *e, double *ke, double *pe, double *virial);
mdg_status mdg_ensemble_rebuilds(mdg_ensemble *e, int64_t *rebuilds, int64_t *steps);
mdg_status mdg_ensemble_set_graph_mode(mdg_ensemble *e, int use_graphs);
/* Force-kernel timers of the ensemble, as mdg_set_kernel_timing /
   mdg_kernel_time for one handle: CUDA events around every force launch
   (one launch covers all replicas) while timing is on. */
mdg_status mdg_ensemble_set_kernel_timing(mdg_ensemble *e, int on);
mdg_status mdg_ensemble_kernel_time(mdg_ensemble *e, double *force_ms, int64_t *force_launches,
                                    int64_t *kernel_launches);
/* Over all replicas: neighbour-list entries of the current lists and the
   unordered pairs closer than the cut-off at the current positions. */
mdg_status mdg_ensemble_list_stats(mdg_ensemble *e, int64_t *list_entries, int64_t *pairs_within_cutoff);
void *mdg_ensemble_stream(mdg_ensemble *e);

/* Replaces, for independent replicas, the reference's assignment of work
   to MPI ranks (ParaInfo, src/parainfo.cc:16-94, which splits one box into a
   grid of equal domains): replica r goes to rank owner[r] so that the
   ranks' loads are balanced, the load of a replica being its atoms times
   (41 + the neighbours expected within search_length, 4/3 pi SL^3 N/V) --
   the list entries a step streams per atom plus the per-atom state traffic
   in the same 4-byte units (164 B).  Largest load first, each to the least
   loaded rank (lowest rank on ties): deterministic.  load (nranks doubles,
   may be NULL) returns every rank's total.  Host-only: no device needed. */
mdg_status mdg_partition_replicas(const mdg_replica *replicas, int nrep, double search_length, int nranks,
                                  int *owner, double *load);

/* ---------------------------------------------------------- slab decomposition
 * One periodic system split into z-slabs of whole cell layers of the
 * single-domain cell grid (int(L/SL) cells per axis), one slab per device
 * (devices may repeat), driven by the calling thread.  Replaces the
 * reference's domain decomposition: migration MDManager::SendParticles
 * (src/mdmanager.cc:317-374), ghost layers refreshed every step
 * MDManager::SendBorderParticles (src/mdmanager.cc:419-489,
 * src/mdunit.cc:140-208), the expiry all-reduce (src/mdmanager.cc:509-518,
 * src/communicator.cc:24-37).  Each slab holds its own atoms plus one ghost
 * layer of cells on each side; every step each slab pushes its two border
 * layers' positions into its neighbours' ghost slots (peer copies); the
 * skin decision, the displacement check and the rebuild are global, and a
 * rebuild migrates the atoms that changed slab.  Lists, force sums and
 * trajectories equal the single domain's.  NVE, FP64 or FP32-mixed;
 * host-driven steps (one host synchronisation per step for the global skin
 * decision).  Layers are split as evenly as their count allows; at least
 * one layer per slab, at least 2 slabs. */
typedef struct mdg_slabs mdg_slabs;
/* params: the whole system's box, capacity (all atoms), cutoff, buffer
   length, time step, precision, check_list_length, threads_per_atom;
   devices: nslabs device ordinals, or NULL for params->device. */
mdg_status mdg_slabs_create(const mdg_params *params, int nslabs, const int *devices, mdg_slabs **out);
mdg_status mdg_slabs_destroy(mdg_slabs *x);
/* n atoms in the reference's AoS layout (as mdg_set_state); each goes to the
   slab of its cell layer; ids are the upload indices. */
mdg_status mdg_slabs_set_state(mdg_slabs *x, const double *q4, const double *v4, const int *type, int n);
/* n x 4 doubles ordered by upload index. */
mdg_status mdg_slabs_get_state(mdg_slabs *x, double *q4, double *v4, int n);
mdg_status mdg_slabs_calculate(mdg_slabs *x, int nsteps);
/* System sums over all slabs, as mdg_observe (MDG_OBSERVE_CURRENT). */
mdg_status mdg_slabs_observe(mdg_slabs *x, double *ke, double *pe, double *virial);
/* Forces (no kick) ordered by upload index, n x 4 doubles, as mdg_forces. */
mdg_status mdg_slabs_forces(mdg_slabs *x, double *f4, int n);
/* Steps, rebuilds, and per slab its own atoms and ghost copies (arrays of
   nslabs ints, may be NULL). */
mdg_status mdg_slabs_info(mdg_slabs *x, int64_t *steps, int64_t *rebuilds, int *owned, int *ghosts);
const char *mdg_slabs_last_error(mdg_slabs *x);

/* ---------------------------------------------------------- box and grid analysis
 * MDManager::ChangeScale (src/mdmanager.cc:573-585) on the device: the list
 * is built (atoms wrapped into the box), the box and every position are
 * scaled by alpha, the cell grid is recomputed and the list rebuilt. */
mdg_status mdg_change_scale(mdg_handle *h, double alpha);
/* Atoms per cell of a regular grid, as BubbleHist::Analyse counts them
 * (src/cavitation.cc:38-58, 117-146): dims[d] = int(L_d / grid_size + 0.5)
 * cells per axis with one edge L_x / dims[0], x fastest, counts as unsigned
 * char (wrapping at 256 like the reference's counters), positions wrapped
 * into the box.  out needs dims[0]*dims[1]*dims[2] bytes (cap).  Unlike
 * BubbleHist::Analyse it does not rebuild the pairlist; call
 * mdg_make_pairlist first for the reference's rebuild schedule. */
mdg_status mdg_density_grid(mdg_handle *h, double grid_size, unsigned char *out, int64_t cap, int dims[3]);

/* ---------------------------------------------------------- checkpoints and snapshots
 * A checkpoint holds the handle's whole state: atoms in slot order with their
 * ids and types, positions at the last list build, the skin budget, step and
 * build counters, simulation time, zeta and the executor's state.  A handle
 * created with the same parameters and loaded from it continues bit for bit
 * as the saved handle would have (the list is rebuilt from the positions of
 * the last build).  The reference's Variables::SaveToStream and
 * LoadFromStream (src/variables.cc:115-136) are not symmetric: the reader
 * expects a header the writer never writes; this format has one. */
mdg_status mdg_save_checkpoint(mdg_handle *h, const char *path);
mdg_status mdg_load_checkpoint(mdg_handle *h, const char *path);
/* The reference's text snapshots, from the device state: CDVIEW as
 * MDUnit::SaveAsCdview ("0 type x y z px py pz", src/mdunit.cc:67-83),
 * CONFIGURATION as Variables::SaveConfiguration ("x y z px py pz",
 * src/variables.cc:49-61).  The device-to-host copy is queued on the
 * handle's stream into pinned buffers the handle keeps (allocated on the
 * first call, grown with the atom count) and a host thread writes the file,
 * so the caller can keep queuing steps.  At most one file is pending: a call
 * first waits for the previous file and, if that write failed, returns
 * MDG_ERR_IO with its name and starts nothing.  mdg_snapshot_wait waits for
 * the pending file and reports its failure the same way; call it before
 * mdg_destroy, which waits too but cannot report. */
enum { MDG_SNAPSHOT_CDVIEW = 0, MDG_SNAPSHOT_CONFIGURATION = 1 };
mdg_status mdg_snapshot_async(mdg_handle *h, const char *path, int format);
mdg_status mdg_snapshot_wait(mdg_handle *h);

/* ---------------------------------------------------------- executors
 * An executor the reference's projects run after every MDManager::Calculate()
 * through MDManager::ExecuteAll, applied here on the device after each step
 * of mdg_calculate (no host round trip, inside the CUDA graphs):
 *   GRAVITY  v[axis] += strength * time_step       GravityImposer, src/phaseflow.cc:58-73
 *   PISTON   wall at z = 0 and a piston at `position` (both the pair-force
 *            expression at the distance), impulse summed; the position then
 *            moves by -velocity                    MyPiston, src/rankine.cc:55-97,117-121
 *   SHELL    spherical wall of radius `radius` around `center`
 *                                                  ShellForce, src/burst.cc:67-99
 * time_step is the dt the executor multiplies by (the reference's executors
 * carry their own). */
enum {
  MDG_EXTERNAL_NONE = 0,
  MDG_EXTERNAL_GRAVITY = 1,
  MDG_EXTERNAL_PISTON = 2,
  MDG_EXTERNAL_SHELL = 3
};
typedef struct mdg_external {
  int kind;
  int axis;
  double strength;
  double time_step;
  double position;
  double velocity;
  double center[3];
  double radius;
} mdg_external;
/* NULL or kind NONE turns the executor off. */
mdg_status mdg_set_external(mdg_handle *h, const mdg_external *x);
/* Piston position now and impulse of the last pass (MyPiston::position, impulse). */
mdg_status mdg_external_state(mdg_handle *h, double *position, double *impulse);

/* ---------------------------------------------------------- adjoint
 * Gradients of a trajectory loss, by a reverse sweep over the steps
 * (mdacp_b200/csrc/mdg_adjoint.cu).  No counterpart in the reference, which
 * computes no gradients.  Potential U(r) = epsilon phi(r/sigma) with the
 * reference's smoothed phi (src/variables.cc:16-33) and the cut-off in units
 * of sigma; steps as MDManager::Calculate (NVE, src/mdmanager.cc:153-186), in
 * FP64.  Loss L = 1/(steps n) sum over the steps' end states of
 * [PE + sum over pairs g((r-lo)/w) g((hi-r)/w)], g the logistic function.
 * Pairs come from a Verlet list of search length cutoff + 0.3 sigma (less in
 * boxes narrower than three such lengths), rebuilt when an atom has moved
 * half the skin; its rows are in ascending partner order, so the sums are a
 * function of the positions alone (and of threads_per_atom). */
typedef struct mdg_adjoint_params {
  double L[3];
  double cutoff;          /* in units of sigma (CUTOFF_LENGTH, include/mdconfig.h:31) */
  double time_step;
  double epsilon, sigma;
  double shell_lo, shell_hi, shell_width;  /* smoothed pair count window */
  int steps;
  int checkpoint_every;   /* states kept every k steps; segments recomputed */
  int threads_per_atom;   /* lanes per atom in the pair kernels: 1, 2, 4, 8, or 0 to
                             time all four once per device and problem shape */
  int device;
} mdg_adjoint_params;

void mdg_adjoint_default_params(mdg_adjoint_params *p);
/* q0, v0: n x 3 doubles.  loss is required; with all three gradient
 * pointers NULL only the forward pass runs.  dloss_dq0: n x 3 doubles.
 * Device memory (checkpoints: 2 x 32 B per atom per checkpoint; the list:
 * 4 B per row entry, rows of up to 1024 entries) is kept per device after
 * the call and reused by later calls whose buffers fit, so repeated calls of
 * one shape allocate nothing; one run at a time per process.
 * MDG_ERR_CAPACITY if a row outgrows its capacity (three times the mean
 * density's count within the search length, plus 64). */
mdg_status mdg_adjoint_run(const mdg_adjoint_params *p, const double *q0, const double *v0, int n, double *loss,
                           double *dloss_deps, double *dloss_dsigma, double *dloss_dq0);
/* Frees the device memory, stream and pinned buffer that mdg_adjoint_run
 * keeps between calls (all devices).  Call it before cudaDeviceReset; a run
 * after a reset without it finds its kept buffers gone and allocates anew. */
void mdg_adjoint_release(void);

const char *mdg_last_error(mdg_handle *h);
const char *mdg_status_string(mdg_status s);
/* Library version string. */
const char *mdg_version(void);

#ifdef __cplusplus
}
#endif
#endif
