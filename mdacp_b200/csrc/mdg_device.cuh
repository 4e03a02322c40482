// Device code of the B200 LJ timestep: cell sort, Verlet list build, force
// kick (FP64 drop-in and FP32-mixed), drift, skin bookkeeping, thermostats
// and FP64 observables.  Host orchestration lives in mdg_api.cu.
//
// Data layout in HBM (n atoms, slots renumbered in cell order at every
// rebuild):
//   q, v      double4[cap]   position (unwrapped between rebuilds), velocity
//   qfix      int4[cap]      fixed-point copy of q for the FP32-mixed force:
//                            x_fix = round(frac(x/L) * 2^32) as uint32, so the
//                            int32 difference of two atoms is the minimum-image
//                            displacement in units of L/2^32 (no shift tables)
//   nbr       int32[maxnb][stride]  full Verlet list, column-major: entry k
//                            of atom i at nbr[k*stride + i] (coalesced per warp)
//   nnbr      int32[cap]     row lengths; rows are padded with the atom's own
//                            index up to a multiple of 4 (the FP32 force loop
//                            walks 4 partners at a time; a self entry has r = 0
//                            and is masked)
//   qloc      float4[cap]    FP32 coordinates at the last build for the list
//                            prefilter: x in box coordinates, y and z
//                            relative to the atom's cell
//   cxyz      int32[cap]     the slot's cell coordinates at the last build,
//                            packed x | y << 11 | z << 22
//   xsub      int32[rows*(8*ms_x+1)]  list-build trim table, one block per
//                            x-row of cells: atoms inside a cell are in x
//                            order, entry 8*cx + k of a row's block is the first
//                            slot of its cell cx at or beyond x0 + k cs_x / 8,
//                            and entry 8*ms_x is the end of the row
//   nbr16     uint2[maxnb/4][stride]  FP32-mixed only: the same rows as 16-bit
//                            indices into the block's staged partner positions
//                            (four per 8-byte load); see k_stage_plan
//   stage_rng int4[blocks][kStageRanges]  per 128-atom block: the cell ranges
//                            whose atoms the force pass stages in shared memory
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mdg {

constexpr int kErrCapacity = 1;
constexpr int kErrTooFast = 2;
constexpr int kErrInvalidPosition = 4;
constexpr int kErrNonFinite = 8;
constexpr int kErrTimeout = 16;
constexpr int kErrStage = 32;  // a staged row index outside its block's stage (an inconsistent plan)

// Geometry and force constants, passed by value to every kernel.
struct Box {
  double L[3];
  double hL[3];        // L/2, minimum-image threshold
  double inv_cs[3];    // 1 / cell size
  int ms[3];           // cells per axis (MeshList::ChangeScale: int(L/SL))
  int ncell;
  double sl;           // SearchLength
  double sl2;          // SearchLength^2
  double rc2;          // CUTOFF_LENGTH^2
  double rc;           // CUTOFF_LENGTH
  double c0, c2;       // smoothed-LJ constants (Variables::C0, C2)
  double dt;           // TimeStep
  double buffer_length;
  float fix_scale[3];  // L / 2^32
  float rc2f;
  float c2x8f;
  int check_list_length;
  double cs[3];        // cell size L / ms
  float sl2_lo, sl2_hi;  // FP32 prefilter band around SearchLength^2
  // z-slab of a decomposed system (slab = 1): the owned cell layers are the
  // global layers z0 .. z0 + nzl - 1, and cell indices, packed cell
  // coordinates and trim-table rows use the local layer z - z0; the trim
  // table has two more blocks of rows, the ghost layers below (block nzl)
  // and above (block nzl + 1).  A single domain has slab = 0, z0 = 0 and
  // nzl = ms[2].
  int slab, z0, nzl;
  long long stage_wait;  // staged FP32 pass: cycles of the first wait for the stage copy
};

// Mutable device-side state of one handle.
struct Status {
  int error;                        // kErr* flags; any set flag halts the step kernels
  int list_stale;                   // 1: next step rebuilds unconditionally
  unsigned long long vmax2_bits;    // max |v|^2 of the last velocity update (double bits)
  double budget;                    // PairList::buffer_length
  unsigned long long dr2max_bits;   // displacement check: max |dq|^2
  int cand_weighted;                // candidate copies (real atoms and ghost images)
  int cand_n;                       // candidate copies stored
  int max_row;                      // longest neighbour row of the last build
  int want_build;                   // this step rebuilds the list
  long long list_entries;
  long long total_images;           // real atoms + ghost images (PairList Nl bound)
  long long rebuilds;
  long long steps;
  long long disp_checks;
  double zeta;                      // Nose-Hoover friction (Variables::Zeta)
  double sim_time;
  double too_fast_v;                // speed that tripped kErrTooFast
  double ext_position;              // external executor: current piston position
  double ext_impulse;               // external executor: impulse of the last pass
  // 1 while Arrays::v_lag holds the velocities of the last second half
  // drift: an executor changed v after the step, and the reconstruction of
  // the reference's half-step-old ghost copies (q - v dt/2) must use the
  // velocities the drift used.  Cleared once the next step's skin check is
  // decided, and by a rebuild (fresh copies).
  int vlag_set;
  // persistent pipeline (mdg_calculate with the persistent pass): the step
  // count the queued launches stop at, the fixed-point buffer the next
  // fused step reads (0: qfix, 1: qfix2), and the steps the persistent
  // pass took
  long long target_steps;
  int fix_parity;
  long long persistent_steps;
  unsigned long long vmax2_ring[3];  // the persistent pass's |v| maxima, step k in slot k % 3
};

// An executor the reference's projects run after every Calculate() (on the
// real atoms' momenta = velocities), applied on the device after each step.
struct External {
  int kind;          // 0 none, 1 gravity, 2 piston, 3 shell wall
  int axis;          // gravity: axis of the acceleration
  double strength;   // gravity: acceleration
  double dt;         // the time step the executor multiplies by
  double velocity;   // piston: displacement per pass (towards -z)
  double center[3];  // shell: centre
  double radius;     // shell: radius of the wall surface
};

struct Arrays {
  double4 *q, *v, *q_old;
  int4 *qfix;
  int4 *qfix2;        // second fixed-point buffer: the fused NVE step reads one and writes the other
  float4 *qloc;       // FP32 coordinates at the last build (list prefilter): x global, y z cell-local
  int *cxyz;          // packed cell coordinates of each slot at the last build
  int *xsub;          // x sub-bin starts of every cell and row ends (list-build trim table)
  int *ids, *type;
  int *cell;          // cell of each slot at the last build
  int *nbr, *nnbr;
  int *cell_count, *cell_start;
  int *slot;          // rank inside the cell from the atomic scatter
  int *perm, *perm2;  // new slot -> old slot
  double4 *q_tmp, *v_tmp;
  double4 *v_lag;     // velocities of the last second half drift (Status::vlag_set); null in slabs
  int *ids_tmp, *type_tmp, *cell_tmp;
  unsigned char *mult; // ghost-border membership at the last build (bits, see border_bits)
  int2 *cand;         // displacement-check candidates: (slot, image code)
  double *disp2;      // per atom: the largest squared copy displacement of the last skin check (k_disp_max); null: not kept
  double *partials;   // per-block partial sums for reductions
  Status *st;
  int stride;         // column stride of nbr (>= cap, multiple of 32)
  int maxnb;          // neighbour-row capacity
  // staged FP32 force (null / 0 when off)
  int4 *stage_rng;    // per block: (first cell, end cell, first atom, offset in the block's stage)
  int *stage_n;       // per block: ranges, -1 = partners gathered from global memory
  uint2 *nbr16;       // rows as stage indices, four 16-bit entries per element
  int stage_cap;      // atoms one block stages at most
};

// The FP32 prefilter band of the list build: candidates whose FP32 r^2 lies
// in [lo, hi] around SearchLength^2 are decided by the exact FP64 test.  The
// prefilter's x coordinate is the box coordinate (error up to one rounding
// of L_x) and y, z are cell-local, so with u = 2^-24 the FP32 r^2 of a
// candidate near the search length is within u (6 L_x / SL + 37) SL^2 of
// the exact value; the band is four times that, and at least 1e-4 SL^2.
inline void prefilter_band(double sl2, double sl, double lx, float *lo, float *hi) {
  const double u = 1.0 / 16777216.0;
  const double rel = fmax(1e-4, 4.0 * u * (6.0 * lx / sl + 37.0));
  *lo = (float)(sl2 * (1.0 - rel));
  *hi = (float)(sl2 * (1.0 + rel));
}

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// The skin budget's cost of one step, 2 vmax dt, each operation separately
// rounded as in PairList::IsPairListExpired (src/pairlist.cc:25-65), so
// every kernel that spends the budget spends the same amount.
__device__ __forceinline__ double skin_cost(double vmax, double dt) { return dmul(dmul(vmax, 2.0), dt); }

__device__ __forceinline__ void atomic_max_double_bits(unsigned long long *addr, double v) {
  // non-negative doubles order like their bit patterns
  atomicMax(addr, (unsigned long long)__double_as_longlong(v));
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide max of a non-negative double, one atomic per block.
template <int BLOCK>
__device__ __forceinline__ void block_max_to(unsigned long long *addr, double v) {
  __shared__ double sm[BLOCK / 32];
  v = warp_max(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sm[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (l < BLOCK / 32) ? sm[l] : 0.0;
    v = warp_max(v);
    if (l == 0) atomic_max_double_bits(addr, v);
  }
}

// Warp maximum folded into a global maximum without a block barrier, so a
// warp that finishes its rows early leaves at once; the atomic is skipped
// when the global value is already at least as large (non-negative v).
__device__ __forceinline__ void warp_max_to(unsigned long long *addr, double v) {
  v = warp_max(v);
  if ((threadIdx.x & 31) == 0 && v > 0.0) {
    const unsigned long long cur = *(volatile unsigned long long *)addr;
    const unsigned long long mine = (unsigned long long)__double_as_longlong(v);
    if (mine > cur) atomicMax(addr, mine);
  }
}

// Fixed order block sum written to partials[blockIdx.x * nsum + k].
template <int BLOCK, int NSUM>
__device__ __forceinline__ void block_sum_to(double (&v)[NSUM], double *partials) {
  __shared__ double sm[NSUM][BLOCK / 32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NSUM; k++) {
    double x = warp_sum(v[k]);
    if (l == 0) sm[k][w] = x;
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < NSUM; k++) {
      double x = (l < BLOCK / 32) ? sm[k][l] : 0.0;
      x = warp_sum(x);
      if (l == 0) partials[(size_t)blockIdx.x * NSUM + k] = x;
    }
  }
}

__device__ __forceinline__ int cell_coord(double x, double inv_cs, int ms) {
  int c = (int)(x * inv_cs);
  return c < 0 ? 0 : (c >= ms ? ms - 1 : c);
}

// Fixed-point image of one coordinate: frac(x / L) * 2^32 rounded, mod 2^32.
__device__ __forceinline__ int fixed_coord(double x, double L) {
  double u = x / L;
  u -= floor(u);
  const long long k = __double2ll_rn(u * 4294967296.0);
  return (int)(unsigned int)(unsigned long long)k;
}

// Minimum-image ghost coordinate as the reference forms it: the copy of
// atom j that lies next to atom i is q_j + diff with diff in {-L, 0, +L}
// (MDUnit::MakeBufferForBorderParticles, src/mdunit.cc:152-192).
__device__ __forceinline__ double image_of(double xj, double xi, double L, double hL) {
  const double t = xj - xi;
  if (t > hL) return dsub(xj, L);
  if (t < -hL) return dadd(xj, L);
  return xj;
}

// ---------------------------------------------------------------- kernels
// Upload indices of a fresh state: slot i holds atom i.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_upload_ids(Arrays a, int n) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  if (i < n) a.ids[i] = i;
}

// Initial |v|^2 maximum (used before the first step after an upload) and a
// finiteness check of the uploaded state.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_vmax(Arrays a, int n) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  double v2 = 0.0;
  if (i < n) {
    const double4 v = a.v[i];
    const double4 q = a.q[i];
    v2 = dadd(dadd(dmul(v.x, v.x), dmul(v.y, v.y)), dmul(v.z, v.z));
    if (!isfinite(v2) || !isfinite(q.x) || !isfinite(q.y) || !isfinite(q.z)) {
      atomicOr(&a.st->error, kErrNonFinite);
      v2 = 0.0;
    }
  }
  block_max_to<BLOCK>(&a.st->vmax2_bits, v2);
}

// PairList::IsPairListExpired (src/pairlist.cc:25-65): budget -= 2 vmax dt
// while the budget is positive (a too-fast atom is an error), then arm the
// displacement check once the budget is spent.  One thread: *disp_out = run
// the displacement check this step; returns whether the step rebuilds
// unconditionally (a stale list).
__device__ __forceinline__ int expiry_decide(Status *st, const Box &b, int *disp_out) {
  int disp = 0, build = 0;
  if (st->error == 0) {
    if (st->list_stale) {
      build = 1;
    } else {
      if (st->budget > 0.0) {
        const double vmax = sqrt(__longlong_as_double((long long)st->vmax2_bits));
        if (skin_cost(vmax, b.dt) > b.buffer_length) {
          st->too_fast_v = vmax;
          atomicOr(&st->error, kErrTooFast);
        } else {
          st->budget = dsub(st->budget, skin_cost(vmax, b.dt));
        }
      }
      if (st->error == 0 && st->budget < 0.0) {
        disp = 1;
        st->dr2max_bits = 0ull;
        st->cand_weighted = 0;
        st->cand_n = 0;
        st->disp_checks++;
      }
    }
  }
  st->want_build = build;
  st->vmax2_bits = 0ull;
  if (!disp) st->vlag_set = 0;  // no displacement check reads the ghost copies this step
  *disp_out = disp;
  return build;
}

// expiry_decide as a kernel: sets the two conditional handles of this
// step's graph (or device flags in eager mode).
static __global__ void k_expiry(Arrays a, Box b, cudaGraphConditionalHandle h_disp,
                                cudaGraphConditionalHandle h_build, int in_graph, int *eager_flags) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Status *st = a.st;
  int disp = 0;
  const int build = expiry_decide(st, b, &disp);
  // the rebuild decision when no displacement check runs; otherwise k_decide,
  // after the check, sets it again
  const int build_now = st->error == 0 && build;
  if (in_graph) {
    cudaGraphSetConditional(h_disp, disp);
    cudaGraphSetConditional(h_build, build_now);
  } else {
    eager_flags[0] = disp;
    eager_flags[1] = build_now;
  }
}

// Sets the rebuild condition of this step from the expiry and displacement
// decisions.
static __global__ void k_decide(Arrays a, cudaGraphConditionalHandle h_build, int in_graph, int *eager_flags) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int build = (a.st->error == 0) && a.st->want_build;
  a.st->vlag_set = 0;  // the displacement check has read the ghost copies
  if (in_graph) cudaGraphSetConditional(h_build, build);
  else eager_flags[1] = build;
}

// ---- ghost copies of the reference, for the skin check -----------------
// The reference checks displacements over real atoms AND their ghost
// copies (src/pairlist.cc:67-121 loops over GetTotalParticleNumber()).  A
// ghost is q + diff with diff = +L for atoms in a low-face strip and -L for a
// high-face strip, per axis, for every combination of the strips the atom was
// in at the last build (the six sequential border passes,
// src/mdmanager.cc:395-401).  Its old position is the build-time copy; its
// current one dates from the last SendBorderParticles, i.e. half a step back
// after a full NVE / Nose-Hoover step (lag = dt/2; 0 otherwise).  An image
// code holds 2 bits per axis: 0 no shift, 1 +L, 2 -L; code 0 is the atom.
__device__ __forceinline__ double image_coord(double x, int c, double L) {
  return c == 1 ? dadd(x, L) : (c == 2 ? dadd(x, -L) : x);
}

// The axis options of an atom's copies: mask bits 2d (low strip) and 2d+1
// (high strip) for axis d.
__device__ __forceinline__ int axis_options(int mask, int d, int opt[2]) {
  int k = 0;
  if (mask & (1 << (2 * d))) opt[k++] = 1;
  if (mask & (1 << (2 * d + 1))) opt[k++] = 2;
  return k;
}

// The state arrays the copy helpers read.
struct CopyView {
  const double4 *q_old, *q, *v;
  const unsigned char *mask;
};

// Old and current position of copy `code` of atom i in a box of lengths L.
__device__ __forceinline__ void copy_positions(const CopyView &cv, const double L[3], int i, int code, double lag,
                                               double old_p[3], double new_p[3]) {
  const double4 o = cv.q_old[i], q = cv.q[i];
  const double oo[3] = {o.x, o.y, o.z};
  double qq[3] = {q.x, q.y, q.z};
  if (code != 0 && lag > 0.0) {
    const double4 v = cv.v[i];
    qq[0] = dsub(q.x, dmul(v.x, lag));
    qq[1] = dsub(q.y, dmul(v.y, lag));
    qq[2] = dsub(q.z, dmul(v.z, lag));
  }
  for (int d = 0; d < 3; d++) {
    const int c = (code >> (2 * d)) & 3;
    old_p[d] = image_coord(oo[d], c, L[d]);
    new_p[d] = image_coord(qq[d], c, L[d]);
  }
}

__device__ __forceinline__ double dist2(const double a[3], const double c[3]) {
  const double dx = dsub(a[0], c[0]), dy = dsub(a[1], c[1]), dz = dsub(a[2], c[2]);
  return dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
}

// Calls f(code, d2) for every copy of atom i (the atom first), d2 the
// squared displacement since the last build as the reference forms it
// (qb_old - q, src/pairlist.cc:75-79).
template <typename F>
__device__ __forceinline__ void for_each_copy(const CopyView &cv, const double L[3], int i, double lag, F f) {
  const int mask = cv.mask[i];
  int ox[3] = {0, 0, 0}, oy[3] = {0, 0, 0}, oz[3] = {0, 0, 0};
  int tx[2], ty[2], tz[2];
  const int nx = axis_options(mask, 0, tx), ny = axis_options(mask, 1, ty), nz = axis_options(mask, 2, tz);
  for (int k = 0; k < nx; k++) ox[k + 1] = tx[k];
  for (int k = 0; k < ny; k++) oy[k + 1] = ty[k];
  for (int k = 0; k < nz; k++) oz[k + 1] = tz[k];
  for (int z = 0; z <= nz; z++)
    for (int y = 0; y <= ny; y++)
      for (int x = 0; x <= nx; x++) {
        const int code = ox[x] | (oy[y] << 2) | (oz[z] << 4);
        double op[3], np[3];
        copy_positions(cv, L, i, code, lag, op, np);
        f(code, dist2(op, np));
      }
}

// Velocities that date the ghost copies: v_lag after an executor changed v.
__device__ __forceinline__ const double4 *lag_velocities(const Arrays &a) {
  return (a.v_lag && a.st->vlag_set) ? a.v_lag : a.v;
}

__device__ __forceinline__ CopyView copy_view(const Arrays &a) {
  return CopyView{a.q_old, a.q, lag_velocities(a), a.mult};
}

// PairList::CheckByDisplacement, first pass: max |qb_old - q|^2 over all
// copies (src/pairlist.cc:67-84).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_disp_max(Arrays a, Box b, int n, double lag) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  double d2 = 0.0;
  if (i < n) for_each_copy(copy_view(a), b.L, i, lag, [&](int, double x) { d2 = fmax(d2, x); });
  if (a.disp2 && i < n) a.disp2[i] = d2;
  block_max_to<BLOCK>(&a.st->dr2max_bits, d2);
}

// Second pass: copies that moved more than BufferLength - sqrt(dr2_max)
// (src/pairlist.cc:86-97); each is stored as (slot, image code).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_disp_collect(Arrays a, Box b, int n, int cand_cap, double lag) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  if (i >= n) return;
  const double c = b.buffer_length - sqrt(__longlong_as_double((long long)a.st->dr2max_bits));
  const double c_d2 = c * c;
  // no copy of this atom moved more than c (k_disp_max's per-atom maximum
  // of the same displacements): nothing to collect
  if (a.disp2 && !(a.disp2[i] > c_d2)) return;
  for_each_copy(copy_view(a), b.L, i, lag, [&](int code, double d2) {
    if (d2 > c_d2) {
      atomicAdd(&a.st->cand_weighted, 1);
      const int k = atomicAdd(&a.st->cand_n, 1);
      if (k < cand_cap) a.cand[k] = make_int2(i, code);
    }
  });
}

// Candidate copies staged in shared memory for the pair test: old and
// current position of each, one array per axis so that consecutive lanes
// read consecutive doubles.  960 copies (45 KB) covers the reference's
// CheckListLength of 500 with room; longer lists are read from global memory.
constexpr int kPairStage = 960;

struct PairStage {
  double o[3][kPairStage], n[3][kPairStage];
};

// The pair test of PairList::CheckByDisplacement (src/pairlist.cc:99-121)
// over rows a = part, part + parts, ... of the candidate list: sets *found
// if a pair of candidate copies (a < b) that was at least SearchLength apart
// at the last build is now inside the cut-off.  Copies carry their shifts,
// so the distances are the reference's direct differences.  The result is
// an "any" over the pairs, so splitting the rows over blocks and the columns
// over threads changes only the time.  l must be the same for every thread
// of the block (the staging pass ends in a barrier).
// The same reading the copies' positions from global memory (any l).
template <int BLOCK>
__device__ __forceinline__ void candidate_pair_test_global(const CopyView &cv, const double L[3], const int2 *cand,
                                                           int l, double lag, double sl2, double rc2, int part,
                                                           int parts, volatile int *found) {
  for (int a = part; a < l - 1 && !*found; a += parts) {
    double o1[3], n1[3];
    copy_positions(cv, L, cand[a].x, cand[a].y, lag, o1, n1);
    for (int c = a + 1 + threadIdx.x; c < l; c += BLOCK) {
      double o2[3], n2[3];
      copy_positions(cv, L, cand[c].x, cand[c].y, lag, o2, n2);
      if (dist2(o1, o2) < sl2) continue;
      if (dist2(n1, n2) < rc2) *found = 1;
    }
  }
}

template <int BLOCK>
__device__ __forceinline__ void candidate_pair_test(const CopyView &cv, const double L[3], const int2 *cand, int l,
                                                    double lag, double sl2, double rc2, int part, int parts,
                                                    PairStage &sm, volatile int *found) {
  if (l <= kPairStage) {
    for (int k = threadIdx.x; k < l; k += BLOCK) {
      const int2 c = cand[k];
      double o[3], p[3];
      copy_positions(cv, L, c.x, c.y, lag, o, p);
      for (int d = 0; d < 3; d++) {
        sm.o[d][k] = o[d];
        sm.n[d][k] = p[d];
      }
    }
    __syncthreads();
    for (int a = part; a < l - 1 && !*found; a += parts) {
      const double o1[3] = {sm.o[0][a], sm.o[1][a], sm.o[2][a]};
      const double n1[3] = {sm.n[0][a], sm.n[1][a], sm.n[2][a]};
      for (int c = a + 1 + threadIdx.x; c < l; c += BLOCK) {
        const double o2[3] = {sm.o[0][c], sm.o[1][c], sm.o[2][c]};
        if (dist2(o1, o2) < sl2) continue;
        const double n2[3] = {sm.n[0][c], sm.n[1][c], sm.n[2][c]};
        if (dist2(n1, n2) < rc2) *found = 1;
      }
    }
  } else {
    candidate_pair_test_global<BLOCK>(cv, L, cand, l, lag, sl2, rc2, part, parts, found);
  }
}

// Third pass, kPairParts blocks sharing the rows: expired if the copies
// found reach min(total copies, CheckListLength), or if the pair test finds
// a pair (src/pairlist.cc:86-121).
constexpr int kPairParts = 16;

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_disp_pairs(Arrays a, Box b, double lag) {
  __shared__ PairStage sm;
  __shared__ volatile int found;
  if (threadIdx.x == 0) found = 0;
  __syncthreads();
  Status *st = a.st;
  const long long tn = st->total_images;
  const int nl = (int)((tn > b.check_list_length) ? b.check_list_length : tn);
  if (st->cand_weighted >= nl) {
    if (threadIdx.x == 0) found = 1;
  } else {
    const int l = min(st->cand_n, b.check_list_length);
    candidate_pair_test<BLOCK>(copy_view(a), b.L, a.cand, l, lag, b.sl2, b.rc2, blockIdx.x, gridDim.x, sm, &found);
  }
  __syncthreads();
  if (threadIdx.x == 0 && found) st->want_build = 1;
}

// ------------------------------------------------------ staged partners
// The FP32-mixed force pass stages, per block of kStageBlock consecutive
// atoms, the fixed-point positions of every atom in the union of the
// block's 27-cell stencils in shared memory, and reads partners from there.
// Atoms are in cell order, so that union is a few runs of consecutive cells
// (the stencil rows of the block's home cells), i.e. a few runs of
// consecutive atoms, which the pass copies with bulk asynchronous copies.
// Rows hold, besides the global partner index, its index in the stage
// (16 bits, four per 8-byte element).  The pair terms and their order are
// the global-gather pass's; only where the positions are read from changes.
constexpr int kStageBlock = 128;
constexpr int kStageRanges = 32;
constexpr int kStageRaw = 96;  // stencil-row cell runs per block before merging

// Offset from a global atom index to its stage index, for an atom of cell nc:
// the plan range that holds nc (ranges are sorted by first cell).
__device__ __forceinline__ int stage_shift(const int4 *plan, int npl, int nc) {
  int lo = 0, hi = npl - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (plan[mid].x <= nc) lo = mid;
    else hi = mid - 1;
  }
  return plan[lo].w - plan[lo].z;
}

// Entry k of atom i's staged row: four 16-bit entries per uint2, written
// when the fourth arrives (rows are padded to a multiple of 4).
__device__ __forceinline__ void stage_entry(uint2 *nbr16, int stride, int i, int k, int v, unsigned &g0,
                                            unsigned &g1) {
  const unsigned val = (unsigned)v & 0xffffu;
  switch (k & 3) {
    case 0: g0 = val; g1 = 0u; break;
    case 1: g0 |= val << 16; break;
    case 2: g1 = val; break;
    default:
      g1 |= val << 16;
      nbr16[(size_t)(k >> 2) * stride + i] = make_uint2(g0, g1);
  }
}

// Rebuild, after the permutation and the cell scan: the stage plan of every
// block of kStageBlock atoms, one thread per block.  The block's home cells
// lie in [cell of its first atom, cell of its last atom]; each run of them
// along x contributes, per (dz, dy), the cells x-1 .. x+1 of that row (one
// or two runs with the periodic wrap).  The runs are sorted and merged; a
// block that needs more than kStageRanges runs or more than stage_cap atoms
// is marked -1 and gathers its partners from global memory.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_stage_plan(Arrays a, Box b, int n) {
  const int blk = blockIdx.x * BLOCK + threadIdx.x;
  const int nblk = (n + kStageBlock - 1) / kStageBlock;
  if (blk >= nblk || a.st->error) return;
  const int i0 = blk * kStageBlock, i1 = min(n, i0 + kStageBlock) - 1;
  const int c_first = a.cell_tmp[i0], c_last = a.cell_tmp[i1];
  const int ms0 = b.ms[0], ms1 = b.ms[1], ms2 = b.ms[2];
  int2 run[kStageRaw];
  int nrun = 0;
  bool over = false;
  for (int c = c_first; c <= c_last && !over;) {
    const int xa = c % ms0, y = (c / ms0) % ms1, z = c / (ms0 * ms1);
    const int xb = min(ms0 - 1, xa + (c_last - c));
    c += xb - xa + 1;
    if (nrun + 18 > kStageRaw) {
      over = true;
      break;
    }
    const int lo = xa - 1, hi = xb + 1;  // inclusive, before the wrap
    int s0, e0, s1 = 0, e1 = 0;
    if (hi - lo + 1 >= ms0) {
      s0 = 0; e0 = ms0;
    } else if (lo < 0) {
      s0 = 0; e0 = hi + 1; s1 = lo + ms0; e1 = ms0;
    } else if (hi >= ms0) {
      s0 = 0; e0 = hi - ms0 + 1; s1 = lo; e1 = ms0;
    } else {
      s0 = lo; e0 = hi + 1;
    }
    for (int dz = -1; dz <= 1; dz++) {
      const int zz = (z + dz + ms2) % ms2;
      for (int dy = -1; dy <= 1; dy++) {
        const int base = (zz * ms1 + (y + dy + ms1) % ms1) * ms0;
        run[nrun++] = make_int2(base + s0, base + e0);
        if (e1 > s1) run[nrun++] = make_int2(base + s1, base + e1);
      }
    }
  }
  int m = 0;
  if (!over) {
    for (int k = 1; k < nrun; k++) {  // insertion sort by first cell
      const int2 x = run[k];
      int j = k - 1;
      while (j >= 0 && run[j].x > x.x) {
        run[j + 1] = run[j];
        j--;
      }
      run[j + 1] = x;
    }
    for (int k = 0; k < nrun; k++) {  // merge overlapping and touching runs
      if (m > 0 && run[k].x <= run[m - 1].y) run[m - 1].y = max(run[m - 1].y, run[k].y);
      else run[m++] = run[k];
    }
    over = m > kStageRanges;
  }
  int total = 0;
  if (!over) {
    for (int r = 0; r < m; r++) {
      const int first = a.cell_start[run[r].x];
      a.stage_rng[blk * kStageRanges + r] = make_int4(run[r].x, run[r].y, first, total);
      total += a.cell_start[run[r].y] - first;
    }
    over = total > a.stage_cap;
  }
  a.stage_n[blk] = over ? -1 : m;
}

// ------------------------------------------------------------- list build
// x sub-bins per cell of the list build's trim table (see xsub above).
constexpr int kXSub = 8;

// Cell coordinates packed into one int (x and y below 2048, z below 1024).
__device__ __forceinline__ int pack_cell(int cx, int cy, int cz) { return cx | (cy << 11) | (cz << 22); }

// Trim-table entries of a cell: the block of its x-row, at its x position.
__device__ __forceinline__ int *trim_entries(int *tab, int ms0, int row, int cx) {
  return tab + (size_t)row * (ms0 * kXSub + 1) + cx * kXSub;
}

// One warp orders the cnt slots perm[beg, beg + cnt) of a cell by (x, upload
// id) into perm2 and writes the cell's entries of the trim table: ent[k] =
// beg + (atoms with x < x0 + k bin), k < kXSub, and for the last cell of a
// row (last) the row's end ent[kXSub] = beg + cnt.  Ties in x (a lattice) go
// by id, so the order is a function of the state alone.
__device__ __forceinline__ void sort_cell_x(const double4 *q, const int *ids, const int *perm, int *perm2, int beg,
                                            int cnt, double x0, double bin, int *ent, bool last, int lane) {
  int below[kXSub];
#pragma unroll
  for (int k = 0; k < kXSub; k++) below[k] = 0;
  for (int base = 0; base < cnt; base += 32) {
    const int me = base + lane;
    int my_slot = -1, my_id = 0x7fffffff;
    double my_x = 0.0;
    if (me < cnt) {
      my_slot = perm[beg + me];
      my_x = q[my_slot].x;
      my_id = ids[my_slot];
    }
    int rank = 0;
    for (int ob = 0; ob < cnt; ob += 32) {
      const int other = ob + lane;
      double ox = 0.0;
      int oid = 0x7fffffff;
      if (other < cnt) {
        const int os = perm[beg + other];
        ox = q[os].x;
        oid = ids[os];
      }
      const int lim = min(32, cnt - ob);
      for (int k = 0; k < lim; k++) {
        const double kx = __shfl_sync(0xffffffffu, ox, k);
        const int kid = __shfl_sync(0xffffffffu, oid, k);
        rank += (kx < my_x || (kx == my_x && kid < my_id)) ? 1 : 0;
      }
    }
    if (me < cnt) perm2[beg + rank] = my_slot;
#pragma unroll
    for (int k = 1; k < kXSub; k++)
      below[k] += __popc(__ballot_sync(0xffffffffu, me < cnt && my_x < x0 + k * bin));
  }
  int v = 0;
#pragma unroll
  for (int k = 1; k < kXSub; k++)
    if (lane == k) v = below[k];
  if (lane < kXSub) ent[lane] = beg + v;
  if (last && lane == 0) ent[kXSub] = beg + cnt;
}

// Rebuild 1/6: wrap into [0,L] (Variables::AdjustPeriodicBoundary,
// src/variables.cc:63-84), validity check, cell index and rank inside the cell.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_cell_assign(Arrays a, Box b, int n) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  if (i >= n || a.st->error) return;
  double4 q = a.q[i];
  double x[3] = {q.x, q.y, q.z};
  int cc[3];
  bool bad = false;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (!isfinite(x[d])) {
      atomicOr(&a.st->error, kErrNonFinite);
      return;
    }
    if (x[d] < 0.0) x[d] = dadd(x[d], b.L[d]);
    else if (x[d] > b.L[d]) x[d] = dsub(x[d], b.L[d]);
    bad |= (x[d] < 0.0 || x[d] > b.L[d]);
    cc[d] = cell_coord(x[d], b.inv_cs[d], b.ms[d]);
  }
  if (bad) {
    atomicOr(&a.st->error, kErrInvalidPosition);
    return;
  }
  q.x = x[0]; q.y = x[1]; q.z = x[2];
  a.q[i] = q;
  if (b.slab) {  // the slab's own layers only (migration moved every other atom away)
    cc[2] -= b.z0;
    if (cc[2] < 0 || cc[2] >= b.nzl) {
      atomicOr(&a.st->error, kErrInvalidPosition);
      return;
    }
  }
  const int c = (cc[2] * b.ms[1] + cc[1]) * b.ms[0] + cc[0];
  a.cell[i] = c;
  a.slot[i] = atomicAdd(&a.cell_count[c], 1);
}

template <int BLOCK>
__device__ __forceinline__ int block_exclusive_scan(int x, int *total) {
  __shared__ int warp_tot[BLOCK / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_tot[w] = inc;
  __syncthreads();
  if (w == 0) {
    int t = lane < BLOCK / 32 ? warp_tot[lane] : 0;
    int ti = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, ti, o);
      if (lane >= o) ti += y;
    }
    if (lane < BLOCK / 32) warp_tot[lane] = ti - t;
    if (lane == BLOCK / 32 - 1) *total = ti;
  }
  __syncthreads();
  const int r = warp_tot[w] + inc - x;
  __syncthreads();
  return r;
}

// Rebuild 2/6: exclusive scan of the cell counts in three passes -- tiles of
// BLOCK cells scanned in parallel, the tile totals scanned by one block,
// the tile offsets added back.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_scan_tiles(Arrays a, int ncell, int *tile_sum) {
  __shared__ int total;
  if (a.st->error) return;
  const int c = blockIdx.x * BLOCK + threadIdx.x;
  const int x = c < ncell ? a.cell_count[c] : 0;
  const int ex = block_exclusive_scan<BLOCK>(x, &total);
  if (c < ncell) a.cell_start[c] = ex;
  if (threadIdx.x == 0) tile_sum[blockIdx.x] = total;
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_scan_tile_sums(Arrays a, int ncell, int *tile_sum, int ntiles) {
  __shared__ int total;
  if (a.st->error) return;
  int carry = 0;
  for (int base = 0; base < ntiles; base += BLOCK) {
    const int k = base + threadIdx.x;
    const int x = k < ntiles ? tile_sum[k] : 0;
    const int ex = block_exclusive_scan<BLOCK>(x, &total);
    if (k < ntiles) tile_sum[k] = carry + ex;
    carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) a.cell_start[ncell] = carry;
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_scan_add(Arrays a, int ncell, const int *tile_sum) {
  if (a.st->error) return;
  const int c = blockIdx.x * BLOCK + threadIdx.x;
  if (c < ncell && blockIdx.x > 0) a.cell_start[c] += tile_sum[blockIdx.x];
}

// The same in one block, for grids of few cells: the carry runs over
// chunks of BLOCK cells (one launch instead of three).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_scan_single(Arrays a, int ncell) {
  __shared__ int total;
  if (a.st->error) return;
  int carry = 0;
  for (int base = 0; base < ncell; base += BLOCK) {
    const int c = base + threadIdx.x;
    const int x = c < ncell ? a.cell_count[c] : 0;
    const int ex = block_exclusive_scan<BLOCK>(x, &total);
    if (c < ncell) a.cell_start[c] = carry + ex;
    carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) a.cell_start[ncell] = carry;
}

// Rebuild 3/6: scatter old slots to their cell ranges.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_scatter(Arrays a, int n) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  if (i >= n || a.st->error) return;
  a.perm[a.cell_start[a.cell[i]] + a.slot[i]] = i;
}

// Rebuild 4/6: order every cell by (x, upload id), one warp per cell, which
// makes the slot order a function of the state alone (independent of
// atomics) and puts each cell's atoms in x order for the list build's trim
// table; the cell's row of that table is written too (sort_cell_x).
static __global__ void k_sort_cells(Arrays a, Box b, int ncell) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= ncell || a.st->error) return;
  const int beg = a.cell_start[warp], cnt = a.cell_start[warp + 1] - beg;
  const int cx = warp % b.ms[0];
  sort_cell_x(a.q, a.ids, a.perm, a.perm2, beg, cnt, cx * b.cs[0], b.cs[0] / kXSub,
              trim_entries(a.xsub, b.ms[0], warp / b.ms[0], cx), cx == b.ms[0] - 1, lane);
}

// Ghost-strip membership of a wrapped position at a build: bit 2d for
// 0 < x_d < SL, bit 2d+1 for L_d - SL < x_d < L_d (MDRect::IsInsideEdge,
// src/mdrect.cc:23-47); the copies are every combination of the strips, so
// their count including the atom is the product over axes of (1 + bits).
__device__ __forceinline__ int border_bits(const double x[3], const Box &b, int *copies) {
  int mask = 0, m = 1;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const int lo = (x[d] < b.sl && x[d] > 0.0) ? 1 : 0;
    const int hi = (x[d] > b.L[d] - b.sl && x[d] < b.L[d]) ? 1 : 0;
    mask |= (lo << (2 * d)) | (hi << (2 * d + 1));
    m *= 1 + lo + hi;
  }
  *copies = m;
  return mask;
}

// Rebuild 5/6: gather into cell order (temporary arrays), snapshot q_old
// (PairList::Init), ghost-strip membership and the total copy count.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_permute(Arrays a, Box b, int n, int4 *pack) {
  const int s = blockIdx.x * BLOCK + threadIdx.x;
  int m = 0;
  if (s < n && !a.st->error) {
    const int o = a.perm2[s];
    const double4 q = a.q[o];
    a.q_tmp[s] = q;
    a.v_tmp[s] = a.v[o];
    a.ids_tmp[s] = a.ids[o];
    a.type_tmp[s] = a.type[o];
    a.cell_tmp[s] = a.cell[o];
    a.q_old[s] = q;
    const double x[3] = {q.x, q.y, q.z};
    a.mult[s] = (unsigned char)border_bits(x, b, &m);
    // FP32 coordinates for the list prefilter (x in box coordinates, y and z
    // relative to the cell) and the packed cell coordinates
    const int c = a.cell_tmp[s];
    const int cx = c % b.ms[0], cy = (c / b.ms[0]) % b.ms[1], cz = c / (b.ms[0] * b.ms[1]);
    const int gz = cz + b.z0;  // global layer (the local one in a slab)
    a.qloc[s] = make_float4((float)q.x, (float)(q.y - cy * b.cs[1]), (float)(q.z - gz * b.cs[2]), 0.f);
    a.cxyz[s] = pack_cell(cx, cy, cz);
    if (pack) {
      // the coming step's first-drift positions for the fused FP32 NVE pass
      const double4 v = a.v[o];
      const double dt2 = b.dt * 0.5;
      pack[s] = make_int4(fixed_coord(dadd(q.x, dmul(v.x, dt2)), b.L[0]),
                          fixed_coord(dadd(q.y, dmul(v.y, dt2)), b.L[1]),
                          fixed_coord(dadd(q.z, dmul(v.z, dt2)), b.L[2]), 0);
    }
  }
  const int tot = __reduce_add_sync(0xffffffffu, m);
  if ((threadIdx.x & 31) == 0 && tot) atomicAdd((unsigned long long *)&a.st->total_images, (unsigned long long)tot);
}

// Strip bits a partner needs for its ghost copy with shift (sx, sy, sz) to
// exist: +L images come from the low-face strip, -L images from the high-face
// strip (MDUnit::MakeBufferForBorderParticles, src/mdunit.cc:156-192).  A
// partner outside the strip -- e.g. exactly on a face, which the strict
// MDRect::IsInsideEdge test leaves out (src/mdrect.cc:27-43) -- has no copy
// there, and the reference's search does not see that pair from this side.
__device__ __forceinline__ int needed_strips(double sx, double sy, double sz) {
  return (sx > 0.0 ? 1 : 0) | (sx < 0.0 ? 2 : 0) | (sy > 0.0 ? 4 : 0) | (sy < 0.0 ? 8 : 0) |
         (sz > 0.0 ? 16 : 0) | (sz < 0.0 ? 32 : 0);
}

// Exact test of one candidate, the reference's arithmetic
// (MeshList::SearchMesh, src/meshlist.cc:276-289): ghost image q_j + diff
// first, then dx = x_i - image, then ((dx*dx + dy*dy) + dz*dz), each
// operation separately rounded; kept when r^2 <= SearchLength^2.
__device__ __forceinline__ bool within_search_exact(const double4 &qi, const double4 &qj, double sx, double sy,
                                                    double sz, double sl2) {
  const double gx = dadd(qj.x, sx), gy = dadd(qj.y, sy), gz = dadd(qj.z, sz);
  const double ex = dsub(qi.x, gx), ey = dsub(qi.y, gy), ez = dsub(qi.z, gz);
  const double r2 = dadd(dadd(dmul(ex, ex), dmul(ey, ey)), dmul(ez, ez));
  return !(r2 > sl2);
}

// Image shift of a stencil piece, 2 bits per axis (0: none, 1: -L, 2: +L).
__device__ __forceinline__ double shift_of(int code, int d, const double L[3]) {
  const int c = (code >> (2 * d)) & 3;
  return c == 1 ? -L[d] : (c == 2 ? L[d] : 0.0);
}

// The exact test of candidate j of atom i through image shift `shift`
// (within_search_exact).  Reached only for candidates in the FP32 band, so
// the FP64 positions and shifts are read here rather than held in registers
// across the candidate loop.
__device__ __forceinline__ bool band_test(const double4 *__restrict__ q, int i, int j, int shift, const Box &b) {
  return within_search_exact(q[i], q[j], shift_of(shift, 0, b.L), shift_of(shift, 1, b.L), shift_of(shift, 2, b.L),
                             b.sl2);
}

// Candidates [beg, end) of one stencil row of atom i, in slot order: FP32
// prefilter r^2 <= hi on the prefilter coordinates moved by the row's base
// (bx, by, bz); the ghost-existence rule for image shifts (NEED); the exact
// FP64 test for candidates in the band [lo, hi] (band_test, image shift
// `shift`); emit(j, k) files partner j as entry k of the row.  SELF: the
// range holds atom i itself.  Four loads are issued before the first test.
//
// With BTPA lanes per atom (the lanes of one atom are consecutive and all
// walk the same ranges), lane s tests candidates beg + s, beg + BTPA + s, ...
// and the lanes file the ones they keep in slot order through a ballot over
// the atom's lanes, so the row is the same for every lane count; cnt stays
// equal on all of them.
template <bool NEED, bool SELF, int BTPA, bool PIPE, typename Emit>
__device__ __forceinline__ void build_range(const float4 *__restrict__ qloc, const double4 *__restrict__ q,
                                            const unsigned char *__restrict__ mult, int beg, int end, float bx,
                                            float by, float bz, int need, int shift, const Box &b, int i, int &cnt,
                                            Emit &emit) {
  auto keep_of = [&](int j, const float4 &l) {
    const float ex = l.x + bx, ey = l.y + by, ez = l.z + bz;
    const float r2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
    bool keep = r2 <= b.sl2_hi;
    if (SELF) keep = keep && j != i;
    if (NEED) keep = keep && (mult[j] & need) == need;
    if (keep && r2 >= b.sl2_lo) keep = band_test(q, i, j, shift, b);
    return keep;
  };
  if (BTPA == 1) {
    // four candidates at a time: the four prefilter tests are independent
    // (one pass over them), the rare band candidates are decided in one
    // branch, then the kept ones are filed in slot order; the loads run one
    // batch ahead
    auto prefilter = [&](int j, const float4 &l, float &r2) {
      const float ex = l.x + bx, ey = l.y + by, ez = l.z + bz;
      r2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
      bool keep = r2 <= b.sl2_hi;
      if (SELF) keep = keep && j != i;
      return keep;
    };
    // PIPE: the next four candidates' loads are issued before this four's
    // tests (four more float4 registers)
    int j = beg;
    float4 n0, n1, n2, n3;
    if (PIPE && j + 4 <= end) {
      n0 = __ldg(qloc + j);
      n1 = __ldg(qloc + j + 1);
      n2 = __ldg(qloc + j + 2);
      n3 = __ldg(qloc + j + 3);
    }
    for (; j + 4 <= end; j += 4) {
      float4 l0, l1, l2, l3;
      if (PIPE) {
        l0 = n0;
        l1 = n1;
        l2 = n2;
        l3 = n3;
        if (j + 8 <= end) {
          n0 = __ldg(qloc + j + 4);
          n1 = __ldg(qloc + j + 5);
          n2 = __ldg(qloc + j + 6);
          n3 = __ldg(qloc + j + 7);
        }
      } else {
        l0 = __ldg(qloc + j);
        l1 = __ldg(qloc + j + 1);
        l2 = __ldg(qloc + j + 2);
        l3 = __ldg(qloc + j + 3);
      }
      float r0, r1, r2, r3;
      bool k0 = prefilter(j, l0, r0), k1 = prefilter(j + 1, l1, r1), k2 = prefilter(j + 2, l2, r2),
           k3 = prefilter(j + 3, l3, r3);
      if (NEED) {
        k0 = k0 && (mult[j] & need) == need;
        k1 = k1 && (mult[j + 1] & need) == need;
        k2 = k2 && (mult[j + 2] & need) == need;
        k3 = k3 && (mult[j + 3] & need) == need;
      }
      const float lo = b.sl2_lo;
      if ((k0 && r0 >= lo) || (k1 && r1 >= lo) || (k2 && r2 >= lo) || (k3 && r3 >= lo)) {
        if (k0 && r0 >= lo) k0 = band_test(q, i, j, shift, b);
        if (k1 && r1 >= lo) k1 = band_test(q, i, j + 1, shift, b);
        if (k2 && r2 >= lo) k2 = band_test(q, i, j + 2, shift, b);
        if (k3 && r3 >= lo) k3 = band_test(q, i, j + 3, shift, b);
      }
      if (k0) emit(j, cnt);
      cnt += k0;
      if (k1) emit(j + 1, cnt);
      cnt += k1;
      if (k2) emit(j + 2, cnt);
      cnt += k2;
      if (k3) emit(j + 3, cnt);
      cnt += k3;
    }
    for (; j < end; j++) {
      if (keep_of(j, __ldg(qloc + j))) {
        emit(j, cnt);
        cnt++;
      }
    }
  } else {
    const int lane = threadIdx.x & 31, sub = lane & (BTPA - 1), first = lane & ~(BTPA - 1);
    const unsigned gmask = (BTPA == 32) ? 0xffffffffu : (((1u << BTPA) - 1u) << first);
    const unsigned below = (1u << sub) - 1u;
    auto file = [&](int j, bool keep) {
      const unsigned m = __ballot_sync(gmask, keep) >> first;
      if (keep) emit(j, cnt + __popc(m & below));
      cnt += __popc(m);
    };
    for (int base = beg; base < end; base += 2 * BTPA) {
      const int j0 = base + sub, j1 = base + BTPA + sub;
      float4 l0 = make_float4(0.f, 0.f, 0.f, 0.f), l1 = l0;
      if (j0 < end) l0 = __ldg(qloc + j0);
      if (j1 < end) l1 = __ldg(qloc + j1);
      const bool k0 = j0 < end && keep_of(j0, l0);
      const bool k1 = j1 < end && keep_of(j1, l1);
      file(j0, k0);
      file(j1, k1);
    }
  }
}

// The full Verlet row of atom i (MeshList::SearchMesh's pair set, src/
// meshlist.cc:242-292, seen from i): the 27 cells around i's own cell
// (periodic, >= 3 cells per axis so they are distinct) are walked as 9 rows
// along x.  Cells of a row are consecutive in slot order and atoms inside a
// cell are in x order, so one row is one contiguous slot range (two or
// three where the periodic wrap splits it), trimmed at both ends through the
// trim table to the sub-bins that reach within SearchLength of x_i; rows
// whose y-z gap to i already exceeds SearchLength are skipped.  Row order:
// rows in (dz, dy) order, then x order across the row's cells -- the cells
// in dx order, as a 27-cell walk visits them.  Returns the partners found
// (entries beyond the capacity are counted, not filed).
template <bool SLAB = false, int BTPA = 1, bool PIPE = true, typename Emit>
__device__ __forceinline__ int build_rows(const Box &b, const float4 *__restrict__ qloc,
                                          const double4 *__restrict__ q, const unsigned char *__restrict__ mult,
                                          const int *__restrict__ tab, int pc, int i, Emit &emit) {
  const float4 li = qloc[i];
  const int cx = pc & 2047, cy = (pc >> 11) & 2047, lz = pc >> 22;
  const int cz = SLAB ? b.z0 + lz : lz;  // global layer
  const int ms0 = b.ms[0], ms1 = b.ms[1], ms2 = b.ms[2];
  const float hi = b.sl2_hi;
  const int mx = ms0 * kXSub;
  // x_i in sub-bins from the start of the virtual row of cells cx-1 .. cx+1
  // (unwrapped x; bins of width cs/kXSub from each cell's lower face, as the
  // trim table counts them), and the x bases of the three pieces (image
  // shifts -L, 0, +L; prefilter x is global)
  const int vbase = (cx - 1) * kXSub;
  float ubin, per_binf, bxm, bx0, bxp;
  {
    const double qx = q[i].x;
    const double cs0 = b.cs[0], per_bin = kXSub / cs0;
    ubin = (float)((qx - (cx - 1) * cs0) * per_bin);
    per_binf = (float)per_bin;
    bxm = (float)(-b.L[0] - qx);
    bx0 = (float)(-qx);
    bxp = (float)(b.L[0] - qx);
  }
  const float csy = (float)b.cs[1], csz = (float)b.cs[2];
  int cnt = 0;
  for (int dz = -1; dz <= 1; dz++) {
    int z = cz + dz, zc = 0;  // zc: the row's image shift along z (shift_of's code)
    if (z < 0) { z += ms2; zc = 1; } else if (z >= ms2) { z -= ms2; zc = 2; }
    const double sz = zc == 1 ? -b.L[2] : (zc == 2 ? b.L[2] : 0.0);
    const float bz = (float)((z - cz) * b.cs[2] + sz) - li.z;
    const float gz = dz == 0 ? 0.f : (dz < 0 ? li.z : csz - li.z);
    // the layer's block of trim-table rows: the global layer in a single
    // domain; in a slab an owned local layer or one of the two ghost blocks
    int blk = z;
    if (SLAB) {
      const int nl = lz + dz;
      blk = nl < 0 ? b.nzl : (nl >= b.nzl ? b.nzl + 1 : nl);
    }
    for (int dy = -1; dy <= 1; dy++) {
      const float gy = dy == 0 ? 0.f : (dy < 0 ? li.y : csy - li.y);
      const float g2 = fmaf(gy, gy, gz * gz);
      if (g2 > hi) continue;  // the whole row is out of reach
      // sub-bins [vlo, vhi) of the row that can hold a partner: every bin
      // that reaches x_i -/+ sqrt(hi - g2), the x reach left by the row's
      // y-z gap g (hi is above SearchLength^2 by more than the FP32 error of
      // g2; the bin edges get 1e-3 of a bin more)
      const float reach = sqrtf(hi - g2) * per_binf;
      int vlo = vbase + (int)floorf(ubin - reach - 1e-3f);
      int vhi = vbase + (int)floorf(ubin + reach + 1e-3f) + 1;
      vlo = max(vlo, vbase);
      vhi = min(vhi, vbase + 3 * kXSub);
      int y = cy + dy, yc = 0;
      if (y < 0) { y += ms1; yc = 1; } else if (y >= ms1) { y -= ms1; yc = 2; }
      const double sy = yc == 1 ? -b.L[1] : (yc == 2 ? b.L[1] : 0.0);
      const float by = (float)((y - cy) * b.cs[1] + sy) - li.y;
      const int *xr = tab + (size_t)(blk * ms1 + y) * (mx + 1);
      const int yz = (yc << 2) | (zc << 4);
      if (vlo < 0)  // through the -x face: the row's last cells, image shift -L
        build_range<true, false, BTPA, PIPE>(qloc, q, mult, xr[vlo + mx], xr[mx], bxm, by, bz,
                                       needed_strips(-b.L[0], sy, sz), 1 | yz, b, i, cnt, emit);
      {
        const int a0 = max(vlo, 0), a1 = min(vhi, mx);
        const int beg = xr[a0], end = xr[a1];
        const int need = needed_strips(0.0, sy, sz);
        if (dz == 0 && dy == 0)
          build_range<false, true, BTPA, PIPE>(qloc, q, mult, beg, end, bx0, by, bz, 0, yz, b, i, cnt, emit);
        else if (need)
          build_range<true, false, BTPA, PIPE>(qloc, q, mult, beg, end, bx0, by, bz, need, yz, b, i, cnt, emit);
        else
          build_range<false, false, BTPA, PIPE>(qloc, q, mult, beg, end, bx0, by, bz, 0, yz, b, i, cnt, emit);
      }
      if (vhi > mx)  // through the +x face: the row's first cells, image shift +L
        build_range<true, false, BTPA, PIPE>(qloc, q, mult, xr[0], xr[vhi - mx], bxp, by, bz,
                                       needed_strips(b.L[0], sy, sz), 2 | yz, b, i, cnt, emit);
    }
  }
  return cnt;
}

// Stage offset of global slot j: the plan range whose atoms hold j (ranges
// are sorted by first cell, so by first atom).
__device__ __forceinline__ int stage_shift_atom(const int4 *plan, int npl, int j) {
  int lo = 0, hi = npl - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (plan[mid].z <= j) lo = mid;
    else hi = mid - 1;
  }
  return plan[lo].w - plan[lo].z;
}

// Rebuild 6/6: full Verlet list, one thread per atom (build_rows).  Each
// candidate is first tested in FP32; only candidates whose FP32 r^2 falls in
// a band around SearchLength^2 -- wider than the FP32 error bound, which
// mdg_create derives from the box -- are decided by the exact FP64 test, so
// the pair set is the reference's bit for bit.  Rows are padded with the
// atom's own index to a multiple of 4.
template <int BLOCK, bool STAGE, bool SLAB = false, int BTPA = 1>
__global__ void __launch_bounds__(BLOCK) k_build(Arrays a, Box b, int n) {
  static_assert(!(STAGE && SLAB), "staged rows are single-domain only");
  static_assert(!STAGE || BTPA == 1, "staged rows are built one lane per atom");
  const int t = blockIdx.x * BLOCK + threadIdx.x;
  const int i = t / BTPA, sub = t % BTPA;
  int cnt = 0;
  // STAGE: also the rows as stage indices (FP32-mixed staged force), from
  // the block's stage plan, see k_stage_plan
  __shared__ int4 plan[STAGE ? kStageRanges : 1];
  __shared__ int nplan;
  __shared__ int nstaged;
  int npl = -1, staged_atoms = 0;
  if (STAGE) {
    static_assert(!STAGE || BLOCK == kStageBlock, "stage plans are per kStageBlock atoms");
    if (threadIdx.x == 0) {
      const int m = a.nbr16 ? a.stage_n[blockIdx.x] : -1;
      nplan = (m > 0 && m <= kStageRanges) ? m : -1;
    }
    __syncthreads();
    npl = nplan;
    if ((int)threadIdx.x < npl) plan[threadIdx.x] = a.stage_rng[blockIdx.x * kStageRanges + threadIdx.x];
    __syncthreads();
    if (threadIdx.x == 0 && npl > 0) {
      const int4 last = plan[npl - 1];
      nstaged = last.w + a.cell_start[last.y] - last.z;
    }
    __syncthreads();
    // a stage index outside the stage would be a plan that misses a stencil
    // cell: flagged, and the entry points at the atom's own slot 0 instead
    staged_atoms = npl > 0 ? nstaged : 0;
  }
  unsigned g0 = 0u, g1 = 0u;  // the row's current group of four stage indices
  // one decision per atom: the lanes of an atom must walk its rows together
  // (their ballots name each other), so they all see its first lane's read
  // of the error flag
  int err = a.st->error;
  if (BTPA > 1) err = __shfl_sync(0xffffffffu, err, (threadIdx.x & 31) & ~(BTPA - 1));
  if (i < n && !err) {
    const int maxnb = a.maxnb, stride = a.stride;
    int *__restrict__ nbr = a.nbr;
    auto emit = [&](int j, int k) {
      if (k >= maxnb) return;
      nbr[(size_t)k * stride + i] = j;
      if (STAGE && npl > 0) {
        int v = j + stage_shift_atom(plan, npl, j);
        if (v < 0 || v >= staged_atoms) {
          atomicOr(&a.st->error, kErrStage);
          v = 0;
        }
        stage_entry(a.nbr16, stride, i, k, v, g0, g1);
      }
    };
    cnt = build_rows<SLAB, BTPA>(b, a.qloc, a.q, a.mult, a.xsub, a.cxyz[i], i, emit);
    if (sub == 0) a.nnbr[i] = min(cnt, maxnb);
    if (cnt > maxnb) {
      if (sub == 0) atomicOr(&a.st->error, kErrCapacity);
    } else if (sub == 0) {
      int self = (STAGE && npl > 0) ? i + stage_shift(plan, npl, a.cell_tmp[i]) : 0;
      if (STAGE && npl > 0 && (self < 0 || self >= staged_atoms)) {
        atomicOr(&a.st->error, kErrStage);
        self = 0;
      }
      for (int k = cnt; k < ((cnt + 3) & ~3); k++) {
        nbr[(size_t)k * stride + i] = i;
        if (STAGE && npl > 0) stage_entry(a.nbr16, stride, i, k, self, g0, g1);
      }
    }
  }
  if (sub != 0) cnt = 0;  // the atom's row is counted once
  const int wmax = __reduce_max_sync(0xffffffffu, cnt);
  const int wsum = __reduce_add_sync(0xffffffffu, cnt);
  if ((threadIdx.x & 31) == 0 && wsum) {
    atomicMax(&a.st->max_row, wmax);
    atomicAdd((unsigned long long *)&a.st->list_entries, (unsigned long long)wsum);
  }
}

// Before a build: clear the build counters.
static __global__ void k_build_begin(Arrays a) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  a.st->max_row = 0;
  a.st->list_entries = 0;
  a.st->total_images = 0;
}

// k_build_begin and the clear of the cell counts in one launch.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_build_begin_clear(Arrays a, int ncell) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    a.st->max_row = 0;
    a.st->list_entries = 0;
    a.st->total_images = 0;
  }
  for (int c = blockIdx.x * BLOCK + threadIdx.x; c < ncell; c += gridDim.x * BLOCK) a.cell_count[c] = 0;
}

// The permuted state back into place (q, v, ids, types), one launch.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_copy_back(Arrays a, int n) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  if (i >= n) return;
  a.q[i] = a.q_tmp[i];
  a.v[i] = a.v_tmp[i];
  a.ids[i] = a.ids_tmp[i];
  a.type[i] = a.type_tmp[i];
}

// After a build: fresh skin budget (PairList::Init, src/pairlist.cc:10-23),
// counters, |v|^2 max for the next expiry test is untouched.
static __global__ void k_build_done(Arrays a, Box b) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Status *st = a.st;
  if (st->error) return;
  st->budget = b.buffer_length;
  st->list_stale = 0;
  st->vlag_set = 0;  // fresh ghost copies, and v_lag is in the old slot order
  st->rebuilds++;
}

// q += v dt/2 (ForceCalculator::UpdatePositionHalf, src/fcalculator.cc:17-30);
// FIX also writes the fixed-point copy used by the FP32-mixed force.
template <int BLOCK, bool FIX>
__global__ void __launch_bounds__(BLOCK) k_drift(Arrays a, Box b, int n, int track_vmax) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  double v2 = 0.0;
  if (i < n && !a.st->error) {
    const double dt2 = b.dt * 0.5;
    double4 q = a.q[i];
    const double4 v = a.v[i];
    q.x = dadd(q.x, dmul(v.x, dt2));
    q.y = dadd(q.y, dmul(v.y, dt2));
    q.z = dadd(q.z, dmul(v.z, dt2));
    a.q[i] = q;
    if (FIX) a.qfix[i] = make_int4(fixed_coord(q.x, b.L[0]), fixed_coord(q.y, b.L[1]),
                                   fixed_coord(q.z, b.L[2]), 0);
    if (track_vmax) {
      v2 = dadd(dadd(dmul(v.x, v.x), dmul(v.y, v.y)), dmul(v.z, v.z));
      if (!isfinite(v2) || !isfinite(q.x + q.y + q.z)) atomicOr(&a.st->error, kErrNonFinite);
    }
  }
  if (track_vmax) block_max_to<BLOCK>(&a.st->vmax2_bits, v2);
}

// ------------------------------------------------------------ executors
// The wall term of the reference's executors: the pair-force expression at
// distance d, each operation separately rounded (src/rankine.cc:78-82,
// src/burst.cc:91-93).
__device__ __forceinline__ double wall_df(double d, double c2, double dt) {
  const double r2 = dmul(d, d);
  const double r6 = dmul(dmul(r2, r2), r2);
  return dmul(dadd(ddiv(dsub(dmul(24.0, r6), 48.0), dmul(dmul(r6, r6), r2)), dmul(c2, 8.0)), dt);
}

// Before an executor pass: the pass re-takes the |v| maximum the next skin
// check reads (PairList::IsPairListExpired reads the momenta after it).
static __global__ void k_external_begin(Arrays a) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && !a.st->error) {
    a.st->vmax2_bits = 0ull;
    if (a.v_lag) a.st->vlag_set = 1;  // k_external keeps the pre-pass velocities
  }
}

// One executor pass over all atoms: GravityImposer (src/phaseflow.cc:58-73),
// MyPiston (src/rankine.cc:55-97), ShellForce (src/burst.cc:67-99); block
// partial sums of the piston impulse into a.partials.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_external(Arrays a, Box b, External x, int n) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  double v2 = 0.0, imp = 0.0;
  if (i < n && !a.st->error) {
    const double4 q = a.q[i];
    double4 v = a.v[i];
    if (a.v_lag) a.v_lag[i] = v;  // the velocities the step's second drift used
    const double CL = b.rc;
    if (x.kind == 1) {
      const double g = dmul(x.strength, x.dt);
      if (x.axis == 0) v.x = dadd(v.x, g);
      else if (x.axis == 1) v.y = dadd(v.y, g);
      else v.z = dadd(v.z, g);
    } else if (x.kind == 2) {
      if (q.z < CL) {
        const double df = wall_df(q.z, b.c2, x.dt);
        v.z = dsub(v.z, dmul(df, q.z));
      }
      const double pos = a.st->ext_position;
      if (q.z > pos) {
        const double dz = dadd(dsub(pos, q.z), CL);
        const double df = wall_df(dz, b.c2, x.dt);
        v.z = dadd(v.z, dmul(df, dz));
        imp = -dmul(df, dz);
      }
    } else if (x.kind == 3) {
      const double dx = dsub(q.x, x.center[0]), dy = dsub(q.y, x.center[1]), dz = dsub(q.z, x.center[2]);
      const double r = dsub(x.radius, sqrt(dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz))));
      if (!(dmul(r, r) > b.rc2)) {
        const double df = wall_df(r, b.c2, x.dt);
        v.x = dadd(v.x, dmul(df, dx));
        v.y = dadd(v.y, dmul(df, dy));
        v.z = dadd(v.z, dmul(df, dz));
      }
    }
    a.v[i] = v;
    v2 = dadd(dadd(dmul(v.x, v.x), dmul(v.y, v.y)), dmul(v.z, v.z));
  }
  block_max_to<BLOCK>(&a.st->vmax2_bits, v2);
  double s1[1] = {imp};
  block_sum_to<BLOCK, 1>(s1, a.partials);
}

// After a pass: impulse (fixed-order sum of the block partials) and the
// piston's move, as Rankine::Run moves it after each pass
// (src/rankine.cc:117-121).
static __global__ void k_external_done(Arrays a, External x, int nblocks) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || a.st->error) return;
  double s = 0.0;
  for (int k = 0; k < nblocks; k++) s += a.partials[k];
  a.st->ext_impulse = s;
  if (x.kind == 2) a.st->ext_position = dsub(a.st->ext_position, x.velocity);
}

// Variables::ChangeScale (src/variables.cc:141-148): q *= alpha.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_scale_positions(Arrays a, int n, double alpha) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  if (i >= n) return;
  double4 q = a.q[i];
  q.x = dmul(q.x, alpha);
  q.y = dmul(q.y, alpha);
  q.z = dmul(q.z, alpha);
  a.q[i] = q;
}

// Atoms per cell of a regular grid (BubbleHist::AnalyseSub,
// src/cavitation.cc:117-146): index int((x - 0) / grid_size) per axis on the
// wrapped position, x fastest; counts kept in int, cast to unsigned char by
// the caller as the reference's counters wrap.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_density(Arrays a, Box b, int n, double gsinv, int gx, int gy, int gz,
                                                   int *count) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  if (i >= n) return;
  const double4 q = a.q[i];
  double x[3] = {q.x, q.y, q.z};
  int g[3] = {gx, gy, gz}, c[3];
  for (int d = 0; d < 3; d++) {
    x[d] -= b.L[d] * floor(x[d] / b.L[d]);
    const int k = (int)(x[d] * gsinv);
    c[d] = k < 0 ? 0 : (k >= g[d] ? g[d] - 1 : k);
  }
  atomicAdd(&count[c[0] + c[1] * gx + c[2] * gx * gy], 1);
}

// Packs q + v dt/2 (the coming step's first half drift) into out without
// moving atoms: the fixed-point copy the fused NVE force pass reads.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_pack_half(Arrays a, Box b, int n, int4 *out) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  if (i >= n || a.st->error) return;
  const double4 q = a.q[i];
  const double4 v = a.v[i];
  const double dt2 = b.dt * 0.5;
  out[i] = make_int4(fixed_coord(dadd(q.x, dmul(v.x, dt2)), b.L[0]), fixed_coord(dadd(q.y, dmul(v.y, dt2)), b.L[1]),
                     fixed_coord(dadd(q.z, dmul(v.z, dt2)), b.L[2]), 0);
}

// Writes the fixed-point copy of q without moving atoms.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_pack_fix(Arrays a, Box b, int n) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  if (i >= n) return;
  const double4 q = a.q[i];
  a.qfix[i] = make_int4(fixed_coord(q.x, b.L[0]), fixed_coord(q.y, b.L[1]), fixed_coord(q.z, b.L[2]), 0);
}

enum ForceMode { kKick = 0, kForceOut = 1, kKickNoseHoover = 2, kKickLangevin = 3 };

__device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
    const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = lo1; c[2] = n2; c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// Three standard normals for (atom id, step) from one Philox4x32-10 block and
// two Box-Muller pairs; the same stream as the oracle's ljo_langevin_normals.
__device__ __forceinline__ void langevin_normals(unsigned long long seed, uint32_t id,
                                                 unsigned long long step, double z[3]) {
  uint32_t c[4] = {id, (uint32_t)step, (uint32_t)(step >> 32), 0x4C414E47u};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double scale = 2.3283064365386963e-10;
  const double u0 = ((double)c[0] + 0.5) * scale, u1 = ((double)c[1] + 0.5) * scale;
  const double u2 = ((double)c[2] + 0.5) * scale, u3 = ((double)c[3] + 0.5) * scale;
  const double twopi = 6.283185307179586;
  const double r0 = sqrt(-2.0 * log(u0)), r1 = sqrt(-2.0 * log(u2));
  z[0] = r0 * cos(twopi * u1);
  z[1] = r0 * sin(twopi * u1);
  z[2] = r1 * cos(twopi * u3);
}

struct Thermo {
  double gamma, noise_sd;      // Langevin friction and noise amplitude sqrt(2 gamma T / dt)
  unsigned long long seed;     // Langevin key; the counter is the device step count
};

// Per-atom epilogue shared by both precisions: apply the kick in the mode's
// form and emit the quantities the next kernels need.
template <int MODE>
__device__ __forceinline__ void finish_atom(Arrays &a, const Box &b, const Thermo &th, int i,
                                            double fx, double fy, double fz, double &v2,
                                            double &ke) {
  if (MODE == kForceOut) {
    a.v_tmp[i] = make_double4(fx, fy, fz, 0.0);
    return;
  }
  double4 v = a.v[i];
  double exp1 = 1.0;
  if (MODE == kKickNoseHoover) {
    exp1 = exp(-(b.dt * 0.5) * a.st->zeta);
    v.x = dmul(v.x, exp1); v.y = dmul(v.y, exp1); v.z = dmul(v.z, exp1);
  }
  v.x = dadd(v.x, fx); v.y = dadd(v.y, fy); v.z = dadd(v.z, fz);
  if (MODE == kKickNoseHoover) {
    v.x = dmul(v.x, exp1); v.y = dmul(v.y, exp1); v.z = dmul(v.z, exp1);
    ke = dadd(dadd(dmul(dmul(0.5, v.x), v.x), dmul(dmul(0.5, v.y), v.y)), dmul(dmul(0.5, v.z), v.z));
  }
  if (MODE == kKickLangevin) {
    // ForceCalculator::Langevin, src/fcalculator.cc:1001-1017
    double z[3];
    langevin_normals(th.seed, (uint32_t)a.ids[i], (unsigned long long)a.st->steps, z);
    const double dt = b.dt;
    v.x = dadd(v.x, dmul(dadd(dmul(-th.gamma, v.x), dmul(th.noise_sd, z[0])), dt));
    v.y = dadd(v.y, dmul(dadd(dmul(-th.gamma, v.y), dmul(th.noise_sd, z[1])), dt));
    v.z = dadd(v.z, dmul(dadd(dmul(-th.gamma, v.z), dmul(th.noise_sd, z[2])), dt));
    v2 = dadd(dadd(dmul(v.x, v.x), dmul(v.y, v.y)), dmul(v.z, v.z));
  }
  a.v[i] = v;
}

// FP64 force kick, one thread per atom over its full row.  Every pair term is
// the reference's (ForceCalculator::CalculateForceNext, src/fcalculator.cc:
// 228-290): dx = image(q_j) - q_i, r2 = (dx*dx + dy*dy) + dz*dz, skipped if
// r2 > rc^2, r6 = (r2*r2)*r2, df = ((24 r6 - 48) / ((r6*r6)*r2) + 8 C2) * dt,
// term = df * dx, all separately rounded; only the summation order differs.
template <int BLOCK, int MODE>
__global__ void __launch_bounds__(BLOCK) k_force_fp64(Arrays a, Box b, int n, Thermo th) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  double v2 = 0.0, ke = 0.0;
  if (i < n && !a.st->error) {
    const double4 qi = a.q[i];
    const int nn = a.nnbr[i];
    const double c2x8 = b.c2 * 8.0;
    const double dt = (MODE == kForceOut) ? 1.0 : b.dt;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    const int *row = a.nbr + i;
    // software pipeline: the next partner's position and the entry after it
    // are in flight while a pair term is formed
    int jn = nn > 1 ? row[a.stride] : i;
    double4 qn = a.q[nn > 0 ? row[0] : i];
    for (int k = 0; k < nn; k++) {
      const double4 qj = qn;
      qn = a.q[jn];
      jn = (k + 2 < nn) ? row[(size_t)(k + 2) * a.stride] : i;
      const double dx = dsub(image_of(qj.x, qi.x, b.L[0], b.hL[0]), qi.x);
      const double dy = dsub(image_of(qj.y, qi.y, b.L[1], b.hL[1]), qi.y);
      const double dz = dsub(image_of(qj.z, qi.z, b.L[2], b.hL[2]), qi.z);
      const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
      if (r2 > b.rc2) continue;
      const double r6 = dmul(dmul(r2, r2), r2);
      const double df = dmul(dadd(ddiv(dsub(dmul(24.0, r6), 48.0), dmul(dmul(r6, r6), r2)), c2x8), dt);
      fx = dadd(fx, dmul(df, dx));
      fy = dadd(fy, dmul(df, dy));
      fz = dadd(fz, dmul(df, dz));
    }
    finish_atom<MODE>(a, b, th, i, fx, fy, fz, v2, ke);
  }
  if (MODE == kKickLangevin) warp_max_to(&a.st->vmax2_bits, v2);
  if (MODE == kKickNoseHoover) {
    double s[1] = {ke};
    block_sum_to<BLOCK, 1>(s, a.partials);
  }
}

// FP32 reciprocal on the special-function unit (rcp.approx.ftz.f32, PTX ISA):
// relative error at most one unit in the last place, well inside the FP32
// force error budget.
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// One FP32 pair term from fixed-point positions: the wrapped int32
// difference is the minimum-image displacement in units of L/2^32.  r^2 = 0
// (the padding entries, the atom itself) contributes nothing: the unsigned
// compare of the float bits keeps 0 < r^2 <= rc^2 in one test.
__device__ __forceinline__ void lj_pair_fp32(const int4 &pi, const int4 &pj, float sx, float sy, float sz,
                                             unsigned rc2_bits, float c2x8, float &fx, float &fy, float &fz) {
  const float dx = (float)(pj.x - pi.x) * sx;
  const float dy = (float)(pj.y - pi.y) * sy;
  const float dz = (float)(pj.z - pi.z) * sz;
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  const float ir2 = rcp_approx(r2);
  const float ir6 = ir2 * ir2 * ir2;
  float df = fmaf(ir2 * ir6, fmaf(-48.f, ir6, 24.f), c2x8);
  df = (__float_as_uint(r2) - 1u < rc2_bits) ? df : 0.f;
  fx = fmaf(df, dx, fx);
  fy = fmaf(df, dy, fy);
  fz = fmaf(df, dz, fz);
}

// The per-atom end of an FP32-mixed force pass: the FP64 kick and, with
// DRIFT, the second half drift (DRIFT == 2 also this step's first half
// drift of the atom itself and the pack of the next step's first-drift
// position into qf_next).
template <int MODE, int DRIFT>
__device__ __forceinline__ void fp32_finish(Arrays &a, const Box &b, const Thermo &th, int i, double Fx, double Fy,
                                            double Fz, int4 *qf_next, double &v2, double &ke) {
  const double dt = (MODE == kForceOut) ? 1.0 : b.dt;
  const double dt2 = b.dt * 0.5;
  double4 q = a.q[i];
  if (DRIFT == 2) {
    // this step's first half drift (the neighbours' copies in qf already have it)
    const double4 v0 = a.v[i];
    q.x = dadd(q.x, dmul(v0.x, dt2));
    q.y = dadd(q.y, dmul(v0.y, dt2));
    q.z = dadd(q.z, dmul(v0.z, dt2));
  }
  finish_atom<MODE>(a, b, th, i, Fx * dt, Fy * dt, Fz * dt, v2, ke);
  if (DRIFT) {
    const double4 v = a.v[i];
    q.x = dadd(q.x, dmul(v.x, dt2));
    q.y = dadd(q.y, dmul(v.y, dt2));
    q.z = dadd(q.z, dmul(v.z, dt2));
    a.q[i] = q;
    v2 = dadd(dadd(dmul(v.x, v.x), dmul(v.y, v.y)), dmul(v.z, v.z));
    if (!isfinite(v2) || !isfinite(q.x + q.y + q.z)) atomicOr(&a.st->error, kErrNonFinite);
    if (DRIFT == 2) {
      // the next step's first half drift, packed for its force pass
      qf_next[i] = make_int4(fixed_coord(dadd(q.x, dmul(v.x, dt2)), b.L[0]),
                             fixed_coord(dadd(q.y, dmul(v.y, dt2)), b.L[1]),
                             fixed_coord(dadd(q.z, dmul(v.z, dt2)), b.L[2]), 0);
    }
  }
}

// ------------------------------------------------ FP32 row sums, 1-4 lanes per atom
// The row sum of an atom in one fixed order whatever the number of lanes
// that share the row, so that 1, 2 or 4 lanes per atom give bit-identical
// forces.  The row's G groups of four entries (rows are padded to a
// multiple of 4 with masked self entries) form chunks of two groups (the
// last chunk may hold one): chunk c is groups 2c and 2c + 1, its eight pair
// terms summed in FP32 in entry order from 0; the row sum is the FP64 sum
// of the chunk sums in chunk order, S = ((0 + s_0) + s_1) + ...  With TPA
// lanes per atom, lane s sums chunks s, s + TPA, s + 2 TPA, ...; after each
// round of TPA chunks every lane of the atom reads the round's chunk sums
// from its neighbours (shuffles of FP32 values) and adds them in chunk
// order, so every lane holds S at the end.  Chunks past the row's end add
// +0.0, which leaves S unchanged (S starts at +0.0 and is never -0.0).

// Partner positions of a lane's groups from the global fixed-point copy.
// The list entries of the group after the next are in flight while a group
// is summed (the list is the pass's one stream from HBM); with AHEAD the
// next group's positions are too (software pipeline: the gathers are the
// pass's long-latency loads; four more int4 registers).  Group -1 is none:
// its entries are the atom itself.
template <bool AHEAD = true>
struct GlobalGroups {
  const int *row;  // nbr + atom
  int st;          // list stride
  const int4 *qf;
  int self;
  int n0, n1, n2, n3;      // entries of the current group (without AHEAD)
  int m0, m1, m2, m3;      // entries of the next group
  int4 c0, c1, c2, c3;     // positions of the current group (with AHEAD)
  __device__ __forceinline__ void load(int g, int &x0, int &x1, int &x2, int &x3) const {
    if (g < 0) {
      x0 = x1 = x2 = x3 = self;
      return;
    }
    const int *r = row + (size_t)(4 * g) * st;
    x0 = __ldg(r);
    x1 = __ldg(r + st);
    x2 = __ldg(r + 2 * st);
    x3 = __ldg(r + 3 * st);
  }
  // the lane's first two groups
  __device__ __forceinline__ void start(int ga, int gb) {
    load(ga, n0, n1, n2, n3);
    if (AHEAD) {
      c0 = __ldg(qf + n0);
      c1 = __ldg(qf + n1);
      c2 = __ldg(qf + n2);
      c3 = __ldg(qf + n3);
    }
    load(gb, m0, m1, m2, m3);
  }
  // positions of the lane's current group; the entries of the group after
  // the next (gnext) start loading, with AHEAD also the next group's positions
  __device__ __forceinline__ void take(int gnext, int4 &p0, int4 &p1, int4 &p2, int4 &p3) {
    if (AHEAD) {
      p0 = c0;
      p1 = c1;
      p2 = c2;
      p3 = c3;
      c0 = __ldg(qf + m0);
      c1 = __ldg(qf + m1);
      c2 = __ldg(qf + m2);
      c3 = __ldg(qf + m3);
    } else {
      p0 = __ldg(qf + n0);
      p1 = __ldg(qf + n1);
      p2 = __ldg(qf + n2);
      p3 = __ldg(qf + n3);
      n0 = m0;
      n1 = m1;
      n2 = m2;
      n3 = m3;
    }
    load(gnext, m0, m1, m2, m3);
  }
};

// The same from the block's stage in shared memory: one 8-byte load brings
// four 16-bit stage indices; indices outside the stage are flagged and read
// as entry 0.  One lane per atom.
__device__ __forceinline__ unsigned stage_index(unsigned v, unsigned nstage, bool &bad) {
  const bool out = v >= nstage;
  bad |= out;
  return out ? 0u : v;
}

struct StagedGroups {
  const uint2 *row;  // nbr16 + atom
  int st;
  const int4 *pos;   // the stage
  unsigned nstage;
  bool bad;
  uint2 g0, g1;
  __device__ __forceinline__ uint2 load(int g) const {
    return g < 0 ? make_uint2(0u, 0u) : __ldg(row + (size_t)g * st);
  }
  __device__ __forceinline__ void start(int ga, int gb) {
    bad = false;
    g0 = load(ga);
    g1 = load(gb);
  }
  __device__ __forceinline__ void take(int gnext, int4 &p0, int4 &p1, int4 &p2, int4 &p3) {
    p0 = pos[stage_index(g0.x & 0xffffu, nstage, bad)];
    p1 = pos[stage_index(g0.x >> 16, nstage, bad)];
    p2 = pos[stage_index(g0.y & 0xffffu, nstage, bad)];
    p3 = pos[stage_index(g0.y >> 16, nstage, bad)];
    g0 = g1;
    g1 = load(gnext);
  }
};

// Fixed-point scales and force constants of the FP32 pair term.
struct PairConst {
  float sx, sy, sz;
  unsigned rc2_bits;
  float c2x8;
};

__device__ __forceinline__ PairConst pair_const(const float fix_scale[3], float rc2f, float c2x8f) {
  return PairConst{fix_scale[0], fix_scale[1], fix_scale[2], __float_as_uint(rc2f), c2x8f};
}

__device__ __forceinline__ void lj_group_fp32(const int4 &pi, const int4 &p0, const int4 &p1, const int4 &p2,
                                              const int4 &p3, const PairConst &k, float &fx, float &fy, float &fz) {
  lj_pair_fp32(pi, p0, k.sx, k.sy, k.sz, k.rc2_bits, k.c2x8, fx, fy, fz);
  lj_pair_fp32(pi, p1, k.sx, k.sy, k.sz, k.rc2_bits, k.c2x8, fx, fy, fz);
  lj_pair_fp32(pi, p2, k.sx, k.sy, k.sz, k.rc2_bits, k.c2x8, fx, fy, fz);
  lj_pair_fp32(pi, p3, k.sx, k.sy, k.sz, k.rc2_bits, k.c2x8, fx, fy, fz);
}

// Row sum of an atom with G groups (see above), lane `sub` of TPA.  All TPA
// lanes of the atom must call together (they exchange chunk sums); every
// lane returns the row sum.
template <int TPA, typename Groups>
__device__ __forceinline__ void fp32_row(Groups &f, int G, int sub, const int4 &pi, const PairConst &k, double &Fx,
                                         double &Fy, double &Fz) {
  static_assert(TPA == 1 || TPA == 2 || TPA == 4, "1, 2 or 4 lanes per atom");
  double Sx = 0.0, Sy = 0.0, Sz = 0.0;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  if (TPA == 1) {
    f.start(G > 0 ? 0 : -1, G > 1 ? 1 : -1);
    for (int g = 0; g < G; g++) {
      int4 p0, p1, p2, p3;
      f.take(g + 2 < G ? g + 2 : -1, p0, p1, p2, p3);
      lj_group_fp32(pi, p0, p1, p2, p3, k, fx, fy, fz);
      if (g & 1) {
        Sx += (double)fx;
        Sy += (double)fy;
        Sz += (double)fz;
        fx = fy = fz = 0.f;
      }
    }
    Sx += (double)fx;  // the last chunk when it holds one group (else +0)
    Sy += (double)fy;
    Sz += (double)fz;
  } else {
    const int lane = threadIdx.x & 31;
    const unsigned amask = ((1u << TPA) - 1u) << (lane & ~(TPA - 1));
    const int C = (G + 1) >> 1, R = (C + TPA - 1) / TPA;
    // the lane's m-th group: group 2c + (m & 1) of chunk c = sub + (m >> 1) TPA
    auto grp = [&](int m) {
      const int g = 2 * (sub + (m >> 1) * TPA) + (m & 1);
      return g < G ? g : -1;
    };
    f.start(grp(0), grp(1));
    for (int r = 0; r < R; r++) {
      const int ga = grp(2 * r), gb = grp(2 * r + 1);
      int4 p0, p1, p2, p3;
      fx = fy = fz = 0.f;
      f.take(grp(2 * r + 2), p0, p1, p2, p3);
      if (ga >= 0) lj_group_fp32(pi, p0, p1, p2, p3, k, fx, fy, fz);
      f.take(grp(2 * r + 3), p0, p1, p2, p3);
      if (gb >= 0) lj_group_fp32(pi, p0, p1, p2, p3, k, fx, fy, fz);
#pragma unroll
      for (int j = 0; j < TPA; j++) {
        Sx += (double)__shfl_sync(amask, fx, j, TPA);
        Sy += (double)__shfl_sync(amask, fy, j, TPA);
        Sz += (double)__shfl_sync(amask, fz, j, TPA);
      }
    }
  }
  Fx = Sx;
  Fy = Sy;
  Fz = Sz;
}

// fp32_row<1> over the global fixed-point copy in one plain loop (the same
// sums in the same order): rows are padded to a multiple of 4 with the atom
// itself, so the row is walked four partners at a time without masks, with
// the list entries of the next two groups always in flight.  Measured at
// 0.282 ms per fused pass on the 2.05M-atom liquid against 0.304 ms for
// fp32_row<1> over GlobalGroups (whose per-group selects the compiler
// schedules worse).
__device__ __forceinline__ void fp32_row_global(const Arrays &a, const Box &b, const int4 *qf, int i,
                                                const int4 &pi, int nn4, double &Fx, double &Fy, double &Fz) {
  const float sx = b.fix_scale[0], sy = b.fix_scale[1], sz = b.fix_scale[2];
  const unsigned rc2_bits = __float_as_uint(b.rc2f);
  const float c2x8 = b.c2x8f;
  const int *row = a.nbr + i;
  const int st = a.stride;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  int n0 = i, n1 = i, n2 = i, n3 = i;
  int m0 = i, m1 = i, m2 = i, m3 = i;
  if (nn4 > 0) {
    n0 = __ldg(row);
    n1 = __ldg(row + st);
    n2 = __ldg(row + 2 * st);
    n3 = __ldg(row + 3 * st);
  }
  if (nn4 > 4) {
    m0 = __ldg(row + 4 * st);
    m1 = __ldg(row + 5 * st);
    m2 = __ldg(row + 6 * st);
    m3 = __ldg(row + 7 * st);
  }
  Fx = Fy = Fz = 0.0;
  for (int k = 0; k < nn4; k += 4) {
    const int4 p0 = __ldg(qf + n0);
    const int4 p1 = __ldg(qf + n1);
    const int4 p2 = __ldg(qf + n2);
    const int4 p3 = __ldg(qf + n3);
    n0 = m0;
    n1 = m1;
    n2 = m2;
    n3 = m3;
    if (k + 8 < nn4) {
      const int *r = row + (size_t)(k + 8) * st;
      m0 = __ldg(r);
      m1 = __ldg(r + st);
      m2 = __ldg(r + 2 * st);
      m3 = __ldg(r + 3 * st);
    }
    lj_pair_fp32(pi, p0, sx, sy, sz, rc2_bits, c2x8, fx, fy, fz);
    lj_pair_fp32(pi, p1, sx, sy, sz, rc2_bits, c2x8, fx, fy, fz);
    lj_pair_fp32(pi, p2, sx, sy, sz, rc2_bits, c2x8, fx, fy, fz);
    lj_pair_fp32(pi, p3, sx, sy, sz, rc2_bits, c2x8, fx, fy, fz);
    if (k & 4) {  // the second group of a chunk
      Fx += (double)fx;
      Fy += (double)fy;
      Fz += (double)fz;
      fx = fy = fz = 0.f;
    }
  }
  Fx += (double)fx;  // the last chunk when it holds one group (else +0)
  Fy += (double)fy;
  Fz += (double)fz;
}

// The error flag as one lane of the warp read it: the lanes of an atom must
// agree on whether they take its row (they exchange values), and the flag
// can be raised by another block at any time.  All lanes must call.
__device__ __forceinline__ int warp_error(const Status *st) {
  return __shfl_sync(0xffffffffu, *(volatile const int *)&st->error, 0);
}

// Sum of one value per atom over a block's BLOCK / TPA atoms (consecutive
// atoms, TPA lanes each, the value on the atom's first lane), written to
// partials[blockIdx.x].  The tree is block_sum_to<BLOCK / TPA, 1>'s over
// one lane per atom whatever TPA is, so the sum does not depend on the lane
// count.  All threads of the block must call.
template <int BLOCK, int TPA>
__device__ __forceinline__ void atom_block_sum(double x, double *partials) {
  constexpr int ATOMS = BLOCK / TPA;
  static_assert(ATOMS % 32 == 0, "whole warps of atoms");
  __shared__ double per_atom[TPA > 1 ? ATOMS : 1];
  __shared__ double per_warp[ATOMS / 32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (TPA > 1) {
    if (threadIdx.x % TPA == 0) per_atom[threadIdx.x / TPA] = x;
    __syncthreads();
    x = threadIdx.x < ATOMS ? per_atom[threadIdx.x] : 0.0;
  }
  if (w < ATOMS / 32) {
    const double s = warp_sum(x);
    if (l == 0) per_warp[w] = s;
  }
  __syncthreads();
  if (w == 0) {
    double y = l < ATOMS / 32 ? per_warp[l] : 0.0;
    y = warp_sum(y);
    if (l == 0) partials[blockIdx.x] = y;
  }
}

// FP32-mixed force kick, TPA lanes per atom (BLOCK / TPA atoms per block).
// Displacements come from the fixed-point copy (no ghost atoms, no shift
// codes); the row sum is fp32_row's fixed-order sum and the kick is FP64
// (the atom's first lane).  With DRIFT the second half drift q += v dt/2 and the |v| maximum
// of the step are done in the same pass: this kernel reads only the
// fixed-point copy, so moving q here races with no other thread.  DRIFT == 2
// is the whole NVE step in one pass: qf holds every atom's position after
// this step's first half drift (packed by the previous step's pass, or by
// k_pack_half after a rebuild); the kernel applies that drift to its own
// atom, kicks, drifts again and packs the next step's first-drift position
// into qf_next (the other buffer, so no thread overwrites a copy that
// another still reads).  The arithmetic is the separate drift kernels',
// operation for operation.
template <int BLOCK, int MODE, int DRIFT, int TPA>
__global__ void __launch_bounds__(BLOCK) k_force_fp32(Arrays a, Box b, int n, Thermo th, const int4 *qf,
                                                      int4 *qf_next) {
  const int t = blockIdx.x * BLOCK + threadIdx.x;
  const int i = t / TPA, sub = t % TPA;
  double v2 = 0.0, ke = 0.0;
  if (DRIFT == 2 && MODE == kKick && t == 0 && !a.st->error) {
    // the step counter (k_step_done's work): nothing in this pass reads it
    a.st->steps++;
    a.st->sim_time += b.dt;
  }
  const int err = TPA > 1 ? warp_error(a.st) : a.st->error;
  if (i < n && !err) {
    const int4 pi = qf[i];
    double Fx, Fy, Fz;
    const PairConst k = pair_const(b.fix_scale, b.rc2f, b.c2x8f);
    if (TPA == 1) {
      fp32_row_global(a, b, qf, i, pi, (a.nnbr[i] + 3) & ~3, Fx, Fy, Fz);
    } else {
      GlobalGroups<> f{a.nbr + i, a.stride, qf, i};
      fp32_row<TPA>(f, (a.nnbr[i] + 3) >> 2, sub, pi, k, Fx, Fy, Fz);
    }
    if (sub == 0) fp32_finish<MODE, DRIFT>(a, b, th, i, Fx, Fy, Fz, qf_next, v2, ke);
  }
  if (MODE == kKickLangevin || DRIFT) warp_max_to(&a.st->vmax2_bits, v2);
  if (MODE == kKickNoseHoover) atom_block_sum<BLOCK, TPA>(ke, a.partials);
}

// ---------------------------------------------- mbarrier and bulk copies
// (PTX ISA: mbarrier, cp.async.bulk; sm_90 and later)
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

// Bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned)
// from global to shared memory, completing on the mbarrier's transaction
// count.  A plain load: no multicast.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// Waits for the mbarrier's phase `parity` to complete, for at most `limit`
// clock cycles; false if it gave up.  The test is the non-blocking
// mbarrier.test_wait (PTX ISA), polled with a short sleep, so that a short
// limit is kept to within a poll.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit) {
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) return false;
    __nanosleep(20);
  }
}

// About one second at the B200's clocks: a stage copy takes microseconds.
constexpr long long kStageWaitCycles = 2000000000ll;

// The staged FP32-mixed pass: k_force_fp32 with the partners' positions read
// from the block's stage (k_stage_plan) in dynamic shared memory, which one
// thread fills with one bulk copy per plan range while the others wait on an
// mbarrier.  Blocks without a plan (-1) gather from global memory.  If the
// wait gives up (Box::stage_wait cycles, mdg_params.stage_wait_cycles), the
// block sets kErrTimeout, waits once more (up to kStageWaitCycles) for its
// copies in flight, and kicks no atom.
template <int BLOCK, int MODE, int DRIFT>
__global__ void __launch_bounds__(BLOCK) k_force_fp32_staged(Arrays a, Box b, int n, Thermo th, const int4 *qf,
                                                             int4 *qf_next) {
  extern __shared__ __align__(16) int4 pos[];
  __shared__ __align__(8) uint64_t bar;
  static_assert(BLOCK == kStageBlock, "stage plans are per kStageBlock atoms");
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  double v2 = 0.0, ke = 0.0;
  if (DRIFT == 2 && MODE == kKick && i == 0 && !a.st->error) {
    a.st->steps++;
    a.st->sim_time += b.dt;
  }
  // thread 0 checks the plan against the stage and the atom count (a plan
  // left from an earlier layout is never copied) and fills the stage
  __shared__ int staged;
  __shared__ unsigned nstage;
  uint32_t total = 0;
  if (threadIdx.x == 0) {
    const int npl = a.stage_n[blockIdx.x];
    int use = npl > 0 && npl <= kStageRanges && !a.st->error;
    const int4 *plan = a.stage_rng + (size_t)blockIdx.x * kStageRanges;
    for (int r = 0; use && r < npl; r++) {
      const int4 pr = plan[r];
      if (pr.x < 0 || pr.y > b.ncell || pr.x >= pr.y) {
        use = 0;
        break;
      }
      const int cnt = a.cell_start[pr.y] - pr.z;
      if (cnt < 0 || pr.z < 0 || pr.z + cnt > n || pr.w != (int)total || pr.w + cnt > a.stage_cap) use = 0;
      // bulk copies start on 16-byte boundaries at both ends
      if (cnt > 0 && (((smem_addr(pos + pr.w) | (uint32_t)(uintptr_t)(qf + pr.z)) & 15u) != 0u)) use = 0;
      total += (uint32_t)cnt;
    }
    if (!use && npl > 0 && npl <= kStageRanges && !a.st->error) atomicOr(&a.st->error, kErrStage);
    if (use) mbar_init(&bar, 1);
    staged = use;
    nstage = use ? total : 0u;
  }
  __syncthreads();
  const bool use_stage = staged != 0;
  bool ok = true;
  if (use_stage) {
    if (threadIdx.x == 0) {
      const int npl = a.stage_n[blockIdx.x];
      const int4 *plan = a.stage_rng + (size_t)blockIdx.x * kStageRanges;
      mbar_arrive_expect_tx(&bar, total * (uint32_t)sizeof(int4));
      for (int r = 0; r < npl; r++) {
        const int4 pr = plan[r];
        const int cnt = a.cell_start[pr.y] - pr.z;
        if (cnt > 0) bulk_load(pos + pr.w, qf + pr.z, (uint32_t)cnt * (uint32_t)sizeof(int4), &bar);
      }
    }
    ok = mbar_wait(&bar, 0, b.stage_wait);
    if (!ok) {
      atomicOr(&a.st->error, kErrTimeout);
      mbar_wait(&bar, 0, kStageWaitCycles);
    }
  }
  if (ok && i < n && !a.st->error) {
    const int4 pi = qf[i];
    const int G = (a.nnbr[i] + 3) >> 2;
    const PairConst k = pair_const(b.fix_scale, b.rc2f, b.c2x8f);
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    if (use_stage) {
      StagedGroups f{a.nbr16 + i, a.stride, pos, nstage};
      fp32_row<1>(f, G, 0, pi, k, Fx, Fy, Fz);
      if (f.bad) atomicOr(&a.st->error, kErrStage);
    } else {
      GlobalGroups<> f{a.nbr + i, a.stride, qf, i};
      fp32_row<1>(f, G, 0, pi, k, Fx, Fy, Fz);
    }
    fp32_finish<MODE, DRIFT>(a, b, th, i, Fx, Fy, Fz, qf_next, v2, ke);
  }
  if (MODE == kKickLangevin || DRIFT) warp_max_to(&a.st->vmax2_bits, v2);
  if (MODE == kKickNoseHoover) {
    double s[1] = {ke};
    block_sum_to<BLOCK, 1>(s, a.partials);
  }
}

// ------------------------------------------- persistent multi-step NVE pass
// Grid barrier for a cooperative launch (every block resident): a counter
// and a generation number.  A block waits at most `limit` polls; one that
// gives up sets kErrTimeout and returns false, and the caller leaves its
// loop (so does every other block at its next barrier).
struct GridBarrier {
  unsigned count;
  unsigned gen;
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Every block of the (cooperative, fully resident) grid arrives; false if
// this block gave up waiting after `limit` polls (kErrTimeout is set).  The
// block's writes before the barrier are visible to every block after it:
// a gpu-scope fence before the arrival, acquire loads while waiting.
__device__ __forceinline__ bool grid_barrier(GridBarrier *g, Status *st, long long limit) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    const unsigned gen = ld_acquire_gpu(&g->gen);
    __threadfence();
    if (atomicAdd(&g->count, 1u) + 1u == gridDim.x) {
      g->count = 0u;  // no block arrives at the next barrier before gen moves
      __threadfence();
      atomicAdd(&g->gen, 1u);
    } else {
      long long polls = 0;
      while (ld_acquire_gpu(&g->gen) == gen) {
        if (++polls > limit) {
          atomicOr(&st->error, kErrTimeout);
          ok = 0;
          break;
        }
        __nanosleep(20);
      }
    }
  }
  __syncthreads();
  return ok != 0;
}

// About a second of polling (a poll and a 20 ns sleep take some 60 ns): a
// step takes microseconds.
constexpr long long kBarrierPolls = 16000000ll;

// The expiry test of PairList::IsPairListExpired (k_expiry's arithmetic)
// for a step the persistent pass may take on its own: the list is current,
// the skin budget is positive and stays non-negative after this step's
// 2 vmax dt.  Only then is the budget spent and the |v| maximum cleared;
// otherwise nothing changes and the caller's ordinary step (k_expiry, the
// displacement check, the rebuild) takes this step.
__device__ __forceinline__ bool take_step_alone(Status *st, const Box &b) {
  if (st->error || st->list_stale || !(st->budget > 0.0)) return false;
  const double vmax = sqrt(__longlong_as_double((long long)st->vmax2_bits));
  if (skin_cost(vmax, b.dt) > b.buffer_length) return false;  // k_expiry reports the too-fast atom
  const double budget = dsub(st->budget, skin_cost(vmax, b.dt));
  if (budget < 0.0) return false;
  st->budget = budget;
  st->vmax2_bits = 0ull;
  st->vlag_set = 0;
  return true;
}

// FP32-mixed NVE steps in one cooperative launch, for systems small enough
// that per-step launch latency dominates: each step is the fused pass of
// k_force_fp32<.., kKick, 2, TPA> over all atoms (grid-stride) followed by
// one grid barrier.  Every decision of PairList::IsPairListExpired and
// CheckByDisplacement is a function of values every block holds or reads
// after a barrier, so every block takes it by itself:
// - the skin budget lives in a register (budget -= 2 vmax dt while
//   positive; a check once it is negative);
// - the step's |v| maximum comes from a ring of three slots (pass k fills
//   slot k % 3; block 0 clears slot k + 1 during step k, which no block
//   reads any more and none fills before the next barrier);
// - a displacement check runs as k_disp_max, k_disp_collect and
//   k_disp_pairs do it (copies dated `lag` back), three phases each ending
//   in a grid barrier, and every block reads the verdict (want_build) after
//   the last one; block 0 clears the check's counters after it (the next
//   check starts at least one barrier later) and want_build while the next
//   check's first phase runs.
// The pass stops before the first step that needs a rebuild -- it marks the
// list stale, so the caller's ordinary step rebuilds without deciding again
// -- before a step whose atom is too fast (the caller's step reports it),
// or when the step count reaches Status::target_steps; block 0 then writes
// the budget, the |v| maximum, the counters and the buffer parity back.
// Errors raised inside the passes stop the work of later passes (they
// check the flag) and are reported by the caller; the decisions never read
// the flag, which a block may raise while another still decides.  The
// fixed-point buffer the next step reads comes from, and goes back to,
// Status::fix_parity (0: qf0, 1: qf1).  The arithmetic is k_force_fp32's
// and the decisions are the graph path's, so trajectories and counters
// equal the graph path's bit for bit.
template <int BLOCK, int TPA>
__global__ void __launch_bounds__(BLOCK) k_nve_persistent(Arrays a, Box b, int n, int4 *qf0, int4 *qf1, double lag,
                                                          GridBarrier *bar) {
  __shared__ volatile int found;
  const Thermo th{};
  const PairConst k = pair_const(b.fix_scale, b.rc2f, b.c2x8f);
  const long long nthreads = (long long)n * TPA;
  const long long stride = (long long)gridDim.x * BLOCK;
  const int gtid = blockIdx.x * BLOCK + threadIdx.x, gthreads = gridDim.x * BLOCK;
  Status *st = a.st;
  const bool lead = blockIdx.x == 0 && threadIdx.x == 0;
  // the values the decisions start from, read by every block before any is
  // written (the first barrier)
  int parity = *(volatile int *)&st->fix_parity;
  double budget = *(volatile double *)&st->budget;
  unsigned long long vmax2 = *(volatile unsigned long long *)&st->vmax2_bits;
  const long long steps0 = *(volatile long long *)&st->steps;
  const long long target = *(volatile long long *)&st->target_steps;
  const bool startable = !*(volatile int *)&st->error && !*(volatile int *)&st->list_stale;
  double sim_time = st->sim_time;  // block 0's copy
  if (lead) {
    st->vmax2_ring[0] = st->vmax2_ring[1] = 0ull;
    st->dr2max_bits = 0ull;
    st->cand_weighted = 0;
    st->cand_n = 0;
  }
  if (!grid_barrier(bar, st, kBarrierPolls)) return;
  bool stale = false, checked = false;
  long long taken = 0, checks = 0;
  for (;; taken++) {
    // 0: stop; 1: take the step; 2: check displacements first
    int g = 0;
    if (startable && steps0 + taken < target) {
      if (budget > 0.0) {
        const double cost = skin_cost(sqrt(__longlong_as_double((long long)vmax2)), b.dt);
        if (cost <= b.buffer_length) {  // else too fast: the caller's step reports it
          budget = dsub(budget, cost);
          g = budget < 0.0 ? 2 : 1;
        }
      } else {
        g = budget < 0.0 ? 2 : 1;
      }
    }
    checked = false;
    if (g == 2) {
      checks++;
      checked = true;
      if (lead) st->want_build = 0;
      double d2 = 0.0;
      for (int i = gtid; i < n; i += gthreads)
        for_each_copy(copy_view(a), b.L, i, lag, [&](int, double x) { d2 = fmax(d2, x); });
      block_max_to<BLOCK>(&st->dr2max_bits, d2);
      if (!grid_barrier(bar, st, kBarrierPolls)) break;
      const double c = b.buffer_length - sqrt(__longlong_as_double(*(volatile long long *)&st->dr2max_bits));
      const double c_d2 = c * c;
      for (int i = gtid; i < n; i += gthreads)
        for_each_copy(copy_view(a), b.L, i, lag, [&](int code, double x) {
          if (x > c_d2) {
            atomicAdd(&st->cand_weighted, 1);
            const int kk = atomicAdd(&st->cand_n, 1);
            if (kk < b.check_list_length) a.cand[kk] = make_int2(i, code);
          }
        });
      if (!grid_barrier(bar, st, kBarrierPolls)) break;
      if (threadIdx.x == 0) found = 0;
      __syncthreads();
      const long long tn = st->total_images;
      const int nl = (int)((tn > b.check_list_length) ? b.check_list_length : tn);
      if (*(volatile int *)&st->cand_weighted >= nl) {
        if (threadIdx.x == 0) found = 1;
      } else {
        const int l = min(*(volatile int *)&st->cand_n, b.check_list_length);
        candidate_pair_test_global<BLOCK>(copy_view(a), b.L, a.cand, l, lag, b.sl2, b.rc2, blockIdx.x, gridDim.x,
                                          &found);
      }
      __syncthreads();
      if (threadIdx.x == 0 && found) st->want_build = 1;
      if (!grid_barrier(bar, st, kBarrierPolls)) break;
      stale = *(volatile int *)&st->want_build != 0;
      if (lead) {
        // the check is over: its counters are free for the next one
        st->dr2max_bits = 0ull;
        st->cand_weighted = 0;
        st->cand_n = 0;
        st->vlag_set = 0;  // k_decide: the check has read the ghost copies
      }
      if (stale) break;  // a rebuild is left to the caller's ordinary step
    }
    if (g == 0) break;
    // the step: block 0 clears the ring slot step taken + 1 will fill
    if (lead) {
      st->vmax2_ring[(taken + 1) % 3] = 0ull;
      if (!checked) st->vlag_set = 0;  // expiry_decide's clear: no check reads the copies this step
      sim_time += b.dt;
    }
    const int4 *qf = parity ? qf1 : qf0;
    int4 *qf_next = parity ? qf0 : qf1;
    unsigned long long *ring = &st->vmax2_ring[taken % 3];
    // warps walk whole warps of threads, so the lane shuffles stay converged
    for (long long base = (long long)blockIdx.x * BLOCK + (threadIdx.x & ~31); base < nthreads; base += stride) {
      const long long t = base + (threadIdx.x & 31);
      const int i = (int)(t / TPA), sub = (int)(t % TPA);
      const int err = warp_error(st);
      double v2 = 0.0, ke = 0.0;
      if (t < nthreads && !err) {
        const int4 pi = qf[i];
        double Fx, Fy, Fz;
        GlobalGroups<> f{a.nbr + i, a.stride, qf, i};
        fp32_row<TPA>(f, (a.nnbr[i] + 3) >> 2, sub, pi, k, Fx, Fy, Fz);
        if (sub == 0) fp32_finish<kKick, 2>(a, b, th, i, Fx, Fy, Fz, qf_next, v2, ke);
      }
      warp_max_to(ring, v2);
    }
    parity ^= 1;
    if (!grid_barrier(bar, st, kBarrierPolls)) {
      taken++;
      break;
    }
    vmax2 = *(volatile unsigned long long *)ring;
  }
  if (lead) {
    st->steps = steps0 + taken;
    st->sim_time = sim_time;
    st->budget = budget;
    // expiry_decide's clear at a step that stopped for a rebuild; else the
    // last pass's maximum, which the next decision reads
    st->vmax2_bits = checked && stale ? 0ull : vmax2;
    st->disp_checks += checks;
    if (stale) {
      st->list_stale = 1;
      st->want_build = 1;
    }
    st->fix_parity = parity;
    st->persistent_steps += taken;
  }
}

// The rebuild step of the persistent pipeline: queued after each persistent
// launch, it runs only when that launch stopped for a rebuild (a stale
// list, no error, steps left).  Then it takes expiry_decide's stale-list
// branch (want_build, the |v| maximum cleared) and the graph body rebuilds,
// packs buffer 0 and runs the fused step from it.
static __global__ void k_rebuild_guard(Arrays a, Box b, cudaGraphConditionalHandle h_run) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Status *st = a.st;
  int run = !st->error && st->list_stale && st->steps < st->target_steps;
  if (run) {
    int disp = 0;
    run = expiry_decide(st, b, &disp) && !st->error;
  }
  cudaGraphSetConditional(h_run, run);
}

static __global__ void k_set_parity(Arrays a, int parity) {
  if (threadIdx.x == 0 && blockIdx.x == 0 && !a.st->error) a.st->fix_parity = parity;
}

// Start of a persistent pipeline run: the step count to stop at and the
// buffer the next fused step reads.
static __global__ void k_set_target(Arrays a, long long target, int parity) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  a.st->target_steps = target;
  a.st->fix_parity = parity;
}

// Kinetic energy partials (KineticEnergyObserver, src/observer.cc:4-15).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_ke_partial(Arrays a, int n) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  double ke = 0.0;
  if (i < n) {
    const double4 v = a.v[i];
    ke = dadd(dadd(dmul(dmul(0.5, v.x), v.x), dmul(dmul(0.5, v.y), v.y)), dmul(dmul(0.5, v.z), v.z));
  }
  double s[1] = {ke};
  block_sum_to<BLOCK, 1>(s, a.partials);
}

// Sums nblocks partials in a fixed order; Nose-Hoover: T = KE/N/1.5,
// zeta += (T - T0)/tau^2 * dt/2 (ForceCalculator::HeatbathZeta, src/fcalculator.cc:979-985).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_zeta(Arrays a, Box b, int nblocks, int n, double aimed_t,
                                                double tau) {
  __shared__ double sm[BLOCK];
  double s = 0.0;
  for (int k = threadIdx.x; k < nblocks; k += BLOCK) s += a.partials[k];
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int off = BLOCK / 2; off > 0; off >>= 1) {
    if (threadIdx.x < off) sm[threadIdx.x] += sm[threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0 && !a.st->error) {
    const double t = sm[0] / (double)n / 1.5;
    const double t1 = (t - aimed_t) / (tau * tau);
    a.st->zeta += t1 * (b.dt * 0.5);
  }
}

// Observers: KE, PE, virial per atom over the full list, x 1/2 for pair sums
// (PotentialEnergyObserver / VirialObserver, src/observer.cc:17-79: each
// pair term formed as the reference forms it).  lag > 0 reproduces what the
// reference's observers see after a full NVE or Nose-Hoover step: a partner
// reached through the periodic boundary is a ghost copy refreshed after the
// first half drift (MDManager::SendBorderParticles, src/mdmanager.cc:165-167),
// i.e. the partner's position lag = dt/2 earlier, q_j - v_j dt/2.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_observe(Arrays a, Box b, int n, double lag) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  double ke = 0.0, pe = 0.0, vir = 0.0;
  if (i < n) {
    const double4 v = a.v[i];
    ke = dadd(dadd(dmul(dmul(0.5, v.x), v.x), dmul(dmul(0.5, v.y), v.y)), dmul(dmul(0.5, v.z), v.z));
    const double4 qi = a.q[i];
    const double4 *vl = lag_velocities(a);
    const int nn = a.nnbr[i];
    for (int k = 0; k < nn; k++) {
      const int j = a.nbr[(size_t)k * a.stride + i];
      double4 qj = a.q[j];
      if (lag > 0.0 && (fabs(qj.x - qi.x) > b.hL[0] || fabs(qj.y - qi.y) > b.hL[1] ||
                        fabs(qj.z - qi.z) > b.hL[2])) {
        const double4 vj = vl[j];
        qj.x = dsub(qj.x, dmul(vj.x, lag));
        qj.y = dsub(qj.y, dmul(vj.y, lag));
        qj.z = dsub(qj.z, dmul(vj.z, lag));
      }
      const double dx = dsub(qi.x, image_of(qj.x, qi.x, b.L[0], b.hL[0]));
      const double dy = dsub(qi.y, image_of(qj.y, qi.y, b.L[1], b.hL[1]));
      const double dz = dsub(qi.z, image_of(qj.z, qi.z, b.L[2], b.hL[2]));
      const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
      if (r2 > b.rc2) continue;
      const double r4 = dmul(r2, r2), r6 = dmul(r4, r2), r8 = dmul(r6, r2), r10 = dmul(r8, r2),
                   r12 = dmul(r10, r2);
      const double e = dmul(4.0, dadd(dadd(dsub(ddiv(1.0, r12), ddiv(1.0, r6)), dmul(b.c2, r2)), b.c0));
      pe = dadd(pe, e);
      const double r6v = dmul(dmul(r2, r2), r2);
      const double w = dmul(dadd(ddiv(dsub(dmul(24.0, r6v), 48.0), dmul(dmul(r6v, r6v), r2)), b.c2 * 8.0), r2);
      vir = dadd(vir, w);
    }
  }
  double s[3] = {ke, 0.5 * pe, 0.5 * vir};
  block_sum_to<BLOCK, 3>(s, a.partials);
}

// Fixed-order final sum of NSUM-wide partials into out[0..NSUM).
template <int BLOCK, int NSUM>
__global__ void __launch_bounds__(BLOCK) k_final_sum(const double *partials, int nblocks, double *out) {
  __shared__ double sm[NSUM][BLOCK];
  for (int k = 0; k < NSUM; k++) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += BLOCK) s += partials[(size_t)b * NSUM + k];
    sm[k][threadIdx.x] = s;
  }
  __syncthreads();
  for (int off = BLOCK / 2; off > 0; off >>= 1) {
    if (threadIdx.x < off)
      for (int k = 0; k < NSUM; k++) sm[k][threadIdx.x] += sm[k][threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < NSUM; k++) out[k] = sm[k][0];
}

// Directed list entries within the cut-off (the pairs whose force is
// evaluated), with the reference's r^2 test (src/fcalculator.cc:268), summed
// into counts[0]; counts[1] gets all list entries.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_count_pairs(Arrays a, Box b, int n, unsigned long long *counts) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  int within = 0, nn = 0;
  if (i < n) {
    const double4 qi = a.q[i];
    nn = a.nnbr[i];
    for (int k = 0; k < nn; k++) {
      const double4 qj = a.q[a.nbr[(size_t)k * a.stride + i]];
      const double dx = dsub(image_of(qj.x, qi.x, b.L[0], b.hL[0]), qi.x);
      const double dy = dsub(image_of(qj.y, qi.y, b.L[1], b.hL[1]), qi.y);
      const double dz = dsub(image_of(qj.z, qi.z, b.L[2], b.hL[2]), qi.z);
      const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
      within += (r2 > b.rc2) ? 0 : 1;
    }
  }
  const int ws = __reduce_add_sync(0xffffffffu, within);
  const int ns = __reduce_add_sync(0xffffffffu, nn);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&counts[0], (unsigned long long)ws);
    atomicAdd(&counts[1], (unsigned long long)ns);
  }
}

// End of step bookkeeping (MDManager::Calculate: s_time += TimeStep).
static __global__ void k_step_done(Arrays a, Box b) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (a.st->error) return;
  a.st->steps++;
  a.st->sim_time += b.dt;
}

// Langevin alone (ForceCalculator::Langevin, src/fcalculator.cc:1001-1017),
// for callers that run the step piece by piece; the noise counter is the
// device step count, as in the fused kick.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_langevin(Arrays a, Box b, int n, Thermo th) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  if (i >= n || a.st->error) return;
  double4 v = a.v[i];
  double z[3];
  langevin_normals(th.seed, (uint32_t)a.ids[i], (unsigned long long)a.st->steps, z);
  const double dt = b.dt;
  v.x = dadd(v.x, dmul(dadd(dmul(-th.gamma, v.x), dmul(th.noise_sd, z[0])), dt));
  v.y = dadd(v.y, dmul(dadd(dmul(-th.gamma, v.y), dmul(th.noise_sd, z[1])), dt));
  v.z = dadd(v.z, dmul(dadd(dmul(-th.gamma, v.z), dmul(th.noise_sd, z[2])), dt));
  a.v[i] = v;
}

// HeatbathMomenta alone (src/fcalculator.cc:987-999).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_scale_v(Arrays a, int n, double dt2) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  if (i >= n) return;
  const double e = exp(-dt2 * a.st->zeta);
  double4 v = a.v[i];
  v.x = dmul(v.x, e); v.y = dmul(v.y, e); v.z = dmul(v.z, e);
  a.v[i] = v;
}

}  // namespace mdg
