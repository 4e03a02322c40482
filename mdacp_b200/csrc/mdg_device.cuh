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
//   qloc      float4[cap]    cell-local FP32 coordinates at the last build
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
  float4 *qloc;       // cell-local FP32 coordinates at the last build (list prefilter)
  int *ids, *type;
  int *cell;          // cell of each slot at the last build
  int *nbr, *nnbr;
  int *cell_count, *cell_start;
  int *slot;          // rank inside the cell from the atomic scatter
  int *perm, *perm2;  // new slot -> old slot
  double4 *q_tmp, *v_tmp;
  int *ids_tmp, *type_tmp, *cell_tmp;
  unsigned char *mult; // ghost-border membership at the last build (bits, see border_bits)
  int2 *cand;         // displacement-check candidates: (slot, image code)
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

// ------------------------------------------------------------------ helpers
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

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
// displacement check once the budget is spent.  Sets the two conditional
// handles of this step's graph (or device flags in eager mode).
static __global__ void k_expiry(Arrays a, Box b, cudaGraphConditionalHandle h_disp,
                                cudaGraphConditionalHandle h_build, int in_graph, int *eager_flags) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Status *st = a.st;
  int disp = 0, build = 0;
  if (st->error == 0) {
    if (st->list_stale) {
      build = 1;
    } else {
      if (st->budget > 0.0) {
        const double vmax = sqrt(__longlong_as_double((long long)st->vmax2_bits));
        if (vmax * 2.0 * b.dt > b.buffer_length) {
          st->too_fast_v = vmax;
          atomicOr(&st->error, kErrTooFast);
        } else {
          st->budget = st->budget - vmax * 2.0 * b.dt;
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

__device__ __forceinline__ CopyView copy_view(const Arrays &a) { return CopyView{a.q_old, a.q, a.v, a.mult}; }

// PairList::CheckByDisplacement, first pass: max |qb_old - q|^2 over all
// copies (src/pairlist.cc:67-84).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_disp_max(Arrays a, Box b, int n, double lag) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  double d2 = 0.0;
  if (i < n) for_each_copy(copy_view(a), b.L, i, lag, [&](int, double x) { d2 = fmax(d2, x); });
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

// Rebuild 3/6: scatter old slots to their cell ranges.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_scatter(Arrays a, int n) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  if (i >= n || a.st->error) return;
  a.perm[a.cell_start[a.cell[i]] + a.slot[i]] = i;
}

// Rebuild 4/6: order every cell by upload id (one warp per cell), which makes
// the slot order a function of the state alone, independent of atomics.
static __global__ void k_sort_cells(Arrays a, int ncell) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= ncell || a.st->error) return;
  const int beg = a.cell_start[warp], cnt = a.cell_start[warp + 1] - beg;
  for (int base = 0; base < cnt; base += 32) {
    const int me = base + lane;
    int my_slot = -1, my_key = 0x7fffffff;
    if (me < cnt) {
      my_slot = a.perm[beg + me];
      my_key = a.ids[my_slot];
    }
    int rank = 0;
    for (int ob = 0; ob < cnt; ob += 32) {
      const int other = ob + lane;
      int okey = 0x7fffffff;
      if (other < cnt) okey = a.ids[a.perm[beg + other]];
      for (int k = 0; k < 32; k++) {
        const int kk = __shfl_sync(0xffffffffu, okey, k);
        if (ob + k < cnt && kk < my_key) rank++;
      }
    }
    if (me < cnt) a.perm2[beg + rank] = my_slot;
  }
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
    // cell-local FP32 coordinates for the list prefilter
    const int c = a.cell_tmp[s];
    const int cx = c % b.ms[0], cy = (c / b.ms[0]) % b.ms[1], cz = c / (b.ms[0] * b.ms[1]);
    a.qloc[s] = make_float4((float)(q.x - cx * b.cs[0]), (float)(q.y - cy * b.cs[1]),
                            (float)(q.z - cz * b.cs[2]), 0.f);
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

// Rebuild 6/6: full Verlet list.  One thread per atom walks the 27 cells
// around its own (periodic, >= 3 cells per axis so they are distinct).  Each
// candidate is first tested in FP32 on cell-local coordinates (one FADD per
// axis: the neighbour cell's offset is folded into a per-cell base); only
// candidates whose FP32 r^2 falls in a thin band around SearchLength^2 --
// wider than the FP32 error by a factor of about 40 -- are decided by the
// exact FP64 test, so the pair set is the reference's bit for bit.  Row
// order: cells in (dz,dy,dx) order, slots ascending; rows padded with the
// atom's own index to a multiple of 4.
template <int BLOCK, bool STAGE>
__global__ void __launch_bounds__(BLOCK) k_build(Arrays a, Box b, int n) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
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
  if (i < n && !a.st->error) {
    const float4 li = a.qloc[i];
    const int c = a.cell_tmp[i];
    const int cx = c % b.ms[0], cy = (c / b.ms[0]) % b.ms[1], cz = c / (b.ms[0] * b.ms[1]);
    const int maxnb = a.maxnb, stride = a.stride;
    const float lo = b.sl2_lo, hi = b.sl2_hi;
    for (int dz = -1; dz <= 1; dz++) {
      int z = cz + dz;
      double sz = 0.0;
      if (z < 0) { z += b.ms[2]; sz = -b.L[2]; } else if (z >= b.ms[2]) { z -= b.ms[2]; sz = b.L[2]; }
      const float bz = (float)((z - cz) * b.cs[2] + sz) - li.z;
      for (int dy = -1; dy <= 1; dy++) {
        int y = cy + dy;
        double sy = 0.0;
        if (y < 0) { y += b.ms[1]; sy = -b.L[1]; } else if (y >= b.ms[1]) { y -= b.ms[1]; sy = b.L[1]; }
        const float by = (float)((y - cy) * b.cs[1] + sy) - li.y;
        for (int dx = -1; dx <= 1; dx++) {
          int x = cx + dx;
          double sx = 0.0;
          if (x < 0) { x += b.ms[0]; sx = -b.L[0]; } else if (x >= b.ms[0]) { x -= b.ms[0]; sx = b.L[0]; }
          const float bx = (float)((x - cx) * b.cs[0] + sx) - li.x;
          const int nc = (z * b.ms[1] + y) * b.ms[0] + x;
          const int beg = a.cell_start[nc], end = a.cell_start[nc + 1];
          const int need = needed_strips(sx, sy, sz);
          const int shift = (STAGE && npl > 0) ? stage_shift(plan, npl, nc) : 0;
          // one candidate, in row order (FP32 prefilter, ghost rule, exact band)
          auto accept = [&](int j, float r2) {
            if (r2 > hi || j == i) return;
            if (need && (a.mult[j] & need) != need) return;
            if (r2 >= lo && !within_search_exact(a.q[i], a.q[j], sx, sy, sz, b.sl2)) return;
            if (cnt < maxnb) {
              a.nbr[(size_t)cnt * stride + i] = j;
              if (STAGE && npl > 0) {
                int v = j + shift;
                if (v < 0 || v >= staged_atoms) {
                  atomicOr(&a.st->error, kErrStage);
                  v = 0;
                }
                stage_entry(a.nbr16, stride, i, cnt, v, g0, g1);
              }
            }
            cnt++;
          };
          auto dist2f = [&](const float4 &lj) {
            const float ex = lj.x + bx, ey = lj.y + by, ez = lj.z + bz;
            return fmaf(ex, ex, fmaf(ey, ey, ez * ez));
          };
          // two candidates per iteration: both loads issue before either
          // test (the loop is bound by their latency)
          int j = beg;
          for (; j + 1 < end; j += 2) {
            const float4 l0 = a.qloc[j], l1 = a.qloc[j + 1];
            const float r0 = dist2f(l0), r1 = dist2f(l1);
            accept(j, r0);
            accept(j + 1, r1);
          }
          if (j < end) accept(j, dist2f(a.qloc[j]));
        }
      }
    }
    a.nnbr[i] = min(cnt, maxnb);
    if (cnt > maxnb) {
      atomicOr(&a.st->error, kErrCapacity);
    } else {
      int self = (STAGE && npl > 0) ? i + stage_shift(plan, npl, c) : 0;
      if (STAGE && npl > 0 && (self < 0 || self >= staged_atoms)) {
        atomicOr(&a.st->error, kErrStage);
        self = 0;
      }
      for (int k = cnt; k < ((cnt + 3) & ~3); k++) {
        a.nbr[(size_t)k * stride + i] = i;
        if (STAGE && npl > 0) stage_entry(a.nbr16, stride, i, k, self, g0, g1);
      }
    }
  }
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

// After a build: fresh skin budget (PairList::Init, src/pairlist.cc:10-23),
// counters, |v|^2 max for the next expiry test is untouched.
static __global__ void k_build_done(Arrays a, Box b) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Status *st = a.st;
  if (st->error) return;
  st->budget = b.buffer_length;
  st->list_stale = 0;
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
  if (threadIdx.x == 0 && blockIdx.x == 0 && !a.st->error) a.st->vmax2_bits = 0ull;
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
    int j = nn > 0 ? row[0] : 0;
    for (int k = 0; k < nn; k++) {
      const int jn = (k + 1 < nn) ? row[(size_t)(k + 1) * a.stride] : 0;
      const double4 qj = a.q[j];
      const double dx = dsub(image_of(qj.x, qi.x, b.L[0], b.hL[0]), qi.x);
      const double dy = dsub(image_of(qj.y, qi.y, b.L[1], b.hL[1]), qi.y);
      const double dz = dsub(image_of(qj.z, qi.z, b.L[2], b.hL[2]), qi.z);
      const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
      j = jn;
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

// Row sum of atom i from the global fixed-point copy: rows are padded to a
// multiple of 4, so the row is walked four partners at a time without
// per-lane masks, with the indices of the next eight partners already in
// flight (the list is the one stream from HBM, so its loads are issued two
// groups ahead); FP32 partial sums over 8 partners are folded into the FP64
// sums.
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
    if (k & 4) {
      Fx += (double)fx;
      Fy += (double)fy;
      Fz += (double)fz;
      fx = fy = fz = 0.f;
    }
  }
  Fx += (double)fx;
  Fy += (double)fy;
  Fz += (double)fz;
}

// The same row sum from the block's stage in shared memory: one 8-byte load
// brings four stage indices; the next two groups are in flight.
__device__ __forceinline__ unsigned stage_index(unsigned v, unsigned nstage, bool &bad) {
  const bool out = v >= nstage;
  bad |= out;
  return out ? 0u : v;
}

__device__ __forceinline__ void fp32_row_staged(const Arrays &a, const Box &b, const int4 *pos, unsigned nstage,
                                                int i, const int4 &pi, int nn4, double &Fx, double &Fy,
                                                double &Fz) {
  const float sx = b.fix_scale[0], sy = b.fix_scale[1], sz = b.fix_scale[2];
  const unsigned rc2_bits = __float_as_uint(b.rc2f);
  const float c2x8 = b.c2x8f;
  const uint2 *row = a.nbr16 + i;
  const int st = a.stride;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  uint2 g = make_uint2(0u, 0u), gn = make_uint2(0u, 0u);
  bool bad = false;  // an index outside the stage: flagged, the read skipped
  if (nn4 > 0) g = __ldg(row);
  if (nn4 > 4) gn = __ldg(row + st);
  for (int k = 0; k < nn4; k += 4) {
    const int4 p0 = pos[stage_index(g.x & 0xffffu, nstage, bad)];
    const int4 p1 = pos[stage_index(g.x >> 16, nstage, bad)];
    const int4 p2 = pos[stage_index(g.y & 0xffffu, nstage, bad)];
    const int4 p3 = pos[stage_index(g.y >> 16, nstage, bad)];
    g = gn;
    if (k + 8 < nn4) gn = __ldg(row + (size_t)((k + 8) >> 2) * st);
    lj_pair_fp32(pi, p0, sx, sy, sz, rc2_bits, c2x8, fx, fy, fz);
    lj_pair_fp32(pi, p1, sx, sy, sz, rc2_bits, c2x8, fx, fy, fz);
    lj_pair_fp32(pi, p2, sx, sy, sz, rc2_bits, c2x8, fx, fy, fz);
    lj_pair_fp32(pi, p3, sx, sy, sz, rc2_bits, c2x8, fx, fy, fz);
    if (k & 4) {
      Fx += (double)fx;
      Fy += (double)fy;
      Fz += (double)fz;
      fx = fy = fz = 0.f;
    }
  }
  Fx += (double)fx;
  Fy += (double)fy;
  Fz += (double)fz;
  if (bad) atomicOr(&a.st->error, kErrStage);
}

// FP32-mixed force kick.  Displacements come from the fixed-point copy (no
// ghost atoms, no shift codes); the row sum is fp32_row_global's and the
// kick is FP64.  With DRIFT the second half drift q += v dt/2 and the |v|
// maximum of the step are done in the same pass: this kernel reads only the
// fixed-point copy, so moving q here races with no other thread.  DRIFT == 2
// is the whole NVE step in one pass: qf holds every atom's position after
// this step's first half drift (packed by the previous step's pass, or by
// k_pack_half after a rebuild); the kernel applies that drift to its own
// atom, kicks, drifts again and packs the next step's first-drift position
// into qf_next (the other buffer, so no thread overwrites a copy that
// another still reads).  The arithmetic is the separate drift kernels',
// operation for operation.
template <int BLOCK, int MODE, int DRIFT>
__global__ void __launch_bounds__(BLOCK) k_force_fp32(Arrays a, Box b, int n, Thermo th, const int4 *qf,
                                                      int4 *qf_next) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  double v2 = 0.0, ke = 0.0;
  if (DRIFT == 2 && MODE == kKick && i == 0 && !a.st->error) {
    // the step counter (k_step_done's work): nothing in this pass reads it
    a.st->steps++;
    a.st->sim_time += b.dt;
  }
  if (i < n && !a.st->error) {
    const int4 pi = qf[i];
    const int nn4 = (a.nnbr[i] + 3) & ~3;
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    fp32_row_global(a, b, qf, i, pi, nn4, Fx, Fy, Fz);
    fp32_finish<MODE, DRIFT>(a, b, th, i, Fx, Fy, Fz, qf_next, v2, ke);
  }
  if (MODE == kKickLangevin || DRIFT) warp_max_to(&a.st->vmax2_bits, v2);
  if (MODE == kKickNoseHoover) {
    double s[1] = {ke};
    block_sum_to<BLOCK, 1>(s, a.partials);
  }
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

// Waits for the mbarrier's phase `parity` to complete, for at most
// `limit` clock cycles; false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit) {
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) return false;
  }
}

// About one second at the B200's clocks: a stage copy takes microseconds.
constexpr long long kStageWaitCycles = 2000000000ll;

// The staged FP32-mixed pass: k_force_fp32 with the partners' positions read
// from the block's stage (k_stage_plan) in dynamic shared memory, which one
// thread fills with one bulk copy per plan range while the others wait on an
// mbarrier.  Blocks without a plan (-1) gather from global memory.  If the
// wait gives up (kStageWaitCycles), the block sets kErrTimeout, waits once
// more for its copies in flight, and kicks no atom.
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
    ok = mbar_wait(&bar, 0, kStageWaitCycles);
    if (!ok) {
      atomicOr(&a.st->error, kErrTimeout);
      mbar_wait(&bar, 0, kStageWaitCycles);
    }
  }
  if (ok && i < n && !a.st->error) {
    const int4 pi = qf[i];
    const int nn4 = (a.nnbr[i] + 3) & ~3;
    double Fx = 0.0, Fy = 0.0, Fz = 0.0;
    if (use_stage) fp32_row_staged(a, b, pos, nstage, i, pi, nn4, Fx, Fy, Fz);
    else fp32_row_global(a, b, qf, i, pi, nn4, Fx, Fy, Fz);
    fp32_finish<MODE, DRIFT>(a, b, th, i, Fx, Fy, Fz, qf_next, v2, ke);
  }
  if (MODE == kKickLangevin || DRIFT) warp_max_to(&a.st->vmax2_bits, v2);
  if (MODE == kKickNoseHoover) {
    double s[1] = {ke};
    block_sum_to<BLOCK, 1>(s, a.partials);
  }
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
    const int nn = a.nnbr[i];
    for (int k = 0; k < nn; k++) {
      const int j = a.nbr[(size_t)k * a.stride + i];
      double4 qj = a.q[j];
      if (lag > 0.0 && (fabs(qj.x - qi.x) > b.hL[0] || fabs(qj.y - qi.y) > b.hL[1] ||
                        fabs(qj.z - qi.z) > b.hL[2])) {
        const double4 vj = a.v[j];
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
