// Replica ensembles: many independent periodic LJ systems of different
// size, density and temperature advanced together.  Every kernel of a step
// covers all replicas in one launch: atoms of all replicas are concatenated,
// a per-atom replica index selects the replica's row of the offset tables
// (box, cell grid, cell and atom offsets), and skin budgets, displacement
// checks and pairlist rebuilds are per replica -- a rebuild pass only
// touches the replicas whose lists expired.  Steps are captured in CUDA
// graphs with IF conditional nodes on "some replica needs a displacement
// check / a rebuild", exactly like the single-system handle.
//
// The arithmetic of every kernel is the single-system kernels' (shared
// device helpers from mdg_device.cuh), and rows are built in the same order,
// so a replica advanced in an ensemble is bit-identical to the same system
// advanced alone.  Replicas with fewer than 3 cells per axis (boxes under
// 3 x SearchLength) are searched all-pairs with the minimum image, which
// needs L > 2 x SearchLength.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "mdacp_b200.h"
#include "mdg_device.cuh"

namespace mdg {
namespace {

constexpr int kEB = 256;        // streaming kernels
constexpr int kEF = 128;        // pair kernels
constexpr int kEStepsPerGraph = 20;
constexpr int kEPairParts = 8;  // blocks per replica in the candidate-pair test

struct Rep {
  double L[3], hL[3], inv_cs[3], cs[3];
  float fix_scale[3];
  int ms[3];
  int ncell, cell_off, atom_off, n;
  long long tab_off;  // first entry of the replica's rows in the trim table
  int small;  // all-pairs search (fewer than 3 cells along an axis)
  // the replica's BufferLength, SearchLength = cut-off + it, and the FP32
  // prefilter band around SearchLength^2
  double buffer_length, sl, sl2;
  float sl2_lo, sl2_hi;
};

struct RepStatus {
  unsigned long long vmax2_bits;
  unsigned long long dr2max_bits;
  double budget;
  int cand_weighted, cand_n;
  int disp, want_build, build, list_stale;
  int max_row, pad;
  long long total_images, rebuilds, steps, disp_checks;
  long long list_entries;  // neighbour entries of the last build
};

// The replicas a skin check or a rebuild acts on, compacted in replica order
// (ke_make_list), with the prefix sums that map a work index to an atom or
// a cell: the per-atom and per-cell kernels of those branches sweep only
// these atoms and cells.
struct WorkList {
  int *rep;          // [count[0]] acting replicas, ascending
  int *atom_prefix;  // [count[0] + 1] first work atom of each
  int *cell_prefix;  // [count[0] + 1] first work cell of each
  int *count;        // replicas, atoms, cells
};

struct Ens {
  const Rep *rep;
  RepStatus *rs;
  const int *rep_of;  // replica of each atom slot (fixed: atoms move only within their replica)
  double4 *q, *v, *q_old;
  int4 *qfix;
  float4 *qloc;
  int *cxyz, *xsub;  // packed cell coordinates and the list-build trim table (as the single-system arrays)
  int *ids, *cell, *cell_tmp, *nbr, *nnbr, *cell_count, *cell_start, *slot, *perm, *perm2;
  double lag;  // age of the reference's ghost copies at the skin check
  double4 *q_tmp, *v_tmp;
  int *ids_tmp;
  unsigned char *mult;
  int2 *cand;  // nrep x cll candidate copies (slot, image code)
  double *disp2;  // per atom: the largest squared copy displacement of the last skin check (ke_disp_max)
  int *error;
  double *sums;  // nrep x 3 observer sums
  WorkList wd, wb;  // skin-check and rebuild work lists
  int stride, maxnb, nrep, ntot, cll;
  double rc2, c0, c2, dt;
  float rc2f, c2x8f;
};

// Box of a replica in the single-system kernels' layout.
__device__ __forceinline__ Box box_of(const Ens &e, const Rep &r) {
  Box b;
  for (int d = 0; d < 3; d++) {
    b.L[d] = r.L[d];
    b.hL[d] = r.hL[d];
    b.inv_cs[d] = r.inv_cs[d];
    b.cs[d] = r.cs[d];
    b.ms[d] = r.ms[d];
    b.fix_scale[d] = r.fix_scale[d];
  }
  b.ncell = r.ncell;
  b.sl = r.sl;
  b.sl2 = r.sl2;
  b.rc2 = e.rc2;
  b.c0 = e.c0;
  b.c2 = e.c2;
  b.dt = e.dt;
  b.buffer_length = r.buffer_length;
  b.rc2f = e.rc2f;
  b.c2x8f = e.c2x8f;
  b.check_list_length = e.cll;
  b.sl2_lo = r.sl2_lo;
  b.sl2_hi = r.sl2_hi;
  b.slab = 0;
  b.z0 = 0;
  b.nzl = r.ms[2];
  return b;
}

// Max of a non-negative double into the replica's slot.  A warp whose
// active lanes all belong to one replica (all but the few warps that
// straddle a replica boundary) reduces first and issues one atomic; the
// others issue one atomic per active lane.  All lanes must call.
__device__ __forceinline__ void rep_max(unsigned long long *slot_base, size_t stride_bytes, int r, double v,
                                        bool active) {
  const int rr = active ? r : -1;
  const int r0 = __shfl_sync(0xffffffffu, rr, 0);
  const bool uniform = __all_sync(0xffffffffu, rr == r0) && r0 >= 0;
  if (uniform) {
    double m = v;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) {
      unsigned long long *p = (unsigned long long *)((char *)slot_base + stride_bytes * r0);
      atomicMax(p, (unsigned long long)__double_as_longlong(m));
    }
  } else if (active) {
    unsigned long long *p = (unsigned long long *)((char *)slot_base + stride_bytes * r);
    atomicMax(p, (unsigned long long)__double_as_longlong(v));
  }
}

// Sum of a count into the replica's slot, with the warp reduction of
// rep_max for warps whose active lanes share one replica.  All lanes must call.
__device__ __forceinline__ void rep_add(long long *slot_base, size_t stride_bytes, int r, long long v,
                                        bool active) {
  const int rr = active ? r : -1;
  const int r0 = __shfl_sync(0xffffffffu, rr, 0);
  const bool uniform = __all_sync(0xffffffffu, rr == r0) && r0 >= 0;
  if (uniform) {
    long long m = v;
    for (int o = 16; o > 0; o >>= 1) m += __shfl_xor_sync(0xffffffffu, m, o);
    if ((threadIdx.x & 31) == 0 && m) {
      long long *p = (long long *)((char *)slot_base + stride_bytes * r0);
      atomicAdd((unsigned long long *)p, (unsigned long long)m);
    }
  } else if (active && v) {
    long long *p = (long long *)((char *)slot_base + stride_bytes * r);
    atomicAdd((unsigned long long *)p, (unsigned long long)v);
  }
}

// Index k of the work-list replica that holds work item g (the largest k
// with prefix[k] <= g; nk >= 1).
__device__ __forceinline__ int work_find(const int *prefix, int nk, int g) {
  int lo = 0, hi = nk - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (prefix[mid] <= g) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Replica and atom slot of work atom g of list w.
__device__ __forceinline__ int work_atom(const Ens &e, const WorkList &w, int g, int *r) {
  const int k = work_find(w.atom_prefix, w.count[0], g);
  *r = w.rep[k];
  return e.rep[*r].atom_off + (g - w.atom_prefix[k]);
}

// One block, 1024 threads: the work list of the replicas whose disp (WHICH
// 0) or build (WHICH 1) flag is set.
template <int WHICH>
__global__ void __launch_bounds__(1024) ke_make_list(Ens e) {
  const WorkList w = WHICH ? e.wb : e.wd;
  __shared__ int base_k, base_a, base_c, tk, ta, tc;
  if (threadIdx.x == 0) base_k = base_a = base_c = 0;
  __syncthreads();
  for (int r0 = 0; r0 < e.nrep; r0 += 1024) {
    const int r = r0 + threadIdx.x;
    int f = 0, na = 0, nc = 0;
    if (r < e.nrep) {
      f = WHICH ? e.rs[r].build : e.rs[r].disp;
      f = f != 0;
      if (f) {
        na = e.rep[r].n;
        nc = e.rep[r].ncell;
      }
    }
    const int k = block_exclusive_scan<1024>(f, &tk);
    const int a = block_exclusive_scan<1024>(na, &ta);
    const int c = block_exclusive_scan<1024>(nc, &tc);
    if (f) {
      w.rep[base_k + k] = r;
      w.atom_prefix[base_k + k] = base_a + a;
      w.cell_prefix[base_k + k] = base_c + c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      base_k += tk;
      base_a += ta;
      base_c += tc;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    w.atom_prefix[base_k] = base_a;
    w.cell_prefix[base_k] = base_c;
    w.count[0] = base_k;
    w.count[1] = base_a;
    w.count[2] = base_c;
  }
}

// --------------------------------------------------------------- step kernels
__global__ void ke_expiry(Ens e, cudaGraphConditionalHandle h_disp, int in_graph, int *flags) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int r = threadIdx.x; r < e.nrep; r += blockDim.x) {
    RepStatus &st = e.rs[r];
    int disp = 0, build = 0;
    if (*e.error == 0) {
      if (st.list_stale) {
        build = 1;
      } else {
        if (st.budget > 0.0) {
          const double vmax = sqrt(__longlong_as_double((long long)st.vmax2_bits));
          if (skin_cost(vmax, e.dt) > e.rep[r].buffer_length) atomicOr(e.error, kErrTooFast);
          else st.budget = dsub(st.budget, skin_cost(vmax, e.dt));
        }
        if (st.budget < 0.0) {
          disp = 1;
          st.dr2max_bits = 0ull;
          st.cand_weighted = 0;
          st.cand_n = 0;
          st.disp_checks++;
        }
      }
    }
    st.disp = disp;
    st.want_build = build;
    st.vmax2_bits = 0ull;
    if (disp) any = 1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (in_graph) cudaGraphSetConditional(h_disp, any);
    else flags[0] = any;
    if (any) flags[2]++;  // steps that launch the skin-check branch
  }
}

__device__ __forceinline__ CopyView ens_view(const Ens &e) { return CopyView{e.q_old, e.q, e.v, e.mult}; }

// Skin check per replica, over the reference's copies (see for_each_copy).
// (The atoms of the checked replicas, through the skin-check work list;
// block-uniform sweeps, so every lane reaches rep_max.)
__global__ void __launch_bounds__(kEB) ke_disp_max(Ens e) {
  const int total = e.wd.count[1];
  for (int base = blockIdx.x * kEB; base < total; base += gridDim.x * kEB) {
    const int g = base + threadIdx.x;
    const bool active = g < total;
    int r = 0;
    double d2 = 0.0;
    if (active) {
      const int i = work_atom(e, e.wd, g, &r);
      for_each_copy(ens_view(e), e.rep[r].L, i, e.lag, [&](int, double x) { d2 = fmax(d2, x); });
      e.disp2[i] = d2;
    }
    rep_max(&e.rs[0].dr2max_bits, sizeof(RepStatus), r, d2, active);
  }
}

__global__ void __launch_bounds__(kEB) ke_disp_collect(Ens e) {
  const int total = e.wd.count[1];
  for (int g = blockIdx.x * kEB + threadIdx.x; g < total; g += gridDim.x * kEB) {
    int r;
    const int i = work_atom(e, e.wd, g, &r);
    RepStatus &st = e.rs[r];
    const double c = e.rep[r].buffer_length - sqrt(__longlong_as_double((long long)st.dr2max_bits));
    const double c_d2 = c * c;
    // no copy of this atom moved more than c (ke_disp_max's per-atom
    // maximum of the same displacements): nothing to collect
    if (!(e.disp2[i] > c_d2)) continue;
    for_each_copy(ens_view(e), e.rep[r].L, i, e.lag, [&](int code, double d2) {
      if (d2 > c_d2) {
        atomicAdd(&st.cand_weighted, 1);
        const int k = atomicAdd(&st.cand_n, 1);
        if (k < e.cll) e.cand[(size_t)r * e.cll + k] = make_int2(i, code);
      }
    });
  }
}

// kEPairParts blocks per replica (blockIdx.y) share the rows of the
// candidate-pair test of PairList::CheckByDisplacement.
__global__ void __launch_bounds__(256) ke_disp_pairs(Ens e) {
  const int r = blockIdx.x;
  RepStatus &st = e.rs[r];
  if (!st.disp) return;
  __shared__ PairStage sm;
  __shared__ volatile int found;
  if (threadIdx.x == 0) found = 0;
  __syncthreads();
  const Rep rep = e.rep[r];
  const long long tn = st.total_images;
  const int nl = (int)((tn > e.cll) ? e.cll : tn);
  if (st.cand_weighted >= nl) {
    if (threadIdx.x == 0) found = 1;
  } else {
    const int l = min(st.cand_n, e.cll);
    candidate_pair_test<256>(ens_view(e), rep.L, e.cand + (size_t)r * e.cll, l, e.lag, rep.sl2, e.rc2, blockIdx.y,
                             gridDim.y, sm, &found);
  }
  __syncthreads();
  if (threadIdx.x == 0 && found) st.want_build = 1;
}

__global__ void ke_decide(Ens e, cudaGraphConditionalHandle h_build, int in_graph, int *flags) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int r = threadIdx.x; r < e.nrep; r += blockDim.x) {
    RepStatus &st = e.rs[r];
    const int b = (*e.error == 0) && st.want_build;
    st.build = b;
    st.disp = 0;
    if (b) {
      any = 1;
      st.max_row = 0;
      st.total_images = 0;
      st.list_entries = 0;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (in_graph) cudaGraphSetConditional(h_build, any);
    else flags[1] = any;
    if (any) flags[3]++;  // steps that launch the rebuild branch
  }
}

// ---------------------------------------------------------- rebuild kernels
__global__ void __launch_bounds__(kEB) ke_clear_cells(Ens e) {
  const int r = blockIdx.x;
  if (!e.rs[r].build) return;
  const Rep rep = e.rep[r];
  for (int c = threadIdx.x; c < rep.ncell; c += kEB) e.cell_count[rep.cell_off + c] = 0;
}

// Wraps atom i of replica r into its box (Variables::AdjustPeriodicBoundary,
// src/variables.cc:63-84), checks it, and files it in its cell.
__device__ __forceinline__ void cell_assign_atom(const Ens &e, int r, int i) {
  const Rep &rep = e.rep[r];
  double4 q = e.q[i];
  double x[3] = {q.x, q.y, q.z};
  int cc[3];
  bool bad = false;
  for (int d = 0; d < 3; d++) {
    if (!isfinite(x[d])) {
      atomicOr(e.error, kErrNonFinite);
      return;
    }
    if (x[d] < 0.0) x[d] = dadd(x[d], rep.L[d]);
    else if (x[d] > rep.L[d]) x[d] = dsub(x[d], rep.L[d]);
    bad |= (x[d] < 0.0 || x[d] > rep.L[d]);
    cc[d] = cell_coord(x[d], rep.inv_cs[d], rep.ms[d]);
  }
  if (bad) {
    atomicOr(e.error, kErrInvalidPosition);
    return;
  }
  q.x = x[0]; q.y = x[1]; q.z = x[2];
  e.q[i] = q;
  const int c = rep.cell_off + (cc[2] * rep.ms[1] + cc[1]) * rep.ms[0] + cc[0];
  e.cell[i] = c;
  e.slot[i] = atomicAdd(&e.cell_count[c], 1);
}

// Atoms of the rebuilding replicas (rebuild work list) from here to ke_build.
__global__ void __launch_bounds__(kEB) ke_cell_assign(Ens e) {
  if (*e.error) return;
  const int total = e.wb.count[1];
  for (int g = blockIdx.x * kEB + threadIdx.x; g < total; g += gridDim.x * kEB) {
    int r;
    const int i = work_atom(e, e.wb, g, &r);
    cell_assign_atom(e, r, i);
  }
}

// One block per rebuilding replica: exclusive scan of its cells, offset by
// the replica's first atom slot.
__global__ void __launch_bounds__(kEB) ke_scan_cells(Ens e) {
  const int r = blockIdx.x;
  if (!e.rs[r].build || *e.error) return;
  const Rep rep = e.rep[r];
  __shared__ int sums[kEB];
  const int t = threadIdx.x;
  const int chunk = (rep.ncell + kEB - 1) / kEB;
  const int beg = min(t * chunk, rep.ncell), end = min(beg + chunk, rep.ncell);
  int s = 0;
  for (int c = beg; c < end; c++) s += e.cell_count[rep.cell_off + c];
  sums[t] = s;
  __syncthreads();
  for (int off = 1; off < kEB; off <<= 1) {
    const int x = (t >= off) ? sums[t - off] : 0;
    __syncthreads();
    sums[t] += x;
    __syncthreads();
  }
  int run = rep.atom_off + sums[t] - s;
  for (int c = beg; c < end; c++) {
    e.cell_start[rep.cell_off + c] = run;
    run += e.cell_count[rep.cell_off + c];
  }
}

__global__ void __launch_bounds__(kEB) ke_scatter(Ens e) {
  if (*e.error) return;
  const int total = e.wb.count[1];
  for (int g = blockIdx.x * kEB + threadIdx.x; g < total; g += gridDim.x * kEB) {
    int r;
    const int i = work_atom(e, e.wb, g, &r);
    e.perm[e.cell_start[e.cell[i]] + e.slot[i]] = i;
  }
}

// Warp per cell of a rebuilding replica (the cells of the rebuild work
// list): order by (x, upload id) and the cell's row of the trim table, as
// the single-system k_sort_cells.
__device__ __forceinline__ void sort_cell(const Ens &e, const Rep &rep, int cell, int lane) {
  const int beg = e.cell_start[cell], cnt = e.cell_start[cell + 1] - beg;
  const int c = cell - rep.cell_off, cx = c % rep.ms[0];
  sort_cell_x(e.q, e.ids, e.perm, e.perm2, beg, cnt, cx * rep.cs[0], rep.cs[0] / kXSub,
              trim_entries(e.xsub + rep.tab_off, rep.ms[0], c / rep.ms[0], cx), cx == rep.ms[0] - 1, lane);
}

__global__ void __launch_bounds__(kEB) ke_sort_cells(Ens e) {
  if (*e.error) return;
  const int total = e.wb.count[2], nk = e.wb.count[0];
  const int lane = threadIdx.x & 31;
  const int wstride = gridDim.x * (kEB / 32);
  for (int gc = blockIdx.x * (kEB / 32) + (threadIdx.x >> 5); gc < total; gc += wstride) {
    const int k = work_find(e.wb.cell_prefix, nk, gc);
    const Rep &rep = e.rep[e.wb.rep[k]];
    sort_cell(e, rep, rep.cell_off + (gc - e.wb.cell_prefix[k]), lane);
  }
}

// Gathers the atom that goes to slot s of replica r into the temporary
// arrays, snapshots q_old (PairList::Init), its ghost-strip membership and
// cell-local coordinates; returns its copy count (atom + ghost images).
__device__ __forceinline__ int permute_atom(const Ens &e, int r, int s) {
  const Rep rep = e.rep[r];
  const Box b = box_of(e, rep);
  const int o = e.perm2[s];
  const double4 q = e.q[o];
  e.q_tmp[s] = q;
  e.v_tmp[s] = e.v[o];
  e.ids_tmp[s] = e.ids[o];
  const int cg = e.cell[o];
  e.cell_tmp[s] = cg;
  e.q_old[s] = q;
  const double x[3] = {q.x, q.y, q.z};
  int m = 1;
  e.mult[s] = (unsigned char)border_bits(x, b, &m);
  const int c = cg - rep.cell_off;
  const int cx = c % rep.ms[0], cy = (c / rep.ms[0]) % rep.ms[1], cz = c / (rep.ms[0] * rep.ms[1]);
  e.qloc[s] = make_float4((float)q.x, (float)(q.y - cy * rep.cs[1]), (float)(q.z - cz * rep.cs[2]), 0.f);
  e.cxyz[s] = pack_cell(cx, cy, cz);
  return m;
}

__global__ void __launch_bounds__(kEB) ke_permute(Ens e) {
  const bool err = *e.error != 0;
  const int total = e.wb.count[1];
  for (int base = blockIdx.x * kEB; base < total; base += gridDim.x * kEB) {
    const int g = base + threadIdx.x;
    const bool active = g < total && !err;
    int r = 0, m = 0;
    if (active) {
      const int s = work_atom(e, e.wb, g, &r);
      m = permute_atom(e, r, s);
    }
    rep_add(&e.rs[0].total_images, sizeof(RepStatus), r, m, active);
  }
}

__global__ void __launch_bounds__(kEB) ke_copy_back(Ens e) {
  if (*e.error) return;
  const int total = e.wb.count[1];
  for (int g = blockIdx.x * kEB + threadIdx.x; g < total; g += gridDim.x * kEB) {
    int r;
    const int s = work_atom(e, e.wb, g, &r);
    e.q[s] = e.q_tmp[s];
    e.v[s] = e.v_tmp[s];
    e.ids[s] = e.ids_tmp[s];
  }
}

// One atom's row of the list build, as the single-system build makes it
// (build_rows: same rows in the same order); all-pairs with the minimum
// image for small replicas.  Returns the entries kept.
__device__ __forceinline__ int ens_build_row(const Ens &e, int i) {
  const int r = e.rep_of[i];
  RepStatus &st = e.rs[r];
  const Rep rep = e.rep[r];
  const int maxnb = e.maxnb, stride = e.stride;
  int cnt = 0;
  if (rep.small) {
    const double4 qi = e.q[i];
    for (int j = rep.atom_off; j < rep.atom_off + rep.n; j++) {
      if (j == i) continue;
      const double4 qj = e.q[j];
      // the minimum-image shift per axis (unique: L > 2 SearchLength)
      const double tx = qj.x - qi.x, ty = qj.y - qi.y, tz = qj.z - qi.z;
      const double sx = tx > rep.hL[0] ? -rep.L[0] : (tx < -rep.hL[0] ? rep.L[0] : 0.0);
      const double sy = ty > rep.hL[1] ? -rep.L[1] : (ty < -rep.hL[1] ? rep.L[1] : 0.0);
      const double sz = tz > rep.hL[2] ? -rep.L[2] : (tz < -rep.hL[2] ? rep.L[2] : 0.0);
      const int need = needed_strips(sx, sy, sz);
      if (need && (e.mult[j] & need) != need) continue;
      if (!within_search_exact(qi, qj, sx, sy, sz, rep.sl2)) continue;
      if (cnt < maxnb) e.nbr[(size_t)cnt * stride + i] = j;
      cnt++;
    }
  } else {
    auto emit = [&](int j, int k) {
      if (k < maxnb) e.nbr[(size_t)k * stride + i] = j;
    };
    // without the load pipeline: it takes ke_build from 72 to 152 registers
    cnt = build_rows<false, 1, false>(box_of(e, rep), e.qloc, e.q, e.mult, e.xsub + rep.tab_off, e.cxyz[i], i, emit);
  }
  e.nnbr[i] = min(cnt, maxnb);
  if (cnt > maxnb) {
    atomicOr(e.error, kErrCapacity);
  } else {
    for (int k = cnt; k < ((cnt + 3) & ~3); k++) e.nbr[(size_t)k * stride + i] = i;
  }
  atomicMax(&st.max_row, cnt);
  return min(cnt, maxnb);
}

__global__ void __launch_bounds__(kEF) ke_build(Ens e) {
  const int total = e.wb.count[1];
  for (int base = blockIdx.x * kEF; base < total; base += gridDim.x * kEF) {
    const int g = base + threadIdx.x;
    const bool active = g < total && !*e.error;
    int r = 0, kept = 0;
    if (active) kept = ens_build_row(e, work_atom(e, e.wb, g, &r));
    rep_add(&e.rs[0].list_entries, sizeof(RepStatus), r, kept, active);
  }
}

__global__ void ke_build_done(Ens e) {
  for (int r = threadIdx.x; r < e.nrep; r += blockDim.x) {
    RepStatus &st = e.rs[r];
    if (!st.build || *e.error) continue;
    st.budget = e.rep[r].buffer_length;
    st.list_stale = 0;
    st.rebuilds++;
  }
}

// ------------------------------------------------------------- integrate
template <bool FIX>
__global__ void __launch_bounds__(kEB) ke_drift(Ens e, int track_vmax) {
  const int i = blockIdx.x * kEB + threadIdx.x;
  int r = 0;
  double v2 = 0.0;
  const bool active = i < e.ntot && !*e.error;
  if (active) {
    r = e.rep_of[i];
    const double dt2 = e.dt * 0.5;
    double4 q = e.q[i];
    const double4 v = e.v[i];
    q.x = dadd(q.x, dmul(v.x, dt2));
    q.y = dadd(q.y, dmul(v.y, dt2));
    q.z = dadd(q.z, dmul(v.z, dt2));
    e.q[i] = q;
    if (FIX) {
      const Rep &rep = e.rep[r];
      e.qfix[i] = make_int4(fixed_coord(q.x, rep.L[0]), fixed_coord(q.y, rep.L[1]), fixed_coord(q.z, rep.L[2]), 0);
    }
    if (track_vmax) {
      v2 = dadd(dadd(dmul(v.x, v.x), dmul(v.y, v.y)), dmul(v.z, v.z));
      if (!isfinite(v2) || !isfinite(q.x + q.y + q.z)) atomicOr(e.error, kErrNonFinite);
    }
  }
  if (track_vmax) rep_max(&e.rs[0].vmax2_bits, sizeof(RepStatus), r, v2, active);
}

// FP32-mixed kick with the second half drift fused (the single-system
// k_force_fp32 loop on the replica's fixed-point scale).
template <int TPA>
__global__ void __launch_bounds__(kEF) ke_force_fp32(Ens e) {
  const int t = blockIdx.x * kEF + threadIdx.x;
  const int i = t / TPA, sub = t % TPA;
  int r = 0;
  double v2 = 0.0;
  // the lanes of an atom exchange chunk sums: they agree on the error flag
  const int err = __shfl_sync(0xffffffffu, *(volatile const int *)e.error, 0);
  const bool active = i < e.ntot && !err;
  double Fx = 0.0, Fy = 0.0, Fz = 0.0;
  if (active) {
    r = e.rep_of[i];
    const Rep &rep = e.rep[r];
    // positions not loaded a group ahead: at 64 registers this pass is
    // faster without (0.324 vs 0.353 ms on the 256-replica ensemble)
    GlobalGroups<false> f{e.nbr + i, e.stride, e.qfix, i};
    fp32_row<TPA>(f, (e.nnbr[i] + 3) >> 2, sub, e.qfix[i], pair_const(rep.fix_scale, e.rc2f, e.c2x8f), Fx, Fy, Fz);
  }
  if (active && sub == 0) {
    const double dt = e.dt;
    double4 v = e.v[i];
    v.x = dadd(v.x, Fx * dt);
    v.y = dadd(v.y, Fy * dt);
    v.z = dadd(v.z, Fz * dt);
    e.v[i] = v;
    double4 q = e.q[i];
    const double dt2 = dt * 0.5;
    q.x = dadd(q.x, dmul(v.x, dt2));
    q.y = dadd(q.y, dmul(v.y, dt2));
    q.z = dadd(q.z, dmul(v.z, dt2));
    e.q[i] = q;
    v2 = dadd(dadd(dmul(v.x, v.x), dmul(v.y, v.y)), dmul(v.z, v.z));
    if (!isfinite(v2) || !isfinite(q.x + q.y + q.z)) atomicOr(e.error, kErrNonFinite);
  }
  rep_max(&e.rs[0].vmax2_bits, sizeof(RepStatus), r, v2, active);  // v2 = 0 on lanes other than 0
}

// FP64 kick (the single-system k_force_fp64 pair terms).
__global__ void __launch_bounds__(kEF) ke_force_fp64(Ens e) {
  const int i = blockIdx.x * kEF + threadIdx.x;
  if (i >= e.ntot || *e.error) return;
  const Rep &rep = e.rep[e.rep_of[i]];
  const double4 qi = e.q[i];
  const int nn = e.nnbr[i];
  const double c2x8 = e.c2 * 8.0;
  const double dt = e.dt;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  const int *row = e.nbr + i;
  int j = nn > 0 ? row[0] : 0;
  for (int k = 0; k < nn; k++) {
    const int jn = (k + 1 < nn) ? row[(size_t)(k + 1) * e.stride] : 0;
    const double4 qj = e.q[j];
    const double dx = dsub(image_of(qj.x, qi.x, rep.L[0], rep.hL[0]), qi.x);
    const double dy = dsub(image_of(qj.y, qi.y, rep.L[1], rep.hL[1]), qi.y);
    const double dz = dsub(image_of(qj.z, qi.z, rep.L[2], rep.hL[2]), qi.z);
    const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
    j = jn;
    if (r2 > e.rc2) continue;
    const double r6 = dmul(dmul(r2, r2), r2);
    const double df = dmul(dadd(ddiv(dsub(dmul(24.0, r6), 48.0), dmul(dmul(r6, r6), r2)), c2x8), dt);
    fx = dadd(fx, dmul(df, dx));
    fy = dadd(fy, dmul(df, dy));
    fz = dadd(fz, dmul(df, dz));
  }
  double4 v = e.v[i];
  v.x = dadd(v.x, fx);
  v.y = dadd(v.y, fy);
  v.z = dadd(v.z, fz);
  e.v[i] = v;
}

__global__ void ke_step_done(Ens e) {
  if (*e.error) return;
  for (int r = threadIdx.x; r < e.nrep; r += blockDim.x) e.rs[r].steps++;
}

// Observer sums per replica (KE, PE, virial x 3), pair terms as k_observe.
__global__ void __launch_bounds__(kEB) ke_observe(Ens e) {
  const int i = blockIdx.x * kEB + threadIdx.x;
  if (i >= e.ntot) return;
  const int r = e.rep_of[i];
  const Rep &rep = e.rep[r];
  const double4 v = e.v[i];
  const double ke = dadd(dadd(dmul(dmul(0.5, v.x), v.x), dmul(dmul(0.5, v.y), v.y)), dmul(dmul(0.5, v.z), v.z));
  const double4 qi = e.q[i];
  double pe = 0.0, vir = 0.0;
  const int nn = e.nnbr[i];
  for (int k = 0; k < nn; k++) {
    const double4 qj = e.q[e.nbr[(size_t)k * e.stride + i]];
    const double dx = dsub(qi.x, image_of(qj.x, qi.x, rep.L[0], rep.hL[0]));
    const double dy = dsub(qi.y, image_of(qj.y, qi.y, rep.L[1], rep.hL[1]));
    const double dz = dsub(qi.z, image_of(qj.z, qi.z, rep.L[2], rep.hL[2]));
    const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
    if (r2 > e.rc2) continue;
    const double r4 = dmul(r2, r2), r6 = dmul(r4, r2), r8 = dmul(r6, r2), r10 = dmul(r8, r2), r12 = dmul(r10, r2);
    pe = dadd(pe, dmul(4.0, dadd(dadd(dsub(ddiv(1.0, r12), ddiv(1.0, r6)), dmul(e.c2, r2)), e.c0)));
    vir = dadd(vir, dmul(dadd(ddiv(dsub(dmul(24.0, r6), 48.0), dmul(dmul(r6, r6), r2)), e.c2 * 8.0), r2));
  }
  atomicAdd(&e.sums[3 * r + 0], ke);
  atomicAdd(&e.sums[3 * r + 1], 0.5 * pe);
  atomicAdd(&e.sums[3 * r + 2], 0.5 * vir);
}

// Ordered pairs with r^2 <= rc^2 over the current lists (the FP64 pair
// test of the force and observer kernels), summed over all replicas.
__global__ void __launch_bounds__(kEB) ke_count_pairs(Ens e, unsigned long long *count) {
  const int i = blockIdx.x * kEB + threadIdx.x;
  int c = 0;
  if (i < e.ntot) {
    const Rep &rep = e.rep[e.rep_of[i]];
    const double4 qi = e.q[i];
    const int nn = e.nnbr[i];
    for (int k = 0; k < nn; k++) {
      const double4 qj = e.q[e.nbr[(size_t)k * e.stride + i]];
      const double dx = dsub(image_of(qj.x, qi.x, rep.L[0], rep.hL[0]), qi.x);
      const double dy = dsub(image_of(qj.y, qi.y, rep.L[1], rep.hL[1]), qi.y);
      const double dz = dsub(image_of(qj.z, qi.z, rep.L[2], rep.hL[2]), qi.z);
      const double r2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
      c += r2 <= e.rc2;
    }
  }
  const int w = __reduce_add_sync(0xffffffffu, c);
  if ((threadIdx.x & 31) == 0 && w) atomicAdd(count, (unsigned long long)w);
}

__global__ void __launch_bounds__(kEB) ke_vmax_init(Ens e) {
  const int i = blockIdx.x * kEB + threadIdx.x;
  int r = 0;
  double v2 = 0.0;
  const bool active = i < e.ntot;
  if (active) {
    r = e.rep_of[i];
    const double4 v = e.v[i], q = e.q[i];
    v2 = dadd(dadd(dmul(v.x, v.x), dmul(v.y, v.y)), dmul(v.z, v.z));
    if (!isfinite(v2) || !isfinite(q.x) || !isfinite(q.y) || !isfinite(q.z)) {
      atomicOr(e.error, kErrNonFinite);
      v2 = 0.0;
    }
  }
  rep_max(&e.rs[0].vmax2_bits, sizeof(RepStatus), r, v2, active);
}

int nb(int n, int b) { return n > 0 ? (n + b - 1) / b : 1; }

}  // namespace
}  // namespace mdg

using namespace mdg;

struct mdg_ensemble {
  mdg_params prm{};
  Ens e{};
  std::vector<Rep> reps;
  int ncell_tot = 0;
  int *d_flags = nullptr;
  unsigned long long *d_count = nullptr;  // ke_count_pairs
  int *d_lists = nullptr;                 // storage of the two work lists
  int work_blocks = 0;                    // grid of the work-list sweeps
  cudaStream_t stream = nullptr, cap_stream = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool graph_dirty = true;
  bool use_graphs = true;
  bool state_set = false;
  int64_t kernel_launches = 0;
  int graph_kernels = 0;
  // force-kernel timers (mdg_ensemble_set_kernel_timing)
  bool timing = false;
  std::vector<cudaEvent_t> ev;  // 2 per captured step
  double force_ms = 0.0;
  int64_t force_launches = 0;
  // lanes per atom of the FP32 force pass: chosen (1, 2, 4) or 0 while the
  // first steps time each candidate (tune_lanes is the one the next eager
  // step uses); the forces are bit-identical for every choice
  int tpa = 0;
  int tune_lanes = 1;
  float tune_ms[3] = {0.f, 0.f, 0.f};
};

namespace {

#define ECUDA(expr)                      \
  do {                                   \
    if ((expr) != cudaSuccess) return MDG_ERR_CUDA; \
  } while (0)

template <typename T>
cudaError_t edalloc(T **p, size_t count) {
  return cudaMalloc((void **)p, std::max<size_t>(count, 1) * sizeof(T));
}

void e_free(mdg_ensemble *x) {
  Ens &e = x->e;
  void *ptrs[] = {(void *)e.rep, e.rs, (void *)e.rep_of, e.q, e.v, e.q_old, e.qfix, e.qloc, e.cxyz, e.xsub, e.ids, e.cell,
                  e.cell_tmp, e.nbr, e.nnbr, e.cell_count, e.cell_start, e.slot, e.perm, e.perm2, e.q_tmp,
                  e.v_tmp, e.ids_tmp, e.mult, e.cand, e.disp2, e.error, e.sums, x->d_flags, x->d_count,
                  x->d_lists};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (x->exec) cudaGraphExecDestroy(x->exec);
  x->exec = nullptr;
}

// Kernels launched by one skin-check and one rebuild branch.
constexpr int kEDispKernels = 4, kEBuildKernels = 10;

// The per-atom and per-cell kernels of the branches sweep the work list with
// a grid of at most x->work_blocks blocks (full occupancy of every SM).
void e_launch_disp(mdg_ensemble *x, cudaStream_t s) {
  Ens &e = x->e;
  const int gb = std::min(nb(e.ntot, kEB), x->work_blocks);
  ke_make_list<0><<<1, 1024, 0, s>>>(e);
  ke_disp_max<<<gb, kEB, 0, s>>>(e);
  ke_disp_collect<<<gb, kEB, 0, s>>>(e);
  ke_disp_pairs<<<dim3(e.nrep, kEPairParts), 256, 0, s>>>(e);
}

void e_launch_build(mdg_ensemble *x, cudaStream_t s) {
  Ens &e = x->e;
  const int gb = std::min(nb(e.ntot, kEB), x->work_blocks);
  const int gf = std::min(nb(e.ntot, kEF), 2 * x->work_blocks);
  const int gc = std::min(nb(x->ncell_tot * 32, kEB), x->work_blocks);
  ke_make_list<1><<<1, 1024, 0, s>>>(e);
  ke_clear_cells<<<e.nrep, kEB, 0, s>>>(e);
  ke_cell_assign<<<gb, kEB, 0, s>>>(e);
  ke_scan_cells<<<e.nrep, kEB, 0, s>>>(e);
  ke_scatter<<<gb, kEB, 0, s>>>(e);
  ke_sort_cells<<<gc, kEB, 0, s>>>(e);
  ke_permute<<<gb, kEB, 0, s>>>(e);
  ke_copy_back<<<gb, kEB, 0, s>>>(e);
  ke_build<<<gf, kEF, 0, s>>>(e);
  ke_build_done<<<1, 1024, 0, s>>>(e);
}

// The step after the skin decision; e0/e1 (optional) bracket the force
// kernel.  Inside a stream capture an event record must be external to be
// recorded when the graph runs (a plain record only orders the capture).
int e_launch_tail(mdg_ensemble *x, cudaStream_t s, cudaEvent_t e0 = nullptr, cudaEvent_t e1 = nullptr,
                  bool capture = false) {
  Ens &e = x->e;
  auto rec = [&](cudaEvent_t ev) {
    if (!ev) return;
    if (capture) cudaEventRecordWithFlags(ev, s, cudaEventRecordExternal);
    else cudaEventRecord(ev, s);
  };
  if (x->prm.precision == MDG_FP32_MIXED) {
    ke_drift<true><<<nb(e.ntot, kEB), kEB, 0, s>>>(e, 0);
    rec(e0);
    const int lanes = x->tpa > 0 ? x->tpa : x->tune_lanes;
    const int blocks = (int)(((long long)e.ntot * lanes + kEF - 1) / kEF);
    if (lanes == 4) ke_force_fp32<4><<<blocks, kEF, 0, s>>>(e);
    else if (lanes == 2) ke_force_fp32<2><<<blocks, kEF, 0, s>>>(e);
    else ke_force_fp32<1><<<blocks, kEF, 0, s>>>(e);
    rec(e1);
    ke_step_done<<<1, 1024, 0, s>>>(e);
    return 3;
  }
  ke_drift<false><<<nb(e.ntot, kEB), kEB, 0, s>>>(e, 0);
  rec(e0);
  ke_force_fp64<<<nb(e.ntot, kEF), kEF, 0, s>>>(e);
  rec(e1);
  ke_drift<false><<<nb(e.ntot, kEB), kEB, 0, s>>>(e, 1);
  ke_step_done<<<1, 1024, 0, s>>>(e);
  return 4;
}

void e_destroy_events(mdg_ensemble *x) {
  for (cudaEvent_t ev : x->ev) cudaEventDestroy(ev);
  x->ev.clear();
}

struct ECapture {
  cudaStream_t s;
  cudaGraph_t g;
  std::vector<cudaGraphNode_t> deps;
};

cudaError_t e_begin(ECapture &c) {
  return cudaStreamBeginCaptureToGraph(c.s, c.g, c.deps.empty() ? nullptr : c.deps.data(), nullptr, c.deps.size(),
                                       cudaStreamCaptureModeThreadLocal);
}

cudaError_t e_end(ECapture &c) {
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t *d = nullptr;
  size_t nd = 0;
  cudaError_t err = cudaStreamGetCaptureInfo(c.s, &cs, nullptr, nullptr, &d, &nd);
  if (err != cudaSuccess) return err;
  std::vector<cudaGraphNode_t> f(d, d + nd);
  cudaGraph_t out = nullptr;
  err = cudaStreamEndCapture(c.s, &out);
  if (err != cudaSuccess) return err;
  if (!f.empty()) c.deps = f;
  return cudaSuccess;
}

cudaError_t e_add_if(ECapture &c, cudaGraphConditionalHandle hc, cudaGraph_t *body) {
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = hc;
  p.conditional.type = cudaGraphCondTypeIf;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  cudaError_t err = cudaGraphAddNode(&node, c.g, c.deps.empty() ? nullptr : c.deps.data(), c.deps.size(), &p);
  if (err != cudaSuccess) return err;
  *body = p.conditional.phGraph_out[0];
  c.deps.assign(1, node);
  return cudaSuccess;
}

mdg_status e_build_graph(mdg_ensemble *x) {
  if (x->exec) cudaGraphExecDestroy(x->exec);
  x->exec = nullptr;
  e_destroy_events(x);
  if (x->timing) {
    x->ev.resize(2 * kEStepsPerGraph);
    for (auto &ev : x->ev) ECUDA(cudaEventCreate(&ev));
  }
  cudaGraph_t g;
  ECUDA(cudaGraphCreate(&g, 0));
  ECapture c{x->cap_stream, g, {}};
  int kernels = 0;
  for (int s = 0; s < kEStepsPerGraph; s++) {
    cudaGraphConditionalHandle hd, hb;
    ECUDA(cudaGraphConditionalHandleCreate(&hd, g, 0, cudaGraphCondAssignDefault));
    ECUDA(cudaGraphConditionalHandleCreate(&hb, g, 0, cudaGraphCondAssignDefault));
    ECUDA(e_begin(c));
    ke_expiry<<<1, 1024, 0, c.s>>>(x->e, hd, 1, x->d_flags);
    ECUDA(e_end(c));
    cudaGraph_t body;
    ECUDA(e_add_if(c, hd, &body));
    {
      ECapture bc{x->cap_stream, body, {}};
      ECUDA(e_begin(bc));
      e_launch_disp(x, bc.s);
      ECUDA(e_end(bc));
    }
    ECUDA(e_begin(c));
    ke_decide<<<1, 1024, 0, c.s>>>(x->e, hb, 1, x->d_flags);
    ECUDA(e_end(c));
    ECUDA(e_add_if(c, hb, &body));
    {
      ECapture bc{x->cap_stream, body, {}};
      ECUDA(e_begin(bc));
      e_launch_build(x, bc.s);
      ECUDA(e_end(bc));
    }
    ECUDA(e_begin(c));
    kernels += 2 + e_launch_tail(x, c.s, x->timing ? x->ev[2 * s] : nullptr,
                                 x->timing ? x->ev[2 * s + 1] : nullptr, true);
    ECUDA(e_end(c));
  }
  cudaError_t err = cudaGraphInstantiate(&x->exec, g, 0);
  cudaGraphDestroy(g);
  if (err != cudaSuccess) return MDG_ERR_CUDA;
  x->graph_kernels = kernels;
  x->graph_dirty = false;
  return MDG_OK;
}

mdg_status e_step_eager(mdg_ensemble *x, float *force_ms_out = nullptr) {
  int flags[2] = {0, 0};
  ke_expiry<<<1, 1024, 0, x->stream>>>(x->e, 0, 0, x->d_flags);
  ECUDA(cudaMemcpyAsync(flags, x->d_flags, sizeof flags, cudaMemcpyDeviceToHost, x->stream));
  ECUDA(cudaStreamSynchronize(x->stream));
  x->kernel_launches++;
  if (flags[0]) e_launch_disp(x, x->stream);  // counted on the device (ke_expiry)
  ke_decide<<<1, 1024, 0, x->stream>>>(x->e, 0, 0, x->d_flags);
  ECUDA(cudaMemcpyAsync(flags, x->d_flags, sizeof flags, cudaMemcpyDeviceToHost, x->stream));
  ECUDA(cudaStreamSynchronize(x->stream));
  x->kernel_launches++;
  if (flags[1]) e_launch_build(x, x->stream);  // counted on the device (ke_decide)
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const bool timed = x->timing || force_ms_out;
  if (timed) {
    ECUDA(cudaEventCreate(&e0));
    ECUDA(cudaEventCreate(&e1));
  }
  x->kernel_launches += e_launch_tail(x, x->stream, e0, e1);
  ECUDA(cudaGetLastError());
  if (timed) {
    float ms = 0.f;
    cudaError_t err = cudaEventSynchronize(e1);
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ECUDA(err);
    if (x->timing) {
      x->force_ms += ms;
      x->force_launches++;
    }
    if (force_ms_out) *force_ms_out = ms;
  }
  return MDG_OK;
}

mdg_status e_status(mdg_ensemble *x, int *error, std::vector<RepStatus> *rs) {
  ECUDA(cudaMemcpyAsync(error, x->e.error, sizeof(int), cudaMemcpyDeviceToHost, x->stream));
  if (rs) {
    rs->resize(x->e.nrep);
    ECUDA(cudaMemcpyAsync(rs->data(), x->e.rs, sizeof(RepStatus) * x->e.nrep, cudaMemcpyDeviceToHost, x->stream));
  }
  ECUDA(cudaStreamSynchronize(x->stream));
  return MDG_OK;
}

mdg_status e_translate(int err) {
  if (err & kErrTooFast) return MDG_ERR_TOO_FAST;
  if (err & kErrNonFinite) return MDG_ERR_NONFINITE;
  if (err & kErrInvalidPosition) return MDG_ERR_INVALID_POSITION;
  if (err & kErrCapacity) return MDG_ERR_CAPACITY;
  return err ? MDG_ERR_CUDA : MDG_OK;
}

mdg_status e_alloc_neighbors(mdg_ensemble *x, int maxnb) {
  maxnb = std::max(8, (maxnb + 7) / 8 * 8);
  if (x->e.nbr && maxnb <= x->e.maxnb) return MDG_OK;
  ECUDA(cudaStreamSynchronize(x->stream));
  if (x->e.nbr) cudaFree(x->e.nbr);
  x->e.nbr = nullptr;
  ECUDA(edalloc(&x->e.nbr, (size_t)maxnb * x->e.stride));
  x->e.maxnb = maxnb;
  if (x->exec) cudaGraphExecDestroy(x->exec);
  x->exec = nullptr;
  x->graph_dirty = true;
  return MDG_OK;
}

// Marks every replica stale and clears the device error.
mdg_status e_mark_all_stale(mdg_ensemble *x) {
  std::vector<RepStatus> rs;
  int err = 0;
  mdg_status r = e_status(x, &err, &rs);
  if (r) return r;
  for (auto &s : rs) {
    s.list_stale = 1;
    s.build = 0;
    s.want_build = 0;
    s.disp = 0;
  }
  const int zero = 0;
  ECUDA(cudaMemcpyAsync(x->e.rs, rs.data(), sizeof(RepStatus) * rs.size(), cudaMemcpyHostToDevice, x->stream));
  ECUDA(cudaMemcpyAsync(x->e.error, &zero, sizeof(int), cudaMemcpyHostToDevice, x->stream));
  ECUDA(cudaStreamSynchronize(x->stream));
  return MDG_OK;
}

}  // namespace

extern "C" {

mdg_status mdg_ensemble_create(const mdg_params *prm, int nrep, const mdg_replica *replicas, mdg_ensemble **out) {
  if (!prm || !replicas || !out || nrep < 1 || prm->cutoff <= 0.0 || prm->time_step <= 0.0 ||
      prm->buffer_length < 0.0 || prm->check_list_length < 1 ||
      (prm->precision != MDG_FP64 && prm->precision != MDG_FP32_MIXED))
    return MDG_ERR_INVALID_ARGUMENT;
  if (prm->thermostat != MDG_NVE) return MDG_ERR_INVALID_ARGUMENT;  // ensembles run NVE
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MDG_ERR_NO_DEVICE;
  if (prm->device < 0 || prm->device >= ndev) return MDG_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(prm->device) != cudaSuccess) return MDG_ERR_CUDA;
  mdg_ensemble *x = new mdg_ensemble();
  x->prm = *prm;
  if (prm->threads_per_atom != 0 && prm->threads_per_atom != 1 && prm->threads_per_atom != 2 &&
      prm->threads_per_atom != 4) {
    delete x;
    return MDG_ERR_INVALID_ARGUMENT;
  }
  x->tpa = prm->threads_per_atom;
  x->reps.resize(nrep);
  long long atoms = 0, tab_entries = 0;
  int cells = 0;
  for (int r = 0; r < nrep; r++) {
    Rep &rp = x->reps[r];
    memset(&rp, 0, sizeof rp);
    if (replicas[r].n < 0 || !(replicas[r].buffer_length >= 0.0) || !std::isfinite(replicas[r].buffer_length)) {
      delete x;
      return MDG_ERR_INVALID_ARGUMENT;
    }
    rp.buffer_length = replicas[r].buffer_length > 0.0 ? replicas[r].buffer_length : prm->buffer_length;
    const double SL = prm->cutoff + rp.buffer_length;
    rp.sl = SL;
    rp.sl2 = SL * SL;
    prefilter_band(rp.sl2, SL, replicas[r].L[0], &rp.sl2_lo, &rp.sl2_hi);
    int small = 0;
    for (int d = 0; d < 3; d++) {
      const double L = replicas[r].L[d];
      if (!(L > 2.0 * SL) || !std::isfinite(L)) {
        delete x;
        return MDG_ERR_BOX_TOO_SMALL;
      }
      rp.L[d] = L;
      rp.hL[d] = 0.5 * L;
      rp.ms[d] = (int)(L / SL);
      if (rp.ms[d] < 3) small = 1;
      rp.fix_scale[d] = (float)(L / 4294967296.0);
    }
    if (small)
      for (int d = 0; d < 3; d++) rp.ms[d] = 1;
    for (int d = 0; d < 3; d++) {
      rp.inv_cs[d] = (double)rp.ms[d] / rp.L[d];
      rp.cs[d] = rp.L[d] / (double)rp.ms[d];
    }
    rp.small = small;
    if (rp.ms[0] >= 2048 || rp.ms[1] >= 2048 || rp.ms[2] >= 1024) {  // packed cell coordinates (pack_cell)
      delete x;
      return MDG_ERR_INVALID_ARGUMENT;
    }
    rp.ncell = rp.ms[0] * rp.ms[1] * rp.ms[2];
    rp.cell_off = cells;
    rp.tab_off = tab_entries;
    tab_entries += (long long)rp.ms[1] * rp.ms[2] * (rp.ms[0] * kXSub + 1);
    rp.atom_off = (int)atoms;
    rp.n = replicas[r].n;
    cells += rp.ncell;
    atoms += replicas[r].n;
  }
  if (atoms > (1LL << 30)) {
    delete x;
    return MDG_ERR_CAPACITY;
  }
  Ens &e = x->e;
  e.nrep = nrep;
  e.ntot = (int)atoms;
  e.cll = prm->check_list_length;
  e.stride = (e.ntot + 31) / 32 * 32;
  e.rc2 = prm->cutoff * prm->cutoff;
  {
    const double s2 = 1.0 / (prm->cutoff * prm->cutoff);
    const double s6 = s2 * s2 * s2, s8 = s6 * s2, s12 = s6 * s6, s14 = s12 * s2;
    e.c2 = 6.0 * s14 - 3.0 * s8;
    e.c0 = -s12 + s6 - e.c2 / s2;
  }
  e.dt = prm->time_step;
  e.lag = 0.5 * prm->time_step;  // NVE: ghosts refreshed before the last half drift
  e.rc2f = (float)e.rc2;
  e.c2x8f = (float)(e.c2 * 8.0);
  x->ncell_tot = cells;
  const size_t n = (size_t)std::max<long long>(atoms, 1);
  cudaError_t err = cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking);
  if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&x->cap_stream, cudaStreamNonBlocking);
  Rep *drep = nullptr;
  int *drep_of = nullptr;
  if (err == cudaSuccess) err = edalloc(&drep, nrep);
  if (err == cudaSuccess) err = edalloc(&e.rs, nrep);
  if (err == cudaSuccess) err = edalloc(&drep_of, n);
  e.rep = drep;
  e.rep_of = drep_of;
  if (err == cudaSuccess) err = edalloc(&e.q, n);
  if (err == cudaSuccess) err = edalloc(&e.v, n);
  if (err == cudaSuccess) err = edalloc(&e.q_old, n);
  if (err == cudaSuccess) err = edalloc(&e.qfix, n);
  if (err == cudaSuccess) err = edalloc(&e.qloc, n);
  if (err == cudaSuccess) err = edalloc(&e.cxyz, n);
  if (err == cudaSuccess) err = edalloc(&e.xsub, (size_t)tab_entries);
  if (err == cudaSuccess) err = edalloc(&e.ids, n);
  if (err == cudaSuccess) err = edalloc(&e.cell, n);
  if (err == cudaSuccess) err = edalloc(&e.cell_tmp, n);
  if (err == cudaSuccess) err = edalloc(&e.nnbr, n);
  if (err == cudaSuccess) err = edalloc(&e.cell_count, cells);
  if (err == cudaSuccess) err = edalloc(&e.cell_start, cells + 1);
  if (err == cudaSuccess) err = edalloc(&e.slot, n);
  if (err == cudaSuccess) err = edalloc(&e.perm, n);
  if (err == cudaSuccess) err = edalloc(&e.perm2, n);
  if (err == cudaSuccess) err = edalloc(&e.q_tmp, n);
  if (err == cudaSuccess) err = edalloc(&e.v_tmp, n);
  if (err == cudaSuccess) err = edalloc(&e.ids_tmp, n);
  if (err == cudaSuccess) err = edalloc(&e.mult, n);
  if (err == cudaSuccess) err = edalloc(&e.cand, (size_t)nrep * e.cll);
  if (err == cudaSuccess) err = edalloc(&e.disp2, n);
  if (err == cudaSuccess) err = edalloc(&e.error, 1);
  if (err == cudaSuccess) err = edalloc(&e.sums, (size_t)3 * nrep);
  if (err == cudaSuccess) err = edalloc(&x->d_flags, 4);
  if (err == cudaSuccess) err = cudaMemsetAsync(x->d_flags, 0, 4 * sizeof(int), x->stream);
  if (err == cudaSuccess) err = edalloc(&x->d_count, 1);
  if (err == cudaSuccess) err = edalloc(&x->d_lists, 2 * (3 * (size_t)nrep + 5));
  if (err == cudaSuccess) {
    // each list: rep[nrep], atom_prefix[nrep + 1], cell_prefix[nrep + 1], count[3]
    WorkList *w[2] = {&e.wd, &e.wb};
    int *p = x->d_lists;
    for (WorkList *l : w) {
      l->rep = p;
      l->atom_prefix = p + nrep;
      l->cell_prefix = p + 2 * nrep + 1;
      l->count = p + 3 * nrep + 2;
      p += 3 * nrep + 5;
    }
    err = cudaMemsetAsync(x->d_lists, 0, sizeof(int) * 2 * (3 * (size_t)nrep + 5), x->stream);
  }
  if (err == cudaSuccess) {
    int nsm = 0;
    err = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, prm->device);
    x->work_blocks = std::max(1, nsm) * 8;
  }
  if (err == cudaSuccess) {
    std::vector<int> rep_of(n, 0);
    for (int r = 0; r < nrep; r++)
      for (int k = 0; k < x->reps[r].n; k++) rep_of[x->reps[r].atom_off + k] = r;
    err = cudaMemcpy(drep, x->reps.data(), sizeof(Rep) * nrep, cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemcpy(drep_of, rep_of.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    // the slot after every replica's last cell is the next replica's first atom
    std::vector<int> starts(cells + 1, 0);
    for (int r = 0; r < nrep; r++) starts[x->reps[r].cell_off] = x->reps[r].atom_off;
    starts[cells] = e.ntot;
    if (err == cudaSuccess) err = cudaMemcpy(e.cell_start, starts.data(), sizeof(int) * (cells + 1), cudaMemcpyHostToDevice);
    if (err == cudaSuccess) err = cudaMemset(e.rs, 0, sizeof(RepStatus) * nrep);
    if (err == cudaSuccess) err = cudaMemset(e.error, 0, sizeof(int));
  }
  if (err != cudaSuccess) {
    e_free(x);
    delete x;
    return MDG_ERR_CUDA;
  }
  *out = x;
  return MDG_OK;
}

mdg_status mdg_ensemble_destroy(mdg_ensemble *x) {
  if (!x) return MDG_ERR_INVALID_ARGUMENT;
  cudaSetDevice(x->prm.device);
  cudaStreamSynchronize(x->stream);
  e_free(x);
  e_destroy_events(x);
  if (x->cap_stream) cudaStreamDestroy(x->cap_stream);
  if (x->stream) cudaStreamDestroy(x->stream);
  delete x;
  return MDG_OK;
}

mdg_status mdg_ensemble_set_state(mdg_ensemble *x, const double *q4, const double *v4) {
  if (!x || !q4 || !v4) return MDG_ERR_INVALID_ARGUMENT;
  Ens &e = x->e;
  ECUDA(cudaSetDevice(x->prm.device));
  ECUDA(cudaStreamSynchronize(x->stream));
  const int n = e.ntot;
  ECUDA(cudaMemcpyAsync(e.q, q4, sizeof(double4) * n, cudaMemcpyHostToDevice, x->stream));
  ECUDA(cudaMemcpyAsync(e.v, v4, sizeof(double4) * n, cudaMemcpyHostToDevice, x->stream));
  std::vector<int> ids(n);
  int maxnb = 8;
  for (int r = 0; r < e.nrep; r++) {
    const Rep &rp = x->reps[r];
    for (int k = 0; k < rp.n; k++) ids[rp.atom_off + k] = k;  // upload index within the replica
    // neighbour-row capacity from the replica's density
    const double vol = rp.L[0] * rp.L[1] * rp.L[2];
    const double sphere = 4.0 / 3.0 * M_PI * rp.sl * rp.sl * rp.sl;
    maxnb = std::max(maxnb, std::min(rp.n, (int)std::ceil(1.6 * (rp.n / vol) * sphere + 32.0)));
  }
  ECUDA(cudaMemcpyAsync(e.ids, ids.data(), sizeof(int) * n, cudaMemcpyHostToDevice, x->stream));
  mdg_status r = e_alloc_neighbors(x, maxnb);
  if (r) return r;
  std::vector<RepStatus> rs(e.nrep);
  ECUDA(cudaMemcpyAsync(rs.data(), e.rs, sizeof(RepStatus) * e.nrep, cudaMemcpyDeviceToHost, x->stream));
  ECUDA(cudaStreamSynchronize(x->stream));
  for (int k = 0; k < e.nrep; k++) {
    RepStatus &s = rs[k];
    s.list_stale = 1;
    s.vmax2_bits = 0;
    s.budget = x->reps[k].buffer_length;
    s.build = s.want_build = s.disp = 0;
  }
  const int zero = 0;
  ECUDA(cudaMemcpyAsync(e.rs, rs.data(), sizeof(RepStatus) * e.nrep, cudaMemcpyHostToDevice, x->stream));
  ECUDA(cudaMemcpyAsync(e.error, &zero, sizeof(int), cudaMemcpyHostToDevice, x->stream));
  ke_vmax_init<<<nb(n, kEB), kEB, 0, x->stream>>>(e);
  int err = 0;
  ECUDA(cudaMemcpyAsync(&err, e.error, sizeof(int), cudaMemcpyDeviceToHost, x->stream));
  ECUDA(cudaStreamSynchronize(x->stream));
  if (err) {
    ECUDA(cudaMemcpy(e.error, &zero, sizeof(int), cudaMemcpyHostToDevice));
    return MDG_ERR_NONFINITE;
  }
  x->state_set = true;
  return MDG_OK;
}

mdg_status mdg_ensemble_get_state(mdg_ensemble *x, double *q4, double *v4, int *ids) {
  if (!x || !x->state_set) return MDG_ERR_STATE;
  const int n = x->e.ntot;
  if (q4) ECUDA(cudaMemcpyAsync(q4, x->e.q, sizeof(double4) * n, cudaMemcpyDeviceToHost, x->stream));
  if (v4) ECUDA(cudaMemcpyAsync(v4, x->e.v, sizeof(double4) * n, cudaMemcpyDeviceToHost, x->stream));
  if (ids) ECUDA(cudaMemcpyAsync(ids, x->e.ids, sizeof(int) * n, cudaMemcpyDeviceToHost, x->stream));
  ECUDA(cudaStreamSynchronize(x->stream));
  return MDG_OK;
}

mdg_status mdg_ensemble_calculate(mdg_ensemble *x, int nsteps) {
  if (!x || nsteps < 0) return MDG_ERR_INVALID_ARGUMENT;
  if (!x->state_set) return MDG_ERR_STATE;
  if (nsteps == 0 || x->e.ntot == 0) return MDG_OK;
  ECUDA(cudaSetDevice(x->prm.device));
  std::vector<RepStatus> rs;
  int err = 0;
  mdg_status r = e_status(x, &err, &rs);
  if (r) return r;
  if (err) return e_translate(err);
  const long long target = rs[0].steps + nsteps;
  for (int attempt = 0; attempt < 8; attempt++) {
    long long left = target - rs[0].steps;
    if (left <= 0) break;
    // FP32-mixed with the lanes per atom to be chosen: the first steps run
    // one candidate each (1, 2, 4 lanes) with the force pass timed; the
    // steps are the trajectory's own (every choice gives the same forces)
    while (x->prm.precision == MDG_FP32_MIXED && x->tpa == 0 && left > 0) {
      const int k = x->tune_lanes == 1 ? 0 : (x->tune_lanes == 2 ? 1 : 2);
      if ((r = e_step_eager(x, &x->tune_ms[k]))) return r;
      left--;
      if (k < 2) {
        x->tune_lanes *= 2;
      } else {
        int best = 0;
        for (int c = 1; c < 3; c++)
          if (x->tune_ms[c] < x->tune_ms[best]) best = c;
        x->tpa = 1 << best;
        x->graph_dirty = true;
      }
    }
    if (x->use_graphs && left >= kEStepsPerGraph && x->graph_dirty) {
      if ((r = e_build_graph(x))) return r;
    }
    while (x->use_graphs && left >= kEStepsPerGraph) {
      ECUDA(cudaGraphLaunch(x->exec, x->stream));
      x->kernel_launches += x->graph_kernels;
      left -= kEStepsPerGraph;
      if (x->timing) {
        ECUDA(cudaStreamSynchronize(x->stream));
        for (int s = 0; s < kEStepsPerGraph; s++) {
          float ms = 0.f;
          ECUDA(cudaEventElapsedTime(&ms, x->ev[2 * s], x->ev[2 * s + 1]));
          x->force_ms += ms;
          x->force_launches++;
        }
      }
    }
    while (left > 0) {
      if ((r = e_step_eager(x))) return r;
      left--;
    }
    if ((r = e_status(x, &err, &rs))) return r;
    if (err == kErrCapacity) {
      int need = 0;
      for (auto &s : rs) need = std::max(need, s.max_row);
      if ((r = e_alloc_neighbors(x, (int)(need * 1.25) + 8))) return r;
      if ((r = e_mark_all_stale(x))) return r;
      if ((r = e_status(x, &err, &rs))) return r;
      continue;
    }
    if (err) return e_translate(err);
  }
  if (rs[0].steps < target) return MDG_ERR_CAPACITY;
  return MDG_OK;
}

mdg_status mdg_ensemble_observe(mdg_ensemble *x, double *ke, double *pe, double *virial) {
  if (!x || !x->state_set) return MDG_ERR_STATE;
  Ens &e = x->e;
  // a stale list (fresh upload) is built first
  std::vector<RepStatus> rs;
  int err = 0;
  mdg_status r = e_status(x, &err, &rs);
  if (r) return r;
  if (err) return e_translate(err);
  bool stale = false;
  for (auto &s : rs) stale |= s.list_stale != 0;
  if (stale) {
    for (auto &s : rs) s.build = s.list_stale;
    ECUDA(cudaMemcpyAsync(e.rs, rs.data(), sizeof(RepStatus) * e.nrep, cudaMemcpyHostToDevice, x->stream));
    e_launch_build(x, x->stream);
    if ((r = e_status(x, &err, &rs))) return r;
    if (err) return e_translate(err);
  }
  ECUDA(cudaMemsetAsync(e.sums, 0, sizeof(double) * 3 * e.nrep, x->stream));
  ke_observe<<<nb(e.ntot, kEB), kEB, 0, x->stream>>>(e);
  std::vector<double> sums(3 * e.nrep);
  ECUDA(cudaMemcpyAsync(sums.data(), e.sums, sizeof(double) * 3 * e.nrep, cudaMemcpyDeviceToHost, x->stream));
  ECUDA(cudaStreamSynchronize(x->stream));
  for (int k = 0; k < e.nrep; k++) {
    if (ke) ke[k] = sums[3 * k];
    if (pe) pe[k] = sums[3 * k + 1];
    if (virial) virial[k] = sums[3 * k + 2] / 3.0;
  }
  return MDG_OK;
}

mdg_status mdg_ensemble_rebuilds(mdg_ensemble *x, int64_t *rebuilds, int64_t *steps) {
  if (!x) return MDG_ERR_INVALID_ARGUMENT;
  std::vector<RepStatus> rs;
  int err = 0;
  mdg_status r = e_status(x, &err, &rs);
  if (r) return r;
  for (int k = 0; k < x->e.nrep; k++) {
    if (rebuilds) rebuilds[k] = rs[k].rebuilds;
    if (steps) steps[k] = rs[k].steps;
  }
  return MDG_OK;
}

mdg_status mdg_ensemble_set_graph_mode(mdg_ensemble *x, int use_graphs) {
  if (!x) return MDG_ERR_INVALID_ARGUMENT;
  x->use_graphs = use_graphs != 0;
  return MDG_OK;
}

mdg_status mdg_ensemble_set_kernel_timing(mdg_ensemble *x, int on) {
  if (!x) return MDG_ERR_INVALID_ARGUMENT;
  if ((on != 0) != x->timing) {
    ECUDA(cudaStreamSynchronize(x->stream));
    x->timing = on != 0;
    x->graph_dirty = true;
  }
  x->force_ms = 0.0;
  x->force_launches = 0;
  x->kernel_launches = 0;
  ECUDA(cudaMemsetAsync(x->d_flags + 2, 0, 2 * sizeof(int), x->stream));
  ECUDA(cudaStreamSynchronize(x->stream));
  return MDG_OK;
}

mdg_status mdg_ensemble_list_stats(mdg_ensemble *x, int64_t *list_entries, int64_t *pairs_within_cutoff) {
  if (!x || !x->state_set) return MDG_ERR_STATE;
  Ens &e = x->e;
  std::vector<RepStatus> rs;
  int err = 0;
  mdg_status r = e_status(x, &err, &rs);
  if (r) return r;
  if (err) return e_translate(err);
  long long entries = 0;
  for (auto &st : rs) entries += st.list_entries;
  if (list_entries) *list_entries = entries;
  if (pairs_within_cutoff) {
    unsigned long long h = 0;
    ECUDA(cudaMemsetAsync(x->d_count, 0, sizeof(unsigned long long), x->stream));
    ke_count_pairs<<<nb(e.ntot, kEB), kEB, 0, x->stream>>>(e, x->d_count);
    ECUDA(cudaGetLastError());
    ECUDA(cudaMemcpyAsync(&h, x->d_count, sizeof h, cudaMemcpyDeviceToHost, x->stream));
    ECUDA(cudaStreamSynchronize(x->stream));
    *pairs_within_cutoff = (int64_t)(h / 2);
  }
  return MDG_OK;
}

mdg_status mdg_ensemble_kernel_time(mdg_ensemble *x, double *force_ms, int64_t *force_launches,
                                    int64_t *kernel_launches) {
  if (!x) return MDG_ERR_INVALID_ARGUMENT;
  if (force_ms) *force_ms = x->force_ms;
  if (force_launches) *force_launches = x->force_launches;
  if (kernel_launches) {
    // the host counts the unconditional kernels; the branches taken (in
    // graphs or eager steps) are counted on the device
    int branch[2] = {0, 0};
    ECUDA(cudaMemcpyAsync(branch, x->d_flags + 2, sizeof branch, cudaMemcpyDeviceToHost, x->stream));
    ECUDA(cudaStreamSynchronize(x->stream));
    *kernel_launches = x->kernel_launches + (long long)kEDispKernels * branch[0] +
                       (long long)kEBuildKernels * branch[1];
  }
  return MDG_OK;
}

void *mdg_ensemble_stream(mdg_ensemble *x) { return x ? (void *)x->stream : nullptr; }

}  // extern "C"

// ------------------------------------------------------- replica partition
extern "C" mdg_status mdg_partition_replicas(const mdg_replica *replicas, int nrep, double search_length,
                                             int nranks, int *owner, double *load) {
  if (nrep < 0 || nranks < 1 || !(search_length > 0.0) || (nrep > 0 && (!replicas || !owner)))
    return MDG_ERR_INVALID_ARGUMENT;
  std::vector<double> cost(nrep);
  const double sphere = 4.0 / 3.0 * M_PI * search_length * search_length * search_length;
  for (int r = 0; r < nrep; r++) {
    const mdg_replica &x = replicas[r];
    if (x.n < 0 || !(x.L[0] > 0.0) || !(x.L[1] > 0.0) || !(x.L[2] > 0.0)) return MDG_ERR_INVALID_ARGUMENT;
    const double rho = (double)x.n / (x.L[0] * x.L[1] * x.L[2]);
    cost[r] = (double)x.n * (41.0 + sphere * rho);
  }
  std::vector<int> order(nrep);
  for (int r = 0; r < nrep; r++) order[r] = r;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<double> tot(nranks, 0.0);
  for (int r : order) {
    int best = 0;
    for (int k = 1; k < nranks; k++)
      if (tot[k] < tot[best]) best = k;
    owner[r] = best;
    tot[best] += cost[r];
  }
  if (load)
    for (int k = 0; k < nranks; k++) load[k] = tot[k];
  return MDG_OK;
}

