// One periodic system decomposed into z-slabs of whole cell layers, one
// slab per device (several slabs may share a device), driven by one host
// thread: the multi-GPU domain decomposition of the reference
// (MDManager::SendParticles / SendBorderParticles, src/mdmanager.cc:317-489;
// MDUnit::MakeBufferForSendingParticle .. ReceiveBorderParticles,
// src/mdunit.cc:93-208; the expiry all-reduce, src/mdmanager.cc:509-518 and
// src/communicator.cc:24-37) on the B200 data layout.
//
// Each slab owns the global cell layers z0 .. z0 + nzl - 1 of the
// single-domain cell grid (int(L / SL) cells per axis) and stores, after
// every rebuild,
//   slots [0, n_own)                  its own atoms, cell-sorted (z-major), so
//                                     its bottom and top layers are the
//                                     contiguous ranges [0, n_bot) and
//                                     [n_own - n_top, n_own)
//   slots [n_own, n_own + ng_lo)      ghost copies of the top layer of the
//                                     slab below (global layer z0 - 1)
//   slots [.., + ng_hi)               ghost copies of the bottom layer of the
//                                     slab above (global layer z0 + nzl)
// in global box coordinates; the trim table of the list build has one block
// of rows for each own layer and one for each ghost layer.  The 27-cell walk
// of an own atom therefore sees exactly the atoms a single-domain walk sees,
// in the same order, so the lists, the force sums and the trajectory are the
// single domain's bit for bit.
//
// Per step: every slab drifts its own atoms, pushes the positions of its two
// border layers into its neighbours' ghost slots (two contiguous device-to-
// device copies, peer copies across devices), and kicks its own atoms once
// both neighbours' pushes have landed.  The skin bookkeeping is global: the
// |v| maximum and the displacement maximum are maxima over the slabs, the
// candidate copies of the displacement check are gathered from all slabs
// and tested together, and every slab rebuilds at the same step.  A rebuild
// first migrates the atoms that left a slab's layers (at most one layer per
// rebuild: the skin bounds the motion) to the neighbouring slab.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "mdacp_b200.h"
#include "mdg_device.cuh"

using namespace mdg;

namespace {

constexpr int kSB = 256;   // streaming kernels
constexpr int kSF = 128;   // pair kernels
constexpr int kSScan = 1024;

int sblocks(long long n, int b) { return n > 0 ? (int)((n + b - 1) / b) : 1; }

// Where the atoms leaving a slab at a rebuild go: kept (into the slab's
// temporary arrays), or to the slab below / above (send buffers).
struct Outbound {
  double4 *q[2], *v[2];
  int *ids[2], *type[2];
  int *count;  // [kept, below, above]
  int cap;     // atoms a send buffer holds
};

// Rebuild of a slab, first pass: every own atom is wrapped into the box
// (Variables::AdjustPeriodicBoundary, src/variables.cc:63-84, as
// k_cell_assign wraps it) and filed by the global cell layer it is in now.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_slab_sort_out(Arrays a, Box b, int n, Outbound ob) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  if (i >= n || a.st->error) return;
  double4 q = a.q[i];
  double x[3] = {q.x, q.y, q.z};
  for (int d = 0; d < 3; d++) {
    if (!isfinite(x[d])) {
      atomicOr(&a.st->error, kErrNonFinite);
      return;
    }
    if (x[d] < 0.0) x[d] = mdg::dadd(x[d], b.L[d]);
    else if (x[d] > b.L[d]) x[d] = mdg::dsub(x[d], b.L[d]);
    if (x[d] < 0.0 || x[d] > b.L[d]) {
      atomicOr(&a.st->error, kErrInvalidPosition);
      return;
    }
  }
  q.x = x[0]; q.y = x[1]; q.z = x[2];
  const int gz = cell_coord(x[2], b.inv_cs[2], b.ms[2]);
  const int lz = gz - b.z0;
  int where;
  if (lz >= 0 && lz < b.nzl) where = 0;
  else if (gz == (b.z0 - 1 + b.ms[2]) % b.ms[2]) where = 1;
  else if (gz == (b.z0 + b.nzl) % b.ms[2]) where = 2;
  else {  // farther than the neighbouring layer: the skin cannot allow it
    atomicOr(&a.st->error, kErrInvalidPosition);
    return;
  }
  const int k = atomicAdd(&ob.count[where], 1);
  if (where == 0) {
    a.q_tmp[k] = q;
    a.v_tmp[k] = a.v[i];
    a.ids_tmp[k] = a.ids[i];
    a.type_tmp[k] = a.type[i];
  } else if (k < ob.cap) {
    ob.q[where - 1][k] = q;
    ob.v[where - 1][k] = a.v[i];
    ob.ids[where - 1][k] = a.ids[i];
    ob.type[where - 1][k] = a.type[i];
  } else {
    atomicOr(&a.st->error, kErrCapacity);
  }
}

// Adds delta to n trim-table entries (ghost rows copied from their owner,
// whose slot numbers differ by delta).
__global__ void k_slab_shift(int *tab, int n, int delta) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) tab[k] += delta;
}

// Old and current positions of the slab's displacement-check candidates
// (PairList::CheckByDisplacement's copies, see for_each_copy), 6 rows of
// stride doubles: old x, y, z, current x, y, z.
__global__ void k_slab_cand_positions(Arrays a, Box b, int count, double lag, double *out, int stride) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= count) return;
  const int2 c = a.cand[k];
  double o[3], p[3];
  copy_positions(copy_view(a), b.L, c.x, c.y, lag, o, p);
  for (int d = 0; d < 3; d++) {
    out[d * stride + k] = o[d];
    out[(3 + d) * stride + k] = p[d];
  }
}

// The pair test of PairList::CheckByDisplacement (src/pairlist.cc:99-121)
// over the candidate copies of all slabs (positions as k_slab_cand_positions
// writes them): *found = 1 if a pair that was at least SearchLength apart at
// the last build is now within the cut-off.  Rows a = blockIdx.x,
// blockIdx.x + gridDim.x, ...; an "any", so the split changes only the time.
__global__ void __launch_bounds__(256) k_slab_pairs(const double *pos, int stride, int l, double sl2, double rc2,
                                                    int *found) {
  for (int a = blockIdx.x; a < l - 1; a += gridDim.x) {
    const double o1[3] = {pos[a], pos[stride + a], pos[2 * stride + a]};
    const double n1[3] = {pos[3 * stride + a], pos[4 * stride + a], pos[5 * stride + a]};
    for (int c = a + 1 + threadIdx.x; c < l; c += blockDim.x) {
      const double o2[3] = {pos[c], pos[stride + c], pos[2 * stride + c]};
      if (dist2(o1, o2) < sl2) continue;
      const double n2[3] = {pos[3 * stride + c], pos[4 * stride + c], pos[5 * stride + c]};
      if (dist2(n1, n2) < rc2) atomicOr(found, 1);
    }
  }
}

struct Slab {
  int dev = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t pushed = nullptr;  // this slab's border positions are in its neighbours' ghost slots
  Box box{};
  Arrays a{};
  int cap = 0;                   // slots (own + ghost)
  int n_own = 0, ng_lo = 0, ng_hi = 0, n_bot = 0, n_top = 0;
  int ncell = 0;                 // own cells
  int *d_tiles = nullptr;
  int *d_flags = nullptr;
  double *d_sums = nullptr;
  double *d_cand = nullptr;      // 6 x cll candidate positions
  int *d_found = nullptr;
  Outbound ob{};
  double4 *sq[2] = {nullptr, nullptr}, *sv[2] = {nullptr, nullptr};
  int *sid[2] = {nullptr, nullptr}, *stype[2] = {nullptr, nullptr};
  int *d_count = nullptr;
};

}  // namespace

struct mdg_slabs {
  mdg_params prm{};
  Box gbox{};                    // the global box (single-domain geometry)
  std::vector<Slab> s;
  int n = 0;                     // atoms in total
  bool state_set = false;
  long long steps = 0, rebuilds = 0, disp_checks = 0;
  int tpa = 1;
  std::string err;
};

namespace {

mdg_status sfail(mdg_slabs *x, mdg_status st, const std::string &msg) {
  if (x) x->err = msg;
  return st;
}

#define SCUDA(x, expr)                                                                         \
  do {                                                                                         \
    cudaError_t e_ = (expr);                                                                   \
    if (e_ != cudaSuccess) return sfail((x), MDG_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
cudaError_t salloc(T **p, size_t count) {
  return cudaMalloc((void **)p, std::max<size_t>(count, 1) * sizeof(T));
}

int below(const mdg_slabs *x, int k) { return (k - 1 + (int)x->s.size()) % (int)x->s.size(); }
int above(const mdg_slabs *x, int k) { return (k + 1) % (int)x->s.size(); }

mdg_status slab_status(mdg_slabs *x, int k, Status *st) {
  Slab &sl = x->s[k];
  SCUDA(x, cudaSetDevice(sl.dev));
  SCUDA(x, cudaMemcpyAsync(st, sl.a.st, sizeof(Status), cudaMemcpyDeviceToHost, sl.stream));
  SCUDA(x, cudaStreamSynchronize(sl.stream));
  return MDG_OK;
}

mdg_status device_error(mdg_slabs *x, int error) {
  if (error & kErrTooFast) return sfail(x, MDG_ERR_TOO_FAST, "Too fast particles exists. Try smaller time step");
  if (error & kErrNonFinite) return sfail(x, MDG_ERR_NONFINITE, "non-finite position or velocity");
  if (error & kErrInvalidPosition) return sfail(x, MDG_ERR_INVALID_POSITION, "Invalid position");
  if (error & kErrCapacity) return sfail(x, MDG_ERR_CAPACITY, "slab or neighbour capacity exceeded");
  return sfail(x, MDG_ERR_STATE, "device error");
}

mdg_status sync_all(mdg_slabs *x) {
  for (Slab &sl : x->s) {
    SCUDA(x, cudaSetDevice(sl.dev));
    SCUDA(x, cudaStreamSynchronize(sl.stream));
  }
  return MDG_OK;
}

// Copies `count` elements of `bytes_each` from slab src's array (at src_off)
// into slab dst's (at dst_off), on the source's stream.
cudaError_t copy_between(const Slab &dst, void *dbase, size_t dst_off, const Slab &src, const void *sbase,
                         size_t src_off, size_t count, size_t bytes_each) {
  if (count == 0) return cudaSuccess;
  return cudaMemcpyPeerAsync((char *)dbase + dst_off * bytes_each, dst.dev, (const char *)sbase + src_off * bytes_each,
                             src.dev, count * bytes_each, src.stream);
}

// Every slab pushes the chosen per-atom array of its border layers into its
// neighbours' ghost slots; `arr` picks the array of a slab and its element
// size.  Each slab's stream then waits until both neighbours have pushed.
template <typename Pick>
mdg_status push_borders(mdg_slabs *x, Pick arr) {
  const int P = (int)x->s.size();
  for (int k = 0; k < P; k++) {
    Slab &sl = x->s[k];
    SCUDA(x, cudaSetDevice(sl.dev));
    const Slab &lo = x->s[below(x, k)], &hi = x->s[above(x, k)];
    size_t es = 0;
    void *src = arr(sl, &es);
    // own top layer -> ghost-low slots of the slab above; own bottom layer ->
    // ghost-high slots of the slab below
    SCUDA(x, copy_between(hi, arr(const_cast<Slab &>(hi), &es), (size_t)hi.n_own, sl, src,
                          (size_t)(sl.n_own - sl.n_top), (size_t)sl.n_top, es));
    SCUDA(x, copy_between(lo, arr(const_cast<Slab &>(lo), &es), (size_t)(lo.n_own + lo.ng_lo), sl, src, 0,
                          (size_t)sl.n_bot, es));
    SCUDA(x, cudaEventRecord(sl.pushed, sl.stream));
  }
  for (int k = 0; k < P; k++) {
    Slab &sl = x->s[k];
    SCUDA(x, cudaSetDevice(sl.dev));
    SCUDA(x, cudaStreamWaitEvent(sl.stream, x->s[below(x, k)].pushed, 0));
    SCUDA(x, cudaStreamWaitEvent(sl.stream, x->s[above(x, k)].pushed, 0));
  }
  return MDG_OK;
}

void *pick_q(Slab &sl, size_t *es) { *es = sizeof(double4); return sl.a.q; }
void *pick_v(Slab &sl, size_t *es) { *es = sizeof(double4); return sl.a.v; }
void *pick_qfix(Slab &sl, size_t *es) { *es = sizeof(int4); return sl.a.qfix; }
void *pick_qloc(Slab &sl, size_t *es) { *es = sizeof(float4); return sl.a.qloc; }
void *pick_mult(Slab &sl, size_t *es) { *es = 1; return sl.a.mult; }
void *pick_ids(Slab &sl, size_t *es) { *es = sizeof(int); return sl.a.ids; }

mdg_status grow_rows(mdg_slabs *x, Slab &sl, int maxnb) {
  maxnb = std::max(8, (maxnb + 7) / 8 * 8);
  if (sl.a.nbr && maxnb <= sl.a.maxnb) return MDG_OK;
  SCUDA(x, cudaSetDevice(sl.dev));
  SCUDA(x, cudaStreamSynchronize(sl.stream));
  if (sl.a.nbr) cudaFree(sl.a.nbr);
  sl.a.nbr = nullptr;
  SCUDA(x, salloc(&sl.a.nbr, (size_t)maxnb * sl.a.stride));
  sl.a.maxnb = maxnb;
  return MDG_OK;
}

// The global rebuild (MDManager::MakePairList over all units): migration,
// the cell sort of every slab's own atoms, the ghost layers and their trim
// rows, the lists of the own atoms, a fresh skin budget.
mdg_status rebuild(mdg_slabs *x) {
  const int P = (int)x->s.size();
  // 1. wrap and sort out the atoms by layer
  for (Slab &sl : x->s) {
    SCUDA(x, cudaSetDevice(sl.dev));
    k_build_begin<<<1, 32, 0, sl.stream>>>(sl.a);
    SCUDA(x, cudaMemsetAsync(sl.d_count, 0, 3 * sizeof(int), sl.stream));
    k_slab_sort_out<kSB><<<sblocks(sl.n_own, kSB), kSB, 0, sl.stream>>>(sl.a, sl.box, sl.n_own, sl.ob);
  }
  std::vector<int> cnt(3 * P);
  for (int k = 0; k < P; k++) {
    Slab &sl = x->s[k];
    SCUDA(x, cudaSetDevice(sl.dev));
    SCUDA(x, cudaMemcpyAsync(&cnt[3 * k], sl.d_count, 3 * sizeof(int), cudaMemcpyDeviceToHost, sl.stream));
  }
  SCUDA(x, cudaGetLastError());
  if (mdg_status r = sync_all(x)) return r;
  for (int k = 0; k < P; k++) {
    Status st;
    if (mdg_status r = slab_status(x, k, &st)) return r;
    if (st.error) return device_error(x, st.error);
  }
  // 2. the new own sets: kept atoms, then arrivals from below and above
  std::vector<int> nown(P);
  for (int k = 0; k < P; k++) {
    const int from_lo = cnt[3 * below(x, k) + 2], from_hi = cnt[3 * above(x, k) + 1];
    nown[k] = cnt[3 * k] + from_lo + from_hi;
    if (nown[k] > x->s[k].cap) return sfail(x, MDG_ERR_CAPACITY, "a slab's atoms exceed its capacity");
  }
  for (int k = 0; k < P; k++) {
    Slab &sl = x->s[k];
    SCUDA(x, cudaSetDevice(sl.dev));
    const int kept = cnt[3 * k];
    SCUDA(x, cudaMemcpyAsync(sl.a.q, sl.a.q_tmp, sizeof(double4) * kept, cudaMemcpyDeviceToDevice, sl.stream));
    SCUDA(x, cudaMemcpyAsync(sl.a.v, sl.a.v_tmp, sizeof(double4) * kept, cudaMemcpyDeviceToDevice, sl.stream));
    SCUDA(x, cudaMemcpyAsync(sl.a.ids, sl.a.ids_tmp, sizeof(int) * kept, cudaMemcpyDeviceToDevice, sl.stream));
    SCUDA(x, cudaMemcpyAsync(sl.a.type, sl.a.type_tmp, sizeof(int) * kept, cudaMemcpyDeviceToDevice, sl.stream));
    int at = kept;
    const int srcs[2] = {below(x, k), above(x, k)};
    const int which[2] = {1, 0};  // the slab below sends its "above" buffer, the slab above its "below" one
    for (int t = 0; t < 2; t++) {
      const Slab &o = x->s[srcs[t]];
      const int m = cnt[3 * srcs[t] + 1 + which[t]];
      const int b = which[t];
      SCUDA(x, cudaMemcpyPeerAsync(sl.a.q + at, sl.dev, o.sq[b], o.dev, sizeof(double4) * m, sl.stream));
      SCUDA(x, cudaMemcpyPeerAsync(sl.a.v + at, sl.dev, o.sv[b], o.dev, sizeof(double4) * m, sl.stream));
      SCUDA(x, cudaMemcpyPeerAsync(sl.a.ids + at, sl.dev, o.sid[b], o.dev, sizeof(int) * m, sl.stream));
      SCUDA(x, cudaMemcpyPeerAsync(sl.a.type + at, sl.dev, o.stype[b], o.dev, sizeof(int) * m, sl.stream));
      at += m;
    }
  }
  if (mdg_status r = sync_all(x)) return r;
  // 3. cell sort of the own atoms (the single-domain rebuild kernels on the
  // slab's layers)
  for (int k = 0; k < P; k++) {
    Slab &sl = x->s[k];
    sl.n_own = nown[k];
    SCUDA(x, cudaSetDevice(sl.dev));
    const int n = sl.n_own;
    cudaStream_t s = sl.stream;
    Arrays &a = sl.a;
    SCUDA(x, cudaMemsetAsync(a.cell_count, 0, sizeof(int) * sl.ncell, s));
    k_cell_assign<kSB><<<sblocks(n, kSB), kSB, 0, s>>>(a, sl.box, n);
    const int ntiles = sblocks(sl.ncell, kSScan);
    k_scan_tiles<kSScan><<<ntiles, kSScan, 0, s>>>(a, sl.ncell, sl.d_tiles);
    k_scan_tile_sums<kSScan><<<1, kSScan, 0, s>>>(a, sl.ncell, sl.d_tiles, ntiles);
    k_scan_add<kSScan><<<ntiles, kSScan, 0, s>>>(a, sl.ncell, sl.d_tiles);
    k_scatter<kSB><<<sblocks(n, kSB), kSB, 0, s>>>(a, n);
    k_sort_cells<<<sblocks((long long)sl.ncell * 32, kSB), kSB, 0, s>>>(a, sl.box, sl.ncell);
    k_permute<kSB><<<sblocks(n, kSB), kSB, 0, s>>>(a, sl.box, n, nullptr);
    SCUDA(x, cudaMemcpyAsync(a.q, a.q_tmp, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s));
    SCUDA(x, cudaMemcpyAsync(a.v, a.v_tmp, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s));
    SCUDA(x, cudaMemcpyAsync(a.ids, a.ids_tmp, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
    SCUDA(x, cudaMemcpyAsync(a.type, a.type_tmp, sizeof(int) * n, cudaMemcpyDeviceToDevice, s));
  }
  SCUDA(x, cudaGetLastError());
  // border layer sizes: the own bottom layer ends at the start of layer 1,
  // the own top layer starts at layer nzl - 1
  std::vector<int> edge(2 * P);
  for (int k = 0; k < P; k++) {
    Slab &sl = x->s[k];
    SCUDA(x, cudaSetDevice(sl.dev));
    const int layer = sl.box.ms[0] * sl.box.ms[1];
    SCUDA(x, cudaMemcpyAsync(&edge[2 * k], sl.a.cell_start + layer, sizeof(int), cudaMemcpyDeviceToHost, sl.stream));
    SCUDA(x, cudaMemcpyAsync(&edge[2 * k + 1], sl.a.cell_start + (sl.box.nzl - 1) * layer, sizeof(int),
                             cudaMemcpyDeviceToHost, sl.stream));
  }
  if (mdg_status r = sync_all(x)) return r;
  for (int k = 0; k < P; k++) {
    Status st;
    if (mdg_status r = slab_status(x, k, &st)) return r;
    if (st.error) return device_error(x, st.error);
  }
  for (int k = 0; k < P; k++) {
    Slab &sl = x->s[k];
    sl.n_bot = edge[2 * k];
    sl.n_top = sl.n_own - edge[2 * k + 1];
  }
  for (int k = 0; k < P; k++) {
    Slab &sl = x->s[k];
    sl.ng_lo = x->s[below(x, k)].n_top;
    sl.ng_hi = x->s[above(x, k)].n_bot;
    if (sl.n_own + sl.ng_lo + sl.ng_hi > sl.cap)
      return sfail(x, MDG_ERR_CAPACITY, "a slab's atoms and ghosts exceed its capacity");
  }
  // 4. ghost layers: positions, velocities, prefilter coordinates, strip
  // bits and ids of the neighbours' border layers, and their trim rows
  for (auto pick : {pick_q, pick_v, pick_qloc, pick_mult, pick_ids})
    if (mdg_status r = push_borders(x, pick)) return r;
  for (int k = 0; k < P; k++) {
    Slab &sl = x->s[k];
    SCUDA(x, cudaSetDevice(sl.dev));
    const Slab &lo = x->s[below(x, k)], &hi = x->s[above(x, k)];
    const int ms1 = sl.box.ms[1], row = sl.box.ms[0] * kXSub + 1, blk = ms1 * row;
    int *own_tab = sl.a.xsub;
    // the block of the slab below's top layer -> ghost-low block (nzl)
    SCUDA(x, cudaMemcpyPeerAsync(own_tab + (size_t)sl.box.nzl * blk, sl.dev, lo.a.xsub + (size_t)(lo.box.nzl - 1) * blk,
                                 lo.dev, sizeof(int) * blk, sl.stream));
    k_slab_shift<<<sblocks(blk, 256), 256, 0, sl.stream>>>(own_tab + (size_t)sl.box.nzl * blk, blk,
                                                           sl.n_own - (lo.n_own - lo.n_top));
    // the block of the slab above's bottom layer -> ghost-high block (nzl + 1)
    SCUDA(x, cudaMemcpyPeerAsync(own_tab + (size_t)(sl.box.nzl + 1) * blk, sl.dev, hi.a.xsub, hi.dev,
                                 sizeof(int) * blk, sl.stream));
    k_slab_shift<<<sblocks(blk, 256), 256, 0, sl.stream>>>(own_tab + (size_t)(sl.box.nzl + 1) * blk, blk,
                                                           sl.n_own + sl.ng_lo);
  }
  // 5. lists of the own atoms; rows that overflow grow the table and are built again
  for (int attempt = 0; attempt < 4; attempt++) {
    for (Slab &sl : x->s) {
      SCUDA(x, cudaSetDevice(sl.dev));
      k_build<kSF, false, true><<<sblocks(sl.n_own, kSF), kSF, 0, sl.stream>>>(sl.a, sl.box, sl.n_own);
    }
    SCUDA(x, cudaGetLastError());
    if (mdg_status r = sync_all(x)) return r;
    bool again = false;
    for (int k = 0; k < P; k++) {
      Status st;
      if (mdg_status r = slab_status(x, k, &st)) return r;
      if (st.error == kErrCapacity) {
        Slab &sl = x->s[k];
        if (mdg_status r = grow_rows(x, sl, (int)(st.max_row * 1.25) + 8)) return r;
        st.error = 0;
        st.max_row = 0;
        st.list_entries = 0;
        SCUDA(x, cudaMemcpyAsync(sl.a.st, &st, sizeof(Status), cudaMemcpyHostToDevice, sl.stream));
        again = true;
      } else if (st.error) {
        return device_error(x, st.error);
      }
    }
    if (!again) break;
    // slabs that did not overflow rebuild too: their counters restart
    for (Slab &sl : x->s) {
      Status st;
      SCUDA(x, cudaSetDevice(sl.dev));
      SCUDA(x, cudaMemcpyAsync(&st, sl.a.st, sizeof(Status), cudaMemcpyDeviceToHost, sl.stream));
      SCUDA(x, cudaStreamSynchronize(sl.stream));
      st.max_row = 0;
      st.list_entries = 0;
      SCUDA(x, cudaMemcpyAsync(sl.a.st, &st, sizeof(Status), cudaMemcpyHostToDevice, sl.stream));
    }
  }
  for (Slab &sl : x->s) {
    SCUDA(x, cudaSetDevice(sl.dev));
    k_build_done<<<1, 32, 0, sl.stream>>>(sl.a, sl.box);
  }
  SCUDA(x, cudaGetLastError());
  x->rebuilds++;
  return sync_all(x);
}

// PairList::CheckByDisplacement over all slabs (src/pairlist.cc:67-121):
// the displacement maximum and the candidate copies are global.  Returns
// the rebuild decision in *expired.
mdg_status displacement_check(mdg_slabs *x, double lag, bool *expired) {
  const int P = (int)x->s.size();
  for (Slab &sl : x->s) {
    SCUDA(x, cudaSetDevice(sl.dev));
    k_disp_max<kSB><<<sblocks(sl.n_own, kSB), kSB, 0, sl.stream>>>(sl.a, sl.box, sl.n_own, lag);
  }
  std::vector<Status> st(P);
  unsigned long long dmax = 0ull;
  for (int k = 0; k < P; k++) {
    if (mdg_status r = slab_status(x, k, &st[k])) return r;
    dmax = std::max(dmax, st[k].dr2max_bits);
  }
  for (Slab &sl : x->s) {
    SCUDA(x, cudaSetDevice(sl.dev));
    SCUDA(x, cudaMemcpyAsync(&sl.a.st->dr2max_bits, &dmax, sizeof dmax, cudaMemcpyHostToDevice, sl.stream));
    k_disp_collect<kSB><<<sblocks(sl.n_own, kSB), kSB, 0, sl.stream>>>(sl.a, sl.box, sl.n_own,
                                                                       x->prm.check_list_length, lag);
  }
  long long weighted = 0, images = 0;
  for (int k = 0; k < P; k++) {
    if (mdg_status r = slab_status(x, k, &st[k])) return r;
    if (st[k].error) return device_error(x, st[k].error);
    weighted += st[k].cand_weighted;
    images += st[k].total_images;
  }
  const long long cll = x->prm.check_list_length;
  const long long nl = images > cll ? cll : images;
  if (weighted >= nl) {
    *expired = true;
    return MDG_OK;
  }
  // every slab's candidates (all stored: weighted < nl <= cll) in one list
  const int stride = (int)cll;
  std::vector<double> all((size_t)6 * stride, 0.0), part((size_t)6 * stride);
  int l = 0;
  for (int k = 0; k < P; k++) {
    Slab &sl = x->s[k];
    const int m = st[k].cand_n;
    if (m == 0) continue;
    SCUDA(x, cudaSetDevice(sl.dev));
    k_slab_cand_positions<<<sblocks(m, 128), 128, 0, sl.stream>>>(sl.a, sl.box, m, lag, sl.d_cand, stride);
    SCUDA(x, cudaMemcpyAsync(part.data(), sl.d_cand, sizeof(double) * 6 * stride, cudaMemcpyDeviceToHost, sl.stream));
    SCUDA(x, cudaStreamSynchronize(sl.stream));
    for (int d = 0; d < 6; d++)
      for (int c = 0; c < m; c++) all[(size_t)d * stride + l + c] = part[(size_t)d * stride + c];
    l += m;
  }
  Slab &s0 = x->s[0];
  SCUDA(x, cudaSetDevice(s0.dev));
  int found = 0;
  SCUDA(x, cudaMemcpyAsync(s0.d_cand, all.data(), sizeof(double) * 6 * stride, cudaMemcpyHostToDevice, s0.stream));
  SCUDA(x, cudaMemsetAsync(s0.d_found, 0, sizeof(int), s0.stream));
  k_slab_pairs<<<16, 256, 0, s0.stream>>>(s0.d_cand, stride, l, x->gbox.sl2, x->gbox.rc2, s0.d_found);
  SCUDA(x, cudaMemcpyAsync(&found, s0.d_found, sizeof(int), cudaMemcpyDeviceToHost, s0.stream));
  SCUDA(x, cudaStreamSynchronize(s0.stream));
  *expired = found != 0;
  return MDG_OK;
}

// One MDManager::Calculate over all slabs (NVE): the global expiry test
// (every slab runs k_expiry on the global |v| maximum, so every slab keeps
// the same skin budget), the global displacement check and rebuild, then
// drift, border push, kick and drift.
mdg_status slab_step(mdg_slabs *x) {
  const int P = (int)x->s.size();
  const bool fp32 = x->prm.precision == MDG_FP32_MIXED;
  unsigned long long vmax = 0ull;
  std::vector<Status> st(P);
  for (int k = 0; k < P; k++) {
    if (mdg_status r = slab_status(x, k, &st[k])) return r;
    if (st[k].error) return device_error(x, st[k].error);
    vmax = std::max(vmax, st[k].vmax2_bits);
  }
  for (Slab &sl : x->s) {
    SCUDA(x, cudaSetDevice(sl.dev));
    SCUDA(x, cudaMemcpyAsync(&sl.a.st->vmax2_bits, &vmax, sizeof vmax, cudaMemcpyHostToDevice, sl.stream));
    k_expiry<<<1, 32, 0, sl.stream>>>(sl.a, sl.box, 0, 0, 0, sl.d_flags);
  }
  int flags[2] = {0, 0};
  {
    Slab &s0 = x->s[0];
    SCUDA(x, cudaSetDevice(s0.dev));
    SCUDA(x, cudaMemcpyAsync(flags, s0.d_flags, sizeof flags, cudaMemcpyDeviceToHost, s0.stream));
  }
  if (mdg_status r = sync_all(x)) return r;
  for (int k = 0; k < P; k++) {
    if (mdg_status r = slab_status(x, k, &st[k])) return r;
    if (st[k].error) return device_error(x, st[k].error);
  }
  bool build = flags[1] != 0;
  if (flags[0]) {
    x->disp_checks++;
    if (mdg_status r = displacement_check(x, 0.5 * x->prm.time_step, &build)) return r;
  }
  if (build)
    if (mdg_status r = rebuild(x)) return r;
  // first half drift of the own atoms (FP32-mixed: and their fixed-point copy)
  for (Slab &sl : x->s) {
    SCUDA(x, cudaSetDevice(sl.dev));
    if (fp32) k_drift<kSB, true><<<sblocks(sl.n_own, kSB), kSB, 0, sl.stream>>>(sl.a, sl.box, sl.n_own, 0);
    else k_drift<kSB, false><<<sblocks(sl.n_own, kSB), kSB, 0, sl.stream>>>(sl.a, sl.box, sl.n_own, 0);
  }
  if (mdg_status r = push_borders(x, fp32 ? pick_qfix : pick_q)) return r;
  const Thermo th{};
  for (Slab &sl : x->s) {
    SCUDA(x, cudaSetDevice(sl.dev));
    const int n = sl.n_own;
    if (fp32) {
      const int nb = sblocks((long long)n * x->tpa, kSF);
      if (x->tpa == 4) k_force_fp32<kSF, kKick, 1, 4><<<nb, kSF, 0, sl.stream>>>(sl.a, sl.box, n, th, sl.a.qfix, nullptr);
      else if (x->tpa == 2) k_force_fp32<kSF, kKick, 1, 2><<<nb, kSF, 0, sl.stream>>>(sl.a, sl.box, n, th, sl.a.qfix, nullptr);
      else k_force_fp32<kSF, kKick, 1, 1><<<nb, kSF, 0, sl.stream>>>(sl.a, sl.box, n, th, sl.a.qfix, nullptr);
    } else {
      k_force_fp64<kSF, kKick><<<sblocks(n, kSF), kSF, 0, sl.stream>>>(sl.a, sl.box, n, th);
      k_drift<kSB, false><<<sblocks(n, kSB), kSB, 0, sl.stream>>>(sl.a, sl.box, n, 1);
    }
  }
  SCUDA(x, cudaGetLastError());
  x->steps++;
  return MDG_OK;
}

void free_slab(Slab &sl) {
  cudaSetDevice(sl.dev);
  if (sl.stream) cudaStreamSynchronize(sl.stream);
  Arrays &a = sl.a;
  void *ptrs[] = {a.q, a.v, a.q_old, a.qfix, a.qfix2, a.qloc, a.cxyz, a.xsub, a.ids, a.type, a.cell, a.nbr, a.nnbr,
                  a.cell_count, a.cell_start, a.slot, a.perm, a.perm2, a.q_tmp, a.v_tmp, a.ids_tmp, a.type_tmp,
                  a.cell_tmp, a.mult, a.cand, a.partials, a.st, sl.d_tiles, sl.d_flags, sl.d_sums, sl.d_cand,
                  sl.d_found, sl.d_count, sl.sq[0], sl.sq[1], sl.sv[0], sl.sv[1], sl.sid[0], sl.sid[1],
                  sl.stype[0], sl.stype[1]};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (sl.pushed) cudaEventDestroy(sl.pushed);
  if (sl.stream) cudaStreamDestroy(sl.stream);
  sl = Slab{};
}

}  // namespace

extern "C" {

mdg_status mdg_slabs_create(const mdg_params *prm, int nslabs, const int *devices, mdg_slabs **out) {
  if (!prm || !out || nslabs < 2) return MDG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (prm->capacity < 1 || prm->cutoff <= 0.0 || prm->buffer_length < 0.0 || prm->time_step <= 0.0 ||
      prm->check_list_length < 1 || (prm->precision != MDG_FP64 && prm->precision != MDG_FP32_MIXED) ||
      prm->thermostat != MDG_NVE ||
      (prm->threads_per_atom != 0 && prm->threads_per_atom != 1 && prm->threads_per_atom != 2 &&
       prm->threads_per_atom != 4))
    return MDG_ERR_INVALID_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MDG_ERR_NO_DEVICE;
  mdg_slabs *x = new mdg_slabs();
  x->prm = *prm;
  x->tpa = prm->threads_per_atom > 0 ? prm->threads_per_atom : 1;
  Box &g = x->gbox;
  const double SL = prm->cutoff + prm->buffer_length;  // src/simulationinfo.cc:6-7
  for (int d = 0; d < 3; d++) {
    const int ms = (int)(prm->L[d] / SL);
    if (!(prm->L[d] > 0.0) || ms < 3) {
      delete x;
      return MDG_ERR_BOX_TOO_SMALL;
    }
    g.L[d] = prm->L[d];
    g.hL[d] = 0.5 * prm->L[d];
    g.ms[d] = ms;
    g.inv_cs[d] = (double)ms / prm->L[d];
    g.fix_scale[d] = (float)(prm->L[d] / 4294967296.0);
    g.cs[d] = prm->L[d] / (double)ms;
  }
  if (g.ms[0] >= 2048 || g.ms[1] >= 2048 || g.ms[2] >= 1024 || nslabs > g.ms[2]) {
    delete x;
    return MDG_ERR_INVALID_ARGUMENT;  // at least one cell layer per slab; packed cell coordinates
  }
  g.ncell = g.ms[0] * g.ms[1] * g.ms[2];
  g.sl = SL;
  g.sl2 = SL * SL;
  prefilter_band(g.sl2, SL, g.L[0], &g.sl2_lo, &g.sl2_hi);
  g.rc = prm->cutoff;
  g.rc2 = prm->cutoff * prm->cutoff;
  {  // Variables::Variables, src/variables.cc:21-27
    const double s2 = 1.0 / (prm->cutoff * prm->cutoff);
    const double s6 = s2 * s2 * s2, s8 = s6 * s2, s12 = s6 * s6, s14 = s12 * s2;
    g.c2 = 6.0 * s14 - 3.0 * s8;
    g.c0 = -s12 + s6 - g.c2 / s2;
  }
  g.dt = prm->time_step;
  g.buffer_length = prm->buffer_length;
  g.rc2f = (float)g.rc2;
  g.c2x8f = (float)(g.c2 * 8.0);
  g.check_list_length = prm->check_list_length;
  g.slab = 0;
  g.z0 = 0;
  g.nzl = g.ms[2];
  // layers per slab: as even as the layer count allows (ParaInfo's equal
  // domains, src/parainfo.cc:16-94, along z)
  const int cap_all = prm->capacity;
  const int layer_atoms = (int)std::ceil(1.5 * cap_all / (double)g.ms[2]) + 64;
  x->s.resize(nslabs);
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < nslabs && e == cudaSuccess; k++) {
    Slab &sl = x->s[k];
    sl.dev = devices ? devices[k] : prm->device;
    if (sl.dev < 0 || sl.dev >= ndev) {
      e = cudaErrorInvalidDevice;
      break;
    }
    sl.box = g;
    sl.box.slab = 1;
    sl.box.z0 = (int)((long long)g.ms[2] * k / nslabs);
    sl.box.nzl = (int)((long long)g.ms[2] * (k + 1) / nslabs) - sl.box.z0;
    sl.ncell = g.ms[0] * g.ms[1] * sl.box.nzl;
    sl.box.ncell = sl.ncell;
    sl.cap = std::min(cap_all, (int)std::ceil(1.5 * cap_all * sl.box.nzl / (double)g.ms[2]) + 4096) + 2 * layer_atoms;
    e = cudaSetDevice(sl.dev);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.pushed, cudaEventDisableTiming);
    Arrays &a = sl.a;
    const int cap = sl.cap;
    a.stride = (cap + 31) / 32 * 32;
    const size_t tab = (size_t)(sl.box.nzl + 2) * g.ms[1] * (g.ms[0] * kXSub + 1);
    if (e == cudaSuccess) e = salloc(&a.q, cap);
    if (e == cudaSuccess) e = salloc(&a.v, cap);
    if (e == cudaSuccess) e = salloc(&a.q_old, cap);
    if (e == cudaSuccess) e = salloc(&a.qfix, cap);
    if (e == cudaSuccess) e = salloc(&a.qloc, cap);
    if (e == cudaSuccess) e = salloc(&a.cxyz, cap);
    if (e == cudaSuccess) e = salloc(&a.xsub, tab);
    if (e == cudaSuccess) e = salloc(&a.ids, cap);
    if (e == cudaSuccess) e = salloc(&a.type, cap);
    if (e == cudaSuccess) e = salloc(&a.cell, cap);
    if (e == cudaSuccess) e = salloc(&a.nnbr, cap);
    if (e == cudaSuccess) e = salloc(&a.cell_count, sl.ncell);
    if (e == cudaSuccess) e = salloc(&a.cell_start, sl.ncell + 1);
    if (e == cudaSuccess) e = salloc(&a.slot, cap);
    if (e == cudaSuccess) e = salloc(&a.perm, cap);
    if (e == cudaSuccess) e = salloc(&a.perm2, cap);
    if (e == cudaSuccess) e = salloc(&a.q_tmp, cap);
    if (e == cudaSuccess) e = salloc(&a.v_tmp, cap);
    if (e == cudaSuccess) e = salloc(&a.ids_tmp, cap);
    if (e == cudaSuccess) e = salloc(&a.type_tmp, cap);
    if (e == cudaSuccess) e = salloc(&a.cell_tmp, cap);
    if (e == cudaSuccess) e = salloc(&a.mult, cap);
    if (e == cudaSuccess) e = salloc(&a.cand, prm->check_list_length);
    if (e == cudaSuccess) e = salloc(&a.partials, (size_t)sblocks(cap, kSF) * 3 + 64);
    if (e == cudaSuccess) e = salloc(&a.st, 1);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.st, 0, sizeof(Status), sl.stream);
    if (e == cudaSuccess) e = salloc(&sl.d_tiles, (size_t)sblocks(sl.ncell, kSScan) + 1);
    if (e == cudaSuccess) e = salloc(&sl.d_flags, 4);
    if (e == cudaSuccess) e = salloc(&sl.d_sums, 8);
    if (e == cudaSuccess) e = salloc(&sl.d_cand, (size_t)6 * prm->check_list_length);
    if (e == cudaSuccess) e = salloc(&sl.d_found, 1);
    if (e == cudaSuccess) e = salloc(&sl.d_count, 3);
    const int mcap = cap / 4 + 4096;  // atoms one rebuild may send to one neighbour
    for (int t = 0; t < 2 && e == cudaSuccess; t++) {
      e = salloc(&sl.sq[t], mcap);
      if (e == cudaSuccess) e = salloc(&sl.sv[t], mcap);
      if (e == cudaSuccess) e = salloc(&sl.sid[t], mcap);
      if (e == cudaSuccess) e = salloc(&sl.stype[t], mcap);
    }
    sl.ob = Outbound{{sl.sq[0], sl.sq[1]}, {sl.sv[0], sl.sv[1]}, {sl.sid[0], sl.sid[1]}, {sl.stype[0], sl.stype[1]},
                     sl.d_count, mcap};
  }
  // peer access between the slabs' devices (a no-op when they share one)
  for (int k = 0; k < nslabs && e == cudaSuccess; k++)
    for (int j = 0; j < nslabs; j++) {
      const int a = x->s[k].dev, b = x->s[j].dev;
      if (a == b) continue;
      int ok = 0;
      cudaDeviceCanAccessPeer(&ok, a, b);
      if (!ok) continue;
      cudaSetDevice(a);
      const cudaError_t pe = cudaDeviceEnablePeerAccess(b, 0);
      if (pe != cudaSuccess && pe != cudaErrorPeerAccessAlreadyEnabled) e = pe;
      cudaGetLastError();
    }
  for (Slab &sl : x->s)
    if (e == cudaSuccess) e = cudaStreamSynchronize(sl.stream);
  if (e != cudaSuccess) {
    for (Slab &sl : x->s) free_slab(sl);
    delete x;
    return MDG_ERR_CUDA;
  }
  *out = x;
  return MDG_OK;
}

mdg_status mdg_slabs_destroy(mdg_slabs *x) {
  if (!x) return MDG_ERR_INVALID_ARGUMENT;
  for (Slab &sl : x->s) free_slab(sl);
  delete x;
  return MDG_OK;
}

mdg_status mdg_slabs_set_state(mdg_slabs *x, const double *q4, const double *v4, const int *type, int n) {
  if (!x || n < 0 || (n > 0 && (!q4 || !v4))) return MDG_ERR_INVALID_ARGUMENT;
  if (n > x->prm.capacity) return sfail(x, MDG_ERR_CAPACITY, "more atoms than the capacity");
  const int P = (int)x->s.size();
  const Box &g = x->gbox;
  // every atom to the slab of its global cell layer (the wrap and the layer
  // as k_slab_sort_out computes them)
  std::vector<std::vector<int>> mine(P);
  std::vector<int> owner_of_layer(g.ms[2]);
  for (int k = 0; k < P; k++)
    for (int z = x->s[k].box.z0; z < x->s[k].box.z0 + x->s[k].box.nzl; z++) owner_of_layer[z] = k;
  for (int i = 0; i < n; i++) {
    double z = q4[4 * i + 2];
    if (!std::isfinite(z) || !std::isfinite(q4[4 * i]) || !std::isfinite(q4[4 * i + 1]))
      return sfail(x, MDG_ERR_NONFINITE, "non-finite value in the uploaded state");
    if (z < 0.0) z += g.L[2];
    else if (z > g.L[2]) z -= g.L[2];
    int c = (int)(z * g.inv_cs[2]);
    c = c < 0 ? 0 : (c >= g.ms[2] ? g.ms[2] - 1 : c);
    mine[owner_of_layer[c]].push_back(i);
  }
  // neighbour-row capacity from the mean density (grown on overflow)
  const double vol = g.L[0] * g.L[1] * g.L[2];
  const int maxnb = (int)std::ceil(1.6 * (n / vol) * 4.0 / 3.0 * M_PI * g.sl * g.sl * g.sl + 32.0);
  for (int k = 0; k < P; k++) {
    Slab &sl = x->s[k];
    const int m = (int)mine[k].size();
    if (m > sl.cap) return sfail(x, MDG_ERR_CAPACITY, "a slab's atoms exceed its capacity");
    std::vector<double4> hq(m), hv(m);
    std::vector<int> hid(m), ht(m);
    for (int t = 0; t < m; t++) {
      const int i = mine[k][t];
      hq[t] = make_double4(q4[4 * i], q4[4 * i + 1], q4[4 * i + 2], 0.0);
      hv[t] = make_double4(v4[4 * i], v4[4 * i + 1], v4[4 * i + 2], 0.0);
      hid[t] = i;
      ht[t] = type ? type[i] : 0;
    }
    if (mdg_status r = grow_rows(x, sl, maxnb)) return r;
    SCUDA(x, cudaSetDevice(sl.dev));
    SCUDA(x, cudaMemcpyAsync(sl.a.q, hq.data(), sizeof(double4) * m, cudaMemcpyHostToDevice, sl.stream));
    SCUDA(x, cudaMemcpyAsync(sl.a.v, hv.data(), sizeof(double4) * m, cudaMemcpyHostToDevice, sl.stream));
    SCUDA(x, cudaMemcpyAsync(sl.a.ids, hid.data(), sizeof(int) * m, cudaMemcpyHostToDevice, sl.stream));
    SCUDA(x, cudaMemcpyAsync(sl.a.type, ht.data(), sizeof(int) * m, cudaMemcpyHostToDevice, sl.stream));
    Status st{};
    st.list_stale = 1;
    st.budget = x->prm.buffer_length;
    SCUDA(x, cudaMemcpyAsync(sl.a.st, &st, sizeof(Status), cudaMemcpyHostToDevice, sl.stream));
    if (m > 0) k_vmax<kSB><<<sblocks(m, kSB), kSB, 0, sl.stream>>>(sl.a, m);
    sl.n_own = m;
    sl.ng_lo = sl.ng_hi = sl.n_bot = sl.n_top = 0;
    SCUDA(x, cudaStreamSynchronize(sl.stream));
    std::vector<double4>().swap(hq);
  }
  SCUDA(x, cudaGetLastError());
  x->n = n;
  x->steps = x->rebuilds = x->disp_checks = 0;
  x->state_set = true;
  return MDG_OK;
}

mdg_status mdg_slabs_calculate(mdg_slabs *x, int nsteps) {
  if (!x || nsteps < 0) return MDG_ERR_INVALID_ARGUMENT;
  if (!x->state_set) return sfail(x, MDG_ERR_STATE, "no state uploaded");
  for (int t = 0; t < nsteps; t++)
    if (mdg_status r = slab_step(x)) return r;
  return sync_all(x);
}

mdg_status mdg_slabs_get_state(mdg_slabs *x, double *q4, double *v4, int n) {
  if (!x || !x->state_set || n != x->n || (n > 0 && (!q4 || !v4))) return MDG_ERR_INVALID_ARGUMENT;
  for (Slab &sl : x->s) {
    const int m = sl.n_own;
    std::vector<double4> hq(m), hv(m);
    std::vector<int> hid(m);
    SCUDA(x, cudaSetDevice(sl.dev));
    SCUDA(x, cudaMemcpyAsync(hq.data(), sl.a.q, sizeof(double4) * m, cudaMemcpyDeviceToHost, sl.stream));
    SCUDA(x, cudaMemcpyAsync(hv.data(), sl.a.v, sizeof(double4) * m, cudaMemcpyDeviceToHost, sl.stream));
    SCUDA(x, cudaMemcpyAsync(hid.data(), sl.a.ids, sizeof(int) * m, cudaMemcpyDeviceToHost, sl.stream));
    SCUDA(x, cudaStreamSynchronize(sl.stream));
    for (int t = 0; t < m; t++) {
      const int i = hid[t];
      if (i < 0 || i >= n) return sfail(x, MDG_ERR_STATE, "slab ids out of range");
      q4[4 * i] = hq[t].x; q4[4 * i + 1] = hq[t].y; q4[4 * i + 2] = hq[t].z; q4[4 * i + 3] = 0.0;
      v4[4 * i] = hv[t].x; v4[4 * i + 1] = hv[t].y; v4[4 * i + 2] = hv[t].z; v4[4 * i + 3] = 0.0;
    }
  }
  return MDG_OK;
}

mdg_status mdg_slabs_observe(mdg_slabs *x, double *ke, double *pe, double *virial) {
  if (!x || !x->state_set) return MDG_ERR_INVALID_ARGUMENT;
  if (x->rebuilds == 0)
    if (mdg_status r = rebuild(x)) return r;
  // the ghosts' current positions and velocities; partners reached through
  // the periodic boundary at their current positions (MDG_OBSERVE_CURRENT)
  if (mdg_status r = push_borders(x, pick_q)) return r;
  if (mdg_status r = push_borders(x, pick_v)) return r;
  double out[3] = {0.0, 0.0, 0.0};
  for (Slab &sl : x->s) {
    SCUDA(x, cudaSetDevice(sl.dev));
    const int nb = sblocks(sl.n_own, kSB);
    k_observe<kSB><<<nb, kSB, 0, sl.stream>>>(sl.a, sl.box, sl.n_own, 0.0);
    k_final_sum<256, 3><<<1, 256, 0, sl.stream>>>(sl.a.partials, nb, sl.d_sums);
    double part[3];
    SCUDA(x, cudaMemcpyAsync(part, sl.d_sums, sizeof part, cudaMemcpyDeviceToHost, sl.stream));
    SCUDA(x, cudaStreamSynchronize(sl.stream));
    for (int c = 0; c < 3; c++) out[c] += part[c];
  }
  if (ke) *ke = out[0];
  if (pe) *pe = out[1];
  if (virial) *virial = out[2] / 3.0;
  return MDG_OK;
}

mdg_status mdg_slabs_forces(mdg_slabs *x, double *f4, int n) {
  if (!x || !x->state_set || n != x->n || (n > 0 && !f4)) return MDG_ERR_INVALID_ARGUMENT;
  if (x->rebuilds == 0)
    if (mdg_status r = rebuild(x)) return r;
  const bool fp32 = x->prm.precision == MDG_FP32_MIXED;
  if (fp32)
    for (Slab &sl : x->s) {
      SCUDA(x, cudaSetDevice(sl.dev));
      k_pack_fix<kSB><<<sblocks(sl.n_own, kSB), kSB, 0, sl.stream>>>(sl.a, sl.box, sl.n_own);
    }
  if (mdg_status r = push_borders(x, fp32 ? pick_qfix : pick_q)) return r;
  const Thermo th{};
  for (Slab &sl : x->s) {
    SCUDA(x, cudaSetDevice(sl.dev));
    const int m = sl.n_own;
    if (fp32) k_force_fp32<kSF, kForceOut, 0, 1><<<sblocks(m, kSF), kSF, 0, sl.stream>>>(sl.a, sl.box, m, th, sl.a.qfix, nullptr);
    else k_force_fp64<kSF, kForceOut><<<sblocks(m, kSF), kSF, 0, sl.stream>>>(sl.a, sl.box, m, th);
    std::vector<double4> hf(m);
    std::vector<int> hid(m);
    SCUDA(x, cudaMemcpyAsync(hf.data(), sl.a.v_tmp, sizeof(double4) * m, cudaMemcpyDeviceToHost, sl.stream));
    SCUDA(x, cudaMemcpyAsync(hid.data(), sl.a.ids, sizeof(int) * m, cudaMemcpyDeviceToHost, sl.stream));
    SCUDA(x, cudaStreamSynchronize(sl.stream));
    for (int t = 0; t < m; t++) {
      const int i = hid[t];
      f4[4 * i] = hf[t].x; f4[4 * i + 1] = hf[t].y; f4[4 * i + 2] = hf[t].z; f4[4 * i + 3] = 0.0;
    }
  }
  return MDG_OK;
}

mdg_status mdg_slabs_info(mdg_slabs *x, int64_t *steps, int64_t *rebuilds, int *owned, int *ghosts) {
  if (!x) return MDG_ERR_INVALID_ARGUMENT;
  if (steps) *steps = x->steps;
  if (rebuilds) *rebuilds = x->rebuilds;
  for (size_t k = 0; k < x->s.size(); k++) {
    if (owned) owned[k] = x->s[k].n_own;
    if (ghosts) ghosts[k] = x->s[k].ng_lo + x->s[k].ng_hi;
  }
  return MDG_OK;
}

const char *mdg_slabs_last_error(mdg_slabs *x) { return x ? x->err.c_str() : "null slabs"; }

}  // extern "C"
