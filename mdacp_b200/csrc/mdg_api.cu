// C ABI of the B200 LJ timestep (include/mdacp_b200.h): handle, buffers,
// the per-step kernel sequence and its CUDA-graph form with device-side
// conditional nodes for the skin check and the pairlist rebuild.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <fstream>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <thread>
#include <vector>

#include "mdacp_b200.h"
#include "mdg_device.cuh"

using namespace mdg;

namespace {

constexpr int kBlock = 256;       // streaming kernels
constexpr int kForceBlock = 128;  // pair kernels
constexpr int kScanSingleCells = 16384;  // cell grids up to this size are scanned by one block
#ifndef MDG_PERSIST_BLOCK
#define MDG_PERSIST_BLOCK 128
#endif
constexpr int kPersistBlock = MDG_PERSIST_BLOCK;  // the persistent pass (fewer, larger blocks: cheaper grid barriers)
constexpr int kScanBlock = 1024;  // cells per tile of the cell-count scan
constexpr int kStepsPerGraph = 20;
// Staged atoms per force block for stage_atoms = -1: 36 KB, six blocks per SM.
// Off by default: on the 2.05M-atom liquid the staged pass takes 0.38 ms per
// launch against 0.28 ms for the global gathers (occupancy-bound: 0.44 ms
// at 2560 atoms, 0.52 ms at 3072).
constexpr int kStageDefault = 2304;
constexpr int kStageMax = 12288;     // 192 KB of shared memory

int blocks_for(int n, int b) { return n > 0 ? (n + b - 1) / b : 1; }

// The box-dependent part of the geometry: MeshList::ChangeScale's cell grid
// int(L / SL) per axis (src/meshlist.cc:50-52), cell edges, the minimum-image
// half box and the fixed-point unit.  False when an axis has < 3 cells.
bool box_geometry(mdg::Box &b, const double L[3], double SL) {
  for (int d = 0; d < 3; d++) {
    const int ms = (int)(L[d] / SL);
    if (ms < 3) return false;
  }
  b.sl = SL;
  b.sl2 = SL * SL;
  mdg::prefilter_band(b.sl2, SL, L[0], &b.sl2_lo, &b.sl2_hi);
  for (int d = 0; d < 3; d++) {
    b.L[d] = L[d];
    b.hL[d] = 0.5 * L[d];
    b.ms[d] = (int)(L[d] / SL);
    b.inv_cs[d] = (double)b.ms[d] / L[d];
    b.fix_scale[d] = (float)(L[d] / 4294967296.0);
    b.cs[d] = L[d] / (double)b.ms[d];
  }
  b.ncell = b.ms[0] * b.ms[1] * b.ms[2];
  b.slab = 0;
  b.z0 = 0;
  b.nzl = b.ms[2];
  return true;
}

// The list build packs cell coordinates into one int (pack_cell).
bool cells_packable(const mdg::Box &b) { return b.ms[0] < 2048 && b.ms[1] < 2048 && b.ms[2] < 1024; }

// Entries of the list build's trim table: one block of 8 ms_x + 1 per x-row.
size_t trim_table_size(const mdg::Box &b) { return (size_t)b.ms[1] * b.ms[2] * (b.ms[0] * kXSub + 1); }

}  // namespace

struct mdg_handle {
  mdg_params prm{};
  Box box{};
  Arrays a{};
  int n = 0;
  int cap = 0;
  int ncell = 0;
  cudaStream_t stream = nullptr;      // work stream (user's or owned)
  bool own_stream = false;
  cudaStream_t cap_stream = nullptr;  // capture stream (always owned)
  int *d_flags = nullptr;             // eager-mode conditional values
  double *d_sums = nullptr;           // reduction outputs
  int *d_tiles = nullptr;             // tile totals of the cell-count scan
  size_t partial_cap = 0;
  bool state_set = false;
  // graph of kStepsPerGraph steps
  cudaGraphExec_t exec = nullptr;
  cudaGraphExec_t rebuild_exec = nullptr;  // persistent pipeline: the guarded rebuild step
  bool rebuild_dirty = true;
  bool graph_dirty = true;
  bool timing = false;
  bool use_graphs = true;
  int observer_mode = 0;              // MDG_OBSERVE_CURRENT or MDG_OBSERVE_GHOST_LAG
  double obs_lag = 0.0;               // half-step lag of the reference's ghost copies, when it applies
  std::vector<cudaEvent_t> ev;        // force-kernel start/stop per step of the graph
  double force_ms = 0.0;
  int64_t force_launches = 0;
  int64_t kernel_launches = 0;
  int graph_kernel_count = 0;         // kernels per graph launch outside conditionals
  // fused FP32 NVE step: which fixed-point buffer (0: qfix, 1: qfix2) holds
  // every atom's position after the coming step's first half drift; -1: none
  int fix_buf = -1;
  int cell_cap = 0;                   // cells the cell tables hold
  int tpa = 0;                        // lanes per atom of the FP32 force pass (0: to be tuned)
  int build_block = 0;                // threads per block of the list build (0: to be tuned)
  int build_tpa = 0;                  // lanes per atom of the list build (0: to be tuned)
  GridBarrier *d_bar = nullptr;       // persistent pass: grid barrier
  int *d_pout = nullptr;              // persistent pass: block 0's decisions
  int64_t persistent_steps = 0;
  int persist_grid = -1;              // blocks of the persistent pass (-1: not computed yet)
  double steps_per_cycle = 4.0;       // persistent pipeline: steps per queued launch pair, as last seen
  External ext{};                     // executor applied after every step (kind 0: none)
  // snapshots: one set of pinned buffers per handle, at most one pending writer
  std::thread writer;
  std::string writer_error;           // failure of the last writer (read after joining it)
  double4 *snap_q = nullptr, *snap_v = nullptr;
  int *snap_t = nullptr;
  int snap_cap = 0;
  cudaEvent_t snap_done = nullptr;
  std::string err;
};

namespace {

mdg_status fail(mdg_handle *h, mdg_status s, const std::string &msg) {
  if (h) h->err = msg;
  return s;
}

#define CUDA_TRY(h, expr)                                                                  \
  do {                                                                                     \
    cudaError_t e_ = (expr);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      return fail((h), MDG_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    }                                                                                      \
  } while (0)

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
  return cudaMalloc((void **)p, std::max<size_t>(count, 1) * sizeof(T));
}

void free_arrays(Arrays &a) {
  void *ptrs[] = {a.q, a.v, a.q_old, a.qfix, a.qfix2, a.qloc, a.cxyz, a.xsub, a.ids, a.type, a.cell, a.nbr, a.nnbr, a.cell_count,
                  a.cell_start, a.slot, a.perm, a.perm2, a.q_tmp, a.v_tmp, a.v_lag, a.ids_tmp, a.type_tmp,
                  a.cell_tmp, a.mult, a.cand, a.partials, a.st, a.stage_rng, a.stage_n, a.nbr16, a.disp2};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  a = Arrays{};
}

void destroy_graph(mdg_handle *h) {
  if (h->exec) cudaGraphExecDestroy(h->exec);
  h->exec = nullptr;
  if (h->rebuild_exec) cudaGraphExecDestroy(h->rebuild_exec);
  h->rebuild_exec = nullptr;
  h->rebuild_dirty = true;
  h->persist_grid = -1;  // lanes per atom or the atom count may have changed
  for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
  h->ev.clear();
  h->graph_dirty = true;
}

mdg_status translate_device_error(mdg_handle *h, const Status &st) {
  if (st.error & kErrTooFast) {
    char buf[160];
    snprintf(buf, sizeof buf,
             "Too fast particles exists. Try smaller time step (max_velocity = %g)", st.too_fast_v);
    return fail(h, MDG_ERR_TOO_FAST, buf);
  }
  if (st.error & kErrNonFinite) return fail(h, MDG_ERR_NONFINITE, "non-finite position or velocity");
  if (st.error & kErrInvalidPosition) return fail(h, MDG_ERR_INVALID_POSITION, "Invalid position");
  if (st.error & kErrCapacity) return fail(h, MDG_ERR_CAPACITY, "neighbour capacity exceeded");
  if (st.error & kErrTimeout) return fail(h, MDG_ERR_TIMEOUT, "device wait timed out");
  if (st.error & kErrStage) return fail(h, MDG_ERR_STATE, "staged partner index outside its block's stage");
  return MDG_OK;
}

mdg_status read_status(mdg_handle *h, Status *st) {
  CUDA_TRY(h, cudaMemcpyAsync(st, h->a.st, sizeof(Status), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return MDG_OK;
}

// (Re)allocates the neighbour table for `maxnb` partners per atom.
mdg_status alloc_neighbors(mdg_handle *h, int maxnb) {
  maxnb = std::max(8, (maxnb + 7) / 8 * 8);
  if (h->a.nbr && maxnb <= h->a.maxnb) return MDG_OK;
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (h->a.nbr) cudaFree(h->a.nbr);
  h->a.nbr = nullptr;
  CUDA_TRY(h, dalloc(&h->a.nbr, (size_t)maxnb * h->a.stride));
  if (h->a.stage_cap > 0) {
    if (h->a.nbr16) cudaFree(h->a.nbr16);
    h->a.nbr16 = nullptr;
    CUDA_TRY(h, dalloc(&h->a.nbr16, (size_t)(maxnb / 4) * h->a.stride));
  }
  h->a.maxnb = maxnb;
  destroy_graph(h);
  return MDG_OK;
}

// Neighbour-row capacity from the densest cell of the uploaded state.
int estimate_max_neighbors(const mdg_handle *h, const double *q4, int n) {
  const Box &b = h->box;
  std::vector<int> count(h->ncell, 0);
  int mx = 0;
  for (int i = 0; i < n; i++) {
    int c[3];
    bool finite = true;
    for (int d = 0; d < 3; d++) {
      double x = q4[4 * i + d];
      if (!std::isfinite(x)) {
        finite = false;
        break;
      }
      x -= b.L[d] * std::floor(x / b.L[d]);
      const double k = std::floor(x * b.inv_cs[d]);
      c[d] = k < 0.0 ? 0 : (k >= b.ms[d] ? b.ms[d] - 1 : (int)k);
    }
    if (!finite) continue;
    const int idx = (c[2] * b.ms[1] + c[1]) * b.ms[0] + c[0];
    mx = std::max(mx, ++count[idx]);
  }
  const double cell_vol = b.L[0] * b.L[1] * b.L[2] / (double)h->ncell;
  const double rho_max = std::max((double)mx / cell_vol, (double)n / (b.L[0] * b.L[1] * b.L[2]));
  const double sphere = 4.0 / 3.0 * M_PI * b.sl * b.sl * b.sl;
  return (int)std::ceil(1.3 * rho_max * sphere + 24.0);
}

// ------------------------------------------------------ kernel sequences
// Displacement check (PairList::CheckByDisplacement).
// lag: age of the reference's ghost copies at this check (see for_each_copy).
void launch_disp(mdg_handle *h, cudaStream_t s, double lag) {
  const int n = h->n;
  k_disp_max<kBlock><<<blocks_for(n, kBlock), kBlock, 0, s>>>(h->a, h->box, n, lag);
  k_disp_collect<kBlock><<<blocks_for(n, kBlock), kBlock, 0, s>>>(h->a, h->box, n,
                                                                   h->prm.check_list_length, lag);
  k_disp_pairs<256><<<kPairParts, 256, 0, s>>>(h->a, h->box, lag);
}

// Ghost age at the skin check of a step: the previous step ended with a half
// drift after the ghosts were refreshed, except in the Langevin branch.
double step_lag(const mdg_handle *h) {
  return h->prm.thermostat == MDG_LANGEVIN ? 0.0 : 0.5 * h->prm.time_step;
}

// Pairlist rebuild (MDManager::MakePairList).
// pack: where to put the coming step's first-drift positions after the
// rebuild (the fused FP32 NVE step), or nullptr.
// Kernels of one rebuild (launch_build).
int build_kernels(const mdg_handle *h) { return (h->ncell <= kScanSingleCells ? 9 : 11) + (h->a.stage_cap > 0 ? 1 : 0); }

// The list build alone (the rows of the atoms' current cell order), with
// `block` threads per block and `lanes` threads per atom.
template <int BLOCK>
void launch_list_build_block(mdg_handle *h, cudaStream_t s, int lanes) {
  const int n = h->n;
  const int nb = (int)std::max<long long>(1, ((long long)n * lanes + BLOCK - 1) / BLOCK);
  if (lanes == 8) k_build<BLOCK, false, false, 8><<<nb, BLOCK, 0, s>>>(h->a, h->box, n);
  else if (lanes == 4) k_build<BLOCK, false, false, 4><<<nb, BLOCK, 0, s>>>(h->a, h->box, n);
  else if (lanes == 2) k_build<BLOCK, false, false, 2><<<nb, BLOCK, 0, s>>>(h->a, h->box, n);
  else k_build<BLOCK, false, false, 1><<<nb, BLOCK, 0, s>>>(h->a, h->box, n);
}

void launch_list_build(mdg_handle *h, cudaStream_t s, int block, int lanes) {
  if (block == 64) launch_list_build_block<64>(h, s, lanes);
  else if (block == 256) launch_list_build_block<256>(h, s, lanes);
  else launch_list_build_block<128>(h, s, lanes);
}

void launch_build(mdg_handle *h, cudaStream_t s, int4 *pack = nullptr) {
  const int n = h->n;
  Arrays &a = h->a;
  k_build_begin_clear<kBlock><<<std::min(blocks_for(h->ncell, kBlock), 1024), kBlock, 0, s>>>(a, h->ncell);
  k_cell_assign<kBlock><<<blocks_for(n, kBlock), kBlock, 0, s>>>(a, h->box, n);
  if (h->ncell <= kScanSingleCells) {
    k_scan_single<kScanBlock><<<1, kScanBlock, 0, s>>>(a, h->ncell);
  } else {
    const int ntiles = blocks_for(h->ncell, kScanBlock);
    k_scan_tiles<kScanBlock><<<ntiles, kScanBlock, 0, s>>>(a, h->ncell, h->d_tiles);
    k_scan_tile_sums<kScanBlock><<<1, kScanBlock, 0, s>>>(a, h->ncell, h->d_tiles, ntiles);
    k_scan_add<kScanBlock><<<ntiles, kScanBlock, 0, s>>>(a, h->ncell, h->d_tiles);
  }
  k_scatter<kBlock><<<blocks_for(n, kBlock), kBlock, 0, s>>>(a, n);
  k_sort_cells<<<blocks_for(h->ncell * 32, kBlock), kBlock, 0, s>>>(a, h->box, h->ncell);
  k_permute<kBlock><<<blocks_for(n, kBlock), kBlock, 0, s>>>(a, h->box, n, pack);
  k_copy_back<kBlock><<<blocks_for(n, kBlock), kBlock, 0, s>>>(a, n);
  if (a.stage_cap > 0) {
    static_assert(kForceBlock == kStageBlock, "the build writes stage rows per force block");
    k_stage_plan<kBlock><<<blocks_for(blocks_for(n, kStageBlock), kBlock), kBlock, 0, s>>>(a, h->box, n);
    k_build<kForceBlock, true><<<blocks_for(n, kForceBlock), kForceBlock, 0, s>>>(a, h->box, n);
  } else {
    launch_list_build(h, s, h->build_block > 0 ? h->build_block : kForceBlock, h->build_tpa > 0 ? h->build_tpa : 1);
  }
  k_build_done<<<1, 32, 0, s>>>(a, h->box);
}

// The FP32-mixed NVE step runs as one force pass per step (both half
// drifts fused, the next step's fixed-point copy packed into the other
// buffer).
bool fused_step(const mdg_handle *h) {
  return h->prm.precision == MDG_FP32_MIXED && h->prm.thermostat == MDG_NVE && h->ext.kind == 0;
}

// The executor pass after a step (nothing when none is set); returns kernels.
int launch_external(mdg_handle *h, cudaStream_t s) {
  if (h->ext.kind == 0) return 0;
  const int nb = blocks_for(h->n, kBlock);
  k_external_begin<<<1, 32, 0, s>>>(h->a);
  k_external<kBlock><<<nb, kBlock, 0, s>>>(h->a, h->box, h->ext, h->n);
  k_external_done<<<1, 32, 0, s>>>(h->a, h->ext, nb);
  return 3;
}

int4 *fix_buffer(mdg_handle *h, int k) { return k ? h->a.qfix2 : h->a.qfix; }

// Dynamic shared memory of every staged force instantiation.
template <int MODE>
cudaError_t set_stage_smem_mode(int bytes) {
  cudaError_t e = cudaFuncSetAttribute(k_force_fp32_staged<kForceBlock, MODE, 0>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_force_fp32_staged<kForceBlock, MODE, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_force_fp32_staged<kForceBlock, MODE, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             bytes);
  return e;
}

cudaError_t set_stage_smem(int atoms) {
  const int bytes = atoms * (int)sizeof(int4);
  cudaError_t e = set_stage_smem_mode<kKick>(bytes);
  if (e == cudaSuccess) e = set_stage_smem_mode<kKickNoseHoover>(bytes);
  if (e == cudaSuccess) e = set_stage_smem_mode<kKickLangevin>(bytes);
  if (e == cudaSuccess) e = set_stage_smem_mode<kForceOut>(bytes);
  return e;
}

// The FP32-mixed force pass with TPA lanes per atom (drift as below).
// Blocks hold kForceBlock atoms whatever TPA is, so the Nose-Hoover kinetic
// energy partials cover the same atoms as k_zeta expects.
template <int MODE, int TPA>
void launch_fp32(mdg_handle *h, cudaStream_t s, const Thermo &th, int drift, const int4 *qf, int4 *qf_next) {
  constexpr int kThreads = kForceBlock * TPA;
  const int n = h->n;
  if (n == 0) return;
  const int nb = blocks_for(n, kForceBlock);
  if (drift == 2)
    k_force_fp32<kThreads, MODE, 2, TPA><<<nb, kThreads, 0, s>>>(h->a, h->box, n, th, qf, qf_next);
  else if (drift)
    k_force_fp32<kThreads, MODE, 1, TPA><<<nb, kThreads, 0, s>>>(h->a, h->box, n, th, qf, nullptr);
  else
    k_force_fp32<kThreads, MODE, 0, TPA><<<nb, kThreads, 0, s>>>(h->a, h->box, n, th, qf, nullptr);
}

// drift: 1 also applies the second half drift in the same pass, 2 the whole
// fused NVE step reading qf and packing into qf_next (FP32-mixed only);
// returns false when the caller still has to launch the second drift.
template <int MODE>
bool launch_force_mode(mdg_handle *h, cudaStream_t s, const Thermo &th, int drift = 0, const int4 *qf = nullptr,
                       int4 *qf_next = nullptr) {
  const int n = h->n;
  const int nb = blocks_for(n, kForceBlock);
  if (!qf) qf = h->a.qfix;
  if (h->prm.precision == MDG_FP32_MIXED && h->a.stage_cap > 0) {
    const size_t smem = (size_t)h->a.stage_cap * sizeof(int4);
    if (drift == 2)
      k_force_fp32_staged<kForceBlock, MODE, 2><<<nb, kForceBlock, smem, s>>>(h->a, h->box, n, th, qf, qf_next);
    else if (drift)
      k_force_fp32_staged<kForceBlock, MODE, 1><<<nb, kForceBlock, smem, s>>>(h->a, h->box, n, th, qf, nullptr);
    else
      k_force_fp32_staged<kForceBlock, MODE, 0><<<nb, kForceBlock, smem, s>>>(h->a, h->box, n, th, qf, nullptr);
    return drift != 0;
  }
  if (h->prm.precision == MDG_FP32_MIXED) {
    const int tpa = h->tpa > 0 ? h->tpa : 1;
    if (tpa == 4) launch_fp32<MODE, 4>(h, s, th, drift, qf, qf_next);
    else if (tpa == 2) launch_fp32<MODE, 2>(h, s, th, drift, qf, qf_next);
    else launch_fp32<MODE, 1>(h, s, th, drift, qf, qf_next);
    return drift != 0;
  }
  k_force_fp64<kForceBlock, MODE><<<nb, kForceBlock, 0, s>>>(h->a, h->box, n, th);
  return false;
}

Thermo thermo_of(const mdg_handle *h) {
  Thermo th{};
  th.gamma = h->prm.heatbath_gamma;
  th.noise_sd = std::sqrt(2.0 * h->prm.heatbath_gamma * h->prm.aimed_temperature / h->prm.time_step);
  th.seed = h->prm.seed;
  return th;
}

void launch_drift(mdg_handle *h, cudaStream_t s, bool pack_fix, int track_vmax) {
  const int nb = blocks_for(h->n, kBlock);
  if (pack_fix)
    k_drift<kBlock, true><<<nb, kBlock, 0, s>>>(h->a, h->box, h->n, track_vmax);
  else
    k_drift<kBlock, false><<<nb, kBlock, 0, s>>>(h->a, h->box, h->n, track_vmax);
}

// Everything of MDManager::Calculate after the rebuild decision; returns the
// number of kernels launched.  ev_start/ev_stop bracket the force kernel.
// parity: the fixed-point buffer the fused NVE step reads (it writes the
// other one).
int launch_step_tail(mdg_handle *h, cudaStream_t s, cudaEvent_t ev_start, cudaEvent_t ev_stop,
                     bool capture, int parity) {
  const bool fix = h->prm.precision == MDG_FP32_MIXED;
  const Thermo th = thermo_of(h);
  const int n = h->n;
  int launches = 0;
  auto rec = [&](cudaEvent_t e) {
    if (!e) return;
    if (capture) cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
    else cudaEventRecord(e, s);
  };
  if (fused_step(h)) {
    // one pass: drift, kick, drift, pack and the step counter
    rec(ev_start);
    launch_force_mode<kKick>(h, s, th, 2, fix_buffer(h, parity), fix_buffer(h, 1 - parity));
    rec(ev_stop);
    return 1;
  }
  launch_drift(h, s, fix, 0);
  launches++;
  if (h->prm.thermostat == MDG_NOSE_HOOVER) {
    const int nbk = blocks_for(n, kBlock);
    k_ke_partial<kBlock><<<nbk, kBlock, 0, s>>>(h->a, n);
    k_zeta<1024><<<1, 1024, 0, s>>>(h->a, h->box, nbk, n, h->prm.aimed_temperature, h->prm.heatbath_tau);
    rec(ev_start);
    // the second drift does not read zeta, so it may precede the zeta update
    const bool drifted = launch_force_mode<kKickNoseHoover>(h, s, th, 1);
    rec(ev_stop);
    k_zeta<1024><<<1, 1024, 0, s>>>(h->a, h->box, blocks_for(n, kForceBlock), n,
                                     h->prm.aimed_temperature, h->prm.heatbath_tau);
    launches += 4;
    if (!drifted) {
      launch_drift(h, s, false, 1);
      launches++;
    }
  } else if (h->prm.thermostat == MDG_LANGEVIN) {
    rec(ev_start);
    launch_force_mode<kKickLangevin>(h, s, th);
    rec(ev_stop);
    launches += 1;
  } else {
    rec(ev_start);
    const bool drifted = launch_force_mode<kKick>(h, s, th, 1);
    rec(ev_stop);
    launches += 1;
    if (!drifted) {
      launch_drift(h, s, false, 1);
      launches++;
    }
  }
  k_step_done<<<1, 32, 0, s>>>(h->a, h->box);
  return launches + 1 + launch_external(h, s);
}

// ---------------------------------------------------------- graph capture
struct Capture {
  cudaStream_t s;
  cudaGraph_t g;
  std::vector<cudaGraphNode_t> deps;
};

cudaError_t begin_capture(Capture &c) {
  return cudaStreamBeginCaptureToGraph(c.s, c.g, c.deps.empty() ? nullptr : c.deps.data(), nullptr,
                                       c.deps.size(), cudaStreamCaptureModeThreadLocal);
}

cudaError_t end_capture(Capture &c) {
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t *d = nullptr;
  size_t nd = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(c.s, &cs, nullptr, nullptr, &d, &nd);
  if (e != cudaSuccess) return e;
  std::vector<cudaGraphNode_t> frontier(d, d + nd);
  cudaGraph_t out = nullptr;
  e = cudaStreamEndCapture(c.s, &out);
  if (e != cudaSuccess) return e;
  if (!frontier.empty()) c.deps = frontier;
  return cudaSuccess;
}

// Appends an IF node on `h_cond` after the current frontier; returns its body.
cudaError_t add_if(Capture &c, cudaGraphConditionalHandle hc, cudaGraph_t *body) {
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = hc;
  p.conditional.type = cudaGraphCondTypeIf;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  cudaError_t e = cudaGraphAddNode(&node, c.g, c.deps.empty() ? nullptr : c.deps.data(),
                                   c.deps.size(), &p);
  if (e != cudaSuccess) return e;
  *body = p.conditional.phGraph_out[0];
  c.deps.assign(1, node);
  return cudaSuccess;
}

mdg_status build_graph(mdg_handle *h) {
  destroy_graph(h);
  cudaGraph_t g;
  CUDA_TRY(h, cudaGraphCreate(&g, 0));
  if (h->timing) {
    h->ev.resize(2 * kStepsPerGraph);
    for (auto &e : h->ev) CUDA_TRY(h, cudaEventCreate(&e));
  }
  Capture c{h->cap_stream, g, {}};
  int kernels = 0;
  for (int s = 0; s < kStepsPerGraph; s++) {
    cudaGraphConditionalHandle hd, hb;
    CUDA_TRY(h, cudaGraphConditionalHandleCreate(&hd, g, 0, cudaGraphCondAssignDefault));
    CUDA_TRY(h, cudaGraphConditionalHandleCreate(&hb, g, 0, cudaGraphCondAssignDefault));
    CUDA_TRY(h, begin_capture(c));
    k_expiry<<<1, 32, 0, c.s>>>(h->a, h->box, hd, hb, 1, h->d_flags);
    CUDA_TRY(h, end_capture(c));
    cudaGraph_t body;
    CUDA_TRY(h, add_if(c, hd, &body));
    {
      Capture bc{h->cap_stream, body, {}};
      CUDA_TRY(h, begin_capture(bc));
      launch_disp(h, bc.s, step_lag(h));
      k_decide<<<1, 32, 0, bc.s>>>(h->a, hb, 1, h->d_flags);
      CUDA_TRY(h, end_capture(bc));
    }
    CUDA_TRY(h, add_if(c, hb, &body));
    {
      Capture bc{h->cap_stream, body, {}};
      CUDA_TRY(h, begin_capture(bc));
      launch_build(h, bc.s, fused_step(h) ? fix_buffer(h, s & 1) : nullptr);
      CUDA_TRY(h, end_capture(bc));
    }
    CUDA_TRY(h, begin_capture(c));
    kernels += 1 + launch_step_tail(h, c.s, h->timing ? h->ev[2 * s] : nullptr,
                                    h->timing ? h->ev[2 * s + 1] : nullptr, true, s & 1);
    CUDA_TRY(h, end_capture(c));
  }
  cudaError_t e = cudaGraphInstantiate(&h->exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(h, MDG_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  h->graph_kernel_count = kernels;
  h->graph_dirty = false;
  return MDG_OK;
}

// One step with host-side decisions (used for partial chunks and by the
// fine-grained entry points).
mdg_status step_eager(mdg_handle *h) {
  int flags[2] = {0, 0};
  k_expiry<<<1, 32, 0, h->stream>>>(h->a, h->box, 0, 0, 0, h->d_flags);
  CUDA_TRY(h, cudaMemcpyAsync(flags, h->d_flags, sizeof flags, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  h->kernel_launches++;
  if (flags[0]) {
    launch_disp(h, h->stream, step_lag(h));
    k_decide<<<1, 32, 0, h->stream>>>(h->a, 0, 0, h->d_flags);
    CUDA_TRY(h, cudaMemcpyAsync(flags, h->d_flags, sizeof flags, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->kernel_launches += 4;
  }
  const int parity = h->fix_buf > 0 ? 1 : 0;
  if (flags[1]) {
    launch_build(h, h->stream, fused_step(h) ? fix_buffer(h, parity) : nullptr);
    h->kernel_launches += build_kernels(h);
  }
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (h->timing) {
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
  }
  h->kernel_launches += launch_step_tail(h, h->stream, e0, e1, false, parity);
  if (fused_step(h)) h->fix_buf = 1 - parity;
  CUDA_TRY(h, cudaGetLastError());
  if (h->timing) {
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    h->force_ms += ms;
    h->force_launches++;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  return MDG_OK;
}

mdg_status check_ready(mdg_handle *h) {
  if (!h) return MDG_ERR_INVALID_ARGUMENT;
  if (!h->state_set) return fail(h, MDG_ERR_STATE, "no state uploaded (mdg_set_state)");
  return MDG_OK;
}

// Builds the list now if it is stale (forces / observers need a valid list).
mdg_status ensure_list(mdg_handle *h) {
  Status st;
  mdg_status r = read_status(h, &st);
  if (r) return r;
  if (st.error) return translate_device_error(h, st);
  if (!st.list_stale) return MDG_OK;
  h->fix_buf = -1;  // the rebuild renumbers the atoms
  for (int attempt = 0; attempt < 4; attempt++) {
    launch_build(h, h->stream);
    h->kernel_launches += build_kernels(h);
    CUDA_TRY(h, cudaGetLastError());
    r = read_status(h, &st);
    if (r) return r;
    if (!(st.error & kErrCapacity)) break;
    // grow the rows and build again
    r = alloc_neighbors(h, (int)(st.max_row * 1.25) + 8);
    if (r) return r;
    const int zero = 0, one = 1;
    CUDA_TRY(h, cudaMemcpyAsync(&h->a.st->error, &zero, sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(&h->a.st->list_stale, &one, sizeof(int), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  }
  if (st.error) return translate_device_error(h, st);
  return MDG_OK;
}

// ------------------------------------------------------------ autotuner
// The lanes per atom of the FP32-mixed force pass (1, 2, 4) and the atoms
// per block of the list build (64, 128, 256), chosen by timing each
// candidate a few times on the handle's own state once its list is built,
// and remembered per device and problem shape (atoms, cells, precision)
// for the rest of the process.  The force candidates run force-only (the
// forces go to scratch, the state is untouched); the build candidates
// rebuild the same rows from the same cell order, and a last build with the
// chosen block leaves the list counters as a normal build does.
std::mutex g_tune_mutex;
std::map<std::tuple<int, int, int, int>, std::tuple<int, int, int>> g_tuned;

template <typename F>
float time_launches(cudaStream_t s, F launch, int reps) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float ms = -1.f;
  if (cudaEventCreate(&e0) != cudaSuccess) return ms;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return ms;
  }
  launch();  // warm-up
  cudaEventRecord(e0, s);
  for (int k = 0; k < reps; k++) launch();
  cudaEventRecord(e1, s);
  if (cudaEventSynchronize(e1) == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms;
}

static __global__ void k_list_counters_reset(Arrays a) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    a.st->max_row = 0;
    a.st->list_entries = 0;
  }
}

mdg_status autotune(mdg_handle *h) {
  const bool fp32 = h->prm.precision == MDG_FP32_MIXED;
  if (!fp32 && h->tpa == 0) h->tpa = 1;            // the FP64 pass has one lane per atom
  if (h->a.stage_cap > 0) {  // stage rows per 128 atoms, one lane per atom
    if (h->build_block == 0) h->build_block = kForceBlock;
    if (h->build_tpa == 0) h->build_tpa = 1;
  }
  if (h->tpa > 0 && h->build_block > 0 && h->build_tpa > 0) return MDG_OK;
  const auto key = std::make_tuple(h->prm.device, h->n, h->ncell, h->prm.precision);
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tuned.find(key);
    if (it != g_tuned.end()) {
      if (h->tpa == 0) h->tpa = std::get<0>(it->second);
      if (h->build_block == 0) h->build_block = std::get<1>(it->second);
      if (h->build_tpa == 0) h->build_tpa = std::get<2>(it->second);
      destroy_graph(h);
      return MDG_OK;
    }
  }
  // the tuner needs a list; a handle whose list is stale (no build since its
  // state was set: the reference's uninitialised PairList, which rebuilds at
  // the first step without spending the skin budget) gets its status back
  // afterwards, so that the first step behaves the same whether the shapes
  // were timed, cached or pinned
  Status before;
  mdg_status r = read_status(h, &before);
  if (r) return r;
  if ((r = ensure_list(h))) return r;
  cudaStream_t s = h->stream;
  const int n = h->n;
  int tpa = h->tpa, bb = h->build_block;
  if (tpa == 0) {
    k_pack_fix<kBlock><<<blocks_for(n, kBlock), kBlock, 0, s>>>(h->a, h->box, n);
    h->fix_buf = -1;  // the copy the fused step reads is repacked before the next step
    const Thermo th = thermo_of(h);
    float best = 0.f;
    const int cand[3] = {1, 2, 4};
    for (int c : cand) {
      const float ms = time_launches(s, [&]() {
        if (c == 4) launch_fp32<kForceOut, 4>(h, s, th, 0, h->a.qfix, nullptr);
        else if (c == 2) launch_fp32<kForceOut, 2>(h, s, th, 0, h->a.qfix, nullptr);
        else launch_fp32<kForceOut, 1>(h, s, th, 0, h->a.qfix, nullptr);
      }, 5);
      if (ms < 0.f) return fail(h, MDG_ERR_CUDA, "autotune: force timing failed");
      if (tpa == 0 || ms < best) {
        best = ms;
        tpa = c;
      }
    }
  }
  int bl = h->build_tpa;
  if (bb == 0 || bl == 0) {
    float best = -1.f;
    int bb_best = 0, bl_best = 0;
    const int blocks[3] = {64, 128, 256}, lanes[4] = {1, 2, 4, 8};
    for (int cb : blocks) {
      if (bb != 0 && cb != bb) continue;
      for (int cl : lanes) {
        if (bl != 0 && cl != bl) continue;
        const float ms = time_launches(s, [&]() { launch_list_build(h, s, cb, cl); }, 3);
        if (ms < 0.f) return fail(h, MDG_ERR_CUDA, "autotune: build timing failed");
        if (best < 0.f || ms < best) {
          best = ms;
          bb_best = cb;
          bl_best = cl;
        }
      }
    }
    bb = bb_best;
    bl = bl_best;
    k_list_counters_reset<<<1, 32, 0, s>>>(h->a);
    launch_list_build(h, s, bb, bl);
  }
  CUDA_TRY(h, cudaGetLastError());
  Status st;
  if ((r = read_status(h, &st))) return r;
  if (st.error) return translate_device_error(h, st);
  if (before.list_stale && !before.error) {
    CUDA_TRY(h, cudaMemcpyAsync(h->a.st, &before, sizeof(Status), cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  }
  h->tpa = tpa;
  h->build_block = bb;
  h->build_tpa = bl;
  destroy_graph(h);
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_tuned[key] = std::make_tuple(tpa, bb, bl);
  return MDG_OK;
}

// ------------------------------------------------------- persistent steps
// Blocks of the persistent pass for this handle: enough for every atom's
// lanes, at most what the device keeps resident at once (a cooperative
// launch needs all of them resident); 0 if the kernel cannot be resident.
template <int TPA>
int persistent_grid_of(mdg_handle *h) {
  int per_sm = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_nve_persistent<kPersistBlock, TPA>, kPersistBlock, 0) !=
          cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->prm.device) != cudaSuccess)
    return 0;
  const long long need = ((long long)h->n * TPA + kPersistBlock - 1) / kPersistBlock;
  return (int)std::min<long long>(need, (long long)per_sm * sms);
}

// Lanes per atom of the persistent pass.  Its steps end in a grid barrier
// whose cost grows with the block count, so it takes fewer lanes than the
// graph path's tuned force pass: one per atom from 16,384 atoms (measured
// on the 32,000-atom liquid: 31 us per step with one lane, 35-40 with two),
// more for smaller systems.  Every lane count gives the same forces.
int persistent_tpa(const mdg_handle *h) { return h->n >= 16384 ? 1 : (h->n >= 8192 ? 2 : 4); }

int persistent_grid(mdg_handle *h) {
  if (h->persist_grid < 0) {
    const int tpa = persistent_tpa(h);
    h->persist_grid = tpa == 4 ? persistent_grid_of<4>(h) : (tpa == 2 ? persistent_grid_of<2>(h) : persistent_grid_of<1>(h));
  }
  return h->persist_grid;
}

// Whether mdg_calculate runs the persistent pass: asked for, or (auto) when
// one wave of resident blocks covers every atom's lanes.
bool use_persistent(mdg_handle *h) {
  // the staged force pass (stage_atoms) runs as graph steps: the persistent
  // pass gathers from global memory
  if (!fused_step(h) || h->prm.step_mode == MDG_STEPS_GRAPHS || h->a.stage_cap > 0) return false;
  const int tpa = persistent_tpa(h);
  const int g = persistent_grid(h);
  if (g <= 0) return false;
  if (h->prm.step_mode == MDG_STEPS_PERSISTENT) return true;
  return (long long)g * kPersistBlock >= (long long)h->n * tpa;
}

// One persistent launch, queued (no wait): it takes steps until one needs a
// rebuild or the step count reaches Status::target_steps.
template <int TPA>
mdg_status enqueue_persistent_tpa(mdg_handle *h) {
  const int grid = persistent_grid(h);
  if (grid <= 0) return fail(h, MDG_ERR_CUDA, "persistent pass: no resident grid");
  CUDA_TRY(h, cudaMemsetAsync(h->d_bar, 0, sizeof(GridBarrier), h->stream));
  int n = h->n;
  int4 *q0 = h->a.qfix, *q1 = h->a.qfix2;
  double lag = step_lag(h);  // the ghost copies' age at a step's displacement check
  void *args[] = {&h->a, &h->box, &n, &q0, &q1, &lag, &h->d_bar};
  CUDA_TRY(h, cudaLaunchCooperativeKernel((const void *)k_nve_persistent<kPersistBlock, TPA>, dim3(grid),
                                          dim3(kPersistBlock), args, 0, h->stream));
  h->kernel_launches++;
  return MDG_OK;
}

mdg_status enqueue_persistent(mdg_handle *h) {
  const int tpa = persistent_tpa(h);
  return tpa == 4 ? enqueue_persistent_tpa<4>(h) : (tpa == 2 ? enqueue_persistent_tpa<2>(h) : enqueue_persistent_tpa<1>(h));
}

// The guarded rebuild step of the persistent pipeline (k_rebuild_guard):
// rebuild with buffer 0 packed, the fused step from buffer 0, parity 1.
mdg_status build_rebuild_graph(mdg_handle *h) {
  if (h->rebuild_exec) cudaGraphExecDestroy(h->rebuild_exec);
  h->rebuild_exec = nullptr;
  cudaGraph_t g;
  CUDA_TRY(h, cudaGraphCreate(&g, 0));
  Capture c{h->cap_stream, g, {}};
  cudaGraphConditionalHandle hr;
  CUDA_TRY(h, cudaGraphConditionalHandleCreate(&hr, g, 0, cudaGraphCondAssignDefault));
  CUDA_TRY(h, begin_capture(c));
  k_rebuild_guard<<<1, 32, 0, c.s>>>(h->a, h->box, hr);
  CUDA_TRY(h, end_capture(c));
  cudaGraph_t body;
  CUDA_TRY(h, add_if(c, hr, &body));
  {
    Capture bc{h->cap_stream, body, {}};
    CUDA_TRY(h, begin_capture(bc));
    launch_build(h, bc.s, h->a.qfix);
    launch_force_mode<kKick>(h, bc.s, thermo_of(h), 2, h->a.qfix, h->a.qfix2);
    k_set_parity<<<1, 32, 0, bc.s>>>(h->a, 1);
    CUDA_TRY(h, end_capture(bc));
  }
  cudaError_t e = cudaGraphInstantiate(&h->rebuild_exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return fail(h, MDG_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  h->rebuild_dirty = false;
  return MDG_OK;
}

// Steps up to `target` through the persistent pipeline: pairs of (persistent
// launch, rebuild step) queued back to back without waiting -- each launch
// stops where a step needs a rebuild, the rebuild step takes that step, and
// both stop at the target, so queued pairs beyond it do nothing -- then one
// wait and a status read per batch of pairs.  *st returns the final status.
mdg_status run_persistent(mdg_handle *h, long long target, Status *st) {
  mdg_status r;
  if (h->fix_buf < 0) {
    k_pack_half<kBlock><<<blocks_for(h->n, kBlock), kBlock, 0, h->stream>>>(h->a, h->box, h->n, h->a.qfix);
    h->kernel_launches++;
    h->fix_buf = 0;
  }
  if (h->rebuild_dirty || !h->rebuild_exec) {
    if ((r = build_rebuild_graph(h))) return r;
  }
  k_set_target<<<1, 32, 0, h->stream>>>(h->a, target, h->fix_buf > 0 ? 1 : 0);
  long long steps = st->steps;
  while (steps < target) {
    const long long left = target - steps;
    const int pairs = (int)std::min<long long>(64, (long long)std::ceil(left / h->steps_per_cycle) + 1);
    for (int k = 0; k < pairs; k++) {
      if ((r = enqueue_persistent(h))) return r;
      CUDA_TRY(h, cudaGraphLaunch(h->rebuild_exec, h->stream));
      h->kernel_launches += 2;
    }
    const long long rebuilds = st->rebuilds;
    if ((r = read_status(h, st))) return r;
    // each launch pair ends with a rebuild, except the last: pairs that did
    // work = rebuilds + 1
    if (st->steps > steps) h->steps_per_cycle = std::max(1.0, (double)(st->steps - steps) / (st->rebuilds - rebuilds + 1));
    if (st->error || st->steps == steps) break;
    steps = st->steps;
  }
  h->fix_buf = st->fix_parity;
  h->persistent_steps = st->persistent_steps;
  return MDG_OK;
}

}  // namespace

// ================================================================== C ABI
extern "C" {

void mdg_default_params(mdg_params *p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->capacity = 1000000;
  p->L[0] = p->L[1] = p->L[2] = 10.0;
  p->cutoff = 3.0;             // CUTOFF_LENGTH, include/mdconfig.h:31
  p->buffer_length = 0.3;      // src/simulationinfo.cc:6
  p->time_step = 0.001;        // src/simulationinfo.cc:9
  p->precision = MDG_FP64;
  p->thermostat = MDG_NVE;
  p->aimed_temperature = 1.0;  // src/simulationinfo.cc:11
  p->heatbath_tau = 0.1;       // src/simulationinfo.cc:13
  p->heatbath_gamma = 0.1;     // src/simulationinfo.cc:14
  p->seed = 0;
  p->check_list_length = 500;  // src/simulationinfo.cc:28
  p->max_neighbors = 0;
  p->device = 0;
  p->stream = nullptr;
  p->stage_atoms = 0;
  p->threads_per_atom = 0;        // timed at the first step
  p->build_block = 0;             // timed at the first step
  p->build_threads_per_atom = 0;  // timed at the first step
  p->step_mode = MDG_STEPS_AUTO;
}

mdg_status mdg_create(const mdg_params *prm, mdg_handle **out) {
  if (!prm || !out) return MDG_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (prm->capacity < 1 || prm->cutoff <= 0.0 || prm->buffer_length < 0.0 || prm->time_step <= 0.0 ||
      prm->check_list_length < 1 || (prm->precision != MDG_FP64 && prm->precision != MDG_FP32_MIXED) ||
      prm->thermostat < MDG_NVE || prm->thermostat > MDG_LANGEVIN || prm->stage_atoms < -1 ||
      prm->stage_atoms > kStageMax || prm->stage_wait_cycles < 0 ||
      (prm->threads_per_atom != 0 && prm->threads_per_atom != 1 && prm->threads_per_atom != 2 &&
       prm->threads_per_atom != 4) ||
      (prm->build_block != 0 && prm->build_block != 64 && prm->build_block != 128 && prm->build_block != 256) ||
      (prm->build_threads_per_atom != 0 && prm->build_threads_per_atom != 1 && prm->build_threads_per_atom != 2 &&
       prm->build_threads_per_atom != 4 && prm->build_threads_per_atom != 8) ||
      prm->step_mode < MDG_STEPS_AUTO || prm->step_mode > MDG_STEPS_PERSISTENT)
    return MDG_ERR_INVALID_ARGUMENT;
  for (int d = 0; d < 3; d++)
    if (!(prm->L[d] > 0.0) || !std::isfinite(prm->L[d])) return MDG_ERR_INVALID_ARGUMENT;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MDG_ERR_NO_DEVICE;
  if (prm->device < 0 || prm->device >= ndev) return MDG_ERR_INVALID_ARGUMENT;

  mdg_handle *h = new mdg_handle();
  h->prm = *prm;
  Box &b = h->box;
  const double SL = prm->cutoff + prm->buffer_length;  // src/simulationinfo.cc:6-7
  if (!box_geometry(b, prm->L, SL)) {
    delete h;
    return MDG_ERR_BOX_TOO_SMALL;
  }
  if (!cells_packable(b)) {
    delete h;
    return MDG_ERR_INVALID_ARGUMENT;
  }
  b.rc2 = prm->cutoff * prm->cutoff;
  b.rc = prm->cutoff;
  {  // Variables::Variables, src/variables.cc:21-27
    const double s2 = 1.0 / (prm->cutoff * prm->cutoff);
    const double s6 = s2 * s2 * s2, s8 = s6 * s2, s12 = s6 * s6, s14 = s12 * s2;
    b.c2 = 6.0 * s14 - 3.0 * s8;
    b.c0 = -s12 + s6 - b.c2 / s2;
  }
  b.dt = prm->time_step;
  b.buffer_length = prm->buffer_length;
  b.rc2f = (float)b.rc2;
  b.c2x8f = (float)(b.c2 * 8.0);
  b.check_list_length = prm->check_list_length;
  b.stage_wait = prm->stage_wait_cycles > 0 ? prm->stage_wait_cycles : kStageWaitCycles;
  h->ncell = b.ncell;
  h->cell_cap = b.ncell;
  h->cap = prm->capacity;
  h->tpa = prm->threads_per_atom;
  h->build_block = prm->build_block;
  h->build_tpa = prm->build_threads_per_atom;

  cudaError_t e = cudaSetDevice(prm->device);
  if (e == cudaSuccess) {
    if (prm->stream) {
      h->stream = (cudaStream_t)prm->stream;
    } else {
      e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
      h->own_stream = true;
    }
  }
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->cap_stream, cudaStreamNonBlocking);
  Arrays &a = h->a;
  const int cap = h->cap;
  a.stride = (cap + 31) / 32 * 32;
  a.maxnb = 0;
  h->partial_cap = (size_t)blocks_for(cap, kForceBlock) * 3 + 64;
  if (e == cudaSuccess) e = dalloc(&a.q, cap);
  if (e == cudaSuccess) e = dalloc(&a.v, cap);
  if (e == cudaSuccess) e = dalloc(&a.q_old, cap);
  if (e == cudaSuccess) e = dalloc(&a.qfix, cap);
  if (e == cudaSuccess) e = dalloc(&a.qfix2, cap);
  if (e == cudaSuccess) e = dalloc(&a.qloc, cap);
  if (e == cudaSuccess) e = dalloc(&a.cxyz, cap);
  if (e == cudaSuccess) e = dalloc(&a.xsub, trim_table_size(b));
  if (e == cudaSuccess) e = dalloc(&a.ids, cap);
  if (e == cudaSuccess) e = dalloc(&a.type, cap);
  if (e == cudaSuccess) e = dalloc(&a.cell, cap);
  if (e == cudaSuccess) e = dalloc(&a.nnbr, cap);
  if (e == cudaSuccess) e = dalloc(&a.cell_count, b.ncell);
  if (e == cudaSuccess) e = dalloc(&a.cell_start, b.ncell + 1);
  if (e == cudaSuccess) e = dalloc(&a.slot, cap);
  if (e == cudaSuccess) e = dalloc(&a.perm, cap);
  if (e == cudaSuccess) e = dalloc(&a.perm2, cap);
  if (e == cudaSuccess) e = dalloc(&a.q_tmp, cap);
  if (e == cudaSuccess) e = dalloc(&a.disp2, cap);
  if (e == cudaSuccess) e = dalloc(&a.v_tmp, cap);
  if (e == cudaSuccess) e = dalloc(&a.v_lag, cap);
  if (e == cudaSuccess) e = dalloc(&a.ids_tmp, cap);
  if (e == cudaSuccess) e = dalloc(&a.type_tmp, cap);
  if (e == cudaSuccess) e = dalloc(&a.cell_tmp, cap);
  if (e == cudaSuccess) e = dalloc(&a.mult, cap);
  if (e == cudaSuccess) e = dalloc(&a.cand, prm->check_list_length);
  if (e == cudaSuccess) e = dalloc(&a.partials, h->partial_cap);
  if (e == cudaSuccess) e = dalloc(&a.st, 1);
  if (e == cudaSuccess) e = dalloc(&h->d_flags, 4);
  if (e == cudaSuccess) e = dalloc(&h->d_sums, 8);
  if (e == cudaSuccess) e = dalloc(&h->d_tiles, (size_t)blocks_for(h->ncell, kScanBlock) + 1);
  if (e == cudaSuccess) e = dalloc(&h->d_bar, 1);
  if (e == cudaSuccess) e = dalloc(&h->d_pout, 4);
  if (prm->precision == MDG_FP32_MIXED && prm->stage_atoms != 0) {
    a.stage_cap = prm->stage_atoms < 0 ? kStageDefault : prm->stage_atoms;
    const int nblk = blocks_for(cap, kStageBlock);
    if (e == cudaSuccess) e = dalloc(&a.stage_rng, (size_t)nblk * kStageRanges);
    if (e == cudaSuccess) e = dalloc(&a.stage_n, nblk);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.stage_n, 0xff, sizeof(int) * nblk, h->stream);  // -1: no plan
    if (e == cudaSuccess) e = set_stage_smem(a.stage_cap);
  }
  if (e == cudaSuccess) e = cudaMemsetAsync(a.st, 0, sizeof(Status), h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    free_arrays(a);
    delete h;
    return MDG_ERR_CUDA;
  }
  if (prm->max_neighbors > 0) {
    mdg_status r = alloc_neighbors(h, prm->max_neighbors);
    if (r) {
      free_arrays(a);
      delete h;
      return r;
    }
  }
  *out = h;
  return MDG_OK;
}

mdg_status mdg_destroy(mdg_handle *h) {
  if (!h) return MDG_ERR_INVALID_ARGUMENT;
  if (h->writer.joinable()) h->writer.join();
  cudaSetDevice(h->prm.device);
  if (h->snap_q) cudaFreeHost(h->snap_q);
  if (h->snap_v) cudaFreeHost(h->snap_v);
  if (h->snap_t) cudaFreeHost(h->snap_t);
  if (h->snap_done) cudaEventDestroy(h->snap_done);
  if (h->stream) cudaStreamSynchronize(h->stream);
  destroy_graph(h);
  free_arrays(h->a);
  if (h->d_flags) cudaFree(h->d_flags);
  if (h->d_sums) cudaFree(h->d_sums);
  if (h->d_tiles) cudaFree(h->d_tiles);
  if (h->d_bar) cudaFree(h->d_bar);
  if (h->d_pout) cudaFree(h->d_pout);
  if (h->cap_stream) cudaStreamDestroy(h->cap_stream);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return MDG_OK;
}

mdg_status mdg_set_state(mdg_handle *h, const double *q4, const double *v4, const int *type, int n) {
  if (!h || n < 0 || (n > 0 && (!q4 || !v4))) return MDG_ERR_INVALID_ARGUMENT;
  if (n > h->cap) return fail(h, MDG_ERR_CAPACITY, "more atoms than the handle's capacity");
  h->fix_buf = -1;
  CUDA_TRY(h, cudaSetDevice(h->prm.device));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (n > 0) {
    CUDA_TRY(h, cudaMemcpyAsync(h->a.q, q4, sizeof(double4) * n, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->a.v, v4, sizeof(double4) * n, cudaMemcpyHostToDevice, h->stream));
    // upload indices made on the device; types copied from the caller's
    // array (0 without one)
    k_upload_ids<kBlock><<<blocks_for(n, kBlock), kBlock, 0, h->stream>>>(h->a, n);
    if (type) CUDA_TRY(h, cudaMemcpyAsync(h->a.type, type, sizeof(int) * n, cudaMemcpyHostToDevice, h->stream));
    else CUDA_TRY(h, cudaMemsetAsync(h->a.type, 0, sizeof(int) * n, h->stream));
    if (h->prm.max_neighbors <= 0 && (!h->a.nbr || n != h->n)) {
      mdg_status r = alloc_neighbors(h, estimate_max_neighbors(h, q4, n));
      if (r) return r;
    }
  } else if (!h->a.nbr) {
    mdg_status r = alloc_neighbors(h, 8);
    if (r) return r;
  }
  // fresh bookkeeping; keep counters of steps / rebuilds / time / zeta
  Status st;
  mdg_status r = read_status(h, &st);
  if (r) return r;
  st.error = 0;
  st.list_stale = 1;
  st.vmax2_bits = 0;
  st.vlag_set = 0;
  st.budget = h->prm.buffer_length;
  CUDA_TRY(h, cudaMemcpyAsync(h->a.st, &st, sizeof(Status), cudaMemcpyHostToDevice, h->stream));
  if (n > 0) k_vmax<kBlock><<<blocks_for(n, kBlock), kBlock, 0, h->stream>>>(h->a, n);
  CUDA_TRY(h, cudaGetLastError());
  if (n != h->n) {
    h->graph_dirty = h->rebuild_dirty = true;
    h->persist_grid = -1;
  }
  h->n = n;
  h->obs_lag = 0.0;
  int dev_error = 0;
  CUDA_TRY(h, cudaMemcpyAsync(&dev_error, &h->a.st->error, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (dev_error) {
    h->state_set = false;
    const int zero = 0;
    CUDA_TRY(h, cudaMemcpy(&h->a.st->error, &zero, sizeof(int), cudaMemcpyHostToDevice));
    return fail(h, MDG_ERR_NONFINITE, "non-finite value in the uploaded state");
  }
  h->state_set = true;
  return MDG_OK;
}

mdg_status mdg_get_state(mdg_handle *h, double *q4, double *v4, int *type, int n) {
  mdg_status r = check_ready(h);
  if (r) return r;
  if (n != h->n) return fail(h, MDG_ERR_INVALID_ARGUMENT, "n differs from the handle's atom count");
  if (n == 0) return MDG_OK;
  if (q4) CUDA_TRY(h, cudaMemcpyAsync(q4, h->a.q, sizeof(double4) * n, cudaMemcpyDeviceToHost, h->stream));
  if (v4) CUDA_TRY(h, cudaMemcpyAsync(v4, h->a.v, sizeof(double4) * n, cudaMemcpyDeviceToHost, h->stream));
  if (type) CUDA_TRY(h, cudaMemcpyAsync(type, h->a.type, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return MDG_OK;
}

mdg_status mdg_set_velocities(mdg_handle *h, const double *v4, int n) {
  mdg_status r = check_ready(h);
  if (r) return r;
  if (n != h->n || (n > 0 && !v4)) return fail(h, MDG_ERR_INVALID_ARGUMENT, "n differs from the handle's atom count");
  if (n == 0) return MDG_OK;
  CUDA_TRY(h, cudaSetDevice(h->prm.device));
  h->fix_buf = -1;  // the fused step's packed first-drift copy used the old velocities
  if (h->obs_lag > 0.0) {
    // the reference's ghost copies date from half a step back: their
    // reconstruction needs the velocities of the last drift, kept once
    // (a second call before the next step keeps the first copy)
    Status st;
    if ((r = read_status(h, &st))) return r;
    if (!st.vlag_set) {
      const int one = 1;
      CUDA_TRY(h, cudaMemcpyAsync(h->a.v_lag, h->a.v, sizeof(double4) * n, cudaMemcpyDeviceToDevice, h->stream));
      CUDA_TRY(h, cudaMemcpyAsync(&h->a.st->vlag_set, &one, sizeof one, cudaMemcpyHostToDevice, h->stream));
    }
  }
  const unsigned long long zero = 0ull;
  CUDA_TRY(h, cudaMemcpyAsync(h->a.v, v4, sizeof(double4) * n, cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaMemcpyAsync(&h->a.st->vmax2_bits, &zero, sizeof zero, cudaMemcpyHostToDevice, h->stream));
  k_vmax<kBlock><<<blocks_for(n, kBlock), kBlock, 0, h->stream>>>(h->a, n);
  CUDA_TRY(h, cudaGetLastError());
  Status st;
  if ((r = read_status(h, &st))) return r;
  if (st.error) return translate_device_error(h, st);
  return MDG_OK;
}

mdg_status mdg_get_ids(mdg_handle *h, int *ids, int n) {
  mdg_status r = check_ready(h);
  if (r) return r;
  if (n != h->n || (n > 0 && !ids)) return fail(h, MDG_ERR_INVALID_ARGUMENT, "bad ids buffer");
  if (n == 0) return MDG_OK;
  CUDA_TRY(h, cudaMemcpyAsync(ids, h->a.ids, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return MDG_OK;
}

mdg_status mdg_particle_number(mdg_handle *h, int *n) {
  if (!h || !n) return MDG_ERR_INVALID_ARGUMENT;
  *n = h->n;
  return MDG_OK;
}

mdg_status mdg_make_pairlist(mdg_handle *h) {
  mdg_status r = check_ready(h);
  if (r) return r;
  h->obs_lag = 0.0;
  if (h->n == 0) return MDG_OK;
  const int one = 1;
  CUDA_TRY(h, cudaMemcpyAsync(&h->a.st->list_stale, &one, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  return ensure_list(h);
}

mdg_status mdg_check_expired(mdg_handle *h, int *expired) {
  mdg_status r = check_ready(h);
  if (r) return r;
  if (!expired) return MDG_ERR_INVALID_ARGUMENT;
  *expired = 0;
  if (h->n == 0) return MDG_OK;
  k_vmax<kBlock><<<blocks_for(h->n, kBlock), kBlock, 0, h->stream>>>(h->a, h->n);
  int flags[2] = {0, 0};
  k_expiry<<<1, 32, 0, h->stream>>>(h->a, h->box, 0, 0, 0, h->d_flags);
  CUDA_TRY(h, cudaMemcpyAsync(flags, h->d_flags, sizeof flags, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (flags[0]) launch_disp(h, h->stream, h->obs_lag);
  k_decide<<<1, 32, 0, h->stream>>>(h->a, 0, 0, h->d_flags);
  CUDA_TRY(h, cudaMemcpyAsync(flags, h->d_flags, sizeof flags, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  Status st;
  r = read_status(h, &st);
  if (r) return r;
  if (st.error) return translate_device_error(h, st);
  *expired = flags[1];
  return MDG_OK;
}

mdg_status mdg_update_position_half(mdg_handle *h) {
  mdg_status r = check_ready(h);
  if (r) return r;
  h->fix_buf = -1;  // q, v or the fixed-point copy change outside the fused step
  h->obs_lag = 0.0;
  if (h->n == 0) return MDG_OK;
  launch_drift(h, h->stream, h->prm.precision == MDG_FP32_MIXED, 0);
  CUDA_TRY(h, cudaGetLastError());
  return MDG_OK;
}

mdg_status mdg_calculate_force(mdg_handle *h) {
  mdg_status r = check_ready(h);
  if (r) return r;
  h->fix_buf = -1;  // q, v or the fixed-point copy change outside the fused step
  h->obs_lag = 0.0;
  if (h->n == 0) return MDG_OK;
  if ((r = ensure_list(h))) return r;
  if (h->prm.precision == MDG_FP32_MIXED)
    k_pack_fix<kBlock><<<blocks_for(h->n, kBlock), kBlock, 0, h->stream>>>(h->a, h->box, h->n);
  launch_force_mode<kKick>(h, h->stream, thermo_of(h));
  CUDA_TRY(h, cudaGetLastError());
  return MDG_OK;
}

mdg_status mdg_heatbath_zeta(mdg_handle *h, double t) {
  mdg_status r = check_ready(h);
  if (r) return r;
  Status st;
  if ((r = read_status(h, &st))) return r;
  const double dt2 = h->prm.time_step * 0.5;
  const double tau = h->prm.heatbath_tau;
  st.zeta += (t - h->prm.aimed_temperature) / (tau * tau) * dt2;
  CUDA_TRY(h, cudaMemcpyAsync(&h->a.st->zeta, &st.zeta, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return MDG_OK;
}

mdg_status mdg_heatbath_momenta(mdg_handle *h) {
  mdg_status r = check_ready(h);
  if (r) return r;
  h->fix_buf = -1;  // q, v or the fixed-point copy change outside the fused step
  h->obs_lag = 0.0;
  if (h->n == 0) return MDG_OK;
  k_scale_v<kBlock><<<blocks_for(h->n, kBlock), kBlock, 0, h->stream>>>(h->a, h->n, h->prm.time_step * 0.5);
  CUDA_TRY(h, cudaGetLastError());
  return MDG_OK;
}

mdg_status mdg_langevin(mdg_handle *h) {
  mdg_status r = check_ready(h);
  if (r) return r;
  h->fix_buf = -1;  // q, v or the fixed-point copy change outside the fused step
  h->obs_lag = 0.0;
  if (h->n == 0) return MDG_OK;
  k_langevin<kBlock><<<blocks_for(h->n, kBlock), kBlock, 0, h->stream>>>(h->a, h->box, h->n, thermo_of(h));
  CUDA_TRY(h, cudaGetLastError());
  return MDG_OK;
}

mdg_status mdg_set_control(mdg_handle *h, int thermostat, double aimed_temperature, double heatbath_tau,
                           double heatbath_gamma) {
  if (!h || thermostat < MDG_NVE || thermostat > MDG_LANGEVIN) return MDG_ERR_INVALID_ARGUMENT;
  if (thermostat != h->prm.thermostat || aimed_temperature != h->prm.aimed_temperature ||
      heatbath_tau != h->prm.heatbath_tau || heatbath_gamma != h->prm.heatbath_gamma) {
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
    h->prm.thermostat = thermostat;
    h->prm.aimed_temperature = aimed_temperature;
    h->prm.heatbath_tau = heatbath_tau;
    h->prm.heatbath_gamma = heatbath_gamma;
    h->fix_buf = -1;
    destroy_graph(h);
  }
  return MDG_OK;
}

mdg_status mdg_set_external(mdg_handle *h, const mdg_external *x) {
  if (!h) return MDG_ERR_INVALID_ARGUMENT;
  External e{};
  if (x && x->kind != MDG_EXTERNAL_NONE) {
    if (x->kind < MDG_EXTERNAL_GRAVITY || x->kind > MDG_EXTERNAL_SHELL || x->axis < 0 || x->axis > 2 ||
        !std::isfinite(x->time_step) || !std::isfinite(x->strength) || !std::isfinite(x->position) ||
        !std::isfinite(x->velocity) || !std::isfinite(x->radius))
      return MDG_ERR_INVALID_ARGUMENT;
    e.kind = x->kind;
    e.axis = x->axis;
    e.strength = x->strength;
    e.dt = x->time_step;
    e.velocity = x->velocity;
    for (int d = 0; d < 3; d++) e.center[d] = x->center[d];
    e.radius = x->radius;
  }
  CUDA_TRY(h, cudaSetDevice(h->prm.device));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  const double pos = x ? x->position : 0.0, zero = 0.0;
  CUDA_TRY(h, cudaMemcpyAsync(&h->a.st->ext_position, &pos, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaMemcpyAsync(&h->a.st->ext_impulse, &zero, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  h->ext = e;
  h->fix_buf = -1;
  destroy_graph(h);
  return MDG_OK;
}

mdg_status mdg_change_scale(mdg_handle *h, double alpha) {
  mdg_status r = check_ready(h);
  if (r) return r;
  if (!(alpha > 0.0) || !std::isfinite(alpha)) return MDG_ERR_INVALID_ARGUMENT;
  CUDA_TRY(h, cudaSetDevice(h->prm.device));
  double L[3];
  for (int d = 0; d < 3; d++) L[d] = h->prm.L[d] * alpha;  // MDManager::ChangeScale, src/mdmanager.cc:573-585
  Box nb = h->box;
  if (!box_geometry(nb, L, h->box.sl)) return fail(h, MDG_ERR_BOX_TOO_SMALL, "scaled box below 3 cells per axis");
  if (!cells_packable(nb)) return fail(h, MDG_ERR_INVALID_ARGUMENT, "scaled box above 2047 x 2047 x 1023 cells");
  // the reference builds the list (wrapping the atoms into the box) before
  // scaling and again after it
  const int one = 1;
  CUDA_TRY(h, cudaMemcpyAsync(&h->a.st->list_stale, &one, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  if ((r = ensure_list(h))) return r;
  if (h->n > 0)
    k_scale_positions<kBlock><<<blocks_for(h->n, kBlock), kBlock, 0, h->stream>>>(h->a, h->n, alpha);
  CUDA_TRY(h, cudaGetLastError());
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  if (nb.ncell > h->cell_cap) {
    cudaFree(h->a.cell_count);
    cudaFree(h->a.cell_start);
    cudaFree(h->a.xsub);
    cudaFree(h->d_tiles);
    h->a.cell_count = h->a.cell_start = h->a.xsub = h->d_tiles = nullptr;
    CUDA_TRY(h, dalloc(&h->a.cell_count, nb.ncell));
    CUDA_TRY(h, dalloc(&h->a.cell_start, nb.ncell + 1));
    CUDA_TRY(h, dalloc(&h->a.xsub, trim_table_size(nb)));
    CUDA_TRY(h, dalloc(&h->d_tiles, (size_t)blocks_for(nb.ncell, kScanBlock) + 1));
    h->cell_cap = nb.ncell;
  }
  h->box = nb;
  h->ncell = nb.ncell;
  for (int d = 0; d < 3; d++) h->prm.L[d] = L[d];
  h->fix_buf = -1;
  destroy_graph(h);
  CUDA_TRY(h, cudaMemcpyAsync(&h->a.st->list_stale, &one, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  return ensure_list(h);
}

mdg_status mdg_density_grid(mdg_handle *h, double grid_size, unsigned char *out, int64_t cap, int dims[3]) {
  mdg_status r = check_ready(h);
  if (r) return r;
  if (!(grid_size > 0.0) || !dims || cap < 0) return MDG_ERR_INVALID_ARGUMENT;
  // BubbleHist (src/cavitation.cc:38-58): grid counts int(w / g + 0.5) per
  // axis, one grid edge from the x width
  int g[3];
  for (int d = 0; d < 3; d++) {
    g[d] = (int)(h->prm.L[d] / grid_size + 0.5);
    if (g[d] < 1) return MDG_ERR_INVALID_ARGUMENT;
    dims[d] = g[d];
  }
  const int64_t cells = (int64_t)g[0] * g[1] * g[2];
  if (!out || cap < cells) return cells <= cap ? MDG_ERR_INVALID_ARGUMENT : fail(h, MDG_ERR_CAPACITY, "grid larger than cap");
  const double gs = h->prm.L[0] / (double)g[0];
  CUDA_TRY(h, cudaSetDevice(h->prm.device));
  int *count = nullptr;
  CUDA_TRY(h, dalloc(&count, (size_t)cells));
  cudaError_t e = cudaMemsetAsync(count, 0, sizeof(int) * cells, h->stream);
  if (e == cudaSuccess && h->n > 0)
    k_density<kBlock><<<blocks_for(h->n, kBlock), kBlock, 0, h->stream>>>(h->a, h->box, h->n, 1.0 / gs, g[0], g[1],
                                                                          g[2], count);
  std::vector<int> hc((size_t)cells);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(hc.data(), count, sizeof(int) * cells, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  cudaFree(count);
  if (e != cudaSuccess) return fail(h, MDG_ERR_CUDA, std::string("density grid: ") + cudaGetErrorString(e));
  for (int64_t k = 0; k < cells; k++) out[k] = (unsigned char)(hc[(size_t)k] & 255);
  return MDG_OK;
}

mdg_status mdg_external_state(mdg_handle *h, double *position, double *impulse) {
  if (!h) return MDG_ERR_INVALID_ARGUMENT;
  Status st;
  mdg_status r = read_status(h, &st);
  if (r) return r;
  if (position) *position = st.ext_position;
  if (impulse) *impulse = st.ext_impulse;
  return MDG_OK;
}

mdg_status mdg_get_list(mdg_handle *h, int *row_len, int *partners, int64_t cap, int64_t *count) {
  mdg_status r = check_ready(h);
  if (r) return r;
  if (!count || cap < 0) return MDG_ERR_INVALID_ARGUMENT;
  *count = 0;
  if (h->n == 0) return MDG_OK;
  if ((r = ensure_list(h))) return r;
  const int n = h->n, stride = h->a.stride;
  std::vector<int> nn(n);
  CUDA_TRY(h, cudaMemcpyAsync(nn.data(), h->a.nnbr, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  const int maxrow = *std::max_element(nn.begin(), nn.end());
  std::vector<int> tab((size_t)maxrow * stride);
  if (maxrow > 0)
    CUDA_TRY(h, cudaMemcpy(tab.data(), h->a.nbr, sizeof(int) * (size_t)maxrow * stride, cudaMemcpyDeviceToHost));
  int64_t c = 0;
  for (int i = 0; i < n; i++) {
    if (row_len) row_len[i] = nn[i];
    for (int k = 0; k < nn[i]; k++) {
      if (c < cap && partners) partners[c] = tab[(size_t)k * stride + i];
      c++;
    }
  }
  *count = c;
  return MDG_OK;
}

mdg_status mdg_get_zeta(mdg_handle *h, double *zeta) {
  if (!h || !zeta) return MDG_ERR_INVALID_ARGUMENT;
  Status st;
  mdg_status r = read_status(h, &st);
  if (r) return r;
  *zeta = st.zeta;
  return MDG_OK;
}

mdg_status mdg_set_zeta(mdg_handle *h, double zeta) {
  if (!h) return MDG_ERR_INVALID_ARGUMENT;
  CUDA_TRY(h, cudaMemcpyAsync(&h->a.st->zeta, &zeta, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return MDG_OK;
}

mdg_status mdg_calculate(mdg_handle *h, int nsteps) {
  mdg_status r = check_ready(h);
  if (r) return r;
  if (nsteps < 0) return MDG_ERR_INVALID_ARGUMENT;
  if (h->n == 0 || nsteps == 0) return MDG_OK;
  CUDA_TRY(h, cudaSetDevice(h->prm.device));
  if ((r = autotune(h))) return r;
  Status st;
  if ((r = read_status(h, &st))) return r;
  if (st.error) return translate_device_error(h, st);
  long long target = st.steps + nsteps;
  for (int attempt = 0; attempt < 8; attempt++) {
    long long left = target - st.steps;
    if (left <= 0) break;
    if (fused_step(h) && h->fix_buf != 0) {
      // the graph's first step reads buffer 0
      k_pack_half<kBlock><<<blocks_for(h->n, kBlock), kBlock, 0, h->stream>>>(h->a, h->box, h->n, h->a.qfix);
      h->kernel_launches++;
      h->fix_buf = 0;
    }
    if (h->use_graphs && use_persistent(h)) {
      if ((r = run_persistent(h, target, &st))) return r;
      left = st.error ? 0 : target - st.steps;  // an error is handled below
    }
    if (h->use_graphs && left >= kStepsPerGraph && h->graph_dirty) {
      if ((r = build_graph(h))) return r;
    }
    while (h->use_graphs && left >= kStepsPerGraph) {
      CUDA_TRY(h, cudaGraphLaunch(h->exec, h->stream));
      h->kernel_launches += h->graph_kernel_count;
      left -= kStepsPerGraph;
      if (h->timing) {
        CUDA_TRY(h, cudaStreamSynchronize(h->stream));
        for (int s = 0; s < kStepsPerGraph; s++) {
          float ms = 0.f;
          CUDA_TRY(h, cudaEventElapsedTime(&ms, h->ev[2 * s], h->ev[2 * s + 1]));
          h->force_ms += ms;
          h->force_launches++;
        }
      }
    }
    while (left > 0) {
      if ((r = step_eager(h))) return r;
      left--;
    }
    if ((r = read_status(h, &st))) return r;
    if (st.error == kErrCapacity) {
      // a rebuild overflowed a neighbour row: grow, rebuild, redo the rest
      if ((r = alloc_neighbors(h, (int)(st.max_row * 1.25) + 8))) return r;
      st.error = 0;
      st.list_stale = 1;
      CUDA_TRY(h, cudaMemcpyAsync(h->a.st, &st, sizeof(Status), cudaMemcpyHostToDevice, h->stream));
      continue;
    }
    if (st.error) return translate_device_error(h, st);
  }
  if (st.steps < target) return fail(h, MDG_ERR_CAPACITY, "could not complete the steps");
  // after a full step the reference's ghost copies date from the first half
  // drift; the Langevin branch has no second drift (src/mdmanager.cc:289-315)
  h->obs_lag = h->prm.thermostat == MDG_LANGEVIN ? 0.0 : 0.5 * h->prm.time_step;
  return MDG_OK;
}

mdg_status mdg_forces(mdg_handle *h, double *f4) {
  mdg_status r = check_ready(h);
  if (r) return r;
  h->fix_buf = -1;  // q, v or the fixed-point copy change outside the fused step
  if (h->n == 0) return MDG_OK;
  if (!f4) return MDG_ERR_INVALID_ARGUMENT;
  if ((r = ensure_list(h))) return r;
  if (h->prm.precision == MDG_FP32_MIXED)
    k_pack_fix<kBlock><<<blocks_for(h->n, kBlock), kBlock, 0, h->stream>>>(h->a, h->box, h->n);
  launch_force_mode<kForceOut>(h, h->stream, thermo_of(h));
  CUDA_TRY(h, cudaGetLastError());
  CUDA_TRY(h, cudaMemcpyAsync(f4, h->a.v_tmp, sizeof(double4) * h->n, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  return MDG_OK;
}

mdg_status mdg_observe(mdg_handle *h, double *ke, double *pe, double *virial) {
  mdg_status r = check_ready(h);
  if (r) return r;
  double out[3] = {0.0, 0.0, 0.0};
  if (h->n > 0) {
    if ((r = ensure_list(h))) return r;
    const int nb = blocks_for(h->n, kBlock);
    const double lag = h->observer_mode ? h->obs_lag : 0.0;
    k_observe<kBlock><<<nb, kBlock, 0, h->stream>>>(h->a, h->box, h->n, lag);
    k_final_sum<256, 3><<<1, 256, 0, h->stream>>>(h->a.partials, nb, h->d_sums);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaMemcpyAsync(out, h->d_sums, sizeof out, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  }
  if (ke) *ke = out[0];
  if (pe) *pe = out[1];
  if (virial) *virial = out[2] / 3.0;
  return MDG_OK;
}

mdg_status mdg_pair_counts(mdg_handle *h, int64_t *within_cutoff, int64_t *list_entries) {
  mdg_status r = check_ready(h);
  if (r) return r;
  unsigned long long c[2] = {0ull, 0ull};
  if (h->n > 0) {
    if ((r = ensure_list(h))) return r;
    unsigned long long *d = reinterpret_cast<unsigned long long *>(h->d_sums);
    CUDA_TRY(h, cudaMemsetAsync(d, 0, 2 * sizeof(unsigned long long), h->stream));
    k_count_pairs<kBlock><<<blocks_for(h->n, kBlock), kBlock, 0, h->stream>>>(h->a, h->box, h->n, d);
    CUDA_TRY(h, cudaGetLastError());
    CUDA_TRY(h, cudaMemcpyAsync(c, d, sizeof c, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  }
  if (within_cutoff) *within_cutoff = (int64_t)c[0];
  if (list_entries) *list_entries = (int64_t)c[1];
  return MDG_OK;
}

mdg_status mdg_set_observer_mode(mdg_handle *h, int mode) {
  if (!h || (mode != MDG_OBSERVE_CURRENT && mode != MDG_OBSERVE_GHOST_LAG)) return MDG_ERR_INVALID_ARGUMENT;
  h->observer_mode = mode;
  return MDG_OK;
}

mdg_status mdg_get_pairs(mdg_handle *h, int *key, int *partner, int64_t cap, int64_t *count) {
  mdg_status r = check_ready(h);
  if (r) return r;
  if (!count || cap < 0) return MDG_ERR_INVALID_ARGUMENT;
  *count = 0;
  if (h->n == 0) return MDG_OK;
  if ((r = ensure_list(h))) return r;
  const int n = h->n, stride = h->a.stride;
  std::vector<int> nn(n), ids(n);
  CUDA_TRY(h, cudaMemcpyAsync(nn.data(), h->a.nnbr, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaMemcpyAsync(ids.data(), h->a.ids, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  const int maxrow = n > 0 ? *std::max_element(nn.begin(), nn.end()) : 0;
  std::vector<int> tab((size_t)maxrow * stride);
  if (maxrow > 0)
    CUDA_TRY(h, cudaMemcpy(tab.data(), h->a.nbr, sizeof(int) * (size_t)maxrow * stride, cudaMemcpyDeviceToHost));
  int64_t c = 0;
  for (int i = 0; i < n; i++) {
    for (int k = 0; k < nn[i]; k++) {
      if (c < cap && key && partner) {
        key[c] = ids[i];
        partner[c] = ids[tab[(size_t)k * stride + i]];
      }
      c++;
    }
  }
  *count = c;
  return MDG_OK;
}

mdg_status mdg_get_info(mdg_handle *h, mdg_info *info) {
  if (!h || !info) return MDG_ERR_INVALID_ARGUMENT;
  Status st;
  mdg_status r = read_status(h, &st);
  if (r) return r;
  info->n = h->n;
  for (int d = 0; d < 3; d++) info->ncell[d] = h->box.ms[d];
  info->max_neighbors = h->a.maxnb;
  info->max_row = st.max_row;
  info->list_entries = st.list_entries;
  info->steps = st.steps;
  info->rebuilds = st.rebuilds;
  info->displacement_checks = st.disp_checks;
  info->simulation_time = st.sim_time;
  info->buffer_left = st.budget;
  info->threads_per_atom = h->tpa;
  info->build_block = h->build_block;
  info->build_threads_per_atom = h->build_tpa;
  info->persistent_steps = h->persistent_steps;
  return MDG_OK;
}

void *mdg_stream(mdg_handle *h) { return h ? (void *)h->stream : nullptr; }

mdg_status mdg_set_graph_mode(mdg_handle *h, int use_graphs) {
  if (!h) return MDG_ERR_INVALID_ARGUMENT;
  h->use_graphs = use_graphs != 0;
  return MDG_OK;
}

mdg_status mdg_set_kernel_timing(mdg_handle *h, int on) {
  if (!h) return MDG_ERR_INVALID_ARGUMENT;
  if ((on != 0) != h->timing) {
    h->timing = on != 0;
    destroy_graph(h);
  }
  h->force_ms = 0.0;
  h->force_launches = 0;
  h->kernel_launches = 0;
  return MDG_OK;
}

mdg_status mdg_kernel_time(mdg_handle *h, double *force_ms, int64_t *force_launches,
                           int64_t *kernel_launches) {
  if (!h) return MDG_ERR_INVALID_ARGUMENT;
  if (force_ms) *force_ms = h->force_ms;
  if (force_launches) *force_launches = h->force_launches;
  if (kernel_launches) *kernel_launches = h->kernel_launches;
  return MDG_OK;
}

const char *mdg_last_error(mdg_handle *h) { return h ? h->err.c_str() : "null handle"; }

const char *mdg_status_string(mdg_status s) {
  switch (s) {
    case MDG_OK: return "ok";
    case MDG_ERR_INVALID_ARGUMENT: return "invalid argument";
    case MDG_ERR_CUDA: return "CUDA error";
    case MDG_ERR_CAPACITY: return "capacity exceeded";
    case MDG_ERR_TOO_FAST: return "too fast particle";
    case MDG_ERR_INVALID_POSITION: return "invalid position";
    case MDG_ERR_NONFINITE: return "non-finite state";
    case MDG_ERR_BOX_TOO_SMALL: return "box too small for the cell list";
    case MDG_ERR_TIMEOUT: return "device wait timed out";
    case MDG_ERR_STATE: return "call out of order";
    case MDG_ERR_NO_DEVICE: return "no CUDA device";
    case MDG_ERR_IO: return "file error";
  }
  return "unknown status";
}

const char *mdg_version(void) { return "mdacp_b200 0.1 (sm_100a)"; }

// ------------------------------------------------------ checkpoints
namespace {
struct CkptHeader {
  char magic[8];
  int version;
  int n;
  double L[3];
  double cutoff, buffer_length, time_step;
  int precision, thermostat;
  double aimed_temperature, heatbath_tau, heatbath_gamma;
  uint64_t seed;
  int check_list_length;
  int observer_mode;
  double obs_lag;
  Status st;
  External ext;
};
const char kCkptMagic[8] = {'M', 'D', 'G', 'C', 'K', 'P', 'T', '1'};
constexpr int kCkptVersion = 2;  // 2: Status::vlag_set, and v_lag after the arrays when it is set
}  // namespace

mdg_status mdg_save_checkpoint(mdg_handle *h, const char *path) {
  mdg_status r = check_ready(h);
  if (r) return r;
  if (!path) return MDG_ERR_INVALID_ARGUMENT;
  CUDA_TRY(h, cudaSetDevice(h->prm.device));
  CkptHeader hd{};
  memcpy(hd.magic, kCkptMagic, 8);
  hd.version = kCkptVersion;
  hd.n = h->n;
  for (int d = 0; d < 3; d++) hd.L[d] = h->prm.L[d];
  hd.cutoff = h->prm.cutoff;
  hd.buffer_length = h->prm.buffer_length;
  hd.time_step = h->prm.time_step;
  hd.precision = h->prm.precision;
  hd.thermostat = h->prm.thermostat;
  hd.aimed_temperature = h->prm.aimed_temperature;
  hd.heatbath_tau = h->prm.heatbath_tau;
  hd.heatbath_gamma = h->prm.heatbath_gamma;
  hd.seed = h->prm.seed;
  hd.check_list_length = h->prm.check_list_length;
  hd.observer_mode = h->observer_mode;
  hd.obs_lag = h->obs_lag;
  hd.ext = h->ext;
  if ((r = read_status(h, &hd.st))) return r;
  if (hd.st.error) return translate_device_error(h, hd.st);
  const int n = h->n;
  std::vector<double4> q(n), v(n), qo(n), vl(hd.st.vlag_set ? n : 0);
  std::vector<int> ids(n), ty(n);
  if (n > 0) {
    if (hd.st.vlag_set)
      CUDA_TRY(h, cudaMemcpyAsync(vl.data(), h->a.v_lag, sizeof(double4) * n, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(q.data(), h->a.q, sizeof(double4) * n, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(v.data(), h->a.v, sizeof(double4) * n, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(qo.data(), h->a.q_old, sizeof(double4) * n, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(ids.data(), h->a.ids, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(ty.data(), h->a.type, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  }
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) return fail(h, MDG_ERR_IO, std::string("cannot write ") + path);
  f.write((const char *)&hd, sizeof hd);
  f.write((const char *)q.data(), sizeof(double4) * n);
  f.write((const char *)v.data(), sizeof(double4) * n);
  f.write((const char *)qo.data(), sizeof(double4) * n);
  f.write((const char *)ids.data(), sizeof(int) * n);
  f.write((const char *)ty.data(), sizeof(int) * n);
  f.write((const char *)vl.data(), sizeof(double4) * vl.size());
  if (!f) return fail(h, MDG_ERR_IO, std::string("write failed: ") + path);
  return MDG_OK;
}

mdg_status mdg_load_checkpoint(mdg_handle *h, const char *path) {
  if (!h || !path) return MDG_ERR_INVALID_ARGUMENT;
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(h, MDG_ERR_IO, std::string("cannot read ") + path);
  CkptHeader hd{};
  f.read((char *)&hd, sizeof hd);
  if (!f || memcmp(hd.magic, kCkptMagic, 8) != 0 || hd.version != kCkptVersion || hd.n < 0)
    return fail(h, MDG_ERR_IO, std::string("not a checkpoint of this library: ") + path);
  for (int d = 0; d < 3; d++)
    if (hd.L[d] != h->prm.L[d]) return fail(h, MDG_ERR_INVALID_ARGUMENT, "checkpoint box differs from the handle's");
  if (hd.cutoff != h->prm.cutoff || hd.buffer_length != h->prm.buffer_length || hd.time_step != h->prm.time_step ||
      hd.precision != h->prm.precision || hd.seed != h->prm.seed ||
      hd.check_list_length != h->prm.check_list_length)
    return fail(h, MDG_ERR_INVALID_ARGUMENT, "checkpoint parameters differ from the handle's");
  const int n = hd.n;
  if (n > h->cap) return fail(h, MDG_ERR_CAPACITY, "checkpoint holds more atoms than the handle's capacity");
  std::vector<double4> q(n), v(n), qo(n), vl(hd.st.vlag_set ? n : 0);
  std::vector<int> ids(n), ty(n);
  f.read((char *)q.data(), sizeof(double4) * n);
  f.read((char *)v.data(), sizeof(double4) * n);
  f.read((char *)qo.data(), sizeof(double4) * n);
  f.read((char *)ids.data(), sizeof(int) * n);
  f.read((char *)ty.data(), sizeof(int) * n);
  f.read((char *)vl.data(), sizeof(double4) * vl.size());
  if (!f) return fail(h, MDG_ERR_IO, std::string("truncated checkpoint: ") + path);
  mdg_status r = mdg_set_control(h, hd.thermostat, hd.aimed_temperature, hd.heatbath_tau, hd.heatbath_gamma);
  if (r) return r;
  CUDA_TRY(h, cudaSetDevice(h->prm.device));
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  const bool stale = hd.st.list_stale != 0;
  if (n > 0) {
    // the list is rebuilt from the positions of the last build: slots come
    // back in the same order and the rows entry for entry
    if (h->prm.max_neighbors <= 0) {
      std::vector<double> q4((size_t)4 * n);
      for (int i = 0; i < n; i++) {
        const double4 &x = stale ? q[i] : qo[i];
        q4[4 * i] = x.x;
        q4[4 * i + 1] = x.y;
        q4[4 * i + 2] = x.z;
        q4[4 * i + 3] = 0.0;
      }
      if ((r = alloc_neighbors(h, estimate_max_neighbors(h, q4.data(), n)))) return r;
    }
    CUDA_TRY(h, cudaMemcpyAsync(h->a.q, stale ? q.data() : qo.data(), sizeof(double4) * n, cudaMemcpyHostToDevice,
                                h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->a.v, v.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->a.ids, ids.data(), sizeof(int) * n, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->a.type, ty.data(), sizeof(int) * n, cudaMemcpyHostToDevice, h->stream));
  }
  Status st = hd.st;
  st.error = 0;
  st.list_stale = 1;
  CUDA_TRY(h, cudaMemcpyAsync(h->a.st, &st, sizeof(Status), cudaMemcpyHostToDevice, h->stream));
  if (n != h->n) {
    h->graph_dirty = h->rebuild_dirty = true;
    h->persist_grid = -1;
  }
  h->n = n;
  h->state_set = true;
  h->fix_buf = -1;
  destroy_graph(h);
  if (n > 0 && !stale) {
    if ((r = ensure_list(h))) return r;
    CUDA_TRY(h, cudaMemcpyAsync(h->a.q, q.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->a.v, v.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, h->stream));
    Status built;
    if ((r = read_status(h, &built))) return r;
    st = hd.st;  // counters, budget, clocks as saved; list figures from the rebuild
    st.max_row = built.max_row;
    st.list_entries = built.list_entries;
    st.total_images = built.total_images;
    if (st.vlag_set)
      CUDA_TRY(h, cudaMemcpyAsync(h->a.v_lag, vl.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->a.st, &st, sizeof(Status), cudaMemcpyHostToDevice, h->stream));
  } else {
    st = hd.st;
    st.list_stale = 1;
    st.vlag_set = 0;  // the next step rebuilds: fresh ghost copies
    CUDA_TRY(h, cudaMemcpyAsync(h->a.st, &st, sizeof(Status), cudaMemcpyHostToDevice, h->stream));
  }
  CUDA_TRY(h, cudaStreamSynchronize(h->stream));
  h->ext = hd.ext;
  h->observer_mode = hd.observer_mode;
  h->obs_lag = hd.obs_lag;
  return MDG_OK;
}

// ------------------------------------------------------ snapshots
namespace {
// Joins the pending writer, if any; MDG_ERR_IO with its message if it failed.
mdg_status join_writer(mdg_handle *h) {
  if (h->writer.joinable()) h->writer.join();
  if (!h->writer_error.empty()) {
    const std::string msg = h->writer_error;
    h->writer_error.clear();
    return fail(h, MDG_ERR_IO, msg);
  }
  return MDG_OK;
}
}  // namespace

mdg_status mdg_snapshot_async(mdg_handle *h, const char *path, int format) {
  mdg_status r = check_ready(h);
  if (r) return r;
  if (!path || (format != MDG_SNAPSHOT_CDVIEW && format != MDG_SNAPSHOT_CONFIGURATION))
    return MDG_ERR_INVALID_ARGUMENT;
  // the previous file is finished (and its failure reported) before its
  // buffers are reused
  if ((r = join_writer(h))) return r;
  CUDA_TRY(h, cudaSetDevice(h->prm.device));
  const int n = h->n;
  if (n > h->snap_cap || !h->snap_q) {
    if (h->snap_q) cudaFreeHost(h->snap_q);
    if (h->snap_v) cudaFreeHost(h->snap_v);
    if (h->snap_t) cudaFreeHost(h->snap_t);
    h->snap_q = h->snap_v = nullptr;
    h->snap_t = nullptr;
    h->snap_cap = 0;
    const int cap = std::max(n, 1);
    CUDA_TRY(h, cudaHostAlloc((void **)&h->snap_q, sizeof(double4) * cap, cudaHostAllocDefault));
    CUDA_TRY(h, cudaHostAlloc((void **)&h->snap_v, sizeof(double4) * cap, cudaHostAllocDefault));
    CUDA_TRY(h, cudaHostAlloc((void **)&h->snap_t, sizeof(int) * cap, cudaHostAllocDefault));
    h->snap_cap = cap;
  }
  if (!h->snap_done) CUDA_TRY(h, cudaEventCreateWithFlags(&h->snap_done, cudaEventDisableTiming));
  if (n > 0) {
    CUDA_TRY(h, cudaMemcpyAsync(h->snap_q, h->a.q, sizeof(double4) * n, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->snap_v, h->a.v, sizeof(double4) * n, cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(h, cudaMemcpyAsync(h->snap_t, h->a.type, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
  }
  CUDA_TRY(h, cudaEventRecord(h->snap_done, h->stream));
  const std::string file(path);
  const int dev = h->prm.device;
  h->writer = std::thread([h, file, format, n, dev]() {
    const double4 *hq = h->snap_q, *hv = h->snap_v;
    const int *ht = h->snap_t;
    cudaSetDevice(dev);
    bool ok = cudaEventSynchronize(h->snap_done) == cudaSuccess;
    if (ok) {
      FILE *fp = fopen(file.c_str(), "w");
      ok = fp != nullptr;
      for (int i = 0; ok && i < n; i++) {
        // the reference streams doubles with the default ostream format (%g)
        if (format == MDG_SNAPSHOT_CDVIEW)
          ok = fprintf(fp, "0 %d %g %g %g %g %g %g\n", ht[i], hq[i].x, hq[i].y, hq[i].z, hv[i].x, hv[i].y,
                       hv[i].z) > 0;
        else
          ok = fprintf(fp, "%g %g %g %g %g %g\n", hq[i].x, hq[i].y, hq[i].z, hv[i].x, hv[i].y, hv[i].z) > 0;
      }
      if (fp && fclose(fp) != 0) ok = false;
    }
    // read by the joining thread only after join()
    if (!ok) h->writer_error = "snapshot not written: " + file;
  });
  return MDG_OK;
}

mdg_status mdg_snapshot_wait(mdg_handle *h) {
  if (!h) return MDG_ERR_INVALID_ARGUMENT;
  return join_writer(h);
}

}  // extern "C"
