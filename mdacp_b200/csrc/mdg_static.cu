// mdg_observe_static: the observer reduction (KE, PE, virial) for callers
// that cannot allocate device memory.
//
// Some callers own every byte of device memory themselves: a host MD code
// that hands this library slices of its own preallocated pools, a
// latency-critical loop that must not hit the implicit device
// synchronisation of cudaMalloc / cudaFree, or a sandboxed plugin whose host
// forbids new allocations.  They cannot create an mdg_handle (which
// allocates its buffers) but can still pass their own device arrays.  For
// them this entry point computes the same sums as mdg_observe while
// allocating nothing: its per-block partial sums live in the file-scope
// device array below (3 x 8192 doubles = 196,608 bytes), which every GPU that
// loads the library holds until the process exits.  It limits a call to
// 8192 blocks of 256 atoms, 2,097,152 atoms; larger inputs are refused with
// MDG_ERR_CAPACITY.
//
// The array's device address comes from cudaGetSymbolAddress with the
// call's device current.  A call on a stream that is not being captured
// looks it up again every time (cheap once the module is loaded), so a
// cudaDeviceReset, after which the module may load the array elsewhere, is
// harmless; a call made during a stream capture uses the address the last
// uncaptured call on that device found, so make one call on each device
// before capturing any.  Every call on a device shares the array and leaves
// its partial sums in it; each call writes every slot it later reads, so
// nothing needs clearing, but calls whose kernels overlap on the GPU
// (different streams, no ordering between them) race on it.
//
// The partner indices are the caller's: an index outside [0, n) is skipped
// (never read) and turns the result's potential energy into NaN, so a bad
// list shows up in the output rather than as a device fault.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "mdacp_b200.h"

namespace mdg {
namespace {

constexpr int kStaticBlock = 256;
constexpr int kStaticMaxBlocks = 8192;  // atoms <= 8192 * 256 = 2,097,152
constexpr int kStaticMaxDevices = 64;

// Shared by every call on a device; each call overwrites the slots it reads.
static __device__ __align__(256) double g_observe_scratch[3 * kStaticMaxBlocks];

std::mutex g_setup_mutex;
double *g_scratch_addr[kStaticMaxDevices];  // device address of g_observe_scratch, per device

// Box and potential constants of one call.
struct StaticBox {
  double L[3], hL[3];
  double rc2, c0, c2;
};

__device__ __forceinline__ double sadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ssub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double smul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double sdiv(double a, double b) { return __ddiv_rn(a, b); }

// The periodic image of x_j next to x_i, formed as the reference forms its
// ghost copies: x_j + diff with diff in {-L, 0, +L} (src/mdunit.cc:152-192).
__device__ __forceinline__ double simage(double xj, double xi, double L, double hL) {
  const double t = xj - xi;
  if (t > hL) return ssub(xj, L);
  if (t < -hL) return sadd(xj, L);
  return xj;
}

__device__ __forceinline__ double swarp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Per-atom sums over a CSR list, each pair term formed as the handle's
// observer forms it (the reference's PotentialEnergyObserver /
// VirialObserver expressions, src/observer.cc:17-79, every operation
// separately rounded); block partials in fixed order into scratch.
__global__ void __launch_bounds__(kStaticBlock)
    k_observe_csr_static(const double4 *q, const double4 *v, int n, const int *row_start, const int *partners,
                         StaticBox b, double *scratch) {
  const int i = blockIdx.x * kStaticBlock + threadIdx.x;
  double ke = 0.0, pe = 0.0, vir = 0.0;
  if (i < n) {
    const double4 vi = v[i];
    ke = sadd(sadd(smul(smul(0.5, vi.x), vi.x), smul(smul(0.5, vi.y), vi.y)), smul(smul(0.5, vi.z), vi.z));
    const double4 qi = q[i];
    for (int k = row_start[i]; k < row_start[i + 1]; k++) {
      const int j = partners[k];
      if ((unsigned)j >= (unsigned)n) {  // not an atom of this call: skipped, reported as NaN
        pe = __longlong_as_double(0x7ff8000000000000ll);
        continue;
      }
      const double4 qj = q[j];
      const double dx = ssub(qi.x, simage(qj.x, qi.x, b.L[0], b.hL[0]));
      const double dy = ssub(qi.y, simage(qj.y, qi.y, b.L[1], b.hL[1]));
      const double dz = ssub(qi.z, simage(qj.z, qi.z, b.L[2], b.hL[2]));
      const double r2 = sadd(sadd(smul(dx, dx), smul(dy, dy)), smul(dz, dz));
      if (r2 > b.rc2) continue;
      const double r4 = smul(r2, r2), r6 = smul(r4, r2), r8 = smul(r6, r2), r10 = smul(r8, r2),
                   r12 = smul(r10, r2);
      pe = sadd(pe, smul(4.0, sadd(sadd(ssub(sdiv(1.0, r12), sdiv(1.0, r6)), smul(b.c2, r2)), b.c0)));
      vir = sadd(vir, smul(sadd(sdiv(ssub(smul(24.0, r6), 48.0), smul(smul(r6, r6), r2)), b.c2 * 8.0), r2));
    }
  }
  __shared__ double sm[3][kStaticBlock / 32];
  const double part[3] = {ke, 0.5 * pe, 0.5 * vir};
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  for (int c = 0; c < 3; c++) {
    const double x = swarp_sum(part[c]);
    if (l == 0) sm[c][w] = x;
  }
  __syncthreads();
  if (w == 0) {
    for (int c = 0; c < 3; c++) {
      double x = (l < kStaticBlock / 32) ? sm[c][l] : 0.0;
      x = swarp_sum(x);
      if (l == 0) scratch[3 * blockIdx.x + c] = x;  // this block's three slots
    }
  }
}

// Fixed-order sum of the block partials into out = (KE, PE, virial / 3).
__global__ void __launch_bounds__(kStaticBlock) k_observe_static_final(const double *scratch, int nblocks,
                                                                       double *out) {
  __shared__ double sm[3][kStaticBlock];
  for (int c = 0; c < 3; c++) {
    double acc = 0.0;
    for (int blk = threadIdx.x; blk < nblocks; blk += kStaticBlock) acc += scratch[3 * blk + c];
    sm[c][threadIdx.x] = acc;
  }
  __syncthreads();
  for (int off = kStaticBlock / 2; off > 0; off >>= 1) {
    if (threadIdx.x < off)
      for (int c = 0; c < 3; c++) sm[c][threadIdx.x] += sm[c][threadIdx.x + off];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = sm[0][0];
    out[1] = sm[1][0];
    out[2] = sm[2][0] / 3.0;
  }
}

// Device address of the scratch array on the current device, with that
// device current.  Outside a stream capture it is looked up on every call
// (and kept); during a capture the kept value of the device is used.
mdg_status scratch_for_current_device(cudaStream_t s, double **out) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return MDG_ERR_NO_DEVICE;
  if (dev < 0 || dev >= kStaticMaxDevices) return MDG_ERR_INVALID_ARGUMENT;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(s, &cs);
  if (e != cudaSuccess) return MDG_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (cs == cudaStreamCaptureStatusNone) {
    void *addr = nullptr;
    e = cudaGetSymbolAddress(&addr, g_observe_scratch);
    if (e != cudaSuccess || !addr) return MDG_ERR_CUDA;
    g_scratch_addr[dev] = static_cast<double *>(addr);
  } else if (!g_scratch_addr[dev]) {
    return MDG_ERR_STATE;  // no uncaptured call on this device yet
  }
  *out = g_scratch_addr[dev];
  return MDG_OK;
}

}  // namespace
}  // namespace mdg

using mdg::kStaticBlock;
using mdg::StaticBox;
using mdg::kStaticMaxBlocks;

extern "C" mdg_status mdg_observe_static(const double *q4, const double *v4, int n, const int *row_start,
                                         const int *partners, const double L[3], double cutoff, double *out,
                                         void *stream) {
  if (n < 0 || !L || !out || !(cutoff > 0.0) || (n > 0 && (!q4 || !v4 || !row_start || !partners)))
    return MDG_ERR_INVALID_ARGUMENT;
  if (n > kStaticBlock * kStaticMaxBlocks)
    return MDG_ERR_CAPACITY;
  StaticBox b{};
  for (int d = 0; d < 3; d++) {
    if (!(L[d] > 0.0) || !std::isfinite(L[d]))
      return MDG_ERR_INVALID_ARGUMENT;
    b.L[d] = L[d];
    b.hL[d] = 0.5 * L[d];
  }
  b.rc2 = cutoff * cutoff;
  const double s2 = 1.0 / (cutoff * cutoff);  // Variables::Variables, src/variables.cc:21-27
  const double s6 = s2 * s2 * s2, s8 = s6 * s2, s12 = s6 * s6, s14 = s12 * s2;
  b.c2 = 6.0 * s14 - 3.0 * s8;
  b.c0 = -s12 + s6 - b.c2 / s2;
  // an error the caller's own earlier work left pending is theirs: report
  // it without clearing it and launch nothing
  if (cudaPeekAtLastError() != cudaSuccess) return MDG_ERR_CUDA;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double *scratch = nullptr;
  mdg_status r = mdg::scratch_for_current_device(s, &scratch);
  if (r) return r;
  const int nblocks = n > 0 ? (n + kStaticBlock - 1) / kStaticBlock : 1;
  mdg::k_observe_csr_static<<<nblocks, kStaticBlock, 0, s>>>(reinterpret_cast<const double4 *>(q4),
                                                        reinterpret_cast<const double4 *>(v4), n, row_start,
                                                        partners, b, scratch);
  mdg::k_observe_static_final<<<1, kStaticBlock, 0, s>>>(scratch, nblocks, out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return MDG_ERR_CUDA;
  return MDG_OK;
}
