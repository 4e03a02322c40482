// Differentiable LJ trajectories: the gradient of a trajectory loss with
// respect to the potential's epsilon and sigma and to the initial positions,
// by a hand-written adjoint (reverse) sweep over the drift-kick-drift steps.
//
// Model (FP64 throughout):
//   U(r) = epsilon * phi(r / sigma), phi(s) = 4 (s^-12 - s^-6 + C2 s^2 + C0)
//   for s <= s_c, 0 beyond: the reference's smoothed potential
//   (Variables::Variables, src/variables.cc:16-33) with the cut-off s_c in
//   units of sigma, so U and U' vanish at the cut-off.
//   Step (MDManager::Calculate, NVE, src/mdmanager.cc:153-186):
//     q_h = q + v dt/2;  v' = v + F(q_h) dt;  q' = q_h + v' dt/2.
//   Loss: L = 1/(T N) sum_{t=1..T} [ PE(q_t) + S(q_t) ], PE the pair energy
//   and S = sum over pairs of g((r - a)/w) g((b - r)/w), a smoothed count of
//   the pairs in the shell a < r < b (g the logistic function).
//
// Reverse sweep, per step, from the adjoints (lq, lv) of (q', v'):
//   lq += dL/dq'          (the loss term of this step)
//   lv' = lv + lq dt/2
//   u = lv' dt;  lq_h = lq - H(q_h) u;  dL/dtheta += u . dF/dtheta
//   lv = lv';  lq = lq_h;  lv += lq_h dt/2
// H(q_h) u is the Hessian-vector product of the pair energy, assembled pair
// by pair: (H u)_i = sum_j K_ij (u_i - u_j), K = U'' d d^T + U'/r (I - d d^T)
// with d the unit separation.  Positions and velocities are checkpointed every
// k steps in the forward pass; each k-step segment is recomputed forward
// (keeping q_h and v') before its reverse sweep.
//
// Pairs are found through a cell grid rebuilt for every evaluation (cells at
// least r_c = s_c sigma wide, >= 3 per axis, atoms in each cell ordered by
// index), so every sum is deterministic and no skin bookkeeping is needed.
// This component has no counterpart in the reference, which has no
// gradients.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "mdacp_b200.h"

namespace {

constexpr int kAB = 128;  // threads per block

struct Pot {
  double eps, sigma, rc2;       // energy scale, length scale, cut-off^2 (absolute)
  double c0, c2;                // smoothed-LJ constants in units of sigma
  double a, b, w;               // shell of the smoothed pair count
  // reciprocals and quotients of the above, formed once on the host
  double inv_sigma, inv_w, inv_eps, eps_sigma, eps_sigma2;  // 1/sigma, 1/w, 1/eps, eps/sigma, eps/sigma^2
};

struct Grid {
  int ms[3];
  double L[3], inv_cs[3], inv_L[3];
  const int *start;   // ncell + 1
  const int *perm;    // atoms in cell order
  const double4 *qs;  // their positions in the same order (made with the grid)
};

// phi(s) and its first two derivatives; one division (1/s).
__device__ __forceinline__ void phi_d(double s, const Pot &p, double &phi, double &d1, double &d2) {
  const double is = 1.0 / s;
  const double is2 = is * is;
  const double is6 = is2 * is2 * is2;
  const double is12 = is6 * is6;
  phi = 4.0 * (is12 - is6 + p.c2 * s * s + p.c0);
  d1 = 4.0 * (-12.0 * is12 + 6.0 * is6 + 2.0 * p.c2 * s * s) * is;
  d2 = 4.0 * (156.0 * is12 - 42.0 * is6 + 2.0 * p.c2 * s * s) * is2;
}

// U(r), U'(r), U''(r)
__device__ __forceinline__ void pair_u(double r, const Pot &p, double &u, double &u1, double &u2) {
  double f, f1, f2;
  phi_d(r * p.inv_sigma, p, f, f1, f2);
  u = p.eps * f;
  u1 = p.eps_sigma * f1;
  u2 = p.eps_sigma2 * f2;
}

__device__ __forceinline__ double logistic(double x) { return 1.0 / (1.0 + exp(-x)); }

// smoothed shell count of one pair and its derivative in r
__device__ __forceinline__ void shell(double r, const Pot &p, double &s, double &s1) {
  const double x1 = (r - p.a) * p.inv_w, x2 = (p.b - r) * p.inv_w;
  const double g1 = logistic(x1), g2 = logistic(x2);
  s = g1 * g2;
  s1 = (g1 * (1.0 - g1) * g2 - g1 * g2 * (1.0 - g2)) * p.inv_w;
}

__device__ __forceinline__ int cell_axis(double x, double L, double inv_cs, int ms) {
  x -= L * floor(x / L);
  int c = (int)(x * inv_cs);
  return c < 0 ? 0 : (c >= ms ? ms - 1 : c);
}

__device__ __forceinline__ int cell_of(const double4 &q, const Grid &g) {
  const int cx = cell_axis(q.x, g.L[0], g.inv_cs[0], g.ms[0]);
  const int cy = cell_axis(q.y, g.L[1], g.inv_cs[1], g.ms[1]);
  const int cz = cell_axis(q.z, g.L[2], g.inv_cs[2], g.ms[2]);
  return (cz * g.ms[1] + cy) * g.ms[0] + cx;
}

// Calls f(j, d, r) for every partner j != i with r < r_c, d = minimum image of
// q_i - q_j, over the 27 cells around i's, each in index order (partner
// positions read from the grid's cell-ordered copy).  TPA lanes
// share one atom: lane `sub` takes cells sub, sub + TPA, ... of the 27 (the
// caller combines the lanes' sums with group_sum).
template <int TPA, class F>
__device__ __forceinline__ void for_pairs(const double4 *q, const Grid &g, const Pot &p, int i, int sub, F f) {
  const double4 qi = q[i];
  const int cx = cell_axis(qi.x, g.L[0], g.inv_cs[0], g.ms[0]);
  const int cy = cell_axis(qi.y, g.L[1], g.inv_cs[1], g.ms[1]);
  const int cz = cell_axis(qi.z, g.L[2], g.inv_cs[2], g.ms[2]);
  for (int nbh = sub; nbh < 27; nbh += TPA) {
    const int z = (cz + nbh / 9 - 1 + g.ms[2]) % g.ms[2];
    const int y = (cy + (nbh / 3) % 3 - 1 + g.ms[1]) % g.ms[1];
    const int x = (cx + nbh % 3 - 1 + g.ms[0]) % g.ms[0];
    const int c = (z * g.ms[1] + y) * g.ms[0] + x;
    for (int k = g.start[c]; k < g.start[c + 1]; k++) {
      const int j = g.perm[k];
      if (j == i) continue;
      const double4 qj = g.qs[k];
      double d[3] = {qi.x - qj.x, qi.y - qj.y, qi.z - qj.z};
      for (int a = 0; a < 3; a++) d[a] -= g.L[a] * rint(d[a] * g.inv_L[a]);
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (r2 < p.rc2) f(j, d, sqrt(r2));
    }
  }
}

// Sum over the TPA lanes of one atom (fixed butterfly order); every lane of
// the group gets the total.
template <int TPA>
__device__ __forceinline__ double group_sum(double x) {
#pragma unroll
  for (int o = 1; o < TPA; o <<= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// Fixed-order block sum of NS values into part[blockIdx.x * NS + k].
template <int NS>
__device__ __forceinline__ void block_sums(double (&v)[NS], double *part) {
  __shared__ double sm[NS][kAB / 32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NS; k++) {
    double x = v[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (l == 0) sm[k][w] = x;
  }
  __syncthreads();
  if (threadIdx.x < NS) {
    double x = 0.0;
    for (int q = 0; q < kAB / 32; q++) x += sm[threadIdx.x][q];
    part[(size_t)blockIdx.x * NS + threadIdx.x] = x;
  }
}

// ------------------------------------------------------------------ cells
__global__ void a_count(const double4 *q, int n, Grid g, int *cell, int *count) {
  const int i = blockIdx.x * kAB + threadIdx.x;
  if (i >= n) return;
  const int c = cell_of(q[i], g);
  cell[i] = c;
  atomicAdd(&count[c], 1);
}

// exclusive scan of count into start (one block, ncell of any size)
__global__ void a_scan(const int *count, int *start, int ncell) {
  __shared__ int part[1024];
  const int t = threadIdx.x;
  const int chunk = (ncell + 1023) / 1024;
  const int beg = min(t * chunk, ncell), end = min(beg + chunk, ncell);
  int s = 0;
  for (int c = beg; c < end; c++) s += count[c];
  part[t] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int x = t >= o ? part[t - o] : 0;
    __syncthreads();
    part[t] += x;
    __syncthreads();
  }
  int run = part[t] - s;
  for (int c = beg; c < end; c++) {
    start[c] = run;
    run += count[c];
  }
  if (t == 1023) start[ncell] = part[t];
}

__global__ void a_fill(int n, const int *cell, const int *start, int *fill, int *perm) {
  const int i = blockIdx.x * kAB + threadIdx.x;
  if (i >= n) return;
  const int c = cell[i];
  perm[start[c] + atomicAdd(&fill[c], 1)] = i;
}

// Orders every cell by atom index, one warp per cell: each entry's new
// place is the count of smaller indices in the cell (indices are distinct).
// perm_in is the fill order, perm_out the sorted one.
__global__ void a_sort(int ncell, const int *start, const int *perm_in, int *perm_out) {
  const int c = (blockIdx.x * kAB + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= ncell) return;
  const int b = start[c], cnt = start[c + 1] - b;
  for (int base = 0; base < cnt; base += 32) {
    const int me = base + lane;
    const int key = me < cnt ? perm_in[b + me] : 0x7fffffff;
    int rank = 0;
    for (int ob = 0; ob < cnt; ob += 32) {
      const int okey = ob + lane < cnt ? perm_in[b + ob + lane] : 0x7fffffff;
      for (int k = 0; k < 32; k++) rank += (ob + k < cnt) && (__shfl_sync(0xffffffffu, okey, k) < key);
    }
    if (me < cnt) perm_out[b + rank] = key;
  }
}

// Positions in cell order for the pair kernels.
__global__ void a_gather(const double4 *x, const int *perm, double4 *xs, int n) {
  const int k = blockIdx.x * kAB + threadIdx.x;
  if (k < n) xs[k] = x[perm[k]];
}

// --------------------------------------------------------------- physics
template <int TPA>
__global__ void __launch_bounds__(kAB) a_force(const double4 *q, int n, Grid g, Pot p, double4 *f) {
  const int t = blockIdx.x * kAB + threadIdx.x;
  const int i = t / TPA, sub = t % TPA;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  if (i < n) {
    for_pairs<TPA>(q, g, p, i, sub, [&](int, const double *d, double r) {
      double u, u1, u2;
      pair_u(r, p, u, u1, u2);
      const double c = -u1 / r;
      fx += c * d[0];
      fy += c * d[1];
      fz += c * d[2];
    });
  }
  fx = group_sum<TPA>(fx);
  fy = group_sum<TPA>(fy);
  fz = group_sum<TPA>(fz);
  if (i < n && sub == 0) f[i] = make_double4(fx, fy, fz, 0.0);
}

// Loss terms at q: per-block sums of PE, S and dPE/dsigma (pairs counted from
// both ends, halved); with grad, dL_t/dq_i * scale added into lq.
template <int TPA>
__global__ void __launch_bounds__(kAB) a_loss(const double4 *q, int n, Grid g, Pot p, double *part, double4 *lq,
                                              double scale) {
  const int t = blockIdx.x * kAB + threadIdx.x;
  const int i = t / TPA, sub = t % TPA;
  double v[3] = {0.0, 0.0, 0.0};
  double gx = 0.0, gy = 0.0, gz = 0.0;
  if (i < n) {
    for_pairs<TPA>(q, g, p, i, sub, [&](int, const double *d, double r) {
      double u, u1, u2, s, s1;
      pair_u(r, p, u, u1, u2);
      shell(r, p, s, s1);
      v[0] += 0.5 * u;
      v[1] += 0.5 * s;
      v[2] += 0.5 * (-(r * p.inv_sigma) * u1);  // dU/dsigma at fixed r
      const double c = (u1 + s1) / r;
      gx += c * d[0];
      gy += c * d[1];
      gz += c * d[2];
    });
  }
  if (lq) {
    gx = group_sum<TPA>(gx);
    gy = group_sum<TPA>(gy);
    gz = group_sum<TPA>(gz);
    if (i < n && sub == 0) {
      double4 l = lq[i];
      l.x += scale * gx;
      l.y += scale * gy;
      l.z += scale * gz;
      lq[i] = l;
    }
  }
  block_sums<3>(v, part);
}

// w = H(q) u (pair energy Hessian times u); per-block sums of
// sum_i u_i . dF_i/d(eps, sigma).
template <int TPA>
__global__ void __launch_bounds__(kAB) a_hvp(const double4 *q, int n, Grid g, Pot p, const double4 *u, double4 *w,
                                             double *part) {
  const int t = blockIdx.x * kAB + threadIdx.x;
  const int i = t / TPA, sub = t % TPA;
  double v[2] = {0.0, 0.0};
  double wx = 0.0, wy = 0.0, wz = 0.0;
  if (i < n) {
    const double4 ui = u[i];
    for_pairs<TPA>(q, g, p, i, sub, [&](int j, const double *d, double r) {
      double uu, u1, u2;
      pair_u(r, p, uu, u1, u2);
      const double4 uj = u[j];
      const double ir = 1.0 / r;
      const double ex = d[0] * ir, ey = d[1] * ir, ez = d[2] * ir;
      const double dux = ui.x - uj.x, duy = ui.y - uj.y, duz = ui.z - uj.z;
      const double proj = ex * dux + ey * duy + ez * duz;
      const double t = u1 * ir;
      // K du = U'' e (e.du) + U'/r (du - e (e.du))
      wx += u2 * ex * proj + t * (dux - ex * proj);
      wy += u2 * ey * proj + t * (duy - ey * proj);
      wz += u2 * ez * proj + t * (duz - ez * proj);
      // F_i = sum_j -U'(r) e: dF_i/deps = -(U'/eps) e, dF_i/dsigma = (U' + r U'')/sigma e
      const double eu = ex * ui.x + ey * ui.y + ez * ui.z;
      v[0] += -(u1 * p.inv_eps) * eu;
      v[1] += (u1 + r * u2) * p.inv_sigma * eu;
    });
  }
  wx = group_sum<TPA>(wx);
  wy = group_sum<TPA>(wy);
  wz = group_sum<TPA>(wz);
  if (i < n && sub == 0) w[i] = make_double4(wx, wy, wz, 0.0);
  block_sums<2>(v, part);
}

// Fixed-order sum of nb blocks' ns (<= 3) partials into out[k], one block of
// kRB threads: thread t sums blocks t, t + kRB, ... in order, then a fixed
// tree; the per-step sums stay on the device until the end of the run.
constexpr int kRB = 256;
__global__ void __launch_bounds__(kRB) a_reduce(const double *part, int nb, int ns, double *out) {
  __shared__ double sm[3][kRB];
  const int t = threadIdx.x;
  for (int k = 0; k < ns; k++) {
    double x = 0.0;
    for (int b = t; b < nb; b += kRB) x += part[(size_t)b * ns + k];
    sm[k][t] = x;
  }
  __syncthreads();
  for (int o = kRB / 2; o > 0; o >>= 1) {
    if (t < o)
      for (int k = 0; k < ns; k++) sm[k][t] += sm[k][t + o];
    __syncthreads();
  }
  if (t < ns) out[t] = sm[t][0];
}

// --------------------------------------------------------- integration
__global__ void a_drift(double4 *q, const double4 *v, int n, double h) {
  const int i = blockIdx.x * kAB + threadIdx.x;
  if (i >= n) return;
  double4 a = q[i];
  const double4 b = v[i];
  a.x += b.x * h;
  a.y += b.y * h;
  a.z += b.z * h;
  q[i] = a;
}

__global__ void a_kick(double4 *v, const double4 *f, int n, double dt) {
  const int i = blockIdx.x * kAB + threadIdx.x;
  if (i >= n) return;
  double4 a = v[i];
  const double4 b = f[i];
  a.x += b.x * dt;
  a.y += b.y * dt;
  a.z += b.z * dt;
  v[i] = a;
}

// lv' = lv + lq dt/2 (into lv), u = lv' dt
__global__ void a_rev1(const double4 *lq, double4 *lv, double4 *u, int n, double dt) {
  const int i = blockIdx.x * kAB + threadIdx.x;
  if (i >= n) return;
  const double4 a = lq[i];
  double4 b = lv[i];
  b.x += a.x * dt * 0.5;
  b.y += a.y * dt * 0.5;
  b.z += a.z * dt * 0.5;
  lv[i] = b;
  u[i] = make_double4(b.x * dt, b.y * dt, b.z * dt, 0.0);
}

// lq_h = lq - w;  lq = lq_h;  lv += lq_h dt/2
__global__ void a_rev2(double4 *lq, double4 *lv, const double4 *w, int n, double dt) {
  const int i = blockIdx.x * kAB + threadIdx.x;
  if (i >= n) return;
  double4 a = lq[i];
  const double4 c = w[i];
  a.x -= c.x;
  a.y -= c.y;
  a.z -= c.z;
  lq[i] = a;
  double4 b = lv[i];
  b.x += a.x * dt * 0.5;
  b.y += a.y * dt * 0.5;
  b.z += a.z * dt * 0.5;
  lv[i] = b;
}

int nblk(int n) { return n > 0 ? (n + kAB - 1) / kAB : 1; }

struct Run {
  int n = 0, ncell = 0, tpa = 1;
  cudaStream_t s = nullptr;
  Grid g{};
  Pot p{};
  double dt = 0.0;
  double4 *q = nullptr, *v = nullptr, *f = nullptr, *tmp = nullptr;
  double4 *lq = nullptr, *lv = nullptr, *u = nullptr, *w = nullptr;
  double4 *ck_q = nullptr, *ck_v = nullptr;    // checkpoints
  double4 *seg_qh = nullptr, *seg_v = nullptr;  // one segment's q_h and v'
  int *cell = nullptr, *count = nullptr, *start = nullptr, *fill = nullptr, *perm = nullptr, *perm_fill = nullptr;
  double4 *qs = nullptr;                        // positions in cell order
  double *part = nullptr;                       // block partials of the pair kernels
  double *loss_sums = nullptr;                  // per step: PE, S, dPE/dsigma
  double *adj_sums = nullptr;                   // per reverse step: u . dF/d(eps, sigma)
  std::vector<void *> owned;

  template <typename T>
  cudaError_t alloc(T **ptr, size_t count_) {
    cudaError_t e = cudaMalloc((void **)ptr, sizeof(T) * (count_ ? count_ : 1));
    if (e == cudaSuccess) owned.push_back(*ptr);
    return e;
  }
  ~Run() {
    for (void *x : owned) cudaFree(x);
    if (s) cudaStreamDestroy(s);
  }
  int pair_blocks() const { return (int)(((long long)n * tpa + kAB - 1) / kAB); }

  // cell grid of the positions x
  void cells(const double4 *x) {
    cudaMemsetAsync(count, 0, sizeof(int) * ncell, s);
    cudaMemsetAsync(fill, 0, sizeof(int) * ncell, s);
    a_count<<<nblk(n), kAB, 0, s>>>(x, n, g, cell, count);
    a_scan<<<1, 1024, 0, s>>>(count, start, ncell);
    a_fill<<<nblk(n), kAB, 0, s>>>(n, cell, start, fill, perm_fill);
    a_sort<<<nblk(ncell * 32), kAB, 0, s>>>(ncell, start, perm_fill, perm);
    a_gather<<<nblk(n), kAB, 0, s>>>(x, perm, qs, n);
  }
  void force(const double4 *x) {
    const int nb = pair_blocks();
    switch (tpa) {
      case 1: a_force<1><<<nb, kAB, 0, s>>>(x, n, g, p, f); break;
      case 2: a_force<2><<<nb, kAB, 0, s>>>(x, n, g, p, f); break;
      case 4: a_force<4><<<nb, kAB, 0, s>>>(x, n, g, p, f); break;
      default: a_force<8><<<nb, kAB, 0, s>>>(x, n, g, p, f); break;
    }
  }
  void loss(const double4 *x, double4 *grad, double scale) {
    const int nb = pair_blocks();
    switch (tpa) {
      case 1: a_loss<1><<<nb, kAB, 0, s>>>(x, n, g, p, part, grad, scale); break;
      case 2: a_loss<2><<<nb, kAB, 0, s>>>(x, n, g, p, part, grad, scale); break;
      case 4: a_loss<4><<<nb, kAB, 0, s>>>(x, n, g, p, part, grad, scale); break;
      default: a_loss<8><<<nb, kAB, 0, s>>>(x, n, g, p, part, grad, scale); break;
    }
  }
  void hvp(const double4 *x) {
    const int nb = pair_blocks();
    switch (tpa) {
      case 1: a_hvp<1><<<nb, kAB, 0, s>>>(x, n, g, p, u, w, part); break;
      case 2: a_hvp<2><<<nb, kAB, 0, s>>>(x, n, g, p, u, w, part); break;
      case 4: a_hvp<4><<<nb, kAB, 0, s>>>(x, n, g, p, u, w, part); break;
      default: a_hvp<8><<<nb, kAB, 0, s>>>(x, n, g, p, u, w, part); break;
    }
  }
  // one forward step; keeps q_h and v' when asked
  void step(double4 *qh_out, double4 *v_out) {
    a_drift<<<nblk(n), kAB, 0, s>>>(q, v, n, 0.5 * dt);
    cells(q);
    force(q);
    if (qh_out) cudaMemcpyAsync(qh_out, q, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s);
    a_kick<<<nblk(n), kAB, 0, s>>>(v, f, n, dt);
    if (v_out) cudaMemcpyAsync(v_out, v, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s);
    a_drift<<<nblk(n), kAB, 0, s>>>(q, v, n, 0.5 * dt);
  }
  // loss terms at x: sums into out[0..2] (device), gradient into lq when scale != 0
  void loss_at(const double4 *x, double scale, double *out) {
    cells(x);
    loss(x, scale != 0.0 ? lq : nullptr, scale);
    if (out) a_reduce<<<1, kRB, 0, s>>>(part, pair_blocks(), 3, out);
  }
};

// Lanes per atom of the pair kernels, chosen once per device and problem
// shape by timing the force kernel with 1, 2, 4 and 8 lanes (the fastest is
// kept for the process, so repeated runs of one shape use the same lanes and
// give the same sums).
std::mutex g_tune_mutex;
std::map<std::tuple<int, int, int>, int> g_tune;

int autotune_tpa(Run &R, int device) {
  const auto key = std::make_tuple(device, R.n, R.ncell);
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  R.cells(R.q);
  int best = 1;
  float best_ms = 1e30f;
  for (int t : {1, 2, 4, 8}) {
    R.tpa = t;
    R.force(R.q);  // warm-up
    cudaEventRecord(e0, R.s);
    for (int r = 0; r < 3; r++) R.force(R.q);
    cudaEventRecord(e1, R.s);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
      best = t;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_tune[key] = best;
  return best;
}

}  // namespace

extern "C" {

void mdg_adjoint_default_params(mdg_adjoint_params *p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->L[0] = p->L[1] = p->L[2] = 10.0;
  p->cutoff = 2.5;
  p->time_step = 0.005;
  p->epsilon = 1.0;
  p->sigma = 1.0;
  p->shell_lo = 1.0;
  p->shell_hi = 1.5;
  p->shell_width = 0.05;
  p->steps = 200;
  p->checkpoint_every = 20;
  p->threads_per_atom = 0;
  p->device = 0;
}

mdg_status mdg_adjoint_run(const mdg_adjoint_params *prm, const double *q0, const double *v0, int n, double *loss,
                           double *dloss_deps, double *dloss_dsigma, double *dloss_dq0) {
  if (!prm || !q0 || !v0 || !loss || n < 1 || prm->steps < 1 || prm->checkpoint_every < 1 ||
      !(prm->time_step > 0.0) || !(prm->epsilon > 0.0) || !(prm->sigma > 0.0) || !(prm->cutoff > 0.0) ||
      !(prm->shell_width > 0.0) ||
      (prm->threads_per_atom != 0 && prm->threads_per_atom != 1 && prm->threads_per_atom != 2 &&
       prm->threads_per_atom != 4 && prm->threads_per_atom != 8))
    return MDG_ERR_INVALID_ARGUMENT;
  const bool grad = dloss_deps || dloss_dsigma || dloss_dq0;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MDG_ERR_NO_DEVICE;
  if (prm->device < 0 || prm->device >= ndev) return MDG_ERR_INVALID_ARGUMENT;
  if (cudaSetDevice(prm->device) != cudaSuccess) return MDG_ERR_CUDA;

  Run R;
  R.n = n;
  R.dt = prm->time_step;
  const double rc = prm->cutoff * prm->sigma;
  for (int d = 0; d < 3; d++) {
    const double L = prm->L[d];
    if (!(L > 0.0) || !std::isfinite(L)) return MDG_ERR_INVALID_ARGUMENT;
    R.g.ms[d] = (int)(L / rc);
    if (R.g.ms[d] < 3) return MDG_ERR_BOX_TOO_SMALL;
    R.g.L[d] = L;
    R.g.inv_cs[d] = R.g.ms[d] / L;
    R.g.inv_L[d] = 1.0 / L;
  }
  R.ncell = R.g.ms[0] * R.g.ms[1] * R.g.ms[2];
  const double sc = prm->cutoff;
  R.p.eps = prm->epsilon;
  R.p.sigma = prm->sigma;
  R.p.rc2 = rc * rc;
  R.p.c2 = 6.0 * pow(sc, -14.0) - 3.0 * pow(sc, -8.0);
  R.p.c0 = -pow(sc, -12.0) + pow(sc, -6.0) - R.p.c2 * sc * sc;
  R.p.a = prm->shell_lo;
  R.p.b = prm->shell_hi;
  R.p.w = prm->shell_width;
  R.p.inv_sigma = 1.0 / R.p.sigma;
  R.p.inv_w = 1.0 / R.p.w;
  R.p.inv_eps = 1.0 / R.p.eps;
  R.p.eps_sigma = R.p.eps / R.p.sigma;
  R.p.eps_sigma2 = R.p.eps / (R.p.sigma * R.p.sigma);
  const int T = prm->steps, k = prm->checkpoint_every;
  const int nck = (T + k - 1) / k + 1;
  const size_t max_blocks = ((size_t)n * 8 + kAB - 1) / kAB;

  cudaError_t e = cudaStreamCreateWithFlags(&R.s, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = R.alloc(&R.q, n);
  if (e == cudaSuccess) e = R.alloc(&R.v, n);
  if (e == cudaSuccess) e = R.alloc(&R.f, n);
  if (e == cudaSuccess) e = R.alloc(&R.tmp, n);
  if (e == cudaSuccess) e = R.alloc(&R.cell, n);
  if (e == cudaSuccess) e = R.alloc(&R.count, R.ncell);
  if (e == cudaSuccess) e = R.alloc(&R.fill, R.ncell);
  if (e == cudaSuccess) e = R.alloc(&R.start, R.ncell + 1);
  if (e == cudaSuccess) e = R.alloc(&R.perm, n);
  if (e == cudaSuccess) e = R.alloc(&R.perm_fill, n);
  if (e == cudaSuccess) e = R.alloc(&R.qs, n);
  if (e == cudaSuccess) e = R.alloc(&R.part, max_blocks * 3);
  if (e == cudaSuccess) e = R.alloc(&R.loss_sums, (size_t)T * 3);
  if (grad) {
    if (e == cudaSuccess) e = R.alloc(&R.lq, n);
    if (e == cudaSuccess) e = R.alloc(&R.lv, n);
    if (e == cudaSuccess) e = R.alloc(&R.u, n);
    if (e == cudaSuccess) e = R.alloc(&R.w, n);
    if (e == cudaSuccess) e = R.alloc(&R.adj_sums, (size_t)T * 2);
    if (e == cudaSuccess) e = R.alloc(&R.ck_q, (size_t)nck * n);
    if (e == cudaSuccess) e = R.alloc(&R.ck_v, (size_t)nck * n);
    if (e == cudaSuccess) e = R.alloc(&R.seg_qh, (size_t)k * n);
    if (e == cudaSuccess) e = R.alloc(&R.seg_v, (size_t)k * n);
  }
  if (e != cudaSuccess) return e == cudaErrorMemoryAllocation ? MDG_ERR_CAPACITY : MDG_ERR_CUDA;
  R.g.start = R.start;
  R.g.perm = R.perm;
  R.g.qs = R.qs;

  // upload (n x 3 host arrays -> double4)
  {
    std::vector<double4> hq(n), hv(n);
    for (int i = 0; i < n; i++) {
      hq[i] = make_double4(q0[3 * i], q0[3 * i + 1], q0[3 * i + 2], 0.0);
      hv[i] = make_double4(v0[3 * i], v0[3 * i + 1], v0[3 * i + 2], 0.0);
    }
    e = cudaMemcpyAsync(R.q, hq.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, R.s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(R.v, hv.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, R.s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(R.s);
    if (e != cudaSuccess) return MDG_ERR_CUDA;
  }
  R.tpa = prm->threads_per_atom ? prm->threads_per_atom : autotune_tpa(R, prm->device);

  // forward pass: loss terms per step, checkpoints every k steps
  for (int t = 0; t < T; t++) {
    if (grad && t % k == 0) {
      cudaMemcpyAsync(R.ck_q + (size_t)(t / k) * n, R.q, sizeof(double4) * n, cudaMemcpyDeviceToDevice, R.s);
      cudaMemcpyAsync(R.ck_v + (size_t)(t / k) * n, R.v, sizeof(double4) * n, cudaMemcpyDeviceToDevice, R.s);
    }
    R.step(nullptr, nullptr);
    R.loss_at(R.q, 0.0, R.loss_sums + (size_t)3 * t);
  }
  std::vector<double> sums((size_t)T * 3);
  e = cudaMemcpyAsync(sums.data(), R.loss_sums, sizeof(double) * sums.size(), cudaMemcpyDeviceToHost, R.s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(R.s);
  if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) return MDG_ERR_CUDA;
  const double norm = 1.0 / ((double)T * n);
  double l = 0.0, dl_deps = 0.0, dl_dsig = 0.0;
  for (int t = 0; t < T; t++) {
    l += sums[3 * t] + sums[3 * t + 1];
    dl_deps += sums[3 * t] / prm->epsilon;  // PE is linear in epsilon
    dl_dsig += sums[3 * t + 2];
  }
  *loss = l * norm;
  if (!grad) return MDG_OK;
  dl_deps *= norm;
  dl_dsig *= norm;

  // reverse sweep, one checkpointed segment at a time
  cudaMemsetAsync(R.lq, 0, sizeof(double4) * n, R.s);
  cudaMemsetAsync(R.lv, 0, sizeof(double4) * n, R.s);
  for (int seg = (T - 1) / k; seg >= 0; seg--) {
    const int t0 = seg * k, t1 = std::min(T, t0 + k);
    cudaMemcpyAsync(R.q, R.ck_q + (size_t)seg * n, sizeof(double4) * n, cudaMemcpyDeviceToDevice, R.s);
    cudaMemcpyAsync(R.v, R.ck_v + (size_t)seg * n, sizeof(double4) * n, cudaMemcpyDeviceToDevice, R.s);
    for (int t = t0; t < t1; t++) R.step(R.seg_qh + (size_t)(t - t0) * n, R.seg_v + (size_t)(t - t0) * n);
    for (int t = t1 - 1; t >= t0; t--) {
      const double4 *qh = R.seg_qh + (size_t)(t - t0) * n;
      const double4 *vp = R.seg_v + (size_t)(t - t0) * n;
      // q' = q_h + v' dt/2, and this step's loss gradient at q'
      cudaMemcpyAsync(R.tmp, qh, sizeof(double4) * n, cudaMemcpyDeviceToDevice, R.s);
      a_drift<<<nblk(n), kAB, 0, R.s>>>(R.tmp, vp, n, 0.5 * R.dt);
      R.loss_at(R.tmp, norm, nullptr);
      a_rev1<<<nblk(n), kAB, 0, R.s>>>(R.lq, R.lv, R.u, n, R.dt);
      R.cells(qh);
      R.hvp(qh);
      a_reduce<<<1, kRB, 0, R.s>>>(R.part, R.pair_blocks(), 2, R.adj_sums + (size_t)2 * t);
      a_rev2<<<nblk(n), kAB, 0, R.s>>>(R.lq, R.lv, R.w, n, R.dt);
    }
  }
  std::vector<double> adj((size_t)T * 2);
  e = cudaMemcpyAsync(adj.data(), R.adj_sums, sizeof(double) * adj.size(), cudaMemcpyDeviceToHost, R.s);
  std::vector<double4> h(n);
  if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), R.lq, sizeof(double4) * n, cudaMemcpyDeviceToHost, R.s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(R.s);
  if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) return MDG_ERR_CUDA;
  // dynamics terms summed in reverse-sweep order, as the sweep produced them
  for (int t = T - 1; t >= 0; t--) {
    dl_deps += adj[(size_t)2 * t];
    dl_dsig += adj[(size_t)2 * t + 1];
  }
  if (dloss_dq0) {
    for (int i = 0; i < n; i++) {
      dloss_dq0[3 * i] = h[i].x;
      dloss_dq0[3 * i + 1] = h[i].y;
      dloss_dq0[3 * i + 2] = h[i].z;
    }
  }
  if (dloss_deps) *dloss_deps = dl_deps;
  if (dloss_dsigma) *dloss_dsigma = dl_dsig;
  return MDG_OK;
}

}  // extern "C"
