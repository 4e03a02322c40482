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
// Pairs come from a Verlet list of search length r_c + skin (r_c = s_c
// sigma; skin 0.3 sigma, less where the box is narrow), built from a cell
// grid (cells at least r_c + skin wide, >= 3 per axis, atoms in each cell
// ordered by index, rows in cell-walk order, so every sum is deterministic).
// Before each evaluation every atom's displacement from the list's build
// positions is checked; the list is rebuilt when one exceeds skin/2, which
// keeps every pair within r_c in the rows.  This component has no
// counterpart in the reference, which has no gradients.
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

// The Verlet list: row of atom i = entries nbr[k * n + i], k < cnt[i].
struct Rows {
  const int *nbr;
  const int *cnt;
  double inv_L[3], L[3];
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

// Calls f(j, d, r) for every partner j of i's row with r < r_c, d = minimum
// image of q_i - q_j, in row order (ascending j).  Rows hold every pair
// within r_c and more, in ascending j, so the pairs within r_c and their
// order are a function of q alone, whichever build the row comes from.
// TPA lanes share one atom: they test TPA entries at a time, number the
// pairs within r_c in row order, and lane `sub` takes pairs sub, sub + TPA,
// ... of that numbering (shuffled to it from the lane that tested them); the
// caller combines the lanes' sums with group_sum.  All TPA lanes of the atom
// call together.
template <int TPA, class F>
__device__ __forceinline__ void for_pairs(const double4 *q, const Rows &w, const Pot &p, int i, int sub, int n,
                                          F f) {
  const double4 qi = q[i];
  const int m = w.cnt[i];
  auto pair_of = [&](int k, int &j, double (&d)[3]) {
    j = w.nbr[(size_t)k * n + i];
    const double4 qj = q[j];
    d[0] = qi.x - qj.x;
    d[1] = qi.y - qj.y;
    d[2] = qi.z - qj.z;
    for (int a = 0; a < 3; a++) d[a] -= w.L[a] * rint(d[a] * w.inv_L[a]);
    return d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  };
  if (TPA == 1) {
    for (int k = 0; k < m; k++) {
      int j;
      double d[3];
      const double r2 = pair_of(k, j, d);
      if (r2 < p.rc2) f(j, d, sqrt(r2));
    }
    return;
  }
  const int lane = threadIdx.x & 31, first = lane & ~(TPA - 1);
  const unsigned gmask = (TPA == 32) ? 0xffffffffu : (((1u << TPA) - 1u) << first);
  int before = 0;  // pairs within r_c in the entries already tested
  for (int k0 = 0; k0 < m; k0 += TPA) {
    int j = 0;
    double d[3] = {0.0, 0.0, 0.0}, r2 = 0.0;
    bool in = false;
    if (k0 + sub < m) {
      r2 = pair_of(k0 + sub, j, d);
      in = r2 < p.rc2;
    }
    const unsigned bal = (__ballot_sync(gmask, in) >> first) & ((1u << TPA) - 1u);
    const int cnt = __popc(bal);
    // this lane's pair of the batch: number r of the batch's pairs, the one
    // with overall number == sub (mod TPA)
    const int r = (sub - before % TPA + TPA) % TPA;
    int src = 0;
#pragma unroll
    for (int b = 0, c = 0; b < TPA; b++) {
      if ((bal >> b) & 1u) {
        if (c == r) src = b;
        c++;
      }
    }
    const int jj = __shfl_sync(gmask, j, first + src);
    double dd[3];
    dd[0] = __shfl_sync(gmask, d[0], first + src);
    dd[1] = __shfl_sync(gmask, d[1], first + src);
    dd[2] = __shfl_sync(gmask, d[2], first + src);
    const double rr = __shfl_sync(gmask, r2, first + src);
    if (r < cnt) f(jj, dd, sqrt(rr));
    before += cnt;
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
// The grid kernels run only when the list is to be rebuilt (*want != 0).
__global__ void a_clear(int *count, int *fill, int ncell, const int *want) {
  if (!*want) return;
  for (int c = blockIdx.x * kAB + threadIdx.x; c < ncell; c += gridDim.x * kAB) count[c] = fill[c] = 0;
}

__global__ void a_count(const double4 *q, int n, Grid g, int *cell, int *count, const int *want) {
  const int i = blockIdx.x * kAB + threadIdx.x;
  if (i >= n || !*want) return;
  const int c = cell_of(q[i], g);
  cell[i] = c;
  atomicAdd(&count[c], 1);
}

// exclusive scan of count into start (one block, ncell of any size)
__global__ void a_scan(const int *count, int *start, int ncell, const int *want) {
  if (!*want) return;
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

__global__ void a_fill(int n, const int *cell, const int *start, int *fill, int *perm, const int *want) {
  const int i = blockIdx.x * kAB + threadIdx.x;
  if (i >= n || !*want) return;
  const int c = cell[i];
  perm[start[c] + atomicAdd(&fill[c], 1)] = i;
}

// Orders every cell by atom index, one warp per cell: each entry's new
// place is the count of smaller indices in the cell (indices are distinct).
// perm_in is the fill order, perm_out the sorted one.
__global__ void a_sort(int ncell, const int *start, const int *perm_in, int *perm_out, const int *want) {
  const int c = (blockIdx.x * kAB + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= ncell || !*want) return;
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
__global__ void a_gather(const double4 *x, const int *perm, double4 *xs, int n, const int *want) {
  const int k = blockIdx.x * kAB + threadIdx.x;
  if (k < n && *want) xs[k] = x[perm[k]];
}

// The whole grid (clear, count, scan, fill, per-cell index order, gather)
// in one block of 1024 threads, for up to kGrid1Atoms atoms.
constexpr int kGrid1Atoms = 262144;
__global__ void __launch_bounds__(1024) a_grid1(const double4 *x, int n, Grid g, int ncell, int *cell, int *count,
                                                int *start, int *fill, int *perm_fill, int *perm, double4 *qs,
                                                const int *want) {
  if (!*want) return;
  __shared__ int part[1024];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  for (int c = t; c < ncell; c += 1024) count[c] = fill[c] = 0;
  __syncthreads();
  for (int i = t; i < n; i += 1024) {
    const int c = cell_of(x[i], g);
    cell[i] = c;
    atomicAdd(&count[c], 1);
  }
  __syncthreads();
  {  // exclusive scan of count into start, 1024 chunks
    const int chunk = (ncell + 1023) / 1024;
    const int beg = min(t * chunk, ncell), end = min(beg + chunk, ncell);
    int sum = 0;
    for (int c = beg; c < end; c++) sum += count[c];
    part[t] = sum;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      const int v = t >= o ? part[t - o] : 0;
      __syncthreads();
      part[t] += v;
      __syncthreads();
    }
    int run = part[t] - sum;
    for (int c = beg; c < end; c++) {
      start[c] = run;
      run += count[c];
    }
    if (t == 1023) start[ncell] = part[t];
  }
  __syncthreads();
  for (int i = t; i < n; i += 1024) {
    const int c = cell[i];
    perm_fill[start[c] + atomicAdd(&fill[c], 1)] = i;
  }
  __syncthreads();
  for (int c = warp; c < ncell; c += 32) {  // index order inside each cell (as a_sort)
    const int b = start[c], cnt = start[c + 1] - b;
    for (int base = 0; base < cnt; base += 32) {
      const int me = base + lane;
      const int key = me < cnt ? perm_fill[b + me] : 0x7fffffff;
      int rank = 0;
      for (int ob = 0; ob < cnt; ob += 32) {
        const int okey = ob + lane < cnt ? perm_fill[b + ob + lane] : 0x7fffffff;
        for (int k = 0; k < 32; k++) rank += (ob + k < cnt) && (__shfl_sync(0xffffffffu, okey, k) < key);
      }
      if (me < cnt) perm[b + rank] = key;
    }
  }
  __syncthreads();
  for (int k = t; k < n; k += 1024) qs[k] = x[perm[k]];
}

// ---------------------------------------------------------- Verlet list
// flag[0] = 1 if some atom moved more than skin/2 from the list's build
// positions qb (minimum image); flag[0] starts at 1 for the first build.
__global__ void a_check(const double4 *x, const double4 *qb, int n, Rows w, double half_skin2, int *flag) {
  const int i = blockIdx.x * kAB + threadIdx.x;
  if (i >= n) return;
  const double4 a = x[i], b = qb[i];
  double d[3] = {a.x - b.x, a.y - b.y, a.z - b.z};
  for (int k = 0; k < 3; k++) d[k] -= w.L[k] * rint(d[k] * w.inv_L[k]);
  if (d[0] * d[0] + d[1] * d[1] + d[2] * d[2] > half_skin2) atomicOr(flag, 1);
}

// Ascending sort of the 32 E values of a warp, v[e] = element e * 32 + lane
// (bitonic network, fully unrolled).
template <int E>
__device__ __forceinline__ void warp_sort_asc(int (&v)[E], int lane) {
  constexpr int N = 32 * E;
#pragma unroll
  for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
#pragma unroll
      for (int e = 0; e < E; e++) {
        if (j < 32) {  // partner in lane ^ j, same e
          const int g = e * 32 + lane;
          const int o = __shfl_xor_sync(0xffffffffu, v[e], j);
          const bool up = (g & k) == 0, lower = (g & j) == 0;
          v[e] = (lower == up) ? min(v[e], o) : max(v[e], o);
        } else {  // partner e ^ (j / 32) in the same lane
          const int f = e ^ (j / 32);
          if (f > e) {
            const bool up = ((e * 32) & k) == 0;
            const int a = v[e], b = v[f];
            v[e] = up ? min(a, b) : max(a, b);
            v[f] = up ? max(a, b) : min(a, b);
          }
        }
      }
    }
  }
}

// Rows of the list at x, one warp per atom i: the partners j != i with
// |x_i - x_j| <= sl (minimum image), found by walking the 27 cells around
// i's (the lanes test a cell's atoms 32 at a time and gather the kept ones
// in a shared buffer), then sorted ascending (warp_sort_asc, rows of up to
// 32 E entries); x is copied to qb.  Runs only when *want != 0; clears
// *next, the rebuild flag of the next evaluation.  A row longer than maxnb
// (<= 32 E) sets *overflow.
template <int E>
__global__ void __launch_bounds__(kAB) a_rows(const double4 *x, int n, Grid g, double sl2, int maxnb, int *nbr,
                                              int *cnt, double4 *qb, const int *want, int *next, int *overflow) {
  __shared__ int buf[kAB / 32][32 * E];
  const int i = (int)(((long long)blockIdx.x * kAB + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  if (blockIdx.x == 0 && threadIdx.x == 0) *next = 0;
  if (i >= n || !*want) return;  // whole warps leave together
  const double4 qi = x[i];
  if (lane == 0) qb[i] = qi;
  const int cx = cell_axis(qi.x, g.L[0], g.inv_cs[0], g.ms[0]);
  const int cy = cell_axis(qi.y, g.L[1], g.inv_cs[1], g.ms[1]);
  const int cz = cell_axis(qi.z, g.L[2], g.inv_cs[2], g.ms[2]);
  // lane l < 27 holds cell l's first slot and the inclusive prefix of the
  // 27 cells' counts: the candidates are one concatenated range of `total`
  // (the row is sorted afterwards, so the walk order does not matter)
  int beg = 0, pre = 0;
  if (lane < 27) {
    const int z = (cz + lane / 9 - 1 + g.ms[2]) % g.ms[2];
    const int y = (cy + (lane / 3) % 3 - 1 + g.ms[1]) % g.ms[1];
    const int xx = (cx + lane % 3 - 1 + g.ms[0]) % g.ms[0];
    const int c = (z * g.ms[1] + y) * g.ms[0] + xx;
    beg = g.start[c];
    pre = g.start[c + 1] - beg;
  }
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, pre, o);
    if (lane >= o) pre += v;
  }
  const int total = __shfl_sync(0xffffffffu, pre, 26);
  int m = 0;  // partners found (warp-uniform)
  for (int fb = 0; fb < total; fb += 32) {
    const int f = fb + lane;
    // the cell of candidate f: the first cell whose inclusive prefix exceeds f
    int lo = 0, hi = 26;
#pragma unroll
    for (int it = 0; it < 5; it++) {
      const int mid = (lo + hi) >> 1;
      const int pm = __shfl_sync(0xffffffffu, pre, mid);
      if (pm > f) hi = mid;
      else lo = min(mid + 1, hi);
    }
    const int bq = __shfl_sync(0xffffffffu, beg, lo);
    const int pp = __shfl_sync(0xffffffffu, pre, lo > 0 ? lo - 1 : 0);
    const int excl = lo > 0 ? pp : 0;  // candidates in the cells before
    int j = -1;
    bool keep = false;
    if (f < total) {
      const int k = bq + (f - excl);
      j = g.perm[k];
      const double4 qj = g.qs[k];
      double d[3] = {qi.x - qj.x, qi.y - qj.y, qi.z - qj.z};
      for (int a = 0; a < 3; a++) d[a] -= g.L[a] * rint(d[a] * g.inv_L[a]);
      keep = j != i && d[0] * d[0] + d[1] * d[1] + d[2] * d[2] <= sl2;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, keep);
    const int slot = m + __popc(bal & ((1u << lane) - 1u));
    if (keep && slot < maxnb) buf[wib][slot] = j;
    m += __popc(bal);
  }
  __syncwarp();
  const int mm = min(m, maxnb);
  int v[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int s = e * 32 + lane;
    v[e] = s < mm ? buf[wib][s] : 0x7fffffff;
  }
  warp_sort_asc<E>(v, lane);
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int s = e * 32 + lane;
    if (s < mm) nbr[(size_t)s * n + i] = v[e];
  }
  if (lane == 0) {
    cnt[i] = mm;
    if (m > maxnb) atomicOr(overflow, 1);
  }
}

// --------------------------------------------------------------- physics
template <int TPA>
__global__ void __launch_bounds__(kAB) a_force(const double4 *q, int n, Rows g, Pot p, double4 *f) {
  const int t = blockIdx.x * kAB + threadIdx.x;
  const int i = t / TPA, sub = t % TPA;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  if (i < n) {
    for_pairs<TPA>(q, g, p, i, sub, n, [&](int, const double *d, double r) {
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
__global__ void __launch_bounds__(kAB) a_loss(const double4 *q, int n, Rows g, Pot p, double *part, double4 *lq,
                                              double scale) {
  const int t = blockIdx.x * kAB + threadIdx.x;
  const int i = t / TPA, sub = t % TPA;
  double v[3] = {0.0, 0.0, 0.0};
  double gx = 0.0, gy = 0.0, gz = 0.0;
  if (i < n) {
    for_pairs<TPA>(q, g, p, i, sub, n, [&](int, const double *d, double r) {
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
__global__ void __launch_bounds__(kAB) a_hvp(const double4 *q, int n, Rows g, Pot p, const double4 *u, double4 *w,
                                             double *part) {
  const int t = blockIdx.x * kAB + threadIdx.x;
  const int i = t / TPA, sub = t % TPA;
  double v[2] = {0.0, 0.0};
  double wx = 0.0, wy = 0.0, wz = 0.0;
  if (i < n) {
    const double4 ui = u[i];
    for_pairs<TPA>(q, g, p, i, sub, n, [&](int j, const double *d, double r) {
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

// Device buffers, stream and pinned flag copy of the adjoint, kept per
// device between calls: a call takes its buffers in a fixed order and reuses
// every kept buffer that is large enough, replacing the others, so repeated
// calls of one shape allocate nothing.  One run at a time per process
// (g_ws_mutex); mdg_adjoint_release frees everything.
struct Workspace {
  std::vector<void *> buf;
  std::vector<size_t> bytes;
  cudaStream_t s = nullptr;
  int *hflag = nullptr;
};
std::mutex g_ws_mutex;
std::map<int, Workspace> g_ws;

void free_workspace(Workspace &w) {
  for (void *x : w.buf)
    if (x) cudaFree(x);
  if (w.hflag) cudaFreeHost(w.hflag);
  if (w.s) cudaStreamDestroy(w.s);
  w = Workspace();
}

struct Run {
  Workspace *ws = nullptr;
  size_t slot = 0;  // next workspace buffer
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
  // Verlet list (a_rows): rows, row lengths, build positions, flags (the
  // rebuild flags of even and odd evaluations, row overflow) and a host copy
  Rows rows{};
  int *nbr = nullptr, *cnt = nullptr, *flag = nullptr, *hflag = nullptr;
  double4 *qb = nullptr;
  int maxnb = 0;
  double sl2 = 0.0, half_skin2 = 0.0;
  long long evals = 0;  // list preparations so far (picks the flag pair's slot)

  template <typename T>
  cudaError_t alloc(T **ptr, size_t count_) {
    const size_t b = sizeof(T) * (count_ ? count_ : 1);
    if (slot == ws->buf.size()) {
      ws->buf.push_back(nullptr);
      ws->bytes.push_back(0);
    }
    if (ws->bytes[slot] < b) {
      if (ws->buf[slot]) cudaFree(ws->buf[slot]);
      ws->buf[slot] = nullptr;
      ws->bytes[slot] = 0;
      void *p = nullptr;
      const cudaError_t e = cudaMalloc(&p, b);
      if (e != cudaSuccess) return e;
      ws->buf[slot] = p;
      ws->bytes[slot] = b;
    }
    *ptr = static_cast<T *>(ws->buf[slot++]);
    return cudaSuccess;
  }
  int pair_blocks() const { return (int)(((long long)n * tpa + kAB - 1) / kAB); }

  // cell grid of the positions x, when *want != 0
  void cells(const double4 *x, const int *want) {
    if (n <= kGrid1Atoms) {
      a_grid1<<<1, 1024, 0, s>>>(x, n, g, ncell, cell, count, start, fill, perm_fill, perm, qs, want);
      return;
    }
    a_clear<<<std::min(nblk(ncell), 1024), kAB, 0, s>>>(count, fill, ncell, want);
    a_count<<<nblk(n), kAB, 0, s>>>(x, n, g, cell, count, want);
    a_scan<<<1, 1024, 0, s>>>(count, start, ncell, want);
    a_fill<<<nblk(n), kAB, 0, s>>>(n, cell, start, fill, perm_fill, want);
    a_sort<<<nblk(ncell * 32), kAB, 0, s>>>(ncell, start, perm_fill, perm, want);
    a_gather<<<nblk(n), kAB, 0, s>>>(x, perm, qs, n, want);
  }
  // True if a row outgrew maxnb in any build so far (the sums are then
  // incomplete).
  bool rows_overflowed() {
    if (cudaMemcpyAsync(hflag, flag + 2, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return true;
    if (cudaStreamSynchronize(s) != cudaSuccess) return true;
    return hflag[0] != 0;
  }
  // Makes the list valid for an evaluation at x, on the device: a_check
  // raises this evaluation's rebuild flag when an atom has moved more than
  // skin/2 since the list's build, and the grid and row kernels run only
  // then (two flags, used by alternate evaluations: a_rows clears the next
  // one).  No host wait.
  void prepare(const double4 *x) {
    int *want = flag + (evals & 1), *next = flag + ((evals + 1) & 1);
    evals++;
    a_check<<<nblk(n), kAB, 0, s>>>(x, qb, n, rows, half_skin2, want);
    cells(x, want);
    const int wb = (int)(((long long)n * 32 + kAB - 1) / kAB);  // one warp per atom
    int *ov = flag + 2;
    if (maxnb <= 32) a_rows<1><<<wb, kAB, 0, s>>>(x, n, g, sl2, maxnb, nbr, cnt, qb, want, next, ov);
    else if (maxnb <= 64) a_rows<2><<<wb, kAB, 0, s>>>(x, n, g, sl2, maxnb, nbr, cnt, qb, want, next, ov);
    else if (maxnb <= 128) a_rows<4><<<wb, kAB, 0, s>>>(x, n, g, sl2, maxnb, nbr, cnt, qb, want, next, ov);
    else if (maxnb <= 256) a_rows<8><<<wb, kAB, 0, s>>>(x, n, g, sl2, maxnb, nbr, cnt, qb, want, next, ov);
    else if (maxnb <= 512) a_rows<16><<<wb, kAB, 0, s>>>(x, n, g, sl2, maxnb, nbr, cnt, qb, want, next, ov);
    else a_rows<32><<<wb, kAB, 0, s>>>(x, n, g, sl2, maxnb, nbr, cnt, qb, want, next, ov);
  }
  void force(const double4 *x) {
    const int nb = pair_blocks();
    switch (tpa) {
      case 1: a_force<1><<<nb, kAB, 0, s>>>(x, n, rows, p, f); break;
      case 2: a_force<2><<<nb, kAB, 0, s>>>(x, n, rows, p, f); break;
      case 4: a_force<4><<<nb, kAB, 0, s>>>(x, n, rows, p, f); break;
      default: a_force<8><<<nb, kAB, 0, s>>>(x, n, rows, p, f); break;
    }
  }
  void loss(const double4 *x, double4 *grad, double scale) {
    const int nb = pair_blocks();
    switch (tpa) {
      case 1: a_loss<1><<<nb, kAB, 0, s>>>(x, n, rows, p, part, grad, scale); break;
      case 2: a_loss<2><<<nb, kAB, 0, s>>>(x, n, rows, p, part, grad, scale); break;
      case 4: a_loss<4><<<nb, kAB, 0, s>>>(x, n, rows, p, part, grad, scale); break;
      default: a_loss<8><<<nb, kAB, 0, s>>>(x, n, rows, p, part, grad, scale); break;
    }
  }
  void hvp(const double4 *x) {
    const int nb = pair_blocks();
    switch (tpa) {
      case 1: a_hvp<1><<<nb, kAB, 0, s>>>(x, n, rows, p, u, w, part); break;
      case 2: a_hvp<2><<<nb, kAB, 0, s>>>(x, n, rows, p, u, w, part); break;
      case 4: a_hvp<4><<<nb, kAB, 0, s>>>(x, n, rows, p, u, w, part); break;
      default: a_hvp<8><<<nb, kAB, 0, s>>>(x, n, rows, p, u, w, part); break;
    }
  }
  // one forward step; keeps q_h and v' when asked
  void step(double4 *qh_out, double4 *v_out) {
    a_drift<<<nblk(n), kAB, 0, s>>>(q, v, n, 0.5 * dt);
    prepare(q);
    force(q);
    if (qh_out) cudaMemcpyAsync(qh_out, q, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s);
    a_kick<<<nblk(n), kAB, 0, s>>>(v, f, n, dt);
    if (v_out) cudaMemcpyAsync(v_out, v, sizeof(double4) * n, cudaMemcpyDeviceToDevice, s);
    a_drift<<<nblk(n), kAB, 0, s>>>(q, v, n, 0.5 * dt);
  }
  // loss terms at x: sums into out[0..2] (device), gradient into lq when scale != 0
  void loss_at(const double4 *x, double scale, double *out) {
    prepare(x);
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
  R.prepare(R.q);
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

void mdg_adjoint_release(void) {
  std::lock_guard<std::mutex> lock(g_ws_mutex);
  int cur = 0;
  const bool have = cudaGetDevice(&cur) == cudaSuccess;
  for (auto &kv : g_ws) {
    if (cudaSetDevice(kv.first) == cudaSuccess) free_workspace(kv.second);
  }
  g_ws.clear();
  if (have) cudaSetDevice(cur);
}

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
  // list skin: 0.3 sigma, less where a box axis holds fewer than three
  // cells of r_c + skin (no skin at all: the list is rebuilt whenever an
  // atom moved)
  double skin = 0.3 * prm->sigma;
  for (int d = 0; d < 3; d++) {
    const double L = prm->L[d];
    if (!(L > 0.0) || !std::isfinite(L)) return MDG_ERR_INVALID_ARGUMENT;
    if ((int)(L / rc) < 3) return MDG_ERR_BOX_TOO_SMALL;
    skin = std::min(skin, L / 3.0 * (1.0 - 1e-9) - rc);  // cells of L/ms >= r_c + skin, ms >= 3
  }
  skin = std::max(skin, 0.0);
  const double sl = rc + skin;
  for (int d = 0; d < 3; d++) {
    const double L = prm->L[d];
    R.g.ms[d] = std::max(3, (int)(L / sl));
    R.g.L[d] = L;
    R.g.inv_cs[d] = R.g.ms[d] / L;
    R.g.inv_L[d] = 1.0 / L;
    R.rows.L[d] = L;
    R.rows.inv_L[d] = 1.0 / L;
  }
  // rows keep pairs up to sl, a hair wider than the r_c + 2 (skin / 2) that
  // the displacement bound needs
  R.sl2 = sl * sl * (1.0 + 1e-9);
  R.half_skin2 = 0.25 * skin * skin;
  {
    const double vol = prm->L[0] * prm->L[1] * prm->L[2];
    const double est = 4.0 / 3.0 * M_PI * sl * sl * sl * (double)n / vol;
    // twice the mean density's count plus 64, and at least the count at
    // density 1.3 (above a close-packed LJ solid) plus 32, so that a dense
    // region of a dilute box fits; at most 1024 (the row sort's width).  A
    // longer row is MDG_ERR_CAPACITY.
    const double dense = 4.0 / 3.0 * M_PI * sl * sl * sl * 1.3 / (prm->sigma * prm->sigma * prm->sigma);
    const double want = std::max(std::ceil(2.0 * est + 64.0), std::ceil(dense + 32.0));
    R.maxnb = (int)std::min<double>(std::min(std::max(n - 1, 1), 1024), want);
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

  std::lock_guard<std::mutex> ws_lock(g_ws_mutex);
  Workspace &ws = g_ws[prm->device];
  if (!ws.buf.empty()) {
    // buffers of an earlier call: still this context's device memory? (a
    // device reset in between drops them)
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, ws.buf[0]) != cudaSuccess || at.type != cudaMemoryTypeDevice) {
      cudaGetLastError();
      ws = Workspace();
    }
  }
  R.ws = &ws;
  cudaError_t e = cudaSuccess;
  if (!ws.s) e = cudaStreamCreateWithFlags(&ws.s, cudaStreamNonBlocking);
  if (e == cudaSuccess && !ws.hflag) e = cudaMallocHost((void **)&ws.hflag, 2 * sizeof(int));
  R.s = ws.s;
  R.hflag = ws.hflag;
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
  if (e == cudaSuccess) e = R.alloc(&R.nbr, (size_t)R.maxnb * n);
  if (e == cudaSuccess) e = R.alloc(&R.cnt, n);
  if (e == cudaSuccess) e = R.alloc(&R.qb, n);
  if (e == cudaSuccess) e = R.alloc(&R.flag, 3);
  if (e == cudaSuccess) {
    const int first[3] = {1, 0, 0};  // the first evaluation builds the list; no overflow
    e = cudaMemsetAsync(R.qb, 0, sizeof(double4) * n, R.s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(R.flag, first, sizeof(first), cudaMemcpyHostToDevice, R.s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(R.s);
  }
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
  R.rows.nbr = R.nbr;
  R.rows.cnt = R.cnt;

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
  if (!grad) return R.rows_overflowed() ? MDG_ERR_CAPACITY : MDG_OK;
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
      R.prepare(qh);
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
  return R.rows_overflowed() ? MDG_ERR_CAPACITY : MDG_OK;
}

}  // extern "C"
