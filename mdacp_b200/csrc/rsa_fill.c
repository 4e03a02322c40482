/*
 * Random sequential addition of points in a periodic box, for the seeded
 * liquid-vapour slab workload (mdacp_b200/workloads.py): candidates are
 * drawn uniformly inside an axis-aligned region and kept when no kept point
 * (in the whole periodic box) is closer than r_min.  A cell grid of side
 * >= r_min holds the kept points; a candidate is tested against the 27
 * cells around its own.  Deterministic for a given seed (splitmix64 +
 * xoshiro256**, Blackman & Vigna).  Host-side workload generation only.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  uint64_t s[4];
} rng_t;

static uint64_t splitmix64(uint64_t *x) {
  uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t next_u64(rng_t *r) {
  const uint64_t result = rotl(r->s[1] * 5, 7) * 9;
  const uint64_t t = r->s[1] << 17;
  r->s[2] ^= r->s[0];
  r->s[3] ^= r->s[1];
  r->s[1] ^= r->s[2];
  r->s[0] ^= r->s[3];
  r->s[2] ^= t;
  r->s[3] = rotl(r->s[3], 45);
  return result;
}

static double next_unit(rng_t *r) { return (double)(next_u64(r) >> 11) * 0x1.0p-53; }

enum { SLOTS = 8 };

typedef struct {
  double L[3];
  int nc[3];
  double cs[3];
  int *cell;   /* nc0*nc1*nc2*SLOTS point indices, -1 empty */
  int *fill;   /* points per cell */
  double *pts; /* kept points, xyz */
  long n;
} grid_t;

static long cell_index(const grid_t *g, const double *x) {
  int c[3];
  for (int d = 0; d < 3; d++) {
    int k = (int)floor(x[d] / g->cs[d]);
    if (k < 0) k = 0;
    if (k >= g->nc[d]) k = g->nc[d] - 1;
    c[d] = k;
  }
  return ((long)c[2] * g->nc[1] + c[1]) * g->nc[0] + c[0];
}

static int overlaps(const grid_t *g, const double *x, double r2min) {
  int c[3];
  for (int d = 0; d < 3; d++) {
    int k = (int)floor(x[d] / g->cs[d]);
    if (k < 0) k = 0;
    if (k >= g->nc[d]) k = g->nc[d] - 1;
    c[d] = k;
  }
  for (int dz = -1; dz <= 1; dz++)
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        const int z = (c[2] + dz + g->nc[2]) % g->nc[2];
        const int y = (c[1] + dy + g->nc[1]) % g->nc[1];
        const int xx = (c[0] + dx + g->nc[0]) % g->nc[0];
        const long idx = ((long)z * g->nc[1] + y) * g->nc[0] + xx;
        for (int s = 0; s < g->fill[idx]; s++) {
          const double *p = g->pts + 3 * (long)g->cell[idx * SLOTS + s];
          double r2 = 0.0;
          for (int d = 0; d < 3; d++) {
            double t = p[d] - x[d];
            t -= g->L[d] * nearbyint(t / g->L[d]);
            r2 += t * t;
          }
          if (r2 < r2min) return 1;
        }
      }
  return 0;
}

/*
 * Fills `out` (count x 3) with points: the first counts[0] uniform in region
 * 0, the next counts[1] in region 1, ... (regions lo/hi are nreg x 3), all at
 * mutual periodic distance >= r_min in the box L.  Returns the number of
 * points placed (less than the total if max_tries candidates ran out).
 */
long mdg_rsa_fill(const double L[3], double r_min, int nreg, const double *lo, const double *hi,
                  const long *counts, uint64_t seed, long max_tries, double *out) {
  grid_t g;
  memset(&g, 0, sizeof g);
  long total = 0;
  for (int k = 0; k < nreg; k++) total += counts[k];
  long ncell = 1;
  for (int d = 0; d < 3; d++) {
    g.L[d] = L[d];
    g.nc[d] = (int)floor(L[d] / r_min);
    if (g.nc[d] < 3) g.nc[d] = 3;
    g.cs[d] = L[d] / g.nc[d];
    ncell *= g.nc[d];
  }
  if (g.cs[0] < r_min || g.cs[1] < r_min || g.cs[2] < r_min) return -1;
  g.cell = (int *)malloc(sizeof(int) * ncell * SLOTS);
  g.fill = (int *)calloc(ncell, sizeof(int));
  g.pts = out;
  rng_t r;
  uint64_t sm = seed;
  for (int k = 0; k < 4; k++) r.s[k] = splitmix64(&sm);
  const double r2min = r_min * r_min;
  long tries = 0;
  for (int reg = 0; reg < nreg; reg++) {
    long placed = 0;
    while (placed < counts[reg] && tries < max_tries) {
      tries++;
      double x[3];
      for (int d = 0; d < 3; d++) x[d] = lo[3 * reg + d] + next_unit(&r) * (hi[3 * reg + d] - lo[3 * reg + d]);
      if (overlaps(&g, x, r2min)) continue;
      const long c = cell_index(&g, x);
      if (g.fill[c] >= SLOTS) continue;
      memcpy(out + 3 * g.n, x, sizeof x);
      g.cell[c * SLOTS + g.fill[c]] = (int)g.n;
      g.fill[c]++;
      g.n++;
      placed++;
    }
  }
  free(g.cell);
  free(g.fill);
  return g.n;
}
