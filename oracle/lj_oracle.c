/*
 * CPU restatement of the MDACP single-domain LJ timestep.  TEST
 * INFRASTRUCTURE ONLY (the oracle); see lj_oracle.h for the file:line map.
 * Compile with -ffp-contract=off: every floating-point expression below keeps
 * the reference's evaluation order and must not be fused.
 */
#include "lj_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { D_LEFT, D_RIGHT, D_BACK, D_FORWARD, D_DOWN, D_UP, MAX_DIR };

typedef struct {
  int *v;
  int64_t n, cap;
} ivec;

static void iv_push(ivec *a, int x) {
  if (a->n == a->cap) {
    a->cap = a->cap ? 2 * a->cap : 1024;
    a->v = (int *)realloc(a->v, (size_t)a->cap * sizeof(int));
  }
  a->v[a->n++] = x;
}

struct ljo_system {
  ljo_params prm;
  double sl;                 /* SearchLength = CUTOFF_LENGTH + BufferLength */
  double c0, c2;             /* smoothed-LJ constants */
  int pn, tn, cap;           /* real atoms, real+ghost atoms, allocation */
  double (*q)[3], (*p)[3];
  int32_t *type;
  int *src;                  /* real source index of each ghost (self for real atoms) */
  ivec border[MAX_DIR];
  /* mesh */
  double msx, msy, msz;
  int mx, my, mz, nmesh;
  int *mesh_index, *mesh_index2, *mesh_np, *particle_position, *sortbuf;
  int sort_cap;
  /* pairs and CSR */
  ivec kp_key, kp_partner;
  int *number_of_partners, *key_pointer, *key_pointer2, *sorted_list;
  int64_t sorted_cap;
  int constructions;
  /* PairList */
  int initialized;
  double buffer;
  int lifetime;
  double (*qb_old)[3];
  double *disp;
  /* integrator */
  double zeta, time;
  uint64_t step_count;
};

/* ---------------------------------------------------------------- storage */
static void ensure_cap(ljo_system *s, int need) {
  if (need <= s->cap) return;
  int nc = s->cap;
  while (nc < need) nc = nc ? nc + nc / 2 + 1024 : 1024;
  s->q = realloc(s->q, (size_t)nc * sizeof(*s->q));
  s->p = realloc(s->p, (size_t)nc * sizeof(*s->p));
  s->type = realloc(s->type, (size_t)nc * sizeof(*s->type));
  s->src = realloc(s->src, (size_t)nc * sizeof(*s->src));
  s->qb_old = realloc(s->qb_old, (size_t)nc * sizeof(*s->qb_old));
  s->disp = realloc(s->disp, (size_t)nc * sizeof(*s->disp));
  s->number_of_partners = realloc(s->number_of_partners, (size_t)nc * sizeof(int));
  s->key_pointer = realloc(s->key_pointer, (size_t)nc * sizeof(int));
  s->key_pointer2 = realloc(s->key_pointer2, (size_t)nc * sizeof(int));
  s->particle_position = realloc(s->particle_position, (size_t)nc * sizeof(int));
  s->sortbuf = realloc(s->sortbuf, (size_t)nc * sizeof(int));
  for (int i = s->cap; i < nc; i++) {
    s->q[i][0] = s->q[i][1] = s->q[i][2] = 0.0;
    s->p[i][0] = s->p[i][1] = s->p[i][2] = 0.0;
    s->type[i] = 0;
    s->src[i] = i;
  }
  s->cap = nc;
}

/* Variables::Variables, src/variables.cc:16-33 */
static void smoothed_constants(double rc, double *c0, double *c2) {
  const double s2 = 1.0 / (rc * rc);
  const double s6 = s2 * s2 * s2;
  const double s8 = s6 * s2;
  const double s12 = s6 * s6;
  const double s14 = s12 * s2;
  *c2 = 6.0 * s14 - 3.0 * s8;
  *c0 = -s12 + s6 - *c2 / s2;
}

/* MeshList::ChangeScale, src/meshlist.cc:40-65, for a rectangle = whole box */
static void change_scale(ljo_system *s) {
  const double wx = s->prm.L[0], wy = s->prm.L[1], wz = s->prm.L[2];
  const double SL = s->sl;
  int msx = (int)(wx / SL);
  int msy = (int)(wy / SL);
  int msz = (int)(wz / SL);
  s->msx = wx / (double)msx;
  s->msy = wy / (double)msy;
  s->msz = wz / (double)msz;
  s->mx = (int)(wx / s->msx) + 2;
  s->my = (int)(wy / s->msy) + 2;
  s->mz = (int)(wz / s->msz) + 2;
  s->nmesh = s->mx * s->my * s->mz;
  free(s->mesh_index);
  free(s->mesh_index2);
  free(s->mesh_np);
  s->mesh_index = calloc((size_t)s->nmesh, sizeof(int));
  s->mesh_index2 = calloc((size_t)s->nmesh, sizeof(int));
  s->mesh_np = calloc((size_t)s->nmesh, sizeof(int));
}

ljo_system *ljo_create(const ljo_params *prm, int n, const double *q, const double *v,
                       const int32_t *id) {
  ljo_system *s = calloc(1, sizeof(*s));
  s->prm = *prm;
  s->sl = prm->rc + prm->buffer_length;
  smoothed_constants(prm->rc, &s->c0, &s->c2);
  ensure_cap(s, n + 1);
  /* MDUnit::AddParticle -> Variables::AddParticle (src/mdunit.cc:60-65,
     src/variables.cc:35-47): only atoms inside [0, L) are kept. */
  for (int i = 0; i < n; i++) {
    const double *x = q + 3 * i;
    int inside = 1;
    for (int d = 0; d < 3; d++) inside &= (0.0 <= x[d] && x[d] < prm->L[d]);
    if (!inside) continue;
    const int k = s->pn++;
    for (int d = 0; d < 3; d++) {
      s->q[k][d] = x[d];
      s->p[k][d] = v[3 * i + d];
    }
    s->type[k] = id[i];
    s->src[k] = k;
  }
  s->tn = s->pn;
  change_scale(s);
  return s;
}

void ljo_destroy(ljo_system *s) {
  if (!s) return;
  free(s->q); free(s->p); free(s->type); free(s->src);
  for (int d = 0; d < MAX_DIR; d++) free(s->border[d].v);
  free(s->mesh_index); free(s->mesh_index2); free(s->mesh_np);
  free(s->particle_position); free(s->sortbuf);
  free(s->kp_key.v); free(s->kp_partner.v);
  free(s->number_of_partners); free(s->key_pointer); free(s->key_pointer2);
  free(s->sorted_list); free(s->qb_old); free(s->disp);
  free(s);
}

/* ------------------------------------------------------ migration and wrap */
/* MDRect::IsOverBoundary, src/mdrect.cc:4-20 (rect = [0, L)) */
static int over_boundary(const ljo_system *s, int dir, const double *x) {
  switch (dir) {
    case D_LEFT: return x[0] < 0.0;
    case D_RIGHT: return x[0] >= s->prm.L[0];
    case D_BACK: return x[1] < 0.0;
    case D_FORWARD: return x[1] >= s->prm.L[1];
    case D_DOWN: return x[2] < 0.0;
    case D_UP: return x[2] >= s->prm.L[2];
  }
  return 0;
}

/* MakeBufferForSendingParticle + ReceiveParticles with the neighbour being
   this same unit (src/mdunit.cc:93-138, src/mdmanager.cc:317-374): atoms over
   the boundary are removed (order of the rest kept) and appended at the end. */
static void send_particles_sub(ljo_system *s, int dir) {
  const int pn = s->pn;
  double (*bq)[3] = malloc((size_t)(pn + 1) * sizeof(*bq));
  double (*bp)[3] = malloc((size_t)(pn + 1) * sizeof(*bp));
  int32_t *bt = malloc((size_t)(pn + 1) * sizeof(int32_t));
  int nb = 0, index = 0;
  for (int i = 0; i < pn; i++) {
    if (over_boundary(s, dir, s->q[i])) {
      memcpy(bq[nb], s->q[i], sizeof(bq[nb]));
      memcpy(bp[nb], s->p[i], sizeof(bp[nb]));
      bt[nb] = s->type[i];
      nb++;
    } else {
      memmove(s->q[index], s->q[i], sizeof(s->q[index]));
      memmove(s->p[index], s->p[i], sizeof(s->p[index]));
      s->type[index] = s->type[i];
      index++;
    }
  }
  for (int k = 0; k < nb; k++) {
    memcpy(s->q[index], bq[k], sizeof(bq[k]));
    memcpy(s->p[index], bp[k], sizeof(bp[k]));
    s->type[index] = bt[k];
    index++;
  }
  s->pn = index;
  free(bq); free(bp); free(bt);
}

/* Variables::AdjustPeriodicBoundary, src/variables.cc:63-84 */
static int adjust_periodic_boundary(ljo_system *s) {
  for (int i = 0; i < s->pn; i++) {
    for (int d = 0; d < 3; d++) {
      if (s->q[i][d] < 0.0) {
        s->q[i][d] += s->prm.L[d];
      } else if (s->q[i][d] > s->prm.L[d]) {
        s->q[i][d] -= s->prm.L[d];
      }
    }
  }
  for (int i = 0; i < s->pn; i++)
    for (int d = 0; d < 3; d++)
      if (s->q[i][d] < 0.0 || s->q[i][d] > s->prm.L[d]) return -1; /* "Invalid position" */
  return 0;
}

/* ----------------------------------------------------------------- ghosts */
/* MDRect::IsInsideEdge, src/mdrect.cc:23-47 */
static int inside_edge(const ljo_system *s, int dir, const double *x) {
  const double SL = s->sl;
  switch (dir) {
    case D_LEFT: return x[0] < 0.0 + SL && x[0] > 0.0;
    case D_RIGHT: return x[0] > s->prm.L[0] - SL && x[0] < s->prm.L[0];
    case D_BACK: return x[1] < 0.0 + SL && x[1] > 0.0;
    case D_FORWARD: return x[1] > s->prm.L[1] - SL && x[1] < s->prm.L[1];
    case D_DOWN: return x[2] < 0.0 + SL && x[2] > 0.0;
    case D_UP: return x[2] > s->prm.L[2] - SL && x[2] < s->prm.L[2];
  }
  return 0;
}

/* MDUnit::FindBorderParticles, src/mdunit.cc:140-150 (over real + ghosts so far) */
static void find_border_particles(ljo_system *s, int dir) {
  s->border[dir].n = 0;
  for (int i = 0; i < s->tn; i++)
    if (inside_edge(s, dir, s->q[i])) iv_push(&s->border[dir], i);
}

/* MakeBufferForBorderParticles + ReceiveBorderParticles for a single unit
   (src/mdunit.cc:152-208): every face is a periodic boundary, so the copy is
   shifted by +-L along the direction's axis; the ghost coordinate is
   q[j][d] + diff[d] for every component. */
static void send_border_particles_sub(ljo_system *s, int dir) {
  double diff[3] = {0.0, 0.0, 0.0};
  switch (dir) {
    case D_LEFT: diff[0] = s->prm.L[0]; break;
    case D_RIGHT: diff[0] -= s->prm.L[0]; break;
    case D_BACK: diff[1] = s->prm.L[1]; break;
    case D_FORWARD: diff[1] = -s->prm.L[1]; break;
    case D_DOWN: diff[2] = s->prm.L[2]; break;
    case D_UP: diff[2] = -s->prm.L[2]; break;
  }
  const ivec *b = &s->border[dir];
  const int base = s->tn;
  ensure_cap(s, base + (int)b->n + 1);
  for (int64_t k = 0; k < b->n; k++) {
    const int j = b->v[k];
    const int g = base + (int)k;
    s->q[g][0] = s->q[j][0] + diff[0];
    s->q[g][1] = s->q[j][1] + diff[1];
    s->q[g][2] = s->q[j][2] + diff[2];
    s->src[g] = s->src[j];
  }
  s->tn = base + (int)b->n;
}

/* MDManager::SendBorderParticles, src/mdmanager.cc:419-429 */
static void send_border_particles(ljo_system *s) {
  s->tn = s->pn;
  for (int dir = 0; dir < MAX_DIR; dir++) send_border_particles_sub(s, dir);
}

/* ------------------------------------------------------------------- mesh */
static int pos2index(const ljo_system *s, int ix, int iy, int iz) {
  return s->mx * s->my * iz + s->mx * iy + ix;
}

/* MeshList::MakeMesh, src/meshlist.cc:175-228 */
static int make_mesh(ljo_system *s) {
  const int pn = s->tn;
  const double imx = 1.0 / s->msx, imy = 1.0 / s->msy, imz = 1.0 / s->msz;
  for (int i = 0; i < s->nmesh; i++) s->mesh_np[i] = 0;
  for (int i = 0; i < pn; i++) {
    int ix = (int)((s->q[i][0] - 0.0) * imx) + 1;
    int iy = (int)((s->q[i][1] - 0.0) * imy) + 1;
    int iz = (int)((s->q[i][2] - 0.0) * imz) + 1;
    if (ix < 0) ix = s->mx - 1;
    else if (ix >= s->mx) ix = 0;
    if (iy < 0) iy = s->my - 1;
    else if (iy >= s->my) iy = 0;
    if (iz < 0) iz = s->mz - 1;
    else if (iz >= s->mz) iz = 0;
    const int index = s->mx * s->my * iz + s->mx * iy + ix;
    if (index >= s->nmesh || index < 0) return -1; /* "Invalid index" */
    s->particle_position[i] = index;
    s->mesh_np[index]++;
  }
  s->mesh_index[0] = 0;
  int sum = 0;
  for (int i = 0; i < s->nmesh - 1; i++) {
    sum += s->mesh_np[i];
    s->mesh_index[i + 1] = sum;
  }
  for (int i = 0; i < s->nmesh; i++) s->mesh_index2[i] = 0;
  for (int i = 0; i < pn; i++) {
    const int index = s->particle_position[i];
    const int j = s->mesh_index[index] + s->mesh_index2[index];
    s->sortbuf[j] = i;
    s->mesh_index2[index]++;
  }
  return 0;
}

/* MeshList::AppendList, src/meshlist.cc:230-240 */
static void append_list(const ljo_system *s, int ix, int iy, int iz, ivec *v) {
  if (ix < 0 || ix >= s->mx) return;
  if (iy < 0 || iy >= s->my) return;
  if (iz < 0 || iz >= s->mz) return;
  const int index = pos2index(s, ix, iy, iz);
  const int in = s->mesh_np[index];
  const int mi = s->mesh_index[index];
  for (int k = 0; k < in; k++) iv_push(v, s->sortbuf[mi + k]);
}

/* MeshList::RegisterPair, src/meshlist.cc:555-583 (half list, plain build) */
static void register_pair(ljo_system *s, int index1, int index2) {
  int i1, i2;
  if (index1 < index2) {
    i1 = index1;
    i2 = index2;
  } else {
    i1 = index2;
    i2 = index1;
  }
  iv_push(&s->kp_key, i1);
  iv_push(&s->kp_partner, i2);
  s->number_of_partners[i1]++;
}

/* MeshList::SearchMesh, src/meshlist.cc:242-292 */
static void search_mesh(ljo_system *s, int index, ivec *v) {
  int ix = index % s->mx;
  int rest = index / s->mx;
  int iy = rest % s->my;
  int iz = rest / s->my;
  v->n = 0;
  append_list(s, ix, iy, iz, v);
  append_list(s, ix + 1, iy, iz, v);
  append_list(s, ix - 1, iy + 1, iz, v);
  append_list(s, ix, iy + 1, iz, v);
  append_list(s, ix + 1, iy + 1, iz, v);
  append_list(s, ix - 1, iy, iz + 1, v);
  append_list(s, ix, iy, iz + 1, v);
  append_list(s, ix + 1, iy, iz + 1, v);
  append_list(s, ix - 1, iy - 1, iz + 1, v);
  append_list(s, ix, iy - 1, iz + 1, v);
  append_list(s, ix + 1, iy - 1, iz + 1, v);
  append_list(s, ix - 1, iy + 1, iz + 1, v);
  append_list(s, ix, iy + 1, iz + 1, v);
  append_list(s, ix + 1, iy + 1, iz + 1, v);
  const double S2 = s->sl * s->sl;
  const int pn = s->pn;
  const int in = s->mesh_np[index];
  const int64_t ln = v->n;
  for (int i = 0; i < in; i++) {
    const int i1 = v->v[i];
    const double x1 = s->q[i1][0], y1 = s->q[i1][1], z1 = s->q[i1][2];
    for (int64_t j = i + 1; j < ln; j++) {
      const int i2 = v->v[j];
      if (i1 >= pn && i2 >= pn) continue;
      const double dx = x1 - s->q[i2][0];
      const double dy = y1 - s->q[i2][1];
      const double dz = z1 - s->q[i2][2];
      const double r2 = (dx * dx + dy * dy + dz * dz);
      if (r2 > S2) continue;
      register_pair(s, i1, i2);
    }
  }
}

/* MeshList::MakeList, src/meshlist.cc:67-104 (no particle Sort: SortParticle=no) */
static int make_list(ljo_system *s) {
  const int pn = s->tn;
  s->kp_key.n = s->kp_partner.n = 0;
  for (int i = 0; i < pn; i++) s->number_of_partners[i] = 0;
  if (make_mesh(s) != 0) return -1;
  ivec v = {0};
  for (int i = 0; i < s->nmesh; i++) search_mesh(s, i, &v);
  free(v.v);
  const int64_t np = s->kp_key.n;
  int pos = 0;
  s->key_pointer[0] = 0;
  for (int i = 0; i < pn - 1; i++) {
    pos += s->number_of_partners[i];
    s->key_pointer[i + 1] = pos;
  }
  for (int i = 0; i < pn; i++) s->key_pointer2[i] = 0;
  if (np + 1 > s->sorted_cap) {
    s->sorted_cap = np + 1;
    s->sorted_list = realloc(s->sorted_list, (size_t)s->sorted_cap * sizeof(int));
  }
  for (int64_t k = 0; k < np; k++) {
    const int i = s->kp_key.v[k];
    const int j = s->kp_partner.v[k];
    const int index = s->key_pointer[i] + s->key_pointer2[i];
    s->sorted_list[index] = j;
    s->key_pointer2[i]++;
  }
  /* CalculateForceNext reads one entry past a row; the padding entry is atom 0. */
  s->sorted_list[np] = 0;
  s->constructions++;
  return 0;
}

/* PairList::Init, src/pairlist.cc:10-23 */
static void pairlist_init(ljo_system *s) {
  s->initialized = 1;
  s->buffer = s->prm.buffer_length;
  s->lifetime = 0;
  for (int i = 0; i < s->tn; i++) {
    s->qb_old[i][0] = s->q[i][0];
    s->qb_old[i][1] = s->q[i][1];
    s->qb_old[i][2] = s->q[i][2];
  }
}

/* MDManager::MakePairList, src/mdmanager.cc:387-417, for one unit */
int ljo_make_pairlist(ljo_system *s) {
  for (int dir = 0; dir < MAX_DIR; dir++) send_particles_sub(s, dir);
  if (adjust_periodic_boundary(s) != 0) return -1;
  for (int i = 0; i < s->pn; i++) s->src[i] = i;
  s->tn = s->pn;
  for (int dir = 0; dir < MAX_DIR; dir++) {
    find_border_particles(s, dir);
    send_border_particles_sub(s, dir);
  }
  pairlist_init(s);
  return make_list(s);
}

/* ------------------------------------------------------- pairlist validity */
/* PairList::UpdatePairListValidity, src/pairlist.cc:47-65 */
static int update_validity(ljo_system *s) {
  double vmax = s->p[0][0] * s->p[0][0] + s->p[0][1] * s->p[0][1] + s->p[0][2] * s->p[0][2];
  for (int i = 1; i < s->pn; i++) {
    double v = s->p[i][0] * s->p[i][0] + s->p[i][1] * s->p[i][1] + s->p[i][2] * s->p[i][2];
    if (v > vmax) vmax = v;
  }
  vmax = sqrt(vmax);
  if (vmax * 2.0 * s->prm.dt > s->prm.buffer_length) return -1; /* "Too fast particles" */
  s->buffer = s->buffer - vmax * 2.0 * s->prm.dt;
  return 0;
}

/* PairList::CheckByDisplacement, src/pairlist.cc:67-121 */
static int check_by_displacement(ljo_system *s) {
  const int pn = s->tn;
  double dr2_max = 0.0;
  for (int i = 0; i < pn; i++) {
    double dx = s->qb_old[i][0] - s->q[i][0];
    double dy = s->qb_old[i][1] - s->q[i][1];
    double dz = s->qb_old[i][2] - s->q[i][2];
    double dr2 = dx * dx + dy * dy + dz * dz;
    s->disp[i] = dr2;
    if (dr2_max < dr2) dr2_max = dr2;
  }
  const int Nl = (pn > s->prm.check_list_length) ? s->prm.check_list_length : pn;
  ivec v = {0};
  const double c_distance = s->prm.buffer_length - sqrt(dr2_max);
  const double c_d2 = c_distance * c_distance;
  for (int i = 0; i < pn; i++) {
    if (s->disp[i] > c_d2) {
      iv_push(&v, i);
      if ((int)v.n >= Nl) {
        free(v.v);
        return 1;
      }
    }
  }
  const double SL2 = s->sl * s->sl;
  const double CL2 = s->prm.rc * s->prm.rc;
  const int l = (int)v.n;
  int expired = 0;
  for (int i = 0; i < l - 1 && !expired; i++) {
    for (int j = i + 1; j < l; j++) {
      int i1 = v.v[i], i2 = v.v[j];
      double dx = s->qb_old[i1][0] - s->qb_old[i2][0];
      double dy = s->qb_old[i1][1] - s->qb_old[i2][1];
      double dz = s->qb_old[i1][2] - s->qb_old[i2][2];
      double dr2 = dx * dx + dy * dy + dz * dz;
      if (dr2 < SL2) continue;
      dx = s->q[i1][0] - s->q[i2][0];
      dy = s->q[i1][1] - s->q[i2][1];
      dz = s->q[i1][2] - s->q[i2][2];
      dr2 = dx * dx + dy * dy + dz * dz;
      if (dr2 < CL2) {
        expired = 1;
        break;
      }
    }
  }
  free(v.v);
  return expired;
}

/* PairList::IsPairListExpired, src/pairlist.cc:25-45.  Returns 1/0, -1 on error. */
static int is_expired(ljo_system *s) {
  if (!s->initialized) return 1;
  s->lifetime++;
  if (s->buffer > 0.0) {
    if (update_validity(s) != 0) return -1;
  }
  if (s->buffer < 0.0) return check_by_displacement(s);
  return 0;
}

/* -------------------------------------------------------------- integrate */
/* ForceCalculator::UpdatePositionHalf, src/fcalculator.cc:17-30 */
static void update_position_half(ljo_system *s) {
  const double dt2 = s->prm.dt * 0.5;
  for (int i = 0; i < s->pn; i++) {
    s->q[i][0] += s->p[i][0] * dt2;
    s->q[i][1] += s->p[i][1] * dt2;
    s->q[i][2] += s->p[i][2] * dt2;
  }
}

/* ForceCalculator::CalculateForceNext, src/fcalculator.cc:228-290: the kick of
   pair k is applied while the distance of pair k+1 is formed. */
static void calculate_force_next(ljo_system *s, double dt) {
  const double CL2 = s->prm.rc * s->prm.rc;
  const double C2 = s->c2 * 8.0;
  double (*q)[3] = s->q;
  double (*p)[3] = s->p;
  const int pn = s->pn;
  const int *sorted_list = s->sorted_list;
  for (int i = 0; i < pn; i++) {
    const double qx_key = q[i][0], qy_key = q[i][1], qz_key = q[i][2];
    double pfx = 0, pfy = 0, pfz = 0;
    const int kp = s->key_pointer[i];
    int ja = sorted_list[kp];
    double dxa = q[ja][0] - qx_key;
    double dya = q[ja][1] - qy_key;
    double dza = q[ja][2] - qz_key;
    double df = 0.0;
    double dxb = 0.0, dyb = 0.0, dzb = 0.0;
    int jb = 0;
    const int np = s->number_of_partners[i];
    for (int k = kp; k < np + kp; k++) {
      const double dx = dxa, dy = dya, dz = dza;
      double r2 = (dx * dx + dy * dy + dz * dz);
      const int j = ja;
      ja = sorted_list[k + 1];
      dxa = q[ja][0] - qx_key;
      dya = q[ja][1] - qy_key;
      dza = q[ja][2] - qz_key;
      if (r2 > CL2) continue;
      pfx += df * dxb;
      pfy += df * dyb;
      pfz += df * dzb;
      p[jb][0] -= df * dxb;
      p[jb][1] -= df * dyb;
      p[jb][2] -= df * dzb;
      const double r6 = r2 * r2 * r2;
      df = ((24.0 * r6 - 48.0) / (r6 * r6 * r2) + C2) * dt;
      jb = j;
      dxb = dx;
      dyb = dy;
      dzb = dz;
    }
    p[jb][0] -= df * dxb;
    p[jb][1] -= df * dyb;
    p[jb][2] -= df * dzb;
    p[i][0] += pfx + df * dxb;
    p[i][1] += pfy + df * dyb;
    p[i][2] += pfz + df * dzb;
  }
}

/* KineticEnergyObserver, src/observer.cc:4-15 */
static double kinetic_sum(const ljo_system *s) {
  double e = 0;
  for (int i = 0; i < s->pn; i++)
    for (int d = 0; d < 3; d++) e += 0.5 * s->p[i][d] * s->p[i][d];
  return e;
}

/* MDManager::Temperature = KineticEnergy()/1.5, src/mdmanager.cc:530-548 */
static double temperature(const ljo_system *s) {
  return kinetic_sum(s) / (double)s->pn / 1.5;
}

/* ForceCalculator::HeatbathZeta / HeatbathMomenta, src/fcalculator.cc:979-999 */
static void heatbath_zeta(ljo_system *s, double t) {
  const double dt2 = s->prm.dt * 0.5;
  const double tau = s->prm.heatbath_tau;
  double t1 = (t - s->prm.aimed_temperature) / (tau * tau);
  s->zeta += t1 * dt2;
}
static void heatbath_momenta(ljo_system *s) {
  const double dt2 = s->prm.dt * 0.5;
  const double exp1 = exp(-dt2 * s->zeta);
  for (int i = 0; i < s->pn; i++)
    for (int d = 0; d < 3; d++) s->p[i][d] *= exp1;
}

/* ---------------------------------------------------------- Philox noise */
static inline void mulhilo32(uint32_t a, uint32_t b, uint32_t *hi, uint32_t *lo) {
  const uint64_t prod = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(prod >> 32);
  *lo = (uint32_t)prod;
}

void ljo_philox4x32(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; r++) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo32(0xD2511F53u, c0, &hi0, &lo0);
    mulhilo32(0xCD9E8D57u, c2, &hi1, &lo1);
    const uint32_t n0 = hi1 ^ c1 ^ k0;
    const uint32_t n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Counter (id, step lo, step hi, tag) under key (seed lo, seed hi); the four
   32-bit words become uniforms in (0,1) and two Box-Muller pairs; three
   normals are used. */
void ljo_langevin_normals(uint64_t seed, uint32_t id, uint64_t step, double z[3]) {
  const uint32_t ctr[4] = {id, (uint32_t)step, (uint32_t)(step >> 32), 0x4C414E47u};
  const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  uint32_t o[4];
  ljo_philox4x32(ctr, key, o);
  const double scale = 2.3283064365386963e-10; /* 2^-32 */
  const double u0 = ((double)o[0] + 0.5) * scale;
  const double u1 = ((double)o[1] + 0.5) * scale;
  const double u2 = ((double)o[2] + 0.5) * scale;
  const double u3 = ((double)o[3] + 0.5) * scale;
  const double twopi = 6.283185307179586;
  const double r0 = sqrt(-2.0 * log(u0));
  const double r1 = sqrt(-2.0 * log(u2));
  z[0] = r0 * cos(twopi * u1);
  z[1] = r0 * sin(twopi * u1);
  z[2] = r1 * cos(twopi * u3);
}

/* ForceCalculator::Langevin, src/fcalculator.cc:1001-1017, with Philox noise */
static void langevin(ljo_system *s) {
  const double dt = s->prm.dt;
  const double hb_gamma = s->prm.heatbath_gamma;
  const double T = s->prm.aimed_temperature;
  const double hb_D = sqrt(2.0 * hb_gamma * T / dt);
  for (int i = 0; i < s->pn; i++) {
    double z[3];
    ljo_langevin_normals(s->prm.seed, (uint32_t)s->type[i], s->step_count, z);
    for (int d = 0; d < 3; d++) {
      const double r = hb_D * z[d];
      s->p[i][d] += (-hb_gamma * s->p[i][d] + r) * dt;
    }
  }
}

/* MDManager::Calculate, src/mdmanager.cc:153-186, and its three force branches
   CalculateForce (:226-252), CalculateNoseHoover (:254-287),
   CalculateLangevin (:289-315, which has no second half drift). */
int ljo_step(ljo_system *s, int nsteps) {
  for (int k = 0; k < nsteps; k++) {
    const int e = is_expired(s);
    if (e < 0) return -1;
    if (e) {
      if (ljo_make_pairlist(s) != 0) return -1;
    }
    update_position_half(s);
    send_border_particles(s);
    if (s->prm.thermostat == LJO_NOSE_HOOVER) {
      heatbath_zeta(s, temperature(s));
      heatbath_momenta(s);
      calculate_force_next(s, s->prm.dt);
      heatbath_momenta(s);
      heatbath_zeta(s, temperature(s));
      update_position_half(s);
    } else if (s->prm.thermostat == LJO_LANGEVIN) {
      calculate_force_next(s, s->prm.dt);
      langevin(s);
    } else {
      calculate_force_next(s, s->prm.dt);
      update_position_half(s);
    }
    s->time += s->prm.dt;
    s->step_count++;
  }
  return 0;
}

/* ------------------------------------------------------------ executors */
/* The reference's wall term: df of a pair at distance d, the pair force's
   expression with the separately rounded operations (src/rankine.cc:78-82,
   src/burst.cc:91-93). */
static double wall_df(double d, double c2, double dt) {
  const double r2 = d * d;
  const double r6 = r2 * r2 * r2;
  return ((24.0 * r6 - 48.0) / (r6 * r6 * r2) + c2 * 8.0) * dt;
}

double ljo_apply_external(ljo_system *s, ljo_external *e) {
  double impulse = 0.0;
  const double CL = s->prm.rc;
  if (e->kind == 1) {
    for (int i = 0; i < s->pn; i++) s->p[i][e->axis] += e->strength * e->time_step;
  } else if (e->kind == 2) {
    for (int i = 0; i < s->pn; i++) {
      if (s->q[i][2] < CL) {
        const double dz = s->q[i][2];
        const double df = wall_df(dz, s->c2, e->time_step);
        s->p[i][2] -= df * dz;
      }
      if (s->q[i][2] > e->position) {
        const double dz = e->position - s->q[i][2] + CL;
        const double df = wall_df(dz, s->c2, e->time_step);
        s->p[i][2] += df * dz;
        impulse -= df * dz;
      }
    }
    e->position -= e->velocity;
  } else if (e->kind == 3) {
    const double CL2 = CL * CL;
    for (int i = 0; i < s->pn; i++) {
      const double dx = s->q[i][0] - e->center[0];
      const double dy = s->q[i][1] - e->center[1];
      const double dz = s->q[i][2] - e->center[2];
      const double r = e->radius - sqrt(dx * dx + dy * dy + dz * dz);
      if (r * r > CL2) continue;
      const double df = wall_df(r, s->c2, e->time_step);
      s->p[i][0] += df * dx;
      s->p[i][1] += df * dy;
      s->p[i][2] += df * dz;
    }
  }
  return impulse;
}

/* ------------------------------------------------------------ accessors */
int ljo_particle_number(const ljo_system *s) { return s->pn; }
int ljo_total_particle_number(const ljo_system *s) { return s->tn; }
int64_t ljo_pair_number(const ljo_system *s) { return s->kp_key.n; }
int ljo_constructions(const ljo_system *s) { return s->constructions; }
double ljo_zeta(const ljo_system *s) { return s->zeta; }

void ljo_get_state(const ljo_system *s, double *q, double *v, int32_t *id) {
  for (int i = 0; i < s->pn; i++) {
    for (int d = 0; d < 3; d++) {
      if (q) q[3 * i + d] = s->q[i][d];
      if (v) v[3 * i + d] = s->p[i][d];
    }
    if (id) id[i] = s->type[i];
  }
}

int64_t ljo_get_pairs(const ljo_system *s, int32_t *key_id, int32_t *partner_id, int64_t cap) {
  int64_t n = 0;
  for (int64_t k = 0; k < s->kp_key.n; k++) {
    const int a = s->kp_key.v[k], b = s->kp_partner.v[k];
    if (a < s->pn && b < s->pn) {
      if (n < cap) { key_id[n] = s->type[a]; partner_id[n] = s->type[b]; }
      n++;
      if (n < cap) { key_id[n] = s->type[b]; partner_id[n] = s->type[a]; }
      n++;
    } else {
      const int real = a < s->pn ? a : b;
      const int ghost = a < s->pn ? b : a;
      if (n < cap) { key_id[n] = s->type[real]; partner_id[n] = s->type[s->src[ghost]]; }
      n++;
    }
  }
  return n;
}

void ljo_forces(ljo_system *s, double *f) {
  double (*save)[3] = malloc((size_t)s->tn * sizeof(*save));
  memcpy(save, s->p, (size_t)s->tn * sizeof(*save));
  for (int i = 0; i < s->tn; i++) s->p[i][0] = s->p[i][1] = s->p[i][2] = 0.0;
  calculate_force_next(s, 1.0);
  for (int i = 0; i < s->pn; i++)
    for (int d = 0; d < 3; d++) f[3 * i + d] = s->p[i][d];
  memcpy(s->p, save, (size_t)s->tn * sizeof(*save));
  free(save);
}

/* PotentialEnergyObserver / VirialObserver, src/observer.cc:17-79 (half list) */
void ljo_observe(const ljo_system *s, double *ke, double *pe, double *virial) {
  const double CL2 = s->prm.rc * s->prm.rc;
  const double C2 = s->c2, C0 = s->c0;
  const int pn = s->pn;
  double energy = 0.0, phi = 0.0;
  for (int64_t k = 0; k < s->kp_key.n; k++) {
    const int i = s->kp_key.v[k], j = s->kp_partner.v[k];
    double dx = s->q[i][0] - s->q[j][0];
    double dy = s->q[i][1] - s->q[j][1];
    double dz = s->q[i][2] - s->q[j][2];
    const double r2 = (dx * dx + dy * dy + dz * dz);
    if (r2 > CL2) continue;
    double e = 4.0 * (1.0 / (r2 * r2 * r2 * r2 * r2 * r2) - 1.0 / (r2 * r2 * r2) + C2 * r2 + C0);
    if (i >= pn || j >= pn) e *= 0.5;
    energy += e;
  }
  for (int64_t k = 0; k < s->kp_key.n; k++) {
    const int i = s->kp_key.v[k], j = s->kp_partner.v[k];
    double dx = s->q[j][0] - s->q[i][0];
    double dy = s->q[j][1] - s->q[i][1];
    double dz = s->q[j][2] - s->q[i][2];
    const double r2 = (dx * dx + dy * dy + dz * dz);
    if (r2 > CL2) continue;
    const double r6 = r2 * r2 * r2;
    double df = ((24.0 * r6 - 48.0) / (r6 * r6 * r2) + C2 * 8.0) * r2;
    if (i >= pn || j >= pn) df *= 0.5;
    phi += df;
  }
  if (ke) *ke = kinetic_sum(s);
  if (pe) *pe = energy;
  if (virial) *virial = phi / 3.0;
}

/* Neumaier's compensated sum (a running sum plus a correction term): the
   checker's own summation error stays near one rounding however many terms
   are added, where a plain running sum of n terms can drift by up to n
   roundings when the terms are alike (a lattice). */
typedef struct { double s, c; } ljo_csum;
static void csum_add(ljo_csum *a, double x) {
  const double t = a->s + x;
  if (fabs(a->s) >= fabs(x)) a->c += (a->s - t) + x;
  else a->c += (x - t) + a->s;
  a->s = t;
}

/* The sums of ljo_observe, each term formed exactly as there (the reference's
   expression trees), added with compensation.  Test infrastructure: the
   checker for sums over millions of pairs, where the reference's own running
   sum carries more rounding than the 1e-12 parity bar allows. */
void ljo_observe_compensated(const ljo_system *s, double *ke, double *pe, double *virial) {
  const double CL2 = s->prm.rc * s->prm.rc;
  const double C2 = s->c2, C0 = s->c0;
  const int pn = s->pn;
  ljo_csum energy = {0.0, 0.0}, phi = {0.0, 0.0}, kin = {0.0, 0.0};
  for (int64_t k = 0; k < s->kp_key.n; k++) {
    const int i = s->kp_key.v[k], j = s->kp_partner.v[k];
    double dx = s->q[i][0] - s->q[j][0];
    double dy = s->q[i][1] - s->q[j][1];
    double dz = s->q[i][2] - s->q[j][2];
    const double r2 = (dx * dx + dy * dy + dz * dz);
    if (r2 > CL2) continue;
    double e = 4.0 * (1.0 / (r2 * r2 * r2 * r2 * r2 * r2) - 1.0 / (r2 * r2 * r2) + C2 * r2 + C0);
    if (i >= pn || j >= pn) e *= 0.5;
    csum_add(&energy, e);
  }
  for (int64_t k = 0; k < s->kp_key.n; k++) {
    const int i = s->kp_key.v[k], j = s->kp_partner.v[k];
    double dx = s->q[j][0] - s->q[i][0];
    double dy = s->q[j][1] - s->q[i][1];
    double dz = s->q[j][2] - s->q[i][2];
    const double r2 = (dx * dx + dy * dy + dz * dz);
    if (r2 > CL2) continue;
    const double r6 = r2 * r2 * r2;
    double df = ((24.0 * r6 - 48.0) / (r6 * r6 * r2) + C2 * 8.0) * r2;
    if (i >= pn || j >= pn) df *= 0.5;
    csum_add(&phi, df);
  }
  for (int i = 0; i < pn; i++)
    for (int d = 0; d < 3; d++) csum_add(&kin, 0.5 * s->p[i][d] * s->p[i][d]);
  if (ke) *ke = kin.s + kin.c;
  if (pe) *pe = energy.s + energy.c;
  if (virial) *virial = (phi.s + phi.c) / 3.0;
}
