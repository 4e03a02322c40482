// Drop-in Variables (interface of include/variables.h:12-49 in the reference).
#include "variables.h"

#include <assert.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cstdlib>
#include <fstream>
#include <random>

#include "mpistream.h"

void mdg_check(mdg_handle *h, mdg_status s, const char *what) {
  if (s == MDG_OK) return;
  // the reference's error convention: show_error + exit(1) (include/mdconfig.h:37)
  mout << "# Error at " << what << std::endl;
  mout << mdg_status_string(s) << ": " << (h ? mdg_last_error(h) : "") << std::endl;
  exit(1);
}

Variables::Variables(void) : Variables(N) {}

Variables::Variables(int capacity_)
    : particle_number(0), total_particle_number(0), capacity(capacity_), device(nullptr),
      host_dirty(false), momenta_dirty(false), device_newer(false), pending_steps(0), Zeta(0.0), SimulationTime(0.0) {
  // smoothed-LJ constants (src/variables.cc:21-27)
  const double s2 = 1.0 / (CUTOFF_LENGTH * CUTOFF_LENGTH);
  const double s6 = s2 * s2 * s2;
  const double s8 = s6 * s2;
  const double s12 = s6 * s6;
  const double s14 = s12 * s2;
  C2 = 6.0 * s14 - 3.0 * s8;
  C0 = -s12 + s6 - C2 / s2;
  q = static_cast<double(*)[D]>(aligned_alloc(64, sizeof(double) * D * (size_t)capacity));
  p = static_cast<double(*)[D]>(aligned_alloc(64, sizeof(double) * D * (size_t)capacity));
  type = static_cast<int *>(malloc(sizeof(int) * (size_t)capacity));
  memset(q, 0, sizeof(double) * D * (size_t)capacity);
  memset(p, 0, sizeof(double) * D * (size_t)capacity);
  memset(type, 0, sizeof(int) * (size_t)capacity);
}

Variables::~Variables(void) {
  free(q);
  free(p);
  free(type);
}

void Variables::AddParticle(double x[D], double v[D], int t) {
  if (particle_number >= capacity) {
    mout << "# Error: more particles than Capacity=" << capacity << std::endl;
    exit(1);
  }
  q[particle_number][X] = x[X];
  q[particle_number][Y] = x[Y];
  q[particle_number][Z] = x[Z];
  q[particle_number][3] = 0.0;
  p[particle_number][X] = v[X];
  p[particle_number][Y] = v[Y];
  p[particle_number][Z] = v[Z];
  p[particle_number][3] = 0.0;
  type[particle_number] = t;
  particle_number++;
  total_particle_number = particle_number;
  host_dirty = true;
}

void Variables::SaveConfiguration(std::ostream &fs) {
  for (int i = 0; i < particle_number; i++) {
    fs << q[i][X] << " " << q[i][Y] << " " << q[i][Z] << " " << p[i][X] << " " << p[i][Y] << " "
       << p[i][Z] << "\n";
  }
}

// Same wrap as the reference (src/variables.cc:63-84); the device applies it
// at every pairlist construction, this host version serves direct callers.
void Variables::AdjustPeriodicBoundary(SimulationInfo *sinfo) {
  for (int i = 0; i < particle_number; i++) {
    for (int d = 0; d < 3; d++) {
      if (q[i][d] < 0.0) q[i][d] += sinfo->L[d];
      else if (q[i][d] > sinfo->L[d]) q[i][d] -= sinfo->L[d];
    }
  }
  for (int i = 0; i < particle_number; i++) {
    for (int d = 0; d < 3; d++) {
      if (q[i][d] < 0.0 || q[i][d] > sinfo->L[d]) {
        mout << "# Error: Invalid position" << std::endl;
        printf("%f: %d %d %f\n", SimulationTime, i, d, q[i][d]);
        exit(1);
      }
    }
  }
  host_dirty = true;
}

// Initial velocities: speed V0 in a uniformly random direction from
// std::mt19937(seed), then the mean removed -- the reference's generator
// (src/variables.cc:86-113), so seeded runs start from the same state.
void Variables::SetInitialVelocity(const double V0, const int seed) {
  std::mt19937 mt(seed);
  std::uniform_real_distribution<double> ud(0.0, 1.0);
  for (int i = 0; i < particle_number; i++) {
    double z = ud(mt) * 2.0 - 1.0;
    double phi = ud(mt) * 2.0 * M_PI;
    p[i][X] = V0 * sqrt(1 - z * z) * cos(phi);
    p[i][Y] = V0 * sqrt(1 - z * z) * sin(phi);
    p[i][Z] = V0 * z;
  }
  double av[3] = {0.0, 0.0, 0.0};
  for (int i = 0; i < particle_number; i++)
    for (int d = 0; d < 3; d++) av[d] += p[i][d];
  for (int d = 0; d < 3; d++) av[d] /= static_cast<double>(particle_number);
  for (int i = 0; i < particle_number; i++)
    for (int d = 0; d < 3; d++) p[i][d] -= av[d];
  host_dirty = true;
}

void Variables::SaveToStream(std::ostream &fs) {
  for (int i = 0; i < particle_number; i++) {
    for (int d = 0; d < D; d++) {
      fs.write((const char *)&q[i][d], sizeof(double));
      fs.write((const char *)&p[i][d], sizeof(double));
    }
  }
}

void Variables::LoadFromStream(std::istream &fs) {
  fs.read((char *)&particle_number, sizeof(particle_number));
  fs.read((char *)&SimulationTime, sizeof(SimulationTime));
  fs.read((char *)&Zeta, sizeof(Zeta));
  for (int i = 0; i < particle_number; i++) {
    for (int d = 0; d < D; d++) {
      fs.read((char *)&q[i][d], sizeof(double));
      fs.read((char *)&p[i][d], sizeof(double));
    }
  }
  total_particle_number = particle_number;
  host_dirty = true;
}

void Variables::ChangeScale(double alpha) {
  for (int i = 0; i < particle_number; i++) {
    q[i][X] *= alpha;
    q[i][Y] *= alpha;
    q[i][Z] *= alpha;
  }
  host_dirty = true;
}

void Variables::Shuffle(void) {
  std::mt19937 mt(12345);
  for (int i = particle_number - 1; i > 0; i--) {
    std::uniform_int_distribution<int> u(0, i);
    const int j = u(mt);
    for (int d = 0; d < D; d++) {
      std::swap(q[i][d], q[j][d]);
      std::swap(p[i][d], p[j][d]);
    }
    std::swap(type[i], type[j]);
  }
  host_dirty = true;
}

void Variables::SyncToDevice(void) {
  if (!device) return;
  if (host_dirty) {
    mdg_check(device, mdg_set_state(device, &q[0][0], &p[0][0], type, particle_number), "mdg_set_state");
    mdg_check(device, mdg_set_zeta(device, Zeta), "mdg_set_zeta");
    host_dirty = false;
    momenta_dirty = false;
    device_newer = false;
  } else if (momenta_dirty) {
    mdg_check(device, mdg_set_velocities(device, &p[0][0], particle_number), "mdg_set_velocities");
    momenta_dirty = false;
    device_newer = false;
  }
  if (pending_steps > 0) {
    while (pending_steps > 0) {
      const int chunk = (int)std::min<long>(pending_steps, 1 << 20);
      mdg_check(device, mdg_calculate(device, chunk), "mdg_calculate");
      pending_steps -= chunk;
    }
    device_newer = true;
  }
}

void Variables::SyncToHost(void) {
  if (!device) return;
  // Host changes not yet uploaded leave the host arrays current: they go up
  // before the next device step, not here (an executor that calls
  // MDUnit::GetVariables several times would otherwise upload the whole
  // state between its calls, which rebuilds the list and loses the ghost
  // copies' age).  Queued steps run first, after the upload.
  if (pending_steps > 0) SyncToDevice();
  if (device_newer) {
    mdg_check(device, mdg_get_state(device, &q[0][0], &p[0][0], type, particle_number), "mdg_get_state");
    mdg_check(device, mdg_get_zeta(device, &Zeta), "mdg_get_zeta");
    total_particle_number = particle_number;
    device_newer = false;
  }
}
