// Drop-in Variables: the reference's particle-state interface
// (include/variables.h:12-49) over a GPU-resident state.  The public arrays
// are a host mirror of the device state: they are current after any call
// that hands control to user code (Executor, observers of host data,
// SaveAsCdview) and uploaded again before the next device step when they
// may have changed.  The layout is the reference's padded AoS double[n][D]
// with the arrays held by pointer, as in the reference's GPU build
// (include/variables.h:19-24).
#ifndef variables_h
#define variables_h
#include <iostream>
#include "mdconfig.h"
#include "simulationinfo.h"
#include "mdacp_b200.h"

class Variables {
 private:
  int particle_number;
  int total_particle_number;
  int capacity;
  double C0, C2;
  mdg_handle *device;     // GPU state (owned by MDUnit)
  bool host_dirty;        // host arrays changed since the last upload
  bool momenta_dirty;     // only p changed since the last upload (an executor's kick)
  bool device_newer;      // device state advanced since the last download
  long pending_steps;     // MDManager::Calculate calls not yet run on the device

 public:
  Variables(void);
  explicit Variables(int capacity_);
  ~Variables(void);
  int *type;
  double (*q)[D];
  double (*p)[D];
  double Zeta;
  double SimulationTime;
  double GetC0(void) { return C0; }
  double GetC2(void) { return C2; }
  int GetParticleNumber(void) { return particle_number; }
  int GetTotalParticleNumber(void) { return total_particle_number; }
  int GetCapacity(void) { return capacity; }

  void AddParticle(double x[D], double v[D], int t = 0);
  void SaveToStream(std::ostream &fs);
  void LoadFromStream(std::istream &fs);
  void SaveConfiguration(std::ostream &fs);
  void SetParticleNumber(int pn) { particle_number = pn; }
  void SetTotalParticleNumber(int pn) { total_particle_number = pn; }
  void AdjustPeriodicBoundary(SimulationInfo *sinfo);
  void SetInitialVelocity(double V0, const int id);
  void ChangeScale(double alpha);
  void Shuffle(void);

  // --- host/device mirror (no counterpart in the reference)
  void AttachDevice(mdg_handle *h) { device = h; host_dirty = true; device_newer = false; }
  mdg_handle *Device(void) { return device; }
  void MarkHostDirty(void) { host_dirty = true; }
  // The host changed p only (positions, atom count and order as downloaded):
  // the upload replaces the velocities and keeps the device's list, skin
  // budget and ghost age (mdg_set_velocities).
  void MarkMomentaDirty(void) {
    host_dirty = false;
    momenta_dirty = true;
  }
  void MarkDeviceNewer(void) { device_newer = true; }
  void QueueSteps(long n) { pending_steps += n; }
  // Runs queued steps, uploads host changes: after this the device is current.
  void SyncToDevice(void);
  // Runs queued steps (uploading host changes first) and downloads: after
  // this the host arrays are current.
  void SyncToHost(void);
};
// Aborts like the reference's show_error + exit(1) on a failed device call.
void mdg_check(mdg_handle *h, mdg_status s, const char *what);
#endif
