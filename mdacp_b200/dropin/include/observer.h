// Drop-in observers: the reference's interfaces (include/observer.h:8-39).
// KineticEnergy / PotentialEnergy / Virial observers are FP64 reductions on
// the GPU; a user-defined DoubleObserver sees the synchronised host mirror.
#ifndef observe_h
#define observe_h
#include "variables.h"
#include "meshlist.h"
#include "simulationinfo.h"

class IntegerObserver {
 public:
  virtual ~IntegerObserver() {}
  virtual int Observe(Variables *vars, MeshList *mesh) = 0;
};

class DoubleObserver {
 public:
  virtual ~DoubleObserver() {}
  virtual double Observe(Variables *vars, MeshList *mesh) = 0;
  // true: computed on the device, the host mirror need not be current
  virtual bool OnDevice(void) { return false; }
};

class ParticleNumberObserver : public IntegerObserver {
 public:
  int Observe(Variables *vars, MeshList *mesh = NULL) { return vars->GetParticleNumber(); }
};

class KineticEnergyObserver : public DoubleObserver {
 public:
  double Observe(Variables *vars, MeshList *mesh);
  bool OnDevice(void) { return true; }
};

class PotentialEnergyObserver : public DoubleObserver {
 private:
  SimulationInfo *sinfo;
 public:
  PotentialEnergyObserver(SimulationInfo *sinfo_) { sinfo = sinfo_; }
  double Observe(Variables *vars, MeshList *mesh);
  bool OnDevice(void) { return true; }
};

class VirialObserver : public DoubleObserver {
 public:
  double Observe(Variables *vars, MeshList *mesh);
  bool OnDevice(void) { return true; }
};
#endif
