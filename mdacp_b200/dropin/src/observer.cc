// Drop-in observers (interfaces of include/observer.h:8-39 in the
// reference): FP64 reductions over the device state and list.
#include "observer.h"

namespace {
void observe(Variables *vars, double *ke, double *pe, double *vir) {
  vars->SyncToDevice();
  mdg_check(vars->Device(), mdg_observe(vars->Device(), ke, pe, vir), "mdg_observe");
  vars->MarkDeviceNewer();  // a stale list is rebuilt first, which renumbers slots
}
}  // namespace

double KineticEnergyObserver::Observe(Variables *vars, MeshList *mesh) {
  double ke = 0.0;
  observe(vars, &ke, nullptr, nullptr);
  return ke;
}

double PotentialEnergyObserver::Observe(Variables *vars, MeshList *mesh) {
  double pe = 0.0;
  observe(vars, nullptr, &pe, nullptr);
  return pe;
}

double VirialObserver::Observe(Variables *vars, MeshList *mesh) {
  double vir = 0.0;
  observe(vars, nullptr, nullptr, &vir);
  return vir;
}
