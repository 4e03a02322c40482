// Drop-in ForceCalculator (interface of include/fcalculator.h:10-44 in the
// reference): every entry point runs its GPU kernel on the device state.
#include "fcalculator.h"

namespace {
mdg_handle *dev(Variables *vars) {
  vars->SyncToDevice();
  return vars->Device();
}
}  // namespace

void ForceCalculator::UpdatePositionHalf(Variables *vars, SimulationInfo *sinfo) {
  mdg_check(dev(vars), mdg_update_position_half(dev(vars)), "mdg_update_position_half");
  vars->MarkDeviceNewer();
}

void ForceCalculator::CalculateForce(Variables *vars, MeshList *mesh, SimulationInfo *sinfo) {
  mdg_check(dev(vars), mdg_calculate_force(dev(vars)), "mdg_calculate_force");
  vars->MarkDeviceNewer();
}

void ForceCalculator::CalculateForceBruteforce(Variables *vars, SimulationInfo *sinfo) {
  CalculateForce(vars, nullptr, sinfo);
}
void ForceCalculator::CalculateForceUnroll(Variables *vars, MeshList *mesh, SimulationInfo *sinfo) {
  CalculateForce(vars, mesh, sinfo);
}
void ForceCalculator::CalculateForceSorted(Variables *vars, MeshList *mesh, SimulationInfo *sinfo) {
  CalculateForce(vars, mesh, sinfo);
}
void ForceCalculator::CalculateForceNext(Variables *vars, MeshList *mesh, SimulationInfo *sinfo) {
  CalculateForce(vars, mesh, sinfo);
}
void ForceCalculator::CalculateForcePair(Variables *vars, MeshList *mesh, SimulationInfo *sinfo) {
  CalculateForce(vars, mesh, sinfo);
}
void ForceCalculator::CalculateForceReactless(Variables *vars, MeshList *mesh, SimulationInfo *sinfo,
                                              const int beg) {
  CalculateForce(vars, mesh, sinfo);
}

void ForceCalculator::HeatbathZeta(Variables *vars, double ct, SimulationInfo *sinfo) {
  mdg_check(dev(vars), mdg_heatbath_zeta(dev(vars), ct), "mdg_heatbath_zeta");
  mdg_check(vars->Device(), mdg_get_zeta(vars->Device(), &vars->Zeta), "mdg_get_zeta");
}

void ForceCalculator::HeatbathMomenta(Variables *vars, SimulationInfo *sinfo, const int beg) {
  mdg_check(dev(vars), mdg_heatbath_momenta(dev(vars)), "mdg_heatbath_momenta");
  vars->MarkDeviceNewer();
}

void ForceCalculator::Langevin(Variables *vars, SimulationInfo *sinfo) {
  mdg_check(dev(vars), mdg_langevin(dev(vars)), "mdg_langevin");
  vars->MarkDeviceNewer();
}
