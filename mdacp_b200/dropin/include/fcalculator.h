// Drop-in ForceCalculator: the reference's free functions
// (include/fcalculator.h:10-44) over the GPU kernels.  The reference's
// variant names (Next, AVX2, Reactless, ...) all select the same kernel here.
#ifndef fcalculator_h
#define fcalculator_h
#include "mdconfig.h"
#include "variables.h"
#include "meshlist.h"
#include "simulationinfo.h"

namespace ForceCalculator {
void CalculateForceBruteforce(Variables *vars, SimulationInfo *sinfo);
void CalculateForceUnroll(Variables *vars, MeshList *mesh, SimulationInfo *sinfo);
void CalculateForceSorted(Variables *vars, MeshList *mesh, SimulationInfo *sinfo);
void CalculateForceNext(Variables *vars, MeshList *mesh, SimulationInfo *sinfo);
void CalculateForcePair(Variables *vars, MeshList *mesh, SimulationInfo *sinfo);
void CalculateForceReactless(Variables *vars, MeshList *mesh, SimulationInfo *sinfo, const int beg = 0);
void UpdatePositionHalf(Variables *vars, SimulationInfo *sinfo);
void CalculateForce(Variables *vars, MeshList *mesh, SimulationInfo *sinfo);
void HeatbathZeta(Variables *vars, double ct, SimulationInfo *sinfo);
void HeatbathMomenta(Variables *vars, SimulationInfo *sinfo, const int beg = 0);
void Langevin(Variables *vars, SimulationInfo *sinfo);
};  // namespace ForceCalculator
#endif
