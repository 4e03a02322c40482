// Drop-in PairList (interface of include/pairlist.h:10-31 in the reference).
#include "pairlist.h"

void PairList::Init(Variables *vars, SimulationInfo *sinfo) {
  initialized = true;
  is_fresh = true;
  lifetime = 0;
}

bool PairList::IsPairListExpired(Variables *vars, MeshList *mesh, SimulationInfo *sinfo) {
  if (!initialized) return true;
  is_fresh = false;
  lifetime++;
  vars->SyncToDevice();
  int expired = 0;
  mdg_check(vars->Device(), mdg_check_expired(vars->Device(), &expired), "mdg_check_expired");
  return expired != 0;
}
