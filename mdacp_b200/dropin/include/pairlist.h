// Drop-in PairList: the reference's skin bookkeeping interface
// (include/pairlist.h:10-31); the budget and displacement test run on the GPU.
#ifndef pairlist_h
#define pairlist_h
#include "mdconfig.h"
#include "meshlist.h"
#include "variables.h"

class PairList {
 private:
  int lifetime;
  bool initialized;
  bool is_fresh;

 public:
  PairList(void) : lifetime(0), initialized(false), is_fresh(false) {}
  void Init(Variables *vars, SimulationInfo *sinfo);
  bool IsFresh(void) { return is_fresh; }
  void SetFresh(bool b) { is_fresh = b; }
  bool IsPairListExpired(Variables *vars, MeshList *mesh, SimulationInfo *sinfo);
  int GetLifeTime(void) { return lifetime; }
};
#endif
