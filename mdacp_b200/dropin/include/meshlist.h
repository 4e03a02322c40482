// Drop-in MeshList: the reference's cell list / Verlet list interface
// (include/meshlist.h:13-102).  The list lives on the GPU (full list, cell
// order); the CSR accessors below present the reference's half list
// (key = lower index, src/meshlist.cc:555-583) of the current slot order,
// downloaded on first use after each construction.
#ifndef meshlist_h
#define meshlist_h
#include <vector>
#include "mdconfig.h"
#include "variables.h"
#include "mdrect.h"

class MeshList {
 private:
  Variables *vars_;
  long cached_rebuild;
  std::vector<int> key_pointer, number_of_partners, sorted_list;
  std::vector<int> pairs;  // key, partner, key, partner, ...
  int number_of_constructions_base;
  void Fetch(void);

 public:
  MeshList(SimulationInfo *sinfo, MDRect &r);
  ~MeshList(void) {}
  void Attach(Variables *vars) { vars_ = vars; }
  void ChangeScale(SimulationInfo *sinfo, MDRect &myrect);

  enum { KEY = 0, PARTNER = 1 };
  int (*GetKeyPartnerPairs(void))[2];
  int GetPairNumber(void);
  int GetPartnerNumber(int i);
  int GetKeyPointer(int i);
  int *GetSortedList(void);
  int *GetKeyPointerP(void);
  int *GetNumberOfPartners(void);

  void Sort(Variables *vars, SimulationInfo *sinfo, MDRect &myrect);
  int GetNumberOfConstructions(void);
  void ClearNumberOfConstructions(void);
  void MakeList(Variables *vars, SimulationInfo *sinfo, MDRect &myrect);
  void MakeListBruteforce(Variables *vars, SimulationInfo *sinfo, MDRect &myrect);
  void ShowPairs(void);
  void ShowSortedList(Variables *vars);
};
#endif
