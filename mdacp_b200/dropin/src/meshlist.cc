// Drop-in MeshList (interface of include/meshlist.h:13-102 in the reference).
#include "meshlist.h"

#include <cstdio>

#include "mpistream.h"

MeshList::MeshList(SimulationInfo *sinfo, MDRect &r)
    : vars_(nullptr), cached_rebuild(-1), number_of_constructions_base(0) {}

void MeshList::ChangeScale(SimulationInfo *sinfo, MDRect &myrect) { cached_rebuild = -1; }

// Downloads the device list once per construction and derives the
// reference's half-list CSR (key = lower slot index, partners in row order).
void MeshList::Fetch(void) {
  mdg_handle *h = vars_->Device();
  vars_->SyncToHost();
  mdg_info info;
  mdg_check(h, mdg_get_info(h, &info), "mdg_get_info");
  if (info.rebuilds == cached_rebuild && cached_rebuild >= 0) return;
  int64_t count = 0;
  mdg_check(h, mdg_get_list(h, nullptr, nullptr, 0, &count), "mdg_get_list");
  const int n = vars_->GetParticleNumber();
  std::vector<int> rows(n), part(count);
  mdg_check(h, mdg_get_list(h, rows.data(), part.data(), count, &count), "mdg_get_list");
  // the list may have been (re)built by the readout: refresh the host mirror
  vars_->MarkDeviceNewer();
  vars_->SyncToHost();
  mdg_check(h, mdg_get_info(h, &info), "mdg_get_info");
  number_of_partners.assign(n, 0);
  key_pointer.assign(n, 0);
  sorted_list.clear();
  pairs.clear();
  int64_t off = 0;
  for (int i = 0; i < n; i++) {
    for (int k = 0; k < rows[i]; k++) {
      const int j = part[off + k];
      if (i < j) {
        number_of_partners[i]++;
        sorted_list.push_back(j);
        pairs.push_back(i);
        pairs.push_back(j);
      }
    }
    off += rows[i];
  }
  int pos = 0;
  for (int i = 0; i < n; i++) {
    key_pointer[i] = pos;
    pos += number_of_partners[i];
  }
  sorted_list.push_back(0);  // one padding entry, as CalculateForceNext reads one past a row
  cached_rebuild = info.rebuilds;
}

int (*MeshList::GetKeyPartnerPairs(void))[2] {
  Fetch();
  return reinterpret_cast<int(*)[2]>(pairs.data());
}
int MeshList::GetPairNumber(void) {
  Fetch();
  return (int)(pairs.size() / 2);
}
int MeshList::GetPartnerNumber(int i) {
  Fetch();
  return number_of_partners[i];
}
int MeshList::GetKeyPointer(int i) {
  Fetch();
  return key_pointer[i];
}
int *MeshList::GetSortedList(void) {
  Fetch();
  return sorted_list.data();
}
int *MeshList::GetKeyPointerP(void) {
  Fetch();
  return key_pointer.data();
}
int *MeshList::GetNumberOfPartners(void) {
  Fetch();
  return number_of_partners.data();
}

// Atoms are kept in cell order on the device at every construction, which is
// what the reference's optional Sort (src/meshlist.cc:139-173) provides.
void MeshList::Sort(Variables *vars, SimulationInfo *sinfo, MDRect &myrect) {}

int MeshList::GetNumberOfConstructions(void) {
  mdg_info info;
  mdg_check(vars_->Device(), mdg_get_info(vars_->Device(), &info), "mdg_get_info");
  return (int)info.rebuilds - number_of_constructions_base;
}

void MeshList::ClearNumberOfConstructions(void) {
  mdg_info info;
  mdg_check(vars_->Device(), mdg_get_info(vars_->Device(), &info), "mdg_get_info");
  number_of_constructions_base = (int)info.rebuilds;
}

void MeshList::MakeList(Variables *vars, SimulationInfo *sinfo, MDRect &myrect) {
  vars->SyncToDevice();
  mdg_check(vars->Device(), mdg_make_pairlist(vars->Device()), "mdg_make_pairlist");
  vars->MarkDeviceNewer();
  cached_rebuild = -1;
}

void MeshList::MakeListBruteforce(Variables *vars, SimulationInfo *sinfo, MDRect &myrect) {
  MakeList(vars, sinfo, myrect);
}

void MeshList::ShowPairs(void) {
  Fetch();
  for (size_t k = 0; k + 1 < pairs.size(); k += 2) printf("(%05d,%05d)\n", pairs[k], pairs[k + 1]);
}

void MeshList::ShowSortedList(Variables *vars) {
  Fetch();
  for (size_t i = 0; i < key_pointer.size(); i++)
    for (int k = 0; k < number_of_partners[i]; k++)
      printf("(%05d,%05d)\n", (int)i, sorted_list[key_pointer[i] + k]);
}
