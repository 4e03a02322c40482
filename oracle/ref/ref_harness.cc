// Test-only MDACP "Project" that drives the reference's own hot path on an
// injected state.  It is compiled together with the unmodified reference
// sources (src/*.cc of kohnakagawa/mdacp) into oracle/_ref/ and is used only
// to make golden fixtures and as the timed CPU baseline.  It is never
// linked into the product.
//
// Registration follows the reference's own plugin mechanism: a static
// Project object calls ProjectManager::AddProject in its constructor
// (include/projectmanager.h:8-24, src/benchmark.cc:10, include/benchmark.h:10-12).
//
// Modes (key Mode= in the input file, read by ProjectManager::ExecuteProject,
// src/projectmanager.cc:26-42):
//   OracleDump  - inject state, MakePairList, dump pairlist / observables /
//                 forces, optionally run Steps x Calculate() and dump the end state.
//   OracleBench - inject state, MakePairList, Warmup + Steps x Calculate(),
//                 print one "ORACLE_BENCH" line with the atom-steps/s.
//
// State file (little endian): int64 n; double q[n][3]; double v[n][3]; int32 id[n].
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#include "projectmanager.h"
#include "mdmanager.h"
#include "mdunit.h"
#include "observer.h"
#include "communicator.h"
#include "mpistream.h"

namespace {

struct InjectedState {
  int64_t n = 0;
  std::vector<double> q, v;
  std::vector<int32_t> id;
  bool Load(const std::string &path) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return false;
    bool ok = fread(&n, sizeof(n), 1, f) == 1;
    if (ok) {
      q.resize(3 * n);
      v.resize(3 * n);
      id.resize(n);
      ok = fread(q.data(), sizeof(double), 3 * n, f) == (size_t)(3 * n) &&
           fread(v.data(), sizeof(double), 3 * n, f) == (size_t)(3 * n) &&
           fread(id.data(), sizeof(int32_t), n, f) == (size_t)n;
    }
    fclose(f);
    return ok;
  }
};

// Adds every injected atom whose position lies in the unit's rectangle
// (MDUnit::AddParticle tests MDRect::IsInside, src/mdunit.cc:60-65); the
// atom's id travels in Variables::type through migration.
class StateInjector : public Executor {
 public:
  explicit StateInjector(const InjectedState *s) : s_(s) {}
  void Execute(MDUnit *mdu) override {
    for (int64_t i = 0; i < s_->n; i++) {
      double x[D] = {s_->q[3 * i], s_->q[3 * i + 1], s_->q[3 * i + 2], 0.0};
      double v[D] = {s_->v[3 * i], s_->v[3 * i + 1], s_->v[3 * i + 2], 0.0};
      mdu->AddParticle(x, v, s_->id[i]);
    }
  }
 private:
  const InjectedState *s_;
};

// Zeroes p so that one force kick leaves p = F * TimeStep.
class ZeroMomenta : public Executor {
 public:
  void Execute(MDUnit *mdu) override {
    Variables *vars = mdu->GetVariables();
    const int pn = vars->GetParticleNumber();
    for (int i = 0; i < pn; i++) {
      vars->p[i][X] = vars->p[i][Y] = vars->p[i][Z] = 0.0;
    }
  }
};

class ForceKick : public Executor {
 public:
  void Execute(MDUnit *mdu) override { mdu->CalculateForce(); }
};

// Observers receive the unit's MeshList (MDUnit::ObserveDouble,
// include/mdunit.h:97); this one writes the unit's raw CSR and positions.
class PairDumper : public DoubleObserver {
 public:
  explicit PairDumper(const std::string &path) : path_(path) {}
  double Observe(Variables *vars, MeshList *mesh) override {
    FILE *f = fopen(path_.c_str(), "wb");
    if (!f) return -1.0;
    const int32_t pn = vars->GetParticleNumber();
    const int32_t tn = vars->GetTotalParticleNumber();
    fwrite(&pn, 4, 1, f);
    fwrite(&tn, 4, 1, f);
    for (int i = 0; i < tn; i++) fwrite(vars->q[i], sizeof(double), 3, f);
    fwrite(vars->type, 4, pn, f);
    std::vector<int32_t> np(tn), kp(tn);
    int64_t total = 0;
    for (int i = 0; i < tn; i++) {
      np[i] = mesh->GetPartnerNumber(i);
      kp[i] = mesh->GetKeyPointer(i);
      total += np[i];
    }
    fwrite(np.data(), 4, tn, f);
    fwrite(kp.data(), 4, tn, f);
    fwrite(&total, 8, 1, f);
    const int *sl = mesh->GetSortedList();
    for (int i = 0; i < tn; i++) fwrite(sl + kp[i], 4, np[i], f);
    fclose(f);
    return 0.0;
  }
 private:
  std::string path_;
};

class ConstructionCounter : public DoubleObserver {
 public:
  double Observe(Variables *, MeshList *mesh) override {
    return static_cast<double>(mesh->GetNumberOfConstructions());
  }
};

// Writes q, p, type of the unit's real atoms (appending to one file).
class StateDumper : public DoubleObserver {
 public:
  explicit StateDumper(FILE *f) : f_(f) {}
  double Observe(Variables *vars, MeshList *) override {
    const int pn = vars->GetParticleNumber();
    for (int i = 0; i < pn; i++) {
      fwrite(vars->q[i], sizeof(double), 3, f_);
      fwrite(vars->p[i], sizeof(double), 3, f_);
      int32_t t = vars->type[i];
      fwrite(&t, 4, 1, f_);
    }
    return static_cast<double>(pn);
  }
 private:
  FILE *f_;
};

void DumpObservables(MDManager *mdm, FILE *f, const char *tag) {
  VirialObserver vobs;
  const double n = static_cast<double>(mdm->GetTotalParticleNumber());
  const double virial = mdm->ObserveDouble(&vobs);
  fprintf(f, "%s n %.17g ke %.17g pe %.17g virial %.17g temperature %.17g pressure %.17g time %.17g\n",
          tag, n, mdm->KineticEnergy(), mdm->PotentialEnergy(), virial,
          mdm->Temperature(), mdm->Pressure(), mdm->GetSimulationTime());
}

void DumpForcesOrState(MDManager *mdm, const std::string &path) {
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) return;
  StateDumper d(f);
  // Units are visited one by one so the file writes are sequential.
  for (int i = 0; i < mdm->GetTotalThreads(); i++) mdm->GetMDUnit(i)->ObserveDouble(&d);
  fclose(f);
}

class OracleDump : public Project {
 public:
  OracleDump() { ProjectManager::GetInstance().AddProject("OracleDump", this); }
  void Run(MDManager *mdm) override {
    Parameter *param = mdm->GetParameter();
    InjectedState st;
    if (!st.Load(param->GetString("StateFile"))) {
      mout << "# OracleDump: cannot read StateFile" << std::endl;
      return;
    }
    const std::string prefix = param->GetStringDef("DumpPrefix", "oracle");
    StateInjector inj(&st);
    mdm->ExecuteAll(&inj);
    mdm->MakePairList();
    for (int u = 0; u < mdm->GetTotalThreads(); u++) {
      PairDumper pd(prefix + "_pairs_u" + std::to_string(u) + ".bin");
      mdm->GetMDUnit(u)->ObserveDouble(&pd);
    }
    FILE *obs = fopen((prefix + "_obs.txt").c_str(), "w");
    DumpObservables(mdm, obs, "initial");
    if (param->GetBooleanDef("DumpForces", false)) {
      // p <- 0, one kick with the configured TimeStep: p = F * TimeStep.
      ZeroMomenta z;
      mdm->ExecuteAll(&z);
      ForceKick k;
      mdm->ExecuteAll(&k);
      DumpForcesOrState(mdm, prefix + "_forces.bin");
    } else {
      const int steps = param->GetIntegerDef("Steps", 0);
      const int every = param->GetIntegerDef("ObserveLoop", 0);
      for (int s = 0; s < steps; s++) {
        mdm->Calculate();
        if (every > 0 && (s + 1) % every == 0) {
          DumpObservables(mdm, obs, ("step" + std::to_string(s + 1)).c_str());
        }
      }
      ConstructionCounter cc;
      fprintf(obs, "constructions %.17g\n", mdm->ObserveDouble(&cc));
      DumpObservables(mdm, obs, "final");
      DumpForcesOrState(mdm, prefix + "_state.bin");
    }
    fclose(obs);
  }
};

class OracleBench : public Project {
 public:
  OracleBench() { ProjectManager::GetInstance().AddProject("OracleBench", this); }
  void Run(MDManager *mdm) override {
    Parameter *param = mdm->GetParameter();
    InjectedState st;
    if (!st.Load(param->GetString("StateFile"))) {
      mout << "# OracleBench: cannot read StateFile" << std::endl;
      return;
    }
    StateInjector inj(&st);
    mdm->ExecuteAll(&inj);
    const int warmup = param->GetIntegerDef("Warmup", 1);
    const int steps = param->GetIntegerDef("Steps", 10);
    const double t_setup0 = Communicator::GetTime();
    mdm->MakePairList();
    for (int s = 0; s < warmup; s++) mdm->Calculate();
    ConstructionCounter cc;
    const double c0 = mdm->ObserveDouble(&cc);
    const double t0 = Communicator::GetTime();
    for (int s = 0; s < steps; s++) mdm->Calculate();
    const double t1 = Communicator::GetTime();
    const double c1 = mdm->ObserveDouble(&cc);
    const double n = static_cast<double>(mdm->GetTotalParticleNumber());
    printf("ORACLE_BENCH n %.0f steps %d sec %.9g atom_steps_per_s %.9g rebuilds %.0f units %d setup_sec %.6g\n",
           n, steps, t1 - t0, steps * n / (t1 - t0), c1 - c0, mdm->GetTotalThreads(),
           t0 - t_setup0);
    fflush(stdout);
  }
};

OracleDump g_oracle_dump;
OracleBench g_oracle_bench;

}  // namespace
