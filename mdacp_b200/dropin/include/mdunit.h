// Drop-in MDUnit: the reference's domain unit (include/mdunit.h:16-104) as
// one unit covering the whole periodic box, backed by one mdacp_b200
// handle.  Migration and ghost exchange (MakeBufferFor*, Receive*) have no
// work to do: the periodic wrap happens inside the GPU cell stencil.
#ifndef mdunit_h
#define mdunit_h
#include <stdio.h>
#include <fstream>
#include <vector>
#include "mdconfig.h"
#include "parainfo.h"
#include "simulationinfo.h"
#include "mdrect.h"
#include "parameter.h"
#include "variables.h"
#include "meshlist.h"
#include "pairlist.h"
#include "observer.h"
#include "fcalculator.h"

class MDUnit;

class Executor {
 public:
  virtual ~Executor() {}
  virtual void Execute(MDUnit *mdu) {}
};

class MDUnit {
 private:
  Variables *vars;
  SimulationInfo *sinfo;
  ParaInfo *pinfo;
  MeshList *mesh;
  PairList *plist;
  const int id;
  MDRect myrect;
  mdg_handle *dev;
  int precision;
  Variables *probe;  // while set, GetVariables hands out this scratch set (ProbeUniformKick)
  void CreateDevice(void);

 public:
  MDUnit(int id_, SimulationInfo *si, ParaInfo *pi, int capacity = N, int precision_ = MDG_FP64);
  ~MDUnit(void);
  std::vector<ParticleInfo> send_buffer;
  int GetID(void) { return id; }
  MDRect *GetRect(void) { return &myrect; }
  Variables *GetVariables(void);
  void SaveConfiguration(void);
  void SaveAsCdview(std::ofstream &ofs);
  void AddParticle(double x[D], double v[D], int type = 1);
  void AddParticle(double x[D], int type = 1);
  double *GetSystemSize(void) { return sinfo->L; }
  double GetTimeStep(void) { return sinfo->TimeStep; }
  void SetInitialVelocity(double v0) { vars->SyncToHost(); vars->SetInitialVelocity(v0, id); vars->MarkHostDirty(); }
  int GetParticleNumber(void) { return vars->GetParticleNumber(); }
  int GetTotalParticleNumber(void) { return vars->GetTotalParticleNumber(); }
  void SetTotalParticleNumber(int n) { vars->SetTotalParticleNumber(n); }

  void CalculateForce(void) { ForceCalculator::CalculateForce(vars, mesh, sinfo); }
  void UpdatePositionHalf(void) { ForceCalculator::UpdatePositionHalf(vars, sinfo); }
  void HeatbathZeta(double t) { ForceCalculator::HeatbathZeta(vars, t, sinfo); }
  void HeatbathMomenta(void) { ForceCalculator::HeatbathMomenta(vars, sinfo); }
  void Langevin(void) { ForceCalculator::Langevin(vars, sinfo); }

  void MakeBufferForSendingParticle(const int dir) { send_buffer.clear(); }
  void FindBorderParticles(const int dir) {}
  void MakeBufferForBorderParticles(const int dir) { send_buffer.clear(); }
  void ReceiveParticles(std::vector<ParticleInfo> &recv_buffer) {}
  void AdjustPeriodicBoundary(void) { vars->SyncToHost(); vars->AdjustPeriodicBoundary(sinfo); vars->MarkHostDirty(); }
  void ReceiveBorderParticles(std::vector<ParticleInfo> &recv_buffer) {}
  double ObserveDouble(DoubleObserver *obs);
  int IntegerDouble(IntegerObserver *obs) { return obs->Observe(vars, mesh); }
  void Execute(Executor *ex);
  void MakePairList(void);
  void ShowPairs(void) { mesh->ShowPairs(); }
  bool IsPairListExpired(void) { return plist->IsPairListExpired(vars, mesh, sinfo); }
  void ChangeScale(double alpha);

  // --- device access (no counterpart in the reference)
  mdg_handle *Device(void) { return dev; }
  Variables *Vars(void) { return vars; }
  void SetControl(void);
  // Runs ex on two scratch atoms (at different places, first at rest, then
  // moving) instead of the unit's own: true, with the change of p in dp, if
  // ex gave both the same kick whatever their place and velocity and moved
  // neither -- a uniform kick (dp as read from the atoms at rest).
  bool ProbeUniformKick(Executor *ex, double dp[D]);
};
#endif
