// Drop-in MDManager: the reference's orchestrator interface
// (include/mdmanager.h:10-84) running one MDUnit over the whole box on one
// GPU.  Calculate() queues MD steps; they run as CUDA-graph batches on the
// device when something needs the state (observers, Executors, snapshots,
// pairlist rebuild requests), so a project's step loop runs without a host
// round trip per step.  Extra input keys (no counterpart in the reference):
//   Precision=FP64|FP32Mixed   (default FP64, the drop-in arithmetic)
//   Capacity=<atoms>           (default mdconfig.h N)
//   Device=<cuda ordinal>      (default 0)
//   DeviceExecutors=yes|no     (default yes) an executor the drop-in knows
//                              runs on the device after every step instead of
//                              on the host mirror (see ExecuteAll)
#ifndef mdmanager_h
#define mdmanager_h
#include <vector>
#include "mdunit.h"
#include "parainfo.h"
#include "simulationinfo.h"
#include "parameter.h"

class MDManager {
 private:
  int num_threads;
  int num_procs;
  int rank;
  ParaInfo *pinfo;
  SimulationInfo *sinfo;
  std::vector<MDUnit *> mdv;
  Parameter param;
  bool IsMyUnit(int id) { return id == 0; }
  int GetLocalID(int id) { return 0; }
  bool IsPairListExpired(void);
  double s_time;
  bool control_synced;
  void SyncControl(void);
  bool device_executors;
  Executor *routed;  // the executor running on the device, if any
  bool RouteToDevice(Executor *ex);

 public:
  MDManager(int &argc, char **&argv);
  ~MDManager(void);
  bool IsValid(void);
  Parameter *GetParameter(void) { return &param; }
  MDUnit *GetMDUnit(int index);
  int GetRank(void) { return rank; }
  int GetTotalThreads(void) { return num_threads; }
  int GetTotalUnits(void) { return num_threads * num_procs; }
  int GetTotalProcs(void) { return num_procs; }
  void GetGridSize(int g[D]) { pinfo->GetGridSize(g); }
  double *GetSystemSize(void) { return sinfo->L; }
  double GetTimeStep(void) { return sinfo->TimeStep; }

  void Calculate(void);
  void CalculateForce(void);
  void CalculateNoseHoover(void);
  void CalculateLangevin(void);
  void SetInitialVelocity(double v0);
  void SaveConfiguration(void);
  void SaveAsCdviewSequential(void);
  void SaveAsCdview(const char *filename);
  void SendParticlesSub(const int dir) {}
  void SendParticles(void) {}
  void MakePairList(void);
  void SendBorderParticles(void) {}
  void SendBorderParticlesSub(const int dir) {}
  void ExecuteAll(Executor *ex);

  double GetSimulationTime(void) { return s_time; }
  double ObserveDouble(DoubleObserver *obs);
  unsigned long int GetTotalParticleNumber(void);
  double KineticEnergy(void);
  double PotentialEnergy(void);
  double TotalEnergy(void);
  double Temperature(void);
  double ConfigurationTemperature(void);
  double Pressure(void);

  void SetControlTemperature(bool b) { sinfo->ControlTemperature = b; control_synced = false; }
  void SetAimedTemperature(double t) { sinfo->AimedTemperature = t; control_synced = false; }
  void ShowSystemInformation(void);
  void ChangeScale(double alpha);
};
#endif
