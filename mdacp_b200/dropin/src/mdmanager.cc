// Drop-in MDManager (interface of include/mdmanager.h:10-84 in the
// reference): one unit over the whole box on one GPU; MD steps are queued by
// Calculate() and run as CUDA-graph batches on the device.
#include "mdmanager.h"

#include <mpi.h>

#include <cxxabi.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <typeinfo>

#include "cmdline.h"
#include "communicator.h"
#include "mpistream.h"
#include "observer.h"

MDManager::MDManager(int &argc, char **&argv) : control_synced(false), device_executors(true), routed(nullptr) {
  MPI_Init(&argc, &argv);
  MPI_Comm_size(MPI_COMM_WORLD, &num_procs);
  MPI_Comm_rank(MPI_COMM_WORLD, &rank);
  mout.SetRank(rank);
  mout << "# " << MDACP_VERSION << " on " << mdg_version() << std::endl;
  cmdline::parser arg_parser;
  arg_parser.add<std::string>("in", 'i', "input file name", false, "input.cfg");
  arg_parser.parse_check(argc, argv);
  const std::string inputfile = arg_parser.get<std::string>("in");
  param.LoadFromFile(inputfile.c_str());
  if (num_procs != 1) {
    show_error("the GPU drop-in runs one MPI process (one domain per GPU)");
    exit(1);
  }
  num_threads = 1;
  mout << "# " << num_procs << " MPI Process(es), " << num_threads << " OpenMP Thread(s), Total "
       << num_procs * num_threads << " Unit(s)" << std::endl;
  // one unit: the decomposition keys (GridX.., LocalGridX..) do not apply
  Parameter no_grid;
  pinfo = new ParaInfo(num_procs, num_threads, no_grid);
  int grid_size[D];
  pinfo->GetGridSize(grid_size);
  sinfo = new SimulationInfo(param, grid_size);
  const std::string prec = param.GetStringDef("Precision", "FP64");
  const int precision = (prec == "FP32Mixed" || prec == "FP32") ? MDG_FP32_MIXED : MDG_FP64;
  const int capacity = param.GetIntegerDef("Capacity", N);
  device_executors = param.GetBooleanDef("DeviceExecutors", true);
  mdv.push_back(new MDUnit(0, sinfo, pinfo, capacity, precision));
  s_time = 0.0;
}

MDManager::~MDManager(void) {
  for (unsigned int i = 0; i < mdv.size(); i++) delete mdv[i];
  delete pinfo;
  delete sinfo;
  MPI_Finalize();
}

bool MDManager::IsValid(void) { return pinfo->IsValid() && param.IsValid(); }

MDUnit *MDManager::GetMDUnit(int index) {
  // callers reach the arrays through the unit: hand over a current mirror
  mdv[index]->Vars()->SyncToHost();
  mdv[index]->Vars()->MarkHostDirty();
  return mdv[index];
}

void MDManager::SetInitialVelocity(double v0) {
  for (size_t i = 0; i < mdv.size(); i++) mdv[i]->SetInitialVelocity(v0);
}

void MDManager::SaveAsCdviewSequential(void) {
  static int index = 0;
  char filename[256];
  snprintf(filename, sizeof filename, "conf%04d.cd", index);
  index++;
  SaveAsCdview(filename);
}

void MDManager::SaveAsCdview(const char *filename) {
  // one unit (the GPU domain): the device copies its state on the stream and
  // a host thread writes the file (mdg_snapshot_async), so the steps queued
  // after this call are not held up by the file write
  if (mdv.size() == 1 && mdv[0]->Vars()->Device()) {
    Variables *vars = mdv[0]->Vars();
    vars->SyncToDevice();
    mdg_check(vars->Device(), mdg_snapshot_async(vars->Device(), filename, MDG_SNAPSHOT_CDVIEW),
              "mdg_snapshot_async");
    return;
  }
  std::ofstream ofs(filename);
  for (size_t i = 0; i < mdv.size(); i++) mdv[i]->SaveAsCdview(ofs);
}

void MDManager::SaveConfiguration(void) {
  for (size_t i = 0; i < mdv.size(); i++) mdv[i]->SaveConfiguration();
}

void MDManager::SyncControl(void) {
  if (control_synced) return;
  mdv[0]->Vars()->SyncToDevice();
  mdv[0]->SetControl();
  control_synced = true;
}

// One MDManager::Calculate (src/mdmanager.cc:153-186): expiry test,
// conditional rebuild, half drift, force kick in the thermostat's form, half
// drift.  Queued; runs on the device in batches.
void MDManager::Calculate(void) {
  SyncControl();
  mdv[0]->Vars()->QueueSteps(1);
  s_time += sinfo->TimeStep;
}

// The three force branches of Calculate as separate calls, for projects that
// drive the step themselves (src/mdmanager.cc:226-315).
void MDManager::CalculateForce(void) {
  mdv[0]->CalculateForce();
  mdv[0]->UpdatePositionHalf();
}

void MDManager::CalculateNoseHoover(void) {
  double t = Temperature();
  mdv[0]->HeatbathZeta(t);
  mdv[0]->HeatbathMomenta();
  mdv[0]->CalculateForce();
  mdv[0]->HeatbathMomenta();
  t = Temperature();
  mdv[0]->HeatbathZeta(t);
  mdv[0]->UpdatePositionHalf();
}

void MDManager::CalculateLangevin(void) {
  mdv[0]->CalculateForce();
  mdv[0]->Langevin();
}

void MDManager::MakePairList(void) {
  SyncControl();
  mdv[0]->MakePairList();
}

void MDManager::ExecuteAll(Executor *ex) {
  if (device_executors && RouteToDevice(ex)) return;
  for (size_t i = 0; i < mdv.size(); i++) mdv[i]->Execute(ex);
}

// Executors the device applies itself after every step (mdg_set_external),
// recognised by their class name: GravityImposer (src/phaseflow.cc:58-73),
// a uniform kick p += G dt along one axis, whose kick is read by running it
// once on two scratch atoms.  The project calls ExecuteAll with it after
// every Calculate(), which is when the device applies it; the first call
// hands it to the device (steps already queued get it too, as they come
// before that call in the project's loop) and later calls are no-ops.  Any
// other executor, or one whose probe is not a uniform kick along one axis,
// runs on the host mirror as in the reference.
bool MDManager::RouteToDevice(Executor *ex) {
  if (routed == ex) return true;
  if (routed || mdv.size() != 1 || !mdv[0]->Device()) return false;
  int status = 0;
  char *name = abi::__cxa_demangle(typeid(*ex).name(), nullptr, nullptr, &status);
  const std::string cls = (status == 0 && name) ? name : typeid(*ex).name();
  free(name);
  if (cls != "GravityImposer") return false;
  double dp[D] = {0.0, 0.0, 0.0, 0.0};
  if (!mdv[0]->ProbeUniformKick(ex, dp)) return false;
  int axis = -1;
  for (int d = 0; d < 3; d++)
    if (dp[d] != 0.0) axis = (axis < 0) ? d : 3;
  if (axis < 0 || axis > 2) return false;
  mdg_external x;
  memset(&x, 0, sizeof x);
  x.kind = MDG_EXTERNAL_GRAVITY;
  x.axis = axis;
  x.strength = dp[axis];  // G dt, applied as strength x time_step with time_step 1
  x.time_step = 1.0;
  mdg_check(mdv[0]->Device(), mdg_set_external(mdv[0]->Device(), &x), "mdg_set_external");
  routed = ex;
  mout << "# " << cls << " runs on the device" << std::endl;
  return true;
}

bool MDManager::IsPairListExpired(void) { return mdv[0]->IsPairListExpired(); }

void MDManager::ShowSystemInformation(void) {
  const unsigned long int pn = GetTotalParticleNumber();
  sinfo->ShowAll(pn);
  mout << "# Precision = " << param.GetStringDef("Precision", "FP64") << " (GPU drop-in)" << std::endl;
}

unsigned long int MDManager::GetTotalParticleNumber(void) {
  unsigned long int pn = 0;
  for (size_t i = 0; i < mdv.size(); i++) pn += static_cast<unsigned long int>(mdv[i]->GetParticleNumber());
  return pn;
}

double MDManager::ObserveDouble(DoubleObserver *obs) {
  double e = 0.0;
  for (size_t i = 0; i < mdv.size(); i++) e += mdv[i]->ObserveDouble(obs);
  return e;
}

double MDManager::Temperature(void) { return KineticEnergy() / 1.5; }

double MDManager::ConfigurationTemperature(void) {
  VirialObserver obs;
  const double pn = static_cast<double>(GetTotalParticleNumber());
  return ObserveDouble(&obs) / pn;
}

double MDManager::KineticEnergy(void) {
  KineticEnergyObserver obs;
  const double pn = static_cast<double>(GetTotalParticleNumber());
  return ObserveDouble(&obs) / pn;
}

double MDManager::PotentialEnergy(void) {
  PotentialEnergyObserver obs(sinfo);
  const double pn = static_cast<double>(GetTotalParticleNumber());
  return ObserveDouble(&obs) / pn;
}

double MDManager::TotalEnergy(void) { return KineticEnergy() + PotentialEnergy(); }

double MDManager::Pressure(void) {
  VirialObserver obs;
  const double pn = static_cast<double>(GetTotalParticleNumber());
  const double phi = ObserveDouble(&obs) / pn;
  const double T = Temperature();
  const double V = sinfo->L[X] * sinfo->L[Y] * sinfo->L[Z];
  return (T - phi) * pn / V;
}

void MDManager::ChangeScale(double alpha) {
  MakePairList();
  sinfo->L[X] = sinfo->L[X] * alpha;
  sinfo->L[Y] = sinfo->L[Y] * alpha;
  sinfo->L[Z] = sinfo->L[Z] * alpha;
  for (size_t i = 0; i < mdv.size(); i++) mdv[i]->ChangeScale(alpha);
  control_synced = false;
  MakePairList();
  mout << "# Change Scale " << alpha << std::endl;
}
