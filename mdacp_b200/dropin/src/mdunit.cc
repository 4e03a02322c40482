// Drop-in MDUnit (interface of include/mdunit.h:16-104 in the reference):
// one unit spanning the whole periodic box, backed by one GPU handle.
#include "mdunit.h"

#include <cstdio>
#include <cstring>

#include "mpistream.h"

MDUnit::MDUnit(int id_, SimulationInfo *si, ParaInfo *pi, int capacity, int precision_)
    : sinfo(si), pinfo(pi), id(id_), dev(nullptr), precision(precision_), probe(nullptr) {
  vars = new Variables(capacity);
  plist = new PairList();
  int grid_size[D], grid_position[D];
  pinfo->GetGridSize(grid_size);
  pinfo->GetGridPosition(id, grid_position);
  double s[D], e[D];
  for (int d = 0; d < D; d++) {
    const double ul = sinfo->L[d] / static_cast<double>(grid_size[d]);
    s[d] = ul * static_cast<double>(grid_position[d]);
    e[d] = s[d] + ul;
  }
  myrect = MDRect(s, e);
  mesh = new MeshList(sinfo, myrect);
  CreateDevice();
}

MDUnit::~MDUnit(void) {
  if (dev) {
    vars->SyncToDevice();  // run queued steps before the state goes away
    // the last snapshot file is written before the handle goes; a failed
    // write stops the run as the reference's own file output would
    mdg_check(dev, mdg_snapshot_wait(dev), "mdg_snapshot_wait");
    mdg_destroy(dev);
  }
  delete vars;
  delete mesh;
  delete plist;
}

int thermostat_of(SimulationInfo *sinfo) {
  if (!sinfo->ControlTemperature) return MDG_NVE;
  return sinfo->HeatbathType == HT_LANGEVIN ? MDG_LANGEVIN : MDG_NOSE_HOOVER;
}

void MDUnit::CreateDevice(void) {
  mdg_params prm;
  mdg_default_params(&prm);
  prm.capacity = vars->GetCapacity();
  for (int d = 0; d < 3; d++) prm.L[d] = sinfo->L[d];
  prm.cutoff = CUTOFF_LENGTH;
  prm.buffer_length = sinfo->BufferLength;
  prm.time_step = sinfo->TimeStep;
  prm.precision = precision;
  prm.thermostat = thermostat_of(sinfo);
  prm.aimed_temperature = sinfo->AimedTemperature;
  prm.heatbath_tau = sinfo->HeatbathTau;
  prm.heatbath_gamma = sinfo->HeatbathGamma;
  prm.check_list_length = sinfo->CheckListLength;
  prm.seed = static_cast<uint64_t>(id);
  mdg_handle *h = nullptr;
  mdg_check(nullptr, mdg_create(&prm, &h), "mdg_create");
  // observers see the reference's half-step-old ghost copies (see mdacp_b200.h)
  mdg_check(h, mdg_set_observer_mode(h, MDG_OBSERVE_GHOST_LAG), "mdg_set_observer_mode");
  dev = h;
  vars->AttachDevice(dev);
  mesh->Attach(vars);
}

void MDUnit::SetControl(void) {
  mdg_check(dev, mdg_set_control(dev, thermostat_of(sinfo), sinfo->AimedTemperature, sinfo->HeatbathTau,
                                 sinfo->HeatbathGamma), "mdg_set_control");
}

Variables *MDUnit::GetVariables(void) {
  if (probe) return probe;
  // the caller may read and write the arrays: hand over a current mirror and
  // upload it again before the next device step
  vars->SyncToHost();
  vars->MarkHostDirty();
  return vars;
}

bool MDUnit::ProbeUniformKick(Executor *ex, double dp[D]) {
  Variables scratch(4);
  double x0[D] = {0.31 * sinfo->L[X], 0.47 * sinfo->L[Y], 0.53 * sinfo->L[Z], 0.0};
  double x1[D] = {0.77 * sinfo->L[X], 0.19 * sinfo->L[Y], 0.61 * sinfo->L[Z], 0.0};
  double v0[D] = {0.25, -0.5, 0.125, 0.0}, v1[D] = {-1.5, 0.75, 2.0, 0.0};
  scratch.AddParticle(x0, v0, 0);
  scratch.AddParticle(x1, v1, 1);
  probe = &scratch;
  ex->Execute(this);
  probe = nullptr;
  if (scratch.GetParticleNumber() != 2) return false;
  bool uniform = true;
  for (int d = 0; d < 3; d++) {
    dp[d] = scratch.p[0][d] - v0[d];
    uniform = uniform && scratch.q[0][d] == x0[d] && scratch.q[1][d] == x1[d] &&
              scratch.p[1][d] - v1[d] == dp[d];
  }
  return uniform;
}

void MDUnit::AddParticle(double x[D], int type) {
  double v[D] = {0.0, 0.0, 0.0, 0.0};
  AddParticle(x, v, type);
}

void MDUnit::AddParticle(double x[D], double v[D], int type) {
  if (myrect.IsInside(x)) {
    vars->SyncToHost();
    vars->AddParticle(x, v, type);
  }
}

void MDUnit::SaveAsCdview(std::ofstream &ofs) {
  vars->SyncToHost();
  double(*q)[D] = vars->q;
  double(*p)[D] = vars->p;
  const int pn = vars->GetParticleNumber();
  for (int i = 0; i < pn; i++) {
    ofs << "0 " << vars->type[i] << " " << q[i][X] << " " << q[i][Y] << " " << q[i][Z] << " " << p[i][X]
        << " " << p[i][Y] << " " << p[i][Z] << "\n";
  }
}

void MDUnit::SaveConfiguration(void) {
  vars->SyncToHost();
  char filename[256];
  snprintf(filename, sizeof filename, "conf%03d.cnf", id);
  std::ofstream fs(filename);
  vars->SaveConfiguration(fs);
}

double MDUnit::ObserveDouble(DoubleObserver *obs) {
  if (obs->OnDevice()) {
    vars->SyncToDevice();
  } else {
    vars->SyncToHost();
  }
  return obs->Observe(vars, mesh);
}

void MDUnit::Execute(Executor *ex) {
  vars->SyncToHost();
  ex->Execute(this);
  vars->MarkHostDirty();
}

void MDUnit::MakePairList(void) {
  plist->Init(vars, sinfo);
  mesh->MakeList(vars, sinfo, myrect);
}

void MDUnit::ChangeScale(double alpha) {
  // the device scales its box and positions and rebuilds its cell grid
  // (mdg_change_scale); the host mirror follows on its next download
  vars->SyncToDevice();
  myrect.ChangeScale(alpha);
  mesh->ChangeScale(sinfo, myrect);
  mdg_check(dev, mdg_change_scale(dev, alpha), "mdg_change_scale");
  vars->MarkDeviceNewer();
}
