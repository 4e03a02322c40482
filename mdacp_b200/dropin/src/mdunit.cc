// Drop-in MDUnit (interface of include/mdunit.h:16-104 in the reference):
// one unit spanning the whole periodic box, backed by one GPU handle.
#include "mdunit.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>
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
  // two atoms at rest at different places: the kick each gets is exact (0 + k)
  // and must be the same; two moving atoms: the same kick up to the rounding
  // of v + k - v, and no atom may move
  const double xs[2][D] = {{0.31 * sinfo->L[X], 0.47 * sinfo->L[Y], 0.53 * sinfo->L[Z], 0.0},
                           {0.77 * sinfo->L[X], 0.19 * sinfo->L[Y], 0.61 * sinfo->L[Z], 0.0}};
  const double vs[2][D] = {{0.25, -0.5, 0.125, 0.0}, {-1.5, 0.75, 2.0, 0.0}};
  double kick[2][2][D];
  for (int moving = 0; moving < 2; moving++) {
    Variables scratch(4);
    for (int a = 0; a < 2; a++) {
      double x[D], v[D];
      for (int d = 0; d < D; d++) {
        x[d] = xs[a][d];
        v[d] = moving ? vs[a][d] : 0.0;
      }
      scratch.AddParticle(x, v, a);
    }
    probe = &scratch;
    ex->Execute(this);
    probe = nullptr;
    if (scratch.GetParticleNumber() != 2) return false;
    for (int a = 0; a < 2; a++)
      for (int d = 0; d < 3; d++) {
        if (scratch.q[a][d] != xs[a][d]) return false;
        kick[moving][a][d] = scratch.p[a][d] - (moving ? vs[a][d] : 0.0);
      }
  }
  for (int d = 0; d < 3; d++) {
    dp[d] = kick[0][0][d];
    if (kick[0][1][d] != dp[d]) return false;
    const double tol = 1e-12 * std::fabs(dp[d]) + 1e-15 * 4.0;
    for (int a = 0; a < 2; a++)
      if (std::fabs(kick[1][a][d] - dp[d]) > tol) return false;
  }
  return true;
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
  // an executor that leaves positions and atoms alone (the reference's
  // gravity, piston and shell wall change momenta only) goes up as new
  // velocities, which keeps the list and the skin budget as the reference's
  // PairList keeps them; any other change uploads the whole state
  const int pn = vars->GetParticleNumber();
  std::vector<double> q0(&vars->q[0][0], &vars->q[0][0] + (size_t)D * pn);
  std::vector<int> t0(vars->type, vars->type + pn);
  ex->Execute(this);
  const bool same = vars->GetParticleNumber() == pn &&
                    std::equal(q0.begin(), q0.end(), &vars->q[0][0]) && std::equal(t0.begin(), t0.end(), vars->type);
  if (same) vars->MarkMomentaDirty();
  else vars->MarkHostDirty();
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
