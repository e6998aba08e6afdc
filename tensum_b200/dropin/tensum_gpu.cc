// tensum_gpu -- the TENSUM solver with its residual/update loop on the B200.
//
// The drop-in caller of include/tensum_gpu.h: the reference's own command
// line (src/process_command_line.cc), parameter reader, part-file reader,
// Grid::preproc, initial conditions, Monte Carlo sample loop and writers, built
// unchanged from the reference's sources, with FiniteVolume::solve's loop
// (src/fv.cc:2273-2343) replaced by the library's calls: per step tg_advance
// (store_conserved_old, compute_dt, the stages, the residual norm and the
// time update on the device), then the reference's own log_messages,
// compute_forces, compute_global, output and output_restart on the state the
// device hands back.  FiniteVolume::run (src/fv.cc:2401-2492) is followed
// step for step; the members it uses are private in src/fv.h, so this
// translation unit opens them with a preprocessor override before including
// the header (the reference files are untouched).
//
//   tensum_gpu -i <param file> -L <case dir>     (the reference's options)
//
// One partition (NPART = 1): the device path has no MPI.  compute_global and
// compute_forces read the whole state every step, so when the parameter file
// asks for them the state comes back to the host every step; without them it
// comes back only at output and restart times.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <vector>
#include <chrono>
#include <algorithm>
#include <complex>
#include <limits>
#include <iomanip>
#include <stdint.h>
#include <dlfcn.h>
#include <mpi.h>
#include <cuda_runtime.h>

#include "tensum_gpu.h"

// Every system header the reference pulls in is included above, so the
// override below only reaches the reference's own class definitions.
#define private public
#include "fv.h"
#undef private

// Globals normally defined in src/main.cc:10-31.
Dimension dim;
bool debug;
bool restart;
bool preprocess;
bool bounds;
bool verbose;
bool PERIODIC;
std::map<std::string, double> constants;
unsigned int NPART;
unsigned int N_MC_GROUPS;
std::vector<double> rnd_nos;

void process_command_line(int argc, char* argv[], int& ifile, int& iloc, unsigned int& NPART);

namespace {

[[noreturn]] void die(const std::string& what, const char* detail) {
  std::cerr << "tensum_gpu: " << what << (detail && *detail ? ": " : "") << (detail ? detail : "") << std::endl;
  std::exit(1);
}

void check(tg_status st, const char* call, tg_handle* h) {
  if (st != TG_OK) die(call, tg_last_error(h));
}

// Host arrays of tg_mesh, built from the reference's Grid after Grid::preproc.
struct MeshArrays {
  std::vector<double> xy, cnrm, carea, fnrm, bnrm, vr, fr, cr;
  std::vector<int> cv, fv, ft, fl, frc, bv, bt, bl, poff, pmem;
  std::vector<unsigned char> bper;
  tg_mesh mesh{};
};

void build_mesh(const Grid& g, MeshArrays& a) {
  for (const Vertex& v : g.vertex) { a.xy.push_back(v.coord.x); a.xy.push_back(v.coord.y); }
  for (const Cell& c : g.cell) {
    for (int k = 0; k < 3; ++k) {
      a.cv.push_back((int)c.vertex[k]);
      a.cnrm.push_back(c.normal[k].x);
      a.cnrm.push_back(c.normal[k].y);
    }
    a.carea.push_back(c.area);
  }
  for (const Face& f : g.face) {
    a.fv.push_back((int)f.vertex[0]); a.fv.push_back((int)f.vertex[1]);
    a.ft.push_back((int)f.type);
    a.fnrm.push_back(f.normal.x); a.fnrm.push_back(f.normal.y);
    a.fl.push_back(f.lcell); a.frc.push_back(f.rcell);
  }
  for (const Face& f : g.bface) {
    a.bv.push_back((int)f.vertex[0]); a.bv.push_back((int)f.vertex[1]);
    a.bt.push_back((int)f.type);
    a.bnrm.push_back(f.normal.x); a.bnrm.push_back(f.normal.y);
    a.bl.push_back(f.lcell);
    a.bper.push_back(f.periodic ? 1 : 0);
  }
  a.poff.push_back(0);
  for (const PERIODIC_LISTS& p : g.periodic_lists) {
    for (int v : p.P_ij) a.pmem.push_back(v);
    a.poff.push_back((int)a.pmem.size());
  }
  if (dim == axi) {   // the radii Grid::compute_radius set (src/grid_preproc.cc:750-777)
    for (const Vertex& v : g.vertex) a.vr.push_back(v.radius);
    for (const Face& f : g.face) a.fr.push_back(f.radius);
    for (const Cell& c : g.cell) a.cr.push_back(c.radius);
  }
  tg_mesh& m = a.mesh;
  m.n_vertex = (int)g.n_vertex; m.coords = a.xy.data(); m.dcarea = g.dcarea.data(); m.mcarea = g.mcarea.data();
  m.n_cell = (int)g.n_cell; m.cell_vertex = a.cv.data(); m.cell_normal = a.cnrm.data(); m.cell_area = a.carea.data();
  m.n_face = (int)g.face.size(); m.face_vertex = a.fv.data(); m.face_type = a.ft.data();
  m.face_normal = a.fnrm.data(); m.face_lcell = a.fl.data(); m.face_rcell = a.frc.data();
  m.n_bface = (int)g.bface.size(); m.bface_vertex = a.bv.data(); m.bface_type = a.bt.data();
  m.bface_normal = a.bnrm.data(); m.bface_lcell = a.bl.data(); m.bface_periodic = a.bper.data();
  m.n_periodic = (int)g.periodic_lists.size(); m.periodic_offsets = a.poff.data(); m.periodic_members = a.pmem.data();
  m.vertex_radius = a.vr.empty() ? nullptr : a.vr.data();
  m.face_radius = a.fr.empty() ? nullptr : a.fr.data();
  m.cell_radius = a.cr.empty() ? nullptr : a.cr.data();
}

// Boundary values per boundary-face vertex, evaluated once by the reference's
// own BoundaryCondition::apply (src/bc.h:568-610) on a probe pair of states:
// the state the condition writes holds the expressions' values there.
struct BcArrays {
  std::vector<int> tags, kinds;
  std::vector<unsigned char> adiabatic;
  std::vector<double> values;
  tg_bc_table bc{};
};

void build_bc(FiniteVolume& fv, BcArrays& a) {
  for (auto& it : fv.param.boundary_condition) {
    a.tags.push_back(it.first);
    a.kinds.push_back((int)it.second.type);
    a.adiabatic.push_back(it.second.adiabatic ? 1 : 0);
  }
  const Grid& g = fv.grid;
  a.values.assign(g.bface.size() * 10, 0.0);
  for (size_t b = 0; b < g.bface.size(); ++b) {
    const Face& f = g.bface[b];
    auto it = fv.param.boundary_condition.find((int)f.type);
    if (it == fv.param.boundary_condition.end()) continue;
    BoundaryCondition& bc = it->second;
    // the state a kind writes: vertex state 0 for no-slip and inlet, the ghost state 1
    // for far field and pressure outlet; slip, outlet and periodic take no values
    int slot = -1;
    switch ((int)bc.type) {
      case TG_BC_NOSLIP: case TG_BC_INLET: slot = 0; break;
      case TG_BC_FARFIELD: case TG_BC_PRESSURE: slot = 1; break;
      default: break;
    }
    if (slot < 0) continue;
    for (int k = 0; k < 2; ++k) {
      std::vector<PrimVar> probe(2);
      for (PrimVar& q : probe) { q.temperature = 1.0; q.pressure = 1.0; q.velocity = 0.0; }
      bc.apply(g.vertex[f.vertex[k]].coord, fv.elapsed_time, f, probe);
      const PrimVar& q = probe[slot];
      double* v = &a.values[(2 * b + k) * 5];
      v[0] = q.temperature; v[1] = q.velocity.x; v[2] = q.velocity.y; v[3] = q.velocity.z; v[4] = q.pressure;
    }
  }
  a.bc.n_types = (int)a.tags.size();
  a.bc.type_tag = a.tags.data();
  a.bc.kind = a.kinds.data();
  a.bc.adiabatic = a.adiabatic.data();
  a.bc.bface_values = a.values.data();
}

tg_material material_of(const Material& m) {
  tg_material t{};
  t.gamma = m.gamma; t.gas_const = m.gas_const; t.prandtl = m.prandtl; t.mu_ref = m.mu_ref;
  t.T_0 = m.T_0; t.T_ref = m.T_ref; t.omega = m.omega; t.ev_mod_alpha = m.ev_mod_alpha;
  t.ev_mod_beta = m.ev_mod_beta; t.tvb_minmod_coef = m.tvb_minmod_coef;
  t.model = (int)m.model; t.flux_scheme = (int)m.flux_scheme; t.mu_model = (int)m.mu_model;
  t.reconstruct_scheme = (int)m.reconstruct_scheme;
  t.nd_active = m.nd_active; t.visc_active = m.visc_active; t.heat_active = m.heat_active;
  return t;
}

tg_options options_of(const Parameter& p) {
  tg_options o{};
  o.time_scheme = p.time_scheme == "rk4" ? TG_TIME_RK4 : p.time_scheme == "heuns" ? TG_TIME_HEUNS : TG_TIME_SSPRK3;
  o.time_mode = p.time_mode == "unsteady" ? TG_UNSTEADY : TG_STEADY;
  o.time_step = p.time_step;
  o.cfl = p.cfl;
  o.final_time = p.final_time;
  o.n_time_stamps = p.n_time_stamps;
  o.max_iter = (long)p.max_iter;
  o.min_residue = p.min_residue;
  o.bad_state_check = 1;
  o.liou_fix = p.liou_fix ? 1 : 0;
  o.bc_strong = p.bc_scheme == Parameter::strong ? 1 : 0;
  return o;
}

// The device state in the reference's arrays: primitive (PrimVar records) and,
// with `grad`, dE as the reference holds it at that point of the loop.
struct HostState {
  double* prim = nullptr;   // pinned, n_vertex x 5
  double* dE = nullptr;     // pinned, n_vertex x 5 x 3
  int nv = 0;
  explicit HostState(int n) : nv(n) {
    if (cudaMallocHost((void**)&prim, sizeof(double) * 5 * (size_t)n) != cudaSuccess ||
        cudaMallocHost((void**)&dE, sizeof(double) * 15 * (size_t)n) != cudaSuccess)
      die("cudaMallocHost", "pinned host buffers");
  }
  ~HostState() { cudaFreeHost(prim); cudaFreeHost(dE); }
};

void fetch_state(FiniteVolume& fv, tg_handle* h, HostState& hs, bool grad, int grad_state) {
  check(tg_output_begin(h, hs.prim, grad ? hs.dE : nullptr, grad_state), "tg_output_begin", h);
  check(tg_output_wait(h), "tg_output_wait", h);
  std::memcpy(reinterpret_cast<double*>(fv.primitive.data()), hs.prim, sizeof(double) * 5 * (size_t)hs.nv);
  if (grad)
    for (int i = 0; i < hs.nv; ++i)
      for (int c = 0; c < 5; ++c) {
        const double* d = hs.dE + ((size_t)i * 5 + c) * 3;
        fv.dE[i][c].x = d[0]; fv.dE[i][c].y = d[1]; fv.dE[i][c].z = d[2];
      }
}

// FiniteVolume::solve (src/fv.cc:2230-2380) with the stage loop on the device.
void solve_gpu(FiniteVolume& fv, tg_handle* h, HostState& hs, int sample_id) {
  fv.t_sample_solve.start_time();
  const Parameter& p = fv.param;
  unsigned long int iter = fv.last_iter;
  fv.residual_norm_total = 1.0e20;
  fv.compute_gradients();   // the reference's own, for the first output's dE
  if (p.write_soln && !restart) {
    fv.output();
    if (p.time_mode == "steady") fv.write_to_master = false;
  }
  if (p.online_stat) fv.increment_moments(sample_id);
  if (fv.counter == 0) fv.counter++;
  unsigned long int term_iter = 0;
  if (p.time_mode == "steady") term_iter = iter;

  check(tg_set_state(h, reinterpret_cast<const double*>(fv.primitive.data()), (int)fv.grid.n_vertex,
                     fv.elapsed_time), "tg_set_state", h);
  const bool every_step = p.has_global || !p.force_data.empty() || bounds;
  while (fv.residual_norm_total > p.min_residue && SafeLess(term_iter, p.max_iter) && fv.elapsed_time < p.final_time) {
    // store_conserved_old, compute_dt, [compute_ssw], n_rks x (compute_residual,
    // [compute_residual_norm], update_solution): one step on the device; the
    // output-time counter it returns tells whether compute_dt clamped the step
    double info[5];
    check(tg_advance(h, fv.counter, 1, info), "tg_advance", h);
    fv.elapsed_time = info[0];
    fv.dt_global = info[1];
    fv.residual_norm_total = info[2];
    if ((int)info[4] > fv.counter) fv.time_instance_reached = true;
    ++iter;
    if (p.time_mode == "steady") term_iter = iter;

    const bool out_now = (p.time_mode == "steady" && iter % p.write_frequency == 0 && p.write_soln) ||
                         (fv.time_instance_reached && p.time_mode == "unsteady");
    const bool restart_now = p.write_restart && (iter % p.restart_write_frequency == 0 || fv.elapsed_time == p.final_time);
    const bool last = !(fv.residual_norm_total > p.min_residue && SafeLess(term_iter, p.max_iter) &&
                        fv.elapsed_time < p.final_time);
    if (every_step || out_now || restart_now || last) fetch_state(fv, h, hs, out_now, TG_GRAD_LAST_STAGE);

    if (p.write_log) fv.log_messages(iter);
    fv.compute_forces(iter);     // Navier-Stokes: forms dE of the current state on the host (src/force.cc:124)
    fv.compute_global(iter);

    if (p.time_mode == "steady" && iter % p.write_frequency == 0 && p.write_soln) {
      fv.output();
    } else if (fv.time_instance_reached && p.time_mode == "unsteady") {
      if (p.write_soln) fv.output();
      if (p.online_stat) fv.increment_moments(sample_id);
      fv.counter++;
      fv.time_instance_reached = false;
    }
    if (restart_now) {
      double r0 = 0.0;
      check(tg_query(h, TG_Q_RESIDUAL_NORM0, &r0), "tg_query", h);
      fv.residual_norm_total0 = r0;
      fv.output_restart(iter);
    }
  }
  if (p.time_mode == "steady") {
    fv.write_to_master = true;
    fv.time_instance[1] = fv.elapsed_time;
    if (p.write_soln) fv.output();
    if (p.online_stat) fv.increment_moments(sample_id);
    MPI_LOC_ASSERT(fv.counter == 1);
  } else {
    MPI_LOC_ASSERT(SafeEq(fv.counter, fv.time_instance.size()));
  }
  if (p.find_error) fv.compute_error_norm();
  fv.t_sample_solve.add_time();
}

// FiniteVolume::run (src/fv.cc:2401-2492).
void run_gpu(FiniteVolume& fv) {
  fv.t_total.start_time();
  fv.t_grid.start_time();
  fv.grid.read(fv.param);
  fv.t_grid.add_time();
  if (preprocess) return;
  fv.create_force_face_list();
  fv.initialize();

  MeshArrays ma;
  build_mesh(fv.grid, ma);
  BcArrays ba;
  build_bc(fv, ba);
  const tg_material mat = material_of(fv.param.material);
  const tg_options opt = options_of(fv.param);
  tg_handle* h = nullptr;
  check(tg_create(&ma.mesh, &mat, &ba.bc, &opt, &h), "tg_create", nullptr);
  HostState hs((int)fv.grid.n_vertex);

  std::cout << "  Starting simulations ...\n    Samples completed:\n";
  for (int ind = fv.param.sample_start_ind; ind <= fv.param.sample_end_ind; ++ind) {
    int sample_no = fv.param.SAMPLE_LIST[ind];
    fv.counter = 0;
    fv.initialize_sample_run(ind);
    if ((fv.elapsed_time < fv.param.final_time && fv.param.time_mode == "unsteady") ||
        (fv.last_iter < fv.param.max_iter && fv.param.time_mode == "steady"))
      solve_gpu(fv, h, hs, ind);
    fv.end_sample_run();
    if (check_group_base()) std::cout << "     --- " << sample_no << " ... " << std::endl;
  }
  tg_destroy(h);

  if (fv.param.online_stat && !fv.found_stop_file) {
    fv.reduce_moments();
    for (fv.counter = 0; SafeLess(fv.counter, fv.time_instance.size()); ++fv.counter) {
      fv.output_mean();
      fv.output_sec_mom();
      fv.output_var();
    }
    fv.compute_stat_norm();
    fv.reduce_stat_norm();
    fv.save_stat_norm();
  }
  fv.t_total.add_time();
}

}  // namespace

int main(int argc, char* argv[]) {
  mpi_init(argc, argv);
  int ifile = 0, iloc = 0;
  process_command_line(argc, argv, ifile, iloc, NPART);
  PERIODIC = false;
  if (NPART != 1) die("one partition only", "the device path has no MPI (-npart 1)");
  N_MC_GROUPS = 1;
  FiniteVolume problem(argv[ifile], argv[iloc]);
  // src/fv.h:171 leaves found_stop_file uninitialised; its stop-file check is commented out
  problem.found_stop_file = false;
  run_gpu(problem);
  std::cout << "\n\n---------------Solver has finished!!----------------------\n";
  mpi_finalize();
  return 0;
}
