// Caller-side smoke of the C++ drop-in (include/md_b200.hpp), written the way
// the reference's drivers use MDSimulation / EnergyMinimizer
// (tests/nph/nph_smoke.cpp, tests/run_test/run_test.cpp in MD_Simulation_CUDA):
// config from JSON plus overrides, lattice construction, NVE / Nose-Hoover /
// NPH / piston steps, observables, save_env and the constructor from a PFRAME
// file, and the two-particle FIRE quench. Exits 0 and prints "shim smoke OK"
// when every check holds.
//
//   shim_smoke <config.json> <scratch.pframe>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "md_b200.hpp"

namespace {

int failures = 0;

void expect(bool ok, const char* what) {
  if (!ok) {
    std::fprintf(stderr, "FAILED: %s\n", what);
    ++failures;
  }
}

bool finite_frame(const std::vector<Particle>& f) {
  for (const Particle& p : f)
    if (!std::isfinite(p.pos.x) || !std::isfinite(p.pos.y) || !std::isfinite(p.vel.x) ||
        !std::isfinite(p.vel.y) || !std::isfinite(p.acc.x) || !std::isfinite(p.acc.y))
      return false;
  return true;
}

struct FakeComm {};  // stands in for MPI_Comm; the drop-in ignores it

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: shim_smoke <config.json> <scratch.pframe>\n");
    return 2;
  }
  try {
    MDConfigManager cm = MDConfigManager::config_from_json(argv[1]);
    std::string key, value;
    expect(MDConfigManager::parse_override_argument("--DT_init=1.0", key, value),
           "parse_override_argument");
    expect(key == "T_init" && value == "1.0", "override key/value");
    expect(cm.apply_override(key, value), "apply_override");
    expect(!cm.apply_override("no_such_key", "1"), "unknown override rejected");
    expect(cm.config.T_init == 1.0, "T_init applied");
    MDConfigManager round;
    round.deserialize(cm.serialize());
    expect(round.serialize() == cm.serialize(), "serialize/deserialize round trip");

    const FakeComm comm;
    MDSimulation sim(cm, comm);
    const double E0 = sim.cal_total_K() + sim.cal_total_U();
    for (int s = 0; s < 200; ++s) sim.step_single_NVE();
    const double E1 = sim.cal_total_K() + sim.cal_total_U();
    expect(std::isfinite(E0) && std::fabs(E1 - E0) <= 1e-3 * std::fabs(E0), "NVE energy");

    for (int s = 0; s < 50; ++s) sim.step_single_nose_hoover();
    expect(std::isfinite(sim.get_xi()), "Nose-Hoover xi finite");

    const double A0 = sim.get_Lx() * sim.get_Ly();
    for (int s = 0; s < 50; ++s) sim.step_single_NPH(1.0);
    const double P = sim.cal_instant_pressure();
    expect(std::isfinite(P) && std::isfinite(sim.get_last_instant_pressure()), "NPH pressure");
    expect(sim.get_Lx() * sim.get_Ly() != A0, "NPH moves the box");
    expect(std::fabs(sim.get_Lx() / sim.get_Ly() - cm.config.box_w_global /
                                                       cm.config.box_h_global) < 1e-9,
           "NPH keeps the aspect ratio");

    for (int s = 0; s < 20; ++s) sim.step_single_NPH_piston(1.0);
    expect(std::isfinite(sim.get_nph_piston_velocity()) &&
               std::isfinite(sim.get_nph_piston_force()),
           "piston observables");

    sim.sample_collect();
    std::vector<Particle> frame;
    sim.get_host_particles(frame);
    expect((int)frame.size() == cm.config.n_particles_global, "frame size");
    expect(finite_frame(frame), "frame finite");

    std::remove(argv[2]);
    sim.save_env(argv[2], 7);
    MDSimulation again(cm, comm, argv[2], 7);
    std::vector<Particle> back;
    again.sample_collect();
    again.get_host_particles(back);
    bool same = back.size() == frame.size();
    for (size_t i = 0; same && i < frame.size(); ++i)
      same = back[i].pos.x == frame[i].pos.x && back[i].pos.y == frame[i].pos.y &&
             back[i].vel.x == frame[i].vel.x && back[i].type == frame[i].type;
    expect(same, "save_env + constructor from file");

    std::vector<double> prof = again.get_pressure_profile(8);
    expect(prof.size() == 24 && std::isfinite(prof[0]), "get_pressure_profile");
    std::vector<int> counts = again.get_N_profile(8);
    int total = 0;
    for (int c : counts) total += c;
    expect(total == cm.config.n_particles_global, "get_N_profile counts every particle");
    expect(std::isfinite(again.cal_partial_U_lambda(0.01)), "cal_partial_U_lambda");

    bool threw = false;
    try {
      MDConfigManager bad = cm;
      bad.config.box_w_global = -1.0;
      MDSimulation broken(bad, comm);
    } catch (const mdb200::Error& e) {
      threw = e.code() == MDB_ERR_BOX;
    }
    expect(threw, "invalid box raises mdb200::Error(MDB_ERR_BOX)");

    // run_test.cpp's FIRE smoke: (1,1) and (3,1) in a 10 x 10 box, sigma =
    // epsilon = 1; here run to convergence, which puts r at 2^(1/6).
    MDConfig c2;
    c2.n_particles_global = 2;
    c2.n_particles_type0 = 2;
    c2.box_w_global = 10.0;
    c2.box_h_global = 10.0;
    c2.SIGMA_AA = c2.SIGMA_BB = c2.SIGMA_AB = 1.0;
    c2.EPSILON_AA = c2.EPSILON_BB = c2.EPSILON_AB = 1.0;
    c2.dt = 1e-3;
    EnergyMinimizer em(MDConfigManager(c2), comm);
    std::vector<Particle> two(2);
    two[0] = Particle{{1.0, 1.0}, {0.0, 0.0}, {0.0, 0.0}, 0, 0.0};
    two[1] = Particle{{3.0, 1.0}, {0.0, 0.0}, {0.0, 0.0}, 0, 0.0};
    MinimizeResult r = em.minimize_frame(two, 1e-6, 20000, FireParams::from_config(c2));
    const double dx = r.frame[1].pos.x - r.frame[0].pos.x;
    expect(r.converged, "FIRE converged");
    expect(std::fabs(dx - std::pow(2.0, 1.0 / 6.0)) < 1e-4, "FIRE distance 2^(1/6)");
    expect(!r.energy_steps.empty() && r.energy_steps.front() == 0, "FIRE energy trace");
  } catch (const std::exception& e) {
    std::fprintf(stderr, "exception: %s\n", e.what());
    return 1;
  }
  if (failures) return 1;
  std::printf("shim smoke OK\n");
  return 0;
}
