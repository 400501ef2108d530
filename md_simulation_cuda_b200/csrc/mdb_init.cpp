// Reference-style initial frame for MDSimulation(cfg, comm) without a file
// (MDSimulation::init_particles, src/md_env.cu:1276-1445):
//  - type 0 on a square lattice filling a central band of width devide_p*Lx,
//    type 1 on its own lattice over the rest, each lattice spacing shrunk by
//    1% until rows*cols covers its count; x shifted so the band is centred;
//  - positions jittered uniformly by +-1e-5, std::mt19937 seeded 12345;
//  - Gaussian velocities with sigma = sqrt(T_init/m), net momentum removed,
//    rescaled to K = (2N-2) T_init / 2;
//  - theta uniform in [0, 2 pi).
// The standard-library distributions of the same C++ runtime reproduce the
// reference's random streams.
#include <math.h>

#include <random>
#include <vector>

#include "mdb200.h"
#include "mdb_util.h"

namespace mdb {

namespace {
void fit_lattice(double width, double height, int count, double& spacing, int& cols, int& rows) {
  auto dims = [&]() {
    rows = (int)(height / spacing);
    cols = (int)(width / spacing);
    if (rows <= 0) rows = 1;
    if (cols <= 0) cols = 1;
  };
  dims();
  while ((long long)rows * cols < count) {
    spacing *= 0.99;
    dims();
  }
}
}  // namespace

int reference_initial_frame(const mdb_config_t& cfg, std::vector<mdb_particle_t>& out) {
  const int N = cfg.n_particles_global;
  const int N0 = cfg.n_particles_type0;
  const int N1 = N - N0;
  const double Lx = cfg.box_w_global, Ly = cfg.box_h_global;
  if (!(Lx > 0.0) || !(Ly > 0.0) || !std::isfinite(Lx) || !std::isfinite(Ly))
    return set_error(MDB_ERR_BOX, "box_w_global and box_h_global must be positive");
  if (N <= 0 || N0 <= 0 || N1 <= 0)
    return set_error(MDB_ERR_CONFIG,
                     "lattice initialisation needs n_particles_global > n_particles_type0 > 0");
  out.assign((size_t)N, mdb_particle_t{});
  const double band = Lx * cfg.devide_p;
  const double shift = Lx * (0.5 - cfg.devide_p / 2.0);
  std::mt19937 rng(12345);
  std::uniform_real_distribution<double> jitter(-1.0e-5, 1.0e-5);

  double sp0 = sqrt(band * Ly / N0);
  double sp1 = sqrt((Lx - band) * Ly / N1);
  int c0, r0, c1, r1;
  fit_lattice(band, Ly, N0, sp0, c0, r0);
  fit_lattice(Lx - band, Ly, N1, sp1, c1, r1);

  for (int j = 0; j < r0; ++j) {
    for (int i = 0; i < c0; ++i) {
      const int idx = j * c0 + i;
      if (idx >= N0) break;
      const double xl = (i + 0.5) * sp0;
      const double y = (j + 0.5) * sp0;
      if (xl >= band || y >= Ly) continue;
      const double x = fmod(xl + shift + Lx, Lx);
      out[idx].pos.x = x + jitter(rng);
      out[idx].pos.y = y + jitter(rng);
      out[idx].type = 0;
    }
  }
  for (int j = 0; j < r1; ++j) {
    for (int i = 0; i < c1; ++i) {
      const int idx = j * c1 + i + N0;
      if (idx >= N) break;
      const double xl = (i + 0.5) * sp1 + band;
      const double y = (j + 0.5) * sp1;
      if (xl >= Lx || y >= Ly) continue;
      const double x = fmod(xl + shift + Lx, Lx);
      out[idx].pos.x = x + jitter(rng);
      out[idx].pos.y = y + jitter(rng);
      out[idx].type = 1;
    }
  }

  const double mA = cfg.MASS_A, mB = cfg.MASS_B;
  const double total_mass = N0 * mA + N1 * mB;
  double px = 0.0, py = 0.0;
  for (int i = 0; i < N; ++i) {
    const double m = out[i].type == 0 ? mA : mB;
    std::normal_distribution<double> g(0.0, sqrt(cfg.T_init / m));
    out[i].vel.x = g(rng);
    out[i].vel.y = g(rng);
    px += m * out[i].vel.x;
    py += m * out[i].vel.y;
  }
  const double vcx = px / total_mass, vcy = py / total_mass;
  for (int i = 0; i < N; ++i) {
    out[i].vel.x -= vcx;
    out[i].vel.y -= vcy;
  }
  double K = 0.0;
  const double K_target = (2 * (double)N - 2) * 0.5 * cfg.T_init;
  for (int i = 0; i < N; ++i) {
    const double m = out[i].type == 0 ? mA : mB;
    K += 0.5 * m * (out[i].vel.x * out[i].vel.x + out[i].vel.y * out[i].vel.y);
  }
  const double f = sqrt(K_target / K);
  for (int i = 0; i < N; ++i) {
    out[i].vel.x *= f;
    out[i].vel.y *= f;
  }
  std::uniform_real_distribution<double> ang(0.0, 2.0 * M_PI);
  for (int i = 0; i < N; ++i) out[i].theta = ang(rng);
  return MDB_OK;
}

}  // namespace mdb
