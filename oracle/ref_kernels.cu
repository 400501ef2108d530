// Host driver for the reference's own CUDA kernels.
//
// TEST INFRASTRUCTURE ONLY. oracle/build_ref.py compiles the reference's
// unmodified src/md_cuda_common.cu (with the stand-in RAFT/RMM headers of
// oracle/ref_stubs/) together with this file into oracle/_ref/libref_kernels.so.
// The parity tests run the reference's kernels through it to pin the oracle
// and the product against the reference's own arithmetic, and bench.py times
// the reference's single-GPU step with it. Nothing in the product links it.
//
// What this file restates is the reference's HOST logic around those kernels,
// at MPI world size 1 and without MPI:
//   cal_forces / cal_forces_piston        src/md_env.cu:1511-1574
//   step_single_NVE                       src/md_env.cu:1576-1637
//   step_single_nose_hoover               src/md_env.cu:1639-1728
//   init_nph_state_if_needed, step_single_NPH      src/md_env.cu:1757-1778, 1795-1918
//   init_nph_piston_state_if_needed, step_single_NPH_piston  :1780-1793, 1920-2023
//   cal_total_K / compute_kinetic_energy_local     :2141-2146, 2268-2303
//   evaluate_piston_wall_observables      :2148-2203
//   cal_total_scalar_pressure             :2205-2252
//   compute_U_energy_local / cal_total_U  :2305-2360
//   update_halo at world size 1           :757-998 (left = right = self)
// Every kernel launched here is the reference's (declared in
// include/md_cuda_common.hpp); block partial sums are copied to the host and
// summed in block order, as the reference does. With ws1_halo = 0 no halo is
// built (the physically correct force); with ws1_halo = 1 the world-size-1
// self-halo of update_halo is rebuilt before every force evaluation, where
// the reference rebuilds it. Particle migration (update_d_particles) is the
// identity at world size 1 for wrapped positions and is not restated.
#include <cuda_runtime.h>
#include <thrust/device_vector.h>
#include <thrust/scan.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "md_cuda_common.hpp"
#include "md_particle.hpp"

extern "C" {

typedef struct refk_lj {
  double sigma[3];   // AA, BB, AB
  double epsilon[3]; // AA, BB, AB
  double mass_a, mass_b, cutoff;
} refk_lj_t;

typedef struct refk_params {
  double dt, Q, T_target, barostat_mass, k_piston, area_rate_init, hmin_ratio, hmax_ratio;
  int64_t n_global;
  int32_t threads;   // THREADS_PER_BLOCK
  int32_t ws1_halo;  // rebuild the world-size-1 self-halo before each force call
} refk_params_t;

typedef struct refk_state {
  double Lx, Ly, Lx0, Ly0, t, xi;
  double nph_area_momentum, nph_aspect_ratio, piston_velocity, piston_force, last_P;
  int32_t nph_init, piston_vel_init, piston_active, n_halo_left, n_halo_right, pad;
} refk_state_t;

}  // extern "C"

namespace {

struct Sim {
  refk_lj_t lj;
  refk_params_t prm;
  refk_state_t st;
  int n = 0;
  thrust::device_vector<Particle> d;
  thrust::device_vector<Particle> halo_left, halo_right;
  thrust::device_vector<int> flags_left, flags_right, pos_left, pos_right;
  thrust::device_vector<double> partial, partial2;
};

int check(cudaError_t e) { return e == cudaSuccess ? 0 : 100 + (int)e; }
int last() { return check(cudaGetLastError()); }

int threads_of(const Sim& s) { return s.prm.threads > 0 ? s.prm.threads : 256; }
int blocks_of(const Sim& s) { return (s.n + threads_of(s) - 1) / threads_of(s); }
Particle* P(Sim& s) { return thrust::raw_pointer_cast(s.d.data()); }
Particle* HL(Sim& s) { return thrust::raw_pointer_cast(s.halo_left.data()); }
Particle* HR(Sim& s) { return thrust::raw_pointer_cast(s.halo_right.data()); }

// update_halo (src/md_env.cu:757-998) at world size 1: the strip within
// halo_width of x_min = 0 is sent left and comes back as the right halo; the
// strip near x_max = Lx is sent right and comes back as the left halo.
int update_halo(Sim& s) {
  s.st.n_halo_left = 0;
  s.st.n_halo_right = 0;
  if (!s.prm.ws1_halo || s.n <= 0) return 0;
  const double smax = std::max(s.lj.sigma[0], std::max(s.lj.sigma[1], s.lj.sigma[2]));
  const double halo_width = s.lj.cutoff * smax * 1.2;
  const int n = s.n, th = threads_of(s), bl = blocks_of(s);
  s.flags_left.resize(n);
  s.flags_right.resize(n);
  s.pos_left.resize(n);
  s.pos_right.resize(n);
  mark_halo_kernel<<<bl, th>>>(P(s), n, 0.0, s.st.Lx, s.st.Lx, halo_width,
                               thrust::raw_pointer_cast(s.flags_left.data()),
                               thrust::raw_pointer_cast(s.flags_right.data()));
  if (int e = last()) return e;
  if (int e = check(cudaDeviceSynchronize())) return e;
  thrust::exclusive_scan(s.flags_left.begin(), s.flags_left.end(), s.pos_left.begin());
  thrust::exclusive_scan(s.flags_right.begin(), s.flags_right.end(), s.pos_right.begin());
  const int send_left = (int)s.pos_left[n - 1] + (int)s.flags_left[n - 1];
  const int send_right = (int)s.pos_right[n - 1] + (int)s.flags_right[n - 1];
  s.halo_right.resize(std::max(send_left, 1));
  s.halo_left.resize(std::max(send_right, 1));
  if (send_left > 0)
    pack_halo_kernel<<<bl, th>>>(P(s), n, thrust::raw_pointer_cast(s.flags_left.data()),
                                 thrust::raw_pointer_cast(s.pos_left.data()), send_left, HR(s));
  if (send_right > 0)
    pack_halo_kernel<<<bl, th>>>(P(s), n, thrust::raw_pointer_cast(s.flags_right.data()),
                                 thrust::raw_pointer_cast(s.pos_right.data()), send_right, HL(s));
  if (int e = last()) return e;
  if (int e = check(cudaDeviceSynchronize())) return e;
  s.st.n_halo_left = send_right;
  s.st.n_halo_right = send_left;
  return 0;
}

int cal_forces(Sim& s, int periodic_y) {
  if (s.n <= 0) return 0;
  li_force_kernel<<<blocks_of(s), threads_of(s)>>>(
      P(s), HL(s), HR(s), s.n, s.st.n_halo_left, s.st.n_halo_right, s.st.Lx, s.st.Ly,
      s.lj.sigma[0], s.lj.sigma[1], s.lj.sigma[2], s.lj.epsilon[0], s.lj.epsilon[1],
      s.lj.epsilon[2], s.lj.cutoff, s.lj.mass_a, s.lj.mass_b, periodic_y);
  if (int e = last()) return e;
  return check(cudaDeviceSynchronize());
}

// Sum of per-block partials in block order (the reference's host loops).
int host_sum(thrust::device_vector<double>& part, int blocks, double* total, double* out) {
  std::vector<double> h((size_t)blocks);
  if (int e = check(cudaMemcpy(h.data(), thrust::raw_pointer_cast(part.data()),
                               sizeof(double) * (size_t)blocks, cudaMemcpyDeviceToHost)))
    return e;
  double acc = 0.0;
  for (int i = 0; i < blocks; ++i) acc += h[(size_t)i];
  *total = acc;
  if (out) std::memcpy(out, h.data(), sizeof(double) * (size_t)blocks);
  return 0;
}

int total_K(Sim& s, double* K, double* partials) {
  *K = 0.0;
  if (s.n <= 0) return 0;
  const int th = threads_of(s), bl = blocks_of(s);
  s.partial.resize(bl);
  cal_local_K_kernel<<<bl, th, th * (int)sizeof(double)>>>(
      P(s), s.n, s.lj.mass_a, s.lj.mass_b, thrust::raw_pointer_cast(s.partial.data()));
  if (int e = last()) return e;
  if (int e = check(cudaDeviceSynchronize())) return e;
  return host_sum(s.partial, bl, K, partials);
}

int pressure_sum(Sim& s, int periodic_y, double* sum, double* partials) {
  *sum = 0.0;
  if (s.n <= 0) return 0;
  const int th = threads_of(s), bl = blocks_of(s);
  s.partial.resize(bl);
  cal_local_pressure_scalar_kernel<<<bl, th, th * (int)sizeof(double)>>>(
      P(s), HL(s), HR(s), s.n, s.st.n_halo_left, s.st.n_halo_right, s.st.Lx, s.st.Ly,
      s.lj.mass_a, s.lj.mass_b, s.lj.sigma[0], s.lj.sigma[1], s.lj.sigma[2], s.lj.epsilon[0],
      s.lj.epsilon[1], s.lj.epsilon[2], s.lj.cutoff, thrust::raw_pointer_cast(s.partial.data()),
      periodic_y);
  if (int e = last()) return e;
  if (int e = check(cudaDeviceSynchronize())) return e;
  return host_sum(s.partial, bl, sum, partials);
}

int scalar_pressure(Sim& s, int periodic_y, double* Pout) {
  double sum = 0.0;
  if (int e = pressure_sum(s, periodic_y, &sum, nullptr)) return e;
  const double area = s.st.Lx * s.st.Ly;
  *Pout = (area > 0.0) ? sum / (2.0 * area) : 0.0;
  return 0;
}

int total_U_pairs(Sim& s, int periodic_y, double* U, double* partials) {
  *U = 0.0;
  if (s.n <= 0) return 0;
  const int th = threads_of(s), bl = blocks_of(s);
  s.partial.resize(bl);
  cal_local_U_kernel<<<bl, th, th * (int)sizeof(double)>>>(
      P(s), HL(s), HR(s), s.n, s.st.n_halo_left, s.st.n_halo_right, s.st.Lx, s.st.Ly,
      s.lj.sigma[0], s.lj.sigma[1], s.lj.sigma[2], s.lj.epsilon[0], s.lj.epsilon[1],
      s.lj.epsilon[2], s.lj.cutoff, thrust::raw_pointer_cast(s.partial.data()), periodic_y);
  if (int e = last()) return e;
  if (int e = check(cudaDeviceSynchronize())) return e;
  return host_sum(s.partial, bl, U, partials);
}

int piston_wall(Sim& s, int update_acc, double* upper, double* energy) {
  *upper = 0.0;
  *energy = 0.0;
  if (s.n <= 0 || !(s.prm.k_piston > 0.0)) return 0;
  const int th = threads_of(s), bl = blocks_of(s);
  s.partial.resize(bl);
  s.partial2.resize(bl);
  piston_wall_kernel<<<bl, th, 2 * th * (int)sizeof(double)>>>(
      P(s), s.n, s.st.Ly, s.prm.k_piston, s.lj.mass_a, s.lj.mass_b, update_acc != 0,
      thrust::raw_pointer_cast(s.partial.data()), thrust::raw_pointer_cast(s.partial2.data()));
  if (int e = last()) return e;
  if (int e = check(cudaDeviceSynchronize())) return e;
  if (int e = host_sum(s.partial, bl, upper, nullptr)) return e;
  return host_sum(s.partial2, bl, energy, nullptr);
}

int total_U(Sim& s, double* U, double* partials) {
  const int periodic_y = s.st.piston_active ? 0 : 1;
  if (int e = total_U_pairs(s, periodic_y, U, partials)) return e;
  if (!s.st.piston_active) return 0;
  double up = 0.0, en = 0.0;
  if (int e = piston_wall(s, 0, &up, &en)) return e;
  *U += en;
  return 0;
}

int cal_forces_piston(Sim& s) {
  if (int e = cal_forces(s, 0)) return e;
  double up = 0.0, en = 0.0;
  if (int e = piston_wall(s, 1, &up, &en)) return e;
  s.st.piston_force = up;
  return 0;
}

double floor_of(const Sim& s) { return std::max(1e-12, s.prm.hmin_ratio * s.st.Ly0); }
double ceil_of(const Sim& s) { return std::max(floor_of(s), s.prm.hmax_ratio * s.st.Ly0); }

int sync_last() {
  if (int e = last()) return e;
  return check(cudaDeviceSynchronize());
}

int step_nve(Sim& s) {
  s.st.piston_active = 0;
  const int th = threads_of(s), bl = blocks_of(s);
  if (s.n > 0) {
    step_half_vv_kernel<<<bl, th>>>(P(s), s.n, s.prm.dt, s.st.Lx, s.st.Ly);
    if (int e = sync_last()) return e;
  }
  if (int e = update_halo(s)) return e;
  if (int e = cal_forces(s, 1)) return e;
  if (s.n > 0) {
    step_2nd_half_vv_kernel<<<bl, th>>>(P(s), s.n, s.prm.dt);
    if (int e = sync_last()) return e;
  }
  s.st.t += s.prm.dt;
  return 0;
}

int step_nh(Sim& s) {
  s.st.piston_active = 0;
  const double dt = s.prm.dt;
  const int th = threads_of(s), bl = blocks_of(s);
  double K = 0.0;
  if (int e = total_K(s, &K, nullptr)) return e;
  const double g_dof = 2.0 * (double)s.prm.n_global - 2.0;
  const double T0 = s.prm.T_target, Q = s.prm.Q;
  s.st.xi += 0.5 * dt * (2.0 * K - g_dof * T0) / Q;
  if (s.n > 0) {
    step_half_vv_nh_kernel<<<bl, th>>>(P(s), s.n, dt, s.st.xi, s.st.Lx, s.st.Ly);
    if (int e = sync_last()) return e;
  }
  if (int e = update_halo(s)) return e;
  if (int e = cal_forces(s, 1)) return e;
  if (int e = total_K(s, &K, nullptr)) return e;
  s.st.xi += 0.5 * dt * (2.0 * K - g_dof * T0) / Q;
  if (s.n > 0) {
    step_2nd_half_vv_nh_kernel<<<bl, th>>>(P(s), s.n, dt, s.st.xi);
    if (int e = sync_last()) return e;
  }
  if (int e = total_K(s, &K, nullptr)) return e;
  s.st.t += dt;
  return 0;
}

void init_nph(Sim& s) {
  if (s.st.nph_init) return;
  s.st.nph_aspect_ratio = s.st.Lx / s.st.Ly;
  s.st.nph_area_momentum = std::max(s.prm.barostat_mass, 1e-12) * s.prm.area_rate_init;
  s.st.nph_init = 1;
}

int step_nph(Sim& s, double p_ext) {
  s.st.piston_active = 0;
  init_nph(s);
  const double dt = s.prm.dt;
  const double W = std::max(s.prm.barostat_mass, 1e-12);
  const int th = threads_of(s), bl = blocks_of(s);
  const double Lx_old = s.st.Lx, Ly_old = s.st.Ly;
  const double area_old = Lx_old * Ly_old;
  if (area_old <= 0.0) return 5;
  double p_old = 0.0;
  if (int e = scalar_pressure(s, 1, &p_old)) return e;
  if (s.n > 0) {
    step_half_nph_velocity_kernel<<<bl, th>>>(P(s), s.n, dt);
    if (int e = sync_last()) return e;
  }
  s.st.nph_area_momentum += 0.5 * dt * (p_old - p_ext);
  double area_new = area_old + dt * (s.st.nph_area_momentum / W);
  if (!(area_new > 0.0) || !std::isfinite(area_new)) return 5;
  if (!(s.st.nph_aspect_ratio > 0.0) || !std::isfinite(s.st.nph_aspect_ratio))
    s.st.nph_aspect_ratio = Lx_old / Ly_old;
  double Ly_new = std::sqrt(area_new / s.st.nph_aspect_ratio);
  double Lx_new = s.st.nph_aspect_ratio * Ly_new;
  const double fl = floor_of(s), ce = ceil_of(s);
  bool clamped = false;
  if (Ly_new < fl) {
    Ly_new = fl;
    Lx_new = s.st.nph_aspect_ratio * Ly_new;
    area_new = Lx_new * Ly_new;
    clamped = true;
  } else if (Ly_new > ce) {
    Ly_new = ce;
    Lx_new = s.st.nph_aspect_ratio * Ly_new;
    area_new = Lx_new * Ly_new;
    clamped = true;
  }
  const double lin = std::sqrt(area_new / area_old);
  const double vsc = 1.0 / lin;
  if (s.n > 0) {
    step_nph_scale_and_drift_kernel<<<bl, th>>>(P(s), s.n, dt, lin, vsc, Lx_new, Ly_new);
    if (int e = sync_last()) return e;
  }
  if (Lx_new <= 0.0 || Ly_new <= 0.0) return 5;
  s.st.Lx = Lx_new;
  s.st.Ly = Ly_new;
  if (int e = update_halo(s)) return e;
  if (int e = cal_forces(s, 1)) return e;
  double p_new = 0.0;
  if (int e = scalar_pressure(s, 1, &p_new)) return e;
  if (s.n > 0) {
    step_2nd_half_vv_kernel<<<bl, th>>>(P(s), s.n, dt);
    if (int e = sync_last()) return e;
  }
  s.st.nph_area_momentum += 0.5 * dt * (p_new - p_ext);
  if (clamped) {
    if (s.st.Ly <= fl && s.st.nph_area_momentum < 0.0) s.st.nph_area_momentum = 0.0;
    if (s.st.Ly >= ce && s.st.nph_area_momentum > 0.0) s.st.nph_area_momentum = 0.0;
  }
  s.st.last_P = p_new;
  s.st.t += dt;
  return 0;
}

int init_piston(Sim& s) {
  if (!s.st.piston_vel_init) {
    s.st.piston_velocity = 0.0;
    s.st.piston_vel_init = 1;
  }
  if (!s.st.piston_active) {
    s.st.piston_active = 1;
    if (int e = cal_forces_piston(s)) return e;
    s.st.last_P = (s.st.Lx > 0.0) ? (s.st.piston_force / s.st.Lx) : 0.0;
  }
  return 0;
}

int step_piston(Sim& s, double p_ext) {
  if (int e = init_piston(s)) return e;
  const double dt = s.prm.dt;
  const double W = std::max(s.prm.barostat_mass, 1e-12);
  const int th = threads_of(s), bl = blocks_of(s);
  const double Lx = s.st.Lx, Ly_old = s.st.Ly;
  if (Lx <= 0.0 || Ly_old <= 0.0) return 5;
  const double acc_old = (s.st.piston_force - p_ext * Lx) / W;
  if (s.n > 0) {
    step_half_vv_piston_kernel<<<bl, th>>>(P(s), s.n, dt, Lx);
    if (int e = sync_last()) return e;
  }
  s.st.piston_velocity += 0.5 * dt * acc_old;
  double Ly_new = Ly_old + dt * s.st.piston_velocity;
  const double fl = floor_of(s), ce = ceil_of(s);
  bool clamped = false;
  if (Ly_new < fl) {
    Ly_new = fl;
    clamped = true;
    if (s.st.piston_velocity < 0.0) s.st.piston_velocity = 0.0;
  } else if (Ly_new > ce) {
    Ly_new = ce;
    clamped = true;
    if (s.st.piston_velocity > 0.0) s.st.piston_velocity = 0.0;
  }
  if (Ly_new <= 0.0) return 5;
  s.st.Ly = Ly_new;
  if (int e = update_halo(s)) return e;
  if (int e = cal_forces_piston(s)) return e;
  if (s.n > 0) {
    step_2nd_half_vv_kernel<<<bl, th>>>(P(s), s.n, dt);
    if (int e = sync_last()) return e;
  }
  const double acc_new = (s.st.piston_force - p_ext * Lx) / W;
  s.st.piston_velocity += 0.5 * dt * acc_new;
  if (clamped) {
    if (s.st.Ly <= fl && s.st.piston_velocity < 0.0) s.st.piston_velocity = 0.0;
    if (s.st.Ly >= ce && s.st.piston_velocity > 0.0) s.st.piston_velocity = 0.0;
  }
  s.st.last_P = s.st.piston_force / Lx;
  s.st.t += dt;
  return 0;
}

int step_one(Sim& s, int kind, double p_ext) {
  switch (kind) {
    case 0: return step_nve(s);
    case 1: return step_nh(s);
    case 2: return step_nph(s, p_ext);
    case 3: return step_piston(s, p_ext);
    default: return 2;
  }
}

Sim& S(void* h) { return *reinterpret_cast<Sim*>(h); }

}  // namespace

extern "C" {

typedef struct refk_sim refk_sim_t;

int refk_device_count(void) {
  int c = 0;
  if (cudaGetDeviceCount(&c) != cudaSuccess) return 0;
  return c;
}

// A simulation over a host frame of n 64-byte Particle records (include/
// md_particle.hpp:31-38), box Lx x Ly. Nothing is computed; the caller then
// calls refk_cal_forces as the MDSimulation constructor does.
int refk_create(const refk_lj_t* lj, const refk_params_t* prm, int32_t n, const void* frame,
                double Lx, double Ly, refk_sim_t** out) {
  if (!lj || !prm || !out || n < 0 || (n > 0 && !frame)) return 2;
  Sim* s = nullptr;
  try {
    s = new Sim();
    s->lj = *lj;
    s->prm = *prm;
    std::memset(&s->st, 0, sizeof(s->st));
    s->st.Lx = Lx;
    s->st.Ly = Ly;
    s->st.Lx0 = Lx;
    s->st.Ly0 = Ly;
    s->n = n;
    std::vector<Particle> h((size_t)n);
    if (n > 0) std::memcpy(h.data(), frame, sizeof(Particle) * (size_t)n);
    s->d = h;
    s->halo_left.resize(1);
    s->halo_right.resize(1);
  } catch (...) {
    delete s;
    return 3;
  }
  *out = reinterpret_cast<refk_sim_t*>(s);
  return check(cudaDeviceSynchronize());
}

void refk_destroy(refk_sim_t* h) { delete reinterpret_cast<Sim*>(h); }

int refk_get_frame(refk_sim_t* h, void* frame) {
  Sim& s = S(h);
  if (s.n > 0)
    return check(cudaMemcpy(frame, P(s), sizeof(Particle) * (size_t)s.n, cudaMemcpyDeviceToHost));
  return 0;
}

int refk_set_frame(refk_sim_t* h, const void* frame) {
  Sim& s = S(h);
  if (s.n > 0)
    return check(cudaMemcpy(P(s), frame, sizeof(Particle) * (size_t)s.n, cudaMemcpyHostToDevice));
  return 0;
}

int refk_get_state(refk_sim_t* h, refk_state_t* out) {
  *out = S(h).st;
  return 0;
}

int refk_set_state(refk_sim_t* h, const refk_state_t* in) {
  S(h).st = *in;
  return 0;
}

// update_halo (world size 1, when ws1_halo) then li_force_kernel.
int refk_cal_forces(refk_sim_t* h, int32_t periodic_y) {
  if (int e = update_halo(S(h))) return e;
  return cal_forces(S(h), periodic_y);
}

int refk_total_K(refk_sim_t* h, double* K, double* partials) {
  return total_K(S(h), K, partials);
}

// cal_local_U_kernel partials (and wall energy in piston mode), block order.
int refk_total_U(refk_sim_t* h, double* U, double* partials) { return total_U(S(h), U, partials); }

// Numerator sum of cal_local_pressure_scalar_kernel (sum m v^2 + 1/2 sum r.F)
// and its block partials; P = sum / (2 Lx Ly).
int refk_pressure_sum(refk_sim_t* h, int32_t periodic_y, double* sum, double* partials) {
  return pressure_sum(S(h), periodic_y, sum, partials);
}

int refk_piston_wall(refk_sim_t* h, int32_t update_acc, double* upper, double* energy) {
  return piston_wall(S(h), update_acc, upper, energy);
}

// cal_partial_U_lambda_kernel (src/md_cuda_common.cu:266-377): block
// partials and their block-order sum.
int refk_partial_U_lambda(refk_sim_t* h, double epsilon_lambda, int32_t periodic_y, double* total,
                          double* partials) {
  Sim& s = S(h);
  *total = 0.0;
  if (s.n <= 0) return 0;
  const int th = threads_of(s), bl = blocks_of(s);
  s.partial.resize(bl);
  cal_partial_U_lambda_kernel<<<bl, th, th * (int)sizeof(double)>>>(
      P(s), HL(s), HR(s), s.n, s.st.n_halo_left, s.st.n_halo_right, s.st.Lx, s.st.Ly,
      s.lj.sigma[0], s.lj.sigma[1], s.lj.sigma[2], s.lj.epsilon[0], s.lj.epsilon[1],
      s.lj.epsilon[2], s.lj.cutoff, epsilon_lambda, thrust::raw_pointer_cast(s.partial.data()),
      periodic_y);
  if (int e = sync_last()) return e;
  return host_sum(s.partial, bl, total, partials);
}

// One integrator kernel of the reference on the resident frame, alone:
// 0 step_half_vv_kernel(dt, Lx, Ly), 1 step_2nd_half_vv_kernel(dt),
// 2 step_half_vv_nh_kernel(dt, xi, Lx, Ly), 3 step_2nd_half_vv_nh_kernel(dt, xi),
// 4 step_half_nph_velocity_kernel(dt),
// 5 step_nph_scale_and_drift_kernel(dt, lin, vsc, Lx_new, Ly_new),
// 6 step_half_vv_piston_kernel(dt, Lx).
int refk_integrator(refk_sim_t* h, int32_t which, double dt, double xi, double lin, double vsc,
                    double Lx_new, double Ly_new) {
  Sim& s = S(h);
  if (s.n <= 0) return 0;
  const int th = threads_of(s), bl = blocks_of(s);
  switch (which) {
    case 0: step_half_vv_kernel<<<bl, th>>>(P(s), s.n, dt, s.st.Lx, s.st.Ly); break;
    case 1: step_2nd_half_vv_kernel<<<bl, th>>>(P(s), s.n, dt); break;
    case 2: step_half_vv_nh_kernel<<<bl, th>>>(P(s), s.n, dt, xi, s.st.Lx, s.st.Ly); break;
    case 3: step_2nd_half_vv_nh_kernel<<<bl, th>>>(P(s), s.n, dt, xi); break;
    case 4: step_half_nph_velocity_kernel<<<bl, th>>>(P(s), s.n, dt); break;
    case 5:
      step_nph_scale_and_drift_kernel<<<bl, th>>>(P(s), s.n, dt, lin, vsc, Lx_new, Ly_new);
      break;
    case 6: step_half_vv_piston_kernel<<<bl, th>>>(P(s), s.n, dt, s.st.Lx); break;
    default: return 2;
  }
  return sync_last();
}

// nsteps of one step kind (0 NVE, 1 Nose-Hoover, 2 NPH, 3 NPH piston). When
// given, K_trace / U_trace receive cal_total_K / cal_total_U after each step
// (outside the step; they add kernel launches of their own).
int refk_step(refk_sim_t* h, int32_t kind, double p_ext, int32_t nsteps, double* K_trace,
              double* U_trace) {
  Sim& s = S(h);
  for (int k = 0; k < nsteps; ++k) {
    if (int e = step_one(s, kind, p_ext)) return e;
    if (K_trace) {
      if (int e = total_K(s, K_trace + k, nullptr)) return e;
    }
    if (U_trace) {
      if (int e = total_U(s, U_trace + k, nullptr)) return e;
    }
  }
  return 0;
}

// Device time of nsteps steps: CUDA events on the default stream around the
// whole host-synchronous loop, which is how the reference issues its work.
int refk_time_steps(refk_sim_t* h, int32_t kind, double p_ext, int32_t nsteps, double* ms_total) {
  Sim& s = S(h);
  cudaEvent_t a, b;
  if (int e = check(cudaEventCreate(&a))) return e;
  if (int e = check(cudaEventCreate(&b))) {
    cudaEventDestroy(a);
    return e;
  }
  int rc = check(cudaDeviceSynchronize());
  if (!rc) rc = check(cudaEventRecord(a, 0));
  for (int k = 0; !rc && k < nsteps; ++k) rc = step_one(s, kind, p_ext);
  if (!rc) rc = check(cudaEventRecord(b, 0));
  if (!rc) rc = check(cudaEventSynchronize(b));
  float ms = 0.f;
  if (!rc) rc = check(cudaEventElapsedTime(&ms, a, b));
  *ms_total = ms;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return rc;
}

}  // extern "C"
