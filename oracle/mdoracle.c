/*
 * mdoracle.c — CPU restatement of the MD stepping path of MD_Simulation_CUDA.
 * TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline); see mdoracle.h
 * for the parity status ("parity unpinned" for the physics, pinned against
 * analytic known answers) and the arithmetic modes.
 *
 * Built with -ffp-contract=off: every fused multiply-add is an explicit fma()
 * / fmaf() call, so the operation order written here is the one executed.
 */
#include "mdoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* pbc_wrap_hd (include/md_cuda_common.hpp:20-29). */
double or_pbc_wrap(double x, double L) {
  if (L <= 0.0) return x;
  x = fmod(x, L);
  if (x < 0.0) x += L;
  return x;
}

/* Type -> LJ parameter set (src/md_cuda_common.cu:218-229): (0,0) AA,
 * (1,1) BB, anything else AB. */
static inline int pair_class(int ti, int tj) {
  if (ti == 0 && tj == 0) return 0;
  if (ti == 1 && tj == 1) return 1;
  return 2;
}

/* Mass of a type (src/md_cuda_common.cu:261): type 0 -> MASS_A, else MASS_B. */
static inline double type_mass(const or_lj_t* lj, int t) { return t == 0 ? lj->mass_a : lj->mass_b; }

/* Energy shift V_c = eps * 4 (c^-12 - c^-6), c = cutoff
 * (src/md_cuda_common.cu:719-727). */
static inline double shift_of(const or_lj_t* lj, int c) {
  const double inv_c = 1.0 / lj->cutoff;
  const double sr2 = inv_c * inv_c;
  const double sr6 = sr2 * sr2 * sr2;
  const double sr12 = sr6 * sr6;
  return lj->epsilon[c] * (4.0 * (sr12 - sr6));
}

typedef struct pair_acc {
  double fx, fy, u, w;
} pair_acc_t;

/* One ordered pair (i, j) in FP64: minimum image with round(), strict cutoff
 * 0 < r^2 < (cutoff*sigma)^2, truncated force, shifted energy. */
static inline void pair_fp64(const or_lj_t* lj, double xi, double yi, int ti, double xj, double yj,
                             int tj, double Lx, double Ly, int periodic_y, pair_acc_t* a) {
  double dx = xi - xj;
  double dy = yi - yj;
  dx = dx - Lx * round(dx / Lx);
  if (periodic_y) dy = dy - Ly * round(dy / Ly);
  const int c = pair_class(ti, tj);
  const double sig = lj->sigma[c];
  const double eps = lj->epsilon[c];
  const double rc = lj->cutoff * sig;
  const double r2 = dx * dx + dy * dy;
  if (r2 > 0.0 && r2 < rc * rc) {
    const double r2i = 1.0 / r2;
    const double sr2 = sig * sig * r2i;
    const double sr6 = sr2 * sr2 * sr2;
    const double sr12 = sr6 * sr6;
    const double tmp = 24.0 * eps * (2.0 * sr12 - sr6) * r2i;
    a->fx += tmp * dx;
    a->fy += tmp * dy;
    a->u += 0.5 * (4.0 * eps * (sr12 - sr6) - shift_of(lj, c));
    a->w += 0.5 * (dx * (tmp * dx) + dy * (tmp * dy));
  }
}

/* One ordered pair in the reference's mixed precision
 * (li_force_kernel src/md_cuda_common.cu:193-254; energy :795-807;
 * virial :676-686): FP64 difference cast to FP32, FP32 minimum image via
 * roundf, FP32 pair term, FP64 accumulation. */
static inline void pair_mixed(const or_lj_t* lj, double xi, double yi, int ti, double xj, double yj,
                              int tj, float Lx_f, float Ly_f, int periodic_y, pair_acc_t* a) {
  float dx_f = (float)(xi - xj);
  float dy_f = (float)(yi - yj);
  dx_f = fmaf(-Lx_f, roundf(dx_f / Lx_f), dx_f);
  if (periodic_y) dy_f = fmaf(-Ly_f, roundf(dy_f / Ly_f), dy_f);
  const int c = pair_class(ti, tj);
  const float sigma_f = (float)lj->sigma[c];
  const float epsilon_f = (float)lj->epsilon[c];
  const float cutoff_f = (float)lj->cutoff;
  const float rc_f = cutoff_f * sigma_f;
  const float rc_sq_f = rc_f * rc_f;
  const float dr_sq_f = fmaf(dx_f, dx_f, dy_f * dy_f);
  if (dr_sq_f > 0.0f && dr_sq_f < rc_sq_f) {
    const float sigma_sq_f = sigma_f * sigma_f;
    const float r2_inv_f = 1.0f / dr_sq_f;
    const float sr2_f = sigma_sq_f * r2_inv_f;
    const float sr6_f = sr2_f * sr2_f * sr2_f;
    const float sr12_f = sr6_f * sr6_f;
    const float tmp_f = (24.0f * epsilon_f) * fmaf(2.0f, sr12_f, -sr6_f) * r2_inv_f;
    const float fx_f = tmp_f * dx_f;
    const float fy_f = tmp_f * dy_f;
    a->fx += (double)fx_f;
    a->fy += (double)fy_f;
    /* the reference's build contracts sr6*sr6 - sr6 into one fused
     * multiply-add in cal_local_U_kernel (pinned against its outputs) */
    const float u_pair_f = (4.0f * epsilon_f) * fmaf(sr6_f, sr6_f, -sr6_f);
    a->u = fma(0.5, (double)u_pair_f - shift_of(lj, c), a->u);
    a->w = fma(0.5, fma((double)dx_f, (double)fx_f, (double)dy_f * (double)fy_f), a->w);
  }
}

static inline void do_pair(const or_lj_t* lj, int mode, double xi, double yi, int ti, double xj,
                           double yj, int tj, double Lx, double Ly, float Lx_f, float Ly_f,
                           int periodic_y, pair_acc_t* a) {
  if (mode == OR_FP64)
    pair_fp64(lj, xi, yi, ti, xj, yj, tj, Lx, Ly, periodic_y, a);
  else
    pair_mixed(lj, xi, yi, ti, xj, yj, tj, Lx_f, Ly_f, periodic_y, a);
}

static void set_threads(int32_t nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
}

/* Halo membership at world size 1 (mark_halo_kernel src/md_cuda_common.cu:67-91
 * with x_min = 0, x_max = Lx, halo_width = 1.2*cutoff*sigma_max from
 * src/md_env.cu:801-805). The halo arrays hold the right strip (received as
 * the left halo) followed by the left strip (the right halo). */
static int64_t build_ws1_halo(const or_lj_t* lj, int64_t n, const double* pos, double Lx,
                              int64_t* idx) {
  double smax = lj->sigma[0];
  if (lj->sigma[1] > smax) smax = lj->sigma[1];
  if (lj->sigma[2] > smax) smax = lj->sigma[2];
  const double h = lj->cutoff * smax * 1.2;
  int64_t m = 0;
  for (int64_t j = 0; j < n; ++j) { /* left halo = particles near x_max */
    const double x = or_pbc_wrap(pos[2 * j], Lx);
    const double dr = Lx - x;
    if (dr <= h && dr >= 0.0) idx[m++] = j;
  }
  for (int64_t j = 0; j < n; ++j) { /* right halo = particles near x_min */
    const double x = or_pbc_wrap(pos[2 * j], Lx);
    const double dl = x - 0.0;
    if (dl <= h && dl >= 0.0) idx[m++] = j;
  }
  return m;
}

/* li_force_kernel / cal_local_U_kernel / pressure pair loop, all pairs
 * (src/md_cuda_common.cu:151-264, 703-825, 591-701): for each i every j != i
 * (then every halo copy), acc_i = F_i / m_i. */
int or_forces_allpairs(const or_lj_t* lj, int64_t n, const double* pos, const int32_t* type,
                       double Lx, double Ly, int32_t periodic_y, int32_t mode, int32_t ws1_halo,
                       double* acc, double* U, double* W, int32_t nthreads) {
  if (n < 0) return 1;
  set_threads(nthreads);
  int64_t* halo = NULL;
  int64_t nh = 0;
  if (ws1_halo) {
    halo = (int64_t*)malloc(sizeof(int64_t) * (size_t)(2 * n + 1));
    if (!halo) return 2;
    nh = build_ws1_halo(lj, n, pos, Lx, halo);
  }
  double* ui = (double*)malloc(sizeof(double) * (size_t)(n + 1));
  double* wi = (double*)malloc(sizeof(double) * (size_t)(n + 1));
  if (!ui || !wi) {
    free(halo);
    free(ui);
    free(wi);
    return 2;
  }
  const float Lx_f = (float)Lx, Ly_f = (float)Ly;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < n; ++i) {
    pair_acc_t a = {0.0, 0.0, 0.0, 0.0};
    const double xi = pos[2 * i], yi = pos[2 * i + 1];
    const int ti = type[i];
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      do_pair(lj, mode, xi, yi, ti, pos[2 * j], pos[2 * j + 1], type[j], Lx, Ly, Lx_f, Ly_f,
              periodic_y, &a);
    }
    for (int64_t k = 0; k < nh; ++k) {
      const int64_t j = halo[k];
      do_pair(lj, mode, xi, yi, ti, pos[2 * j], pos[2 * j + 1], type[j], Lx, Ly, Lx_f, Ly_f,
              periodic_y, &a);
    }
    const double m = type_mass(lj, ti);
    if (acc) {
      acc[2 * i] = a.fx / m;
      acc[2 * i + 1] = a.fy / m;
    }
    ui[i] = a.u;
    wi[i] = a.w;
  }
  double su = 0.0, sw = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    su += ui[i];
    sw += wi[i];
  }
  if (U) *U = su;
  if (W) *W = sw;
  free(ui);
  free(wi);
  free(halo);
  return 0;
}

/* ---- the reference's block-reduced kernels, thread by thread -------------- */

/* The pair quantities the reference's pair loops share, in its mixed
 * arithmetic (src/md_cuda_common.cu:193-249, 616-688, 735-806, 293-361):
 * FP32 displacement and minimum image, strict FP32 cutoff, FP32 tmp and
 * u_pair. In FP64 mode the same quantities in double. */
typedef struct ref_pair {
  int in, c;
  double dx, dy, fx, fy, u; /* fx = double(tmp*dx) etc. (exact FP32 values in mixed mode) */
} ref_pair_t;

static inline ref_pair_t ref_pair_terms(const or_lj_t* lj, int mode, double xi, double yi, int ti,
                                        double xj, double yj, int tj, double Lx, double Ly,
                                        int periodic_y) {
  ref_pair_t r = {0, pair_class(ti, tj), 0.0, 0.0, 0.0, 0.0, 0.0};
  if (mode == OR_FP64) {
    double dx = xi - xj, dy = yi - yj;
    dx = dx - Lx * round(dx / Lx);
    if (periodic_y) dy = dy - Ly * round(dy / Ly);
    const double sig = lj->sigma[r.c], eps = lj->epsilon[r.c], rc = lj->cutoff * sig;
    const double r2 = dx * dx + dy * dy;
    if (!(r2 > 0.0 && r2 < rc * rc)) return r;
    const double r2i = 1.0 / r2;
    const double sr2 = sig * sig * r2i;
    const double sr6 = sr2 * sr2 * sr2;
    const double sr12 = sr6 * sr6;
    const double tmp = 24.0 * eps * (2.0 * sr12 - sr6) * r2i;
    r.in = 1;
    r.dx = dx;
    r.dy = dy;
    r.fx = tmp * dx;
    r.fy = tmp * dy;
    r.u = 4.0 * eps * (sr12 - sr6);
    return r;
  }
  const float Lx_f = (float)Lx, Ly_f = (float)Ly;
  float dx_f = (float)(xi - xj);
  float dy_f = (float)(yi - yj);
  dx_f = fmaf(-Lx_f, roundf(dx_f / Lx_f), dx_f);
  if (periodic_y) dy_f = fmaf(-Ly_f, roundf(dy_f / Ly_f), dy_f);
  const float sigma_f = (float)lj->sigma[r.c];
  const float epsilon_f = (float)lj->epsilon[r.c];
  const float rc_f = (float)lj->cutoff * sigma_f;
  const float rc_sq_f = rc_f * rc_f;
  const float dr_sq_f = fmaf(dx_f, dx_f, dy_f * dy_f);
  if (!(dr_sq_f > 0.0f && dr_sq_f < rc_sq_f)) return r;
  const float r2_inv_f = 1.0f / dr_sq_f;
  const float sr2_f = (sigma_f * sigma_f) * r2_inv_f;
  const float sr6_f = sr2_f * sr2_f * sr2_f;
  const float sr12_f = sr6_f * sr6_f;
  const float tmp_f = (24.0f * epsilon_f) * fmaf(2.0f, sr12_f, -sr6_f) * r2_inv_f;
  r.in = 1;
  r.dx = (double)dx_f;
  r.dy = (double)dy_f;
  r.fx = (double)(tmp_f * dx_f);
  r.fy = (double)(tmp_f * dy_f);
  r.u = (double)((4.0f * epsilon_f) * fmaf(sr6_f, sr6_f, -sr6_f));
  return r;
}

int or_ref_thread_values(const or_lj_t* lj, int64_t n, const double* pos, const double* vel,
                         const int32_t* type, double Lx, double Ly, int32_t periodic_y,
                         int32_t mode, int32_t ws1_halo, int32_t what, double eps_lambda,
                         double* out, int32_t nthreads) {
  if (!lj || n < 0 || !out || what < OR_SUM_U || what > OR_SUM_DUDL) return 1;
  if ((what == OR_SUM_P || what == OR_SUM_K) && !vel) return 1;
  set_threads(nthreads);
  int64_t* halo = NULL;
  int64_t nh = 0;
  if (ws1_halo && what != OR_SUM_K) {
    halo = (int64_t*)malloc(sizeof(int64_t) * (size_t)(2 * n + 1));
    if (!halo) return 2;
    nh = build_ws1_halo(lj, n, pos, Lx, halo);
  }
  double vc[3];
  for (int c = 0; c < 3; ++c) vc[c] = shift_of(lj, c);
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < n; ++i) {
    const int ti = type[i];
    const double m = type_mass(lj, ti);
    double acc = 0.0;
    if (what == OR_SUM_K) {
      const double vx = vel[2 * i], vy = vel[2 * i + 1];
      out[i] = (0.5 * m) * fma(vx, vx, vy * vy);
      continue;
    }
    if (what == OR_SUM_P) {
      const double vx = vel[2 * i], vy = vel[2 * i + 1];
      acc = m * fma(vx, vx, vy * vy);
    }
    const double xi = pos[2 * i], yi = pos[2 * i + 1];
    for (int64_t q = 0; q < n + nh; ++q) {
      if (q == i) continue;
      const int64_t j = q < n ? q : halo[q - n];
      const ref_pair_t r = ref_pair_terms(lj, mode, xi, yi, ti, pos[2 * j], pos[2 * j + 1],
                                          type[j], Lx, Ly, periodic_y);
      if (!r.in) continue;
      if (what == OR_SUM_U) {
        acc = fma(0.5, r.u - vc[r.c], acc);
      } else if (what == OR_SUM_P) {
        acc = fma(0.5, fma(r.dx, r.fx, r.dy * r.fy), acc);
      } else {
        const double pv = -eps_lambda * fma(r.fx, r.dx, -(r.fy * r.dy));
        acc = fma(0.5, pv, acc);
      }
    }
    out[i] = acc;
  }
  free(halo);
  return 0;
}

double or_ref_block_partials(int64_t n, const double* v, int32_t threads, double* partials) {
  if (threads <= 0) threads = 256;
  double* sh = (double*)malloc(sizeof(double) * (size_t)threads);
  if (!sh) return NAN;
  const int64_t nb = (n + threads - 1) / threads;
  double total = 0.0;
  for (int64_t b = 0; b < nb; ++b) {
    for (int32_t t = 0; t < threads; ++t) {
      const int64_t idx = b * threads + t;
      sh[t] = idx < n ? v[idx] : 0.0;
    }
    for (int32_t s = threads / 2; s > 0; s >>= 1)
      for (int32_t t = 0; t < s; ++t) sh[t] += sh[t + s];
    if (partials) partials[b] = sh[0];
    total += sh[0];
  }
  free(sh);
  return total;
}

/* ---- project binning ----------------------------------------------------- */
void or_cell_grid(double Lx, double Ly, double cell_min, int32_t* ncx, int32_t* ncy) {
  double fx = floor(Lx / cell_min);
  double fy = floor(Ly / cell_min);
  int32_t cx = (fx >= 1.0 && fx < 2147483647.0) ? (int32_t)fx : 1;
  int32_t cy = (fy >= 1.0 && fy < 2147483647.0) ? (int32_t)fy : 1;
  if (!(fx >= 1.0)) cx = 1;
  if (!(fy >= 1.0)) cy = 1;
  *ncx = cx;
  *ncy = cy;
}

static inline int32_t bin_axis(double v, int32_t nc) {
  /* v = coordinate * (nc / L); NaN and negatives -> 0, >= nc -> nc-1 */
  if (v >= 0.0 && v < (double)nc) return (int32_t)v;
  if (v >= (double)nc) return nc - 1;
  return 0;
}

void or_cell_bin(int64_t n, const double* pos, double Lx, double Ly, int32_t ncx, int32_t ncy,
                 int32_t* cell) {
  const double inv_wx = (double)ncx / Lx;
  const double inv_wy = (double)ncy / Ly;
  for (int64_t i = 0; i < n; ++i) {
    const int32_t cx = bin_axis(pos[2 * i] * inv_wx, ncx);
    const int32_t cy = bin_axis(pos[2 * i + 1] * inv_wy, ncy);
    cell[i] = cy * ncx + cx;
  }
}

/* Stable counting sort of particle indices by cell. cell_start has
 * ncells+1 entries. */
void or_cell_sort(int64_t n, const int32_t* cell, int32_t ncells, int32_t* perm,
                  int32_t* cell_start) {
  int32_t* cnt = (int32_t*)calloc((size_t)ncells + 1, sizeof(int32_t));
  for (int64_t i = 0; i < n; ++i) cnt[cell[i]]++;
  int32_t run = 0;
  for (int32_t c = 0; c < ncells; ++c) {
    const int32_t k = cnt[c];
    cell_start[c] = run;
    cnt[c] = run;
    run += k;
  }
  cell_start[ncells] = run;
  for (int64_t i = 0; i < n; ++i) perm[cnt[cell[i]]++] = (int32_t)i;
  free(cnt);
}

/* Cell-list force evaluation (cell width >= rc_max): the same pair set as the
 * all-pairs loop for rc < L/2, summed in cell order. */
int or_forces_cells(const or_lj_t* lj, int64_t n, const double* pos, const int32_t* type,
                    double Lx, double Ly, int32_t periodic_y, int32_t mode, double* acc,
                    double* U, double* W, int32_t nthreads) {
  double smax = lj->sigma[0];
  if (lj->sigma[1] > smax) smax = lj->sigma[1];
  if (lj->sigma[2] > smax) smax = lj->sigma[2];
  const double rcmax = lj->cutoff * smax;
  int32_t ncx, ncy;
  or_cell_grid(Lx, Ly, rcmax, &ncx, &ncy);
  if (ncx < 3 || (periodic_y && ncy < 3))
    return or_forces_allpairs(lj, n, pos, type, Lx, Ly, periodic_y, mode, 0, acc, U, W, nthreads);
  set_threads(nthreads);
  const int32_t ncells = ncx * ncy;
  int32_t* cell = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
  int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
  int32_t* start = (int32_t*)malloc(sizeof(int32_t) * (size_t)(ncells + 1));
  double* ui = (double*)malloc(sizeof(double) * (size_t)(n + 1));
  double* wi = (double*)malloc(sizeof(double) * (size_t)(n + 1));
  if (!cell || !perm || !start || !ui || !wi) {
    free(cell);
    free(perm);
    free(start);
    free(ui);
    free(wi);
    return 2;
  }
  or_cell_bin(n, pos, Lx, Ly, ncx, ncy, cell);
  or_cell_sort(n, cell, ncells, perm, start);
  const float Lx_f = (float)Lx, Ly_f = (float)Ly;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    pair_acc_t a = {0.0, 0.0, 0.0, 0.0};
    const double xi = pos[2 * i], yi = pos[2 * i + 1];
    const int ti = type[i];
    const int32_t cx = cell[i] % ncx, cy = cell[i] / ncx;
    for (int dyc = -1; dyc <= 1; ++dyc) {
      int32_t yy = cy + dyc;
      if (periodic_y) {
        if (yy < 0) yy += ncy;
        if (yy >= ncy) yy -= ncy;
      } else if (yy < 0 || yy >= ncy) {
        continue;
      }
      for (int dxc = -1; dxc <= 1; ++dxc) {
        int32_t xx = cx + dxc;
        if (xx < 0) xx += ncx;
        if (xx >= ncx) xx -= ncx;
        const int32_t c = yy * ncx + xx;
        for (int32_t k = start[c]; k < start[c + 1]; ++k) {
          const int32_t j = perm[k];
          if (j == i) continue;
          do_pair(lj, mode, xi, yi, ti, pos[2 * j], pos[2 * j + 1], type[j], Lx, Ly, Lx_f, Ly_f,
                  periodic_y, &a);
        }
      }
    }
    const double m = type_mass(lj, ti);
    if (acc) {
      acc[2 * i] = a.fx / m;
      acc[2 * i + 1] = a.fy / m;
    }
    ui[i] = a.u;
    wi[i] = a.w;
  }
  double su = 0.0, sw = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    su += ui[i];
    sw += wi[i];
  }
  if (U) *U = su;
  if (W) *W = sw;
  free(cell);
  free(perm);
  free(start);
  free(ui);
  free(wi);
  return 0;
}

int or_forces_rows(const or_lj_t* lj, int64_t n, const double* pos, const int32_t* type,
                   double Lx, double Ly, int32_t periodic_y, int32_t mode, int64_t row0,
                   int64_t nrows, double* acc_rows, int32_t nthreads) {
  if (row0 < 0 || nrows < 0 || row0 + nrows > n) return 1;
  set_threads(nthreads);
  const float Lx_f = (float)Lx, Ly_f = (float)Ly;
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t r = 0; r < nrows; ++r) {
    const int64_t i = row0 + r;
    pair_acc_t a = {0.0, 0.0, 0.0, 0.0};
    const double xi = pos[2 * i], yi = pos[2 * i + 1];
    const int ti = type[i];
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      do_pair(lj, mode, xi, yi, ti, pos[2 * j], pos[2 * j + 1], type[j], Lx, Ly, Lx_f, Ly_f,
              periodic_y, &a);
    }
    const double m = type_mass(lj, ti);
    acc_rows[2 * r] = a.fx / m;
    acc_rows[2 * r + 1] = a.fy / m;
  }
  return 0;
}

int64_t or_count_pairs_cells(const or_lj_t* lj, int64_t n, const double* pos,
                             const int32_t* type, double Lx, double Ly, int32_t nthreads) {
  double smax = lj->sigma[0];
  if (lj->sigma[1] > smax) smax = lj->sigma[1];
  if (lj->sigma[2] > smax) smax = lj->sigma[2];
  int32_t ncx, ncy;
  or_cell_grid(Lx, Ly, lj->cutoff * smax, &ncx, &ncy);
  if (ncx < 3 || ncy < 3) return or_count_pairs(lj, n, pos, type, Lx, Ly, 1, nthreads);
  set_threads(nthreads);
  const int32_t ncells = ncx * ncy;
  int32_t* cell = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
  int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
  int32_t* start = (int32_t*)malloc(sizeof(int32_t) * (size_t)(ncells + 1));
  if (!cell || !perm || !start) {
    free(cell);
    free(perm);
    free(start);
    return -1;
  }
  or_cell_bin(n, pos, Lx, Ly, ncx, ncy, cell);
  or_cell_sort(n, cell, ncells, perm, start);
  int64_t total = 0;
#pragma omp parallel for reduction(+ : total) schedule(dynamic, 256)
  for (int64_t i = 0; i < n; ++i) {
    const int32_t cx = cell[i] % ncx, cy = cell[i] / ncx;
    for (int dyc = -1; dyc <= 1; ++dyc) {
      const int32_t yy = (cy + dyc + ncy) % ncy;
      for (int dxc = -1; dxc <= 1; ++dxc) {
        const int32_t xx = (cx + dxc + ncx) % ncx;
        const int32_t c = yy * ncx + xx;
        for (int32_t k = start[c]; k < start[c + 1]; ++k) {
          const int32_t j = perm[k];
          if (j == i) continue;
          double dx = pos[2 * i] - pos[2 * j], dy = pos[2 * i + 1] - pos[2 * j + 1];
          dx = dx - Lx * round(dx / Lx);
          dy = dy - Ly * round(dy / Ly);
          const double rc = lj->cutoff * lj->sigma[pair_class(type[i], type[j])];
          const double r2 = dx * dx + dy * dy;
          if (r2 > 0.0 && r2 < rc * rc) total += 1;
        }
      }
    }
  }
  free(cell);
  free(perm);
  free(start);
  return total;
}

int64_t or_count_pairs(const or_lj_t* lj, int64_t n, const double* pos, const int32_t* type,
                       double Lx, double Ly, int32_t periodic_y, int32_t nthreads) {
  set_threads(nthreads);
  int64_t total = 0;
#pragma omp parallel for reduction(+ : total) schedule(dynamic, 16)
  for (int64_t i = 0; i < n; ++i) {
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      double dx = pos[2 * i] - pos[2 * j];
      double dy = pos[2 * i + 1] - pos[2 * j + 1];
      dx = dx - Lx * round(dx / Lx);
      if (periodic_y) dy = dy - Ly * round(dy / Ly);
      const int c = pair_class(type[i], type[j]);
      const double rc = lj->cutoff * lj->sigma[c];
      const double r2 = dx * dx + dy * dy;
      if (r2 > 0.0 && r2 < rc * rc) total += 1;
    }
  }
  return total;
}

/* cal_partial_U_lambda_kernel (src/md_cuda_common.cu:266-377) and its host
 * sum (src/md_env.cu:2362-2406), all pairs with the nearest image (no halo
 * duplication): sum over ordered pairs of 1/2 * (-eps_lambda) * (Fx dx - Fy dy).
 * OR_REF_MIXED: FP32 pair force, products and sum in FP64 as the kernel does;
 * OR_FP64: every operation in double. *scale receives the same sum with
 * |Fx dx| + |Fy dy| (a magnitude for tolerances). */
int or_partial_U_lambda(const or_lj_t* lj, int64_t n, const double* pos, const int32_t* type,
                        double Lx, double Ly, int32_t periodic_y, int32_t mode,
                        double epsilon_lambda, double* out, double* scale, int32_t nthreads) {
  if (!lj || !pos || !type || !out || n < 0) return 1;
  set_threads(nthreads);
  const float Lx_f = (float)Lx, Ly_f = (float)Ly;
  double total = 0.0, mag = 0.0;
#pragma omp parallel for reduction(+ : total, mag) schedule(dynamic, 16)
  for (int64_t i = 0; i < n; ++i) {
    double ui = 0.0, mi = 0.0;
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const int c = pair_class(type[i], type[j]);
      double fxdx, fydy;
      if (mode == OR_FP64) {
        double dx = pos[2 * i] - pos[2 * j];
        double dy = pos[2 * i + 1] - pos[2 * j + 1];
        dx = dx - Lx * round(dx / Lx);
        if (periodic_y) dy = dy - Ly * round(dy / Ly);
        const double sig = lj->sigma[c], rc = lj->cutoff * sig;
        const double r2 = dx * dx + dy * dy;
        if (!(r2 > 0.0 && r2 < rc * rc)) continue;
        const double r2i = 1.0 / r2;
        const double sr2 = sig * sig * r2i;
        const double sr6 = sr2 * sr2 * sr2;
        const double sr12 = sr6 * sr6;
        const double tmp = 24.0 * lj->epsilon[c] * (2.0 * sr12 - sr6) * r2i;
        fxdx = (tmp * dx) * dx;
        fydy = (tmp * dy) * dy;
      } else {
        float dx_f = (float)(pos[2 * i] - pos[2 * j]);
        float dy_f = (float)(pos[2 * i + 1] - pos[2 * j + 1]);
        dx_f = fmaf(-Lx_f, roundf(dx_f / Lx_f), dx_f);
        if (periodic_y) dy_f = fmaf(-Ly_f, roundf(dy_f / Ly_f), dy_f);
        const float sigma_f = (float)lj->sigma[c];
        const float rc_f = (float)lj->cutoff * sigma_f;
        const float dr_sq_f = fmaf(dx_f, dx_f, dy_f * dy_f);
        if (!(dr_sq_f > 0.0f && dr_sq_f < rc_f * rc_f)) continue;
        const float r2_inv_f = 1.0f / dr_sq_f;
        const float sr2_f = (sigma_f * sigma_f) * r2_inv_f;
        const float sr6_f = sr2_f * sr2_f * sr2_f;
        const float sr12_f = sr6_f * sr6_f;
        const float tmp_f = (24.0f * (float)lj->epsilon[c]) * fmaf(2.0f, sr12_f, -sr6_f) * r2_inv_f;
        fxdx = (double)(tmp_f * dx_f) * (double)dx_f;
        fydy = (double)(tmp_f * dy_f) * (double)dy_f;
      }
      ui += 0.5 * (-epsilon_lambda * (fxdx - fydy));
      mi += 0.5 * fabs(epsilon_lambda) * (fabs(fxdx) + fabs(fydy));
    }
    total += ui;
    mag += mi;
  }
  *out = total;
  if (scale) *scale = mag;
  return 0;
}

/* get_N_profile (src/md_env.cu:3920-3985, kernel src/md_cuda_common.cu:827-871)
 * at world size 1 (x_min = 0, x_max = Lx): counts of type 0 in out[0..nb) and
 * of other types in out[nb..2nb), bin = int(x / Lx * nb) clamped, particles
 * with 0 <= x <= Lx. */
int or_n_profile(int64_t n, const double* pos, const int32_t* type, double Lx, int32_t nb,
                 int32_t* out) {
  if (nb <= 0 || !out) return 1;
  memset(out, 0, sizeof(int32_t) * 2 * (size_t)nb);
  for (int64_t i = 0; i < n; ++i) {
    const double x = pos[2 * i];
    if (!(x >= 0.0 && x <= Lx)) continue;
    int b = (int)(x / Lx * nb);
    if (b < 0) b = 0;
    if (b >= nb) b = nb - 1;
    out[(type[i] == 0 ? 0 : nb) + b] += 1;
  }
  return 0;
}

static int profile_bin(double y, double Ly, int32_t nb, int periodic_y) {
  double yy = periodic_y ? or_pbc_wrap(y, Ly) : y;
  if (!periodic_y) {
    if (yy < 0.0)
      yy = 0.0;
    else if (yy >= Ly && Ly > 0.0)
      yy = Ly * (1.0 - 1e-12);
  }
  const double t = (Ly > 0.0) ? (yy / Ly) : 0.0;
  int b = (int)(t * (double)nb);
  if (b < 0) b = 0;
  if (b >= nb) b = nb - 1;
  return b;
}

/* get_pressure_profile (src/md_env.cu:3821-3918, kernel
 * src/md_cuda_common.cu:873-1030), all pairs with the nearest image:
 * out[0..nb) = P_xx, [nb..2nb) = P_yy, [2nb..3nb) = P_xy per y bin; kinetic
 * m v_a v_b at the bin of y_i, pair 1/2 r_a F_b at the bin of the midpoint
 * y_i - dy/2, each divided by the bin area Lx * Ly / nb. FP64 or the
 * reference's mixed arithmetic. */
int or_pressure_profile(const or_lj_t* lj, int64_t n, const double* pos, const double* vel,
                        const int32_t* type, double Lx, double Ly, int32_t periodic_y,
                        int32_t mode, int32_t nb, double* out) {
  if (nb <= 0 || !out) return 1;
  memset(out, 0, sizeof(double) * 3 * (size_t)nb);
  const float Lx_f = (float)Lx, Ly_f = (float)Ly;
  for (int64_t i = 0; i < n; ++i) {
    const double m = type_mass(lj, type[i]);
    const double vx = vel[2 * i], vy = vel[2 * i + 1];
    const int bk = profile_bin(pos[2 * i + 1], Ly, nb, periodic_y);
    out[bk] += m * vx * vx;
    out[nb + bk] += m * vy * vy;
    out[2 * nb + bk] += m * vx * vy;
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const int c = pair_class(type[i], type[j]);
      double dx, dy, Fx, Fy;
      if (mode == OR_FP64) {
        dx = pos[2 * i] - pos[2 * j];
        dy = pos[2 * i + 1] - pos[2 * j + 1];
        dx = dx - Lx * round(dx / Lx);
        if (periodic_y) dy = dy - Ly * round(dy / Ly);
        const double sig = lj->sigma[c], rc = lj->cutoff * sig;
        const double r2 = dx * dx + dy * dy;
        if (!(r2 > 0.0 && r2 < rc * rc)) continue;
        const double r2i = 1.0 / r2;
        const double sr2 = sig * sig * r2i;
        const double sr6 = sr2 * sr2 * sr2;
        const double sr12 = sr6 * sr6;
        const double tmp = 24.0 * lj->epsilon[c] * (2.0 * sr12 - sr6) * r2i;
        Fx = tmp * dx;
        Fy = tmp * dy;
      } else {
        float dx_f = (float)(pos[2 * i] - pos[2 * j]);
        float dy_f = (float)(pos[2 * i + 1] - pos[2 * j + 1]);
        dx_f = fmaf(-Lx_f, roundf(dx_f / Lx_f), dx_f);
        if (periodic_y) dy_f = fmaf(-Ly_f, roundf(dy_f / Ly_f), dy_f);
        const float sigma_f = (float)lj->sigma[c];
        const float rc_f = (float)lj->cutoff * sigma_f;
        const float dr_sq_f = fmaf(dx_f, dx_f, dy_f * dy_f);
        if (!(dr_sq_f > 0.0f && dr_sq_f < rc_f * rc_f)) continue;
        const float r2_inv_f = 1.0f / dr_sq_f;
        const float sr2_f = (sigma_f * sigma_f) * r2_inv_f;
        const float sr6_f = sr2_f * sr2_f * sr2_f;
        const float sr12_f = sr6_f * sr6_f;
        const float tmp_f = (24.0f * (float)lj->epsilon[c]) * fmaf(2.0f, sr12_f, -sr6_f) * r2_inv_f;
        dx = (double)dx_f;
        dy = (double)dy_f;
        Fx = (double)(tmp_f * dx_f);
        Fy = (double)(tmp_f * dy_f);
      }
      const int bp = profile_bin(pos[2 * i + 1] - 0.5 * dy, Ly, nb, periodic_y);
      out[bp] += 0.5 * dx * Fx;
      out[nb + bp] += 0.5 * dy * Fy;
      out[2 * nb + bp] += 0.5 * dx * Fy;
    }
  }
  const double vol = Lx * (Ly / (double)nb);
  if (vol > 0.0)
    for (int k = 0; k < 3 * nb; ++k) out[k] /= vol;
  return 0;
}

/* ---- engine --------------------------------------------------------------- */
static void sim_forces(or_sim_t* s, int32_t periodic_y, double* acc, double* U, double* W) {
  if (s->use_cells && !s->ws1_halo)
    or_forces_cells(&s->lj, s->n, s->pos, s->type, s->Lx, s->Ly, periodic_y, s->mode, acc, U, W,
                    s->nthreads);
  else
    or_forces_allpairs(&s->lj, s->n, s->pos, s->type, s->Lx, s->Ly, periodic_y, s->mode,
                       s->ws1_halo, acc, U, W, s->nthreads);
}

/* MDSimulation::cal_forces (src/md_env.cu:1511-1542): periodic_y = 1. */
void or_sim_cal_forces(or_sim_t* s, int32_t periodic_y) { sim_forces(s, periodic_y, s->acc, NULL, NULL); }

void or_sim_setup(or_sim_t* s) {
  s->Lx0 = s->Lx;
  s->Ly0 = s->Ly;
  s->t = 0.0;
  s->xi = 0.0;
  s->nph_area_momentum = 0.0;
  s->nph_aspect_ratio = 1.0;
  s->nph_state_initialized = 0;
  s->piston_velocity = 0.0;
  s->piston_force = 0.0;
  s->piston_velocity_initialized = 0;
  s->piston_mode_active = 0;
  s->last_instant_pressure = 0.0;
  s->error = 0;
  or_sim_cal_forces(s, 1);
}

/* Sum of the reference kernel `what` over the system through its block
 * trees (ref_threads per block) and the host's block-order loop. */
static double ref_tree_total(const or_sim_t* s, int what, int32_t periodic_y) {
  double* v = (double*)malloc(sizeof(double) * (size_t)(s->n + 1));
  if (!v) return NAN;
  or_ref_thread_values(&s->lj, s->n, s->pos, s->vel, s->type, s->Lx, s->Ly, periodic_y, s->mode,
                       s->ws1_halo, what, 0.0, v, s->nthreads);
  const double tot = or_ref_block_partials(s->n, v, s->ref_threads, NULL);
  free(v);
  return tot;
}

/* cal_local_K_kernel (src/md_cuda_common.cu:554-589): k = 1/2 m |v|^2. */
double or_total_K(const or_sim_t* s) {
  if (s->ref_threads > 0) return ref_tree_total(s, OR_SUM_K, 1);
  double K = 0.0;
  for (int64_t i = 0; i < s->n; ++i) {
    const double vx = s->vel[2 * i], vy = s->vel[2 * i + 1];
    const double m = type_mass(&s->lj, s->type[i]);
    K += (0.5 * m) * fma(vx, vx, vy * vy);
  }
  return K;
}

/* cal_total_scalar_pressure (src/md_env.cu:2205-2252):
 * (sum m|v|^2 + sum_i 1/2 sum_j r.F) / (2 A). */
double or_scalar_pressure(or_sim_t* s, int32_t periodic_y) {
  const double area = s->Lx * s->Ly;
  if (s->ref_threads > 0) {
    const double sum = ref_tree_total(s, OR_SUM_P, periodic_y);
    return (area > 0.0) ? sum / (2.0 * area) : 0.0;
  }
  double kin = 0.0;
  for (int64_t i = 0; i < s->n; ++i) {
    const double vx = s->vel[2 * i], vy = s->vel[2 * i + 1];
    kin += type_mass(&s->lj, s->type[i]) * fma(vx, vx, vy * vy);
  }
  double W = 0.0;
  sim_forces(s, periodic_y, NULL, NULL, &W);
  if (!(area > 0.0)) return 0.0;
  return (kin + W) / (2.0 * area);
}

/* piston_wall_kernel (src/md_cuda_common.cu:498-552) with the host sums of
 * evaluate_piston_wall_observables (src/md_env.cu:2148-2203). */
static void piston_walls(or_sim_t* s, int update_acc, double* upper, double* energy) {
  double up = 0.0, en = 0.0;
  const double k = s->k_piston;
  double* tv = NULL;
  if (s->ref_threads > 0 && s->n > 0 && k > 0.0)
    tv = (double*)malloc(sizeof(double) * (size_t)(2 * s->n));
  if (s->n > 0 && k > 0.0) {
    for (int64_t i = 0; i < s->n; ++i) {
      const double y = s->pos[2 * i + 1];
      double wf = 0.0, upi = 0.0, eni = 0.0;
      if (y > s->Ly) {
        const double ov = y - s->Ly;
        wf = fma(-k, ov, wf);
        upi = fma(k, ov, upi);
        eni = fma((0.5 * k) * ov, ov, eni);
      }
      if (y < 0.0) {
        const double ov = -y;
        wf = fma(k, ov, wf);
        eni = fma((0.5 * k) * ov, ov, eni);
      }
      if (update_acc && wf != 0.0) {
        const double m = type_mass(&s->lj, s->type[i]);
        s->acc[2 * i + 1] = s->acc[2 * i + 1] + wf / m;
      }
      up += upi;
      en += eni;
      if (tv) {
        tv[i] = upi;
        tv[s->n + i] = eni;
      }
    }
  }
  if (tv) {
    up = or_ref_block_partials(s->n, tv, s->ref_threads, NULL);
    en = or_ref_block_partials(s->n, tv + s->n, s->ref_threads, NULL);
    free(tv);
  }
  *upper = up;
  *energy = en;
}

void or_sim_piston_walls(or_sim_t* s, int32_t update_acc, double* upper, double* energy) {
  piston_walls(s, update_acc, upper, energy);
}

/* cal_total_U (src/md_env.cu:2347-2360). */
double or_total_U(or_sim_t* s) {
  const int periodic_y = s->piston_mode_active ? 0 : 1;
  double U = 0.0;
  if (s->ref_threads > 0)
    U = ref_tree_total(s, OR_SUM_U, periodic_y);
  else
    sim_forces(s, periodic_y, NULL, &U, NULL);
  if (!s->piston_mode_active) return U;
  double up, en;
  piston_walls(s, 0, &up, &en);
  return U + en;
}

/* cal_instant_pressure (src/md_env.cu:2254-2266). */
double or_instant_pressure(or_sim_t* s) {
  if (s->piston_mode_active) {
    double up, en;
    piston_walls(s, 0, &up, &en);
    s->piston_force = up;
    s->last_instant_pressure = (s->Lx > 0.0) ? (s->piston_force / s->Lx) : 0.0;
    return s->last_instant_pressure;
  }
  s->last_instant_pressure = or_scalar_pressure(s, 1);
  return s->last_instant_pressure;
}

/* step_single_NVE (src/md_env.cu:1576-1637) with step_half_vv_kernel
 * (src/md_cuda_common.cu:381-394) and step_2nd_half_vv_kernel (:443-452):
 *   v = fma(dt/2, a, v); x = wrap(fma(dt, v, x)); a = F/m; v = fma(dt/2, a, v). */
void or_step_nve(or_sim_t* s) {
  s->piston_mode_active = 0;
  const double dt = s->dt, h = 0.5 * dt;
  for (int64_t i = 0; i < s->n; ++i) {
    for (int d = 0; d < 2; ++d) {
      const int64_t k = 2 * i + d;
      s->vel[k] = fma(h, s->acc[k], s->vel[k]);
      s->pos[k] = fma(dt, s->vel[k], s->pos[k]);
    }
    s->pos[2 * i] = or_pbc_wrap(s->pos[2 * i], s->Lx);
    s->pos[2 * i + 1] = or_pbc_wrap(s->pos[2 * i + 1], s->Ly);
  }
  or_sim_cal_forces(s, 1);
  for (int64_t k = 0; k < 2 * s->n; ++k) s->vel[k] = fma(h, s->acc[k], s->vel[k]);
  s->t += dt;
}

/* xi += 0.5 dt (2K - g T0) / Q with g = 2N - 2 (src/md_env.cu:1668-1673,
 * 1709-1713), host arithmetic without contraction. */
static double nh_xi_update(const or_sim_t* s, double xi, double K) {
  const double g = 2.0 * (double)s->n_global - 2.0;
  const double t1 = 0.5 * s->dt;
  const double t2 = 2.0 * K;
  const double t3 = g * s->T_target;
  const double t4 = t2 - t3;
  const double t5 = t1 * t4;
  const double t6 = t5 / s->Q;
  return xi + t6;
}

/* step_single_nose_hoover (src/md_env.cu:1639-1728) with
 * step_half_vv_nh_kernel (src/md_cuda_common.cu:454-478) and
 * step_2nd_half_vv_nh_kernel (:480-496): v = fma(dt/2, fma(-xi, v, a), v). */
void or_step_nose_hoover(or_sim_t* s) {
  s->piston_mode_active = 0;
  const double dt = s->dt, h = 0.5 * dt;
  double K = or_total_K(s);
  s->xi = nh_xi_update(s, s->xi, K);
  const double xi1 = s->xi;
  for (int64_t i = 0; i < s->n; ++i) {
    for (int d = 0; d < 2; ++d) {
      const int64_t k = 2 * i + d;
      const double v = s->vel[k];
      s->vel[k] = fma(h, fma(-xi1, v, s->acc[k]), v);
      s->pos[k] = fma(dt, s->vel[k], s->pos[k]);
    }
    s->pos[2 * i] = or_pbc_wrap(s->pos[2 * i], s->Lx);
    s->pos[2 * i + 1] = or_pbc_wrap(s->pos[2 * i + 1], s->Ly);
  }
  or_sim_cal_forces(s, 1);
  K = or_total_K(s);
  s->xi = nh_xi_update(s, s->xi, K);
  const double xi2 = s->xi;
  for (int64_t k = 0; k < 2 * s->n; ++k) {
    const double v = s->vel[k];
    s->vel[k] = fma(h, fma(-xi2, v, s->acc[k]), v);
  }
  s->t += dt;
}

/* step_single_NPH (src/md_env.cu:1795-1918; init :1757-1778; kernels
 * src/md_cuda_common.cu:411-440). */
void or_step_nph(or_sim_t* s, double p_ext) {
  s->piston_mode_active = 0;
  const double bm = s->barostat_mass > 1e-12 ? s->barostat_mass : 1e-12;
  if (!s->nph_state_initialized) {
    if (!(s->Lx > 0.0) || !(s->Ly > 0.0)) {
      s->error = 1;
      return;
    }
    s->nph_aspect_ratio = s->Lx / s->Ly;
    s->nph_area_momentum = bm * s->area_rate_init;
    s->nph_state_initialized = 1;
  }
  const double dt = s->dt, h = 0.5 * dt, W = bm;
  const double Lx_old = s->Lx, Ly_old = s->Ly;
  const double area_old = Lx_old * Ly_old;
  if (area_old <= 0.0) {
    s->error = 1;
    return;
  }
  const double p_old = or_scalar_pressure(s, 1);
  for (int64_t k = 0; k < 2 * s->n; ++k) s->vel[k] = fma(h, s->acc[k], s->vel[k]);
  s->nph_area_momentum = s->nph_area_momentum + h * (p_old - p_ext);
  double area_new = area_old + dt * (s->nph_area_momentum / W);
  if (!(area_new > 0.0) || !isfinite(area_new)) {
    s->error = 1;
    return;
  }
  if (!(s->nph_aspect_ratio > 0.0) || !isfinite(s->nph_aspect_ratio))
    s->nph_aspect_ratio = Lx_old / Ly_old;
  const double g = s->nph_aspect_ratio;
  double Ly_new = sqrt(area_new / g);
  double Lx_new = g * Ly_new;
  const double fl = (s->hmin_ratio * s->Ly0) > 1e-12 ? s->hmin_ratio * s->Ly0 : 1e-12;
  const double ce = (s->hmax_ratio * s->Ly0) > fl ? s->hmax_ratio * s->Ly0 : fl;
  int clamped = 0;
  if (Ly_new < fl) {
    Ly_new = fl;
    Lx_new = g * Ly_new;
    area_new = Lx_new * Ly_new;
    clamped = 1;
  } else if (Ly_new > ce) {
    Ly_new = ce;
    Lx_new = g * Ly_new;
    area_new = Lx_new * Ly_new;
    clamped = 1;
  }
  const double lin = sqrt(area_new / area_old);
  const double vs = 1.0 / lin;
  for (int64_t i = 0; i < s->n; ++i) {
    for (int d = 0; d < 2; ++d) {
      const int64_t k = 2 * i + d;
      s->vel[k] = s->vel[k] * vs;
      s->pos[k] = fma(lin, s->pos[k], dt * s->vel[k]);
    }
    s->pos[2 * i] = or_pbc_wrap(s->pos[2 * i], Lx_new);
    s->pos[2 * i + 1] = or_pbc_wrap(s->pos[2 * i + 1], Ly_new);
  }
  if (Lx_new <= 0.0 || Ly_new <= 0.0) {
    s->error = 1;
    return;
  }
  s->Lx = Lx_new;
  s->Ly = Ly_new;
  or_sim_cal_forces(s, 1);
  const double p_new = or_scalar_pressure(s, 1);
  for (int64_t k = 0; k < 2 * s->n; ++k) s->vel[k] = fma(h, s->acc[k], s->vel[k]);
  s->nph_area_momentum = s->nph_area_momentum + h * (p_new - p_ext);
  if (clamped) {
    if (s->Ly <= fl && s->nph_area_momentum < 0.0) s->nph_area_momentum = 0.0;
    if (s->Ly >= ce && s->nph_area_momentum > 0.0) s->nph_area_momentum = 0.0;
  }
  s->last_instant_pressure = p_new;
  s->t += dt;
}

/* cal_forces_piston (src/md_env.cu:1544-1574): LJ with periodic_y = 0, then
 * the soft walls added to acc.y. */
static void cal_forces_piston(or_sim_t* s) {
  sim_forces(s, 0, s->acc, NULL, NULL);
  double up, en;
  piston_walls(s, 1, &up, &en);
  s->piston_force = up;
}

/* step_single_NPH_piston (src/md_env.cu:1920-2023; init :1780-1793;
 * step_half_vv_piston_kernel src/md_cuda_common.cu:396-409). */
void or_step_nph_piston(or_sim_t* s, double p_ext) {
  if (!s->piston_velocity_initialized) {
    s->piston_velocity = 0.0;
    s->piston_velocity_initialized = 1;
  }
  if (!s->piston_mode_active) {
    s->piston_mode_active = 1;
    cal_forces_piston(s);
    s->last_instant_pressure = (s->Lx > 0.0) ? (s->piston_force / s->Lx) : 0.0;
  }
  const double dt = s->dt, h = 0.5 * dt;
  const double W = s->barostat_mass > 1e-12 ? s->barostat_mass : 1e-12;
  const double Lx = s->Lx, Ly_old = s->Ly;
  if (Lx <= 0.0 || Ly_old <= 0.0) {
    s->error = 1;
    return;
  }
  const double a_old = (s->piston_force - p_ext * Lx) / W;
  for (int64_t i = 0; i < s->n; ++i) {
    for (int d = 0; d < 2; ++d) {
      const int64_t k = 2 * i + d;
      s->vel[k] = fma(h, s->acc[k], s->vel[k]);
      s->pos[k] = fma(dt, s->vel[k], s->pos[k]);
    }
    s->pos[2 * i] = or_pbc_wrap(s->pos[2 * i], Lx);
  }
  s->piston_velocity = s->piston_velocity + h * a_old;
  double Ly_new = Ly_old + dt * s->piston_velocity;
  const double fl = (s->hmin_ratio * s->Ly0) > 1e-12 ? s->hmin_ratio * s->Ly0 : 1e-12;
  const double ce = (s->hmax_ratio * s->Ly0) > fl ? s->hmax_ratio * s->Ly0 : fl;
  int clamped = 0;
  if (Ly_new < fl) {
    Ly_new = fl;
    clamped = 1;
    if (s->piston_velocity < 0.0) s->piston_velocity = 0.0;
  } else if (Ly_new > ce) {
    Ly_new = ce;
    clamped = 1;
    if (s->piston_velocity > 0.0) s->piston_velocity = 0.0;
  }
  s->Ly = Ly_new;
  cal_forces_piston(s);
  for (int64_t k = 0; k < 2 * s->n; ++k) s->vel[k] = fma(h, s->acc[k], s->vel[k]);
  const double a_new = (s->piston_force - p_ext * Lx) / W;
  s->piston_velocity = s->piston_velocity + h * a_new;
  if (clamped) {
    if (s->Ly <= fl && s->piston_velocity < 0.0) s->piston_velocity = 0.0;
    if (s->Ly >= ce && s->piston_velocity > 0.0) s->piston_velocity = 0.0;
  }
  s->last_instant_pressure = s->piston_force / Lx;
  s->t += dt;
}

/* The reference's integrator kernels one at a time (src/md_cuda_common.cu:
 * 379-496), in the arithmetic its build performs (pinned against outputs of
 * the kernels themselves, tests/golden/ref_physics.*). */
int or_ref_integrator(int32_t which, int64_t n, double* pos, double* vel, const double* acc,
                      double dt, double xi, double lin, double vsc, double Lx, double Ly) {
  if (which < 0 || which > 6 || n < 0) return 1;
  const double h = 0.5 * dt;
  for (int64_t i = 0; i < n; ++i) {
    for (int d = 0; d < 2; ++d) {
      const int64_t k = 2 * i + d;
      double v = vel[k];
      switch (which) {
        case 0: /* step_half_vv_kernel :381-394 */
        case 6: /* step_half_vv_piston_kernel :396-409 */
          v = fma(h, acc[k], v);
          pos[k] = fma(dt, v, pos[k]);
          break;
        case 1: /* step_2nd_half_vv_kernel :443-452 */
        case 4: /* step_half_nph_velocity_kernel :411-420 */
          v = fma(h, acc[k], v);
          break;
        case 2: /* step_half_vv_nh_kernel :454-478 */
          v = fma(h, fma(-xi, v, acc[k]), v);
          pos[k] = fma(dt, v, pos[k]);
          break;
        case 3: /* step_2nd_half_vv_nh_kernel :480-496 */
          v = fma(h, fma(-xi, v, acc[k]), v);
          break;
        case 5: /* step_nph_scale_and_drift_kernel :422-440 */
          v = v * vsc;
          pos[k] = fma(lin, pos[k], dt * v);
          break;
      }
      vel[k] = v;
    }
    if (which == 0 || which == 2 || which == 5) {
      pos[2 * i] = or_pbc_wrap(pos[2 * i], Lx);
      pos[2 * i + 1] = or_pbc_wrap(pos[2 * i + 1], Ly);
    } else if (which == 6) {
      pos[2 * i] = or_pbc_wrap(pos[2 * i], Lx);
    }
  }
  return 0;
}

/* ---- FIRE ------------------------------------------------------------------ */
static double fire_potential(const or_lj_t* lj, int64_t n, const double* pos,
                             const int32_t* type, double Lx, double Ly, int32_t mode,
                             int32_t halo, int32_t use_cells, int32_t nthreads) {
  double U = 0.0;
  if (use_cells && !halo)
    or_forces_cells(lj, n, pos, type, Lx, Ly, 1, mode, NULL, &U, NULL, nthreads);
  else
    or_forces_allpairs(lj, n, pos, type, Lx, Ly, 1, mode, halo, NULL, &U, NULL, nthreads);
  return U;
}

/* EnergyMinimizer::minimize_frame (src/md_energy_minimizer.cu:122-272) with
 * velocity_kick / zero_velocity / fire_velocity_mix / drift kernels (:24-71)
 * and reduce_force_metrics (:442-475). */
int or_fire_minimize(const or_lj_t* lj, int64_t n, double* pos, double* vel, double* acc,
                     const int32_t* type, double Lx, double Ly, double force_tol,
                     int32_t max_steps, const or_fire_params_t* p, int32_t mode,
                     int32_t ws1_halo, int32_t use_cells, int32_t nthreads,
                     or_fire_result_t* res, int32_t* energy_steps, double* energy_trace,
                     int64_t trace_cap) {
  if (max_steps <= 0) return 1;
  /* initialize_from_frame (:386-419): wrap, zero v and a, no halos */
  for (int64_t i = 0; i < n; ++i) {
    pos[2 * i] = or_pbc_wrap(pos[2 * i], Lx);
    pos[2 * i + 1] = or_pbc_wrap(pos[2 * i + 1], Ly);
    vel[2 * i] = vel[2 * i + 1] = 0.0;
    acc[2 * i] = acc[2 * i + 1] = 0.0;
  }
  int32_t halo = 0;
  double dt = p->dt_init, alpha = p->alpha0;
  int32_t streak = 0;
  int64_t ns = 0;
#define RECORD(st, u)                          \
  do {                                         \
    if (ns < trace_cap) {                      \
      energy_steps[ns] = (st);                 \
      energy_trace[ns] = (u);                  \
    }                                          \
    ns++;                                      \
  } while (0)
  double last_u = fire_potential(lj, n, pos, type, Lx, Ly, mode, halo, use_cells, nthreads);
  RECORD(0, last_u);
  int converged = 0, steps = 0;
  double max_force = 0.0;
  for (int32_t step = 0; step < max_steps; ++step) {
    if (use_cells && !halo)
      or_forces_cells(lj, n, pos, type, Lx, Ly, 1, mode, acc, NULL, NULL, nthreads);
    else
      or_forces_allpairs(lj, n, pos, type, Lx, Ly, 1, mode, halo, acc, NULL, NULL, nthreads);
    for (int64_t k = 0; k < 2 * n; ++k) vel[k] = fma(dt, acc[k], vel[k]);
    double mf = 0.0, power = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      const double vx = vel[2 * i], vy = vel[2 * i + 1];
      const double fx = acc[2 * i], fy = acc[2 * i + 1];
      const double fm = sqrt(fma(fx, fx, fy * fy));
      if (fm > mf) mf = fm;
      power += fma(vx, fx, vy * fy);
    }
    max_force = mf;
    if (mf < force_tol) {
      converged = 1;
      steps = step;
      last_u = fire_potential(lj, n, pos, type, Lx, Ly, mode, halo, use_cells, nthreads);
      RECORD(step + 1, last_u);
      break;
    }
    if (power > 0.0) {
      streak += 1;
      if (streak > p->N_min) {
        const double d2 = dt * p->f_inc;
        dt = d2 < p->dt_max ? d2 : p->dt_max;
        const double a2 = alpha * 0.99;
        alpha = a2 > 0.0 ? a2 : 0.0;
      }
    } else {
      dt = dt * p->f_dec;
      streak = 0;
      alpha = p->alpha0;
      for (int64_t k = 0; k < 2 * n; ++k) vel[k] = 0.0;
    }
    for (int64_t i = 0; i < n; ++i) {
      const double vx = vel[2 * i], vy = vel[2 * i + 1];
      const double fx = acc[2 * i], fy = acc[2 * i + 1];
      const double vmag = sqrt(fma(vx, vx, vy * vy));
      const double fmag = sqrt(fma(fx, fx, fy * fy));
      if (vmag > 0.0 && fmag > 0.0) {
        const double scale = vmag / fmag;
        vel[2 * i] = fma(alpha * scale, fx, (1.0 - alpha) * vx);
        vel[2 * i + 1] = fma(alpha * scale, fy, (1.0 - alpha) * vy);
      }
    }
    for (int64_t i = 0; i < n; ++i) {
      pos[2 * i] = or_pbc_wrap(fma(dt, vel[2 * i], pos[2 * i]), Lx);
      pos[2 * i + 1] = or_pbc_wrap(fma(dt, vel[2 * i + 1], pos[2 * i + 1]), Ly);
    }
    halo = ws1_halo; /* exchange_particles: halos exist from here on */
    if ((step + 1) % 1000 == 0) {
      last_u = fire_potential(lj, n, pos, type, Lx, Ly, mode, halo, use_cells, nthreads);
      RECORD(step + 1, last_u);
    }
  }
  if (!converged) {
    steps = max_steps;
    const int32_t last_st = (ns > 0 && ns - 1 < trace_cap) ? energy_steps[ns - 1] : -1;
    if (ns == 0 || last_st != max_steps) {
      last_u = fire_potential(lj, n, pos, type, Lx, Ly, mode, halo, use_cells, nthreads);
      RECORD(max_steps, last_u);
    }
  }
#undef RECORD
  res->steps = steps;
  res->converged = converged;
  res->max_force = max_force;
  res->potential_energy = fire_potential(lj, n, pos, type, Lx, Ly, mode, halo, use_cells, nthreads);
  res->n_energy_samples = ns;
  return 0;
}
