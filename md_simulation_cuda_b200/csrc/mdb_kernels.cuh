// Device code of libmdb200: sm_100a kernels for the LJ pair force, the fused
// integrator phases, the reductions and the cell-list rebuild.
//
// Compiled with --fmad=false: every fused multiply-add is an explicit fma()/
// fmaf(), so the FP64 integrator arithmetic is exactly the operation sequence
// written here (the CPU oracle performs the same sequence).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "mdb_internal.h"

namespace mdb {

// ---------------------------------------------------------------- helpers --

// pbc_wrap_hd (include/md_cuda_common.hpp:20-29): fmod(x, L), then + L when
// negative. For -L <= x < 2L the branches below give the same bits as fmod
// (x - L is exact there), which covers every step but pathological jumps.
// Exact remainder of x by L with the sign of x (the value fmod returns), for
// finite x, L. Each pass removes up to 40 bits of the quotient: with
// y = |L| 2^k and r / y < 2^41, q = floor(fl(r / y)) is the true quotient or
// one more (rounding to nearest never falls below an integer the true value
// reaches), so r - q y lies in [-y, y), is a multiple of ulp(y) and is
// computed exactly by one fma; adding y back to a negative remainder is exact
// as well. A particle that jumps 2^90 box lengths in one step (a FIRE start
// with overlapping pairs) takes 3 passes.
__device__ __noinline__ double fmod_exact(double x, double L) {
  if (!isfinite(x) || !isfinite(L) || L == 0.0) return fmod(x, L);
  const double a = fabs(L);
  double r = fabs(x);
  for (int pass = 0; r >= a && pass < 64; ++pass) {
    const int e = ilogb(r) - ilogb(a);
    const double y = ldexp(a, e > 40 ? e - 40 : 0);
    const double q = floor(r / y);
    double rem = fma(-q, y, r);
    if (rem < 0.0) rem += y;
    r = rem;
  }
  return copysign(r, x);
}

__device__ __forceinline__ double pbc_wrap(double x, double L) {
  if (L <= 0.0) return x;
  if (x >= 0.0 && x < L) return x;
  if (x >= L && x < 2.0 * L) return x - L;
  if (x < 0.0 && x >= -L) return x + L;
  x = fmod_exact(x, L);
  if (x < 0.0) x += L;
  return x;
}

// 1/x from the hardware approximation refined by one Newton-Raphson step
// (r1 = r0 + r0 (1 - x r0)); within one ulp of the IEEE quotient.
__device__ __forceinline__ float recip(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return fmaf(r, fmaf(-x, r, 1.0f), r);
}

// Type class for the parameter table (src/md_cuda_common.cu:218-229):
// 0 -> A, 1 -> B, anything else -> "other" (pairs with it use AB).
__device__ __forceinline__ int type_class(int t) { return t == 0 ? 0 : (t == 1 ? 1 : 2); }
// Mass (src/md_cuda_common.cu:261): type 0 -> MASS_A, else MASS_B.
__device__ __forceinline__ double type_mass(const SysParams& P, int t) {
  return t == 0 ? P.massA : P.massB;
}

// Float-float split of a biased coordinate. X = x + off lies in one binade
// [B, 2B), so the difference of two hi parts is exact; lo carries the next 24
// bits. The lowest mantissa bit of each lo part carries one bit of the type
// class (x: bit 0, y: bit 1), which moves the coordinate by at most 2^-47 B
// (1.5e-11 for B = 4096); the hi parts stay positive, so the pair loop can
// subtract x and y together with one packed FP32x2 instruction.
__device__ __forceinline__ float4 encode_ff(double x, double y, int t, double offx, double offy) {
  const double X = x + offx;
  const double Y = y + offy;
  const float xh = __double2float_rn(X);
  const float xl = __double2float_rn(X - (double)xh);
  const float yh = __double2float_rn(Y);
  const float yl = __double2float_rn(Y - (double)yh);
  const uint32_t tc = (uint32_t)type_class(t);
  return make_float4(xh, yh, __uint_as_float((__float_as_uint(xl) & ~1u) | (tc & 1u)),
                     __uint_as_float((__float_as_uint(yl) & ~1u) | (tc >> 1)));
}

// Type class carried by a float-float position (encode_ff).
__device__ __forceinline__ uint32_t ff_class(const float4 q) {
  return (__float_as_uint(q.z) & 1u) | ((__float_as_uint(q.w) << 1) & 2u);
}

// Packed FP32x2 arithmetic of sm_100: one instruction for the x and y lanes,
// each lane rounded exactly as the scalar operation.
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;"
      : "=l"(r)
      : "l"(*reinterpret_cast<unsigned long long*>(&a)),
        "l"(*reinterpret_cast<unsigned long long*>(&b)));
  return *reinterpret_cast<float2*>(&r);
}
__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// Cell index along one axis: v = coordinate * (n / L); NaN and negatives
// bin to 0, v >= n to n-1 (the oracle's or_cell_bin does the same).
__device__ __forceinline__ int bin_axis(double v, int n) {
  if (v >= 0.0 && v < (double)n) return (int)v;
  if (v >= (double)n) return n - 1;
  return 0;
}

__device__ __forceinline__ int grid_n(double L, double rcell, int cap) {
  const double f = floor(L / rcell);
  if (!(f >= 1.0)) return 1;
  if (f >= (double)cap) return cap;
  return (int)f;
}

// Compensated (Kahan) FP32 accumulation; the value is s - c.
__device__ __forceinline__ void kahan(float& s, float& c, float x) {
  const float y = x - c;
  const float t = s + y;
  c = (t - s) - y;
  s = t;
}
// The same for the x and y force components at once (packed FP32x2).
__device__ __forceinline__ void kahan2(float2& s, float2& c, float2 x) {
  const float2 y = f2sub(x, c);
  const float2 t = f2add(s, y);
  c = f2sub(f2sub(t, s), y);
  s = t;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// Fixed-order block reduction of the first NS sums and NM maxima
// (non-negative values); valid in thread 0. The tree depends only on
// blockDim, so results are bit-reproducible.
template <int NS, int NM>
__device__ __forceinline__ void block_reduce(double (&s)[kNP], double (&m)[3]) {
  if (NS == 0 && NM == 0) return;
  __shared__ double sh_s[NS > 0 ? NS : 1][kThreads / 32];
  __shared__ double sh_m[NM > 0 ? NM : 1][kThreads / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < NS; ++k) s[k] = warp_sum(s[k]);
#pragma unroll
  for (int k = 0; k < NM; ++k) m[k] = warp_max(m[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NS; ++k) sh_s[k][w] = s[k];
#pragma unroll
    for (int k = 0; k < NM; ++k) sh_m[k][w] = m[k];
  }
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int k = 0; k < NS; ++k) {
      double v = lane < kThreads / 32 ? sh_s[k][lane] : 0.0;
      s[k] = warp_sum(v);
    }
#pragma unroll
    for (int k = 0; k < NM; ++k) {
      double v = lane < kThreads / 32 ? sh_m[k][lane] : 0.0;
      m[k] = warp_max(v);
    }
  }
  __syncthreads();
}

// Sums (and maxima) of one value set over the blocks of a system, without a
// second launch and independent of block timing: each block publishes its
// partials and counts itself in with one acquire-release atomic (the release
// publishes its partials, the acquire makes every earlier block's visible);
// the block that arrives last sums all partials of the system in a fixed
// order (thread t takes blocks t, t + kThreads, ..., then the block tree).
// Returns true in that final block, whose thread 0 then holds the system
// totals in tot/tmx; its thread 0 resets S->counter when it is done.
// red/mx hold the calling thread's contributions.
template <int NS, int NM>
__device__ __forceinline__ bool reduce_system(const Dev& D, const SysParams& P, SysState* S,
                                              double (&red)[kNP], double (&mx)[3],
                                              double (&tot)[kNP], double (&tmx)[3]) {
  __shared__ int sh_last;
  block_reduce<NS, NM>(red, mx);
  if (threadIdx.x == 0) {
    double* p = D.part + (size_t)blockIdx.x * kNP;
#pragma unroll
    for (int k = 0; k < NS; ++k) p[k] = red[k];
    double* pm = D.partm + (size_t)blockIdx.x * 4;
#pragma unroll
    for (int k = 0; k < NM; ++k) pm[k] = mx[k];
    unsigned prev;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;"
                 : "=r"(prev)
                 : "l"(&S->counter)
                 : "memory");
    sh_last = (prev == (unsigned)(P.nb - 1)) ? 1 : 0;
  }
  __syncthreads();
  if (!sh_last) return false;
#pragma unroll
  for (int k = 0; k < kNP; ++k) tot[k] = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) tmx[k] = 0.0;
  for (int q = threadIdx.x; q < P.nb; q += kThreads) {
    const size_t blk = (size_t)(P.b0 + q);
#pragma unroll
    for (int k = 0; k < NS; ++k) tot[k] += __ldcg(D.part + blk * kNP + k);
#pragma unroll
    for (int k = 0; k < NM; ++k) tmx[k] = fmax(tmx[k], __ldcg(D.partm + blk * 4 + k));
  }
  block_reduce<NS, NM>(tot, tmx);
  return true;
}

// Scalars the force phase's last block reads after the system reduction,
// loaded by thread 0 of every block before it (see DriftTail).
struct ForceTail {
  int64_t steps, target_steps;
  double pA, p_ext, fl, ce, vp, W, f_dt, f_alpha, f_tol, f_inc, f_dt_max, f_dec, f_alpha0;
  double f_hp_below;
  int clamped, f_streak, f_step, f_Nmin, f_fp64;
};
template <int FM>
__device__ __forceinline__ ForceTail force_tail_inputs(const SysParams& P, const SysState* S) {
  ForceTail t{};
  if (FM == FM_NPH || FM == FM_PISTON) {
    t.p_ext = S->p_ext;
    t.clamped = S->clamped;
    t.fl = S->fl;
    t.ce = S->ce;
  }
  if (FM == FM_NPH) t.pA = S->pA;
  if (FM == FM_PISTON) {
    t.vp = S->vp;
    t.W = P.W;
  }
  if (FM == FM_FIRE) {
    t.f_hp_below = P.f_hp_below;
    t.f_fp64 = S->f_fp64;
    t.f_dt = S->f_dt;
    t.f_alpha = S->f_alpha;
    t.f_streak = S->f_streak;
    t.f_step = S->f_step;
    t.f_tol = P.f_tol;
    t.f_inc = P.f_inc;
    t.f_dt_max = P.f_dt_max;
    t.f_dec = P.f_dec;
    t.f_alpha0 = P.f_alpha0;
    t.f_Nmin = P.f_Nmin;
  }
  if (FM != FM_INIT && FM != FM_OBS && FM != FM_FIRE) {
    t.steps = S->steps;
    t.target_steps = P.target_steps;
  }
  return t;
}

// Number of sums / maxima each phase reduces.
template <int FM>
struct ForceRed {
  static constexpr int NS = (FM == FM_OBS) ? 6 : (FM == FM_NPH) ? 3
                          : (FM == FM_INIT || FM == FM_PISTON) ? 2
                          : (FM == FM_NH || FM == FM_FIRE) ? 1 : 0;
  static constexpr int NM = (FM == FM_FIRE) ? 2 : 0;
};

// Counts finished systems; the last one sets the graph condition for the
// rebuild body from the batch-wide flag. Called by thread 0 of a system's
// last block after its own state is final. A lone system sets the condition
// at once from `any` (its own request or one made before this launch).
__device__ __forceinline__ void system_done_and_signal(const Dev& D, int any) {
  if (D.nsys == 1) {
    if (D.use_cond) cudaGraphSetConditional(D.cond, any ? 1u : 0u);
    return;
  }
  __threadfence();
  const unsigned prev = atomicAdd(&D.bg->sys_counter, 1u);
  if (prev == (unsigned)(D.nsys - 1)) {
    D.bg->sys_counter = 0u;
    const int any = atomicOr(&D.bg->any_rebuild, 0);
    if (D.use_cond) cudaGraphSetConditional(D.cond, any ? 1u : 0u);
  }
}

// xi += 0.5 dt (2K - g T0) / Q (src/md_env.cu:1668-1673), host-order
// arithmetic without contraction.
__device__ __forceinline__ double nh_xi(double dt, double g_dof, double T0, double Q, double xi,
                                        double K) {
  const double t1 = 0.5 * dt;
  const double t2 = 2.0 * K;
  const double t3 = g_dof * T0;
  const double t4 = t2 - t3;
  const double t5 = t1 * t4;
  const double t6 = t5 / Q;
  return xi + t6;
}
__device__ __forceinline__ double nh_xi(const SysParams& P, double xi, double K) {
  return nh_xi(P.dt, P.g_dof, P.T0, P.Q, xi, K);
}

// Scalars the drift's last block reads after the system reduction. Thread 0
// of every block loads them before the reduction: after its acquire every
// global load is an L2 round trip, and these would be a chain of them.
struct DriftTail {
  double g_dof, T0, Q, rc_max, skin, Lx_b, Ly_b;
  int ncx, ncy, allpairs, prior;
};
__device__ __forceinline__ DriftTail drift_tail_inputs(const Dev& D, const SysParams& P,
                                                       const SysState* S) {
  DriftTail t;
  t.g_dof = P.g_dof;
  t.T0 = P.T0;
  t.Q = P.Q;
  t.rc_max = P.rc_max;
  t.skin = P.skin;
  t.Lx_b = S->Lx_b;
  t.Ly_b = S->Ly_b;
  t.ncx = S->ncx;
  t.ncy = S->ncy;
  t.allpairs = S->allpairs;
  // a rebuild requested before this launch (a forced rebuild); for a lone
  // system nothing else changes the flag until this block sets it
  t.prior = (D.nsys == 1) ? *((volatile int*)&D.bg->any_rebuild) : 0;
  return t;
}

// --------------------------------------------------------- pair interaction --

struct PairCtx {
  float2 ih, il;        // slot i's float-float position (hi, lo), x and y lanes
  float2 nLh, nLl, invL;  // -L_hi, -L_lo, 1/L_hi per axis (invL.y = 0: walled y)
  uint32_t ts;  // class whose pairs with i use the "same" parameters
  uint32_t tsz;  // pair loop: bit 0 = slot i is class 1 (B)
  uint32_t rc2s_m1, rc2ab_m1;  // pair loop: bits of rc^2, minus 1
  float rc2s, rc2ab, sig2s, sig2ab, e24s, e24ab, e4s, e4ab;
  float r2fs, r2fab;  // FLOOR: smallest r^2 used in the pair term (1e-5 sigma_ij^2)
  double Vcs, Vcab;
};

// Displacement i - j with the nearest image, x and y in the two lanes of
// packed FP32x2 instructions: the hi parts of two coordinates in the same
// binade subtract exactly, the image shift s*L_hi is exact, the lo parts carry
// the remaining bits, one rounding at the end. The walled y axis of the piston
// has invL.y = 0, which makes its shift 0.
// MIC = false: both particles are known to sit on the same side of every
// periodic edge (no image shift needed).
template <bool MIC = true>
__device__ __forceinline__ float pair_r2(const float4 q, const PairCtx& c, float2& d) {
  float2 dh = f2sub(c.ih, make_float2(q.x, q.y));
  float2 dl = f2sub(c.il, make_float2(q.z, q.w));
  if (MIC) {
    const float2 t = f2mul(dh, c.invL);
    const float2 sh = make_float2(rintf(t.x), rintf(t.y));
    dh = f2fma(sh, c.nLh, dh);
    dl = f2fma(sh, c.nLl, dl);
  }
  d = f2add(dh, dl);
  return fmaf(d.x, d.x, d.y * d.y);
}

// The LJ pair term of li_force_kernel (src/md_cuda_common.cu:193-254) for one
// candidate j: strict cutoff 0 < r^2 < rc_ij^2 in FP32, FP32 pair force, Kahan
// FP32 accumulation. ENERGY adds 1/2 (u_ij - V_c) in FP64 (:795-807); VIRIAL
// adds 1/2 r.F (:676-686) as the compensated FP32 sum of tmp*r^2.
template <bool PY, bool ENERGY, bool VIRIAL, bool MIC = true, bool FLOOR = false>
__device__ __forceinline__ void pair_one(const float4 q, const PairCtx& c, float2& fs, float2& fc,
                                         float& ws, float& wc, double& u, double& an) {
  float2 d;
  float r2 = pair_r2<MIC>(q, c, d);
  // j's class equals i's (classes 0 and 1: the lo bits of x and y are 0 / 0
  // and 1 / 0); a class-2 slot i has its "same" parameters set to AB
  const bool same = (((__float_as_uint(q.z) ^ c.tsz) | __float_as_uint(q.w)) & 1u) == 0u;
  // 0 < r2 < rc2 for the non-negative r2 (NaN fails): bits - 1 as unsigned
  if (__float_as_uint(r2) - 1u < (same ? c.rc2s_m1 : c.rc2ab_m1)) {
    // FLOOR (FIRE and observations): pairs closer than ~0.003 sigma (random
    // starts) take the pair term at r^2 = 1e-5 sigma^2, which keeps it finite
    // in FP32; the reference's FP32 term overflows to inf/NaN there.
    if (FLOOR) r2 = fmaxf(r2, same ? c.r2fs : c.r2fab);
    const float sig2 = same ? c.sig2s : c.sig2ab;
    const float e24 = same ? c.e24s : c.e24ab;
    const float r2i = recip(r2);
    const float sr2 = sig2 * r2i;
    const float sr6 = sr2 * sr2 * sr2;
    const float sr12 = sr6 * sr6;
    const float tmp = e24 * fmaf(2.0f, sr12, -sr6) * r2i;
    const float2 f = f2mul(make_float2(tmp, tmp), d);
    kahan2(fs, fc, f);
    if (VIRIAL) kahan(ws, wc, tmp * r2);
    if (ENERGY) {
      const float e4 = same ? c.e4s : c.e4ab;
      const double vc = same ? c.Vcs : c.Vcab;
      u = fma(0.5, (double)(e4 * (sr12 - sr6)) - vc, u);
      // Fx dx - Fy dy of cal_partial_U_lambda_kernel (src/md_cuda_common.cu:
      // 345-355): products of FP32 values, exact in FP64
      an += (double)f.x * (double)d.x - (double)f.y * (double)d.y;
    }
  }
}

// Neighbour-list candidates of slot i. Entry k holds the offset d of the
// partner j from i inside the system's slot range, taken modulo the system
// size n into [-n/2, n/2) (so the stencil rows across the periodic y edge stay
// small): int16 at nlist16[k * ntot + i] when the batch uses 16-bit offsets,
// else int32 at nlist[k * ntot + i]. MIC = false is the interior form: no
// minimum image and no offset wrap (j = i + d). Offsets are fetched several at
// a time before the dependent position gathers to keep loads in flight.
// Position loads of the pair loop. NC: through the read-only data path, for
// kernels that do not write positions. Otherwise a plain (weak, L1-cached)
// load: the multi-step kernel writes the positions between its phases, and
// the acquire of its grid barrier makes those writes visible to it.
template <bool NC>
__device__ __forceinline__ float4 ld_pos(const float4* p) {
  if (NC) return __ldg(p);
  float4 v;
  asm volatile("ld.global.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(p));
  return v;
}

// LANES > 1: the slot's list is shared by LANES lanes; lane `lane` takes the
// entries lane, lane + LANES, ... (the caller adds the lanes' sums).
template <bool PY, bool ENERGY, bool VIRIAL, bool MIC, bool FLOOR, bool NC, int LANES = 1,
          typename IDX>
__device__ __forceinline__ void pair_list(const float4* __restrict__ pff,
                                          const IDX* __restrict__ nlist, int64_t ntot, int64_t i,
                                          int li, int n, int nn, const PairCtx& c, float2& fs,
                                          float2& fc, float& ws, float& wc, double& u,
                                          double& an, int lane = 0) {
  const IDX* __restrict__ p = nlist + i + (int64_t)lane * ntot;
  // MIC: slot 0 of the system and a wrapped index; interior: slot i itself
  const float4* __restrict__ base = MIC ? pff + (i - li) : pff + i;
  constexpr int PF = (LANES > 1) ? 4 : ((ENERGY || VIRIAL) ? 4 : 8);  // prefetch width
  const int64_t step = (int64_t)LANES * ntot;
  nn = (LANES > 1) ? (nn > lane ? (nn - lane + LANES - 1) / LANES : 0) : nn;
  int k = 0;
  for (; k + PF <= nn; k += PF) {
    int j[PF];
#pragma unroll
    for (int q = 0; q < PF; ++q) {
      int t = (int)__ldg(p + (int64_t)(k + q) * step);
      if (MIC) {
        t += li;
        t += (t < 0) ? n : 0;
        t -= (t >= n) ? n : 0;
      }
      j[q] = t;
    }
#pragma unroll
    for (int q = 0; q < PF; ++q)
      pair_one<PY, ENERGY, VIRIAL, MIC, FLOOR>(ld_pos<NC>(base + j[q]), c, fs, fc, ws, wc, u, an);
  }
  for (; k < nn; ++k) {
    int t = (int)__ldg(p + (int64_t)k * step);
    if (MIC) {
      t += li;
      t += (t < 0) ? n : 0;
      t -= (t >= n) ? n : 0;
    }
    pair_one<PY, ENERGY, VIRIAL, MIC, FLOOR>(ld_pos<NC>(base + t), c, fs, fc, ws, wc, u, an);
  }
}

// Candidates j in [j0, j1) (cell stencil rows or the whole system).
template <bool PY, bool ENERGY, bool VIRIAL, bool FLOOR, bool NC, int LANES = 1>
__device__ __forceinline__ void pair_range(const float4* __restrict__ pff, int j0, int j1,
                                           const PairCtx& c, float2& fs, float2& fc, float& ws,
                                           float& wc, double& u, double& an, int lane = 0) {
#pragma unroll 4
  for (int j = j0 + lane; j < j1; j += LANES)
    pair_one<PY, ENERGY, VIRIAL, true, FLOOR>(ld_pos<NC>(pff + j), c, fs, fc, ws, wc, u, an);
}

__device__ __forceinline__ void split_box(double L, float& h, float& l, float& inv) {
  h = __double2float_rn(L);
  l = __double2float_rn(L - (double)h);
  inv = 1.0f / h;
}

// Slot i's position and the box in a pair context; PY = false leaves the y
// image shift at 0 (walled y axis).
template <bool PY>
__device__ __forceinline__ void set_pair_box(PairCtx& c, const float4 qi, double Lx, double Ly) {
  c.ih = make_float2(qi.x, qi.y);
  c.il = make_float2(qi.z, qi.w);
  float h, l, inv;
  split_box(Lx, h, l, inv);
  c.nLh.x = -h;
  c.nLl.x = -l;
  c.invL.x = inv;
  split_box(Ly, h, l, inv);
  c.nLh.y = -h;
  c.nLl.y = -l;
  c.invL.y = PY ? inv : 0.0f;
}

// Pair parameters of slot i's class: "same" for partners of its own class,
// "ab" otherwise (types other than 0/1 always use AB).
__device__ __forceinline__ void set_profile_class(PairCtx& c, const SysParams& P, int tci) {
  c.ts = (tci == 2) ? 99u : (uint32_t)tci;
  const int sc = (tci == 2) ? 2 : tci;
  c.rc2s = P.frc2[sc];
  c.rc2ab = P.frc2[2];
  c.sig2s = P.fsig2[sc];
  c.sig2ab = P.fsig2[2];
  c.e24s = P.feps24[sc];
  c.e24ab = P.feps24[2];
}

// Sum of pair forces on slot i over its 3x3 cell stencil (or every slot of the
// system for grids narrower than 3 cells). Returns F in FP64. tci receives the
// type class of slot i, decoded from its float-float position (encode_ff), so
// the type array is not read.
//
// LANES > 1: lane `lane` of the LANES lanes that share slot i sums its share
// of the candidates (the caller adds the lanes' results in a fixed order).
template <bool PY, bool ENERGY, bool VIRIAL, bool FLOOR = false, bool NC = true, int LANES = 1>
__device__ __forceinline__ void particle_force(const Dev& D, const SysParams& P, const SysState& S,
                                               int64_t i, double Lx, double Ly, double& fx,
                                               double& fy, double& w, double& u, double& an,
                                               int& tci, int lane = 0) {
  PairCtx c;
  const float4 qi = ld_pos<NC>(D.pff + i);
  set_pair_box<PY>(c, qi, Lx, Ly);
  tci = (int)ff_class(qi);
  c.ts = (tci == 2) ? 99u : (uint32_t)tci;
  c.tsz = (tci == 1) ? 1u : 0u;
  const int sc = (tci == 2) ? 2 : tci;
  c.rc2s = P.frc2[sc];
  c.rc2ab = P.frc2[2];
  c.rc2s_m1 = __float_as_uint(c.rc2s) - 1u;
  c.rc2ab_m1 = __float_as_uint(c.rc2ab) - 1u;
  c.sig2s = P.fsig2[sc];
  c.sig2ab = P.fsig2[2];
  c.e24s = P.feps24[sc];
  c.e24ab = P.feps24[2];
  c.e4s = P.feps4[sc];
  c.e4ab = P.feps4[2];
  c.Vcs = P.Vc[sc];
  c.Vcab = P.Vc[2];
  if (FLOOR) {
    c.r2fs = 1e-5f * P.fsig2[sc];
    c.r2fab = 1e-5f * P.fsig2[2];
  }
  float2 fs = make_float2(0.f, 0.f), fc = make_float2(0.f, 0.f);
  float ws = 0.f, wc = 0.f;
  u = 0.0;
  an = 0.0;
  const float4* __restrict__ pff = D.pff;
  const int nc = __ldg(D.ncount + i);
  if (nc >= 0) {
    const int li = (int)(i - P.p0);
    const int nn = nc & (kListInterior - 1);
    if (D.nl16) {
      if (nc & kListInterior)
        pair_list<PY, ENERGY, VIRIAL, false, FLOOR, NC, LANES>(pff, D.nlist16, D.ntot, i, li, P.n, nn, c, fs,
                                                  fc, ws, wc, u, an, lane);
      else
        pair_list<PY, ENERGY, VIRIAL, true, FLOOR, NC, LANES>(pff, D.nlist16, D.ntot, i, li, P.n, nn, c, fs,
                                                 fc, ws, wc, u, an, lane);
    } else {
      if (nc & kListInterior)
        pair_list<PY, ENERGY, VIRIAL, false, FLOOR, NC, LANES>(pff, D.nlist, D.ntot, i, li, P.n, nn, c, fs,
                                                  fc, ws, wc, u, an, lane);
      else
        pair_list<PY, ENERGY, VIRIAL, true, FLOOR, NC, LANES>(pff, D.nlist, D.ntot, i, li, P.n, nn, c, fs,
                                                 fc, ws, wc, u, an, lane);
    }
  } else if (S.allpairs) {
    pair_range<PY, ENERGY, VIRIAL, FLOOR, NC, LANES>(pff, (int)P.p0, (int)(P.p0 + P.n), c, fs, fc, ws, wc,
                                          u, an, lane);
  } else {
    const int ncx = S.ncx, ncy = S.ncy;
    const int cell = D.cell_of[i];
    const int cx = cell % ncx, cy = cell / ncx;
    const int* __restrict__ cs = D.cstart;
#pragma unroll 1
    for (int dr = -1; dr <= 1; ++dr) {
      int yy = cy + dr;
      if (PY) {
        if (yy < 0) yy += ncy;
        if (yy >= ncy) yy -= ncy;
      } else if (yy < 0 || yy >= ncy) {
        continue;
      }
      const int64_t row = P.c0 + (int64_t)yy * ncx;
      if (cx > 0 && cx < ncx - 1) {
        pair_range<PY, ENERGY, VIRIAL, FLOOR, NC, LANES>(pff, __ldg(cs + row + cx - 1),
                                              __ldg(cs + row + cx + 2), c, fs, fc, ws, wc, u, an, lane);
      } else if (cx == 0) {
        pair_range<PY, ENERGY, VIRIAL, FLOOR, NC, LANES>(pff, __ldg(cs + row), __ldg(cs + row + 2), c, fs, fc,
                                              ws, wc, u, an, lane);
        pair_range<PY, ENERGY, VIRIAL, FLOOR, NC, LANES>(pff, __ldg(cs + row + ncx - 1),
                                              __ldg(cs + row + ncx), c, fs, fc, ws, wc, u, an, lane);
      } else {
        pair_range<PY, ENERGY, VIRIAL, FLOOR, NC, LANES>(pff, __ldg(cs + row + ncx - 2),
                                              __ldg(cs + row + ncx), c, fs, fc, ws, wc, u, an, lane);
        pair_range<PY, ENERGY, VIRIAL, FLOOR, NC, LANES>(pff, __ldg(cs + row), __ldg(cs + row + 1), c, fs, fc,
                                              ws, wc, u, an, lane);
      }
    }
  }
  fx = (double)fs.x - (double)fc.x;
  fy = (double)fs.y - (double)fc.y;
  w = 0.5 * ((double)ws - (double)wc);
}

// ------------------------------------------------- FP64 pair terms (FIRE) --
// The same candidates as particle_force with every pair term in FP64: the
// float-float coordinates converted to double are exact (hi and lo together
// hold 48 bits), their difference is exact, the nearest image and the LJ
// term are FP64 and the sums are FP64. Used by FIRE systems near convergence,
// where FP32 pair terms leave a force noise floor near 1e-6.
struct PairCtxD {
  double xi, yi, Lx, Ly, invLx, invLy;
  uint32_t ts;
  double rc2s, rc2ab, sig2s, sig2ab, e24s, e24ab, e4s, e4ab, Vcs, Vcab;
};

template <bool PY, bool ENERGY, bool VIRIAL, bool MIC>
__device__ __forceinline__ void pair_one_hp(const float4 q, const PairCtxD& c, double& fx,
                                            double& fy, double& w, double& u, double& an) {
  double dx = c.xi - ((double)q.x + (double)q.z);
  double dy = c.yi - ((double)q.y + (double)q.w);
  if (MIC) {
    dx = fma(-rint(dx * c.invLx), c.Lx, dx);
    if (PY) dy = fma(-rint(dy * c.invLy), c.Ly, dy);
  }
  const double r2 = fma(dx, dx, dy * dy);
  const bool same = (ff_class(q) == c.ts);
  const double rc2 = same ? c.rc2s : c.rc2ab;
  if (r2 > 0.0 && r2 < rc2) {
    const double sig2 = same ? c.sig2s : c.sig2ab;
    const double r2e = fmax(r2, 1e-5 * sig2);  // the FP32 path's distance floor
    const double r2i = 1.0 / r2e;
    const double sr2 = sig2 * r2i;
    const double sr6 = sr2 * sr2 * sr2;
    const double sr12 = sr6 * sr6;
    const double tmp = (same ? c.e24s : c.e24ab) * fma(2.0, sr12, -sr6) * r2i;
    fx = fma(tmp, dx, fx);
    fy = fma(tmp, dy, fy);
    if (VIRIAL) w = fma(tmp, r2e, w);
    if (ENERGY) {
      u = fma(0.5, (same ? c.e4s : c.e4ab) * (sr12 - sr6) - (same ? c.Vcs : c.Vcab), u);
      an += (tmp * dx) * dx - (tmp * dy) * dy;
    }
  }
}

template <bool PY, bool ENERGY, bool VIRIAL, bool MIC, typename IDX>
__device__ __forceinline__ void pair_list_hp(const float4* __restrict__ pff,
                                             const IDX* __restrict__ nlist, int64_t ntot,
                                             int64_t i, int li, int n, int nn, const PairCtxD& c,
                                             double& fx, double& fy, double& w, double& u,
                                             double& an) {
  const float4* __restrict__ base = MIC ? pff + (i - li) : pff + i;
  for (int k = 0; k < nn; ++k) {
    int t = (int)__ldg(nlist + i + (int64_t)k * ntot);
    if (MIC) {
      t += li;
      t += (t < 0) ? n : 0;
      t -= (t >= n) ? n : 0;
    }
    pair_one_hp<PY, ENERGY, VIRIAL, MIC>(__ldg(base + t), c, fx, fy, w, u, an);
  }
}

template <bool PY, bool ENERGY, bool VIRIAL>
__device__ __forceinline__ void pair_range_hp(const float4* __restrict__ pff, int j0, int j1,
                                              const PairCtxD& c, double& fx, double& fy,
                                              double& w, double& u, double& an) {
  for (int j = j0; j < j1; ++j)
    pair_one_hp<PY, ENERGY, VIRIAL, true>(__ldg(pff + j), c, fx, fy, w, u, an);
}

// FP64 counterpart of particle_force (same outputs; w already halved).
template <bool PY, bool ENERGY, bool VIRIAL>
__device__ __forceinline__ void particle_force_hp(const Dev& D, const SysParams& P,
                                               const SysState& S, int64_t i, double Lx,
                                               double Ly, double& fx, double& fy, double& w,
                                               double& u, double& an) {
  PairCtxD c;
  const float4 qi = __ldg(D.pff + i);
  c.xi = (double)qi.x + (double)qi.z;
  c.yi = (double)qi.y + (double)qi.w;
  c.Lx = Lx;
  c.Ly = Ly;
  c.invLx = 1.0 / Lx;
  c.invLy = 1.0 / Ly;
  const int tci = (int)ff_class(qi);
  c.ts = (tci == 2) ? 99u : (uint32_t)tci;
  const int sc = (tci == 2) ? 2 : tci;
  const double rs = P.cutoff * P.sig[sc], rab = P.cutoff * P.sig[2];
  c.rc2s = rs * rs;
  c.rc2ab = rab * rab;
  c.sig2s = P.sig[sc] * P.sig[sc];
  c.sig2ab = P.sig[2] * P.sig[2];
  c.e24s = 24.0 * P.eps[sc];
  c.e24ab = 24.0 * P.eps[2];
  c.e4s = 4.0 * P.eps[sc];
  c.e4ab = 4.0 * P.eps[2];
  c.Vcs = P.Vc[sc];
  c.Vcab = P.Vc[2];
  fx = fy = w = u = an = 0.0;
  const float4* __restrict__ pff = D.pff;
  const int nc = __ldg(D.ncount + i);
  if (nc >= 0) {
    const int li = (int)(i - P.p0);
    const int nn = nc & (kListInterior - 1);
    const bool interior = (nc & kListInterior) != 0;
    if (D.nl16) {
      if (interior)
        pair_list_hp<PY, ENERGY, VIRIAL, false>(pff, D.nlist16, D.ntot, i, li, P.n, nn, c, fx,
                                                fy, w, u, an);
      else
        pair_list_hp<PY, ENERGY, VIRIAL, true>(pff, D.nlist16, D.ntot, i, li, P.n, nn, c, fx, fy,
                                               w, u, an);
    } else {
      if (interior)
        pair_list_hp<PY, ENERGY, VIRIAL, false>(pff, D.nlist, D.ntot, i, li, P.n, nn, c, fx, fy,
                                                w, u, an);
      else
        pair_list_hp<PY, ENERGY, VIRIAL, true>(pff, D.nlist, D.ntot, i, li, P.n, nn, c, fx, fy,
                                               w, u, an);
    }
  } else if (S.allpairs) {
    for (int64_t j = P.p0; j < P.p0 + P.n; ++j) {
      if (j == i) continue;
      pair_one_hp<PY, ENERGY, VIRIAL, true>(__ldg(pff + j), c, fx, fy, w, u, an);
    }
  } else {
    const int ncx = S.ncx, ncy = S.ncy;
    const int cell = D.cell_of[i];
    const int cx = cell % ncx, cy = cell / ncx;
    const int* __restrict__ cs = D.cstart;
    for (int dr = -1; dr <= 1; ++dr) {
      int yy = cy + dr;
      if (PY) {
        if (yy < 0) yy += ncy;
        if (yy >= ncy) yy -= ncy;
      } else if (yy < 0 || yy >= ncy) {
        continue;
      }
      const int64_t row = P.c0 + (int64_t)yy * ncx;
      if (cx > 0 && cx < ncx - 1) {
        pair_range_hp<PY, ENERGY, VIRIAL>(pff, __ldg(cs + row + cx - 1), __ldg(cs + row + cx + 2),
                                          c, fx, fy, w, u, an);
      } else if (cx == 0) {
        pair_range_hp<PY, ENERGY, VIRIAL>(pff, __ldg(cs + row), __ldg(cs + row + 2), c, fx, fy, w,
                                          u, an);
        pair_range_hp<PY, ENERGY, VIRIAL>(pff, __ldg(cs + row + ncx - 1), __ldg(cs + row + ncx),
                                          c, fx, fy, w, u, an);
      } else {
        pair_range_hp<PY, ENERGY, VIRIAL>(pff, __ldg(cs + row + ncx - 2), __ldg(cs + row + ncx),
                                          c, fx, fy, w, u, an);
        pair_range_hp<PY, ENERGY, VIRIAL>(pff, __ldg(cs + row), __ldg(cs + row + 1), c, fx, fy, w,
                                          u, an);
      }
    }
  }
  w = 0.5 * w;
}

// Soft walls of piston_wall_kernel (src/md_cuda_common.cu:498-552) for one
// particle: returns the y wall force and adds to the upper-wall force and the
// wall energy.
__device__ __forceinline__ double wall_terms(double y, double Ly, double k, double& up,
                                             double& en) {
  double wf = 0.0;
  up = 0.0;
  en = 0.0;
  if (k > 0.0) {
    if (y > Ly) {
      const double ov = y - Ly;
      wf = fma(-k, ov, wf);
      up = fma(k, ov, up);
      en = fma((0.5 * k) * ov, ov, en);
    }
    if (y < 0.0) {
      const double ov = -y;
      wf = fma(k, ov, wf);
      en = fma((0.5 * k) * ov, ov, en);
    }
  }
  return wf;
}

// What follows the pair sum of one slot in the force phase: the kick, the
// reductions and the stores (the sums are the caller's per-thread partials).
template <int FM, bool PY>
struct ForceFinish {
  double red[kNP];
  double mx[3];
  int bad;
  __device__ __forceinline__ void init() {
#pragma unroll
    for (int k = 0; k < kNP; ++k) red[k] = 0.0;
    mx[0] = mx[1] = mx[2] = 0.0;
    bad = 0;
  }
  __device__ __forceinline__ void operator()(const Dev& D, const SysParams& P, double Ly,
                                             double h, double xi2, double fdt, int64_t i,
                                             double fx, double fy, double w, double u, double an,
                                             int tci) {
    const double m = (tci == 0) ? P.massA : P.massB;  // type 0 <=> class 0
    double2 v = D.vel[i];
    if (FM == FM_OBS) {
      red[0] += u;
      red[1] += w;
      red[2] += m * fma(v.x, v.x, v.y * v.y);
      if (!PY) {
        double up, en;
        wall_terms(D.pos[i].y, Ly, P.k_piston, up, en);
        red[3] += up;
        red[4] += en;
      }
      red[5] += an;
    } else {
      // x / 1.0 == x exactly: skip the two FP64 divisions for unit masses
      double ax, ay;
      if (m == 1.0) {
        ax = fx;
        ay = fy;
      } else {
        ax = fx / m;
        ay = fy / m;
      }
      if (!PY && (FM == FM_INIT || FM == FM_PISTON)) {
        double up, en;
        const double wf = wall_terms(D.pos[i].y, Ly, P.k_piston, up, en);
        if (wf != 0.0) ay = ay + wf / m;
        red[0] += up;
        red[1] += en;
      }
      if (FM == FM_NVE || FM == FM_PISTON) {
        v.x = fma(h, ax, v.x);
        v.y = fma(h, ay, v.y);
      } else if (FM == FM_NH) {
        v.x = fma(h, fma(-xi2, v.x, ax), v.x);
        v.y = fma(h, fma(-xi2, v.y, ay), v.y);
        red[0] += (0.5 * m) * fma(v.x, v.x, v.y * v.y);
      } else if (FM == FM_NPH) {
        red[0] += m * fma(v.x, v.x, v.y * v.y);
        v.x = fma(h, ax, v.x);
        v.y = fma(h, ay, v.y);
        red[1] += m * fma(v.x, v.x, v.y * v.y);
        red[2] += w;
      } else if (FM == FM_FIRE) {
        v.x = fma(fdt, ax, v.x);
        v.y = fma(fdt, ay, v.y);
        // ForceMag / PowerVal of reduce_force_metrics (src/md_energy_minimizer.cu:416-446)
        const double fm = sqrt(fma(ax, ax, ay * ay));
        if (fm != fm) {
          mx[1] = 1.0;  // NaN |a|: never converged
        } else {
          mx[0] = fmax(mx[0], fm);
        }
        red[0] += fma(v.x, ax, v.y * ay);
      }
      D.acc[i] = make_double2(ax, ay);
      if (FM != FM_INIT) D.vel[i] = v;
      if (!isfinite(ax) || !isfinite(ay) || !isfinite(v.x) || !isfinite(v.y)) bad = 1;
    }
  }
};

// The force phase's slots of one thread with FP64 pair terms (a FIRE system
// past its switch point, and its observations). Out of line: its registers
// do not count against the FP32 pair loop of the kernel.
template <int FM, bool PY>
__device__ __noinline__ ForceFinish<FM, PY> force_items_hp(Dev D, const SysParams* Pp,
                                                           const SysState* Sp, int64_t base,
                                                           int64_t stride, int64_t end,
                                                           int items, double Lx, double Ly,
                                                           double h, double xi2, double fdt) {
  constexpr bool kEnergy = (FM == FM_OBS);
  constexpr bool kVirial = (FM == FM_OBS || FM == FM_NPH);
  const SysParams& P = *Pp;
  ForceFinish<FM, PY> fin;
  fin.init();
  for (int it = 0; it < items; ++it) {
    const int64_t i = base + (int64_t)it * stride;
    if (i >= end) break;
    double fx, fy, w, u, an;
    const float4 qi = __ldg(D.pff + i);
    const int tci = (int)ff_class(qi);
    particle_force_hp<PY, kEnergy, kVirial>(D, P, *Sp, i, Lx, Ly, fx, fy, w, u, an);
    fin(D, P, Ly, h, xi2, fdt, i, fx, fy, w, u, an, tci);
  }
  return fin;
}

// ------------------------------------------------------------ force phase --
// One thread per slot. FM selects what follows the force evaluation; PY is the
// y image convention (false = the piston's walled y axis, which also applies
// the soft walls in FM_INIT/FM_OBS).
//
// force_phase is the work of block b of the launch; k_force runs it as one
// kernel, k_md_steps as a phase of its multi-step loop (NC = false: plain
// position loads, see ld_pos).
template <int FM, bool PY, bool NC, bool LN>
__device__ __forceinline__ void force_phase(const Dev& D, const int b) {
  const int s = D.sys_of_block[b];
  const SysParams& P = D.sp[s];
  SysState* S = D.st + s;
  if (!LN || P.lanes == 1) {
    // L1 prefetch of this thread's first slot and its first list rows
    const int64_t i0 = P.p0 + (int64_t)(b - P.b0) * kThreads + threadIdx.x;
    if (i0 < P.p0 + P.n) {
      asm volatile("prefetch.global.L1 [%0];" ::"l"(D.pff + i0));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(D.vel + i0));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(D.ncount + i0));
      if (D.nl16 && D.max_nbr >= 8) {
#pragma unroll
        for (int q = 0; q < 8; ++q)
          asm volatile("prefetch.global.L1 [%0];" ::"l"(D.nlist16 + (int64_t)q * D.ntot + i0));
      }
    }
  }
  // a finished batch system is still observed (FM_OBS) and re-evaluated (FM_INIT)
  const bool skip = (FM != FM_OBS && FM != FM_INIT && S->done != 0) || (S->err != 0) ||
                    (FM == FM_FIRE && (S->f_conv != 0 || S->f_step >= P.f_max_steps));
  constexpr bool kEnergy = (FM == FM_OBS);
  constexpr bool kVirial = (FM == FM_OBS || FM == FM_NPH);
  constexpr int kNS = ForceRed<FM>::NS, kNM = ForceRed<FM>::NM;
  const double Lx = S->Lx, Ly = S->Ly;
  const double dt = P.dt, h = 0.5 * dt;
  const int items = P.items;
  // Block b of the system takes the kThreads-slot chunks b, b + nb, b + 2 nb,
  // ...: the chunks of one block come from across the whole system, so dense
  // and sparse regions (different list lengths) even out between blocks.
  const int64_t base = P.p0 + (int64_t)(b - P.b0) * kThreads + threadIdx.x;
  const int64_t stride = (int64_t)P.nb * kThreads;
  const int64_t end = P.p0 + P.n;
  const double xi2 = (FM == FM_NH) ? S->xi : 0.0;
  const double fdt = (FM == FM_FIRE) ? S->f_dt : 0.0;
  // What follows the pair sum of one slot (kick, reductions, stores).
  constexpr bool kHpCapable = (FM == FM_FIRE || FM == FM_OBS || FM == FM_INIT);
  ForceFinish<FM, PY> fin;
  if (kHpCapable && !skip && S->f_fp64 != 0) {
    fin = force_items_hp<FM, PY>(D, &P, S, base, stride, end, items, Lx, Ly, h, xi2, fdt);
  } else if (LN && P.lanes == kLanes) {
    // kLanes lanes per slot: a block covers kThreads / kLanes slots; the
    // lanes of a slot split its candidates, their sums are added in a fixed
    // butterfly (every lane ends with the same bits) and the first lane
    // finishes the slot. items is 1 for these systems.
    fin.init();
    constexpr int spb = kThreads / kLanes;
    const int lane = threadIdx.x % kLanes;
    const int64_t i = P.p0 + (int64_t)(b - P.b0) * spb + threadIdx.x / kLanes;
    double fx = 0.0, fy = 0.0, w = 0.0, u = 0.0, an = 0.0;
    int tci = 0;
    if (!skip && i < end)
      particle_force<PY, kEnergy, kVirial, kHpCapable, NC, kLanes>(D, P, *S, i, Lx, Ly, fx, fy, w,
                                                                 u, an, tci, lane);
#pragma unroll
    for (int o = 1; o < kLanes; o <<= 1) {
      fx += __shfl_xor_sync(0xffffffffu, fx, o);
      fy += __shfl_xor_sync(0xffffffffu, fy, o);
      if (kVirial) w += __shfl_xor_sync(0xffffffffu, w, o);
      if (kEnergy) {
        u += __shfl_xor_sync(0xffffffffu, u, o);
        an += __shfl_xor_sync(0xffffffffu, an, o);
      }
    }
    if (!skip && i < end && lane == 0) fin(D, P, Ly, h, xi2, fdt, i, fx, fy, w, u, an, tci);
  } else {
    fin.init();
    const int q_first = b - P.b0;
#pragma unroll 1
    for (int it = 0; it < items; ++it) {
      // the block's chunk of this pass (every thread of the block agrees)
      // (rotated by half the blocks per pass: a block's chunks spread over
      // the system, each pass still covering one contiguous band of chunks)
      const int q = it * P.nb + (int)((q_first + (int64_t)it * (P.nb / 2)) % P.nb);
      const int64_t cs = P.p0 + (int64_t)q * kThreads;
      if (skip || cs >= end) break;
      const int64_t i = cs + threadIdx.x;
      {
        // L1 prefetch of the next chunk's list rows (lane r of a warp: row r
        // of the warp's 32 slots), counts, velocities and positions, so that
        // its dependent loads do not each wait a DRAM round trip
        const int64_t ncs = cs + (int64_t)P.nb * kThreads;
        const int64_t wslot = ncs + (threadIdx.x & ~31);
        if (wslot < end) {
          const int lane = threadIdx.x & 31;
          if (lane < D.pf_rows && lane < D.max_nbr) {
            if (D.nl16)
              asm volatile("prefetch.global.L1 [%0];" ::"l"(D.nlist16 + (int64_t)lane * D.ntot +
                                                             wslot));
            else
              asm volatile("prefetch.global.L1 [%0];" ::"l"(D.nlist + (int64_t)lane * D.ntot +
                                                             wslot));
          }
          if (ncs + threadIdx.x < end) {
            asm volatile("prefetch.global.L1 [%0];" ::"l"(D.ncount + ncs + threadIdx.x));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(D.vel + ncs + threadIdx.x));
            asm volatile("prefetch.global.L1 [%0];" ::"l"(D.pff + ncs + threadIdx.x));
          }
        }
      }
      double fx, fy, w, u, an;
      int tci;
      if (i < end) {
        particle_force<PY, kEnergy, kVirial, kHpCapable, NC>(D, P, *S, i, Lx, Ly, fx, fy, w, u, an,
                                                         tci);
        fin(D, P, Ly, h, xi2, fdt, i, fx, fy, w, u, an, tci);
      }
    }
  }
  if (fin.bad) atomicOr(&S->nonfinite, 1);
  ForceTail tin;
  if (threadIdx.x == 0) tin = force_tail_inputs<FM>(P, S);
  double tot[kNP];
  double tmx[3];
  if (!reduce_system<kNS, kNM>(D, P, S, fin.red, fin.mx, tot, tmx)) return;
  if (threadIdx.x != 0) return;
  int conv = 0;
  if (!skip) {
    if (FM == FM_NH) {
      S->K = tot[0];
    } else if (FM == FM_NPH) {
      const double A = Lx * Ly;
      const double p_new = (A > 0.0) ? (tot[0] + tot[2]) / (2.0 * A) : 0.0;
      double pA = tin.pA + h * (p_new - tin.p_ext);
      if (tin.clamped) {
        if (Ly <= tin.fl && pA < 0.0) pA = 0.0;
        if (Ly >= tin.ce && pA > 0.0) pA = 0.0;
      }
      S->pA = pA;
      S->last_P = p_new;
      S->P_cur = (A > 0.0) ? (tot[1] + tot[2]) / (2.0 * A) : 0.0;
      S->Wv = tot[2];
    } else if (FM == FM_PISTON) {
      const double Fp = tot[0];
      const double a_new = (Fp - tin.p_ext * Lx) / tin.W;
      double vp = tin.vp + h * a_new;
      if (tin.clamped) {
        if (Ly <= tin.fl && vp < 0.0) vp = 0.0;
        if (Ly >= tin.ce && vp > 0.0) vp = 0.0;
      }
      S->vp = vp;
      S->Fp = Fp;
      S->wallU = tot[1];
      S->last_P = Fp / Lx;
    } else if (FM == FM_INIT) {
      if (!PY) {
        S->Fp = tot[0];
        S->wallU = tot[1];
      }
    } else if (FM == FM_OBS) {
      S->U = tot[0];
      S->Wv = tot[1];
      S->kin = tot[2];
      S->kin2 = tot[3];
      S->wallU = tot[4];
      S->Wani = 0.5 * tot[5];
    } else if (FM == FM_FIRE) {
      // FIRE control (src/md_energy_minimizer.cu:171-203)
      const double maxf = (tmx[1] > 0.0) ? __longlong_as_double(0x7ff8000000000000ULL) : tmx[0];
      S->f_power = tot[0];
      S->f_maxf = maxf;
      // from the next iteration on, FP64 pair terms for this system
      if (!tin.f_fp64 && maxf < tin.f_hp_below) S->f_fp64 = 1;
      if (maxf < tin.f_tol) {
        conv = 1;
        S->f_conv = 1;
        S->f_conv_step = tin.f_step;
      } else {
        if (tot[0] > 0.0) {
          const int streak = tin.f_streak + 1;
          S->f_streak = streak;
          if (streak > tin.f_Nmin) {
            const double d2 = tin.f_dt * tin.f_inc;
            S->f_dt = d2 < tin.f_dt_max ? d2 : tin.f_dt_max;
            const double a2 = tin.f_alpha * 0.99;
            S->f_alpha = a2 > 0.0 ? a2 : 0.0;
          }
          S->f_zero_v = 0;
        } else {
          S->f_dt = tin.f_dt * tin.f_dec;
          S->f_streak = 0;
          S->f_alpha = tin.f_alpha0;
          S->f_zero_v = 1;
        }
        S->f_step = tin.f_step + 1;
      }
    }
    if (FM != FM_INIT && FM != FM_OBS && FM != FM_FIRE) {
      const int64_t steps = tin.steps + 1;
      S->steps = steps;
      // an MD segment of a batch ends after its target number of steps
      if (tin.target_steps > 0 && steps >= tin.target_steps) S->done = 1;
    }
  }
  // (a system that was converged at launch is skipped)
  if (FM == FM_FIRE) S->f_drift = (!skip && !conv) ? 1 : 0;
  S->counter = 0u;
}

// LN: the launch holds systems with several lanes per slot (the kernel
// without them keeps the one-lane code only).
template <int FM, bool PY, bool LN>
__global__ void __launch_bounds__(kThreads, 4) k_force(Dev D) {
  force_phase<FM, PY, true, LN>(D, blockIdx.x);
}

// ------------------------------------------------------------ drift phase --
// First half of a step for one slot: kick + drift + wrap (mode-specific),
// float-float refresh, displacement since the last rebuild. The system's last
// block applies the scalar updates and the rebuild criterion.
struct DriftCtx {
  double dt, h, xi1, lam, vsc, fdt, alpha, Lx, Ly, ilx, ily, ilx_old, ily_old;
  double massA, massB, offx, offy;
  int zero_v, py;
};

// One particle's drift from its loaded state.
template <int DMd>
__device__ __forceinline__ void drift_particle(const Dev& D, const DriftCtx& c, int64_t i,
                                               double2 x, double2 v, const double2 a, int t,
                                               const float2 sb, double& ksum, double& mdx,
                                               double& mdy, double& mjump, int& bad) {
  const double m = t == 0 ? c.massA : c.massB;
  const double2 x0 = x;
  if (DMd == DM_NVE || DMd == DM_PISTON) {
    // step_half_vv_kernel (src/md_cuda_common.cu:381-394), piston (:396-409)
    v.x = fma(c.h, a.x, v.x);
    v.y = fma(c.h, a.y, v.y);
    x.x = fma(c.dt, v.x, x.x);
    x.y = fma(c.dt, v.y, x.y);
  } else if (DMd == DM_NH) {
    // step_half_vv_nh_kernel (src/md_cuda_common.cu:454-478)
    v.x = fma(c.h, fma(-c.xi1, v.x, a.x), v.x);
    v.y = fma(c.h, fma(-c.xi1, v.y, a.y), v.y);
    x.x = fma(c.dt, v.x, x.x);
    x.y = fma(c.dt, v.y, x.y);
    ksum += (0.5 * m) * fma(v.x, v.x, v.y * v.y);
  } else if (DMd == DM_NPH) {
    // step_half_nph_velocity_kernel + step_nph_scale_and_drift_kernel (:411-440)
    v.x = fma(c.h, a.x, v.x);
    v.y = fma(c.h, a.y, v.y);
    v.x = v.x * c.vsc;
    v.y = v.y * c.vsc;
    x.x = fma(c.lam, x.x, c.dt * v.x);
    x.y = fma(c.lam, x.y, c.dt * v.y);
  } else if (DMd == DM_FIRE) {
    // zero_velocity / fire_velocity_mix / drift (src/md_energy_minimizer.cu:32-71)
    if (c.zero_v) {
      v.x = 0.0;
      v.y = 0.0;
    } else {
      const double vmag = sqrt(fma(v.x, v.x, v.y * v.y));
      const double fmag = sqrt(fma(a.x, a.x, a.y * a.y));
      if (vmag > 0.0 && fmag > 0.0) {
        const double scale = vmag / fmag;
        v.x = fma(c.alpha * scale, a.x, (1.0 - c.alpha) * v.x);
        v.y = fma(c.alpha * scale, a.y, (1.0 - c.alpha) * v.y);
      }
    }
    x.x = fma(c.fdt, v.x, x.x);
    x.y = fma(c.fdt, v.y, x.y);
  }
  const double xu = x.x, yu = x.y;
  x.x = pbc_wrap(x.x, c.Lx);
  if (DMd != DM_PISTON) x.y = pbc_wrap(x.y, c.Ly);
  D.pos[i] = x;
  D.vel[i] = v;
  D.pff[i] = encode_ff(x.x, x.y, t, c.offx, c.offy);
  // displacement since the last rebuild and the single-step jump
  float dsx = (float)(x.x * c.ilx) - sb.x;
  dsx -= rintf(dsx);
  const double dxr = (double)fabsf(dsx) * c.Lx;
  double dyr;
  if (c.py && DMd != DM_PISTON) {
    float dsy = (float)(x.y * c.ily) - sb.y;
    dsy -= rintf(dsy);
    dyr = (double)fabsf(dsy) * c.Ly;
  } else {
    dyr = fabs(x.y - (double)sb.y);
  }
  // (only the NPH step rescales the box inside the step)
  const double jx = (DMd == DM_NPH) ? fabs(xu * c.ilx - x0.x * c.ilx_old) * c.Lx : fabs(xu - x0.x);
  const double jy = (DMd == DM_NPH) ? fabs(yu * c.ily - x0.y * c.ily_old) * c.Ly : fabs(yu - x0.y);
  mdx = fmax(mdx, dxr);
  mdy = fmax(mdy, dyr);
  mjump = fmax(mjump, fmax(jx, jy));
  if (!isfinite(x.x) || !isfinite(x.y) || !isfinite(v.x) || !isfinite(v.y)) {
    bad = 1;
    mjump = __longlong_as_double(0x7ff0000000000000ULL);
  }
}

// drift_phase is the work of block b of the launch (k_drift: one kernel;
// k_md_steps: a phase of its multi-step loop).
template <int DMd, bool LN>
__device__ __forceinline__ void drift_phase(const Dev& D, const int b) {
  // (a lone system needs no table lookup: one dependent load less per block)
  const int s = D.nsys == 1 ? 0 : D.sys_of_block[b];
  const SysParams& P = D.sp[s];
  SysState* S = D.st + s;
  {
    // L1 prefetch of this thread's first particle: its DRAM latency overlaps
    // the scalar prologue below
    const int spb0 = LN ? kThreads / P.lanes : kThreads;
    const int64_t i0 = P.p0 + (int64_t)(b - P.b0) * spb0 * P.items + threadIdx.x;
    if ((int)threadIdx.x < spb0 && i0 < P.p0 + P.n) {
      asm volatile("prefetch.global.L1 [%0];" ::"l"(D.pos + i0));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(D.vel + i0));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(D.acc + i0));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(D.type + i0));
      asm volatile("prefetch.global.L1 [%0];" ::"l"(D.sb + i0));
    }
  }
  const bool skip = (S->done != 0) || (S->err != 0) || (DMd == DM_FIRE && S->f_drift == 0);
  constexpr int kNS = (DMd == DM_NH) ? 1 : 0, kNM = 3;
  const double dt = P.dt, h = 0.5 * dt;
  const double Lx_old = S->Lx, Ly_old = S->Ly;
  double Lx = Lx_old, Ly = Ly_old;
  const bool py = S->periodic_y != 0;
  // ---- scalar prelude (identical in every block) ----
  double xi1 = 0.0, lam = 1.0, vsc = 1.0, pA1 = 0.0, vp1 = 0.0, aspect = S->aspect;
  int clamped = 0, boxbad = 0;
  if (DMd == DM_NH) xi1 = nh_xi(P, S->xi, S->K);
  if (DMd == DM_NPH) {
    // step_single_NPH (src/md_env.cu:1795-1881)
    const double A_old = Lx_old * Ly_old;
    pA1 = S->pA + h * (S->P_cur - S->p_ext);
    double A_new = A_old + dt * (pA1 / P.W);
    if (!(A_old > 0.0) || !(A_new > 0.0) || !isfinite(A_new)) boxbad = 1;
    if (!(aspect > 0.0) || !isfinite(aspect)) aspect = Lx_old / Ly_old;
    double Ly_new = sqrt(A_new / aspect);
    double Lx_new = aspect * Ly_new;
    if (Ly_new < S->fl) {
      Ly_new = S->fl;
      Lx_new = aspect * Ly_new;
      A_new = Lx_new * Ly_new;
      clamped = 1;
    } else if (Ly_new > S->ce) {
      Ly_new = S->ce;
      Lx_new = aspect * Ly_new;
      A_new = Lx_new * Ly_new;
      clamped = 1;
    }
    lam = sqrt(A_new / A_old);
    vsc = 1.0 / lam;
    if (Lx_new <= 0.0 || Ly_new <= 0.0) boxbad = 1;
    Lx = Lx_new;
    Ly = Ly_new;
  }
  if (DMd == DM_PISTON) {
    // step_single_NPH_piston (src/md_env.cu:1939-1989)
    if (Lx_old <= 0.0 || Ly_old <= 0.0) boxbad = 1;
    const double a_old = (S->Fp - S->p_ext * Lx_old) / P.W;
    vp1 = S->vp + h * a_old;
    double Ly_new = Ly_old + dt * vp1;
    if (Ly_new < S->fl) {
      Ly_new = S->fl;
      clamped = 1;
      if (vp1 < 0.0) vp1 = 0.0;
    } else if (Ly_new > S->ce) {
      Ly_new = S->ce;
      clamped = 1;
      if (vp1 > 0.0) vp1 = 0.0;
    }
    Ly = Ly_new;
  }
  double fdt = 0.0, alpha = 0.0;
  int zero_v = 0;
  if (DMd == DM_FIRE) {
    fdt = S->f_dt;
    alpha = S->f_alpha;
    zero_v = S->f_zero_v;
  }
  double red[kNP];
#pragma unroll
  for (int k = 0; k < kNP; ++k) red[k] = 0.0;
  double mx[3] = {0.0, 0.0, 0.0};
  int bad = 0;
  const double ilx = 1.0 / Lx, ily = 1.0 / Ly;
  const double ilx_old = 1.0 / Lx_old, ily_old = 1.0 / Ly_old;
  const int items = P.items;
  // a block covers spb slots per pass (kThreads / lanes; the other threads
  // only join the reduction)
  const int spb = LN ? kThreads / P.lanes : kThreads;
  const int64_t base = P.p0 + (int64_t)(b - P.b0) * spb * items + threadIdx.x;
  const int64_t end = (!LN || (int)threadIdx.x < spb) ? P.p0 + P.n : 0;
  DriftCtx dc;
  dc.dt = dt;
  dc.h = h;
  dc.xi1 = xi1;
  dc.lam = lam;
  dc.vsc = vsc;
  dc.fdt = fdt;
  dc.alpha = alpha;
  dc.Lx = Lx;
  dc.Ly = Ly;
  dc.ilx = ilx;
  dc.ily = ily;
  dc.ilx_old = ilx_old;
  dc.ily_old = ily_old;
  dc.massA = P.massA;
  dc.massB = P.massB;
  dc.offx = P.offx;
  dc.offy = P.offy;
  dc.zero_v = zero_v;
  dc.py = py ? 1 : 0;
  if (!skip && !boxbad) {
#pragma unroll 1
    for (int it = 0; it < items; ++it) {
      const int64_t i = base + (int64_t)it * spb;
      if (i >= end) break;
      drift_particle<DMd>(D, dc, i, D.pos[i], D.vel[i], D.acc[i], D.type[i], D.sb[i], red[0],
                          mx[0], mx[1], mx[2], bad);
    }
  }
  if (bad) atomicOr(&S->nonfinite, 1);
  DriftTail tin;
  if (threadIdx.x == 0) tin = drift_tail_inputs(D, P, S);
  double tot[kNP];
  double tmx[3];
  if (!reduce_system<kNS, kNM>(D, P, S, red, mx, tot, tmx)) return;
  if (threadIdx.x != 0) return;
  int need = 0;
  if (!skip) {
    if (boxbad) {
      S->err = 5;  // MDB_ERR_BOX
    } else {
      if (DMd == DM_NH) {
        S->xi = nh_xi(dt, tin.g_dof, tin.T0, tin.Q, xi1, tot[0]);
      } else if (DMd == DM_NPH) {
        S->pA = pA1;
        S->aspect = aspect;
        S->Lx = Lx;
        S->Ly = Ly;
        S->clamped = clamped;
      } else if (DMd == DM_PISTON) {
        S->vp = vp1;
        S->Ly = Ly;
        S->clamped = clamped;
      }
      // Rebuild criterion. Cell stencil: a pair inside the cutoff now was
      // within one cell width (per axis) at the last rebuild while
      // 2*max displacement + rc_max stays below the current cell width.
      // Neighbour lists (radius rc_ij + skin at the last rebuild): with the
      // box scaled by f since then, a pair outside the list is still outside
      // rc while 2*max displacement < f*skin - max(0, 1-f)*rc_max.
      const double slop = 1e-3 + 4e-7 * fmax(Lx, Ly);
      const double wx = Lx / (double)tin.ncx;
      const double wy = (DMd == DM_PISTON) ? (tin.Ly_b / (double)tin.ncy) : Ly / (double)tin.ncy;
      const double fx = Lx / tin.Lx_b;
      const double fy = (DMd == DM_PISTON) ? 1.0 : Ly / tin.Ly_b;
      const double f = fmin(fx, fy);
      const double dmax = sqrt(tmx[0] * tmx[0] + tmx[1] * tmx[1]);
      if (!tin.allpairs) {
        if (2.0 * tmx[0] + slop + tin.rc_max >= wx) need = 1;
        if (2.0 * tmx[1] + slop + tin.rc_max >= wy) need = 1;
        if (2.0 * dmax + slop >= f * tin.skin - fmax(0.0, 1.0 - f) * tin.rc_max) need = 1;
        if (!(tmx[2] <= tin.skin)) need = 1;  // large single-step moves, NaN
      } else {
        need = (!(tmx[2] <= 0.25 * fmin(Lx, Ly))) ? 1 : 0;
      }
      if (need) {
        S->need_rebuild = 1;
        atomicOr(&D.bg->any_rebuild, 1);
      }
    }
  }
  S->counter = 0u;
  system_done_and_signal(D, tin.prior | need);
}

template <int DMd, bool LN>
__global__ void __launch_bounds__(kThreads, 4) k_drift(Dev D) {
  drift_phase<DMd, LN>(D, blockIdx.x);
}

// ------------------------------------------------------ multi-step kernel --
// A single system whose blocks are all resident at once (a cooperative
// launch) runs its steps in one kernel: drift phase, grid barrier, force
// phase, grid barrier, per step. The phases are the kernels' own block
// functions with the same blocks, so every sum has the same operands in the
// same order as with one launch per phase: the results are bit for bit those
// of the per-phase kernels. The kernel returns after the drift of a step that
// needs a rebuild; the graph around it rebuilds, runs that step's force phase
// and launches it again for the remaining steps.

// Polls of a grid-barrier wait before it gives up (at least 32 ns each).
constexpr unsigned kBarrierSpins = 1u << 22;

// Grid-wide barrier. Thread 0 of each block arrives on a counter; the last
// arrival resets it and advances the generation (release), the others poll
// the generation (acquire). A wait that runs out of polls records bar_err
// and returns; the kernel stops at its next check. That error is final for
// the handle: the kernel sets the system's err flag, after which every phase
// skips the system and every call reports it. Each call clears the arrival
// counter before its first launch (k_md_steps_set), so that a later call on
// such a handle passes its barriers and stops at once instead of waiting out
// the polls on arrivals that an abandoned barrier left behind.
__device__ __forceinline__ void grid_barrier(BatchGlobal* bg, unsigned nblocks) {
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned gen, prev;
    __threadfence();  // the block's writes (ordered before by the CTA barrier)
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(gen) : "l"(&bg->bar_gen) : "memory");
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;"
                 : "=r"(prev)
                 : "l"(&bg->bar_count)
                 : "memory");
    if (prev == nblocks - 1) {
      asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(&bg->bar_count), "r"(0u) : "memory");
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(&bg->bar_gen), "r"(gen + 1u)
                   : "memory");
    } else {
      unsigned cur = gen, polls = 0;
      do {
        __nanosleep(32);
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];"
                     : "=r"(cur)
                     : "l"(&bg->bar_gen)
                     : "memory");
      } while (cur == gen && ++polls < kBarrierSpins);
      if (cur == gen) atomicExch(&bg->bar_err, 1);
    }
    __threadfence();
  }
  __syncthreads();
}

__device__ __forceinline__ int ld_volatile(const int32_t* p) { return *(const volatile int32_t*)p; }

// Runs up to bg->steps_left steps of the single system (grid = its blocks).
// On return bg->steps_left holds the steps not finished (the step whose
// drift asked for a rebuild counts as not finished); h_rebuild is set when
// such a step is pending and h_more while steps remain.
// (Two blocks per SM: the drift and force phases in one kernel need more
// than the 64 registers of four, which spilled 270 B; the small systems it
// serves do not need the occupancy.)
template <int DMd, int FM, bool LN>
__global__ void __launch_bounds__(kThreads, 2)
    k_md_steps(Dev D, cudaGraphConditionalHandle h_more, cudaGraphConditionalHandle h_rebuild) {
  BatchGlobal* bg = D.bg;
  const unsigned nb = gridDim.x;
  const int64_t todo = *(const volatile int64_t*)&bg->steps_left;
  int64_t done = 0;
  int rebuild = 0, err = 0;
  while (done < todo) {
    drift_phase<DMd, LN>(D, blockIdx.x);
    grid_barrier(bg, nb);
    if (ld_volatile(&bg->bar_err)) {
      err = 1;
      break;
    }
    if (ld_volatile(&bg->any_rebuild)) {
      rebuild = 1;
      break;
    }
    force_phase<FM, true, false, LN>(D, blockIdx.x);
    grid_barrier(bg, nb);
    if (ld_volatile(&bg->bar_err)) {
      err = 1;
      break;
    }
    ++done;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int64_t left = todo - done;
    bg->steps_left = left;
    if (err) D.st->err = 6;  // MDB_ERR_CUDA: a barrier wait gave up
    cudaGraphSetConditional(h_rebuild, (rebuild && !err) ? 1u : 0u);
    cudaGraphSetConditional(h_more, (left > 0 && !err) ? 1u : 0u);
  }
}

// After the rebuild and the force phase of the pending step.
__global__ void k_md_steps_count(Dev D, cudaGraphConditionalHandle h_more) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int64_t left = D.bg->steps_left - 1;
  D.bg->steps_left = left;
  cudaGraphSetConditional(h_more, left > 0 ? 1u : 0u);
}

__global__ void k_md_steps_set(Dev D, int64_t n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    D.bg->steps_left = n;
    D.bg->bar_count = 0u;  // no multi-step block runs now (stream order)
  }
}

// K = sum 1/2 m |v|^2 (cal_local_K_kernel src/md_cuda_common.cu:554-589) into
// S.K for every system.
__global__ void __launch_bounds__(kThreads) k_reduce_K(Dev D) {
  const int b = blockIdx.x;
  // (a lone system needs no table lookup: one dependent load less per block)
  const int s = D.nsys == 1 ? 0 : D.sys_of_block[b];
  const SysParams& P = D.sp[s];
  SysState* S = D.st + s;
  constexpr int kNS = 1, kNM = 0;
  double red[kNP];
#pragma unroll
  for (int k = 0; k < kNP; ++k) red[k] = 0.0;
  double mx[3] = {0.0, 0.0, 0.0};
  const int spb = kThreads / P.lanes;
  const int64_t base = P.p0 + (int64_t)(b - P.b0) * spb * P.items + threadIdx.x;
  for (int it = 0; it < P.items && (int)threadIdx.x < spb; ++it) {
    const int64_t i = base + (int64_t)it * spb;
    if (i >= P.p0 + P.n) break;
    const double2 v = D.vel[i];
    const double m = type_mass(P, D.type[i]);
    red[0] += (0.5 * m) * fma(v.x, v.x, v.y * v.y);
  }
  double tot[kNP];
  double tmx[3];
  if (!reduce_system<kNS, kNM>(D, P, S, red, mx, tot, tmx)) return;
  if (threadIdx.x != 0) return;
  S->K = tot[0];
  S->counter = 0u;
}

// ------------------------------------------------------ cell-list rebuild --
// All rebuild kernels are grid-stride with a fixed grid and return at once
// when no system asked for a rebuild (the eager path launches them every step;
// the graph path puts them behind a conditional node).

__device__ __forceinline__ bool rebuild_requested(const Dev& D) {
  return *((volatile int*)&D.bg->any_rebuild) != 0;
}

// System owning global cell c (cells of system s are [c0_s, c0_s + ccap_s)).
__device__ __forceinline__ int cell_system(const Dev& D, int64_t c) {
  int lo = 0, hi = D.nsys - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (D.sp[mid].c0 <= c) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ bool sys_rebuilds(const Dev& D, int s) {
  return *((volatile int*)&D.st[s].need_rebuild) != 0;
}

// Zero the cell counters of every system that rebuilds and compute its grid
// for the current box. Systems that do not rebuild keep their counts, so the
// global scan reproduces their cell ranges unchanged.
__global__ void k_rb_zero(Dev D) {
  if (!rebuild_requested(D)) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int64_t c = tid; c < D.ncells; c += stride) {
    if (!sys_rebuilds(D, cell_system(D, c))) continue;
    D.ccount[c] = 0;
    D.ccursor[c] = 0;
  }
  for (int64_t s = tid; s < D.nsys; s += stride) {
    if (!sys_rebuilds(D, (int)s)) continue;
    const SysParams& P = D.sp[s];
    SysState* S = D.st + s;
    const double Lx = S->Lx, Ly = S->Ly;
    const int ncx = grid_n(Lx, P.r_cell, P.ccap_x);
    const int ncy = grid_n(Ly, P.r_cell, P.ccap_y);
    S->ncx = ncx;
    S->ncy = ncy;
    S->allpairs = (ncx < 3 || (S->periodic_y && ncy < 3)) ? 1 : 0;
    S->inv_wx = (double)ncx / Lx;
    S->inv_wy = (double)ncy / Ly;
    S->Lx_b = Lx;
    S->Ly_b = Ly;
    S->nl_overflow = 0;
  }
}

__global__ void k_rb_bin(Dev D) {
  if (!rebuild_requested(D)) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D.ntot; i += stride) {
    const int s = D.sysid[i];
    if (!sys_rebuilds(D, s)) continue;
    const SysState* S = D.st + s;
    const double2 p = D.pos[i];
    const int ncx = S->ncx, ncy = S->ncy;
    const int cx = bin_axis(p.x * S->inv_wx, ncx);
    const int cy = bin_axis(p.y * S->inv_wy, ncy);
    const int key = (int)(D.sp[s].c0 + (int64_t)cy * ncx + cx);
    D.key[i] = key;
    atomicAdd(D.ccount + key, 1);
  }
}

// Exclusive scan of ccount into cstart: per-tile scan, scan of tile sums,
// add. cstart[ncells] receives the total.
__global__ void __launch_bounds__(kScanBlock) k_scan_tiles(Dev D) {
  if (!rebuild_requested(D)) return;
  __shared__ int sh[kScanBlock / 32];
  const int64_t ntiles = (D.ncells + kScanTile - 1) / kScanTile;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t base = tile * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int v[kScanItems];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      v[k] = (base + k < D.ncells) ? D.ccount[base + k] : 0;
      sum += v[k];
    }
    // block exclusive scan of per-thread sums
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
      int t = lane < kScanBlock / 32 ? sh[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += y;
      }
      if (lane < kScanBlock / 32) sh[lane] = t;
    }
    __syncthreads();
    int run = x - sum + (w > 0 ? sh[w - 1] : 0);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      if (base + k < D.ncells) D.cstart[base + k] = run;
      run += v[k];
    }
    if (threadIdx.x == kScanBlock - 1) D.scan_part[tile] = run;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(1024) k_scan_parts(Dev D) {
  if (!rebuild_requested(D)) return;
  __shared__ int sh[32];
  __shared__ int carry;
  const int64_t ntiles = (D.ncells + kScanTile - 1) / kScanTile;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < ntiles; base += 1024) {
    const int64_t k = base + threadIdx.x;
    const int v = k < ntiles ? D.scan_part[k] : 0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
      int t = sh[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, t, o);
        if (lane >= o) t += y;
      }
      sh[lane] = t;
    }
    __syncthreads();
    const int excl = x - v + (w > 0 ? sh[w - 1] : 0) + carry;
    __syncthreads();
    if (k < ntiles) D.scan_part[k] = excl;
    if (threadIdx.x == 1023) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) D.cstart[D.ncells] = carry;
}

__global__ void k_scan_add(Dev D) {
  if (!rebuild_requested(D)) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < D.ncells; c += stride)
    D.cstart[c] += D.scan_part[c / kScanTile];
}

__global__ void k_rb_scatter(Dev D) {
  if (!rebuild_requested(D)) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D.ntot; i += stride) {
    if (!sys_rebuilds(D, D.sysid[i])) continue;
    const int key = D.key[i];
    const int slot = D.cstart[key] + atomicAdd(D.ccursor + key, 1);
    D.perm[slot] = (int)i;
  }
}

// Within a cell the scatter order is arbitrary; sorting each cell's slots by
// source slot makes the permutation the stable sort by cell.
__global__ void k_rb_cellsort(Dev D) {
  if (!rebuild_requested(D)) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < D.ncells; c += stride) {
    if (!sys_rebuilds(D, cell_system(D, c))) continue;
    const int a = D.cstart[c], e = D.cstart[c + 1];
    for (int k = a + 1; k < e; ++k) {
      const int v = D.perm[k];
      int q = k - 1;
      while (q >= a && D.perm[q] > v) {
        D.perm[q + 1] = D.perm[q];
        --q;
      }
      D.perm[q + 1] = v;
    }
  }
}

__global__ void k_rb_permute(Dev D) {
  if (!rebuild_requested(D)) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < D.ntot; k += stride) {
    const int s = D.sysid[k];
    if (!sys_rebuilds(D, s)) continue;
    const int src = D.perm[k];
    const SysParams& P = D.sp[s];
    const SysState* S = D.st + s;
    const double2 p = D.pos[src];
    const int t = D.type[src];
    D.pos2[k] = p;
    D.vel2[k] = D.vel[src];
    D.acc2[k] = D.acc[src];
    D.type2[k] = t;
    D.theta2[k] = D.theta[src];
    D.orig2[k] = D.orig[src];
    D.cell_of[k] = (int)(D.key[src] - P.c0);
    D.pff[k] = encode_ff(p.x, p.y, t, P.offx, P.offy);
    const float sx = (float)(p.x * (1.0 / S->Lx));
    const float sy = S->periodic_y ? (float)(p.y * (1.0 / S->Ly)) : (float)p.y;
    D.sb[k] = make_float2(sx, sy);
  }
}

__global__ void k_rb_copyback(Dev D) {
  if (!rebuild_requested(D)) return;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < D.ntot; k += stride) {
    if (!sys_rebuilds(D, D.sysid[k])) continue;
    D.pos[k] = D.pos2[k];
    D.vel[k] = D.vel2[k];
    D.acc[k] = D.acc2[k];
    D.type[k] = D.type2[k];
    D.theta[k] = D.theta2[k];
    D.orig[k] = D.orig2[k];
  }
}

// Verlet list of one slot: the 3x3 stencil candidates within the list radius
// (rc_ij + skin), same displacement arithmetic as the force loop. MIC = false
// for interior cells (two or more cells from every periodic edge): the
// stencil does not wrap, so the nearest image is the plain difference.
template <bool PY, bool MIC>
__device__ __forceinline__ int build_list(const Dev& D, const SysParams& P, const SysState& S,
                                          int64_t k, int& nowrap) {
  PairCtx c;
  const float4 qi = D.pff[k];
  set_pair_box<PY>(c, qi, S.Lx, S.Ly);
  const uint32_t tci = ff_class(qi);
  const uint32_t ts = (tci == 2u) ? 99u : tci;
  const float rl2s = P.frl2[tci == 2u ? 2 : tci], rl2ab = P.frl2[2];
  const int ncx = S.ncx, ncy = S.ncy;
  const int cell = D.cell_of[k];
  const int cx = cell % ncx, cy = cell / ncx;
  int cnt = 0;
  const int maxn = D.max_nbr;
  const int half = (P.n + 1) / 2;
  nowrap = 1;
  for (int dr = -1; dr <= 1; ++dr) {
    int yy = cy + dr;
    if (PY) {
      if (yy < 0) yy += ncy;
      if (yy >= ncy) yy -= ncy;
    } else if (yy < 0 || yy >= ncy) {
      continue;
    }
    const int64_t row = P.c0 + (int64_t)yy * ncx;
    int r0[2], r1[2], nr;
    if (cx > 0 && cx < ncx - 1) {
      r0[0] = D.cstart[row + cx - 1];
      r1[0] = D.cstart[row + cx + 2];
      nr = 1;
    } else if (cx == 0) {
      r0[0] = D.cstart[row];
      r1[0] = D.cstart[row + 2];
      r0[1] = D.cstart[row + ncx - 1];
      r1[1] = D.cstart[row + ncx];
      nr = 2;
    } else {
      r0[0] = D.cstart[row + ncx - 2];
      r1[0] = D.cstart[row + ncx];
      r0[1] = D.cstart[row];
      r1[1] = D.cstart[row + 1];
      nr = 2;
    }
    // visit(j, q): false when the list must give up (16-bit offsets overflow)
    auto visit = [&](int j, const float4 q) -> bool {
      if (j == k) return true;
      float2 dd;
      const float r2 = pair_r2<MIC>(q, c, dd);
      const float rl2 = (ff_class(q) == ts) ? rl2s : rl2ab;
      if (r2 < rl2) {
        int d = j - (int)k;  // offset modulo n into [-n/2, n/2)
        if (d >= half) {
          d -= P.n;
          nowrap = 0;
        }
        if (d < -half) {
          d += P.n;
          nowrap = 0;
        }
        if (D.nl16 && (d > 32767 || d < -32768)) return false;
        if (cnt < maxn) {
          if (D.nl16)
            D.nlist16[(int64_t)cnt * D.ntot + k] = (int16_t)d;
          else
            D.nlist[(int64_t)cnt * D.ntot + k] = d;
        }
        ++cnt;
      }
      return true;
    };
    for (int r = 0; r < nr; ++r) {
      int j = r0[r];
      const int je = r1[r];
      // four candidates' positions in flight at a time
      for (; j + 4 <= je; j += 4) {
        float4 qq[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) qq[u] = D.pff[j + u];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (!visit(j + u, qq[u])) return maxn + 1;  // use the stencil
      }
      for (; j < je; ++j)
        if (!visit(j, D.pff[j])) return maxn + 1;
    }
  }
  return cnt;
}

// Steps (MD) or iterations (FIRE) the system has run: the clock of its
// rebuild history.
__device__ __forceinline__ int64_t rebuild_clock(const SysParams& P, const SysState& S) {
  return P.kind == K_FIRE ? (int64_t)S.f_step : S.steps;
}

__global__ void k_rb_nlist(Dev D) {
  if (!rebuild_requested(D)) return;
  const bool forced = *((volatile int*)&D.bg->forced) != 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < D.ntot; k += stride) {
    const int s = D.sysid[k];
    if (!sys_rebuilds(D, s)) continue;
    const SysParams& P = D.sp[s];
    SysState* S = D.st + s;
    // a system that rebuilds again within kListMinReuse steps scans its cell
    // stencil instead of a list it would hardly reuse
    const bool recent = !forced && rebuild_clock(P, *S) - S->rb_last < kListMinReuse;
    if (S->allpairs || D.max_nbr <= 0 || recent) {
      D.ncount[k] = -1;
      continue;
    }
    // Interior build cells (two or more cells from each periodic edge) with
    // unwrapped offsets: the partners were binned one cell away at most and
    // move less than half a cell before the next rebuild, so no pair needs
    // the minimum image and j = k + offset directly.
    const int cell = D.cell_of[k];
    const int cx = cell % S->ncx, cy = cell / S->ncx;
    const bool interior = cx >= 2 && cx <= S->ncx - 3 &&
                          (!S->periodic_y || (cy >= 2 && cy <= S->ncy - 3));
    int nowrap = 0;
    int cnt;
    if (S->periodic_y)
      cnt = interior ? build_list<true, false>(D, P, *S, k, nowrap)
                     : build_list<true, true>(D, P, *S, k, nowrap);
    else
      cnt = interior ? build_list<false, false>(D, P, *S, k, nowrap)
                     : build_list<false, true>(D, P, *S, k, nowrap);
    if (cnt > D.max_nbr) {
      D.ncount[k] = -1;  // too many neighbours: the force loop scans the stencil
      atomicAdd(&S->nl_overflow, 1);
      continue;
    }
    D.ncount[k] = cnt | ((interior && nowrap) ? kListInterior : 0);
  }
}

__global__ void k_rb_finish(Dev D) {
  if (!rebuild_requested(D)) return;
  const bool forced = *((volatile int*)&D.bg->forced) != 0;
  for (int s = threadIdx.x; s < D.nsys; s += blockDim.x) {
    SysState* S = D.st + s;
    if (!S->need_rebuild) continue;
    S->need_rebuild = 0;
    S->dmax_x = 0u;
    S->dmax_y = 0u;
    S->jump = 0u;
    S->rebuilds += 1;
    S->rb_last = forced ? kNoRebuildYet : rebuild_clock(D.sp[s], *S);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    D.bg->any_rebuild = 0;
    D.bg->forced = 0;
  }
}

// ------------------------------------------------------------ profiles --
// get_N_profile / get_pressure_profile (src/md_cuda_common.cu:827-1030) for
// system s: per-type counts in x bins, and the Irving-Kirkwood pressure
// tensor in y bins (kinetic m v_a v_b at the bin of y_i, pair 1/2 r_a F_b at
// the bin of the minimum-image midpoint y_i - dy/2). Pairs come from the cell
// stencil of the last rebuild (exact while the rebuild criterion holds).
// Sums are fixed point (2^-24) in 64-bit integers, so atomics give the same
// result in any order.
constexpr double kProfileFix = 16777216.0;

__device__ __forceinline__ int profile_bin(double y, double Ly, int nb, bool py) {
  double yy = py ? pbc_wrap(y, Ly) : y;
  if (!py) {
    if (yy < 0.0)
      yy = 0.0;
    else if (yy >= Ly && Ly > 0.0)
      yy = Ly * (1.0 - 1e-12);
  }
  const double t = (Ly > 0.0) ? (yy / Ly) : 0.0;
  int b = (int)(t * (double)nb);
  return b < 0 ? 0 : (b >= nb ? nb - 1 : b);
}

__device__ __forceinline__ void fix_add(unsigned long long* a, double v) {
  atomicAdd(a, (unsigned long long)__double2ll_rn(v * kProfileFix));
}

template <bool PY>
__global__ void __launch_bounds__(kThreads) k_profiles(Dev D, int s, int nb,
                                                       unsigned long long* ptens, int* counts) {
  const SysParams& P = D.sp[s];
  const SysState& S = D.st[s];
  const double Lx = S.Lx, Ly = S.Ly;
  PairCtx c;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < P.n; k += stride) {
    const int64_t i = P.p0 + k;
    const double2 p = D.pos[i];
    const double2 v = D.vel[i];
    const int ti = D.type[i];
    if (p.x >= 0.0 && p.x <= Lx) {
      int b = (int)(p.x / Lx * nb);
      b = b < 0 ? 0 : (b >= nb ? nb - 1 : b);
      atomicAdd(counts + (ti == 0 ? 0 : nb) + b, 1);
    }
    const double m = type_mass(P, ti);
    const int bk = profile_bin(p.y, Ly, nb, PY);
    fix_add(ptens + bk, m * v.x * v.x);
    fix_add(ptens + nb + bk, m * v.y * v.y);
    fix_add(ptens + 2 * nb + bk, m * v.x * v.y);
    const float4 qi = D.pff[i];
    set_pair_box<PY>(c, qi, Lx, Ly);
    set_profile_class(c, P, type_class(ti));
    // candidate ranges: the whole system, or the 3x3 stencil
    int r0[6], r1[6], nr = 0;
    if (S.allpairs) {
      r0[0] = (int)P.p0;
      r1[0] = (int)(P.p0 + P.n);
      nr = 1;
    } else {
      const int ncx = S.ncx, ncy = S.ncy;
      const int cell = D.cell_of[i];
      const int cx = cell % ncx, cy = cell / ncx;
      for (int dr = -1; dr <= 1; ++dr) {
        int yy = cy + dr;
        if (PY) {
          if (yy < 0) yy += ncy;
          if (yy >= ncy) yy -= ncy;
        } else if (yy < 0 || yy >= ncy) {
          continue;
        }
        const int64_t row = P.c0 + (int64_t)yy * ncx;
        if (cx > 0 && cx < ncx - 1) {
          r0[nr] = D.cstart[row + cx - 1];
          r1[nr++] = D.cstart[row + cx + 2];
        } else if (cx == 0) {
          r0[nr] = D.cstart[row];
          r1[nr++] = D.cstart[row + 2];
          r0[nr] = D.cstart[row + ncx - 1];
          r1[nr++] = D.cstart[row + ncx];
        } else {
          r0[nr] = D.cstart[row + ncx - 2];
          r1[nr++] = D.cstart[row + ncx];
          r0[nr] = D.cstart[row];
          r1[nr++] = D.cstart[row + 1];
        }
      }
    }
    for (int r = 0; r < nr; ++r) {
      for (int j = r0[r]; j < r1[r]; ++j) {
        if (j == i) continue;
        const float4 q = D.pff[j];
        float2 dd;
        const float r2 = pair_r2<true>(q, c, dd);
        const float dx = dd.x, dy = dd.y;
        const bool same = (ff_class(q) == c.ts);
        const float rc2 = same ? c.rc2s : c.rc2ab;
        if (!(r2 > 0.0f && r2 < rc2)) continue;
        const float sig2 = same ? c.sig2s : c.sig2ab;
        const float e24 = same ? c.e24s : c.e24ab;
        const float r2i = 1.0f / r2;
        const float sr2 = sig2 * r2i;
        const float sr6 = sr2 * sr2 * sr2;
        const float sr12 = sr6 * sr6;
        const float tmp = e24 * fmaf(2.0f, sr12, -sr6) * r2i;
        const double ddx = (double)dx, ddy = (double)dy;
        const double Fx = (double)(tmp * dx), Fy = (double)(tmp * dy);
        const int bp = profile_bin(p.y - 0.5 * ddy, Ly, nb, PY);
        fix_add(ptens + bp, 0.5 * ddx * Fx);
        fix_add(ptens + nb + bp, 0.5 * ddy * Fy);
        fix_add(ptens + 2 * nb + bp, 0.5 * ddx * Fy);
      }
    }
  }
}

// ------------------------------------------------------------ frame I/O --
struct DevParticle {  // include/md_particle.hpp:31-38 (64 bytes)
  double2 pos, vel, acc;
  int32_t type, pad;
  double theta;
};

__global__ void k_import(Dev D, const DevParticle* __restrict__ in, int64_t p0, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
    const DevParticle q = in[k];
    const int64_t slot = p0 + k;
    D.pos[slot] = q.pos;
    D.vel[slot] = q.vel;
    D.acc[slot] = q.acc;
    D.type[slot] = q.type;
    D.theta[slot] = q.theta;
    D.orig[slot] = (int32_t)k;
  }
}

// Wraps every position into the box (FIRE initialize_from_frame,
// src/md_energy_minimizer.cu:386-419) and zeroes v and a when asked.
__global__ void k_fire_prepare(Dev D, int64_t p0, int64_t n, int s) {
  const SysState* S = D.st + s;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
    const int64_t slot = p0 + k;
    double2 p = D.pos[slot];
    p.x = pbc_wrap(p.x, S->Lx);
    p.y = pbc_wrap(p.y, S->Ly);
    D.pos[slot] = p;
    D.vel[slot] = make_double2(0.0, 0.0);
    D.acc[slot] = make_double2(0.0, 0.0);
  }
}

__global__ void k_export(Dev D, DevParticle* __restrict__ out, int64_t p0, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
    const int64_t slot = p0 + k;
    DevParticle q;
    q.pos = D.pos[slot];
    q.vel = D.vel[slot];
    q.acc = D.acc[slot];
    q.type = D.type[slot];
    q.pad = 0;
    q.theta = D.theta[slot];
    out[D.orig[slot]] = q;
  }
}

// mdb_sim_observables of system s from its device state into a staging slot.
__global__ void k_observables(Dev D, int s, double t, int piston_active,
                              mdb_observables_t* out) {
  const SysParams& P = D.sp[s];
  const SysState& S = D.st[s];
  mdb_observables_t o;
  memset(&o, 0, sizeof(o));
  o.t = t;
  o.Lx = S.Lx;
  o.Ly = S.Ly;
  o.xi = S.xi;
  o.last_instant_pressure = S.last_P;
  o.nph_area_momentum = S.pA;
  o.nph_area_rate = S.pA / P.W;
  o.nph_piston_velocity = S.vp;
  o.nph_piston_force = S.Fp;
  o.n = P.n;
  o.steps = S.steps;
  o.rebuilds = S.rebuilds;
  o.piston_mode_active = piston_active;
  o.nonfinite = S.nonfinite;
  *out = o;
}

// Rebuild flag for every system (creation, frame import, mode switches).
__global__ void k_force_rebuild(Dev D, int periodic_y) {
  for (int s = threadIdx.x; s < D.nsys; s += blockDim.x) {
    D.st[s].need_rebuild = 1;
    if (periodic_y >= 0) D.st[s].periodic_y = periodic_y;
  }
  if (threadIdx.x == 0) {
    D.bg->any_rebuild = 1;
    D.bg->forced = 1;
  }
}

__global__ void k_set_pext(Dev D, double p) {
  for (int s = threadIdx.x; s < D.nsys; s += blockDim.x) D.st[s].p_ext = p;
}

}  // namespace mdb
