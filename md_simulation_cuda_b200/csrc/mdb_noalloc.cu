// mdb_compute_forces_noalloc: the pair force / energy / virial evaluation of
// mdb_compute_forces for callers that cannot allocate device memory.
//
// Who cannot allocate, and why: hosts that own every byte of device memory
// through their own pool (a framework's caching allocator, a plugin host with
// a fixed budget) and forbid plugins from calling cudaMalloc behind their
// back; and loops that must not stall other streams, since cudaMalloc and
// cudaFree may synchronise the whole device. Such callers hand in device
// buffers they already own and a stream; this entry point issues kernels on
// that stream and allocates nothing.
//
// Scratch: everything the evaluation needs beyond its inputs and outputs (the
// cell binning, the per-cell particle lists, the block partial sums and the
// arrival counter of the last-block reduction) lives in one file-scope
// device array of 1 MiB, g_noalloc_scratch. That fixes the maximum size:
// MDB_NOALLOC_MAX_PARTICLES particles, and at most 128 x 128 cells (larger
// boxes use wider cells, which stays exact). The first call on each device
// looks the array's address up with cudaGetSymbolAddress while that device
// is current; make that first call before any stream capture. The address is
// remembered together with the CUDA context it belongs to: after a
// cudaDeviceReset, or with another context current on the device, the next
// call looks it up again instead of using a stale address.
//
// Cost: the order inside a cell is each particle's rank among the cell's
// indices, found by a scan of the cell, so a cell holding m particles costs
// m^2 comparisons. Ordinary frames hold a few particles per cell; a frame
// with all particles in a few cells (clustered input, or non-finite positions,
// which all bin to cell 0) costs up to n^2, about 4e9 comparisons (seconds)
// at n = 65536.
//
// Every call on a device shares the one array: each call first clears the
// parts that must start at zero (the per-cell counts and the arrival counter)
// on its stream, so consecutive calls on one stream, or on streams ordered by
// events, are independent. Calls whose kernels overlap on the GPU (two host
// threads, or two unordered streams, on one device) race on the array and
// produce wrong results.
//
// Arithmetic: FP64 minimum-image differences, FP32 pair terms with the
// truncated force and the shifted energy of the other force paths, FP64
// accumulation in a fixed order (cells in stencil order, particles in index
// order inside a cell), so a call is deterministic.
#include <cuda.h>
#include <cuda_runtime.h>
#include <math.h>

#include <mutex>

#include "mdb200.h"
#include "mdb_util.h"

namespace mdb {
namespace {

constexpr int kNaThreads = 256;
constexpr int kNaMaxN = MDB_NOALLOC_MAX_PARTICLES;
constexpr int kNaCellAxis = 128;
constexpr int kNaMaxCells = kNaCellAxis * kNaCellAxis;
constexpr int kNaMaxBlocks = kNaMaxN / kNaThreads;
constexpr int kNaScanThreads = 1024;

// Byte offsets of the scratch regions (each 256-byte aligned).
constexpr size_t kOffCell = 0;                                   // int32[kNaMaxN]
constexpr size_t kOffTmp = kOffCell + 4 * (size_t)kNaMaxN;       // int32[kNaMaxN]
constexpr size_t kOffIdx = kOffTmp + 4 * (size_t)kNaMaxN;        // int32[kNaMaxN]
constexpr size_t kOffCount = kOffIdx + 4 * (size_t)kNaMaxN;      // int32[kNaMaxCells]
constexpr size_t kOffStart = kOffCount + 4 * (size_t)kNaMaxCells;  // int32[kNaMaxCells + 1]
constexpr size_t kOffPart = (kOffStart + 4 * (size_t)(kNaMaxCells + 1) + 255) / 256 * 256;
constexpr size_t kOffCounter = kOffPart + 16 * (size_t)kNaMaxBlocks;  // uint32
constexpr size_t kScratchBytes = 1u << 20;
static_assert(kOffCounter + 256 <= kScratchBytes, "scratch regions exceed the array");

}  // namespace

// The scratch array shared by every call on a device (1 MiB).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

struct NaGrid {
  double Lx, Ly, sx, sy;  // sx = ncx / Lx, sy = ncy / Ly
  int ncx, ncy, ncells, py;
};

struct NaPair {
  float rc2[3], sig2[3], e24[3], e4[3];  // AA, BB, AB
  double Vc[3];
  double massA, massB;
};

struct NaScratch {
  int32_t* cell_of;
  int32_t* tmp;
  int32_t* idx;
  int32_t* count;
  int32_t* start;
  double* part;
  unsigned int* counter;
};

__device__ __forceinline__ int na_bin(double v, int n) {
  if (v >= 0.0 && v < (double)n) return (int)v;
  if (v >= (double)n) return n - 1;
  return 0;  // negative or NaN
}

__device__ __forceinline__ int na_cell(double x, double y, const NaGrid& g) {
  const double xw = x - floor(x / g.Lx) * g.Lx;
  const double yw = g.py ? y - floor(y / g.Ly) * g.Ly : y;
  return na_bin(yw * g.sy, g.ncy) * g.ncx + na_bin(xw * g.sx, g.ncx);
}

__device__ __forceinline__ int na_class(int t) { return t == 0 ? 0 : (t == 1 ? 1 : 2); }

// v[k] for a pair class k in {0, 1, 2} by selects (no local-memory copy).
template <typename T>
__device__ __forceinline__ T na_sel(const T (&v)[3], int k) {
  return k == 0 ? v[0] : (k == 1 ? v[1] : v[2]);
}

// Zero the per-cell counts and the arrival counter.
__global__ void k_na_clear(NaScratch s, int ncells) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncells) s.count[c] = 0;
  if (c == 0) *s.counter = 0u;
}

__global__ void k_na_bin(const double* __restrict__ pos, int n, NaGrid g, NaScratch s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = na_cell(pos[2 * i], pos[2 * i + 1], g);
  s.cell_of[i] = c;
  atomicAdd(s.count + c, 1);
}

// Exclusive scan of the counts into start[0..ncells]; resets the counts to
// zero for use as fill cursors.
__global__ void __launch_bounds__(kNaScanThreads) k_na_scan(NaScratch s, int ncells, int n) {
  __shared__ int sh[kNaScanThreads];
  const int per = (ncells + kNaScanThreads - 1) / kNaScanThreads;
  const int c0 = threadIdx.x * per;
  int tot = 0;
  for (int k = 0; k < per; ++k)
    if (c0 + k < ncells) tot += s.count[c0 + k];
  sh[threadIdx.x] = tot;
  __syncthreads();
  for (int off = 1; off < kNaScanThreads; off <<= 1) {
    const int v = threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
    __syncthreads();
    sh[threadIdx.x] += v;
    __syncthreads();
  }
  int run = sh[threadIdx.x] - tot;
  for (int k = 0; k < per; ++k) {
    const int c = c0 + k;
    if (c < ncells) {
      s.start[c] = run;
      run += s.count[c];
      s.count[c] = 0;
    }
  }
  if (threadIdx.x == 0) s.start[ncells] = n;
}

// Unordered fill of each cell's slot range.
__global__ void k_na_fill(int n, NaScratch s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = s.cell_of[i];
  s.tmp[s.start[c] + atomicAdd(s.count + c, 1)] = i;
}

// Deterministic order: particle i goes to its rank among its cell's indices.
__global__ void k_na_rank(int n, NaScratch s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = s.cell_of[i];
  const int a = s.start[c], b = s.start[c + 1];
  int r = 0;
  for (int k = a; k < b; ++k) r += (s.tmp[k] < i) ? 1 : 0;
  s.idx[a + r] = i;
}

__device__ __forceinline__ void na_range(const double* __restrict__ pos,
                                         const int32_t* __restrict__ type, const NaGrid& g,
                                         const NaPair& p, const NaScratch& s, int i, double xi,
                                         double yi, int ci, int a, int b, double& fx, double& fy,
                                         double& u, double& w) {
  for (int k = a; k < b; ++k) {
    const int j = s.idx[k];
    if (j == i) continue;
    double dx = xi - pos[2 * j];
    double dy = yi - pos[2 * j + 1];
    dx -= g.Lx * rint(dx / g.Lx);
    if (g.py) dy -= g.Ly * rint(dy / g.Ly);
    const float dxf = (float)dx, dyf = (float)dy;
    const float r2 = dxf * dxf + dyf * dyf;
    const int cj = na_class(type[j]);
    const int pc = (ci == cj && ci != 2) ? ci : 2;
    if (r2 < na_sel(p.rc2, pc) && r2 > 0.0f) {
      const float r2i = 1.0f / r2;
      const float sr2 = na_sel(p.sig2, pc) * r2i;
      const float sr6 = sr2 * sr2 * sr2;
      const float sr12 = sr6 * sr6;
      const float t = na_sel(p.e24, pc) * fmaf(2.0f, sr12, -sr6) * r2i;
      fx += (double)(t * dxf);
      fy += (double)(t * dyf);
      w += (double)(t * r2);
      u = fma(0.5, (double)(na_sel(p.e4, pc) * (sr12 - sr6)) - na_sel(p.Vc, pc), u);
    }
  }
}

// One thread per particle: stencil of the particle's cell (3x3, or one cell
// along an axis with a single cell), acceleration, and the deterministic
// last-block sum of U and W = 1/2 sum r.F into uw[0..1].
__global__ void __launch_bounds__(kNaThreads) k_na_force(const double* __restrict__ pos,
                                                         const int32_t* __restrict__ type, int n,
                                                         NaGrid g, NaPair p, NaScratch s,
                                                         double* __restrict__ acc,
                                                         double* __restrict__ uw) {
  __shared__ double su[kNaThreads], sw[kNaThreads];
  __shared__ bool last;
  const int i = blockIdx.x * kNaThreads + threadIdx.x;
  double u = 0.0, w = 0.0;
  if (i < n) {
    const double xi = pos[2 * i], yi = pos[2 * i + 1];
    const int ti = type[i];
    const int ci = na_class(ti);
    const int cell = s.cell_of[i];
    const int cx = cell % g.ncx, cy = cell / g.ncx;
    const int rx = g.ncx >= 3 ? 1 : 0;
    const int ry = (!g.py || g.ncy >= 3) ? 1 : 0;
    double fx = 0.0, fy = 0.0;
    for (int dr = -ry; dr <= ry; ++dr) {
      int yy = cy + dr;
      if (g.py) {
        yy += (yy < 0) ? g.ncy : 0;
        yy -= (yy >= g.ncy) ? g.ncy : 0;
      } else if (yy < 0 || yy >= g.ncy) {
        continue;
      }
      for (int dc = -rx; dc <= rx; ++dc) {
        int xx = cx + dc;
        xx += (xx < 0) ? g.ncx : 0;
        xx -= (xx >= g.ncx) ? g.ncx : 0;
        const int c = yy * g.ncx + xx;
        na_range(pos, type, g, p, s, i, xi, yi, ci, s.start[c], s.start[c + 1], fx, fy, u, w);
      }
    }
    const double m = ti == 0 ? p.massA : p.massB;
    acc[2 * i] = fx / m;
    acc[2 * i + 1] = fy / m;
  }
  su[threadIdx.x] = u;
  sw[threadIdx.x] = w;
  __syncthreads();
  for (int h = kNaThreads / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) {
      su[threadIdx.x] += su[threadIdx.x + h];
      sw[threadIdx.x] += sw[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    s.part[2 * blockIdx.x] = su[0];
    s.part[2 * blockIdx.x + 1] = sw[0];
    __threadfence();
    last = (atomicAdd(s.counter, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  double U = 0.0, W = 0.0;
  for (unsigned b = 0; b < gridDim.x; ++b) {
    U += __ldcg(s.part + 2 * b);
    W += __ldcg(s.part + 2 * b + 1);
  }
  uw[0] = U;
  uw[1] = 0.5 * W;
  *s.counter = 0u;
}

std::mutex g_setup_mu;
constexpr int kMaxDevices = 64;
struct ScratchAddr {
  CUcontext ctx = nullptr;
  unsigned char* ptr = nullptr;
};
ScratchAddr g_scratch[kMaxDevices];  // guarded by g_setup_mu

// cuCtxGetCurrent through the runtime's driver entry point (no link against
// the driver library).
using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrentFn>(f);
  }();
  return fn;
}

// Once per device and context, with that device current: the device address
// of the scratch array.
int scratch_for_device(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices)
    return set_error(MDB_ERR_ARG, "mdb_compute_forces_noalloc: device ordinal out of range");
  CtxGetCurrentFn get = ctx_get_current();
  CUcontext ctx = nullptr;
  if (!get || get(&ctx) != CUDA_SUCCESS)
    return set_error(MDB_ERR_CUDA, "mdb_compute_forces_noalloc: cuCtxGetCurrent failed");
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!ctx) {
    // no context yet on this thread: the runtime's first call makes the
    // device's primary context current
    void* addr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    if (get(&ctx) != CUDA_SUCCESS || !ctx)
      return set_error(MDB_ERR_CUDA, "mdb_compute_forces_noalloc: no current CUDA context");
  }
  ScratchAddr& a = g_scratch[dev];
  if (a.ptr == nullptr || a.ctx != ctx) {
    void* addr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_error(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    a.ptr = static_cast<unsigned char*>(addr);
    a.ctx = ctx;
  }
  *out = a.ptr;
  return MDB_OK;
}

int na_grid_axis(double L, double cell_min, bool wrap) {
  const double f = floor(L / cell_min);
  int k = (f >= 1.0) ? (f >= (double)kNaCellAxis ? kNaCellAxis : (int)f) : 1;
  // a periodic axis needs three cells for a stencil without repeats
  if (wrap && k < 3) k = 1;
  return k;
}

}  // namespace
}  // namespace mdb

extern "C" int mdb_compute_forces_noalloc(const mdb_config_t* cfg, const double* pos,
                                          const int32_t* type, int64_t n, double Lx, double Ly,
                                          int32_t periodic_y, void* stream, double* acc,
                                          double* uw) {
  using namespace mdb;
  if (!cfg || !uw || n < 0 || (n > 0 && (!pos || !type || !acc)))
    return set_error(MDB_ERR_ARG, "bad arguments");
  if (n > kNaMaxN)
    return set_error(MDB_ERR_CAPACITY,
                     "mdb_compute_forces_noalloc: n exceeds MDB_NOALLOC_MAX_PARTICLES (65536), "
                     "the capacity of its fixed 1 MiB device scratch array");
  if (!(Lx > 0.0) || !(Ly > 0.0) || !isfinite(Lx) || !isfinite(Ly))
    return set_error(MDB_ERR_BOX, "box lengths must be positive and finite");
  const mdb_config_t& c = *cfg;
  if (!(c.cutoff > 0.0) || !isfinite(c.cutoff))
    return set_error(MDB_ERR_CONFIG, "cutoff must be positive");
  if (!(c.MASS_A > 0.0) || !(c.MASS_B > 0.0))
    return set_error(MDB_ERR_CONFIG, "MASS_A and MASS_B must be positive");
  if (!(c.SIGMA_AA > 0.0) || !(c.SIGMA_BB > 0.0) || !(c.SIGMA_AB > 0.0))
    return set_error(MDB_ERR_CONFIG, "SIGMA_* must be positive");
  int dev = 0;
  MDB_CUDA(cudaGetDevice(&dev));
  unsigned char* base = nullptr;
  const int rc = scratch_for_device(dev, &base);
  if (rc) return rc;
  NaScratch s;
  s.cell_of = reinterpret_cast<int32_t*>(base + kOffCell);
  s.tmp = reinterpret_cast<int32_t*>(base + kOffTmp);
  s.idx = reinterpret_cast<int32_t*>(base + kOffIdx);
  s.count = reinterpret_cast<int32_t*>(base + kOffCount);
  s.start = reinterpret_cast<int32_t*>(base + kOffStart);
  s.part = reinterpret_cast<double*>(base + kOffPart);
  s.counter = reinterpret_cast<unsigned int*>(base + kOffCounter);

  NaPair p;
  const double sig[3] = {c.SIGMA_AA, c.SIGMA_BB, c.SIGMA_AB};
  const double eps[3] = {c.EPSILON_AA, c.EPSILON_BB, c.EPSILON_AB};
  const double inv_c = 1.0 / c.cutoff;
  const double csr6 = inv_c * inv_c * inv_c * inv_c * inv_c * inv_c;
  const float cutoff_f = (float)c.cutoff;
  for (int k = 0; k < 3; ++k) {
    p.Vc[k] = eps[k] * (4.0 * (csr6 * csr6 - csr6));
    const float sf = (float)sig[k], ef = (float)eps[k];
    p.sig2[k] = sf * sf;
    p.e24[k] = 24.0f * ef;
    p.e4[k] = 4.0f * ef;
    const float rcf = cutoff_f * sf;
    p.rc2[k] = rcf * rcf;
  }
  p.massA = c.MASS_A;
  p.massB = c.MASS_B;

  // cells at least the largest cutoff wide (with a margin for the rounding
  // of the binning product)
  const double rc_max = c.cutoff * fmax(sig[0], fmax(sig[1], sig[2]));
  const double cell_min = rc_max * (1.0 + 1e-6);
  NaGrid g;
  g.Lx = Lx;
  g.Ly = Ly;
  g.py = periodic_y ? 1 : 0;
  g.ncx = na_grid_axis(Lx, cell_min, true);
  g.ncy = na_grid_axis(Ly, cell_min, g.py != 0);
  g.ncells = g.ncx * g.ncy;
  g.sx = (double)g.ncx / Lx;
  g.sy = (double)g.ncy / Ly;

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int ni = (int)n;
  const int nb = ni > 0 ? (ni + kNaThreads - 1) / kNaThreads : 1;
  int launches = 1;
  if (ni > 0) {
    k_na_clear<<<(g.ncells + kNaThreads - 1) / kNaThreads, kNaThreads, 0, st>>>(s, g.ncells);
    k_na_bin<<<nb, kNaThreads, 0, st>>>(pos, ni, g, s);
    k_na_scan<<<1, kNaScanThreads, 0, st>>>(s, g.ncells, ni);
    k_na_fill<<<nb, kNaThreads, 0, st>>>(ni, s);
    k_na_rank<<<nb, kNaThreads, 0, st>>>(ni, s);
    launches += 5;
  } else {
    k_na_clear<<<1, kNaThreads, 0, st>>>(s, 0);
    launches += 1;
  }
  k_na_force<<<nb, kNaThreads, 0, st>>>(pos, type, ni, g, p, s, acc, uw);
  MDB_CUDA(cudaGetLastError());
  count_launches(launches);
  return MDB_OK;
}
