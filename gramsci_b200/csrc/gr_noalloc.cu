// gr_count_2pcf_noalloc: the 2PCF path for callers that cannot allocate
// device memory.
//
// Some callers cannot call cudaMalloc: code that runs inside another
// framework's memory pool or under a fixed memory budget, plugins that may
// only use the buffers their host hands them, and callers that must not
// synchronise with the device allocator in the middle of their own stream
// work.  This entry point needs no allocation at all.  The caller passes
// device pointers to the catalogue and to the outputs; every intermediate
// array (cell index, point layout, histograms) lives in one file-scope
// device array, g_noalloc_scratch, of fixed size (kNoAllocBytes, about
// 4.3 MB), which every GPU that loads the library holds until the process
// exits.
//
// Limits (larger inputs are rejected with GR_E_CAPACITY before any kernel
// runs): at most GR_NOALLOC_MAX_POINTS points, at most
// GR_NOALLOC_MAX_BINS radial x mu bins, and a cell grid of at most
// kMaxCells cells (cells are merged to stay below it).
//
// The scratch array is shared by every call on a device and keeps the last
// call's contents; each call clears what must start at zero.  Calls whose
// work overlaps on the GPU (two host threads, or two streams in flight at
// once) race on the scratch and must be serialised by the caller.
//
// Each call waits once on its stream: the catalogue's bounding box is read
// back to size the cell grid before the sweep is queued.
//
// Host code cannot use the array's name as a device address, so the first
// call on each device (and CUDA context), with that device current, looks
// the address up with cudaGetSymbolAddress and caches it; that first call
// should come before any stream capture.  The cache is keyed by the current
// context, so a context created later on the same device (a non-primary
// context, or the primary context again after cudaDeviceReset) gets its own
// lookup.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/gramsci_cuda.h"
#include "gr_kernels.cuh"

namespace gr {
namespace {

constexpr int64_t kMaxPoints = GR_NOALLOC_MAX_POINTS;
constexpr int64_t kMaxCells = 65536;
constexpr int64_t kMaxHist = (int64_t)GR_NOALLOC_MAX_BINS * 4;

constexpr size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// scratch layout (byte offsets)
constexpr size_t kOffMisc = 0;                                            // 16 x u64
constexpr size_t kOffKey = al256(kOffMisc + 16 * 8);                      // int[N]
constexpr size_t kOffSlot = al256(kOffKey + 4 * kMaxPoints);              // int[N]
constexpr size_t kOffTmpPerm = al256(kOffSlot + 4 * kMaxPoints);          // int[N]
constexpr size_t kOffPerm = al256(kOffTmpPerm + 4 * kMaxPoints);          // int[N]
constexpr size_t kOffPos4 = al256(kOffPerm + 4 * kMaxPoints);             // float4[N]
constexpr size_t kOffPosd = al256(kOffPos4 + 16 * kMaxPoints);           // double4[N]
constexpr size_t kOffW = al256(kOffPosd + 32 * kMaxPoints);               // double[N]
constexpr size_t kOffOrig = al256(kOffW + 8 * kMaxPoints);                // int[N]
constexpr size_t kOffFlags = al256(kOffOrig + 4 * kMaxPoints);            // u8[N]
constexpr size_t kOffCellKey = al256(kOffFlags + kMaxPoints);             // int[N]
constexpr size_t kOffCount = al256(kOffCellKey + 4 * kMaxPoints);         // int[C+1]
constexpr size_t kOffStart64 = al256(kOffCount + 4 * (kMaxCells + 1));    // int64[C+1]
constexpr size_t kOffStart = al256(kOffStart64 + 8 * (kMaxCells + 1));    // int[C+1]
constexpr size_t kOffHCnt = al256(kOffStart + 4 * (kMaxCells + 1));       // u64[H]
constexpr size_t kOffHFix = al256(kOffHCnt + 8 * kMaxHist);               // u64[2H]
constexpr size_t kOffStats = al256(kOffHFix + 16 * kMaxHist);             // u64[8]
constexpr size_t kOffWork = al256(kOffStats + 8 * 8);                     // int[4]
constexpr size_t kNoAllocBytes = al256(kOffWork + 16);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// cached device addresses of the scratch array, per (device, context)
struct SymbolEntry {
  int device;
  void* context;
  unsigned char* addr;
};
std::mutex g_symbol_mutex;
std::vector<SymbolEntry> g_symbol_cache;

// misc words: [0..2] min keys, [3..5] max keys, [6] max |coord| key,
// [7] max |w| bits, [8] set when a coordinate or weight is not finite
// (tested directly: a NaN's key does not reliably survive the reductions)
__device__ __forceinline__ unsigned long long na_key(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

__global__ void na_init_kernel(unsigned long long* misc) {
  const int t = threadIdx.x;
  if (t < 3) misc[t] = ~0ull;
  if (t >= 3 && t < 16) misc[t] = 0ull;
}

__global__ void na_bounds_kernel(const double* __restrict__ xyz, const double* __restrict__ w,
                                 int n, unsigned long long* misc) {
  unsigned long long mn[3] = {~0ull, ~0ull, ~0ull}, mx[3] = {0, 0, 0}, ab = 0, wm = 0;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (i0 >= n) return;
  bool bad = false;
  for (int i = i0; i < n; i += gridDim.x * blockDim.x) {
    bad = bad || !isfinite(w[i]);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double v = xyz[3 * (int64_t)i + d];
      bad = bad || !isfinite(v);
      const unsigned long long k = na_key(v);
      mn[d] = k < mn[d] ? k : mn[d];
      mx[d] = k > mx[d] ? k : mx[d];
      const unsigned long long a = na_key(fabs(v));
      ab = a > ab ? a : ab;
    }
    const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(w[i]));
    wm = b > wm ? b : wm;
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    atomicMin(&misc[d], mn[d]);
    atomicMax(&misc[3 + d], mx[d]);
  }
  atomicMax(&misc[6], ab);
  atomicMax(&misc[7], wm);
  if (bad) atomicOr(&misc[8], 1ull);
}

__global__ void na_assign_kernel(const double* __restrict__ xyz, int n, GridGeom g,
                                 int* __restrict__ key, int* __restrict__ slot,
                                 int* __restrict__ count) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int c[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      int v = (int)floor((xyz[3 * (int64_t)i + d] - g.lo[d]) * g.inv_cs[d]);
      c[d] = v < 0 ? 0 : (v >= g.nc[d] ? g.nc[d] - 1 : v);
    }
    const int k = (c[2] * g.nc[1] + c[1]) * g.nc[0] + c[0];
    key[i] = k;
    slot[i] = atomicAdd(&count[k], 1);
  }
}

// exclusive scan of count[0..m) into start64[0..m] and start[0..m], one block
__global__ void na_scan_kernel(const int* __restrict__ count, int m, int64_t* __restrict__ start64,
                               int* __restrict__ start) {
  __shared__ int64_t part[1024];
  const int t = threadIdx.x;
  const int per = (m + blockDim.x - 1) / blockDim.x;
  const int b = t * per, e = min(m, b + per);
  int64_t s = 0;
  for (int i = b; i < e; ++i) s += count[i];
  part[t] = s;
  __syncthreads();
  if (t == 0) {
    int64_t acc = 0;
    for (int k = 0; k < (int)blockDim.x; ++k) {
      const int64_t v = part[k];
      part[k] = acc;
      acc += v;
    }
    start64[m] = acc;
    start[m] = (int)acc;
  }
  __syncthreads();
  int64_t acc = part[t];
  for (int i = b; i < e; ++i) {
    start64[i] = acc;
    start[i] = (int)acc;
    acc += count[i];
  }
}

__global__ void na_scatter_kernel(int n, const int* __restrict__ key, const int* __restrict__ slot,
                                  const int64_t* __restrict__ start, int* __restrict__ tmp_perm) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    tmp_perm[start[key[i]] + slot[i]] = i;
}

// in-cell order by catalogue index, warp per cell
__global__ void na_order_kernel(int ncell, const int64_t* __restrict__ start,
                                const int* __restrict__ tmp_perm, int* __restrict__ perm) {
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int c = warp; c < ncell; c += nwarps) {
    const int b = (int)start[c], cnt = (int)(start[c + 1] - start[c]);
    for (int k = lane; k < cnt; k += 32) {
      const int v = tmp_perm[b + k];
      int r = 0;
      for (int j = 0; j < cnt; ++j) r += tmp_perm[b + j] < v;
      perm[b + r] = v;
    }
  }
}

__global__ void na_gather_kernel(int n, int n_data, const int* __restrict__ perm,
                                 const double* __restrict__ xyz, const double* __restrict__ w,
                                 const int* __restrict__ key, float4* __restrict__ pos4,
                                 double4* __restrict__ posd, double* __restrict__ wl,
                                 int* __restrict__ orig, uint8_t* __restrict__ flags,
                                 int* __restrict__ cell_key) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const int i = perm[p];
    const double x = xyz[3 * (int64_t)i], y = xyz[3 * (int64_t)i + 1], z = xyz[3 * (int64_t)i + 2];
    pos4[p] = make_float4(__double2float_rn(x), __double2float_rn(y), __double2float_rn(z), 0.f);
    posd[p] = make_double4(x, y, z, w[i]);
    wl[p] = w[i];
    orig[p] = i;
    flags[p] = i >= n_data ? FLAG_RANDOM : 0;
    cell_key[p] = key[i];
  }
}

// counts and fixed-point sums -> caller's device outputs
__global__ void na_finish_kernel(const unsigned long long* __restrict__ hcnt,
                                 const unsigned long long* __restrict__ hfix, int nbm,
                                 double inv_scale, int64_t* __restrict__ counts,
                                 double* __restrict__ catsum, double* __restrict__ N2,
                                 double* __restrict__ N3) {
  const int nh = 4 * nbm;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nbm; k += gridDim.x * blockDim.x) {
    double s[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int j = k + nbm * c;
      // one rounding, as gr_count_2pcf converts its sums on the host
      s[c] = fix_to_double(hfix[j], hfix[nh + j], inv_scale);
      if (counts) counts[j] = (int64_t)hcnt[j];
      if (catsum) catsum[j] = s[c];
    }
    if (N2) N2[k] = ((s[0] + s[1]) + s[2]) + s[3];
    if (N3) N3[k] = s[3];
  }
}

// The CUDA context current on this thread (cuCtxGetCurrent, reached through
// the runtime's driver entry point so that the library does not link
// against the driver library); nullptr when it cannot be queried.
void* current_context() {
  typedef int (*CtxGetCurrent)(void**);
  static CtxGetCurrent fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrent>(f);
  }();
  void* ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

// Device address of the scratch array in the current device and context:
// looked up with cudaGetSymbolAddress on the first call there, then cached.
unsigned char* scratch_address(int device, int* status) {
  void* ctx = current_context();
  std::lock_guard<std::mutex> lock(g_symbol_mutex);
  for (const SymbolEntry& e : g_symbol_cache)
    if (e.device == device && e.context == ctx) {
      *status = GR_OK;
      return e.addr;
    }
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
    *status = GR_E_CUDA;
    return nullptr;
  }
  g_symbol_cache.push_back(SymbolEntry{device, ctx, static_cast<unsigned char*>(p)});
  *status = GR_OK;
  return static_cast<unsigned char*>(p);
}

inline double key_value(unsigned long long k) {
  unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
  double v;
  std::memcpy(&v, &b, 8);
  return v;
}

}  // namespace
}  // namespace gr

using namespace gr;

extern "C" int gr_count_2pcf_noalloc(const double* d_xyz, const double* d_w, int64_t n_data,
                                     int64_t n_rand, double rmin, double rmax, int32_t nbins,
                                     int32_t nmu, int64_t* d_counts, double* d_catsum,
                                     double* d_N2, double* d_N3, void* stream) {
  const int64_t n = n_data + n_rand;
  if (n_data < 0 || n_rand < 0 || (n > 0 && (!d_xyz || !d_w))) return GR_E_ARG;
  if (nbins < 1 || nbins > kMaxBins || nmu < 1 || nmu > kMaxBins) return GR_E_ARG;
  if (!(rmax > rmin) || !(rmin >= 0.0) || !std::isfinite(rmax)) return GR_E_ARG;
  if (n > kMaxPoints) return GR_E_CAPACITY;
  if ((int64_t)nbins * nmu > GR_NOALLOC_MAX_BINS) return GR_E_CAPACITY;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  try {
    int device = 0;
    GR_CUDA_TRY(cudaGetDevice(&device));
    int status = GR_OK;
    unsigned char* base = scratch_address(device, &status);
    if (!base) return status;
    unsigned long long* misc = reinterpret_cast<unsigned long long*>(base + kOffMisc);
    int* key = reinterpret_cast<int*>(base + kOffKey);
    int* slot = reinterpret_cast<int*>(base + kOffSlot);
    int* tmp_perm = reinterpret_cast<int*>(base + kOffTmpPerm);
    int* perm = reinterpret_cast<int*>(base + kOffPerm);
    float4* pos4 = reinterpret_cast<float4*>(base + kOffPos4);
    double4* posd = reinterpret_cast<double4*>(base + kOffPosd);
    double* wl = reinterpret_cast<double*>(base + kOffW);
    int* orig = reinterpret_cast<int*>(base + kOffOrig);
    uint8_t* flags = reinterpret_cast<uint8_t*>(base + kOffFlags);
    int* cell_key = reinterpret_cast<int*>(base + kOffCellKey);
    int* count = reinterpret_cast<int*>(base + kOffCount);
    int64_t* start64 = reinterpret_cast<int64_t*>(base + kOffStart64);
    int* start = reinterpret_cast<int*>(base + kOffStart);
    unsigned long long* hcnt = reinterpret_cast<unsigned long long*>(base + kOffHCnt);
    unsigned long long* hfix = reinterpret_cast<unsigned long long*>(base + kOffHFix);
    unsigned long long* stats = reinterpret_cast<unsigned long long*>(base + kOffStats);
    int* work = reinterpret_cast<int*>(base + kOffWork);
    const int nbm = nbins * nmu, nh = 4 * nbm;
    const int ni = (int)n;

    // bounds of the catalogue and of |w|
    na_init_kernel<<<1, 32, 0, s>>>(misc);
    const int nsm = sm_count();
    if (ni > 0) na_bounds_kernel<<<std::min(nsm, (ni + 255) / 256), 256, 0, s>>>(d_xyz, d_w, ni, misc);
    GR_CHECK_LAUNCH();
    unsigned long long h[9];
    GR_CUDA_TRY(cudaMemcpyAsync(h, misc, sizeof(h), cudaMemcpyDeviceToHost, s));
    GR_CUDA_TRY(cudaStreamSynchronize(s));
    if (h[8] != 0) return GR_E_ARG;  // a coordinate or weight is not finite
    double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    double coord_max = 0.0, wmax = 0.0;
    if (ni > 0) {
      for (int d = 0; d < 3; ++d) {
        lo[d] = key_value(h[d]);
        hi[d] = key_value(h[3 + d]);
        if (!std::isfinite(lo[d]) || !std::isfinite(hi[d])) return GR_E_ARG;
      }
      coord_max = key_value(h[6]);
      std::memcpy(&wmax, &h[7], 8);
      if (!std::isfinite(wmax)) return GR_E_ARG;
    }
    // grid: cells at least rmax wide, at most kMaxCells of them (the same
    // geometry as the allocating path's index, with this array's cap)
    GridGeom g;
    const int64_t total = make_grid_geom(lo, hi, rmax, 2048, kMaxCells, g);
    const int ncell = (int)total;

    // cell index in the scratch array
    GR_CUDA_TRY(cudaMemsetAsync(count, 0, sizeof(int) * (ncell + 1), s));
    const int blocks = std::max(1, std::min(4 * nsm, (ni + 255) / 256));
    if (ni > 0) na_assign_kernel<<<blocks, 256, 0, s>>>(d_xyz, ni, g, key, slot, count);
    na_scan_kernel<<<1, 1024, 0, s>>>(count, ncell, start64, start);
    if (ni > 0) {
      na_scatter_kernel<<<blocks, 256, 0, s>>>(ni, key, slot, start64, tmp_perm);
      na_order_kernel<<<std::max(1, std::min(4 * nsm, (ncell * 32 + 255) / 256)), 256, 0, s>>>(
          ncell, start64, tmp_perm, perm);
      na_gather_kernel<<<blocks, 256, 0, s>>>(ni, (int)n_data, perm, d_xyz, d_w, key, pos4, posd,
                                              wl, orig, flags, cell_key);
    }
    GR_CHECK_LAUNCH();

    DevCatalog C;
    C.pos4 = pos4;
    C.posd = posd;
    C.w = wl;
    C.orig = orig;
    C.flags = flags;
    C.cell_key = cell_key;
    C.cell_start = start;
    C.n = ni;
    C.n_data = (int)n_data;
    C.grid.nx = g.nc[0];
    C.grid.ny = g.nc[1];
    C.grid.nz = g.nc[2];
    C.grid.ncell = total;
    C.grid.sub = 1;
    C.cell_region = nullptr;
    C.region_grid = nullptr;
    C.region_cell_off = nullptr;
    PairParams P;
    make_pair_params(P, rmin, rmax, nbins, nmu, 0, coord_max, 0);
    const double fscale = fix_scale(wmax * wmax);

    // histograms start at zero on every call
    GR_CUDA_TRY(cudaMemsetAsync(hcnt, 0, sizeof(unsigned long long) * nh, s));
    GR_CUDA_TRY(cudaMemsetAsync(hfix, 0, sizeof(unsigned long long) * 2 * nh, s));
    GR_CUDA_TRY(cudaMemsetAsync(stats, 0, sizeof(unsigned long long) * 8, s));
    launch_pair2(C, P, true, hcnt, hfix, fscale, stats, work, s);
    na_finish_kernel<<<std::max(1, std::min(nsm, (nbm + 255) / 256)), 256, 0, s>>>(
        hcnt, hfix, nbm, 1.0 / fscale, d_counts, d_catsum, d_N2, d_N3);
    GR_CHECK_LAUNCH();
  } catch (const gr::Error& e) {
    return e.code;
  } catch (...) {
    return GR_E_CUDA;
  }
  return GR_OK;
}
