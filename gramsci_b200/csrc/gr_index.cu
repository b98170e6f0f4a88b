// Sorted-cell index on the device: replaces the kd-tree of the reference
// (src/kdtree2.F90:611-1012) as the structure behind the fixed-radius
// queries.  Points are bucketed into a uniform grid whose cells are at least
// rmax wide, counting-sorted by cell key, and re-laid out in cell order as
// float4 (FP32 fast path) and double4 (FP64 guard band, weight) arrays.
#include "gr_index.cuh"

#include <atomic>
#include <cstring>

namespace gr {

namespace {

// Order-preserving map of doubles onto unsigned 64-bit ints, so that min/max
// reductions can use integer atomics.
__device__ __forceinline__ unsigned long long dbl_key(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

__global__ void bbox_kernel(const double* __restrict__ xyz, int64_t n, unsigned long long* out) {
  // out[0..2] min keys, out[3..5] max keys, out[6] max |coord| key, out[7]
  // set when a coordinate is not finite (tested directly: a NaN's key does
  // not reliably survive the min / max reductions)
  unsigned long long mn[3] = {~0ull, ~0ull, ~0ull}, mx[3] = {0, 0, 0}, ab = 0;
  bool bad = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double v = xyz[3 * i + d];
      bad = bad || !isfinite(v);
      unsigned long long k = dbl_key(v);
      mn[d] = k < mn[d] ? k : mn[d];
      mx[d] = k > mx[d] ? k : mx[d];
      unsigned long long a = dbl_key(fabs(v));
      ab = a > ab ? a : ab;
    }
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(&out[7], 1ull);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      unsigned long long a = __shfl_xor_sync(0xffffffffu, mn[d], o);
      unsigned long long b = __shfl_xor_sync(0xffffffffu, mx[d], o);
      mn[d] = a < mn[d] ? a : mn[d];
      mx[d] = b > mx[d] ? b : mx[d];
    }
    unsigned long long c = __shfl_xor_sync(0xffffffffu, ab, o);
    ab = c > ab ? c : ab;
  }
  // block reduction, then one set of atomics per block
  __shared__ unsigned long long red[32][7];
  const int wid = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      red[wid][d] = mn[d];
      red[wid][3 + d] = mx[d];
    }
    red[wid][6] = ab;
  }
  __syncthreads();
  if (threadIdx.x < 7) {
    const int t = threadIdx.x;
    unsigned long long v = red[0][t];
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
      const unsigned long long u = red[k][t];
      v = (t < 3) ? (u < v ? u : v) : (u > v ? u : v);
    }
    if (t < 3)
      atomicMin(&out[t], v);
    else
      atomicMax(&out[t], v);
  }
}

// Speculative builds: flag [7] = 1 when the new bounding box differs from
// the one the grid was taken from.
__global__ void bbox_check_kernel(const unsigned long long* __restrict__ now,
                                  unsigned long long* __restrict__ prev) {
  if (threadIdx.x == 0) {
    unsigned long long d = 0;
    for (int k = 0; k < 7; ++k) d |= now[k] ^ prev[k];
    // a non-finite coordinate also sends the call to the build with waits,
    // which reports it
    prev[7] = (d != 0 || now[7] != 0) ? 1ull : 0ull;
  }
}

__global__ void init_bbox_kernel(unsigned long long* out) {
  int t = threadIdx.x;
  if (t < 3) out[t] = ~0ull;
  if (t >= 3 && t < 8) out[t] = 0ull;
}

__device__ __forceinline__ int cell_coord(double v, double lo, double inv_cs, int nc) {
  int c = (int)floor((v - lo) * inv_cs);
  return c < 0 ? 0 : (c >= nc ? nc - 1 : c);
}

__global__ void cell_assign_kernel(const double* __restrict__ xyz, int64_t n, GridGeom g,
                                   int* __restrict__ key, int* __restrict__ slot,
                                   int* __restrict__ count) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int cx = cell_coord(xyz[3 * i + 0], g.lo[0], g.inv_cs[0], g.nc[0]);
    int cy = cell_coord(xyz[3 * i + 1], g.lo[1], g.inv_cs[1], g.nc[1]);
    int cz = cell_coord(xyz[3 * i + 2], g.lo[2], g.inv_cs[2], g.nc[2]);
    int k = (cz * g.nc[1] + cy) * g.nc[0] + cx;
    key[i] = k;
    slot[i] = atomicAdd(&count[k], 1);
  }
}

// Place every point at start[key] + (rank of its original index among the
// points of its cell).  The rank makes the layout deterministic: within a
// cell, points keep their catalogue order.
__global__ void cell_scatter_kernel(int64_t n, const int* __restrict__ key,
                                    const int* __restrict__ slot, const int64_t* __restrict__ start,
                                    int* __restrict__ tmp_perm) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    tmp_perm[start[key[i]] + slot[i]] = (int)i;
}

// One warp per cell: rank each member by its catalogue index (O(c^2/32)),
// so that within a cell points keep their catalogue order, and write the
// member's data at its place in the cell-ordered layout (the scattered
// reads of the catalogue happen here, once per point).
__global__ void cell_order_gather_kernel(int64_t ncell, const int64_t* __restrict__ start,
                                         const int* __restrict__ tmp_perm,
                                         const double* __restrict__ xyz,
                                         const double* __restrict__ w,
                                         const int* __restrict__ buffer, int64_t n_data,
                                         float4* __restrict__ pos4, double4* __restrict__ posd,
                                         double* __restrict__ wl, int* __restrict__ orig,
                                         uint8_t* __restrict__ flags, int* __restrict__ cell_key) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c = warp; c < ncell; c += nwarps) {
    const int64_t b = start[c], e = start[c + 1];
    const int cnt = (int)(e - b);
    for (int k = lane; k < cnt; k += 32) {
      const int i = tmp_perm[b + k];
      int r = 0;
      for (int j = 0; j < cnt; ++j) r += tmp_perm[b + j] < i;
      const int64_t p = b + r;
      const double x = xyz[3 * (int64_t)i + 0], y = xyz[3 * (int64_t)i + 1],
                   z = xyz[3 * (int64_t)i + 2];
      const double wi = w[i];
      uint8_t f = (i >= n_data) ? FLAG_RANDOM : 0;
      if (buffer && buffer[i] == 1) f |= FLAG_BUFFER;
      // the fourth component marks buffer points (pair sweeps skip pairs of two)
      pos4[p] = make_float4(__double2float_rn(x), __double2float_rn(y), __double2float_rn(z),
                            (f & FLAG_BUFFER) ? 1.0f : 0.0f);
      posd[p] = make_double4(x, y, z, wi);
      wl[p] = wi;
      orig[p] = i;
      flags[p] = f;
      cell_key[p] = (int)c;
    }
  }
}

inline double key_to_dbl(unsigned long long k) {
  unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
  double v;
  std::memcpy(&v, &b, 8);
  return v;
}

// blocks for n items, at most `waves` blocks per SM
int blocks_for(int64_t n, int threads, int waves = 16) {
  const int64_t cap = (int64_t)waves * sm_count();
  int64_t b = (n + threads - 1) / threads;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (int)b;
}

}  // namespace

void CellIndex::build(const double* d_xyz, const double* d_w, const int* d_buffer, int64_t n_pts,
                      int64_t n_data_pts, double rmax, cudaStream_t s, bool speculate, int sub,
                      double dense_per_cell) {
  const bool auto_sub = sub == 0;
  if (sub != 2) sub = 1;
  n = n_pts;
  n_data = n_data_pts;
  launches = 0;
  bbox_raw.reserve(8);
  bbox_prev.reserve(8);
  init_bbox_kernel<<<1, 32, 0, s>>>(bbox_raw.p);
  launches++;
  if (n > 0) {
    bbox_kernel<<<blocks_for(n, 256, 2), 256, 0, s>>>(d_xyz, n, bbox_raw.p);
    launches++;
  }
  GR_CHECK_LAUNCH();
  unsigned long long h[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  // an automatic choice of sub decides from the bounding box, so it speculates
  // on the previous build's box like the grid does
  speculated = speculate && have_prev && prev_n == n && prev_rmax == rmax &&
               prev_auto == auto_sub && prev_sub == sub;
  if (speculated) {
    std::memcpy(h, prev_raw, sizeof(prev_raw));
    bbox_check_kernel<<<1, 32, 0, s>>>(bbox_raw.p, bbox_prev.p);
    launches++;
    GR_CHECK_LAUNCH();
  } else {
    GR_CUDA_TRY(cudaMemcpyAsync(h, bbox_raw.p, sizeof(h), cudaMemcpyDeviceToHost, s));
    GR_CUDA_TRY(cudaStreamSynchronize(s));
    if (h[7] != 0) throw Error{-1, "catalogue has non-finite coordinates"};
    std::memcpy(prev_raw, h, sizeof(prev_raw));
    prev_n = n;
    prev_rmax = rmax;
    prev_sub = sub;
    prev_auto = auto_sub;
    have_prev = true;
    GR_CUDA_TRY(cudaMemcpyAsync(bbox_prev.p, prev_raw, sizeof(prev_raw), cudaMemcpyHostToDevice, s));
    GR_CUDA_TRY(cudaMemsetAsync(bbox_prev.p + 7, 0, sizeof(unsigned long long), s));
  }
  double lo[3], hi[3];
  for (int d = 0; d < 3; ++d) {
    lo[d] = n > 0 ? key_to_dbl(h[d]) : 0.0;
    hi[d] = n > 0 ? key_to_dbl(h[3 + d]) : 0.0;
  }
  coord_max = n > 0 ? key_to_dbl(h[6]) : 0.0;
  for (int d = 0; d < 3; ++d)
    if (!std::isfinite(lo[d]) || !std::isfinite(hi[d]))
      throw Error{-1, "catalogue has non-finite coordinates"};
  // cells at least rmax (sub 2: rmax/2) wide; the cell table stays O(N)
  GridGeom g;
  {
    const int64_t cells1 = make_grid_geom(lo, hi, rmax, 2048, std::max<int64_t>(4 * n, 4096), g);
    per_cell_rmax = cells1 > 0 ? (double)n / (double)cells1 : 0.0;
    if (auto_sub) sub = (dense_per_cell > 0.0 && per_cell_rmax >= dense_per_cell) ? 2 : 1;
  }
  const int64_t total =
      make_grid_geom(lo, hi, rmax / sub, 2048, std::max<int64_t>(4 * n, 4096), g);
  grid.nx = g.nc[0];
  grid.ny = g.nc[1];
  grid.nz = g.nc[2];
  grid.ncell = total;
  grid.sub = sub;

  cell_count.reserve(total + 1);
  key_orig.reserve(n);
  slot.reserve(n);
  tmp_perm.reserve(n);
  cell_start64.reserve(total + 1);
  cell_start.reserve(total + 1);
  pos4.reserve(n);
  posd.reserve(n);
  w.reserve(n);
  orig.reserve(n);
  flags.reserve(n);
  cell_key.reserve(n);

  GR_CUDA_TRY(cudaMemsetAsync(cell_count.p, 0, sizeof(int) * (total + 1), s));
  if (n > 0) {
    cell_assign_kernel<<<blocks_for(n, 256), 256, 0, s>>>(d_xyz, n, g, key_orig.p, slot.p,
                                                         cell_count.p);
    launches++;
  }
  GR_CHECK_LAUNCH();
  // cell starts as 64-bit offsets and, in the same pass, the 32-bit copy
  // the kernels read
  scan_i32_to_i64(cell_count.p, cell_start64.p, total, s, scan_tmp, cell_start.p);
  launches += 3;
  if (n > 0) {
    cell_scatter_kernel<<<blocks_for(n, 256), 256, 0, s>>>(n, key_orig.p, slot.p, cell_start64.p,
                                                          tmp_perm.p);
    cell_order_gather_kernel<<<blocks_for(total * 32, 256), 256, 0, s>>>(
        total, cell_start64.p, tmp_perm.p, d_xyz, d_w, d_buffer, n_data, pos4.p, posd.p, w.p,
        orig.p, flags.p, cell_key.p);
    launches += 2;
  }
  GR_CHECK_LAUNCH();
}

int sm_count() {
  constexpr int kDev = 64;
  static std::atomic<int> cache[kDev];
  int dev = 0;
  GR_CUDA_TRY(cudaGetDevice(&dev));
  if (dev >= 0 && dev < kDev) {
    const int v = cache[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
  }
  int v = 0;
  GR_CUDA_TRY(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
  if (v < 1) v = 1;
  if (dev >= 0 && dev < kDev) cache[dev].store(v, std::memory_order_relaxed);
  return v;
}

int64_t make_grid_geom(const double lo[3], const double hi[3], double rmax, int max_per_axis,
                       int64_t max_cells, GridGeom& g) {
  double cell_min = rmax * 1.000001;
  if (!(cell_min > 0)) cell_min = 1e300;
  int64_t total = 1;
  for (int d = 0; d < 3; ++d) {
    const double span = hi[d] - lo[d];
    double k = std::floor(span / cell_min);
    if (!(k >= 1)) k = 1;
    if (k > max_per_axis) k = max_per_axis;
    g.nc[d] = (int)k;
    g.lo[d] = lo[d];
    g.inv_cs[d] = 1.0 / (span > 0 ? span / k : 1.0);
    total *= (int64_t)k;
  }
  while (total > max_cells && total > 1) {
    int d = 0;
    for (int k = 1; k < 3; ++k)
      if (g.nc[k] > g.nc[d]) d = k;
    g.nc[d] = std::max(1, g.nc[d] / 2);
    const double span = hi[d] - lo[d];
    g.inv_cs[d] = 1.0 / (span > 0 ? span / g.nc[d] : 1.0);
    total = (int64_t)g.nc[0] * g.nc[1] * g.nc[2];
  }
  return total;
}

DevCatalog CellIndex::view() const {
  DevCatalog c;
  c.pos4 = pos4.p;
  c.posd = posd.p;
  c.w = w.p;
  c.orig = orig.p;
  c.flags = flags.p;
  c.cell_key = cell_key.p;
  c.cell_start = cell_start.p;
  c.n = (int)n;
  c.n_data = (int)n_data;
  c.grid = grid;
  c.cell_region = nullptr;
  c.region_grid = nullptr;
  c.region_cell_off = nullptr;
  return c;
}

// ------------------------------------------------------------------- scan --
namespace {

constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
__device__ __forceinline__ int64_t block_exclusive_scan(int64_t v, int64_t* warp_tot, int64_t& total) {
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int64_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int64_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    int64_t t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int64_t y = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += y;
    }
    if (lane < nw) warp_tot[lane] = t;
  }
  __syncthreads();
  int64_t before = wid > 0 ? warp_tot[wid - 1] : 0;
  total = warp_tot[(blockDim.x >> 5) - 1];
  return before + x - v;
}

template <typename T>
__global__ void scan_tile_sums(const T* __restrict__ in, int64_t n, int64_t* __restrict__ sums) {
  __shared__ int64_t warp_tot[32];
  int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) s += (int64_t)in[base + k];
  int64_t total;
  block_exclusive_scan<T>(s, warp_tot, total);
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <typename T>
__global__ void scan_tile_apply(const T* __restrict__ in, int64_t n, const int64_t* __restrict__ offs,
                                int64_t* __restrict__ out, int* __restrict__ out32) {
  __shared__ int64_t warp_tot[32];
  int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int64_t v[kScanItems];
  int64_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (base + k < n) ? (int64_t)in[base + k] : 0;
    s += v[k];
  }
  int64_t total;
  int64_t ex = block_exclusive_scan<T>(s, warp_tot, total) + (offs ? offs[blockIdx.x] : 0);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) {
      out[base + k] = ex;
      if (out32) out32[base + k] = (int)ex;
    }
    ex += v[k];
  }
  // the last element of the whole array writes the grand total at out[n]
  if (base <= n - 1 && n - 1 < base + kScanItems) {
    out[n] = ex;
    if (out32) out32[n] = (int)ex;
  }
}

// Exclusive scan of in[0, n) into out[0, n] (out[n] = the total); out32,
// when given, receives the same values as 32-bit integers.
template <typename T>
void scan_impl(const T* in, int64_t* out, int64_t n, cudaStream_t s, DevBuf<int64_t>& tmp,
               size_t tmp_off, int* out32 = nullptr) {
  if (n <= 0) {
    GR_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(int64_t), s));
    if (out32) GR_CUDA_TRY(cudaMemsetAsync(out32, 0, sizeof(int), s));
    return;
  }
  int64_t tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 1) {
    scan_tile_apply<T><<<1, kScanThreads, 0, s>>>(in, n, nullptr, out, out32);
    GR_CHECK_LAUNCH();
    return;
  }
  int64_t* sums = tmp.p + tmp_off;
  int64_t* offs = sums + tiles;
  scan_tile_sums<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, sums);
  GR_CHECK_LAUNCH();
  scan_impl<int64_t>(sums, offs, tiles, s, tmp, tmp_off + 2 * tiles + 1);
  scan_tile_apply<T><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, n, offs, out, out32);
  GR_CHECK_LAUNCH();
}

size_t scan_tmp_need(int64_t n) {
  size_t need = 0;
  while (n > kScanTile) {
    int64_t tiles = (n + kScanTile - 1) / kScanTile;
    need += 2 * tiles + 1;
    n = tiles;
  }
  return need + 1;
}

}  // namespace

namespace {

// Buffers from cudaMalloc start 256-byte aligned; each is zeroed with 16-byte
// stores for its body and 4-byte stores for a tail (sizes are multiples of 4).
__global__ void zero_many_kernel(ZeroList z) {
  const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const size_t nthr = (size_t)gridDim.x * blockDim.x;
  for (int k = 0; k < z.n; ++k) {
    const size_t nv = z.bytes[k] / 16;
    uint4* v = reinterpret_cast<uint4*>(z.p[k]);
    for (size_t i = tid; i < nv; i += nthr) v[i] = make_uint4(0u, 0u, 0u, 0u);
    const size_t tail = (z.bytes[k] - nv * 16) / 4;
    uint32_t* t = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(z.p[k]) + nv * 16);
    if (tid < tail) t[tid] = 0u;
  }
}

}  // namespace

void zero_async(const ZeroList& z, cudaStream_t s) {
  if (z.n == 0) return;
  size_t total = 0;
  for (int k = 0; k < z.n; ++k) {
    if ((reinterpret_cast<uintptr_t>(z.p[k]) & 15) != 0 || (z.bytes[k] & 3) != 0)
      throw Error{-2, "zero_async: buffer not 16-byte aligned or size not a multiple of 4"};
    total += z.bytes[k];
  }
  const size_t threads = 256;
  size_t blocks = (total / 16 + threads - 1) / threads;
  if (blocks < 1) blocks = 1;
  if (blocks > (size_t)8 * sm_count()) blocks = (size_t)8 * sm_count();
  zero_many_kernel<<<(unsigned)blocks, (unsigned)threads, 0, s>>>(z);
  GR_CHECK_LAUNCH();
}

void scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s, DevBuf<int64_t>& tmp) {
  size_t need = scan_tmp_need(n);
  if (tmp.n < need) tmp.reserve(need);
  scan_impl<int64_t>(in, out, n, s, tmp, 0);
}

void scan_i32_to_i64(const int* in, int64_t* out, int64_t n, cudaStream_t s, DevBuf<int64_t>& tmp,
                     int* out32) {
  size_t need = scan_tmp_need(n);
  if (tmp.n < need) tmp.reserve(need);
  scan_impl<int>(in, out, n, s, tmp, 0, out32);
}

}  // namespace gr
