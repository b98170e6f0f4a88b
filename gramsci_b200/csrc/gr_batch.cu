// Batched regions: the 2PCF over a domain decomposition of the catalogue in
// one persistent launch, replayed from a CUDA graph.
//
// The reference handles large catalogues by domain decomposition
// (src/domain_decomposition.f90:39-80): region j is the bounding box of its
// points, grown by Rmax on every side (strict inequalities, :64-66); points
// of other regions inside that halo are buffer points, which serve as
// neighbours but never as roots (src/gramsci.F90:363).  Each region is then
// run as a separate program and the outputs summed by hand.  Here the
// catalogue's bounding box is split into nsplit^3 equal subcubes (region of a
// point = its subcube), the region boxes and halos are computed on the
// device in FP64, and every region's members (its own points, plus buffer
// copies of the other points inside its halo) are laid out together: each
// region gets its own cell grid over its halo box, the cells of all regions
// are numbered consecutively (largest region first), and a single launch of
// the warp-per-cell pair kernel processes the cells of every region from
// one work counter.  Galaxy/random flags and the global weight
// normalisation are kept, so the summed histogram equals the unsplit run.
//
// The first call for a given catalogue, binning and split computes the
// geometry on the host (region boxes, halos, member counts, grids) and runs
// eagerly; the device work of every later call (membership, cell sort,
// layout, pair sweep) is replayed from a captured CUDA graph.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "gr_batch.cuh"

namespace gr {

namespace {

__device__ __forceinline__ unsigned long long bkey(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

inline double bkey_value(unsigned long long k) {
  unsigned long long b = (k & 0x8000000000000000ull) ? (k & 0x7fffffffffffffffull) : ~k;
  double v;
  std::memcpy(&v, &b, 8);
  return v;
}

struct SplitGeom {
  double lo[3], inv_span[3];
  int ns;
};

__device__ __forceinline__ int sub_coord(double v, double lo, double inv_span, int ns) {
  int s = (int)floor((v - lo) * inv_span * ns);
  return s < 0 ? 0 : (s >= ns ? ns - 1 : s);
}

// catalogue bounding box: out[0..2] min keys, out[3..5] max keys
__global__ void b_bbox_kernel(const double* __restrict__ xyz, int n, unsigned long long* out) {
  unsigned long long mn[3] = {~0ull, ~0ull, ~0ull}, mx[3] = {0, 0, 0};
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (i0 >= n) return;
  for (int i = i0; i < n; i += gridDim.x * blockDim.x)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const unsigned long long k = bkey(xyz[3 * (int64_t)i + d]);
      mn[d] = k < mn[d] ? k : mn[d];
      mx[d] = k > mx[d] ? k : mx[d];
    }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    atomicMin(&out[d], mn[d]);
    atomicMax(&out[3 + d], mx[d]);
  }
}

// subcube of every point, per-region boxes (6 keys per region) and sizes
__global__ void b_region_box_kernel(const double* __restrict__ xyz, int n, SplitGeom g,
                                    int* __restrict__ sub, unsigned long long* __restrict__ box,
                                    int* __restrict__ own_count) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double x = xyz[3 * (int64_t)i], y = xyz[3 * (int64_t)i + 1], z = xyz[3 * (int64_t)i + 2];
    const int sx = sub_coord(x, g.lo[0], g.inv_span[0], g.ns);
    const int sy = sub_coord(y, g.lo[1], g.inv_span[1], g.ns);
    const int sz = sub_coord(z, g.lo[2], g.inv_span[2], g.ns);
    const int r = (sz * g.ns + sy) * g.ns + sx;
    sub[i] = r;
    atomicMin(&box[6 * r + 0], bkey(x));
    atomicMin(&box[6 * r + 1], bkey(y));
    atomicMin(&box[6 * r + 2], bkey(z));
    atomicMax(&box[6 * r + 3], bkey(x));
    atomicMax(&box[6 * r + 4], bkey(y));
    atomicMax(&box[6 * r + 5], bkey(z));
    atomicAdd(&own_count[r], 1);
  }
}

__global__ void b_init_box_kernel(unsigned long long* box, int nreg) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < 6 * nreg; k += gridDim.x * blockDim.x)
    box[k] = (k % 6) < 3 ? ~0ull : 0ull;
}

__device__ __forceinline__ bool in_halo(const double* h, double x, double y, double z) {
  return x > h[0] && x < h[3] && y > h[1] && y < h[4] && z > h[2] && z < h[5];
}

// Region boxes and sizes from a given region id per point.
__global__ void b_region_box_ids_kernel(const double* __restrict__ xyz, int n,
                                        const int* __restrict__ reg,
                                        unsigned long long* __restrict__ box,
                                        int* __restrict__ own_count) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int r = reg[i];
    const double x = xyz[3 * (int64_t)i], y = xyz[3 * (int64_t)i + 1], z = xyz[3 * (int64_t)i + 2];
    atomicMin(&box[6 * r + 0], bkey(x));
    atomicMin(&box[6 * r + 1], bkey(y));
    atomicMin(&box[6 * r + 2], bkey(z));
    atomicMax(&box[6 * r + 3], bkey(x));
    atomicMax(&box[6 * r + 4], bkey(y));
    atomicMax(&box[6 * r + 5], bkey(z));
    atomicAdd(&own_count[r], 1);
  }
}

// Memberships of point i, f(region, buffer): every point belongs to its own
// region, and in the halo layouts to every other region whose halo
// contains it, as a buffer point.  Subcube split: the own subcube and the 26
// around it (a halo reaches at most Rmax beyond its box, and a region's box
// lies inside its subcube, so farther subcubes cannot qualify when the
// subcubes are at least Rmax wide -- the host checks that).  Region ids: the
// regions the coarse grid lists for the point's coarse cell.  Mocks: the own
// region only (no halos).
enum : int { kMemSplit = 0, kMemIds = 1, kMemMocks = 2 };

template <int MODE, class F>
__device__ __forceinline__ void for_each_membership(double x, double y, double z, int own,
                                                    const RegionGeomDev& G, const CoarseDev& CG,
                                                    F f) {
  if (MODE == kMemSplit) {
    const int sx = own % G.ns, sy = (own / G.ns) % G.ns, sz = own / (G.ns * G.ns);
    for (int dz = -1; dz <= 1; ++dz) {
      const int tz = sz + dz;
      if (tz < 0 || tz >= G.ns) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int ty = sy + dy;
        if (ty < 0 || ty >= G.ns) continue;
        for (int dx = -1; dx <= 1; ++dx) {
          const int tx = sx + dx;
          if (tx < 0 || tx >= G.ns) continue;
          const int r = (tz * G.ns + ty) * G.ns + tx;
          if (in_halo(G.halo + 6 * r, x, y, z)) f(r, r != own);
        }
      }
    }
    return;
  }
  f(own, false);
  if (MODE == kMemMocks) return;
  const double v[3] = {x, y, z};
  int c[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int q = (int)floor((v[d] - CG.lo[d]) * CG.inv[d]);
    c[d] = q < 0 ? 0 : (q >= CG.nc[d] ? CG.nc[d] - 1 : q);
  }
  const int cc = (c[2] * CG.nc[1] + c[1]) * CG.nc[0] + c[0];
  for (int k = CG.off[cc]; k < CG.off[cc + 1]; ++k) {
    const int r = CG.list[k];
    if (r != own && in_halo(G.halo + 6 * r, x, y, z)) f(r, true);
  }
}

// Region members.  PASS 0 (planning): members per region (count).  PASS 1:
// memberships per point (mcount).  PASS 2: the memberships of point i
// written at moff[i] onward (an exclusive scan of PASS 1): catalogue index,
// flags, cell key in the region's grid and slot in that cell.  Only the
// per-cell slots use atomics (many cells, little contention); the members of
// a region need no common counter.  Random flags from pflag when given,
// else from the galaxy / random split.
template <int PASS, int MODE>
__global__ void b_members_kernel(const double* __restrict__ xyz, int n, int n_data,
                                 const int* __restrict__ reg, const uint8_t* __restrict__ pflag,
                                 RegionGeomDev G, CoarseDev CG, int* __restrict__ count,
                                 int* __restrict__ mcount, const int64_t* __restrict__ moff,
                                 int* __restrict__ m_orig, uint8_t* __restrict__ m_flag,
                                 int* __restrict__ m_key, int* __restrict__ m_slot,
                                 int* __restrict__ cell_count) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double x = xyz[3 * (int64_t)i], y = xyz[3 * (int64_t)i + 1], z = xyz[3 * (int64_t)i + 2];
    const int own = reg[i];
    const uint8_t rnd = pflag ? (uint8_t)(pflag[i] & FLAG_RANDOM) : (uint8_t)(i >= n_data ? FLAG_RANDOM : 0);
    if (PASS == 0) {
      for_each_membership<MODE>(x, y, z, own, G, CG, [&](int r, bool) { atomicAdd(&count[r], 1); });
    } else if (PASS == 1) {
      int c = 0;
      for_each_membership<MODE>(x, y, z, own, G, CG, [&](int, bool) { ++c; });
      mcount[i] = c;
    } else {
      int64_t m = moff[i];
      for_each_membership<MODE>(x, y, z, own, G, CG, [&](int r, bool buf) {
        m_orig[m] = i;
        m_flag[m] = (uint8_t)(rnd | (buf ? FLAG_BUFFER : 0));
        const GridParams g = G.grid[r];
        const double v[3] = {x, y, z};
        int c[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const int q = (int)floor((v[d] - G.glo[3 * r + d]) * G.ginv[3 * r + d]);
          const int nc = d == 0 ? g.nx : (d == 1 ? g.ny : g.nz);
          c[d] = q < 0 ? 0 : (q >= nc ? nc - 1 : q);
        }
        const int key = G.cell_off[r] + (c[2] * g.ny + c[1]) * g.nx + c[0];
        m_key[m] = key;
        m_slot[m] = atomicAdd(&cell_count[key], 1);
        ++m;
      });
    }
  }
}

__global__ void b_scatter_kernel(int64_t m, const int* __restrict__ key, const int* __restrict__ slot,
                                 const int64_t* __restrict__ start, int* __restrict__ tmp) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m;
       k += (int64_t)gridDim.x * blockDim.x)
    tmp[start[key[k]] + slot[k]] = (int)k;
}

// members of a cell ordered by catalogue index (deterministic layout)
__global__ void b_order_kernel(int64_t ncell, const int64_t* __restrict__ start,
                               const int* __restrict__ tmp, const int* __restrict__ m_orig,
                               int* __restrict__ perm) {
  const int lane = threadIdx.x & 31;
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c = warp; c < ncell; c += nwarps) {
    const int64_t b = start[c];
    const int cnt = (int)(start[c + 1] - b);
    for (int k = lane; k < cnt; k += 32) {
      const int v = tmp[b + k];
      const int ov = m_orig[v];
      int r = 0;
      for (int j = 0; j < cnt; ++j) r += m_orig[tmp[b + j]] < ov;
      perm[b + r] = v;
    }
  }
}

__global__ void b_gather_kernel(int64_t m, const int* __restrict__ perm,
                                const int* __restrict__ m_orig, const uint8_t* __restrict__ m_flag,
                                const int* __restrict__ m_key, const double* __restrict__ xyz,
                                const double* __restrict__ w, float4* __restrict__ pos4,
                                double4* __restrict__ posd, double* __restrict__ wl,
                                int* __restrict__ orig, uint8_t* __restrict__ flags,
                                int* __restrict__ cell_key) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < m;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int k = perm[p];
    const int i = m_orig[k];
    const double x = xyz[3 * (int64_t)i], y = xyz[3 * (int64_t)i + 1], z = xyz[3 * (int64_t)i + 2];
    const uint8_t f = m_flag[k];
    // the fourth component marks buffer points (pair sweeps skip pairs of two)
    pos4[p] = make_float4(__double2float_rn(x), __double2float_rn(y), __double2float_rn(z),
                          (f & FLAG_BUFFER) ? 1.f : 0.f);
    posd[p] = make_double4(x, y, z, w[i]);
    wl[p] = w[i];
    orig[p] = i;
    flags[p] = f;
    cell_key[p] = m_key[k];
  }
}

__global__ void b_narrow_kernel(const int64_t* __restrict__ in, int* __restrict__ out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (int)in[i];
}

// blocks for n items, at most `waves` blocks per SM
int nblocks(int64_t n, int threads, int waves = 8) {
  const int64_t cap = (int64_t)waves * sm_count();
  int64_t b = (n + threads - 1) / threads;
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, cap));
}

}  // namespace

void RegionLayout::release_graph() {
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  exec = nullptr;
  graph = nullptr;
}

RegionLayout::~RegionLayout() { release_graph(); }

// Host-side geometry (first call): region boxes, halos, member counts,
// grids and offsets; sizes every buffer.
void RegionLayout::plan(const double* d_xyz, int64_t n_pts, int64_t n_data_pts, double rmax_,
                        int nsplit_, cudaStream_t s, int sub_policy, double dense_per_cell) {
  release_graph();
  valid = false;
  n = n_pts;
  n_data = n_data_pts;
  rmax = rmax_;
  if (mode == kRegionsSplit) {
    ns = nsplit_;
    nreg = ns * ns * ns;
    sub.reserve(n + 1);
  } else {
    ns = 0;  // nreg and the region of every point were set by set_ids / set_mocks
  }
  box_raw.reserve(6 * (size_t)nreg + 8);
  own_count.reserve(nreg);
  count.reserve(nreg);
  // catalogue box
  {
    unsigned long long init[6] = {~0ull, ~0ull, ~0ull, 0, 0, 0};
    GR_CUDA_TRY(cudaMemcpyAsync(box_raw.p + 6 * (size_t)nreg, init, sizeof(init),
                                cudaMemcpyHostToDevice, s));
    if (n > 0)
      b_bbox_kernel<<<nblocks(n, 256, 2), 256, 0, s>>>(d_xyz, (int)n, box_raw.p + 6 * (size_t)nreg);
    GR_CHECK_LAUNCH();
  }
  unsigned long long hb[6];
  GR_CUDA_TRY(cudaMemcpyAsync(hb, box_raw.p + 6 * (size_t)nreg, sizeof(hb), cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaStreamSynchronize(s));
  SplitGeom sg;
  sg.ns = ns;
  double cat_lo[3], cat_hi[3];
  for (int d = 0; d < 3; ++d) {
    const double lo = n > 0 ? bkey_value(hb[d]) : 0.0, hi = n > 0 ? bkey_value(hb[3 + d]) : 0.0;
    if (!std::isfinite(lo) || !std::isfinite(hi)) throw Error{-1, "non-finite coordinates"};
    cat_lo[d] = lo;
    cat_hi[d] = hi;
    sg.lo[d] = lo;
    const double span = hi - lo;
    sg.inv_span[d] = span > 0 ? 1.0 / span : 0.0;
    // subcubes narrower than Rmax would let a halo reach beyond the
    // neighbouring subcubes
    if (mode == kRegionsSplit && span > 0 && span / ns < rmax)
      throw Error{-1, "regions narrower than rmax; use a smaller split"};
  }
  b_init_box_kernel<<<nblocks(6 * (int64_t)nreg, 256), 256, 0, s>>>(box_raw.p, nreg);
  GR_CUDA_TRY(cudaMemsetAsync(own_count.p, 0, sizeof(int) * nreg, s));
  if (n > 0) {
    if (mode == kRegionsSplit)
      b_region_box_kernel<<<nblocks(n, 256), 256, 0, s>>>(d_xyz, (int)n, sg, sub.p, box_raw.p,
                                                          own_count.p);
    else
      b_region_box_ids_kernel<<<nblocks(n, 256), 256, 0, s>>>(d_xyz, (int)n, sub.p, box_raw.p,
                                                              own_count.p);
  }
  GR_CHECK_LAUNCH();
  std::vector<unsigned long long> hbox(6 * (size_t)nreg);
  std::vector<int> hown(nreg);
  GR_CUDA_TRY(cudaMemcpyAsync(hbox.data(), box_raw.p, sizeof(unsigned long long) * 6 * nreg,
                              cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaMemcpyAsync(hown.data(), own_count.p, sizeof(int) * nreg, cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaStreamSynchronize(s));
  // halos: box +- rmax, strict; empty regions get an empty halo
  h_halo.assign(6 * (size_t)nreg, 0.0);
  for (int r = 0; r < nreg; ++r) {
    if (hown[r] == 0) {
      for (int d = 0; d < 3; ++d) {
        h_halo[6 * r + d] = 1.0;
        h_halo[6 * r + 3 + d] = -1.0;
      }
      continue;
    }
    // mocks have no halo: the region box bounds the mock's own grid
    const double grow = mode == kRegionsMocks ? 0.0 : rmax;
    for (int d = 0; d < 3; ++d) {
      h_halo[6 * r + d] = bkey_value(hbox[6 * r + d]) - grow;
      h_halo[6 * r + 3 + d] = bkey_value(hbox[6 * r + 3 + d]) + grow;
    }
  }
  halo.reserve(6 * (size_t)nreg);
  GR_CUDA_TRY(cudaMemcpyAsync(halo.p, h_halo.data(), sizeof(double) * 6 * nreg, cudaMemcpyHostToDevice, s));
  // region ids: a coarse grid over the catalogue listing, per cell, the
  // regions whose halo reaches it (each point then tests only those)
  ncoarse = 0;
  if (mode == kRegionsIds) {
    ncoarse = make_grid_geom(cat_lo, cat_hi, rmax, 64, (int64_t)1 << 18, coarse);
    std::vector<int> cnt(ncoarse + 1, 0), lst;
    auto cell_range = [&](int r, int d, int& a, int& b) {
      const double lo = coarse.lo[d], inv = coarse.inv_cs[d];
      const int nc = coarse.nc[d];
      a = (int)std::floor((h_halo[6 * r + d] - lo) * inv);
      b = (int)std::floor((h_halo[6 * r + 3 + d] - lo) * inv);
      a = std::min(std::max(a, 0), nc - 1);
      b = std::min(std::max(b, 0), nc - 1);
    };
    for (int pass = 0; pass < 2; ++pass) {
      std::vector<int> fill;
      if (pass == 1) {
        for (int64_t c = 0; c < ncoarse; ++c) cnt[c + 1] += cnt[c];
        lst.assign(cnt[ncoarse], 0);
        fill.assign(cnt.begin(), cnt.end() - 1);
      }
      for (int r = 0; r < nreg; ++r) {
        if (hown[r] == 0) continue;
        int a[3], b[3];
        for (int d = 0; d < 3; ++d) cell_range(r, d, a[d], b[d]);
        for (int z = a[2]; z <= b[2]; ++z)
          for (int y = a[1]; y <= b[1]; ++y)
            for (int x = a[0]; x <= b[0]; ++x) {
              const int64_t c = ((int64_t)z * coarse.nc[1] + y) * coarse.nc[0] + x;
              if (pass == 0)
                cnt[c + 1]++;
              else
                lst[fill[c]++] = r;
            }
      }
    }
    coarse_off.reserve(ncoarse + 1);
    coarse_list.reserve(lst.size() + 1);
    GR_CUDA_TRY(cudaMemcpyAsync(coarse_off.p, cnt.data(), sizeof(int) * (ncoarse + 1),
                                cudaMemcpyHostToDevice, s));
    if (!lst.empty())
      GR_CUDA_TRY(cudaMemcpyAsync(coarse_list.p, lst.data(), sizeof(int) * lst.size(),
                                  cudaMemcpyHostToDevice, s));
    GR_CUDA_TRY(cudaStreamSynchronize(s));  // the host vectors must outlive the copies
  }
  // member counts
  GR_CUDA_TRY(cudaMemsetAsync(count.p, 0, sizeof(int) * nreg, s));
  RegionGeomDev G{};
  G.halo = halo.p;
  G.ns = ns;
  if (n > 0) launch_members(0, d_xyz, G, s);
  GR_CHECK_LAUNCH();
  h_count.assign(nreg, 0);
  GR_CUDA_TRY(cudaMemcpyAsync(h_count.data(), count.p, sizeof(int) * nreg, cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaStreamSynchronize(s));
  h_mem_off.assign(nreg + 1, 0);
  for (int r = 0; r < nreg; ++r) h_mem_off[r + 1] = h_mem_off[r] + h_count[r];
  n_members = h_mem_off[nreg];
  if (n_members >= ((int64_t)1 << 31)) throw Error{-2, "too many region members"};
  // grids over each halo box, cells at least rmax (or rmax/2) wide; cells
  // numbered region by region, largest region first
  auto region_grid = [&](int r, double cell, GridGeom& gg) {
    double lo3[3], hi3[3];
    for (int d = 0; d < 3; ++d) {
      lo3[d] = h_halo[6 * r + d];
      hi3[d] = h_halo[6 * r + 3 + d];
    }
    return make_grid_geom(lo3, hi3, cell, 1024, std::max<int64_t>(4 * (int64_t)h_count[r], 64), gg);
  };
  grid_sub = sub_policy == 2 ? 2 : 1;
  if (sub_policy == 0) {
    int64_t cells1 = 0;
    for (int r = 0; r < nreg; ++r) {
      GridGeom gg;
      if (h_count[r] > 0) cells1 += region_grid(r, rmax, gg);
    }
    grid_sub = (dense_per_cell > 0.0 && cells1 > 0 &&
                (double)n_members / (double)cells1 >= dense_per_cell)
                   ? 2
                   : 1;
  }
  h_grid.assign(nreg, GridParams{1, 1, 1, 1, grid_sub});
  h_glo.assign(3 * (size_t)nreg, 0.0);
  h_ginv.assign(3 * (size_t)nreg, 1.0);
  std::vector<int> order(nreg);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return h_count[a] > h_count[b]; });
  h_cell_off.assign(nreg + 1, 0);
  std::vector<int> cell_region_h;
  int64_t next = 0;
  std::vector<int64_t> off_by_region(nreg, 0);
  for (int k = 0; k < nreg; ++k) {
    const int r = order[k];
    int nc[3] = {1, 1, 1};
    if (h_count[r] > 0) {
      // keep each region's cell table O(its members)
      GridGeom gg;
      region_grid(r, rmax / grid_sub, gg);
      for (int d = 0; d < 3; ++d) {
        nc[d] = gg.nc[d];
        h_glo[3 * r + d] = gg.lo[d];
        h_ginv[3 * r + d] = gg.inv_cs[d];
      }
    }
    const int64_t cells = h_count[r] > 0 ? (int64_t)nc[0] * nc[1] * nc[2] : 0;
    h_grid[r] = GridParams{nc[0], nc[1], nc[2], cells, grid_sub};
    off_by_region[r] = next;
    cell_region_h.insert(cell_region_h.end(), (size_t)cells, r);
    next += cells;
  }
  ncell = next;
  if (ncell >= ((int64_t)1 << 31)) throw Error{-2, "too many cells"};
  for (int r = 0; r < nreg; ++r) h_cell_off[r] = (int)off_by_region[r];
  h_cell_off[nreg] = (int)ncell;
  // device geometry
  glo.reserve(3 * (size_t)nreg);
  ginv.reserve(3 * (size_t)nreg);
  grid.reserve(nreg);
  cell_off.reserve(nreg + 1);
  cell_region.reserve(ncell + 1);
  GR_CUDA_TRY(cudaMemcpyAsync(glo.p, h_glo.data(), sizeof(double) * 3 * nreg, cudaMemcpyHostToDevice, s));
  GR_CUDA_TRY(cudaMemcpyAsync(ginv.p, h_ginv.data(), sizeof(double) * 3 * nreg, cudaMemcpyHostToDevice, s));
  GR_CUDA_TRY(cudaMemcpyAsync(grid.p, h_grid.data(), sizeof(GridParams) * nreg, cudaMemcpyHostToDevice, s));
  GR_CUDA_TRY(cudaMemcpyAsync(cell_off.p, h_cell_off.data(), sizeof(int) * (nreg + 1), cudaMemcpyHostToDevice, s));
  if (ncell > 0)
    GR_CUDA_TRY(cudaMemcpyAsync(cell_region.p, cell_region_h.data(), sizeof(int) * ncell,
                                cudaMemcpyHostToDevice, s));
  // member and layout buffers
  const int64_t M = n_members;
  mcount.reserve(n + 1);
  moff.reserve(n + 1);
  m_orig.reserve(M + 1);
  m_flag.reserve(M + 1);
  m_key.reserve(M + 1);
  m_slot.reserve(M + 1);
  tmp_perm.reserve(M + 1);
  perm.reserve(M + 1);
  cell_count.reserve(ncell + 1);
  cell_start64.reserve(ncell + 1);
  cell_start.reserve(ncell + 1);
  pos4.reserve(M + 1);
  posd.reserve(M + 1);
  w.reserve(M + 1);
  orig.reserve(M + 1);
  flags.reserve(M + 1);
  cell_key.reserve(M + 1);
  GR_CUDA_TRY(cudaStreamSynchronize(s));  // host vectors above must outlive the copies
  valid = true;
}

// Device work of one call (no host synchronisation; capturable).
void RegionLayout::enqueue_layout(const double* d_xyz, const double* d_w, cudaStream_t s) {
  RegionGeomDev G;
  G.halo = halo.p;
  G.glo = glo.p;
  G.ginv = ginv.p;
  G.grid = grid.p;
  G.cell_off = cell_off.p;
  G.ns = ns;
  GR_CUDA_TRY(cudaMemsetAsync(cell_count.p, 0, sizeof(int) * (ncell + 1), s));
  if (n > 0) {
    // memberships per point, their offsets, then the members themselves
    launch_members(1, d_xyz, G, s);
    scan_i32_to_i64(mcount.p, moff.p, n, s, scan_tmp);
    launch_members(2, d_xyz, G, s);
  }
  GR_CHECK_LAUNCH();
  scan_i32_to_i64(cell_count.p, cell_start64.p, ncell, s, scan_tmp);
  if (n_members > 0) {
    b_scatter_kernel<<<nblocks(n_members, 256), 256, 0, s>>>(n_members, m_key.p, m_slot.p,
                                                             cell_start64.p, tmp_perm.p);
    b_order_kernel<<<nblocks(ncell * 32, 256, 16), 256, 0, s>>>(ncell, cell_start64.p,
                                                                      tmp_perm.p, m_orig.p, perm.p);
    b_gather_kernel<<<nblocks(n_members, 256), 256, 0, s>>>(n_members, perm.p, m_orig.p, m_flag.p,
                                                            m_key.p, d_xyz, d_w, pos4.p, posd.p,
                                                            w.p, orig.p, flags.p, cell_key.p);
  }
  b_narrow_kernel<<<nblocks(ncell + 1, 256), 256, 0, s>>>(cell_start64.p, cell_start.p, ncell + 1);
  GR_CHECK_LAUNCH();
}

void RegionLayout::launch_members(int pass, const double* d_xyz, const RegionGeomDev& G,
                                  cudaStream_t s) {
  const CoarseDev CG = coarse_dev();
  const uint8_t* pf = mode == kRegionsMocks ? pflag.p : nullptr;
  const int blocks = nblocks(n, 256);
#define GR_MEM_LAUNCH(P, M)                                                                     \
  b_members_kernel<P, M><<<blocks, 256, 0, s>>>(d_xyz, (int)n, (int)n_data, sub.p, pf, G, CG,    \
                                                count.p, mcount.p, moff.p, m_orig.p, m_flag.p,   \
                                                m_key.p, m_slot.p, cell_count.p)
#define GR_MEM_MODE(P)                                                                          \
  do {                                                                                          \
    if (mode == kRegionsSplit) GR_MEM_LAUNCH(P, kMemSplit);                                     \
    else if (mode == kRegionsIds) GR_MEM_LAUNCH(P, kMemIds);                                    \
    else GR_MEM_LAUNCH(P, kMemMocks);                                                           \
  } while (0)
  if (pass == 0) GR_MEM_MODE(0);
  else if (pass == 1) GR_MEM_MODE(1);
  else GR_MEM_MODE(2);
#undef GR_MEM_MODE
#undef GR_MEM_LAUNCH
  GR_CHECK_LAUNCH();
}

CoarseDev RegionLayout::coarse_dev() const {
  CoarseDev c{};
  if (mode != kRegionsIds || ncoarse == 0) return c;  // list null: own region only
  c.off = coarse_off.p;
  c.list = coarse_list.p;
  for (int d = 0; d < 3; ++d) {
    c.lo[d] = coarse.lo[d];
    c.inv[d] = coarse.inv_cs[d];
    c.nc[d] = coarse.nc[d];
  }
  return c;
}

void RegionLayout::set_ids(const int* h_ids, int64_t n_pts, int nregions, cudaStream_t s) {
  if (nregions < 1) throw Error{-1, "need at least one region"};
  for (int64_t i = 0; i < n_pts; ++i)
    if (h_ids[i] < 0 || h_ids[i] >= nregions) throw Error{-1, "region id out of range"};
  release_graph();
  sub.reserve(n_pts + 1);
  if (n_pts > 0) {
    GR_CUDA_TRY(cudaMemcpyAsync(sub.p, h_ids, sizeof(int) * n_pts, cudaMemcpyHostToDevice, s));
    GR_CUDA_TRY(cudaStreamSynchronize(s));
  }
  mode = kRegionsIds;
  nreg = nregions;
  valid = false;
}

void RegionLayout::set_mocks(const int64_t* nd, const int64_t* nr, int nmocks, int64_t n_pts,
                             cudaStream_t s) {
  if (nmocks < 1) throw Error{-1, "need at least one mock"};
  int64_t tot = 0;
  for (int m = 0; m < nmocks; ++m) {
    if (nd[m] < 0 || nr[m] < 0) throw Error{-1, "negative mock size"};
    tot += nd[m] + nr[m];
  }
  if (tot != n_pts) throw Error{-1, "mock sizes do not add up to the catalogue"};
  std::vector<int> ids(n_pts + 1);
  std::vector<uint8_t> fl(n_pts + 1);
  int64_t i = 0;
  for (int m = 0; m < nmocks; ++m) {
    for (int64_t k = 0; k < nd[m]; ++k, ++i) {
      ids[i] = m;
      fl[i] = 0;
    }
    for (int64_t k = 0; k < nr[m]; ++k, ++i) {
      ids[i] = m;
      fl[i] = FLAG_RANDOM;
    }
  }
  release_graph();
  sub.reserve(n_pts + 1);
  pflag.reserve(n_pts + 1);
  if (n_pts > 0) {
    GR_CUDA_TRY(cudaMemcpyAsync(sub.p, ids.data(), sizeof(int) * n_pts, cudaMemcpyHostToDevice, s));
    GR_CUDA_TRY(cudaMemcpyAsync(pflag.p, fl.data(), n_pts, cudaMemcpyHostToDevice, s));
    GR_CUDA_TRY(cudaStreamSynchronize(s));
  }
  mode = kRegionsMocks;
  nreg = nmocks;
  valid = false;
}

DevCatalog RegionLayout::view() const {
  DevCatalog c;
  c.pos4 = pos4.p;
  c.posd = posd.p;
  c.w = w.p;
  c.orig = orig.p;
  c.flags = flags.p;
  c.cell_key = cell_key.p;
  c.cell_start = cell_start.p;
  c.n = (int)n_members;
  c.n_data = (int)n_data;
  c.grid = GridParams{1, 1, 1, ncell, grid_sub};
  c.cell_region = cell_region.p;
  c.region_grid = grid.p;
  c.region_cell_off = cell_off.p;
  return c;
}

}  // namespace gr
