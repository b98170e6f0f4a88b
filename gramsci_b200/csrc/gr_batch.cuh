// Batched regions (domain decomposition in one launch), see gr_batch.cu.
#pragma once

#include <vector>

#include "gr_kernels.cuh"

namespace gr {

// Catalogue-wide coarse grid of candidate regions (region-id layouts): cell
// c lists in list[off[c] .. off[c+1]) the regions whose halo reaches it; a
// null list means no halos (every point belongs to its own region only).
struct CoarseDev {
  const int* off;
  const int* list;
  double lo[3], inv[3];
  int nc[3];
};

// Region geometry read by the membership kernels.
struct RegionGeomDev {
  const double* halo;    // 6 per region: lo xyz, hi xyz (strict bounds)
  const double* glo;     // 3 per region: grid origin
  const double* ginv;    // 3 per region: inverse cell size
  const GridParams* grid;
  const int* cell_off;   // nreg + 1
  int ns;                // subcubes per axis (subcube split)
};

// How the catalogue is split into regions.
enum : int {
  kRegionsSplit = 0,  // nsplit^3 equal subcubes of the bounding box, Rmax halos
  kRegionsIds = 1,    // a region id per point (e.g. jackknife regions), Rmax halos
  kRegionsMocks = 2   // independent catalogues one after another, no halos
};

struct RegionLayout {
  bool valid = false;
  int mode = kRegionsSplit;
  int ns = 0, nreg = 0;
  int64_t n = 0, n_data = 0, n_members = 0, ncell = 0;
  double rmax = 0.0;
  // host geometry
  std::vector<double> h_halo, h_glo, h_ginv;
  std::vector<GridParams> h_grid;
  std::vector<int> h_count, h_cell_off;
  std::vector<int64_t> h_mem_off;
  // ids / mocks: the region of every point (in `sub`) and, for mocks, the
  // random flag of every point
  DevBuf<uint8_t> pflag;
  // ids: coarse grid over the catalogue; cell c lists the regions whose halo
  // reaches it (coarse_off[c] .. coarse_off[c+1] in coarse_list)
  GridGeom coarse{};
  int64_t ncoarse = 0;
  DevBuf<int> coarse_off, coarse_list;
  // device geometry
  DevBuf<unsigned long long> box_raw;
  DevBuf<int> own_count, count, sub, cell_off, cell_region;
  DevBuf<int> mcount;      // memberships of every point
  DevBuf<int64_t> moff;    // their exclusive scan (where each point's members go)
  DevBuf<double> halo, glo, ginv;
  DevBuf<GridParams> grid;
  // members and layout
  DevBuf<int> m_orig, m_key, m_slot, tmp_perm, perm, cell_count, cell_start, orig, cell_key;
  DevBuf<uint8_t> m_flag, flags;
  DevBuf<int64_t> cell_start64, scan_tmp;
  DevBuf<float4> pos4;
  DevBuf<double4> posd;
  DevBuf<double> w;
  // replay of the per-call device work
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;

  ~RegionLayout();
  void release_graph();
  // grid_sub: region grids of cells at least rmax (1) or rmax/2 (2) wide;
  // plan's sub_policy 0 picks 2 when the rmax-wide grids would hold at least
  // dense_per_cell members per cell
  int grid_sub = 1;
  void plan(const double* d_xyz, int64_t n, int64_t n_data, double rmax, int nsplit, cudaStream_t s,
            int sub_policy = 1, double dense_per_cell = 0.0);
  // ids: region of every point (host array of n entries in [0, nregions));
  // mocks: galaxies and randoms of each mock, the catalogue being the mocks
  // one after another, each with its galaxies first.  Both replace the
  // subcube split until set_split is called.
  void set_ids(const int* h_ids, int64_t n, int nregions, cudaStream_t s);
  void set_mocks(const int64_t* n_data, const int64_t* n_rand, int nmocks, int64_t n, cudaStream_t s);
  void set_split() {
    mode = kRegionsSplit;
    valid = false;
  }
  void enqueue_layout(const double* d_xyz, const double* d_w, cudaStream_t s);
  DevCatalog view() const;
  CoarseDev coarse_dev() const;
  // membership kernels (pass 0: members per region, 1: memberships per
  // point, 2: the members)
  void launch_members(int pass, const double* d_xyz, const RegionGeomDev& G, cudaStream_t s);
};

}  // namespace gr
