// Batched regions (domain decomposition in one launch), see gr_batch.cu.
#pragma once

#include <vector>

#include "gr_kernels.cuh"

namespace gr {

struct RegionLayout {
  bool valid = false;
  int ns = 0, nreg = 0;
  int64_t n = 0, n_data = 0, n_members = 0, ncell = 0;
  double rmax = 0.0;
  // host geometry
  std::vector<double> h_halo, h_glo, h_ginv;
  std::vector<GridParams> h_grid;
  std::vector<int> h_count, h_cell_off;
  std::vector<int64_t> h_mem_off;
  // device geometry
  DevBuf<unsigned long long> box_raw;
  DevBuf<int> own_count, count, sub, cell_off, mem_off, cell_region;
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
  void enqueue_layout(const double* d_xyz, const double* d_w, cudaStream_t s);
  DevCatalog view() const;
};

}  // namespace gr
