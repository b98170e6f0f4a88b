// Device cell index and upper-triangular CSR adjacency.
#pragma once

// candidates staged per warp and tile by the cell sweeps
#define kCellTile 256

#include <algorithm>
#include <cstring>

#include "gr_internal.cuh"

namespace gr {

// Uniform-grid index over the catalogue, points laid out in cell order.
struct CellIndex {
  int64_t n = 0, n_data = 0;
  double coord_max = 0.0;  // max |coordinate|, bounds the FP32 rounding error
  GridParams grid{};
  int launches = 0;
  DevBuf<unsigned long long> bbox_raw;
  // Speculative build: the grid depends only on the bounding box, the point
  // count and rmax, so a build may take the previous build's bounding box
  // without waiting for the new one and let a device check record whether
  // it differs (bbox_prev[7] = 1); the caller reads the flag with its results
  // and rebuilds without speculation when it is set.
  bool have_prev = false, speculated = false;
  int64_t prev_n = -1;
  double prev_rmax = 0.0;
  int prev_sub = 0;
  bool prev_auto = false;  // the previous build chose sub itself
  unsigned long long prev_raw[7] = {0, 0, 0, 0, 0, 0, 0};
  DevBuf<unsigned long long> bbox_prev;  // previous raw bounding box [0..6], mismatch flag [7]
  DevBuf<int> cell_count, key_orig, slot, tmp_perm, cell_start, orig, cell_key;
  DevBuf<int64_t> cell_start64, scan_tmp;
  DevBuf<float4> pos4;
  DevBuf<double4> posd;
  DevBuf<double> w;
  DevBuf<uint8_t> flags;

  // sub = 1: cells at least rmax wide; sub = 2: at least rmax/2 wide (for
  // the tile pair sweep); sub = 0: 2 when an rmax-wide grid would hold at
  // least dense_per_cell points per cell, else 1.
  void build(const double* d_xyz, const double* d_w, const int* d_buffer, int64_t n, int64_t n_data,
             double rmax, cudaStream_t s, bool speculate = false, int sub = 1,
             double dense_per_cell = 0.0);
  double per_cell_rmax = 0.0;  // points per cell of an rmax-wide grid (last build)
  const unsigned long long* mismatch_flag() const { return bbox_prev.p + 7; }
  DevCatalog view() const;
};


// Upper adjacency: row p lists the neighbours q > p (internal labels) of the
// (rmin, rmax) graph in increasing label order, with packed bin / mu
// metadata.  deg_full[p] is the full degree (the reference's row length nn).
// Rows live in `scratch` at rstart[p] with deg_up[p] records (per-cell
// candidate-bound layout, with gaps); compact() also lays them out as a
// classic CSR (row_ptr, rec) for export and persistence.
struct CSRView {
  const int64_t* start;           // first record of row p
  const int* len;                 // records in row p
  const unsigned long long* rec;  // (meta << 32) | neighbour label
  const int* deg_full;
};

// Roots ordered by upper row length, longest first (lengths above cap share
// the first class), into order[0..n): the counting kernels hand roots out in
// this order so that the costliest start first and no warp ends a launch on
// one of them.  scratch: cap + 1 device ints.
void order_roots_by_length(const CSRView& G, int n, int cap, int* order, int* scratch,
                           cudaStream_t s);

struct UpperCSR {
  int64_t n = 0, n_edges = 0;  // n_edges counts upper (undirected) edges
  int64_t max_deg = 0;         // largest upper degree
  int64_t rechecks = 0, candidates = 0;
  int launches = 0;
  bool compacted = false;      // row_ptr / rec hold the current rows
  DevBuf<int> deg_up, deg_full, work;
  DevBuf<int64_t> row_ptr, scan_tmp, rstart, cbound, cbase;
  DevBuf<unsigned long long> rec;      // compacted rows (compact())
  DevBuf<unsigned long long> scratch;  // rows as built: rstart / deg_up
  DevBuf<unsigned long long> stats;    // [0] FP64 rechecks, [1] candidates, [2] max upper degree
  DevBuf<unsigned long long> ctl;      // [1] out of room, [2] disagreements, [3] edges
  // speculate: one fill with the scratch area as it is and no wait; the
  // caller reads ctl[0..3] and stats[0..2] with its results, calls settle()
  // and rebuilds without speculation when ctl[1] == 1 (out of room).
  void build(const DevCatalog& C, const PairParams& P, cudaStream_t s, bool speculate = false);
  void settle(const unsigned long long hc[4], const unsigned long long hs[3]);
  void compact(cudaStream_t s);
  CSRView view() const { return CSRView{rstart.p, deg_up.p, scratch.p, deg_full.p}; }
};

__device__ __forceinline__ int rec_col(unsigned long long r) { return (int)(uint32_t)r; }
__device__ __forceinline__ uint32_t rec_meta(unsigned long long r) { return (uint32_t)(r >> 32); }

}  // namespace gr
