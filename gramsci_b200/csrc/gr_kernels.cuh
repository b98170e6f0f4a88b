// Launchers of the counting kernels.
#pragma once

#include "gr_index.cuh"

namespace gr {

// Shared-memory budget for a privatised histogram; larger histograms are
// accumulated with global atomics instead.
constexpr size_t kMaxHistSmem = 96 * 1024;

// 2PCF: pairs binned straight from the half-stencil cell sweep.
// g_cnt (nbins*nmu*4) and g_sum (same, weighted only) must be zeroed.
// stats: [0] FP64 rechecks, [1] candidates, [2] binned unordered pairs.
size_t pair2_smem_bytes(const PairParams& P, bool weighted);
void launch_pair2(const DevCatalog& C, const PairParams& P, bool weighted,
                  unsigned long long* g_cnt, double* g_sum, unsigned long long* stats,
                  cudaStream_t s);

struct TriParams {
  int nbins, nmu, ncfg, rsd;
  int cap;                 // per-warp shared row capacity (rows longer go the global path)
  const uint8_t* normal;   // device find_normal table [mu1-1 + nmu*(mu2-1)]
  RankTables rank;         // 3-tuple ranks
};

// 3PCF: triangles p < a < c enumerated once over the upper CSR; each adds to
// the rooted histogram of every non-buffer vertex.  g_cnt / g_sum have
// ncfg*nmu*4 entries.  stats: [0] distinct triangles binned, [1] rooted
// incidences, [2] intersection probes.
void launch_tri3(const DevCatalog& C, const CSRView& G, const TriParams& T, bool weighted,
                 unsigned long long* g_cnt, double* g_sum, unsigned long long* stats,
                 cudaStream_t s);

struct QuadParams {
  int nbins, ncfg;
  int cap;
  RankTables rank;  // 4-tuple ranks
};

// 4PCF: 4-cliques p < a < b < c enumerated once; each adds to the rooted
// histograms of its non-buffer vertices whose perimeter is canonical.
// g_cnt/g_sum: ncfg*nbins*nbins*5; d_cnt/d_sum: ncfg*nbins*nbins*24.
// stats: [0] distinct 4-cliques binned, [1] rooted incidences, [2] probes.
void launch_quad4(const DevCatalog& C, const CSRView& G, const QuadParams& Q, bool weighted,
                  unsigned long long* g_cnt, double* g_sum, unsigned long long* d_cnt,
                  double* d_sum, unsigned long long* stats, cudaStream_t s);

}  // namespace gr
