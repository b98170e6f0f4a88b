// Launchers of the counting kernels.
#pragma once

#include "gr_index.cuh"

namespace gr {

// Shared-memory budget for a privatised histogram; larger histograms are
// accumulated with global atomics instead.
constexpr size_t kMaxHistSmem = 120 * 1024;

// Weighted sums (g_fix / d_fix below) are fixed-point (lo, hi) pairs: the
// nh lo words followed by the nh hi words, scale fscale (fix_add).

// 2PCF: pairs binned straight from the half-stencil cell sweep.
// g_cnt (nh = nbins*nmu*4) and g_fix (2*nh, weighted only) must be zeroed.
// stats: [0] FP64 rechecks, [1] candidates, [2] binned unordered pairs.
// variant: kPairWarpCell (warp per cell, lanes over candidates; sparse
// cells) or kPairDense128/256 (block per cell, thread per root, broadcast
// candidates; dense cells).  The autotuner picks one per workload class.
// kPairWarpQueue / kPairDenseQ128/256: the same sweeps with a
// membership-only test per candidate and the binning of the edges queued and
// run with full warps.
// kPairTile: the tile sweep (gr_tile.cu) on cells at least rmax wide;
// kPairTile2: the same on cells at least rmax/2 wide (the only variant that
// reads such grids).
enum {
  kPairWarpCell = 0,
  kPairDense128 = 1,
  kPairDense256 = 2,
  kPairWarpQueue = 3,
  kPairDenseQ128 = 4,
  kPairDenseQ256 = 5,
  kPairTile = 6,
  kPairTile2 = 7,
  kPairVariants = 8
};
// Points per rmax-wide cell from which the 2PCF sweeps use cells of rmax/2
// and the tile sweep.
constexpr double kDenseCellPoints = 64.0;
size_t pair2_smem_bytes(const PairParams& P, bool weighted);

// Tile sweep for dense cells (gr_tile.cu): warp per cell, lanes over 32
// roots, candidates staged 32 at a time per warp and tested two per packed
// FP32x2 instruction (FP64 path: one per FP64 test), hits binned from a
// per-warp queue; reads grids with cells at least rmax wide (sub 1) or rmax/2
// wide (sub 2).  Same inputs, outputs and results as launch_pair2.
// Histograms private to each warp in shared memory when they need at most
// kMaxTileHistSmem bytes.  per_region (region layouts only): one histogram
// per region, g_cnt nregions*nh and g_fix nregions*2*nh (region r's lo
// words at 2*r*nh, hi words at 2*r*nh + nh), all zeroed.
constexpr size_t kMaxTileHistSmem = 160 * 1024;
size_t pair2_tile_smem_bytes(const PairParams& P, bool weighted);
void launch_pair2_tile(const DevCatalog& C, const PairParams& P, bool weighted,
                       unsigned long long* g_cnt, unsigned long long* g_fix, double fscale,
                       unsigned long long* stats, int* work, cudaStream_t s,
                       bool per_region = false);
void launch_pair2(const DevCatalog& C, const PairParams& P, bool weighted,
                  unsigned long long* g_cnt, unsigned long long* g_fix, double fscale,
                  unsigned long long* stats, int* work, cudaStream_t s, int variant = kPairWarpCell);

struct TriParams {
  int nbins, nmu, ncfg, rsd;
  int equi;                // -equi: only triangles with three equal bins, ncfg = nbins
  int cap;                 // per-warp shared row capacity (rows longer go the global path)
  const uint8_t* normal;   // device find_normal table [mu1-1 + nmu*(mu2-1)]
  RankTables rank;         // 3-tuple ranks
  double fscale[4];        // fixed-point scale of the products with 0..3 randoms
  PairParams P;            // edge predicate and binning of the graph
  int geo;                 // 1: third edges by the geometric pair test, 0: hash probes of rows
  int maxdeg;              // longest upper row
  int long_geo;            // 1: rows beyond cap take a second, geometric launch
  int kmin, kskip;         // roots handled by one launch: kmin < row length <= kskip
};

// 3PCF: triangles p < a < c enumerated once over the upper CSR; each adds to
// the rooted histogram of every non-buffer vertex.  g_cnt (nh = ncfg*nmu*4,
// when counts) and g_lim (2*nh: 128-bit fixed-point sums, lo words then hi
// words, weighted only) must be zeroed.  stats: [0] distinct triangles binned, [1] rooted
// incidences, [2] intersection probes.
// work: one device int used as the dynamic root counter (reset by the launch).
// Returns the number of kernel launches (2 when long rows take a second one).
size_t tri3_smem_bytes(const TriParams& T, bool weighted, bool counts);
int launch_tri3(const DevCatalog& C, const CSRView& G, const TriParams& T, bool weighted,
                 bool counts, unsigned long long* g_cnt, unsigned long long* g_lim,
                 unsigned long long* stats, int* work, cudaStream_t s);

// Weight adjoints: gradient of sum(cot2 * N2) + sum(cot3 * N3) with respect
// to the weights, as 128-bit fixed-point sums (g_lo, g_hi, label order; the
// 2PCF adjoint writes every entry, the 3PCF adjoint needs them zeroed) of
// scale gscale; launch_grad_finish converts them to
// FP64 in catalogue order.  cot3 may be NULL.
void launch_adj2(const DevCatalog& C, const PairParams& P, const double* cot2, const double* cot3,
                 double gscale, unsigned long long* g_lo, unsigned long long* g_hi, int* work,
                 cudaStream_t s, int variant = kPairWarpCell);
int launch_adj3(const DevCatalog& C, const CSRView& G, const TriParams& T, const double* cot2,
                 const double* cot3, double gscale, unsigned long long* g_lo,
                 unsigned long long* g_hi, unsigned long long* stats, int* work, cudaStream_t s);
// The same adjoint with the tile sweep (gr_tile.cu): half stencil, both ends
// of every edge updated; g_lo / g_hi must be zeroed.  Per-warp 64-bit
// partials take at most 32 terms each before they are merged, so gscale
// needs 2^6 of headroom over the largest term: fix_scale(64 * term bound).
// stats as launch_pair2 (zeroed).
void launch_adj2_tile(const DevCatalog& C, const PairParams& P, const double* cot2,
                      const double* cot3, double gscale, unsigned long long* g_lo,
                      unsigned long long* g_hi, unsigned long long* stats, int* work,
                      cudaStream_t s);
void launch_grad_finish(int n, const int* orig, const unsigned long long* g_lo,
                        const unsigned long long* g_hi, double gscale, double* grad,
                        cudaStream_t s);

// 8-byte words per entry of the 4PCF kernels' global fixed-point sums
// (g_fix, d_fix): 16, one 128-byte line per entry.
#ifndef GR_FIX_STRIDE
#define GR_FIX_STRIDE 16
#endif
constexpr int kFixStride = GR_FIX_STRIDE;

struct QuadParams {
  int nbins, ncfg;
  int tetra;  // -tetra: only 4-cliques with six equal bins (histograms by bin)
  int cap;
  RankTables rank;  // 4-tuple ranks
  PairParams P;     // edge predicate and binning of the graph
  int geo;          // 1: edges among R+(p) by the geometric pair test (cap <= 256)
  int split;        // weighted sums as split limbs without returned values (fix_red);
                    // exact while every bin receives fewer than 2^32 updates
  int counts;       // integer counts kept (always for unweighted catalogues)
  const int* order; // roots in the order the work counter hands them out
                    // (order_roots_by_length), or null: label order
  const int* above;  // with order: above[b] = the number of roots whose row
                     // length class (min(length, nclass - 1)) exceeds b, or null
  int nclass;
};

// -tetra histograms (tetra = 1): g_cnt nbins*5, d_cnt nbins*30 (6 terms x 5
// categories: 0..3 number of randoms in the 3-product, 4 = discR).
// 4PCF: 4-cliques p < a < b < c enumerated once; each adds to the rooted
// histograms of its non-buffer vertices whose perimeter is canonical.
// g_cnt: nh = ncfg*nbins*nbins*5 (g_fix 2*nh); d_cnt: nd = ncfg*nbins*nbins*24 (d_fix 2*nd).
// stats (4 entries, zeroed): [0] distinct 4-cliques binned, [1] rooted
// incidences, [2] probes, [3] set when a root's label offsets exceed the
// hash key range (the host reports it).  work: one device int, the dynamic
// root counter (reset by the launch).
// The outputs (g_cnt nh, g_fix 2 nh, d_cnt nd, d_fix 2 nd entries, the fix
// arrays kFixStride words per entry and only when weighted) must be zeroed; the last disc category (discR, equal to the
// all-random one before it) is not written, nd covers the others.
// shared_counts: integer counts in block-private 32-bit shared-memory
// counters (exact while the rooted total stays below 2^32; the caller
// checks stats[1] and reruns without them otherwise).  Returns whether the
// shared counters were used.
bool launch_quad4(const DevCatalog& C, const CSRView& G, const QuadParams& Q, bool weighted,
                  unsigned long long* g_cnt, unsigned long long* g_fix, unsigned long long* d_cnt,
                  unsigned long long* d_fix, int nh, int nd, double fscale, double dscale,
                  bool shared_counts, unsigned long long* stats, int* work, cudaStream_t s);
// Unit-weight 4PCF (tetra = 0, not weighted): the kernels count each rooted
// clique once at (histogram index kk, pattern), pattern = the randomness of
// the root and of the other three vertices in catalogue-id order (bits 0..3);
// g_cnt then holds kQuadPatterns * nbin entries (nh = that, nd = 0).
// quad_expand_patterns forms from them the N2 / N3 counts hc (5 * nbin, by
// number of randoms) and the disconnected-term counts dc (6 * 3 * nbin: term,
// randoms in the pair; a term counts when its gating role is random), as the
// kernels otherwise accumulate them.
constexpr int kQuadPatterns = 16;
void quad_expand_patterns(const unsigned long long* H, int nbin, unsigned long long* hc,
                          unsigned long long* dc);
// 4PCF adjoint: gradient of sum(cot2 N2) + sum(cot3 N3) + sum(cotN discN)
// + sum(cotR discR), cot = [cot2 nbin | cot3 nbin | cotN 6 nbin | cotR 6 nbin]
// (nbin = ncfg nbins^2), into g_lo / g_hi (label order, zeroed) at scale
// gscale.  Q as for launch_quad4 with tetra = 0.
void launch_adj4(const DevCatalog& C, const CSRView& G, const QuadParams& Q, const double* cot,
                 double gscale, unsigned long long* g_lo, unsigned long long* g_hi,
                 unsigned long long* stats, int* work, cudaStream_t s);

}  // namespace gr
