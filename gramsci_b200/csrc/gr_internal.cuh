// Internal declarations shared by the CUDA translation units of
// libgramsci_cuda.so: the pair predicate (FP32 fast path with an FP64 guard
// band, and the exact FP64 reference form), cell-grid helpers, tuple-rank
// tables and small device utilities.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <string>
#include <vector>

namespace gr {

// ------------------------------------------------------------------ errors --
struct Error {
  int code;
  std::string msg;
};

#define GR_CUDA_TRY(call)                                                     \
  do {                                                                        \
    cudaError_t _e = (call);                                                  \
    if (_e != cudaSuccess)                                                    \
      throw ::gr::Error{-3, std::string(#call) + ": " + cudaGetErrorString(_e)}; \
  } while (0)

#define GR_CHECK_LAUNCH() GR_CUDA_TRY(cudaGetLastError())

// ------------------------------------------------------------ device buffer --
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;  // capacity in elements
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  // Grow to at least `count` elements (contents are not preserved).
  void reserve(size_t count) {
    if (count <= n && p) return;
    release();
    size_t c = count > 0 ? count : 1;
    GR_CUDA_TRY(cudaMalloc(&p, c * sizeof(T)));
    n = c;
  }
};

// Pinned host memory for the results a call reads back: copies into it are
// asynchronous, so one stream synchronisation covers all of them (a copy
// into pageable memory blocks the host once per copy).
template <typename T>
struct HostBuf {
  T* p = nullptr;
  size_t n = 0;  // capacity in elements
  HostBuf() = default;
  HostBuf(const HostBuf&) = delete;
  HostBuf& operator=(const HostBuf&) = delete;
  ~HostBuf() { release(); }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    n = 0;
  }
  void reserve(size_t count) {
    if (count <= n && p) return;
    release();
    size_t c = count > 0 ? count : 1;
    GR_CUDA_TRY(cudaMallocHost(&p, c * sizeof(T)));
    n = c;
  }
};

// ------------------------------------------------------------ pair predicate --
// Everything a kernel needs to decide whether (i, j) is an edge of the
// reference graph and which radial / mu bins it falls in.
struct PairParams {
  // exact FP64 form (src/gramsci.F90:136-147, 295-340)
  double rmin, rmax, rmin2, rmax2, inv_dr, log_rmin, mu_scale;
  int nbins, nmu, logbins, rsd;
  // FP32 fast path with guard band
  int f32;           // 1 = FP32 path enabled
  float f_rmin, f_inv_dr, f_mu_scale;
  float rmax2_hi;    // d2 >= rmax2_hi: certainly d >= rmax
  float rmin2_lo;    // d2 <= rmin2_lo: certainly d <= rmin (or -1)
  float rmax2_lo;    // d2 < rmax2_lo: certainly d < rmax (or -1)
  float rmin2_hi;    // d2 > rmin2_hi: certainly d > rmin
  float tguard;      // |t - nearest integer| below this -> FP64
  float d0;          // bound on |d_f - d_true|
  float eA, eB, mB, eC;  // cosine error model eA/(d-d0) + eB/(|m|-mB) + eC
  float f_nmu;
};

// Host: fill PairParams.  coord_max bounds |x|,|y|,|z| over the catalogue.
void make_pair_params(PairParams& P, double rmin, double rmax, int nbins, int nmu, int logbins,
                      double coord_max, int force_fp64);

__device__ __forceinline__ int mu_bin_f64(double th, const PairParams& P) {
  double v = __dmul_rn(__dadd_rn(th, 1.0), P.mu_scale);
  if (!(v == v)) return 1;
  double f = floor(v);
  if (f < -1.0e9) return 1;
  if (f > 1.0e9) return P.nmu;
  int m = (int)f + 1;
  m = m < 1 ? 1 : m;
  m = m > P.nmu ? P.nmu : m;
  return m;
}

// Exact reference predicate in FP64 (separate IEEE multiply / add, no FMA),
// root pi, neighbour pj.  Identical arithmetic to the CPU oracle.
__device__ __forceinline__ bool edge_f64(const double4 pi, const double4 pj, const PairParams& P,
                                         int& bin, int& muf, int& mur) {
  double dx = __dsub_rn(pj.x, pi.x);
  double dy = __dsub_rn(pj.y, pi.y);
  double dz = __dsub_rn(pj.z, pi.z);
  double sd = __dmul_rn(dx, dx);
  sd = __dadd_rn(sd, __dmul_rn(dy, dy));
  sd = __dadd_rn(sd, __dmul_rn(dz, dz));
  if (sd > P.rmax2) return false;
  if (P.rmin > 0.0 && sd <= P.rmin2) return false;
  double d = __dsqrt_rn(sd);
  if (d <= P.rmin || d >= P.rmax) return false;
  double t;
  if (P.logbins)
    t = __dmul_rn(__dsub_rn(log10(d), P.log_rmin), P.inv_dr);
  else
    t = __dmul_rn(__dsub_rn(d, P.rmin), P.inv_dr);
  int b = (int)floor(t) + 1;
  b = b > P.nbins ? P.nbins : b;
  b = b < 1 ? 1 : b;
  bin = b;
  if (P.rsd) {
    double m0 = __dmul_rn(0.5, __dadd_rn(pi.x, pj.x));
    double m1 = __dmul_rn(0.5, __dadd_rn(pi.y, pj.y));
    double m2 = __dmul_rn(0.5, __dadd_rn(pi.z, pj.z));
    double s0 = __dsub_rn(pi.x, pj.x);
    double s1 = __dsub_rn(pi.y, pj.y);
    double s2 = __dsub_rn(pi.z, pj.z);
    double th = __dmul_rn(m0, s0);
    th = __dadd_rn(th, __dmul_rn(m1, s1));
    th = __dadd_rn(th, __dmul_rn(m2, s2));
    double nm = __dmul_rn(m0, m0);
    nm = __dadd_rn(nm, __dmul_rn(m1, m1));
    nm = __dadd_rn(nm, __dmul_rn(m2, m2));
    double ns = __dmul_rn(s0, s0);
    ns = __dadd_rn(ns, __dmul_rn(s1, s1));
    ns = __dadd_rn(ns, __dmul_rn(s2, s2));
    th = __ddiv_rn(th, __dmul_rn(__dsqrt_rn(nm), __dsqrt_rn(ns)));
    muf = mu_bin_f64(th, P);
    mur = mu_bin_f64(-th, P);
  } else {
    muf = 1;
    mur = 1;
  }
  return true;
}

// FP32 classification.  Returns 0: certainly not an edge; 1: edge with the
// bins written; 2: inside the guard band, re-evaluate with edge_f64.
// NEED_BINS=false only decides membership (guards only at rmin and rmax).
// The separation is d2 * rsqrtf(d2) and the cosine and its error bound use
// __fdividef: make_pair_params sizes the guard band for these approximate
// operations (d0 and eC), so outside the band the bins equal the FP64 ones.
template <bool NEED_BINS>
__device__ __forceinline__ int classify_f32(const float4 pi, const float4 pj, const PairParams& P,
                                            int& bin, int& muf, int& mur) {
  const float dx = pj.x - pi.x;
  const float dy = pj.y - pi.y;
  const float dz = pj.z - pi.z;
  const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
  if (d2 >= P.rmax2_hi || d2 <= P.rmin2_lo) return 0;
  // d2 = 0 (coincident points, rmin = 0): t = -rmin/dr, decided in FP64
  const float d = d2 > 0.0f ? d2 * rsqrtf(d2) : 0.0f;
  const float t = (d - P.f_rmin) * P.f_inv_dr;
  const float tn = rintf(t);
  if (NEED_BINS) {
    if (fabsf(t - tn) < P.tguard) return 2;
  } else {
    if ((tn == 0.0f || tn == (float)P.nbins) && fabsf(t - tn) < P.tguard) return 2;
  }
  if (t <= 0.0f || t >= (float)P.nbins) return 0;
  if (!NEED_BINS) return 1;
  bin = (int)t + 1;
  if (P.rsd) {
    // s = pi + pj is twice the midpoint m: the factors of 2 cancel in the
    // cosine th = m.(-d) / (|m| d) and are exact, so th is as with m
    const float dd = d - P.d0;
    const float sx = pi.x + pj.x;
    const float sy = pi.y + pj.y;
    const float sz = pi.z + pj.z;
    const float s2 = fmaf(sz, sz, fmaf(sy, sy, sx * sx));
    const float sn = s2 * rsqrtf(s2);
    const float mmm = fmaf(0.5f, sn, -P.mB);  // |m| - mB
    // one bound for both error terms: eA/dd + eB/mmm <= (eA + eB)/min(dd, mmm);
    // __fdividef needs denominators of at least 2^-126
    const float den = fminf(dd, mmm);
    if (!(den > 1e-30f) || !(s2 > 0.0f)) return 2;
    const float dot = fmaf(sz, -dz, fmaf(sy, -dy, sx * -dx));
    const float th = __fdividef(dot, sn * d);
    const float eth = __fdividef(P.eA + P.eB, den) + P.eC;
    const float ug = eth * P.f_mu_scale + 8.0f * 5.96046448e-8f * P.f_nmu;
    // mu bins of th (root p) and of -th (root q): u2 = (1 - th) nmu/2 is
    // nmu - u1, so the interior bin edges of u2 are those of u1 mirrored
    // and one guard test covers both; outside it the bin of -th is
    // nmu + 1 - (bin of th), also at the clamped ends th = -1 and 1
    const float u1 = (th + 1.0f) * P.f_mu_scale;
    const float k1 = rintf(u1);
    if (k1 >= 1.0f && k1 <= P.f_nmu - 1.0f && fabsf(u1 - k1) < ug) return 2;
    const int a = (int)floorf(u1) + 1;
    muf = a < 1 ? 1 : (a > P.nmu ? P.nmu : a);
    mur = P.nmu + 1 - muf;
  } else {
    muf = 1;
    mur = 1;
  }
  return 1;
}

// Square root for the inversion of the triangular pair index of k members
// (x = floor((2k - 1 - sqrt((2k - 1)^2 - 8t)) / 2), followed by one
// adjustment each way): disc * rsqrtf(disc), within about 3e-7 relative of
// the root.  The adjustments absorb an estimate off by one; checked on the
// CPU for every pair of every k up to 1024 with the root perturbed by
// 4e-7 either way.
__device__ __forceinline__ float pair_index_sqrt(float disc) {
  return disc > 0.0f ? disc * rsqrtf(disc) : 0.0f;
}

// Row x of pair t (0 <= t < k(k-1)/2, k2m1 = 2k - 1) with no adjustment, exact
// for k <= kPairRowExact.  There disc = (2k-1)^2 - 8t is an integer in
// [9, 511^2], exact in FP32; the root from pair_index_sqrt is within 2.5 ulp
// (rsqrtf's 2 ulp and the product's rounding), 1.6e-4 absolute, and
// u = (2k - 1 - root) / 2 comes out within 1.1e-4 of its true value.  The
// true u is an integer or a half-integer when disc is a square, and otherwise
// at least 4.8e-4 from every integer (a root of a non-square below 512^2 is
// at least 1/1024 from every integer).  Adding 2.5e-4 before truncating
// therefore gives floor(u) in every case.  Beyond kPairRowExact the result
// is within one row and the caller adjusts it.  Checked on the CPU for every
// pair of every k up to kPairRowExact with the root 3 ulp off either way.
constexpr int kPairRowExact = 256;
__device__ __forceinline__ int pair_row_biased(int k2m1, int t) {
  const float disc = (float)(k2m1 * k2m1) - 8.0f * (float)t;
  return (int)(0.5f * ((float)k2m1 - pair_index_sqrt(disc)) + 2.5e-4f);
}

// Both points of a pair are buffer points (pos4.w = 1 marks them): the pair
// has no root and adds nothing to any 2PCF histogram or gradient, so the
// pair sweeps skip it before testing it.  (The neighbour graph keeps such
// edges: they close triangles and 4-cliques rooted elsewhere.)
__device__ __forceinline__ bool both_buffer(const float4& a, const float4& b) {
  return a.w != 0.0f && b.w != 0.0f;
}

// Membership only (no bins) from the FP32 squared separation: 0 not an
// edge, 1 an edge, 2 undecided (inside the guard band at rmin or rmax:
// evaluate with edge_f64).
__device__ __forceinline__ int member_f32(const float4 pi, const float4 pj, const PairParams& P) {
  const float dx = pj.x - pi.x;
  const float dy = pj.y - pi.y;
  const float dz = pj.z - pi.z;
  const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
  if (d2 >= P.rmax2_hi || d2 <= P.rmin2_lo) return 0;
  if (d2 > P.rmin2_hi && d2 < P.rmax2_lo) return 1;
  return 2;
}

// Radial bin of a pair already known to be an edge of the graph, exactly as
// the graph build bins it: the FP32 bin outside the guard band around the bin
// edges (where it equals the FP64 one), else the FP64 reference arithmetic.
// a < c are the internal labels, pa / pc their FP32 positions.
__device__ __forceinline__ int edge_rbin(const double4* __restrict__ posd, const PairParams& P,
                                         int a, int c, const float4 pa, const float4 pc) {
  if (P.f32) {
    const float dx = pc.x - pa.x;
    const float dy = pc.y - pa.y;
    const float dz = pc.z - pa.z;
    const float d2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    const float d = d2 > 0.0f ? d2 * rsqrtf(d2) : 0.0f;
    const float t = (d - P.f_rmin) * P.f_inv_dr;
    const float tn = rintf(t);
    if (fabsf(t - tn) >= P.tguard && t > 0.0f && t < (float)P.nbins) return (int)t + 1;
  }
  int b = 1, mf = 1, mr = 1;
  edge_f64(posd[a], posd[c], P, b, mf, mr);
  return b;
}

// ---------------------------------------------------------------- cell grid --
struct GridParams {
  int nx, ny, nz;
  int64_t ncell;
  int sub;  // 0 or 1: cells at least rmax wide (27-cell neighbourhoods);
            // 2: cells at least rmax/2 wide (125-cell neighbourhoods, read
            // only by the tile pair sweep)
};

// Number of SMs of the current device (cudaDevAttrMultiProcessorCount,
// queried once per device ordinal), for grids sized in whole waves.
int sm_count();

// Host-side geometry of a uniform cell grid over the box [lo, hi]: origin,
// inverse cell size and cells per axis.
struct GridGeom {
  double lo[3];
  double inv_cs[3];
  int nc[3];
};

// Cells at least rmax wide (with a relative margin of 1e-6, so that every
// pair closer than rmax lies in the same or adjacent cells despite rounding
// in the cell-coordinate computation), at most max_per_axis per axis, then
// merged (halving the longest axis) until the grid has at most max_cells
// cells.  Every pair sweep relies on the cells being at least rmax wide, so
// all grids over a catalogue come from this one function.  Returns the
// number of cells.
int64_t make_grid_geom(const double lo[3], const double hi[3], double rmax, int max_per_axis,
                       int64_t max_cells, GridGeom& g);

// Forward (half-stencil) candidate ranges of a root at internal label p in
// cell `key`: labels q > p in the root's own cell and the 13 neighbouring
// cells that follow it in key order, as at most 5 contiguous label ranges in
// increasing order.
struct Ranges {
  int n;
  int beg[5], end[5];
};

__device__ __forceinline__ void forward_ranges(int p, int key, const GridParams& g,
                                               const int* __restrict__ cell_start, Ranges& R) {
  // five fixed slots (empty ones have beg == end), written with constant
  // indices so that R stays in registers
  const int cx = key % g.nx;
  const int cy = (key / g.nx) % g.ny;
  const int cz = key / (g.nx * g.ny);
  const int x0 = cx > 0 ? cx - 1 : 0;
  const int x1 = cx + 1 < g.nx ? cx + 1 : cx;
  R.n = 5;
  {
    const int e = cell_start[key + (cx + 1 < g.nx ? 2 : 1)];
    R.beg[0] = p + 1;
    R.end[0] = e > p + 1 ? e : p + 1;
  }
  {
    int b = 0, e = 0;
    if (cy + 1 < g.ny) {
      const int kb = (cz * g.ny + cy + 1) * g.nx;
      b = cell_start[kb + x0];
      e = cell_start[kb + x1 + 1];
    }
    R.beg[1] = b;
    R.end[1] = e > b ? e : b;
  }
#pragma unroll
  for (int dy = -1; dy <= 1; ++dy) {
    const int y = cy + dy;
    int b = 0, e = 0;
    if (cz + 1 < g.nz && y >= 0 && y < g.ny) {
      const int kb = ((cz + 1) * g.ny + y) * g.nx;
      b = cell_start[kb + x0];
      e = cell_start[kb + x1 + 1];
    }
    R.beg[3 + dy] = b;
    R.end[3 + dy] = e > b ? e : b;
  }
}

// Forward candidate ranges on a grid of cells at least rmax/2 wide (sub 2):
// labels from `first` on in the root's own cell and every cell after it in
// key order within two cells on each axis, as 13 contiguous label ranges in
// increasing order: the root's x-row up to two cells on (slot 0), the two
// following rows of its z plane (slots 1-2), and the five rows of each of
// the next two z planes (slots 3-12).  Lane k of the calling warp (k < 13)
// returns slot k's [beg, end).
__device__ __forceinline__ void forward_range2_slot(int k, int first, int key, const GridParams& g,
                                                    const int* __restrict__ cell_start, int& beg,
                                                    int& end) {
  const int cx = key % g.nx;
  const int cy = (key / g.nx) % g.ny;
  const int cz = key / (g.nx * g.ny);
  const int x0 = cx > 1 ? cx - 2 : 0;
  const int x1 = cx + 2 < g.nx ? cx + 2 : g.nx - 1;
  int b = 0, e = 0;
  if (k == 0) {
    b = first;
    e = cell_start[key - cx + x1 + 1];
  } else if (k < 3) {
    const int y = cy + k;
    if (y < g.ny) {
      const int kb = (cz * g.ny + y) * g.nx;
      b = cell_start[kb + x0];
      e = cell_start[kb + x1 + 1];
    }
  } else if (k < 13) {
    const int z = cz + 1 + (k - 3) / 5;
    const int y = cy - 2 + (k - 3) % 5;
    if (z < g.nz && y >= 0 && y < g.ny) {
      const int kb = (z * g.ny + y) * g.nx;
      b = cell_start[kb + x0];
      e = cell_start[kb + x1 + 1];
    }
  }
  beg = b;
  end = e > b ? e : b;
}

// All 27 neighbouring cells (own cell included) as at most 9 contiguous
// label ranges in increasing order.
struct Ranges9 {
  int n;
  int beg[9], end[9];
};

__device__ __forceinline__ void full_ranges(int key, const GridParams& g,
                                            const int* __restrict__ cell_start, Ranges9& R) {
  const int cx = key % g.nx;
  const int cy = (key / g.nx) % g.ny;
  const int cz = key / (g.nx * g.ny);
  const int x0 = cx > 0 ? cx - 1 : 0;
  const int x1 = cx + 1 < g.nx ? cx + 1 : cx;
  R.n = 0;
  for (int dz = -1; dz <= 1; ++dz) {
    const int z = cz + dz;
    if (z < 0 || z >= g.nz) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const int y = cy + dy;
      if (y < 0 || y >= g.ny) continue;
      const int kb = (z * g.ny + y) * g.nx;
      const int b = cell_start[kb + x0], e = cell_start[kb + x1 + 1];
      if (e > b) {
        R.beg[R.n] = b;
        R.end[R.n] = e;
        R.n++;
      }
    }
  }
}

__device__ __forceinline__ int range9_label(const Ranges9& R, const int* pre, int f) {
  int r = 0;
#pragma unroll
  for (int k = 1; k < 9; ++k)
    if (k < R.n && f >= pre[k]) r = k;
  return R.beg[r] + (f - pre[r]);
}

// Map flattened candidate index f (0 <= f < total) to a label.
__device__ __forceinline__ int range_label(const Ranges& R, const int* pre, int f) {
  // constant indices only, so R and pre stay in registers
  int b = R.beg[0], o = pre[0];
#pragma unroll
  for (int k = 1; k < 5; ++k)
    if (k < R.n && f >= pre[k]) {
      b = R.beg[k];
      o = pre[k];
    }
  return b + (f - o);
}

// --------------------------------------------------------- tuple rank tables --
// Rank (1-based) of a non-decreasing k-tuple over [1, n] in lexicographic
// order, as create_binlookup numbers configurations
// (src/gramsci.F90:1398-1477).  F[j][v] = sum_{u<v} C(n-u+1 + (k-j-1) - 1, k-j-1)
// so rank = 1 + sum_j (F[j][x_j] - F[j][x_{j-1}]).
constexpr int kMaxBins = 127;
struct RankTables {
  int n;
  int k;
  int F[4][kMaxBins + 2];
};
void make_rank_tables(RankTables& T, int n, int k);

__device__ __forceinline__ int rank_sorted3(const RankTables& T, int a, int b, int c) {
  // a <= b <= c, 1-based
  return 1 + (T.F[0][a] - T.F[0][1]) + (T.F[1][b] - T.F[1][a]) + (T.F[2][c] - T.F[2][b]);
}

__device__ __forceinline__ int rank_sorted4(const RankTables& T, int a, int b, int c, int d) {
  return 1 + (T.F[0][a] - T.F[0][1]) + (T.F[1][b] - T.F[1][a]) + (T.F[2][c] - T.F[2][b]) +
         (T.F[3][d] - T.F[3][c]);
}

__device__ __forceinline__ void sort3i(int& a, int& b, int& c) {
  int t;
  if (a > b) { t = a; a = b; b = t; }
  if (b > c) { t = b; b = c; c = t; }
  if (a > b) { t = a; a = b; b = t; }
}

// Packed edge metadata of the upper CSR: radial bin, mu seen from the row's
// point, mu seen from the neighbour.
__device__ __forceinline__ uint32_t pack_meta(int bin, int muf, int mur) {
  return (uint32_t)bin | ((uint32_t)muf << 8) | ((uint32_t)mur << 16);
}
__device__ __forceinline__ int meta_bin(uint32_t m) { return (int)(m & 0xff); }
__device__ __forceinline__ int meta_muf(uint32_t m) { return (int)((m >> 8) & 0xff); }
__device__ __forceinline__ int meta_mur(uint32_t m) { return (int)((m >> 16) & 0xff); }

// ---------------------------------------------------------- device catalogue --
// Points in cell order ("internal labels").  orig[p] is the position in the
// reference's catalogue order; random = orig >= n_data.
struct DevCatalog {
  const float4* pos4;    // float x, y, z, (unused)
  const double4* posd;   // double x, y, z, w
  const double* w;       // weight
  const int* orig;       // original index
  const uint8_t* flags;  // bit0 random, bit1 buffer
  const int* cell_key;   // cell of each point
  const int* cell_start; // ncell + 1
  int n;
  int n_data;
  GridParams grid;
  // Batched regions: when cell_region is set, cells are grouped by region;
  // region r owns cells [region_cell_off[r], region_cell_off[r+1]) laid out
  // on its own grid region_grid[r].  NULL for a single grid.
  const int* cell_region;
  const GridParams* region_grid;
  const int* region_cell_off;
};

// Grid, cell-start table and local key of a cell (single grid or region).
__device__ __forceinline__ void cell_grid(const DevCatalog& C, int cell, GridParams& g,
                                          const int*& cs, int& lkey) {
  if (C.cell_region) {
    const int r = C.cell_region[cell];
    const int off = C.region_cell_off[r];
    g = C.region_grid[r];
    cs = C.cell_start + off;
    lkey = cell - off;
  } else {
    g = C.grid;
    cs = C.cell_start;
    lkey = cell;
  }
}

enum : uint8_t { FLAG_RANDOM = 1, FLAG_BUFFER = 2 };

// 2PCF weight adjoint: coefficient of the pair (p, q) in dL/dw, the
// cotangents of the bins the pair lands in from each non-buffer end (cot3
// only for random-random pairs); the pair adds coef * w_q to dL/dw_p and
// coef * w_p to dL/dw_q.
__device__ __forceinline__ double pair_coef(const double* c2, const double* c3, int nbins, int b,
                                            int mf, int mr, uint8_t fp, uint8_t fq) {
  const bool rr = (fp & fq & FLAG_RANDOM) != 0;
  double c = 0.0;
  if (!(fp & FLAG_BUFFER)) {
    const int k = (b - 1) + nbins * (mf - 1);
    c += rr ? c2[k] + c3[k] : c2[k];
  }
  if (!(fq & FLAG_BUFFER)) {
    const int k = (b - 1) + nbins * (mr - 1);
    c += rr ? c2[k] + c3[k] : c2[k];
  }
  return c;
}

// ------------------------------------------------------- fixed-point sums --
// Weighted sums are accumulated as signed 128-bit fixed-point integers with
// 64-bit integer atomics: a product x becomes V = round(x * 2^e) (|V| < 2^63,
// e chosen per launch from the largest possible |product|) and is added in
// two's complement to a (lo, hi) pair.  Integer addition is exact and
// order-independent, so the sums are deterministic; the only rounding is the
// quantisation of each product, at most 2^-(e+1) absolute.
__device__ __forceinline__ void fix_add(unsigned long long* lo, unsigned long long* hi, double x,
                                        double scale) {
  const long long v = __double2ll_rn(x * scale);
  const unsigned long long add = (unsigned long long)v;
  const unsigned long long old = atomicAdd(lo, add);
  const unsigned long long carry = (old + add < old) ? 1ull : 0ull;
  const unsigned long long d = (v < 0 ? ~0ull : 0ull) + carry;
  if (d) atomicAdd(hi, d);
}

// the same for an integer already scaled (|v| < 2^62)
__device__ __forceinline__ void fix_add_int(unsigned long long* lo, unsigned long long* hi,
                                            long long v) {
  const unsigned long long add = (unsigned long long)v;
  const unsigned long long old = atomicAdd(lo, add);
  const unsigned long long carry = (old + add < old) ? 1ull : 0ull;
  const unsigned long long d = (v < 0 ? ~0ull : 0ull) + carry;
  if (d) atomicAdd(hi, d);
}

// Fixed-point sums whose updates return nothing: V = round(x * scale)
// (|V| < 2^62) is split into its low 32 bits (unsigned) and its high part
// V >> 32 (signed), and each is added with a reduction, so the issuing warp
// never waits for an atomic's old value (the carry of fix_add needs it).
// The pair (lo, hi) then holds sum(low limbs) and sum(high limbs); its value
// is hi * 2^32 + lo (fix_split_value).  Exact while a sum receives fewer
// than 2^32 updates (the low-limb sum stays below 2^64).
__device__ __forceinline__ void fix_red(unsigned long long* lo, unsigned long long* hi, double x,
                                        double scale) {
  const long long v = __double2ll_rn(x * scale);
  atomicAdd(lo, (unsigned long long)(v & 0xffffffffll));
  atomicAdd(hi, (unsigned long long)(v >> 32));
}

// merge a partial (lo, hi) pair into another with atomics
__device__ __forceinline__ void fix_merge(unsigned long long* lo, unsigned long long* hi,
                                          unsigned long long plo, unsigned long long phi) {
  const unsigned long long old = atomicAdd(lo, plo);
  const unsigned long long d = phi + ((old + plo < old) ? 1ull : 0ull);
  if (d) atomicAdd(hi, d);
}

// A 128-bit fixed-point accumulator held in registers.
struct Fix128 {
  unsigned long long lo, hi;
};

__device__ __forceinline__ void fix_acc(Fix128& a, double x, double scale) {
  const long long v = __double2ll_rn(x * scale);
  const unsigned long long add = (unsigned long long)v;
  const unsigned long long old = a.lo;
  a.lo += add;
  a.hi += (v < 0 ? ~0ull : 0ull) + (a.lo < old ? 1ull : 0ull);
}

// Exact warp sum of 128-bit accumulators (every lane gets the total).
__device__ __forceinline__ Fix128 fix_warp_sum(Fix128 a) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long l2 = __shfl_xor_sync(0xffffffffu, a.lo, o);
    const unsigned long long h2 = __shfl_xor_sync(0xffffffffu, a.hi, o);
    const unsigned long long s = a.lo + l2;
    a.hi = a.hi + h2 + (s < a.lo ? 1ull : 0ull);
    a.lo = s;
  }
  return a;
}

// Value of the signed 128-bit integer (hi, lo) as a double, rounded once
// (to nearest, ties to even), on the host and on the device alike: the
// magnitude's top 64 bits are converted with the bits below them folded
// into a sticky bit, then scaled by a power of two (exact).
__host__ __device__ __forceinline__ double i128_to_double(unsigned long long lo,
                                                          unsigned long long hi) {
  const bool neg = (long long)hi < 0;
  if (neg) {
    lo = ~lo + 1ull;
    hi = ~hi + (lo == 0ull ? 1ull : 0ull);
  }
  double mag;
  if (hi == 0ull) {
#ifdef __CUDA_ARCH__
    mag = __ull2double_rn(lo);
#else
    mag = (double)lo;
#endif
  } else {
#ifdef __CUDA_ARCH__
    const int sh = 64 - __clzll((long long)hi);  // significant bits of hi, 1..64
#else
    const int sh = 64 - __builtin_clzll(hi);
#endif
    unsigned long long top = sh == 64 ? hi : ((hi << (64 - sh)) | (lo >> sh));
    const unsigned long long rest = sh == 64 ? lo : (lo << (64 - sh));
    top |= rest != 0ull ? 1ull : 0ull;
#ifdef __CUDA_ARCH__
    mag = ldexp(__ull2double_rn(top), sh);
#else
    mag = std::ldexp((double)top, sh);
#endif
  }
  return neg ? -mag : mag;
}

// Device: value of a signed 128-bit (lo, hi) pair divided by scale (a power
// of two, so the division adds no rounding).
__device__ __forceinline__ double fix_to_double(unsigned long long lo, unsigned long long hi,
                                                double inv_scale) {
  return i128_to_double(lo, hi) * inv_scale;
}

// Host: scale 2^e with max_abs_product * 2^e < 2^62.
double fix_scale(double max_abs_product);
// Host: value of a (lo, hi) pair.
double fix_value(unsigned long long lo, unsigned long long hi, double scale);
// Host: value of a split-limb pair written by fix_red.
double fix_split_value(unsigned long long lo, unsigned long long hi, double scale);

// -------------------------------------------------------------- host launch --
// Zero up to 8 device buffers in one launch (instead of one memset each).
struct ZeroList {
  void* p[8];
  size_t bytes[8];
  int n = 0;
  void add(void* ptr, size_t b) {
    if (b > 0) {
      p[n] = ptr;
      bytes[n] = b;
      ++n;
    }
  }
};
void zero_async(const ZeroList& z, cudaStream_t s);

// Exclusive scan of n int32 values into n+1 int64 values (out[n] = total).
// out32 (optional): the scan also as 32-bit integers (values below 2^31)
void scan_i32_to_i64(const int* in, int64_t* out, int64_t n, cudaStream_t s, DevBuf<int64_t>& tmp,
                     int* out32 = nullptr);
void scan_i64(const int64_t* in, int64_t* out, int64_t n, cudaStream_t s, DevBuf<int64_t>& tmp);

}  // namespace gr
