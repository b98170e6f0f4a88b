// 4PCF 4-clique counting: replaces query_4pcf_all2 (src/gramsci.F90:662-825),
// whose per-root triple loop performs three find_dist binary searches per
// candidate triple, and the -tetra counter query_graph_tetrahedron
// (:548-660).
//
// Every 4-clique is enumerated exactly once, from its smallest label p.  A
// warp takes roots from a work counter and stages R+(p) in shared memory
// (catalogue id, flags, weight, row start and length of every neighbour)
// with a per-root hash table (label offset -> row position).  For each a in
// R+(p) it builds X = R+(a) ∩ R+(p) beyond a's position, as a compacted list
// and a bitmask over R+(p)'s positions; then the work items (b, d) for b in X
// and d in R+(b) are flattened over the lanes (warp OR-reduction owners, as
// in the triangle kernel), d is looked up in the hash table and tested in
// the bitmask, and hits (cliques p < a < b < d) are queued and binned 32 at
// a time with all their data in shared memory.  A clique contributes, for
// every vertex r that is a root in the reference (not a buffer point, row
// length > 3), with the other three vertices taken in catalogue-id order
// (k1 < k2 < k3 of the reference), if the perimeter r-k1-k2-k3-r is
// canonical (bintable entry > 0), to N2 / N3 at (cfg, bin(r,k2), bin(k1,k3))
// and to the six disconnected pair terms.
//
// A second kernel (quad4g_kernel, the geometric mode) finds the edges among
// the members of R+(p) with the graph's own membership test on their
// positions instead of probing the members' rows; it is used whenever the
// rows fit (up to 256 members).
#include <algorithm>
#include <type_traits>

#include "gr_kernels.cuh"

namespace gr {

namespace {

constexpr int kQuadMaxWarps = 16;   // weighted / adjoint kernels (up to 128 registers)
constexpr int kQuadMaxWarpsU = 24;  // unweighted kernels (up to 85 registers)
#ifndef GR_QUADG_WEIGHTED_WARPS
#define GR_QUADG_WEIGHTED_WARPS 24
#endif
// Weighted geometric kernel: 24 warps (at most 85 registers, a few bytes
// spilled) measured 4.47 ms on the 4PCF workload against 4.64 ms at 20,
// 5.04 ms at 16 (106 registers), 4.84 ms at 28 and 5.29 ms at 32 (spills)
// once its sums had a line per bin; before that the reductions, not the
// warps, bounded it.  (The high limb in the
// low limb's line instead of a line of its own: 4.58 ms.)
constexpr int kQuadGWarpsW = GR_QUADG_WEIGHTED_WARPS;
// Geometric adjoint kernel: 24 warps (at most 85 registers, ~50 bytes
// spilled) measured 6.13 ms on the 4PCF workload against 6.67 ms at 20 and
// 7.27 ms at 16 (116 registers), identical gradients.
constexpr int kQuadGWarpsA = 24;
constexpr size_t kQuadSmemLimit = 227 * 1024;
constexpr int kQQueue = 96;         // hit queue entries per warp (< 32 left + 64 pushed)
constexpr int kQMaxOffset = 1 << 22;  // hash entries: (label offset << 10) | position
constexpr uint8_t kFlagDeg4 = 4;    // staged flag: full row length > 3 (a reference root)
// The longest rows (a root's cost grows with the cube of its row length) are
// handed out as kSplitParts work items each, every item staging the root in
// full and taking every kSplitParts-th share of its cliques: a heavy root on
// one warp otherwise ends the launch alone (measured on the 4PCF workload:
// one SM busy for 8.0M cycles while the others were done after 5.1M).  The
// split roots are the longest ones, at least kSplitRow long, few enough that
// their items fill at most a quarter of the launch's warps (measured on the
// 4PCF workload, unit weights: 2.98 ms at an eighth, 2.64 ms at a quarter,
// 2.62 ms at a half; 16 items per root: 3.01 ms).
constexpr int kSplitRow = 32;
constexpr int kSplitParts = 8;

// The root and part of work item `item` (QuadParams::order / nheavy).
// Items [0, nheavy * parts) are the parts of the heavy roots, then one item
// per remaining root.  Returns false past the last root.
__device__ __forceinline__ bool quad_item(const QuadParams& Q, int n, int item, int nh, int parts,
                                          int& p, int& part) {
  int slot;
  part = 0;
  if (item < nh * parts) {
    slot = item / parts;
    part = item - slot * parts;
  } else {
    slot = nh + (item - nh * parts);
  }
  if (slot >= n) return false;
  p = Q.order ? Q.order[slot] : slot;
  return true;
}
__device__ __forceinline__ int quad_split_parts(const QuadParams& Q, int& nh) {
  nh = 0;
  if (!Q.order || !Q.above || Q.nclass <= kSplitRow) return 1;
  const int limit = (int)gridDim.x * (int)(blockDim.x >> 5) / (4 * kSplitParts);
  // above[] does not increase with b: the smallest b >= kSplitRow - 1 with
  // above[b] <= limit
  int lo = kSplitRow - 1, hi = Q.nclass - 1;
  if (Q.above[hi] > limit) return 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (Q.above[mid] <= limit) hi = mid;
    else lo = mid + 1;
  }
  nh = Q.above[lo];
  return nh > 0 ? kSplitParts : 1;
}

__host__ __device__ inline size_t qalign8(size_t x) { return (x + 7) & ~(size_t)7; }

__host__ __device__ inline int qhash_lg_max(int cap) {
  int lg = 6;
  while ((1 << lg) < 4 * cap) ++lg;
  return lg;
}

struct QuadLayout {
  size_t off_rank, off_cnt, off_warp, warp_bytes, total;
  // per-warp sub-offsets
  size_t o_rs, o_w, o_mo, o_g, o_col, o_len, o_xm, o_hkey, o_q, o_xy, o_xz, o_bits;
};

// ncounts: block-private 32-bit counters in shared memory (0: none);
// adj: per-neighbour 128-bit gradient accumulators (adjoint mode)
__host__ __device__ inline QuadLayout quad_layout(int nbins, int cap, int nwarps, int ncounts,
                                                  bool adj = false) {
  QuadLayout L;
  size_t o = 0;
  L.off_rank = o;
  o = qalign8(o + sizeof(int) * 4 * (size_t)(nbins + 2));
  L.off_cnt = o;
  o = qalign8(o + sizeof(unsigned int) * (size_t)ncounts);
  L.off_warp = o;
  size_t w = 0;
  L.o_rs = w;   w += (size_t)cap * 8;   // row start of each neighbour
  L.o_w = w;    w += (size_t)cap * 8;   // weight
  L.o_mo = w;   w += (size_t)cap * 8;   // (catalogue id << 32) | flags << 24 | meta(p, a)
  L.o_g = w;    w += adj ? (size_t)cap * 16 : 0;  // gradient (lo, hi) of each neighbour
  L.o_col = w;  w += (size_t)cap * 4;   // label
  L.o_len = w;  w += (size_t)cap * 4;   // row length
  L.o_xm = w;   w += (size_t)cap * 4;   // X entry z: meta(a, b)
  L.o_hkey = w; w += (size_t)(1u << qhash_lg_max(cap)) * 4;
  L.o_q = w;    w += (size_t)kQQueue * 8;
  L.o_xy = w;   w += (size_t)cap * 2;   // X entry z: position of b in R+(p)
  L.o_xz = w;   w += (size_t)cap * 2;   // position y: X entry (when its bit is set)
  L.o_bits = w; w += (size_t)((cap + 31) / 32) * 4;
  L.warp_bytes = qalign8(w);
  L.total = o + L.warp_bytes * nwarps;
  return L;
}

struct QuadCtx {
  const int* F;  // 4 x (nbins+2)
  int nbins, ncfg, nbin, tetra;
  unsigned long long *cnt, *dcnt;
  unsigned int *scnt, *sdcnt;  // block-private 32-bit counts in shared memory, or null
  unsigned long long *fix, *dfix;  // fixed-point (lo, hi) sums, hi at +5*nbin / +dhi
  int dhi;                          // disc entries on the device (hi offset in dfix)
  int split;                        // 1: sums as split limbs (fix_red), 0: carries (fix_add)
  int counts;                       // 0: weighted sums only, no integer counts
  double fscale;  // scale of the 4-point products
  double dscale;  // scale of the pair products of the disconnected terms
  // adjoint: cotangents of N2, N3 (nbin each), discN, discR (6 nbin each)
  const double *c2, *c3, *cN, *cR;
};

// Logical entry i of a global fixed-point array: one entry per kFixStride
// 8-byte words, so that every entry has a 128-byte line of its own.  The
// hottest bins are neighbours in the dense order; packed 16 to a line they
// were served by a few L2 slices, and the weighted 4PCF kernel's time then
// depended on where the arrays happened to lie (measured 5.4 to 6.9 ms for
// the same launch as the arrays were moved in steps of 4 KB).
__device__ __forceinline__ unsigned long long* qfx(unsigned long long* a, int i) {
  return a + (size_t)i * kFixStride;
}

// one weighted update of a global fixed-point sum
__device__ __forceinline__ void qfix(const QuadCtx& X, unsigned long long* lo, unsigned long long* hi,
                                     double x, double scale) {
  if (X.split)
    fix_red(lo, hi, x, scale);
  else
    fix_add(lo, hi, x, scale);
}

template <bool SHC>
__device__ __forceinline__ void qcount(const QuadCtx& X, int k) {
  if (SHC) atomicAdd(&X.scnt[k], 1u);
  else if (X.counts) atomicAdd(&X.cnt[k], 1ull);
}
template <bool SHC>
__device__ __forceinline__ void qdcount(const QuadCtx& X, int k) {
  if (SHC) atomicAdd(&X.sdcnt[k], 1u);
  else if (X.counts) atomicAdd(&X.dcnt[k], 1ull);
}

// The four vertices of a clique: flags (with kFlagDeg4), catalogue ids and
// weights.
struct QVerts {
  uint8_t fl[4];
  int og[4];
  double w[4];
};

// Disconnected term t (t = 1..6 of gramsci.F90:754-818, here 0..5): the
// role whose randomness gates it and the two roles of its pair product
// (roles: 0 = root, 1..3 = the other vertices in catalogue-id order).  The
// -tetra terms (:591-646) use the same gate with the 3-product (gate, pu, pv).
// Written as functions of a loop index that is unrolled, so every use folds
// to a constant and no table is indexed at run time.
__host__ __device__ constexpr int term_gate(int t) { return t < 2 ? 3 : (t == 2 ? 1 : 0); }
__host__ __device__ constexpr int term_pu(int t) { return t < 3 ? 0 : (t == 3 ? 1 : 3); }
__host__ __device__ constexpr int term_pv(int t) { return t < 3 ? t + 1 : (t == 5 ? 1 : 2); }

// index (0..5) of the clique edge between vertices u != v: (0,1) (0,2) (0,3)
// (1,2) (1,3) (2,3)
__device__ __forceinline__ int qedge(int u, int v) {
  const int a = min(u, v), b = max(u, v);
  return a * (7 - a) / 2 - 1 + b - a;
}
// radial bin of edge (u, v) from the six bins packed a byte each
__device__ __forceinline__ int qbin(unsigned long long packed, int u, int v) {
  return (int)((packed >> (8 * qedge(u, v))) & 0xffull);
}
__device__ __forceinline__ double qsel(int i, const QVerts& V) {
  return i == 0 ? V.w[0] : (i == 1 ? V.w[1] : (i == 2 ? V.w[2] : V.w[3]));
}

// The three vertices other than root r, ordered by catalogue id (the
// reference's id-sorted row): a three-element sorting network on registers.
template <int R>
__device__ __forceinline__ void others_by_id(const QVerts& V, int& u0, int& u1, int& u2) {
  constexpr int O0 = R == 0 ? 1 : 0, O1 = R <= 1 ? 2 : 1, O2 = R <= 2 ? 3 : 2;
  int g0 = V.og[O0], g1 = V.og[O1], g2 = V.og[O2];
  u0 = O0;
  u1 = O1;
  u2 = O2;
  int t;
  if (g0 > g1) { t = g0; g0 = g1; g1 = t; t = u0; u0 = u1; u1 = t; }
  if (g1 > g2) { t = g1; g1 = g2; g2 = t; t = u1; u1 = u2; u2 = t; }
  if (g0 > g1) { t = g0; g0 = g1; g1 = t; t = u0; u0 = u1; u1 = t; }
}

// query_graph_tetrahedron: a 4-clique with all six edges in bin b counts from
// each non-buffer vertex (no row-length condition).
template <bool WEIGHTED, bool SHC, int R>
__device__ __forceinline__ int tetra_root(const QuadCtx& X, const QVerts& V, int b, unsigned rndm,
                                          int nr) {
  if (V.fl[R] & FLAG_BUFFER) return 0;
  int u0, u1, u2;
  others_by_id<R>(V, u0, u1, u2);
  const int role[4] = {R, u0, u1, u2};
  const int nb = X.nbins;
  qcount<SHC>(X, (b - 1) + nb * nr);
  if (WEIGHTED)
    qfix(X, qfx(X.fix, (b - 1) + nb * nr), qfx(X.fix, (b - 1) + nb * (nr + 5)),
            ((V.w[R] * qsel(u0, V)) * qsel(u1, V)) * qsel(u2, V), X.fscale);
#pragma unroll
  for (int tt = 0; tt < 6; ++tt) {
    if (!((rndm >> role[term_gate(tt)]) & 1u)) continue;
    const int ua = role[term_gate(tt)], ub = role[term_pu(tt)], uc = role[term_pv(tt)];
    const int nr3 = (int)((rndm >> ua) & 1u) + (int)((rndm >> ub) & 1u) + (int)((rndm >> uc) & 1u);
    const int kt = (b - 1) + nb * tt;
    const double qv = WEIGHTED ? (qsel(ua, V) * qsel(ub, V)) * qsel(uc, V) : 0.0;
    // discR (all three random) equals category 3 and is copied on the host
    qdcount<SHC>(X, kt + nb * 6 * nr3);
    if (WEIGHTED) qfix(X, qfx(X.dfix, kt + nb * 6 * nr3), qfx(X.dfix, kt + nb * 6 * nr3 + X.dhi), qv, X.dscale);
  }
  return 1;
}

template <bool WEIGHTED, bool SHC>
__device__ __forceinline__ int tetra_contrib(const QuadCtx& X, const QVerts& V, const uint32_t m[6]) {
  const int b = meta_bin(m[0]);
#pragma unroll
  for (int k = 1; k < 6; ++k)
    if (meta_bin(m[k]) != b) return 0;
  unsigned rndm = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) rndm |= (unsigned)(V.fl[k] & FLAG_RANDOM) << k;
  const int nr = __popc(rndm);
  return tetra_root<WEIGHTED, SHC, 0>(X, V, b, rndm, nr) + tetra_root<WEIGHTED, SHC, 1>(X, V, b, rndm, nr) +
         tetra_root<WEIGHTED, SHC, 2>(X, V, b, rndm, nr) + tetra_root<WEIGHTED, SHC, 3>(X, V, b, rndm, nr);
}

// Root R of a 4-clique for query_4pcf_all2: the histogram index of its
// contribution, (cfg, bin(r,k2), bin(k1,k3)) with k1 < k2 < k3 the other
// vertices in catalogue-id order (returned in u0..u2), or -1 when R is no
// root (buffer point, row length <= 3) or its perimeter is not canonical.
template <int R>
__device__ __forceinline__ int quad_root_index(const QuadCtx& X, const QVerts& V,
                                               unsigned long long packed, int& u0, int& u1,
                                               int& u2) {
  if (V.fl[R] & FLAG_BUFFER) return -1;
  if (!(V.fl[R] & kFlagDeg4)) return -1;
  others_by_id<R>(V, u0, u1, u2);
  const int b1 = qbin(packed, R, u0), b2 = qbin(packed, u0, u1), b3 = qbin(packed, u1, u2),
            b4 = qbin(packed, R, u2);
  if (!(b1 <= b2 && b2 <= b3 && b3 <= b4)) return -1;
  const int nb2 = X.nbins + 2;
  const int cfg = 1 + (X.F[b1] - X.F[1]) + (X.F[nb2 + b2] - X.F[nb2 + b1]) +
                  (X.F[2 * nb2 + b3] - X.F[2 * nb2 + b2]) + (X.F[3 * nb2 + b4] - X.F[3 * nb2 + b3]);
  const int d1 = qbin(packed, R, u1), d2 = qbin(packed, u0, u2);
  return (cfg - 1) + X.ncfg * ((d1 - 1) + X.nbins * (d2 - 1));
}

// N2 / N3 and the six disconnected terms of root R.  Unit weights: one
// count at (histogram index, randomness of the four roles) instead, the
// pattern histogram from which quad_expand_patterns forms the N2 / N3 and
// disconnected-term counts (which roles are random decides the category of
// each and which terms are gated in).
template <bool WEIGHTED, bool SHC, int R>
__device__ __forceinline__ int quad_root(const QuadCtx& X, const QVerts& V, unsigned long long packed,
                                         unsigned rndm, int nr) {
  int u0, u1, u2;
  const int kk = quad_root_index<R>(X, V, packed, u0, u1, u2);
  if (kk < 0) return 0;
  if constexpr (!WEIGHTED) {
    const unsigned pat = ((rndm >> R) & 1u) | (((rndm >> u0) & 1u) << 1) |
                         (((rndm >> u1) & 1u) << 2) | (((rndm >> u2) & 1u) << 3);
    qcount<SHC>(X, kk + X.nbin * (int)pat);
    return 1;
  }
  qcount<SHC>(X, kk + X.nbin * nr);
  if (WEIGHTED)
    qfix(X, qfx(X.fix, kk + X.nbin * nr), qfx(X.fix, kk + X.nbin * (nr + 5)),
            ((V.w[R] * qsel(u0, V)) * qsel(u1, V)) * qsel(u2, V), X.fscale);
  const int role[4] = {R, u0, u1, u2};
#pragma unroll
  for (int tt = 0; tt < 6; ++tt) {
    if (!((rndm >> role[term_gate(tt)]) & 1u)) continue;
    const int u = role[term_pu(tt)], vv = role[term_pv(tt)];
    const int npr = (int)((rndm >> u) & 1u) + (int)((rndm >> vv) & 1u);
    const int kt = kk + X.nbin * tt;
    const double q = WEIGHTED ? qsel(u, V) * qsel(vv, V) : 0.0;
    // discR (both random) equals category 2 and is copied on the host
    qdcount<SHC>(X, kt + X.nbin * 6 * npr);
    if (WEIGHTED)
      qfix(X, qfx(X.dfix, kt + X.nbin * 6 * npr), qfx(X.dfix, kt + X.nbin * 6 * npr + X.dhi), q, X.dscale);
  }
  return 1;
}

// m: bins of (0,1) (0,2) (0,3) (1,2) (1,3) (2,3) for vertices 0 = p, 1 = a,
// 2 = b, 3 = d.
template <bool WEIGHTED, bool SHC>
__device__ __forceinline__ int quad_contrib(const QuadCtx& X, const QVerts& V, const uint32_t m[6]) {
  unsigned long long packed = 0;
#pragma unroll
  for (int e = 0; e < 6; ++e) packed |= (unsigned long long)meta_bin(m[e]) << (8 * e);
  unsigned rndm = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) rndm |= (unsigned)(V.fl[k] & FLAG_RANDOM) << k;
  const int nr = __popc(rndm);
  return quad_root<WEIGHTED, SHC, 0>(X, V, packed, rndm, nr) + quad_root<WEIGHTED, SHC, 1>(X, V, packed, rndm, nr) +
         quad_root<WEIGHTED, SHC, 2>(X, V, packed, rndm, nr) + quad_root<WEIGHTED, SHC, 3>(X, V, packed, rndm, nr);
}

// Vertex indices 0..3 in ascending catalogue id, two bits each (the
// register sorting network the flattened drain and the gradient use).
__device__ __forceinline__ unsigned id_order(const QVerts& V) {
  int g0 = V.og[0], g1 = V.og[1], g2 = V.og[2], g3 = V.og[3];
  unsigned a0 = 0, a1 = 1, a2 = 2, a3 = 3;
  auto cx = [](int& ga, int& gb, unsigned& ia, unsigned& ib) {
    if (ga > gb) {
      const int t = ga; ga = gb; gb = t;
      const unsigned u = ia; ia = ib; ib = u;
    }
  };
  cx(g0, g1, a0, a1);
  cx(g2, g3, a2, a3);
  cx(g0, g2, a0, a2);
  cx(g1, g3, a1, a3);
  cx(g1, g2, a1, a2);
  return a0 | (a1 << 2) | (a2 << 4) | (a3 << 6);
}

// Gradient of the cotangent-weighted sums with respect to the four vertex
// weights of one clique (g[v] = d/dw_v, vertices as in quad_contrib).  The
// sums are multilinear: a 4-product contributes its cotangent times the
// product of the other three weights, a pair term its cotangent times the
// partner's weight.  The valid roots' cotangents are gathered into one
// 4-product coefficient c4 and one coefficient per clique edge D[e] (edges
// 0 (0,1) 1 (0,2) 2 (0,3) 3 (1,2) 4 (1,3) 5 (2,3)); the roots are a loop
// that is not unrolled (fully unrolled, the gradient code overflowed the
// instruction cache).
__device__ __forceinline__ int quad_grad_c(const QuadCtx& X, const QVerts& V, const uint32_t m[6],
                                           double g[4]) {
  unsigned long long packed = 0;
#pragma unroll
  for (int e = 0; e < 6; ++e) packed |= (unsigned long long)meta_bin(m[e]) << (8 * e);
  unsigned rndm = 0, flw = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    rndm |= (unsigned)(V.fl[k] & FLAG_RANDOM) << k;
    flw |= (unsigned)V.fl[k] << (8 * k);
  }
  const int nr = __popc(rndm);
  const unsigned perm = id_order(V);
  double c4 = 0.0, D[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  int n = 0;
#pragma unroll 1
  for (int R = 0; R < 4; ++R) {
    const unsigned fr = flw >> (8 * R);
    if ((fr & FLAG_BUFFER) || !(fr & kFlagDeg4)) continue;
    int pos = 0;
#pragma unroll
    for (int i = 1; i < 4; ++i)
      if ((int)((perm >> (2 * i)) & 3u) == R) pos = i;
    const unsigned lowm = (1u << (2 * pos)) - 1u;
    const unsigned oth = (perm & lowm) | ((perm >> (2 * pos + 2)) << (2 * pos));
    const int u0 = (int)(oth & 3u), u1 = (int)((oth >> 2) & 3u), u2 = (int)((oth >> 4) & 3u);
    const int b1 = qbin(packed, R, u0), b2 = qbin(packed, u0, u1), b3 = qbin(packed, u1, u2),
              b4 = qbin(packed, R, u2);
    if (!(b1 <= b2 && b2 <= b3 && b3 <= b4)) continue;
    const int nb2 = X.nbins + 2;
    const int cfg = 1 + (X.F[b1] - X.F[1]) + (X.F[nb2 + b2] - X.F[nb2 + b1]) +
                    (X.F[2 * nb2 + b3] - X.F[2 * nb2 + b2]) + (X.F[3 * nb2 + b4] - X.F[3 * nb2 + b3]);
    const int d1 = qbin(packed, R, u1), d2 = qbin(packed, u0, u2);
    const int kk = (cfg - 1) + X.ncfg * ((d1 - 1) + X.nbins * (d2 - 1));
    ++n;
    c4 += __ldg(&X.c2[kk]) + (nr == 4 ? __ldg(&X.c3[kk]) : 0.0);
    const unsigned rp = (unsigned)R | ((unsigned)u0 << 2) | ((unsigned)u1 << 4) | ((unsigned)u2 << 6);
#pragma unroll
    for (int tt = 0; tt < 6; ++tt) {
      const int ga = (int)((rp >> (2 * term_gate(tt))) & 3u);
      if (!((rndm >> ga) & 1u)) continue;
      const int u = (int)((rp >> (2 * term_pu(tt))) & 3u), vv = (int)((rp >> (2 * term_pv(tt))) & 3u);
      const int kt = kk + X.nbin * tt;
      const bool both = ((rndm >> u) & 1u) && ((rndm >> vv) & 1u);
      const double cd = __ldg(&X.cN[kt]) + (both ? __ldg(&X.cR[kt]) : 0.0);
      const int e = qedge(u, vv);
#pragma unroll
      for (int ee = 0; ee < 6; ++ee)
        if (ee == e) D[ee] += cd;
    }
  }
  const double w0 = V.w[0], w1 = V.w[1], w2 = V.w[2], w3 = V.w[3];
  g[0] = c4 * (w1 * w2 * w3) + D[0] * w1 + D[1] * w2 + D[2] * w3;
  g[1] = c4 * (w0 * w2 * w3) + D[0] * w0 + D[3] * w2 + D[4] * w3;
  g[2] = c4 * (w0 * w1 * w3) + D[1] * w0 + D[3] * w1 + D[5] * w3;
  g[3] = c4 * (w0 * w1 * w2) + D[2] * w0 + D[4] * w1 + D[5] * w2;
  return n;
}

__device__ __forceinline__ uint32_t qfib_slot(uint32_t off, int lg) {
  return (off * 2654435769u) >> (32 - lg);
}

// Block-level context shared by the 4-clique kernels: rank tables in shared
// memory, output pointers, block-private counters (SHC), cotangents (ADJ).
template <bool SHC, bool ADJ>
__device__ __forceinline__ void quad_setup(QuadCtx& X, const QuadParams& Q, unsigned char* rank_smem,
                                           unsigned char* cnt_smem, unsigned long long* g_cnt,
                                           unsigned long long* g_fix, unsigned long long* d_cnt,
                                           unsigned long long* d_fix, int nh, int nd,
                                           double fscale, double dscale, const double* cot) {
  int* s_F = reinterpret_cast<int*>(rank_smem);
  const int nb2 = Q.nbins + 2;
  for (int k = threadIdx.x; k < 4 * nb2; k += blockDim.x) s_F[k] = Q.rank.F[k / nb2][k % nb2];
  __syncthreads();
  X.F = s_F;
  X.nbins = Q.nbins;
  X.ncfg = Q.ncfg;
  X.nbin = Q.tetra ? Q.nbins : Q.ncfg * Q.nbins * Q.nbins;
  X.tetra = Q.tetra;
  X.cnt = g_cnt;
  X.dcnt = d_cnt;
  X.fix = g_fix;
  X.dfix = d_fix;
  X.dhi = nd;
  X.split = Q.split;
  X.counts = Q.counts;
  X.scnt = nullptr;
  X.sdcnt = nullptr;
  if (SHC) {
    unsigned int* sc = reinterpret_cast<unsigned int*>(cnt_smem);
    for (int k = threadIdx.x; k < nh + nd; k += blockDim.x) sc[k] = 0u;
    __syncthreads();
    X.scnt = sc;
    X.sdcnt = sc + nh;
  }
  X.fscale = fscale;
  X.dscale = dscale;
  X.c2 = cot;
  X.c3 = ADJ ? cot + X.nbin : nullptr;
  X.cN = ADJ ? cot + 2 * (size_t)X.nbin : nullptr;
  X.cR = ADJ ? cot + 8 * (size_t)X.nbin : nullptr;
}

// Weighted 4PCF contributions of the warp's cliques, flattened: every lane
// first evaluates the four roots of its clique (act: the lane holds one)
// without branching -- root validity, histogram index and the other three
// vertices in catalogue-id order -- then the warp takes the valid (clique,
// root) pairs 32 at a time, every lane updating one root's N2 / N3 sum and
// its gated pair terms.  The compact per-clique loops diverge (a quarter of
// the lanes active on average); here every lane is busy in both stages.
// The pairs are ordered by root index, then lane: one ballot per root index
// gives each pair's lane with no search, and the vertex weights are read
// from the staged weights (s_w at the positions packed 10 bits each in vpos
// for vertices 1..3; vertex 0 is the warp's root, weight wp).  Products and
// histogram indices are those of quad_root.
// Returns this lane's number of rooted contributions.
template <bool SHC>
__device__ __forceinline__ int quad_contrib_flat(const QuadCtx& X, const QVerts& V,
                                                 const uint32_t m[6], bool act, unsigned vpos,
                                                 const double* s_w, double wp) {
  const int lane = threadIdx.x & 31;
  unsigned long long packed = 0;
#pragma unroll
  for (int e = 0; e < 6; ++e) packed |= (unsigned long long)meta_bin(m[e]) << (8 * e);
  unsigned rndm = 0, flw = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    rndm |= (unsigned)(V.fl[k] & FLAG_RANDOM) << k;
    flw |= (unsigned)V.fl[k] << (8 * k);
  }
  const unsigned perm = id_order(V);
  // stage 1: the four roots of this lane's clique
  unsigned vm = 0, rpk = 0;
  int kk[4];
#pragma unroll
  for (int R = 0; R < 4; ++R) {
    kk[R] = 0;
    const unsigned fr = flw >> (8 * R);
    int pos = 0;
#pragma unroll
    for (int i = 1; i < 4; ++i)
      if ((int)((perm >> (2 * i)) & 3u) == R) pos = i;
    const unsigned lowm = (1u << (2 * pos)) - 1u;
    const unsigned oth = (perm & lowm) | ((perm >> (2 * pos + 2)) << (2 * pos));
    const int u0 = (int)(oth & 3u), u1 = (int)((oth >> 2) & 3u), u2 = (int)((oth >> 4) & 3u);
    const int b1 = qbin(packed, R, u0), b2 = qbin(packed, u0, u1), b3 = qbin(packed, u1, u2),
              b4 = qbin(packed, R, u2);
    const bool ok = act && !(fr & FLAG_BUFFER) && (fr & kFlagDeg4) && b1 <= b2 && b2 <= b3 &&
                    b3 <= b4;
    if (ok) {
      const int nb2 = X.nbins + 2;
      const int cfg = 1 + (X.F[b1] - X.F[1]) + (X.F[nb2 + b2] - X.F[nb2 + b1]) +
                      (X.F[2 * nb2 + b3] - X.F[2 * nb2 + b2]) +
                      (X.F[3 * nb2 + b4] - X.F[3 * nb2 + b3]);
      const int d1 = qbin(packed, R, u1), d2 = qbin(packed, u0, u2);
      kk[R] = (cfg - 1) + X.ncfg * ((d1 - 1) + X.nbins * (d2 - 1));
      vm |= 1u << R;
    }
    rpk |= ((unsigned)R | ((unsigned)u0 << 2) | ((unsigned)u1 << 4) | ((unsigned)u2 << 6)) << (8 * R);
  }
  // stage 2: pairs (root index R, lane) in that order
  unsigned mr[4];
  int c0, c1, c2, total;
#pragma unroll
  for (int R = 0; R < 4; ++R) mr[R] = __ballot_sync(0xffffffffu, (vm >> R) & 1u);
  c0 = __popc(mr[0]);
  c1 = c0 + __popc(mr[1]);
  c2 = c1 + __popc(mr[2]);
  total = c2 + __popc(mr[3]);
  for (int i0 = 0; i0 < total; i0 += 32) {
    const int i = i0 + lane;
    const int R = i < c0 ? 0 : (i < c1 ? 1 : (i < c2 ? 2 : 3));
    const int base = R == 0 ? 0 : (R == 1 ? c0 : (R == 2 ? c1 : c2));
    const unsigned mR = R == 0 ? mr[0] : (R == 1 ? mr[1] : (R == 2 ? mr[2] : mr[3]));
    const int o = i < total ? (int)__fns(mR, 0, i - base + 1) : 0;
    // every lane takes part in each shuffle; the select comes after
    const unsigned orp = __shfl_sync(0xffffffffu, rpk, o);
    const unsigned ornd = __shfl_sync(0xffffffffu, rndm, o);
    const unsigned opos = __shfl_sync(0xffffffffu, vpos, o);
    const int k0 = __shfl_sync(0xffffffffu, kk[0], o), k1 = __shfl_sync(0xffffffffu, kk[1], o),
              k2 = __shfl_sync(0xffffffffu, kk[2], o), k3 = __shfl_sync(0xffffffffu, kk[3], o);
    if (i >= total) continue;
    const int kr = R == 0 ? k0 : (R == 1 ? k1 : (R == 2 ? k2 : k3));
    const int onr = __popc(ornd);
    const unsigned rp = (orp >> (8 * R)) & 0xffu;
    const int u0 = (int)((rp >> 2) & 3u), u1 = (int)((rp >> 4) & 3u), u2 = (int)((rp >> 6) & 3u);
    const double w1 = s_w[opos & 0x3ffu], w2 = s_w[(opos >> 10) & 0x3ffu],
                 w3 = s_w[(opos >> 20) & 0x3ffu];
    auto wsel = [&](int v) { return v == 0 ? wp : (v == 1 ? w1 : (v == 2 ? w2 : w3)); };
    qcount<SHC>(X, kr + X.nbin * onr);
    qfix(X, qfx(X.fix, kr + X.nbin * onr), qfx(X.fix, kr + X.nbin * (onr + 5)),
         ((wsel(R) * wsel(u0)) * wsel(u1)) * wsel(u2), X.fscale);
#pragma unroll
    for (int tt = 0; tt < 6; ++tt) {
      const int ga = (int)((rp >> (2 * term_gate(tt))) & 3u);
      if (!((ornd >> ga) & 1u)) continue;
      const int u = (int)((rp >> (2 * term_pu(tt))) & 3u), vv = (int)((rp >> (2 * term_pv(tt))) & 3u);
      const int npr = (int)((ornd >> u) & 1u) + (int)((ornd >> vv) & 1u);
      const int kt = kr + X.nbin * tt;
      qdcount<SHC>(X, kt + X.nbin * 6 * npr);
      qfix(X, qfx(X.dfix, kt + X.nbin * 6 * npr), qfx(X.dfix, kt + X.nbin * 6 * npr + X.dhi),
           wsel(u) * wsel(vv), X.dscale);
    }
  }
  return __popc(vm);
}

// One 4-clique (p, a, b, d) = vertices 0..3 with edge metas m: its
// contributions to the histograms, or (ADJ) its weight gradient: the root's
// to racc, those of a, b, d to the per-neighbour accumulators at positions
// ya, yb, yd.  Returns the number of rooted contributions.
template <bool WEIGHTED, bool SHC, bool ADJ, bool COMPACT, bool TETRA>
__device__ __forceinline__ int quad_emit(const QuadCtx& X, const QVerts& V, const uint32_t m[6],
                                         double gscale, Fix128& racc, unsigned long long* s_glo,
                                         unsigned long long* s_ghi, int ya, int yb, int yd) {
  if constexpr (ADJ) {
    double g[4];
    const int nroot = quad_grad_c(X, V, m, g);
    if (nroot) {
      fix_acc(racc, g[0], gscale);
      fix_add(&s_glo[ya], &s_ghi[ya], g[1], gscale);
      fix_add(&s_glo[yb], &s_ghi[yb], g[2], gscale);
      fix_add(&s_glo[yd], &s_ghi[yd], g[3], gscale);
    }
    return nroot;
  } else if constexpr (TETRA) {
    return tetra_contrib<WEIGHTED, SHC>(X, V, m);
  } else {
    static_assert(!(WEIGHTED && COMPACT), "weighted 4PCF sums take the flattened drain");
    return quad_contrib<WEIGHTED, SHC>(X, V, m);
  }
}

// SHC: integer counts in block-private 32-bit shared-memory counters,
// added to the global histograms at the end of the block.
// ADJ: instead of the histograms, the weight gradient (g_lo / g_hi, label
// order, scale gscale) of sum(c2 N2) + sum(c3 N3) + sum(cN discN) +
// sum(cR discR), cot = [c2 | c3 | cN | cR].
// COMPACT: the weighted 4PCF sums through the flattened drain
// (quad_contrib_flat) instead of the unrolled per-clique quad_contrib.
// TETRA: the -tetra counts (query_graph_tetrahedron) instead of the 4PCF;
// a template argument so that each kernel holds the code of one form only.
template <bool WEIGHTED, bool SHC, bool ADJ, bool COMPACT, bool TETRA>
__global__ void __launch_bounds__((WEIGHTED || ADJ ? kQuadMaxWarps : kQuadMaxWarpsU) * 32) quad4_kernel(
    DevCatalog C, CSRView G, QuadParams Q, unsigned long long* __restrict__ g_cnt,
    unsigned long long* __restrict__ g_fix, unsigned long long* __restrict__ d_cnt,
    unsigned long long* __restrict__ d_fix, int nh, int nd, double fscale, double dscale,
    unsigned long long* __restrict__ stats, int* __restrict__ work,
    const double* __restrict__ cot, double gscale, unsigned long long* __restrict__ g_lo,
    unsigned long long* __restrict__ g_hi) {
  constexpr bool LW = WEIGHTED || ADJ;  // weights staged
  extern __shared__ __align__(16) unsigned char smem[];
  const QuadLayout L = quad_layout(Q.nbins, Q.cap, blockDim.x >> 5, SHC ? nh + nd : 0, ADJ);
  QuadCtx X;
  quad_setup<SHC, ADJ>(X, Q, smem + L.off_rank, smem + L.off_cnt, g_cnt, g_fix, d_cnt, d_fix, nh,
                       nd, fscale, dscale, cot);

  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  unsigned char* wb = smem + L.off_warp + L.warp_bytes * (threadIdx.x >> 5);
  long long* s_rs = reinterpret_cast<long long*>(wb + L.o_rs);
  double* s_w = reinterpret_cast<double*>(wb + L.o_w);
  unsigned long long* s_mo = reinterpret_cast<unsigned long long*>(wb + L.o_mo);
  int* s_col = reinterpret_cast<int*>(wb + L.o_col);
  int* s_len = reinterpret_cast<int*>(wb + L.o_len);
  uint32_t* s_xm = reinterpret_cast<uint32_t*>(wb + L.o_xm);
  uint32_t* s_hkey = reinterpret_cast<uint32_t*>(wb + L.o_hkey);
  unsigned long long* s_q = reinterpret_cast<unsigned long long*>(wb + L.o_q);
  uint16_t* s_xy = reinterpret_cast<uint16_t*>(wb + L.o_xy);
  uint16_t* s_xz = reinterpret_cast<uint16_t*>(wb + L.o_xz);
  uint32_t* s_bits = reinterpret_cast<uint32_t*>(wb + L.o_bits);
  unsigned long long* s_glo = reinterpret_cast<unsigned long long*>(wb + L.o_g);
  unsigned long long* s_ghi = s_glo + Q.cap;
  const int cap = Q.cap;
  const int lg_max = qhash_lg_max(cap);
  unsigned long long quads = 0, rooted = 0, probes = 0;

  // position of label c in R+(p) via the hash table, or -1
  auto lookup = [&](int c, int p, int lg, bool live) -> int {
    const int off = c - p;
    live = live && off > 0 && off < kQMaxOffset;
    const int hs = 1 << lg;
    uint32_t h = qfib_slot((uint32_t)off, lg);
    uint32_t e = live ? s_hkey[h] : 0u;
    bool hit = live && (e >> 10) == (uint32_t)off;
    bool open = live && !hit && e != 0u;
    for (int it = 1; it < hs && __any_sync(0xffffffffu, open); ++it) {
      if (open) {
        h = (h + 1) & (uint32_t)(hs - 1);
        e = s_hkey[h];
        hit = (e >> 10) == (uint32_t)off;
        open = !hit && e != 0u;
      }
    }
    return hit ? (int)(e & 0x3ffu) : -1;
  };

  int nheavy;
  const int parts = quad_split_parts(Q, nheavy);
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(work, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    int p, part;
    if (!quad_item(Q, C.n, item, nheavy, parts, p, part)) break;
    const int nparts = item < nheavy * parts ? parts : 1;
    const int64_t b0 = G.start[p];
    const int k = G.len[p];
    if (k < 3 && Q.order) break;  // longest rows first: every later root is as short
    if (k < 3 || k > cap) continue;  // rows longer than cap are rejected on the host
    if (rec_col(G.rec[b0 + k - 1]) - p >= kQMaxOffset) {
      if (lane == 0) atomicMax(&stats[3], 1ull);  // reported to the host
      continue;
    }
    const uint8_t fp = C.flags[p] | (G.deg_full[p] > 3 ? kFlagDeg4 : 0);
    const int op = C.orig[p];
    const double wp = LW ? C.w[p] : 0.0;
    Fix128 racc = {0ull, 0ull};  // adjoint: gradient of the root, per lane
    int lg = 6;
    while (lg < lg_max && (1 << lg) < 8 * k) ++lg;
    const int hs = 1 << lg;
    __syncwarp();
    for (int h = lane; h < hs; h += 32) s_hkey[h] = 0u;
    __syncwarp();
    for (int xb = 0; xb < k; xb += 32) {
      const int x = xb + lane;
      if (x < k) {
        const unsigned long long r = G.rec[b0 + x];
        const int a = rec_col(r);
        s_col[x] = a;
        s_rs[x] = G.start[a];
        s_len[x] = G.len[a];
        const uint8_t fa = C.flags[a] | (G.deg_full[a] > 3 ? kFlagDeg4 : 0);
        s_mo[x] = ((unsigned long long)(uint32_t)C.orig[a] << 32) |
                  (rec_meta(r) | ((uint32_t)fa << 24));
        if (LW) s_w[x] = C.w[a];
        if (ADJ) {
          s_glo[x] = 0ull;
          s_ghi[x] = 0ull;
        }
        const uint32_t off = (uint32_t)(a - p);
        const uint32_t key = (off << 10) | (uint32_t)x;
        uint32_t h = qfib_slot(off, lg);
        for (int t = 0; t < hs; ++t) {
          if (atomicCAS(&s_hkey[h], 0u, key) == 0u) break;
          h = (h + 1) & (uint32_t)(hs - 1);
        }
      }
    }
    __syncwarp();
    const int nwords = (k + 31) >> 5;
    for (int x = part; x < k - 2; x += nparts) {  // a split root: every nparts-th a
      // X = R+(a) ∩ R+(p) beyond position x, listed in label order and
      // marked in the bitmask
      for (int wd = lane; wd < nwords; wd += 32) s_bits[wd] = 0u;
      __syncwarp();
      const int64_t ra = s_rs[x];
      const int ka = s_len[x];
      if (lane == 0) probes += (unsigned long long)ka;
      int nx = 0;
      for (int j0 = 0; j0 < ka; j0 += 32) {
        const int j = j0 + lane;
        unsigned long long rr = 0;
        if (j < ka) rr = G.rec[ra + j];
        const int y = lookup(rec_col(rr), p, lg, j < ka);
        const bool found = y > x;
        const unsigned msk = __ballot_sync(0xffffffffu, found);
        if (found) {
          const int z = nx + __popc(msk & lt);
          s_xy[z] = (uint16_t)y;
          s_xm[z] = rec_meta(rr);
          s_xz[y] = (uint16_t)z;
          atomicOr(&s_bits[y >> 5], 1u << (y & 31));
        }
        nx += __popc(msk);
      }
      __syncwarp();
      if (nx < 2) continue;
      const unsigned long long mpa_w = s_mo[x];
      int qn = 0;
      // one queued clique: (p, a = row x, b = X entry z, d = row y_d), one
      // per lane (act: the lane holds entry e).  The weighted 4PCF bins the
      // warp's cliques together (quad_contrib_flat), so every lane takes
      // part; a lane without a clique reads nothing and holds zero bins
      // (no valid root).  Every other mode bins one clique per lane.
      auto drain_one = [&](int e, bool act) {
        constexpr bool FLAT = WEIGHTED && COMPACT && !ADJ && !TETRA;
        if (!act && !FLAT) return;
        QVerts V;
        uint32_t m[6] = {0u, 0u, 0u, 0u, 0u, 0u};
        int yb = 0, yd = 0;
        V.fl[0] = V.fl[1] = V.fl[2] = V.fl[3] = 0;
        V.og[0] = V.og[1] = V.og[2] = V.og[3] = 0;
        V.w[0] = V.w[1] = V.w[2] = V.w[3] = 0.0;
        if (act) {
          const unsigned long long qe = s_q[e];
          const int z = (int)(qe & 0x3ffu);
          yd = (int)((qe >> 10) & 0x3ffu);
          const uint32_t mbd = (uint32_t)(qe >> 32);
          yb = s_xy[z];
          const unsigned long long mpb_w = s_mo[yb], mpd_w = s_mo[yd];
          V.fl[0] = fp;
          V.fl[1] = (uint8_t)((uint32_t)mpa_w >> 24);
          V.fl[2] = (uint8_t)((uint32_t)mpb_w >> 24);
          V.fl[3] = (uint8_t)((uint32_t)mpd_w >> 24);
          V.og[0] = op;
          V.og[1] = (int)(mpa_w >> 32);
          V.og[2] = (int)(mpb_w >> 32);
          V.og[3] = (int)(mpd_w >> 32);
          V.w[0] = wp;
          V.w[1] = LW ? s_w[x] : 0.0;
          V.w[2] = LW ? s_w[yb] : 0.0;
          V.w[3] = LW ? s_w[yd] : 0.0;
          // m: (p,a) (p,b) (p,d) (a,b) (a,d) (b,d)
          m[0] = (uint32_t)mpa_w & 0xffffffu;
          m[1] = (uint32_t)mpb_w & 0xffffffu;
          m[2] = (uint32_t)mpd_w & 0xffffffu;
          m[3] = s_xm[z];
          m[4] = s_xm[s_xz[yd]];
          m[5] = mbd;
        }
        int nroot;
        if constexpr (FLAT)
          nroot = quad_contrib_flat<SHC>(X, V, m, act,
                                         (unsigned)x | ((unsigned)yb << 10) | ((unsigned)yd << 20),
                                         s_w, wp);
        else
          nroot = quad_emit<WEIGHTED, SHC, ADJ, COMPACT, TETRA>(X, V, m, gscale, racc, s_glo, s_ghi,
                                                                x, yb, yd);
        quads += nroot > 0;
        rooted += nroot;
      };
      // Work items (b = X[z], d in R+(b)): X entries in batches of 32, the
      // rows of a batch flattened over the lanes in windows of 32 items.
      // One loop over the windows, with a last pass (fin) that drains the
      // cliques still queued, so that the long binning code has one call
      // site (the X data of this a are replaced next).
      int zb = 0, tot = 0, t0 = 0, nrows = 0, incl = 0, excl = 0, cz = 0, done = 0;
      long long crs = 0;
      bool fin = false;
      for (;;) {
        while (!fin && t0 >= tot) {
          if (zb >= nx) {
            fin = true;
            break;
          }
          // the next batch of X entries with their rows
          const int z = zb + lane;
          int len = 0;
          long long rs = 0;
          if (z < nx) {
            const int yb = s_xy[z];
            len = s_len[yb];
            rs = s_rs[yb];
          }
          const unsigned nz = __ballot_sync(0xffffffffu, len > 0);
          nrows = __popc(nz);
          const int src = lane < nrows ? (int)__fns(nz, 0, lane + 1) : 0;
          // every lane takes part in each shuffle; the select comes after
          const int slen = __shfl_sync(0xffffffffu, len, src);
          const int clen = lane < nrows ? slen : 0;
          crs = __shfl_sync(0xffffffffu, rs, src);
          cz = zb + src;
          incl = clen;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int yv = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += yv;
          }
          tot = __shfl_sync(0xffffffffu, incl, 31);
          excl = incl - clen;
          if (lane == 0) probes += (unsigned long long)tot;
          done = 0;  // compacted rows that ended before the window
          t0 = 0;
          zb += 32;
        }
        if (!fin) {
          const int last = incl - 1 - t0;
          const unsigned bit = (lane < nrows && last >= 0 && last < 32) ? (1u << last) : 0u;
          const unsigned ends = __reduce_or_sync(0xffffffffu, bit);
          const int j = (done + __popc(ends & lt)) & 31;
          done += __popc(ends);
          const long long ors = __shfl_sync(0xffffffffu, crs, j);
          const int oex = __shfl_sync(0xffffffffu, excl, j);
          const int oz = __shfl_sync(0xffffffffu, cz, j);
          const int t = t0 + lane;
          unsigned long long rr = 0;
          if (t < tot) rr = G.rec[ors + (t - oex)];
          const int yd = lookup(rec_col(rr), p, lg, t < tot);
          const bool hit = yd >= 0 && ((s_bits[yd >> 5] >> (yd & 31)) & 1u);
          const unsigned m = __ballot_sync(0xffffffffu, hit);
          if (hit) {
            const int pos = qn + __popc(m & lt);
            s_q[pos] = ((unsigned long long)rec_meta(rr) << 32) | (uint32_t)(oz | (yd << 10));
          }
          qn += __popc(m);
          t0 += 32;
        }
        if (qn >= 32 || (fin && qn > 0)) {
          const int nq = min(qn, 32);
          __syncwarp();
          drain_one(qn - nq + lane, lane < nq);
          qn -= nq;
          __syncwarp();
        }
        if (fin && qn == 0) break;
      }
      __syncwarp();
    }
    if (ADJ) {
      // flush the gradients of this root and of its neighbours
      for (int x = lane; x < k; x += 32) {
        const unsigned long long lo = s_glo[x], hi = s_ghi[x];
        if (lo | hi) fix_merge(&g_lo[s_col[x]], &g_hi[s_col[x]], lo, hi);
      }
      racc = fix_warp_sum(racc);
      if (lane == 0 && (racc.lo | racc.hi)) fix_merge(&g_lo[p], &g_hi[p], racc.lo, racc.hi);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    quads += __shfl_xor_sync(0xffffffffu, quads, o);
    rooted += __shfl_xor_sync(0xffffffffu, rooted, o);
    probes += __shfl_xor_sync(0xffffffffu, probes, o);
  }
  if (lane == 0) {
    if (quads) atomicAdd(&stats[0], quads);
    if (rooted) atomicAdd(&stats[1], rooted);
    if (probes) atomicAdd(&stats[2], probes);
  }
  if (SHC) {
    __syncthreads();
    for (int k = threadIdx.x; k < nh + nd; k += blockDim.x) {
      const unsigned int v = X.scnt[k];
      if (v) atomicAdd(k < nh ? &X.cnt[k] : &X.dcnt[k - nh], (unsigned long long)v);
    }
  }
}

// Geometric mode.  The edges among the members of R+(p) are exactly the
// pairs that pass the graph's membership test, so the warp tests the
// k(k-1)/2 pairs of R+(p) once (closed-form inversion of the triangular pair
// index over the lanes) and records them as one adjacency bitmask row per
// member (bits of the later members).  The 4-cliques p < a < b < d are then
// the set bits d of row(a) AND row(b) for every edge (a, b): the edges are
// queued 32 at a time, each lane ANDs its two rows word by word and emits one
// clique per set bit into the clique queue.  The bins of (a, b), (a, d) and
// (b, d) are computed from the positions as the graph build computes them
// (edge_rbin), the bin of (a, b) once per edge.  No row other than R+(p) is
// read; the tests are k(k-1)/2 per root instead of the sum over R+(p) of the
// members' row lengths.  Rows up to 256 members (8-bit positions).
constexpr int kQEdgeQueue = 64;  // edge queue entries per warp (< 32 left + 32 pushed)

struct QuadGLayout {
  size_t off_rank, off_cnt, off_warp, warp_bytes, total;
  size_t o_pos, o_w, o_mo, o_g, o_col, o_adj, o_q, o_eq;
};

__host__ __device__ inline QuadGLayout quadg_layout(int nbins, int cap, int nwarps, int ncounts,
                                                    bool adj, bool lw) {
  QuadGLayout L;
  size_t o = 0;
  L.off_rank = o;
  o = qalign8(o + sizeof(int) * 4 * (size_t)(nbins + 2));
  L.off_cnt = o;
  o = o + sizeof(unsigned int) * (size_t)ncounts;
  o = (o + 15) & ~(size_t)15;
  L.off_warp = o;
  const size_t nwd = (size_t)(cap + 31) / 32;
  size_t w = 0;
  L.o_pos = w;  w += (size_t)cap * 16;              // float4 position of each member
  L.o_w = w;    w += lw ? (size_t)cap * 8 : 0;      // weight
  L.o_mo = w;   w += (size_t)cap * 8;               // (catalogue id << 32) | flags << 24 | meta(p, a)
  L.o_g = w;    w += adj ? (size_t)cap * 16 : 0;    // gradient (lo, hi)
  L.o_col = w;  w += (size_t)cap * 4;               // label
  L.o_adj = w;  w += (size_t)cap * nwd * 4;         // adjacency rows
  L.o_q = w;    w += (size_t)kQQueue * 4;           // cliques: a | b << 8 | d << 16 | bin(a,b) << 24
  L.o_eq = w;   w += (size_t)kQEdgeQueue * 4;       // edges: a | b << 8
  L.warp_bytes = (w + 15) & ~(size_t)15;
  L.total = o + L.warp_bytes * nwarps;
  return L;
}

template <bool WEIGHTED, bool SHC, bool ADJ, bool COMPACT, bool TETRA>
__global__ void __launch_bounds__((ADJ ? kQuadGWarpsA : (WEIGHTED ? kQuadGWarpsW : kQuadMaxWarpsU)) * 32)
    quad4g_kernel(
    DevCatalog C, CSRView G, QuadParams Q, unsigned long long* __restrict__ g_cnt,
    unsigned long long* __restrict__ g_fix, unsigned long long* __restrict__ d_cnt,
    unsigned long long* __restrict__ d_fix, int nh, int nd, double fscale, double dscale,
    unsigned long long* __restrict__ stats, int* __restrict__ work,
    const double* __restrict__ cot, double gscale, unsigned long long* __restrict__ g_lo,
    unsigned long long* __restrict__ g_hi) {
  constexpr bool LW = WEIGHTED || ADJ;
  extern __shared__ __align__(16) unsigned char smem[];
  const QuadGLayout L = quadg_layout(Q.nbins, Q.cap, blockDim.x >> 5, SHC ? nh + nd : 0, ADJ, LW);
  QuadCtx X;
  quad_setup<SHC, ADJ>(X, Q, smem + L.off_rank, smem + L.off_cnt, g_cnt, g_fix, d_cnt, d_fix, nh,
                       nd, fscale, dscale, cot);
  const PairParams& P = Q.P;

  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  unsigned char* wb = smem + L.off_warp + L.warp_bytes * (threadIdx.x >> 5);
  float4* s_pos = reinterpret_cast<float4*>(wb + L.o_pos);
  double* s_w = reinterpret_cast<double*>(wb + L.o_w);
  unsigned long long* s_mo = reinterpret_cast<unsigned long long*>(wb + L.o_mo);
  unsigned long long* s_glo = reinterpret_cast<unsigned long long*>(wb + L.o_g);
  unsigned long long* s_ghi = s_glo + Q.cap;
  int* s_col = reinterpret_cast<int*>(wb + L.o_col);
  uint32_t* s_adj = reinterpret_cast<uint32_t*>(wb + L.o_adj);
  uint32_t* s_q = reinterpret_cast<uint32_t*>(wb + L.o_q);
  uint32_t* s_eq = reinterpret_cast<uint32_t*>(wb + L.o_eq);
  unsigned long long quads = 0, rooted = 0, probes = 0;

  int nheavy;
  const int parts = quad_split_parts(Q, nheavy);
  for (;;) {
    int item = 0;
    if (lane == 0) item = atomicAdd(work, 1);
    item = __shfl_sync(0xffffffffu, item, 0);
    int p, part;
    if (!quad_item(Q, C.n, item, nheavy, parts, p, part)) break;
    const int nparts = item < nheavy * parts ? parts : 1;
    const int64_t b0 = G.start[p];
    const int k = G.len[p];
    if (k < 3 && Q.order) break;  // longest rows first: every later root is as short
    if (k < 3 || k > Q.cap) continue;  // rows longer than cap are rejected on the host
    const uint8_t fp = C.flags[p] | (G.deg_full[p] > 3 ? kFlagDeg4 : 0);
    const int op = C.orig[p];
    const double wp = LW ? C.w[p] : 0.0;
    Fix128 racc = {0ull, 0ull};
    const int nwk = (k + 31) >> 5;  // adjacency words per row for this root
    __syncwarp();
    for (int x = lane; x < k; x += 32) {
      const unsigned long long r = G.rec[b0 + x];
      const int a = rec_col(r);
      s_col[x] = a;
      s_pos[x] = C.pos4[a];
      const uint8_t fa = C.flags[a] | (G.deg_full[a] > 3 ? kFlagDeg4 : 0);
      s_mo[x] = ((unsigned long long)(uint32_t)C.orig[a] << 32) | (rec_meta(r) | ((uint32_t)fa << 24));
      if (LW) s_w[x] = C.w[a];
      if (ADJ) {
        s_glo[x] = 0ull;
        s_ghi[x] = 0ull;
      }
    }
    for (int i = lane; i < k * nwk; i += 32) s_adj[i] = 0u;
    __syncwarp();
    // pass 1: adjacency among the members of R+(p)
    const int npair = k * (k - 1) / 2;
    const int k2m1 = 2 * k - 1;
    if (lane == 0 && part == 0) probes += (unsigned long long)npair;  // once per root
    auto pair_of = [&](int t, int& x, int& y) {
      // x: the largest row with x (2k - 1 - x) / 2 <= t pairs before it
      // (exact up to kPairRowExact members, else one adjustment each way)
      x = pair_row_biased(k2m1, t);
      if (k > kPairRowExact) {
        x = max(0, min(x, k - 2));
        if ((x + 1) * (k2m1 - x - 1) / 2 <= t) ++x;
        if (x * (k2m1 - x) / 2 > t) --x;
      }
      y = t - (int)((unsigned)(x * (k2m1 - x)) >> 1) + x + 1;
    };
    for (int t = lane; t < npair; t += 32) {
      int x, y;
      pair_of(t, x, y);
      int r = P.f32 ? member_f32(s_pos[x], s_pos[y], P) : 2;
      if (r == 2) {
        int b, mf, mr;
        r = edge_f64(C.posd[s_col[x]], C.posd[s_col[y]], P, b, mf, mr) ? 1 : 0;
      }
      if (r == 1) atomicOr(&s_adj[x * nwk + (y >> 5)], 1u << (y & 31));
    }
    __syncwarp();
    int qn = 0, en = 0;
    // one queued clique: (p, a = member x, b = member y, d = member z), one
    // per lane (act: the lane holds entry e).  The weighted 4PCF bins the
    // warp's cliques together (quad_contrib_flat): every lane takes part, a
    // lane without a clique reads nothing and holds no valid root.
    auto drain_one = [&](int e, bool act) {
      constexpr bool FLAT = WEIGHTED && COMPACT && !ADJ && !TETRA;
      if (!act && !FLAT) return;
      QVerts V;
      uint32_t m[6] = {0u, 0u, 0u, 0u, 0u, 0u};
      int x = 0, y = 0, z = 0;
      V.fl[0] = V.fl[1] = V.fl[2] = V.fl[3] = 0;
      V.og[0] = V.og[1] = V.og[2] = V.og[3] = 0;
      V.w[0] = V.w[1] = V.w[2] = V.w[3] = 0.0;
      if (act) {
        const uint32_t qe = s_q[e];
        x = (int)(qe & 0xffu);
        y = (int)((qe >> 8) & 0xffu);
        z = (int)((qe >> 16) & 0xffu);
        const int bxy = (int)(qe >> 24);
        const int bxz = edge_rbin(C.posd, P, s_col[x], s_col[z], s_pos[x], s_pos[z]);
        const int byz = edge_rbin(C.posd, P, s_col[y], s_col[z], s_pos[y], s_pos[z]);
        const unsigned long long ma = s_mo[x], mb = s_mo[y], md = s_mo[z];
        V.fl[0] = fp;
        V.fl[1] = (uint8_t)((uint32_t)ma >> 24);
        V.fl[2] = (uint8_t)((uint32_t)mb >> 24);
        V.fl[3] = (uint8_t)((uint32_t)md >> 24);
        V.og[0] = op;
        V.og[1] = (int)(ma >> 32);
        V.og[2] = (int)(mb >> 32);
        V.og[3] = (int)(md >> 32);
        V.w[0] = wp;
        V.w[1] = LW ? s_w[x] : 0.0;
        V.w[2] = LW ? s_w[y] : 0.0;
        V.w[3] = LW ? s_w[z] : 0.0;
        // m: (p,a) (p,b) (p,d) (a,b) (a,d) (b,d)
        m[0] = (uint32_t)ma & 0xffffffu;
        m[1] = (uint32_t)mb & 0xffffffu;
        m[2] = (uint32_t)md & 0xffffffu;
        m[3] = pack_meta(bxy, 1, 1);
        m[4] = pack_meta(bxz, 1, 1);
        m[5] = pack_meta(byz, 1, 1);
      }
      int nroot;
      if constexpr (FLAT)
        nroot = quad_contrib_flat<SHC>(X, V, m, act,
                                       (unsigned)x | ((unsigned)y << 10) | ((unsigned)z << 20), s_w,
                                       wp);
      else
        nroot = quad_emit<WEIGHTED, SHC, ADJ, COMPACT, TETRA>(X, V, m, gscale, racc, s_glo, s_ghi,
                                                              x, y, z);
      quads += nroot > 0;
      rooted += nroot;
    };
    // the cliques of up to 32 queued edges (entry e, or none when e < 0);
    // every lane takes part.  fin: also drain the cliques still queued.
    // (One call site each for this and drain_one: their code is long.)
    auto run_edges = [&](int e, bool fin) {
      const bool live = e >= 0;
      int x = 0, y = 0, bxy = 0, cw = 0;
      unsigned cm = 0u;
      if (live) {
        const uint32_t ent = s_eq[e];
        x = (int)(ent & 0xffu);
        y = (int)((ent >> 8) & 0xffu);
        cw = y >> 5;
        cm = s_adj[x * nwk + cw] & s_adj[y * nwk + cw];
        bxy = edge_rbin(C.posd, P, s_col[x], s_col[y], s_pos[x], s_pos[y]);
      }
      for (;;) {
        if (live)
          while (cm == 0u && cw + 1 < nwk) {
            ++cw;
            cm = s_adj[x * nwk + cw] & s_adj[y * nwk + cw];
          }
        const bool has = live && cm != 0u;
        const unsigned hm = __ballot_sync(0xffffffffu, has);
        if (has) {
          const int z = cw * 32 + __ffs(cm) - 1;
          cm &= cm - 1u;
          s_q[qn + __popc(hm & lt)] = (uint32_t)(x | (y << 8) | (z << 16) | (bxy << 24));
        }
        qn += __popc(hm);
        if (qn >= 32 || (fin && hm == 0u && qn > 0)) {
          const int nq = min(qn, 32);
          __syncwarp();
          drain_one(qn - nq + lane, lane < nq);
          qn -= nq;
          __syncwarp();
        }
        if (hm == 0u && (!fin || qn == 0)) break;
      }
    };
    // pass 2: the edges in pair order, 32 at a time, then what is queued
    // (a split root: every nparts-th chunk of 32 pairs)
    for (int t0 = 0;; t0 += 32) {
      if (t0 < npair && ((t0 >> 5) % nparts) == part) {
        const int t = t0 + lane;
        bool edge = false;
        int x = 0, y = 0;
        if (t < npair) {
          pair_of(t, x, y);
          edge = (s_adj[x * nwk + (y >> 5)] >> (y & 31)) & 1u;
        }
        const unsigned em = __ballot_sync(0xffffffffu, edge);
        if (edge) s_eq[en + __popc(em & lt)] = (uint32_t)(x | (y << 8));
        en += __popc(em);
      }
      const bool last = t0 + 32 >= npair;
      if (en >= 32 || last) {
        const int ne = min(en, 32);
        const bool fin = last && en == ne;
        __syncwarp();
        run_edges(lane < ne ? en - ne + lane : -1, fin);
        en -= ne;
        __syncwarp();
        if (fin) break;
      }
    }
    if (ADJ) {
      for (int x = lane; x < k; x += 32) {
        const unsigned long long lo = s_glo[x], hi = s_ghi[x];
        if (lo | hi) fix_merge(&g_lo[s_col[x]], &g_hi[s_col[x]], lo, hi);
      }
      racc = fix_warp_sum(racc);
      if (lane == 0 && (racc.lo | racc.hi)) fix_merge(&g_lo[p], &g_hi[p], racc.lo, racc.hi);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    quads += __shfl_xor_sync(0xffffffffu, quads, o);
    rooted += __shfl_xor_sync(0xffffffffu, rooted, o);
    probes += __shfl_xor_sync(0xffffffffu, probes, o);
  }
  if (lane == 0) {
    if (quads) atomicAdd(&stats[0], quads);
    if (rooted) atomicAdd(&stats[1], rooted);
    if (probes) atomicAdd(&stats[2], probes);
  }
  if (SHC) {
    __syncthreads();
    for (int k = threadIdx.x; k < nh + nd; k += blockDim.x) {
      const unsigned int v = X.scnt[k];
      if (v) atomicAdd(k < nh ? &X.cnt[k] : &X.dcnt[k - nh], (unsigned long long)v);
    }
  }
}

// Warps per block: as many as fit in shared memory (at most maxw).
int quad4_warps(int nbins, int cap, int ncounts, bool adj = false, int maxw = kQuadMaxWarps) {
  int nw = maxw;
  while (nw > 1 && quad_layout(nbins, cap, nw, ncounts, adj).total > kQuadSmemLimit) nw -= 1;
  return nw;
}

}  // namespace

// Warps per block of the geometric kernel (at most maxw).
static int quadg_warps(int nbins, int cap, int ncounts, bool adj, bool lw, int maxw) {
  int nw = maxw;
  while (nw > 1 && quadg_layout(nbins, cap, nw, ncounts, adj, lw).total > kQuadSmemLimit) nw -= 1;
  return nw;
}

// Launch of either 4-clique kernel: grid of resident blocks, dynamic roots.
template <typename K>
static void launch_quad_grid(K kfn, int nw, size_t smem, int n, int* work, cudaStream_t s,
                             const DevCatalog& C, const CSRView& G, const QuadParams& Q,
                             unsigned long long* g_cnt, unsigned long long* g_fix,
                             unsigned long long* d_cnt, unsigned long long* d_fix, int nh, int nd,
                             double fscale, double dscale, unsigned long long* stats,
                             const double* cot, double gscale, unsigned long long* g_lo,
                             unsigned long long* g_hi) {
  if (smem > kQuadSmemLimit) throw Error{-2, "4PCF: per-warp shared memory exceeds the SM limit"};
  GR_CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  GR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, nw * 32, smem));
  if (per_sm < 1) per_sm = 1;
  int64_t blocks = (int64_t)per_sm * sm_count();
  const int64_t need = ((int64_t)n + nw - 1) / nw;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  GR_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int), s));
  kfn<<<(unsigned)blocks, nw * 32, smem, s>>>(C, G, Q, g_cnt, g_fix, d_cnt, d_fix, nh, nd, fscale,
                                              dscale, stats, work, cot, gscale, g_lo, g_hi);
  GR_CHECK_LAUNCH();
}

bool launch_quad4(const DevCatalog& C, const CSRView& G, const QuadParams& Q, bool weighted,
                  unsigned long long* g_cnt, unsigned long long* g_fix, unsigned long long* d_cnt,
                  unsigned long long* d_fix, int nh, int nd, double fscale, double dscale,
                  bool shared_counts, unsigned long long* stats, int* work, cudaStream_t s) {
  if (C.n <= 0) return false;
  const bool geo = Q.geo != 0;
  const int maxw = weighted ? (geo ? kQuadGWarpsW : kQuadMaxWarps) : kQuadMaxWarpsU;
  auto warps = [&](int ncounts, int mw) {
    return geo ? quadg_warps(Q.nbins, Q.cap, ncounts, false, weighted, mw)
               : quad4_warps(Q.nbins, Q.cap, ncounts, false, mw);
  };
  // integer counts in block-private counters when they leave room for at
  // least 8 warps (weighted sums without counts need none)
  const int ncnt = nh + nd;
  if ((weighted && !Q.counts) || warps(ncnt, kQuadMaxWarps) < 8) shared_counts = false;
  const int nc = shared_counts ? ncnt : 0;
  const int nw = warps(nc, maxw);
  const size_t smem = geo ? quadg_layout(Q.nbins, Q.cap, nw, nc, false, weighted).total
                          : quad_layout(Q.nbins, Q.cap, nw, nc).total;
  // weighted: the compact contribution code (the unrolled form of its long
  // fixed-point updates overflows the instruction cache); unweighted: unrolled
  auto go = [&](auto kfn) {
    launch_quad_grid(kfn, nw, smem, C.n, work, s, C, G, Q, g_cnt, g_fix, d_cnt, d_fix, nh, nd,
                     fscale, dscale, stats, nullptr, 1.0, nullptr, nullptr);
  };
  auto pick = [&](auto geo_t, auto tetra_t) {
    constexpr bool GEO = decltype(geo_t)::value, TT = decltype(tetra_t)::value;
    if constexpr (GEO) {
      if (weighted && shared_counts) go(quad4g_kernel<true, true, false, true, TT>);
      else if (weighted) go(quad4g_kernel<true, false, false, true, TT>);
      else if (shared_counts) go(quad4g_kernel<false, true, false, false, TT>);
      else go(quad4g_kernel<false, false, false, false, TT>);
    } else {
      if (weighted && shared_counts) go(quad4_kernel<true, true, false, true, TT>);
      else if (weighted) go(quad4_kernel<true, false, false, true, TT>);
      else if (shared_counts) go(quad4_kernel<false, true, false, false, TT>);
      else go(quad4_kernel<false, false, false, false, TT>);
    }
  };
  using T1 = std::true_type;
  using T0 = std::false_type;
  if (geo)
    Q.tetra ? pick(T1{}, T1{}) : pick(T1{}, T0{});
  else
    Q.tetra ? pick(T0{}, T1{}) : pick(T0{}, T0{});
  return shared_counts;
}

void launch_adj4(const DevCatalog& C, const CSRView& G, const QuadParams& Q, const double* cot,
                 double gscale, unsigned long long* g_lo, unsigned long long* g_hi,
                 unsigned long long* stats, int* work, cudaStream_t s) {
  if (C.n <= 0) return;
  if (Q.geo) {
    const int nw = quadg_warps(Q.nbins, Q.cap, 0, true, true, kQuadGWarpsA);
    const size_t smem = quadg_layout(Q.nbins, Q.cap, nw, 0, true, true).total;
    launch_quad_grid(quad4g_kernel<false, false, true, true, false>, nw, smem, C.n, work, s, C, G, Q,
                     nullptr, nullptr, nullptr, nullptr, 0, 0, 1.0, 1.0, stats, cot, gscale, g_lo,
                     g_hi);
  } else {
    const int nw = quad4_warps(Q.nbins, Q.cap, 0, true);
    const size_t smem = quad_layout(Q.nbins, Q.cap, nw, 0, true).total;
    launch_quad_grid(quad4_kernel<false, false, true, true, false>, nw, smem, C.n, work, s, C, G, Q,
                     nullptr, nullptr, nullptr, nullptr, 0, 0, 1.0, 1.0, stats, cot, gscale, g_lo,
                     g_hi);
  }
}

void quad_expand_patterns(const unsigned long long* H, int nbin, unsigned long long* hc,
                          unsigned long long* dc) {
  std::fill(hc, hc + (size_t)nbin * 5, 0ull);
  std::fill(dc, dc + (size_t)nbin * 6 * 3, 0ull);
  for (int pat = 0; pat < kQuadPatterns; ++pat) {
    const int nr = __builtin_popcount((unsigned)pat);
    for (int k = 0; k < nbin; ++k) {
      const unsigned long long v = H[k + (size_t)nbin * pat];
      if (!v) continue;
      hc[k + (size_t)nbin * nr] += v;
      for (int tt = 0; tt < 6; ++tt) {
        if (!((pat >> term_gate(tt)) & 1)) continue;
        const int npr = ((pat >> term_pu(tt)) & 1) + ((pat >> term_pv(tt)) & 1);
        dc[k + (size_t)nbin * tt + (size_t)nbin * 6 * npr] += v;
      }
    }
  }
}

size_t quad4_smem_bytes(int nbins, int cap) {
  return quad_layout(nbins, cap, quad4_warps(nbins, cap, 0), 0).total;
}

}  // namespace gr
