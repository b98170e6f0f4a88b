// CPU oracle for the N-point-correlation hot path of Gramsci (csabiu/Gramsci).
//
// TEST INFRASTRUCTURE ONLY.  This file restates, on the CPU and in plain IEEE
// FP64 with no FMA contraction, the algorithm of the reference program
// (src/gramsci.F90, src/kdtree2.F90, src/sorting_module.F90).  Only tests/,
// the smoke check and the CPU-baseline leg of bench.py load it, and only to
// check the library's results or as the timed CPU baseline.  The CUDA library
// never calls it.
//
// Parity status: UNPINNED against reference outputs.  The reference is
// Fortran; no Fortran compiler exists in the build container or on the GPU
// host, and the only known-answer values the reference ships
// (tests/run_correlation_tests.py:28-29,39-40) need example/test.gal and
// example/test.ran, which are missing from the reference tree.  The oracle is
// instead pinned by (1) hand-derived configurations (tests/golden), (2) an
// independent brute-force enumeration in the Python tests, and (3) agreement
// between two independent range searches (uniform grid and kd-tree).
//
// Floating-point convention.  The reference is built with gfortran -Ofast,
// whose FMA contraction and reassociation choices cannot be reproduced
// without the compiler.  This oracle fixes one evaluation: left-to-right
// sums, separate multiply and add (compile with -ffp-contract=off).  Results
// can differ from a given reference binary only for pairs whose separation
// or line-of-sight cosine lies within about one ulp of a bin edge.
//
// Definitions of reference undefined behaviour (kept identical in the CUDA
// library):
//  * radial bin nbins+1 (d within rounding of rmax) is clamped to nbins
//    (the reference indexes one past the histogram, gramsci.F90:337);
//  * a NaN line-of-sight cosine (pair midpoint at the origin) gives mu bin 1;
//  * non-canonical 4PCF bin-table entries are 0 (gramsci.F90:1402-1414 leave
//    them uninitialised);
//  * find_normal with a negative radicand gives bin 1 (gramsci.F90:1619).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#else
static inline int omp_get_max_threads() { return 1; }
static inline int omp_get_thread_num() { return 0; }
#endif

#if defined(__FP_FAST_FMA) && !defined(ORACLE_ALLOW_FMA)
// Contraction is switched off by the build recipe; this guard only documents
// that the oracle's arithmetic must not be fused.
#endif

typedef long double acc_t;  // reference-grade accumulator for category sums

namespace {

// ---------------------------------------------------------------- binning --
// gramsci.F90:88-96 (radial_bins), :136-145 (delta_r, inv_delta_r, log_rmin),
// :147 (mu_scale = 0.5*nmu), :1216-1223 (RSD when nmu >= 2).
struct Bins {
  double rmin, rmax, rmin2, rmax2, delta_r, inv_dr, log_rmin, mu_scale;
  int nbins, nmu;
  bool logbins, rsd;
};

Bins make_bins(double rmin, double rmax, int nbins, int nmu, int logbins) {
  Bins b;
  b.rmin = rmin;
  b.rmax = rmax;
  b.rmin2 = rmin * rmin;  // kdtree2 ball size r2=rmin*rmin (gramsci.F90:302)
  b.rmax2 = rmax * rmax;  // r2=rmax*rmax (gramsci.F90:296)
  b.nbins = nbins;
  b.nmu = nmu;
  b.logbins = logbins != 0;
  b.rsd = nmu >= 2;
  b.log_rmin = 0.0;
  if (b.logbins) {
    b.delta_r = (std::log10(rmax) - std::log10(rmin)) / (double)nbins;
    b.inv_dr = 1.0 / b.delta_r;
    b.log_rmin = std::log10(rmin);
  } else {
    b.delta_r = (rmax - rmin) / (double)nbins;
    b.inv_dr = 1.0 / b.delta_r;
  }
  b.mu_scale = (double)(0.5f * (float)nmu);
  return b;
}

// mu bin of a line-of-sight cosine: floor((theta+1)*mu_scale)+1 clamped to
// [1,nmu] (gramsci.F90:326-328).  NaN -> 1.
inline int mu_bin(double theta, const Bins& B) {
  double v = (theta + 1.0) * B.mu_scale;
  if (!(v == v)) return 1;
  double f = std::floor(v);
  if (f < -1.0e9) return 1;
  if (f > 1.0e9) return B.nmu;
  int m = (int)f + 1;
  if (m < 1) m = 1;
  if (m > B.nmu) m = B.nmu;
  return m;
}

// The reference edge predicate and bin assignment for root i, neighbour j.
// kdtree2.F90:1685-1690 accumulates sd = (x_j-x_i)^2 + (y_j-y_i)^2 +
// (z_j-z_i)^2 left to right; the r2=rmax^2 search keeps sd <= rmax^2, the
// first nn1 results (sd <= rmin^2, self included) are skipped
// (gramsci.F90:295-311), then dist() recomputes d = sqrt(sd) and keeps
// rmin < d < rmax (gramsci.F90:313-317).  Radial bin :337, mu :320-332.
// mu_rev is the bin seen from j (theta exactly negated).
inline bool edge_eval(const double* pi, const double* pj, const Bins& B,
                      int* bin, int* mu_fwd, int* mu_rev) {
  double dx = pj[0] - pi[0];
  double dy = pj[1] - pi[1];
  double dz = pj[2] - pi[2];
  double sd = dx * dx;
  sd = sd + dy * dy;
  sd = sd + dz * dz;
  if (sd > B.rmax2) return false;
  if (B.rmin > 0.0 && sd <= B.rmin2) return false;
  double d = std::sqrt(sd);
  if (d <= B.rmin) return false;
  if (d >= B.rmax) return false;
  double t;
  if (B.logbins)
    t = (std::log10(d) - B.log_rmin) * B.inv_dr;
  else
    t = (d - B.rmin) * B.inv_dr;
  int b = (int)std::floor(t) + 1;
  if (b > B.nbins) b = B.nbins;
  if (b < 1) b = 1;
  *bin = b;
  if (B.rsd) {
    double m0 = 0.5 * (pi[0] + pj[0]);
    double m1 = 0.5 * (pi[1] + pj[1]);
    double m2 = 0.5 * (pi[2] + pj[2]);
    double s0 = pi[0] - pj[0];
    double s1 = pi[1] - pj[1];
    double s2 = pi[2] - pj[2];
    double th = m0 * s0;
    th = th + m1 * s1;
    th = th + m2 * s2;
    double nm = m0 * m0;
    nm = nm + m1 * m1;
    nm = nm + m2 * m2;
    double ns = s0 * s0;
    ns = ns + s1 * s1;
    ns = ns + s2 * s2;
    th = th / (std::sqrt(nm) * std::sqrt(ns));
    *mu_fwd = mu_bin(th, B);
    *mu_rev = mu_bin(-th, B);
  } else {
    *mu_fwd = 1;
    *mu_rev = 1;
  }
  return true;
}

// ------------------------------------------------------------ bin tables --
// Rank of a non-decreasing k-tuple over [1,n] in lexicographic order, i.e.
// the value create_binlookup assigns (gramsci.F90:1398-1477).  3PCF tables
// are symmetric (any permutation maps to the rank of the sorted triple);
// 4PCF tables hold only the canonical entries, everything else is 0.
int64_t ncomb_multiset(int64_t m, int r) {  // C(m+r-1, r)
  if (r == 0) return 1;
  if (m <= 0) return 0;
  int64_t num = 1, den = 1;
  for (int i = 0; i < r; ++i) {
    num *= (m + i);
    den *= (i + 1);
  }
  return num / den;
}

int64_t rank_sorted(const int* x, int k, int n) {  // x 1-based, non-decreasing
  int64_t rank = 0;
  int prev = 1;
  for (int j = 0; j < k; ++j) {
    for (int v = prev; v < x[j]; ++v) rank += ncomb_multiset(n - v + 1, k - j - 1);
    prev = x[j];
  }
  return rank + 1;
}

int bintable3(int a, int b, int c, int n) {
  int x[3] = {a, b, c};
  std::sort(x, x + 3);
  return (int)rank_sorted(x, 3, n);
}

int bintable4(int a, int b, int c, int d, int n) {
  if (!(a <= b && b <= c && c <= d)) return 0;
  int x[4] = {a, b, c, d};
  return (int)rank_sorted(x, 4, n);
}

// find_normal (gramsci.F90:1611-1625) in single precision.  variant 0:
// separate IEEE operations left to right; variant 1: the FMA contraction an
// FMA-capable gfortran -Ofast build would plausibly emit.
int find_normal(int mu1, int mu2, int nmu, double mu_scale, int variant) {
  volatile float a = (float)((double)((float)mu1 - 0.5f) / mu_scale - 1.0);
  volatile float b = (float)((double)((float)mu2 - 0.5f) / mu_scale - 1.0);
  float r;
  if (variant == 0) {
    volatile float t1 = a * a;
    volatile float s1 = 0.75f - t1;
    volatile float t2 = b * b;
    volatile float s2 = s1 - t2;
    volatile float t3 = a * b;
    r = s2 + t3;
  } else {
    float s1 = std::fmaf(-a, a, 0.75f);
    float s2 = std::fmaf(-b, b, s1);
    r = std::fmaf(a, b, s2);
  }
  volatile float sq = std::sqrt(r);
  volatile float v = 1.1547f * sq;
  volatile float v2 = v * (float)nmu;
  if (!(v2 == v2)) return 1;
  float f = std::floor(v2);
  int m = (int)f + 1;
  if (m < 1) m = 1;
  if (m > nmu) m = nmu;
  return m;
}

// ----------------------------------------------------------- neighbour grid --
struct Grid {
  double lo[3], cs[3];
  int nc[3];
  std::vector<int64_t> start;  // per cell, size ncells+1
  std::vector<int32_t> idx;    // point indices grouped by cell, ascending
};

void build_grid(const double* xyz, int64_t n, double rmax, Grid& g) {
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  if (n > 0) {
    for (int d = 0; d < 3; ++d) lo[d] = hi[d] = xyz[d];
    for (int64_t i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) {
        lo[d] = std::min(lo[d], xyz[3 * i + d]);
        hi[d] = std::max(hi[d], xyz[3 * i + d]);
      }
  }
  double cell_min = rmax * 1.000001 + 1e-300;
  int64_t total = 1;
  for (int d = 0; d < 3; ++d) {
    double span = hi[d] - lo[d];
    int64_t k = (int64_t)std::floor(span / cell_min);
    if (k < 1) k = 1;
    if (k > 1024) k = 1024;
    g.nc[d] = (int)k;
    g.lo[d] = lo[d];
    g.cs[d] = span > 0 ? span / (double)k : 1.0;
    total *= k;
  }
  g.start.assign(total + 1, 0);
  std::vector<int64_t> key(n);
  for (int64_t i = 0; i < n; ++i) {
    int c[3];
    for (int d = 0; d < 3; ++d) {
      int v = (int)std::floor((xyz[3 * i + d] - g.lo[d]) / g.cs[d]);
      c[d] = std::min(std::max(v, 0), g.nc[d] - 1);
    }
    key[i] = ((int64_t)c[2] * g.nc[1] + c[1]) * g.nc[0] + c[0];
    g.start[key[i] + 1]++;
  }
  for (int64_t c = 0; c < total; ++c) g.start[c + 1] += g.start[c];
  g.idx.resize(n);
  std::vector<int64_t> fill(g.start.begin(), g.start.end() - 1);
  for (int64_t i = 0; i < n; ++i) g.idx[fill[key[i]]++] = (int32_t)i;
}

// ------------------------------------------------------------------ graph --
struct Graph {
  int64_t n = 0;
  Bins B;
  std::vector<int64_t> row_ptr;  // n+1
  std::vector<int32_t> col;      // 0-based neighbour index, rows ascending
  std::vector<uint8_t> bin;      // radial bin 1..nbins
  std::vector<uint8_t> mu;       // mu bin seen from the row's point
};

void graph_from_rows(std::vector<std::vector<int64_t>>& rows, Graph& G) {
  // row entries are packed (j << 16) | (bin << 8) | mu
  G.row_ptr.assign(G.n + 1, 0);
  for (int64_t i = 0; i < G.n; ++i) G.row_ptr[i + 1] = G.row_ptr[i] + (int64_t)rows[i].size();
  int64_t E = G.row_ptr[G.n];
  G.col.resize(E);
  G.bin.resize(E);
  G.mu.resize(E);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < G.n; ++i) {
    int64_t o = G.row_ptr[i];
    for (size_t k = 0; k < rows[i].size(); ++k) {
      int64_t v = rows[i][k];
      G.col[o + k] = (int32_t)(v >> 16);
      G.bin[o + k] = (uint8_t)((v >> 8) & 0xff);
      G.mu[o + k] = (uint8_t)(v & 0xff);
    }
  }
}

void build_graph_grid(const double* xyz, int64_t n, const Bins& B, Graph& G) {
  G.n = n;
  G.B = B;
  Grid g;
  build_grid(xyz, n, B.rmax, g);
  std::vector<std::vector<int64_t>> rows(n);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    const double* pi = xyz + 3 * i;
    int c[3];
    for (int d = 0; d < 3; ++d) {
      int v = (int)std::floor((pi[d] - g.lo[d]) / g.cs[d]);
      c[d] = std::min(std::max(v, 0), g.nc[d] - 1);
    }
    std::vector<int64_t>& row = rows[i];
    for (int dz = -1; dz <= 1; ++dz) {
      int z = c[2] + dz;
      if (z < 0 || z >= g.nc[2]) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        int y = c[1] + dy;
        if (y < 0 || y >= g.nc[1]) continue;
        for (int dx = -1; dx <= 1; ++dx) {
          int x = c[0] + dx;
          if (x < 0 || x >= g.nc[0]) continue;
          int64_t cell = ((int64_t)z * g.nc[1] + y) * g.nc[0] + x;
          for (int64_t k = g.start[cell]; k < g.start[cell + 1]; ++k) {
            int32_t j = g.idx[k];
            if (j == i) continue;
            int b, mf, mr;
            if (edge_eval(pi, xyz + 3 * (int64_t)j, B, &b, &mf, &mr))
              row.push_back(((int64_t)j << 16) | ((int64_t)b << 8) | mf);
          }
        }
      }
    }
    std::sort(row.begin(), row.end());
  }
  graph_from_rows(rows, G);
}

// ------------------------------------------------ kd-tree (timing baseline) --
// A restatement of the kdtree2 algorithm the reference uses for the graph
// build (kdtree2.F90:611-1012 build, 1204-1269/1381-1472/1630-1719 fixed-ball
// search, 1875-1929 heap sort by distance): buckets of at most 10 points,
// cut on the widest coordinate at the mean, a bounding box per node.  Per
// point: a ball search of radius rmax, a ball count of radius rmin, the first
// nn1 results (sorted by distance) skipped, the rest filtered and binned, and
// the row sorted by id with the O(k^2) selection sort of
// sorting_module.F90:36-47.  Used to time the reference algorithm on the host
// cores; its graph equals build_graph_grid's.
struct KdNode {
  int32_t l, u;          // range in perm
  int32_t left, right;   // children or -1
  int32_t cut_dim;
  double cut_val, cut_left, cut_right;
  double box_lo[3], box_hi[3];
};

struct KdTree {
  std::vector<double> data;  // rearranged coordinates, 3 per point
  std::vector<int32_t> perm;
  std::vector<KdNode> nodes;
};

int kd_build_range(KdTree& T, const double* xyz, int32_t l, int32_t u) {
  KdNode node;
  node.l = l;
  node.u = u;
  node.left = node.right = -1;
  node.cut_dim = 0;
  node.cut_val = node.cut_left = node.cut_right = 0.0;
  for (int d = 0; d < 3; ++d) {
    double lo = xyz[3 * (int64_t)T.perm[l] + d], hi = lo;
    for (int32_t k = l; k <= u; ++k) {
      double v = xyz[3 * (int64_t)T.perm[k] + d];
      lo = std::min(lo, v);
      hi = std::max(hi, v);
    }
    node.box_lo[d] = lo;
    node.box_hi[d] = hi;
  }
  int32_t id = (int32_t)T.nodes.size();
  T.nodes.push_back(node);
  if (u - l + 1 <= 10) return id;
  int cd = 0;
  double best = -1.0;
  for (int d = 0; d < 3; ++d) {
    double s = node.box_hi[d] - node.box_lo[d];
    if (s > best) {
      best = s;
      cd = d;
    }
  }
  double mean = 0.0;
  for (int32_t k = l; k <= u; ++k) mean += xyz[3 * (int64_t)T.perm[k] + cd];
  mean /= (double)(u - l + 1);
  int32_t lo = l, hi = u;
  while (lo <= hi) {
    if (xyz[3 * (int64_t)T.perm[lo] + cd] <= mean)
      ++lo;
    else
      std::swap(T.perm[lo], T.perm[hi--]);
  }
  int32_t m = lo - 1;  // last index of the left part
  if (m < l || m >= u) m = (l + u) / 2;  // degenerate spread: split evenly
  int32_t left = kd_build_range(T, xyz, l, m);
  int32_t right = kd_build_range(T, xyz, m + 1, u);
  KdNode& me = T.nodes[id];
  me.left = left;
  me.right = right;
  me.cut_dim = cd;
  me.cut_val = mean;
  me.cut_left = T.nodes[left].box_hi[cd];
  me.cut_right = T.nodes[right].box_lo[cd];
  return id;
}

void kd_build(KdTree& T, const double* xyz, int64_t n) {
  T.perm.resize(n);
  for (int64_t i = 0; i < n; ++i) T.perm[i] = (int32_t)i;
  T.nodes.clear();
  if (n > 0) kd_build_range(T, xyz, 0, (int32_t)n - 1);
  T.data.resize(3 * n);
  for (int64_t k = 0; k < n; ++k)
    for (int d = 0; d < 3; ++d) T.data[3 * k + d] = xyz[3 * (int64_t)T.perm[k] + d];
}

struct KdHit {
  double dis;
  int32_t idx;
};

inline double dis2_bound(double x, double lo, double hi) {
  if (x > hi) return (x - hi) * (x - hi);
  if (x < lo) return (lo - x) * (lo - x);
  return 0.0;
}

void kd_search(const KdTree& T, int32_t nid, const double* q, double r2,
               std::vector<KdHit>* out, int64_t* count) {
  const KdNode& nd = T.nodes[nid];
  if (nd.left < 0) {
    for (int32_t k = nd.l; k <= nd.u; ++k) {
      const double* p = &T.data[3 * (int64_t)k];
      double sd = 0.0;
      double t = p[0] - q[0];
      sd = sd + t * t;
      if (sd > r2) continue;
      t = p[1] - q[1];
      sd = sd + t * t;
      if (sd > r2) continue;
      t = p[2] - q[2];
      sd = sd + t * t;
      if (sd > r2) continue;
      if (out)
        out->push_back({sd, T.perm[k]});
      else
        ++*count;
    }
    return;
  }
  double qv = q[nd.cut_dim];
  int32_t closer, farther;
  double dis;
  if (qv < nd.cut_val) {
    closer = nd.left;
    farther = nd.right;
    dis = (nd.cut_right - qv) * (nd.cut_right - qv);
  } else {
    closer = nd.right;
    farther = nd.left;
    dis = (nd.cut_left - qv) * (nd.cut_left - qv);
  }
  kd_search(T, closer, q, r2, out, count);
  if (dis <= r2) {
    const KdNode& fn = T.nodes[farther];
    for (int d = 0; d < 3; ++d) {
      if (d == nd.cut_dim) continue;
      dis += dis2_bound(q[d], fn.box_lo[d], fn.box_hi[d]);
      if (dis > r2) return;
    }
    kd_search(T, farther, q, r2, out, count);
  }
}

void heap_sort_hits(std::vector<KdHit>& a) {
  auto cmp = [](const KdHit& x, const KdHit& y) { return x.dis < y.dis; };
  std::make_heap(a.begin(), a.end(), cmp);
  std::sort_heap(a.begin(), a.end(), cmp);
}

void selection_sort_row(std::vector<int32_t>& id, std::vector<uint8_t>& b, std::vector<uint8_t>& m) {
  size_t k = id.size();
  for (size_t i = 0; i + 1 < k; ++i) {
    size_t loc = i;
    int32_t mn = id[i];
    for (size_t j = i + 1; j < k; ++j)
      if (id[j] < mn) {
        mn = id[j];
        loc = j;
      }
    std::swap(id[i], id[loc]);
    std::swap(b[i], b[loc]);
    std::swap(m[i], m[loc]);
  }
}

void build_graph_kdtree(const double* xyz, int64_t n, const Bins& B, Graph& G) {
  G.n = n;
  G.B = B;
  KdTree T;
  kd_build(T, xyz, n);
  std::vector<std::vector<int32_t>> rid(n);
  std::vector<std::vector<uint8_t>> rb(n), rm(n);
  if (n > 0) {
#pragma omp parallel
    {
      std::vector<KdHit> hits;
#pragma omp for schedule(dynamic)
      for (int64_t i = 0; i < n; ++i) {
        const double* pi = xyz + 3 * i;
        hits.clear();
        kd_search(T, 0, pi, B.rmax2, &hits, nullptr);
        heap_sort_hits(hits);
        int64_t nn1 = 1;
        if (B.rmin > 0.0) {
          nn1 = 0;
          kd_search(T, 0, pi, B.rmin2, nullptr, &nn1);
        }
        std::vector<int32_t>& id = rid[i];
        std::vector<uint8_t>& bb = rb[i];
        std::vector<uint8_t>& mm = rm[i];
        for (int64_t j = nn1; j < (int64_t)hits.size(); ++j) {
          int b, mf, mr;
          int32_t jj = hits[j].idx;
          if (jj == i) continue;  // a duplicate point may sort ahead of i
          if (!edge_eval(pi, xyz + 3 * (int64_t)jj, B, &b, &mf, &mr)) continue;
          id.push_back(jj);
          bb.push_back((uint8_t)b);
          mm.push_back((uint8_t)mf);
        }
        selection_sort_row(id, bb, mm);
      }
    }
  }
  G.row_ptr.assign(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) G.row_ptr[i + 1] = G.row_ptr[i] + (int64_t)rid[i].size();
  int64_t E = G.row_ptr[n];
  G.col.resize(E);
  G.bin.resize(E);
  G.mu.resize(E);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    int64_t o = G.row_ptr[i];
    std::copy(rid[i].begin(), rid[i].end(), G.col.begin() + o);
    std::copy(rb[i].begin(), rb[i].end(), G.bin.begin() + o);
    std::copy(rm[i].begin(), rm[i].end(), G.mu.begin() + o);
  }
}

// find_dist (gramsci.F90:1579-1609): binary search of id2 in the id-sorted
// row of id1; returns the stored position or -1.
inline int64_t find_edge(const Graph& G, int32_t id1, int32_t id2) {
  const int32_t* b = G.col.data() + G.row_ptr[id1];
  const int32_t* e = G.col.data() + G.row_ptr[id1 + 1];
  if (b == e) return -1;
  const int32_t* p = std::lower_bound(b, e, id2);
  if (p == e || *p != id2) return -1;
  return p - G.col.data();
}

inline int find_dist(const Graph& G, int32_t id1, int32_t id2) {
  int64_t p = find_edge(G, id1, id2);
  return p < 0 ? 0 : G.bin[p];
}

}  // namespace

// ====================================================================== C ABI
extern "C" {

struct orc_graph;

// Builds the neighbour graph.  method 0: uniform grid; 1: kd-tree restatement
// of the reference's search (same edge set).  xyz is points(3,N) in Fortran
// order, i.e. x,y,z interleaved; ids are 0-based positions in that array.
orc_graph* orc_graph_new(const double* xyz, int64_t n, double rmin, double rmax,
                         int32_t nbins, int32_t nmu, int32_t logbins, int32_t method,
                         int32_t nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
  Graph* G = new Graph();
  Bins B = make_bins(rmin, rmax, nbins, nmu, logbins);
  if (method == 1)
    build_graph_kdtree(xyz, n, B, *G);
  else
    build_graph_grid(xyz, n, B, *G);
  return reinterpret_cast<orc_graph*>(G);
}

void orc_graph_free(orc_graph* h) { delete reinterpret_cast<Graph*>(h); }

int64_t orc_graph_nedges(const orc_graph* h) {
  const Graph* G = reinterpret_cast<const Graph*>(h);
  return G->row_ptr.empty() ? 0 : G->row_ptr[G->n];
}

void orc_graph_copy(const orc_graph* h, int64_t* row_ptr, int32_t* col, uint8_t* bin, uint8_t* mu) {
  const Graph* G = reinterpret_cast<const Graph*>(h);
  int64_t E = orc_graph_nedges(h);
  if (row_ptr) std::copy(G->row_ptr.begin(), G->row_ptr.end(), row_ptr);
  if (col) std::copy(G->col.begin(), G->col.begin() + E, col);
  if (bin) std::copy(G->bin.begin(), G->bin.begin() + E, bin);
  if (mu) std::copy(G->mu.begin(), G->mu.begin() + E, mu);
}

// Single-pair evaluation of the reference predicate (used by the tests to
// probe bin edges).  Returns 1 for an edge and writes bin / mu bins.
int32_t orc_edge_eval(const double* pi, const double* pj, double rmin, double rmax,
                      int32_t nbins, int32_t nmu, int32_t logbins, int32_t* out3) {
  Bins B = make_bins(rmin, rmax, nbins, nmu, logbins);
  int b = 0, mf = 0, mr = 0;
  bool e = edge_eval(pi, pj, B, &b, &mf, &mr);
  out3[0] = b;
  out3[1] = mf;
  out3[2] = mr;
  return e ? 1 : 0;
}

void orc_normal_table(int32_t nmu, int32_t variant, int32_t* out /* nmu*nmu, [mu1-1 + nmu*(mu2-1)] */) {
  double mu_scale = (double)(0.5f * (float)nmu);
  for (int b = 1; b <= nmu; ++b)
    for (int a = 1; a <= nmu; ++a) out[(a - 1) + nmu * (b - 1)] = find_normal(a, b, nmu, mu_scale, variant);
}

int32_t orc_bintable3(int32_t a, int32_t b, int32_t c, int32_t n) { return bintable3(a, b, c, n); }
int32_t orc_bintable4(int32_t a, int32_t b, int32_t c, int32_t d, int32_t n) { return bintable4(a, b, c, d, n); }

// Weight normalisation of read_files_2 (gramsci.F90:1390-1391): galaxies
// divided by their sum, randoms negated and divided by theirs.  Sums are
// taken left to right.
void orc_normalise(double* w, int64_t n_data, int64_t n_rand) {
  double sg = 0.0, sr = 0.0;
  for (int64_t i = 0; i < n_data; ++i) sg = sg + w[i];
  for (int64_t i = n_data; i < n_data + n_rand; ++i) sr = sr + w[i];
  for (int64_t i = 0; i < n_data; ++i) w[i] = w[i] / sg;
  for (int64_t i = n_data; i < n_data + n_rand; ++i) w[i] = -1.0 * w[i] / sr;
}

// ------------------------------------------------------------------ 2PCF --
// query_graph_2pcf (gramsci.F90:352-379).  Outputs (Fortran order):
//   N2, N3     (nbins, nmu)          plain FP64 sums as the reference forms them
//   counts     (nbins, nmu, 4)       rooted directed pairs by category
//                                     cat = 2*random(root) + random(neighbour)
//   catsum     (nbins, nmu, 4)       sum of w_i*w_j per category, long double
//                                     accumulated, rounded to FP64
// buffer may be NULL (no buffer points).
void orc_2pcf(const orc_graph* h, const double* w, const int32_t* buffer, int64_t n_data,
              double* N2, double* N3, int64_t* counts, double* catsum) {
  const Graph& G = *reinterpret_cast<const Graph*>(h);
  const int nb = G.B.nbins, nm = G.B.nmu;
  const int nbin = nb * nm;
  int nt = omp_get_max_threads();
  std::vector<double> n2(nt * nbin, 0.0), n3(nt * nbin, 0.0);
  std::vector<int64_t> cnt(nt * nbin * 4, 0);
  std::vector<acc_t> cs(nt * nbin * 4, 0.0L);
#pragma omp parallel
  {
    int t = omp_get_thread_num();
    double* a2 = &n2[t * nbin];
    double* a3 = &n3[t * nbin];
    int64_t* ac = &cnt[t * nbin * 4];
    acc_t* as = &cs[t * nbin * 4];
#pragma omp for schedule(dynamic, 64)
    for (int64_t i = 0; i < G.n; ++i) {
      if (buffer && buffer[i] == 1) continue;
      bool ri = i >= n_data;
      for (int64_t e = G.row_ptr[i]; e < G.row_ptr[i + 1]; ++e) {
        int32_t j = G.col[e];
        int b = G.bin[e];
        int m = G.B.rsd ? G.mu[e] : 1;
        int k = (b - 1) + nb * (m - 1);
        double p = w[i] * w[j];
        bool rj = j >= n_data;
        if (ri && rj) a3[k] = a3[k] + p;
        a2[k] = a2[k] + p;
        int cat = 2 * (int)ri + (int)rj;
        ac[k + nbin * cat] += 1;
        as[k + nbin * cat] += (acc_t)p;
      }
    }
  }
  for (int k = 0; k < nbin; ++k) {
    double s2 = 0.0, s3 = 0.0;
    for (int t = 0; t < nt; ++t) {
      s2 += n2[t * nbin + k];
      s3 += n3[t * nbin + k];
    }
    if (N2) N2[k] = s2;
    if (N3) N3[k] = s3;
  }
  for (int k = 0; k < nbin * 4; ++k) {
    int64_t c = 0;
    acc_t s = 0.0L;
    for (int t = 0; t < nt; ++t) {
      c += cnt[t * nbin * 4 + k];
      s += cs[t * nbin * 4 + k];
    }
    if (counts) counts[k] = c;
    if (catsum) catsum[k] = (double)s;
  }
}

// ------------------------------------------------------------------ 3PCF --
// query_graph_3pcf_all (gramsci.F90:463-510).  cfg = symmetric bin table of
// the three radial bins; mu bin = find_normal(mu(k1), mu(k2)) with k1 < k2
// in the id-sorted row (normal_table indexed [mu1-1 + nmu*(mu2-1)]).
// Outputs (Fortran order, ncfg = C(nbins+2,3)):
//   N2, N3   (ncfg, nmu)     reference sums (N3 accumulates -w_i w_a w_b)
//   counts   (ncfg, nmu, 4)  rooted triangles by number of randoms
//   catsum   (ncfg, nmu, 4)  sum of w_i*w_a*w_b by number of randoms
void orc_3pcf(const orc_graph* h, const double* w, const int32_t* buffer, int64_t n_data,
              const int32_t* normal_table, double* N2, double* N3, int64_t* counts,
              double* catsum) {
  const Graph& G = *reinterpret_cast<const Graph*>(h);
  const int nb = G.B.nbins, nm = G.B.nmu;
  const int ncfg = (int)ncomb_multiset(nb, 3);
  const int nbin = ncfg * nm;
  std::vector<int> tab(nb * nb * nb);
  for (int a = 1; a <= nb; ++a)
    for (int b = 1; b <= nb; ++b)
      for (int c = 1; c <= nb; ++c) tab[(a - 1) + nb * ((b - 1) + nb * (c - 1))] = bintable3(a, b, c, nb);
  int nt = omp_get_max_threads();
  std::vector<double> n2(nt * nbin, 0.0), n3(nt * nbin, 0.0);
  std::vector<int64_t> cnt(nt * nbin * 4, 0);
  std::vector<acc_t> cs(nt * nbin * 4, 0.0L);
#pragma omp parallel
  {
    int t = omp_get_thread_num();
    double* a2 = &n2[t * nbin];
    double* a3 = &n3[t * nbin];
    int64_t* ac = &cnt[t * nbin * 4];
    acc_t* as = &cs[t * nbin * 4];
#pragma omp for schedule(dynamic, 16)
    for (int64_t i = 0; i < G.n; ++i) {
      if (buffer && buffer[i] == 1) continue;
      bool ri = i >= n_data;
      int64_t r0 = G.row_ptr[i], r1 = G.row_ptr[i + 1];
      for (int64_t k1 = r0; k1 < r1; ++k1) {
        int32_t id1 = G.col[k1];
        int b1 = G.bin[k1];
        double wi_w1 = w[i] * w[id1];
        bool r_1 = id1 >= n_data;
        for (int64_t k2 = k1 + 1; k2 < r1; ++k2) {
          int32_t id2 = G.col[k2];
          int b2 = G.bin[k2];
          int b3 = find_dist(G, id1, id2);
          if (b3 == 0) continue;
          int cfg = tab[(b1 - 1) + nb * ((b2 - 1) + nb * (b3 - 1))];
          int m = 1;
          if (G.B.rsd) m = normal_table[(G.mu[k1] - 1) + nm * (G.mu[k2] - 1)];
          int k = (cfg - 1) + ncfg * (m - 1);
          double p = wi_w1 * w[id2];
          bool r_2 = id2 >= n_data;
          if (ri && r_1 && r_2) a3[k] = a3[k] - p;
          a2[k] = a2[k] + p;
          int nr = (int)ri + (int)r_1 + (int)r_2;
          ac[k + nbin * nr] += 1;
          as[k + nbin * nr] += (acc_t)p;
        }
      }
    }
  }
  for (int k = 0; k < nbin; ++k) {
    double s2 = 0.0, s3 = 0.0;
    for (int t = 0; t < nt; ++t) {
      s2 += n2[t * nbin + k];
      s3 += n3[t * nbin + k];
    }
    if (N2) N2[k] = s2;
    if (N3) N3[k] = s3;
  }
  for (int k = 0; k < nbin * 4; ++k) {
    int64_t c = 0;
    acc_t s = 0.0L;
    for (int t = 0; t < nt; ++t) {
      c += cnt[t * nbin * 4 + k];
      s += cs[t * nbin * 4 + k];
    }
    if (counts) counts[k] = c;
    if (catsum) catsum[k] = (double)s;
  }
}

// ------------------------------------------------------------------ 4PCF --
// query_4pcf_all2 (gramsci.F90:662-825).  Root i (non-buffer, row length >
// 3); a<b<c in its id-sorted row with all of ab, bc, ac present; cfg =
// bintable(b_ia, b_ab, b_bc, b_ic) if canonical; diagonals d1 = b_ib,
// d2 = b_ac.  Outputs (Fortran order, ncfg = C(nbins+3,4)):
//   N2, N3        (ncfg, nbins, nbins)
//   discN, discR  (ncfg, nbins, nbins, 6)     the six pair terms of :754-818
//   counts        (ncfg, nbins, nbins, 5)     rooted quads by number of randoms
//   catsum        (ncfg, nbins, nbins, 5)     sum of the 4-products by randoms
//   dcount        (ncfg, nbins, nbins, 6, 4)  disc pair terms: categories
//                                             0..2 = discN by number of
//                                             randoms in the pair, 3 = discR
//   dsum          (ncfg, nbins, nbins, 6, 4)  matching sums
void orc_4pcf(const orc_graph* h, const double* w, const int32_t* buffer, int64_t n_data,
              double* N2, double* N3, double* discN, double* discR, int64_t* counts,
              double* catsum, int64_t* dcount, double* dsum) {
  const Graph& G = *reinterpret_cast<const Graph*>(h);
  const int nb = G.B.nbins;
  const int ncfg = (int)ncomb_multiset(nb, 4);
  const int nbin = ncfg * nb * nb;
  int nt = omp_get_max_threads();
  std::vector<double> n2(nt * nbin, 0.0), n3(nt * nbin, 0.0);
  std::vector<double> dn(nt * nbin * 6, 0.0), dr(nt * nbin * 6, 0.0);
  std::vector<int64_t> cnt(nt * nbin * 5, 0), dcnt(nt * nbin * 24, 0);
  std::vector<acc_t> cs(nt * nbin * 5, 0.0L), dcs(nt * nbin * 24, 0.0L);
  // disc term t (0-based 0..5 for the reference's 1..6): gate vertex and pair
  // vertices, with vertices 0=i, 1=a(id1), 2=b(id2), 3=c(id3).
  static const int gate[6] = {3, 3, 1, 0, 0, 0};
  static const int pu[6] = {0, 0, 0, 1, 3, 3};
  static const int pv[6] = {1, 2, 3, 2, 2, 1};
#pragma omp parallel
  {
    int t = omp_get_thread_num();
    double* a2 = &n2[t * nbin];
    double* a3 = &n3[t * nbin];
    double* adn = &dn[t * nbin * 6];
    double* adr = &dr[t * nbin * 6];
    int64_t* ac = &cnt[t * nbin * 5];
    acc_t* as = &cs[t * nbin * 5];
    int64_t* adc = &dcnt[t * nbin * 24];
    acc_t* ads = &dcs[t * nbin * 24];
#pragma omp for schedule(dynamic, 8)
    for (int64_t i = 0; i < G.n; ++i) {
      if (buffer && buffer[i] == 1) continue;
      int64_t r0 = G.row_ptr[i], r1 = G.row_ptr[i + 1];
      if (r1 - r0 <= 3) continue;
      for (int64_t k1 = r0; k1 < r1; ++k1) {
        int32_t id1 = G.col[k1];
        int ind1 = G.bin[k1];
        for (int64_t k2 = k1 + 1; k2 < r1; ++k2) {
          int32_t id2 = G.col[k2];
          int ind2 = G.bin[k2];
          int ind4 = find_dist(G, id1, id2);
          if (ind4 == 0) continue;
          for (int64_t k3 = k2 + 1; k3 < r1; ++k3) {
            int32_t id3 = G.col[k3];
            int ind3 = G.bin[k3];
            int ind5 = find_dist(G, id2, id3);
            if (ind5 == 0) continue;
            int ind6 = find_dist(G, id1, id3);
            if (ind6 == 0) continue;
            int cfg = bintable4(ind1, ind4, ind5, ind3, nb);
            if (cfg <= 0) continue;
            int k = (cfg - 1) + ncfg * ((ind2 - 1) + nb * (ind6 - 1));
            double p = w[i] * w[id1] * w[id2] * w[id3];
            int64_t v[4] = {i, id1, id2, id3};
            bool r[4] = {i >= n_data, id1 >= n_data, id2 >= n_data, id3 >= n_data};
            a2[k] = a2[k] + p;
            if (r[0] && r[1] && r[2] && r[3]) a3[k] = a3[k] + p;
            int nr = (int)r[0] + (int)r[1] + (int)r[2] + (int)r[3];
            ac[k + nbin * nr] += 1;
            as[k + nbin * nr] += (acc_t)p;
            for (int tt = 0; tt < 6; ++tt) {
              if (!r[gate[tt]]) continue;
              double q = w[v[pu[tt]]] * w[v[pv[tt]]];
              int kt = k + nbin * tt;
              adn[kt] = adn[kt] + q;
              int npr = (int)r[pu[tt]] + (int)r[pv[tt]];
              adc[kt + nbin * 6 * npr] += 1;
              ads[kt + nbin * 6 * npr] += (acc_t)q;
              if (r[pu[tt]] && r[pv[tt]]) {
                adr[kt] = adr[kt] + q;
                adc[kt + nbin * 6 * 3] += 1;
                ads[kt + nbin * 6 * 3] += (acc_t)q;
              }
            }
          }
        }
      }
    }
  }
  for (int k = 0; k < nbin; ++k) {
    double s2 = 0.0, s3 = 0.0;
    for (int t = 0; t < nt; ++t) {
      s2 += n2[t * nbin + k];
      s3 += n3[t * nbin + k];
    }
    if (N2) N2[k] = s2;
    if (N3) N3[k] = s3;
  }
  for (int k = 0; k < nbin * 6; ++k) {
    double s = 0.0, q = 0.0;
    for (int t = 0; t < nt; ++t) {
      s += dn[t * nbin * 6 + k];
      q += dr[t * nbin * 6 + k];
    }
    if (discN) discN[k] = s;
    if (discR) discR[k] = q;
  }
  for (int k = 0; k < nbin * 5; ++k) {
    int64_t c = 0;
    acc_t s = 0.0L;
    for (int t = 0; t < nt; ++t) {
      c += cnt[t * nbin * 5 + k];
      s += cs[t * nbin * 5 + k];
    }
    if (counts) counts[k] = c;
    if (catsum) catsum[k] = (double)s;
  }
  for (int k = 0; k < nbin * 24; ++k) {
    int64_t c = 0;
    acc_t s = 0.0L;
    for (int t = 0; t < nt; ++t) {
      c += dcnt[t * nbin * 24 + k];
      s += dcs[t * nbin * 24 + k];
    }
    if (dcount) dcount[k] = c;
    if (dsum) dsum[k] = (double)s;
  }
}

// ------------------------------------------------------- -equi and -tetra --
// query_graph_equilateral_triangle (gramsci.F90:402-448): triangles whose
// three edges share one radial bin b, from every non-buffer root.  With RSD
// the mu bin is find_normal of the root's two edges and only N2 is summed;
// without RSD N3 accumulates minus the all-random products.
// Outputs (Fortran order): N2, N3 (nbins, nmu); counts, catsum (nbins, nmu, 4)
// by number of randoms.
void orc_equi(const orc_graph* h, const double* w, const int32_t* buffer, int64_t n_data,
              const int32_t* normal_table, double* N2, double* N3, int64_t* counts,
              double* catsum) {
  const Graph& G = *reinterpret_cast<const Graph*>(h);
  const int nb = G.B.nbins, nm = G.B.nmu;
  const int nbin = nb * nm;
  std::vector<double> n2(nbin, 0.0), n3(nbin, 0.0);
  std::vector<int64_t> cnt(nbin * 4, 0);
  std::vector<acc_t> cs(nbin * 4, 0.0L);
  for (int64_t i = 0; i < G.n; ++i) {
    if (buffer && buffer[i] == 1) continue;
    const bool ri = i >= n_data;
    const int64_t r0 = G.row_ptr[i], r1 = G.row_ptr[i + 1];
    for (int64_t k1 = r0; k1 < r1; ++k1) {
      const int ind1 = G.bin[k1];
      const int32_t id1 = G.col[k1];
      for (int64_t k2 = k1 + 1; k2 < r1; ++k2) {
        if (G.bin[k2] != ind1) continue;
        const int32_t id2 = G.col[k2];
        if (find_dist(G, id1, id2) != ind1) continue;
        const double p = w[i] * w[id1] * w[id2];
        const bool allr = ri && id1 >= n_data && id2 >= n_data;
        int m = 1;
        if (G.B.rsd) {
          m = normal_table[(G.mu[k1] - 1) + nm * (G.mu[k2] - 1)];
        } else if (allr) {
          n3[ind1 - 1] = n3[ind1 - 1] - p;
        }
        const int k = (ind1 - 1) + nb * (m - 1);
        n2[k] = n2[k] + p;
        const int nr = (int)ri + (int)(id1 >= n_data) + (int)(id2 >= n_data);
        cnt[k + nbin * nr] += 1;
        cs[k + nbin * nr] += (acc_t)p;
      }
    }
  }
  for (int k = 0; k < nbin; ++k) {
    if (N2) N2[k] = n2[k];
    if (N3) N3[k] = n3[k];
  }
  for (int k = 0; k < nbin * 4; ++k) {
    if (counts) counts[k] = cnt[k];
    if (catsum) catsum[k] = (double)cs[k];
  }
}

// query_graph_tetrahedron (gramsci.F90:548-660): 4-cliques whose six edges
// share one radial bin b, from every non-buffer root (no row-length
// condition), a < b < c in id order.  N2(b) / N3(b) sum the 4-products; the
// six disconnected terms are 3-products gated on one vertex being a random:
//   t  gate  product        discR also needs
//   1  c     w_c w_i w_a    i, a random
//   2  c     w_c w_i w_b    i, b random
//   3  a     w_a w_i w_c    i, c random
//   4  i     w_i w_a w_b    a, b random
//   5  i     w_i w_c w_b    c, b random
//   6  i     w_i w_c w_a    c, a random
// Outputs (Fortran order): N2, N3 (nbins); discN, discR (nbins, 6);
// counts, catsum (nbins, 5) by number of randoms; dcount, dsum (nbins, 6, 5):
// categories 0..3 = discN by number of randoms in the product, 4 = discR.
void orc_tetra(const orc_graph* h, const double* w, const int32_t* buffer, int64_t n_data,
               double* N2, double* N3, double* discN, double* discR, int64_t* counts,
               double* catsum, int64_t* dcount, double* dsum) {
  const Graph& G = *reinterpret_cast<const Graph*>(h);
  const int nb = G.B.nbins;
  std::vector<double> n2(nb, 0.0), n3(nb, 0.0), dn(nb * 6, 0.0), dr(nb * 6, 0.0);
  std::vector<int64_t> cnt(nb * 5, 0), dcnt(nb * 30, 0);
  std::vector<acc_t> cs(nb * 5, 0.0L), dcs(nb * 30, 0.0L);
  static const int gate[6] = {3, 3, 1, 0, 0, 0};
  static const int pa[6] = {3, 3, 1, 0, 0, 0};
  static const int pb[6] = {0, 0, 0, 1, 3, 3};
  static const int pc[6] = {1, 2, 3, 2, 2, 1};
  for (int64_t i = 0; i < G.n; ++i) {
    if (buffer && buffer[i] == 1) continue;
    const int64_t r0 = G.row_ptr[i], r1 = G.row_ptr[i + 1];
    for (int64_t k1 = r0; k1 < r1; ++k1) {
      const int ind1 = G.bin[k1];
      const int32_t id1 = G.col[k1];
      for (int64_t k2 = k1 + 1; k2 < r1; ++k2) {
        const int32_t id2 = G.col[k2];
        if (G.bin[k2] != ind1) continue;
        if (find_dist(G, id1, id2) != ind1) continue;
        for (int64_t k3 = k2 + 1; k3 < r1; ++k3) {
          if (G.bin[k3] != ind1) continue;
          const int32_t id3 = G.col[k3];
          if (find_dist(G, id2, id3) != ind1) continue;
          if (find_dist(G, id1, id3) != ind1) continue;
          const int64_t v[4] = {i, id1, id2, id3};
          const bool r[4] = {i >= n_data, id1 >= n_data, id2 >= n_data, id3 >= n_data};
          const int b = ind1 - 1;
          for (int t = 0; t < 6; ++t) {
            if (!r[gate[t]]) continue;
            const double q = w[v[pa[t]]] * w[v[pb[t]]] * w[v[pc[t]]];
            const int kt = b + nb * t;
            dn[kt] = dn[kt] + q;
            const int nr3 = (int)r[pa[t]] + (int)r[pb[t]] + (int)r[pc[t]];
            dcnt[kt + nb * 6 * nr3] += 1;
            dcs[kt + nb * 6 * nr3] += (acc_t)q;
            if (r[pb[t]] && r[pc[t]]) {
              dr[kt] = dr[kt] + q;
              dcnt[kt + nb * 6 * 4] += 1;
              dcs[kt + nb * 6 * 4] += (acc_t)q;
            }
          }
          const double p = w[i] * w[id1] * w[id2] * w[id3];
          n2[b] = n2[b] + p;
          if (r[0] && r[1] && r[2] && r[3]) n3[b] = n3[b] + p;
          const int nr = (int)r[0] + (int)r[1] + (int)r[2] + (int)r[3];
          cnt[b + nb * nr] += 1;
          cs[b + nb * nr] += (acc_t)p;
        }
      }
    }
  }
  for (int k = 0; k < nb; ++k) {
    if (N2) N2[k] = n2[k];
    if (N3) N3[k] = n3[k];
  }
  for (int k = 0; k < nb * 6; ++k) {
    if (discN) discN[k] = dn[k];
    if (discR) discR[k] = dr[k];
  }
  for (int k = 0; k < nb * 5; ++k) {
    if (counts) counts[k] = cnt[k];
    if (catsum) catsum[k] = (double)cs[k];
  }
  for (int k = 0; k < nb * 30; ++k) {
    if (dcount) dcount[k] = dcnt[k];
    if (dsum) dsum[k] = (double)dcs[k];
  }
}

// --------------------------------------------------------------- adjoints --
// Gradient of L = sum(cot2 * N2) + sum(cot3 * N3) with respect to the signed
// normalised weights, for the 2PCF of orc_2pcf.  dN2_b/dw_k = sum of w_j over
// edges (k,j) in bin b counted from each non-buffer endpoint.  Computed per
// point from the symmetric graph, long double accumulation.
void orc_adjoint_2pcf(const orc_graph* h, const double* w, const int32_t* buffer, int64_t n_data,
                      const double* cot2, const double* cot3, double* grad) {
  const Graph& G = *reinterpret_cast<const Graph*>(h);
  const int nb = G.B.nbins;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t k = 0; k < G.n; ++k) {
    acc_t g = 0.0L;
    bool rk = k >= n_data;
    bool bk = buffer && buffer[k] == 1;
    for (int64_t e = G.row_ptr[k]; e < G.row_ptr[k + 1]; ++e) {
      int32_t j = G.col[e];
      int b = G.bin[e];
      bool rj = j >= n_data;
      bool bj = buffer && buffer[j] == 1;
      acc_t c = 0.0L;
      if (!bk) {
        int m = G.B.rsd ? G.mu[e] : 1;
        int idx = (b - 1) + nb * (m - 1);
        c += cot2[idx];
        if (rk && rj && cot3) c += cot3[idx];
      }
      if (!bj) {
        int m = 1;
        if (G.B.rsd) {
          int64_t r = find_edge(G, j, (int32_t)k);
          m = G.mu[r];
        }
        int idx = (b - 1) + nb * (m - 1);
        c += cot2[idx];
        if (rk && rj && cot3) c += cot3[idx];
      }
      g += c * (acc_t)w[j];
    }
    grad[k] = (double)g;
  }
}

// Gradient of L = sum(cot2 * N2) + sum(cot3 * N3) for the 3PCF of orc_3pcf.
// Each triangle {k,x,y} adds, for every non-buffer root r among its vertices,
// coef(r) * w_x * w_y to grad[k], where coef(r) = cot2[cfg, m_r] minus
// cot3[cfg, m_r] when all three are randoms and m_r is find_normal of r's two
// edges taken in id order.
void orc_adjoint_3pcf(const orc_graph* h, const double* w, const int32_t* buffer, int64_t n_data,
                      const int32_t* normal_table, const double* cot2, const double* cot3,
                      double* grad) {
  const Graph& G = *reinterpret_cast<const Graph*>(h);
  const int nb = G.B.nbins, nm = G.B.nmu;
  const int ncfg = (int)ncomb_multiset(nb, 3);
  auto mu_of = [&](int32_t from, int32_t to) -> int {
    if (!G.B.rsd) return 1;
    return G.mu[find_edge(G, from, to)];
  };
  auto coef = [&](int32_t r, int32_t u, int32_t v, int cfg, bool allr) -> acc_t {
    if (buffer && buffer[r] == 1) return 0.0L;
    int m = 1;
    if (G.B.rsd) {
      int32_t f = std::min(u, v), s = std::max(u, v);
      m = normal_table[(mu_of(r, f) - 1) + nm * (mu_of(r, s) - 1)];
    }
    int idx = (cfg - 1) + ncfg * (m - 1);
    acc_t c = cot2[idx];
    if (allr && cot3) c -= cot3[idx];
    return c;
  };
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t k = 0; k < G.n; ++k) {
    acc_t g = 0.0L;
    int64_t r0 = G.row_ptr[k], r1 = G.row_ptr[k + 1];
    for (int64_t e1 = r0; e1 < r1; ++e1) {
      int32_t x = G.col[e1];
      for (int64_t e2 = e1 + 1; e2 < r1; ++e2) {
        int32_t y = G.col[e2];
        int bxy = find_dist(G, x, y);
        if (bxy == 0) continue;
        int cfg = bintable3(G.bin[e1], G.bin[e2], bxy, nb);
        bool allr = k >= n_data && x >= n_data && y >= n_data;
        acc_t c = coef((int32_t)k, x, y, cfg, allr) + coef(x, (int32_t)k, y, cfg, allr) +
                  coef(y, (int32_t)k, x, cfg, allr);
        g += c * (acc_t)w[x] * (acc_t)w[y];
      }
    }
    grad[k] = (double)g;
  }
}

// Gradient of L = sum(cot2 N2) + sum(cot3 N3) + sum(cotN discN) +
// sum(cotR discR) for the 4PCF of orc_4pcf (the same enumeration: root i,
// a < b < c in its row).  Each rooted quad adds to every one of its four
// vertices (cot2[k] + cot3[k] if all four are randoms) times the product of
// the other three weights; each gated pair term t adds (cotN[kt] + cotR[kt]
// if both pair vertices are randoms) times the partner's weight to each of
// its two vertices.  Per-thread long double gradients, summed at the end.
void orc_adjoint_4pcf(const orc_graph* h, const double* w, const int32_t* buffer, int64_t n_data,
                      const double* cot2, const double* cot3, const double* cotN,
                      const double* cotR, double* grad) {
  const Graph& G = *reinterpret_cast<const Graph*>(h);
  const int nb = G.B.nbins;
  const int ncfg = (int)ncomb_multiset(nb, 4);
  const int64_t nbin = (int64_t)ncfg * nb * nb;
  const int nt = omp_get_max_threads();
  std::vector<acc_t> part((size_t)nt * G.n, 0.0L);
  static const int gate[6] = {3, 3, 1, 0, 0, 0};
  static const int pu[6] = {0, 0, 0, 1, 3, 3};
  static const int pv[6] = {1, 2, 3, 2, 2, 1};
#pragma omp parallel
  {
    acc_t* g = &part[(size_t)omp_get_thread_num() * G.n];
#pragma omp for schedule(dynamic, 8)
    for (int64_t i = 0; i < G.n; ++i) {
      if (buffer && buffer[i] == 1) continue;
      int64_t r0 = G.row_ptr[i], r1 = G.row_ptr[i + 1];
      if (r1 - r0 <= 3) continue;
      for (int64_t k1 = r0; k1 < r1; ++k1) {
        int32_t id1 = G.col[k1];
        for (int64_t k2 = k1 + 1; k2 < r1; ++k2) {
          int32_t id2 = G.col[k2];
          int ind4 = find_dist(G, id1, id2);
          if (ind4 == 0) continue;
          for (int64_t k3 = k2 + 1; k3 < r1; ++k3) {
            int32_t id3 = G.col[k3];
            int ind5 = find_dist(G, id2, id3);
            if (ind5 == 0) continue;
            int ind6 = find_dist(G, id1, id3);
            if (ind6 == 0) continue;
            int cfg = bintable4(G.bin[k1], ind4, ind5, G.bin[k3], nb);
            if (cfg <= 0) continue;
            int64_t k = (cfg - 1) + ncfg * ((G.bin[k2] - 1) + nb * (int64_t)(ind6 - 1));
            int64_t v[4] = {i, id1, id2, id3};
            bool r[4] = {i >= n_data, id1 >= n_data, id2 >= n_data, id3 >= n_data};
            acc_t c4 = cot2[k];
            if (cot3 && r[0] && r[1] && r[2] && r[3]) c4 += cot3[k];
            for (int a = 0; a < 4; ++a) {
              acc_t p = c4;
              for (int b = 0; b < 4; ++b)
                if (b != a) p *= (acc_t)w[v[b]];
              g[v[a]] += p;
            }
            for (int tt = 0; tt < 6; ++tt) {
              if (!r[gate[tt]]) continue;
              int64_t kt = k + nbin * tt;
              acc_t cd = cotN ? (acc_t)cotN[kt] : 0.0L;
              if (cotR && r[pu[tt]] && r[pv[tt]]) cd += cotR[kt];
              g[v[pu[tt]]] += cd * (acc_t)w[v[pv[tt]]];
              g[v[pv[tt]]] += cd * (acc_t)w[v[pu[tt]]];
            }
          }
        }
      }
    }
  }
#pragma omp parallel for
  for (int64_t k = 0; k < G.n; ++k) {
    acc_t s = 0.0L;
    for (int t = 0; t < nt; ++t) s += part[(size_t)t * G.n + k];
    grad[k] = (double)s;
  }
}

int32_t orc_max_threads() { return omp_get_max_threads(); }

}  // extern "C"
