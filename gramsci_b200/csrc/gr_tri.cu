// 3PCF triangle counting: replaces query_graph_3pcf_all
// (src/gramsci.F90:463-510), whose per-root double loop looks up the third
// edge with a binary search into another vertex's row (find_dist,
// :1579-1609).
//
// Every triangle is enumerated exactly once, from its smallest internal
// label p.  A warp takes a root p and stages its upper row R+(p) in shared
// memory together with the flags, catalogue ids and weights of those
// neighbours, their row starts and lengths, and a per-root open-addressing
// hash table (label offset -> row position, one 32-bit word per entry,
// Fibonacci hashing).  The work items (a, c) for c in R+(a) are flattened
// over batches of 32 rows and spread over the lanes; a lane finds the row
// of its item by a binary search over the lanes' prefix sums (register
// shuffles), loads one 8-byte CSR record and probes the hash table for c.
// Hits (triangles p < a < c) are pushed to a per-warp queue that is drained
// 32 at a time, so the binning work runs with every lane busy.
//
// Geometric mode (TriParams::geo): the third edge (a, c) of a triangle joins
// two members of R+(p), and it is an edge exactly when the pair passes the
// graph's own membership test (FP32 squared separation, FP64 inside the
// guard band).  The warp stages the positions of R+(p) instead of the row
// starts and the hash table, spreads the k(k-1)/2 pairs of R+(p) over the
// lanes (closed-form inversion of the triangular pair index) and queues the
// pairs that pass; the drain bins (a, c) with the graph's binning.  It tests
// k(k-1)/2 pairs per root instead of the sum of |R+(a)| and reads no other
// rows, but bins every third edge again: it wins at high degree and without
// mu bins, the hash mode at low degree with mu bins.  Both give identical
// results.
//
// A triangle contributes to the rooted histogram of each non-buffer vertex r
// with the bins of its three edges (symmetric bin table), the find_normal mu
// bin of r's two edges taken in catalogue-id order (k1 < k2 in the
// reference's id-sorted row) and the weight product, accumulated as 128-bit
// fixed point with a scale per number of randoms.
#include "gr_kernels.cuh"

#include <algorithm>

namespace gr {

namespace {

constexpr int kTriMaxWarps = 32;  // block size is chosen at launch to fit shared memory
constexpr size_t kSmemLimit = 227 * 1024;
constexpr int kQueue = 96;   // hit queue entries per warp (< 32 left + 64 pushed)
constexpr int kChunk = 1;    // roots taken per work-counter increment (more causes tail imbalance)
constexpr int kCfgTableBins = 16;  // nbins up to which the configuration table is used

__host__ __device__ inline size_t align8(size_t x) { return (x + 7) & ~(size_t)7; }
struct TriLayout {
  size_t off_cnt, off_lim, off_cot, off_norm, off_rank, off_cfg, off_fsc, off_warp, warp_bytes, total;
  // per-warp sub-offsets
  size_t o_pos, o_rs, o_w, o_g, o_col, o_mo, o_len, o_hkey, o_q;
};

// Largest per-root hash table: a power of two >= 4 * cap (load <= 1/4).
__host__ __device__ inline int hash_lg_max(int cap) {
  int lg = 6;
  while ((1 << lg) < 4 * cap) ++lg;
  return lg;
}

// adj: the adjoint variant (cotangent tables, per-neighbour gradient
// accumulators) instead of histograms.  geo: neighbour positions instead of
// row starts, lengths and the hash table.
__host__ __device__ inline TriLayout tri_layout(int nh, int nmu, int nbins, int cap, bool shist,
                                                bool weighted, bool counts, int nwarps,
                                                bool adj = false, bool geo = false) {
  TriLayout L;
  size_t o = 0;
  L.off_cnt = o;
  if (shist && counts) o += (size_t)nh * 8;
  L.off_lim = o;
  if (shist && weighted) o += (size_t)nh * 16;
  L.off_cot = o;
  if (adj) o += (size_t)nh / 4 * 2 * 8;  // cot2, cot3: ncfg * nmu doubles each
  L.off_fsc = o;
  o += 4 * 8;
  L.off_norm = o;
  o = align8(o + (size_t)nmu * nmu);
  L.off_rank = o;
  o = align8(o + sizeof(int) * 3 * (size_t)(nbins + 2));
  L.off_cfg = o;  // configuration of every (b1, b2, b3), small nbins only
  if (nbins <= kCfgTableBins) o = align8(o + sizeof(uint16_t) * (size_t)nbins * nbins * nbins);
  o = (o + 15) & ~(size_t)15;  // float4 positions in the warp areas
  L.off_warp = o;
  const int hs = 1 << hash_lg_max(cap);
  size_t w = 0;
  L.o_pos = w;  if (geo) w += (size_t)cap * 16;  // float4 position per neighbour
  L.o_rs = w;   if (!geo) w += (size_t)cap * 8;
  L.o_w = w;    if (weighted || adj) w += (size_t)cap * 8;
  L.o_g = w;    if (adj) w += (size_t)cap * 8;  // signed 64-bit gradient per neighbour
  L.o_col = w;  w += (size_t)cap * 4;
  L.o_mo = w;   w += (size_t)cap * 8;  // (catalogue id << 32) | flags << 24 | edge meta
  L.o_len = w;  if (!geo) w += (size_t)cap * 4;
  L.o_hkey = w; if (!geo) w += (size_t)hs * 4;
  L.o_q = w;    w += (size_t)kQueue * 8;
  L.warp_bytes = (w + 15) & ~(size_t)15;
  L.total = o + L.warp_bytes * nwarps;
  return L;
}

struct TriCtx {
  const uint8_t* norm;
  const int* F;  // 3 x (nbins+2)
  const uint16_t* cfgtab;  // symmetric configuration table or NULL
  const double* fsc;       // fixed-point scale by number of randoms
  int nbins, nmu, ncfg, rsd, nh, equi;
  unsigned long long* cnt;
  unsigned long long* lim;  // fixed-point sums: lim[k] (lo), lim[nh + k] (hi)
  // adjoint
  const double* c2;  // cot2 (ncfg, nmu)
  const double* c3;  // cot3 (ncfg, nmu)
  double gscale;
};

__device__ __forceinline__ int rank3_s(const int* F, int nb2, int a, int b, int c) {
  return 1 + (F[a] - F[1]) + (F[nb2 + b] - F[nb2 + a]) + (F[2 * nb2 + c] - F[2 * nb2 + b]);
}

// symmetric bin table of the three radial bins (gramsci.F90:1459-1474)
__device__ __forceinline__ int tri_cfg(const TriCtx& X, int b1, int b2, int b3) {
  if (X.cfgtab) return X.cfgtab[(b1 - 1) + X.nbins * ((b2 - 1) + X.nbins * (b3 - 1))];
  sort3i(b1, b2, b3);
  return rank3_s(X.F, X.nbins + 2, b1, b2, b3);
}

__device__ __forceinline__ int normal_bin(const TriCtx& X, int mu1, int mu2, bool first_is_1) {
  if (!X.rsd) return 1;
  return first_is_1 ? X.norm[(mu1 - 1) + X.nmu * (mu2 - 1)] : X.norm[(mu2 - 1) + X.nmu * (mu1 - 1)];
}

template <bool WEIGHTED, bool COUNTS>
__device__ __forceinline__ void tri_add(const TriCtx& X, int k, int n, long long v) {
  if (COUNTS) atomicAdd(&X.cnt[k], (unsigned long long)n);
  if (WEIGHTED) fix_add_int(&X.lim[k], &X.lim[X.nh + k], v * n);
}

// One triangle (p, a, c) with p < a < c in labels.  It adds to the rooted
// histogram of each non-buffer vertex r: the bins of its three edges
// (symmetric bin table), the find_normal mu bin of r's two edges taken in
// catalogue-id order (k1 < k2 in the reference's id-sorted row) and the
// weight product w_p w_a w_c (one product for all roots: the orders the
// reference multiplies in differ from it by at most an ulp).  Roots that land
// in the same bin share one update.  Returns the number of rooted
// contributions.
template <bool WEIGHTED, bool COUNTS>
__device__ __forceinline__ int tri_bin(const TriCtx& X, uint8_t fp, int op, double wp, uint8_t fa,
                                       int oa, double wa, uint8_t fc, int oc, double wc,
                                       uint32_t mpa, uint32_t mpc, uint32_t mac) {
  int cfg;
  if (X.equi) {  // query_graph_equilateral_triangle: three equal bins
    const int b1 = meta_bin(mpa);
    if (meta_bin(mpc) != b1 || meta_bin(mac) != b1) return 0;
    cfg = b1;
  } else {
    cfg = tri_cfg(X, meta_bin(mpa), meta_bin(mpc), meta_bin(mac));
  }
  const int nr = (fp & FLAG_RANDOM) + (fa & FLAG_RANDOM) + (fc & FLAG_RANDOM);
  long long v = 0;
  if (WEIGHTED) v = __double2ll_rn(((wp * wa) * wc) * X.fsc[nr]);
  int m0 = 1, m1 = 1, m2 = 1;
  if (X.rsd) {
    m0 = normal_bin(X, meta_muf(mpa), meta_muf(mpc), oa < oc);  // root p: a, c
    m1 = normal_bin(X, meta_mur(mpa), meta_muf(mac), op < oc);  // root a: p, c
    m2 = normal_bin(X, meta_mur(mpc), meta_mur(mac), op < oa);  // root c: p, a
  }
  int c0 = (fp & FLAG_BUFFER) ? 0 : 1;
  int c1 = (fa & FLAG_BUFFER) ? 0 : 1;
  int c2 = (fc & FLAG_BUFFER) ? 0 : 1;
  const int total = c0 + c1 + c2;
  if (c1 && m1 == m0 && c0) { c0 += c1; c1 = 0; }
  if (c2 && m2 == m0 && c0) { c0 += c2; c2 = 0; }
  else if (c2 && m2 == m1 && c1) { c1 += c2; c2 = 0; }
  const int base = (cfg - 1) + X.ncfg * X.nmu * nr;
  if (c0) tri_add<WEIGHTED, COUNTS>(X, base + X.ncfg * (m0 - 1), c0, v);
  if (c1) tri_add<WEIGHTED, COUNTS>(X, base + X.ncfg * (m1 - 1), c1, v);
  if (c2) tri_add<WEIGHTED, COUNTS>(X, base + X.ncfg * (m2 - 1), c2, v);
  return total;
}

// Adjoint of one triangle (p, a, c): every non-buffer root r contributes
// (cot2 - [all random] cot3)[cfg, m_r] (N3 accumulates minus the product);
// with C the sum, dL/dw_p += C w_a w_c, dL/dw_a += C w_p w_c, dL/dw_c +=
// C w_p w_a.  p's term goes to the lane's register accumulator, a's and c's
// to the given fixed-point accumulators: S64, signed 64-bit partial sums of
// one root (alo / clo; the scale leaves room for 1024 terms), else 128-bit
// (lo, hi) pairs.
template <bool S64>
__device__ __forceinline__ int tri_grad(const TriCtx& X, uint8_t fp, int op, double wp,
                                        uint8_t fa, int oa, double wa, uint8_t fc, int oc,
                                        double wc, uint32_t mpa, uint32_t mpc, uint32_t mac,
                                        Fix128& racc, unsigned long long* alo,
                                        unsigned long long* ahi, unsigned long long* clo,
                                        unsigned long long* chi) {
  const int cfg = tri_cfg(X, meta_bin(mpa), meta_bin(mpc), meta_bin(mac));
  const bool allr = (fp & fa & fc & FLAG_RANDOM) != 0;
  double C = 0.0;
  int n = 0;
  if (!(fp & FLAG_BUFFER)) {
    const int k = (cfg - 1) + X.ncfg * (normal_bin(X, meta_muf(mpa), meta_muf(mpc), oa < oc) - 1);
    C += allr ? X.c2[k] - X.c3[k] : X.c2[k];
    n++;
  }
  if (!(fa & FLAG_BUFFER)) {
    const int k = (cfg - 1) + X.ncfg * (normal_bin(X, meta_mur(mpa), meta_muf(mac), op < oc) - 1);
    C += allr ? X.c2[k] - X.c3[k] : X.c2[k];
    n++;
  }
  if (!(fc & FLAG_BUFFER)) {
    const int k = (cfg - 1) + X.ncfg * (normal_bin(X, meta_mur(mpc), meta_mur(mac), op < oa) - 1);
    C += allr ? X.c2[k] - X.c3[k] : X.c2[k];
    n++;
  }
  if (C != 0.0) {
    fix_acc(racc, C * (wa * wc), X.gscale);
    if (S64) {
      atomicAdd(alo, (unsigned long long)__double2ll_rn(C * (wp * wc) * X.gscale));
      atomicAdd(clo, (unsigned long long)__double2ll_rn(C * (wp * wa) * X.gscale));
    } else {
      fix_add(alo, ahi, C * (wp * wc), X.gscale);
      fix_add(clo, chi, C * (wp * wa), X.gscale);
    }
  }
  return n;
}

// first index in sorted a[0..n) with a[i] >= v
__device__ __forceinline__ int lower_bound_g(const unsigned long long* a, int n, int v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (rec_col(a[mid]) < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Fibonacci hashing of a label offset into a table of 2^lg slots: runs of
// consecutive offsets (the common case: a cell's points are consecutive
// labels) spread evenly over the table.
__device__ __forceinline__ uint32_t fib_slot(uint32_t off, int lg) {
  return (off * 2654435769u) >> (32 - lg);
}

// Hash entries: (offset << 8) | position, offset = label - p in [1, 2^24);
// 0 marks an empty slot.
constexpr int kMaxOffset = 1 << 24;

// ADJ: accumulate the weight gradient (g_lo / g_hi, label order) of
// L = sum cot2 N2 + cot3 N3 instead of the histograms.
template <bool WEIGHTED, bool COUNTS, bool SHIST, bool ADJ, bool GEO>
__global__ void __launch_bounds__(kTriMaxWarps * 32) tri3_kernel(DevCatalog C, CSRView G, TriParams T,
                                                           unsigned long long* __restrict__ g_cnt,
                                                           unsigned long long* __restrict__ g_lim,
                                                           unsigned long long* __restrict__ stats,
                                                           int* __restrict__ work,
                                                           const double* __restrict__ cot2,
                                                           const double* __restrict__ cot3,
                                                           double gscale,
                                                           unsigned long long* __restrict__ g_lo,
                                                           unsigned long long* __restrict__ g_hi) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int nh = T.ncfg * T.nmu * 4;
  const TriLayout L =
      tri_layout(nh, T.nmu, T.nbins, T.cap, SHIST, WEIGHTED, COUNTS, blockDim.x >> 5, ADJ, GEO);
  TriCtx X;
  X.nbins = T.nbins;
  X.nmu = T.nmu;
  X.ncfg = T.ncfg;
  X.rsd = T.rsd;
  X.equi = T.equi;
  X.nh = nh;
  X.cnt = SHIST ? reinterpret_cast<unsigned long long*>(smem + L.off_cnt) : g_cnt;
  X.lim = SHIST ? reinterpret_cast<unsigned long long*>(smem + L.off_lim) : g_lim;
  uint8_t* s_norm = smem + L.off_norm;
  int* s_F = reinterpret_cast<int*>(smem + L.off_rank);
  X.norm = s_norm;
  X.F = s_F;
  double* s_fsc = reinterpret_cast<double*>(smem + L.off_fsc);
  X.fsc = s_fsc;
  if (threadIdx.x < 4) s_fsc[threadIdx.x] = T.fscale[threadIdx.x];
  X.gscale = gscale;
  if (ADJ) {
    double* s_cot = reinterpret_cast<double*>(smem + L.off_cot);
    const int nc = T.ncfg * T.nmu;
    for (int k = threadIdx.x; k < nc; k += blockDim.x) {
      s_cot[k] = cot2[k];
      s_cot[nc + k] = cot3 ? cot3[k] : 0.0;
    }
    X.c2 = s_cot;
    X.c3 = s_cot + nc;
  }
  if (SHIST) {
    for (int k = threadIdx.x; k < nh; k += blockDim.x) {
      if (COUNTS) X.cnt[k] = 0ull;
      if (WEIGHTED) {
        X.lim[k] = 0ull;
        X.lim[nh + k] = 0ull;
      }
    }
  }
  for (int k = threadIdx.x; k < T.nmu * T.nmu; k += blockDim.x) s_norm[k] = T.rsd ? T.normal[k] : 1;
  const int nb2 = T.nbins + 2;
  for (int k = threadIdx.x; k < 3 * nb2; k += blockDim.x) s_F[k] = T.rank.F[k / nb2][k % nb2];
  __syncthreads();
  X.cfgtab = nullptr;
  if (T.nbins <= kCfgTableBins) {
    uint16_t* tab = reinterpret_cast<uint16_t*>(smem + L.off_cfg);
    const int nb = T.nbins;
    for (int k = threadIdx.x; k < nb * nb * nb; k += blockDim.x) {
      int a = k % nb + 1, b = (k / nb) % nb + 1, c = k / (nb * nb) + 1;
      sort3i(a, b, c);
      tab[k] = (uint16_t)rank3_s(s_F, nb2, a, b, c);
    }
    __syncthreads();
    X.cfgtab = tab;
  }

  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  unsigned char* wb = smem + L.off_warp + L.warp_bytes * (threadIdx.x >> 5);
  float4* s_pos = reinterpret_cast<float4*>(wb + L.o_pos);
  long long* s_rs = reinterpret_cast<long long*>(wb + L.o_rs);
  double* s_w = reinterpret_cast<double*>(wb + L.o_w);
  int* s_col = reinterpret_cast<int*>(wb + L.o_col);
  unsigned long long* s_mo = reinterpret_cast<unsigned long long*>(wb + L.o_mo);
  int* s_len = reinterpret_cast<int*>(wb + L.o_len);
  uint32_t* s_hkey = reinterpret_cast<uint32_t*>(wb + L.o_hkey);
  // queue entry: (meta of edge (a, c) << 32) | row of a | (row of c << 16)
  unsigned long long* s_q = reinterpret_cast<unsigned long long*>(wb + L.o_q);
  unsigned long long* s_g = reinterpret_cast<unsigned long long*>(wb + L.o_g);
  const int lg_max = hash_lg_max(T.cap);

  unsigned long long tris = 0, rooted = 0, probes = 0;

  // one queued triangle (p, a = row qx, c = row qy) with edge meta (a, c)
  auto drain_one = [&](int e, uint8_t fp, int op, double wp, Fix128& racc) -> int {
    const unsigned long long qe = s_q[e];
    const int qx = (int)(qe & 0xffffu), qy = (int)((qe >> 16) & 0xffffu);
    uint32_t mac = (uint32_t)(qe >> 32);
    if (GEO) {
      // bins of the edge (a, c) exactly as the graph build computes them
      int b = 1, mf = 1, mr = 1;
      const int r = T.P.f32 ? classify_f32<true>(s_pos[qx], s_pos[qy], T.P, b, mf, mr) : 2;
      if (r == 2) edge_f64(C.posd[s_col[qx]], C.posd[s_col[qy]], T.P, b, mf, mr);
      mac = pack_meta(b, mf, mr);
    }
    const unsigned long long moa = s_mo[qx], moc = s_mo[qy];
    const uint32_t ma = (uint32_t)moa, mc = (uint32_t)moc;
    const int oa = (int)(moa >> 32), oc = (int)(moc >> 32);
    const uint8_t fa = (uint8_t)(ma >> 24), fc = (uint8_t)(mc >> 24);
    if (ADJ)
      return tri_grad<true>(X, fp, op, wp, fa, oa, s_w[qx], fc, oc, s_w[qy], ma, mc, mac, racc,
                            &s_g[qx], nullptr, &s_g[qy], nullptr);
    return tri_bin<WEIGHTED, COUNTS>(X, fp, op, wp, fa, oa, WEIGHTED ? s_w[qx] : 0.0, fc, oc,
                                     WEIGHTED ? s_w[qy] : 0.0, ma, mc, mac);
  };

  for (;;) {
    int base_root = 0;
    if (lane == 0) base_root = atomicAdd(work, kChunk);
    base_root = __shfl_sync(0xffffffffu, base_root, 0);
    if (base_root >= C.n) break;
    const int end_root = min(base_root + kChunk, C.n);
    for (int p = base_root; p < end_root; ++p) {
      const int64_t b0 = G.start[p];
      const int k = G.len[p];
      if (k < 2 || k <= T.kmin || k > T.kskip) continue;  // rows of the other launch
      const uint8_t fp = C.flags[p];
      const int op = C.orig[p];
      const double wp = (WEIGHTED || ADJ) ? C.w[p] : 0.0;
      Fix128 racc = {0ull, 0ull};
      // rows are sorted: the last entry has the largest label offset
      if (k <= T.cap && (GEO || rec_col(G.rec[b0 + k - 1]) - p < kMaxOffset)) {
        // per-root table: >= 8 slots per entry, at most the capacity's table
        int lg = 6;
        while (lg < lg_max && (1 << lg) < 8 * k) ++lg;
        const int hs = 1 << lg;
        __syncwarp();
        if (!GEO)
          for (int h = lane; h < hs; h += 32) s_hkey[h] = 0u;
        __syncwarp();
        // stage R+(p) and the data of its vertices; insert into the hash table
        for (int xb = 0; xb < k; xb += 32) {
          const int x = xb + lane;
          if (x < k) {
            const unsigned long long r = G.rec[b0 + x];
            const int a = rec_col(r);
            s_col[x] = a;
            if (GEO) {
              s_pos[x] = C.pos4[a];
            } else {
              const long long rs = G.start[a];
              const int len = G.len[a];
              s_rs[x] = rs;
              s_len[x] = len;
              probes += (unsigned long long)len;
            }
            // the vertex flags ride in the top byte of the edge meta word
            s_mo[x] = ((unsigned long long)(uint32_t)C.orig[a] << 32) |
                      (rec_meta(r) | ((uint32_t)C.flags[a] << 24));
            if (WEIGHTED || ADJ) s_w[x] = C.w[a];
            if (ADJ) s_g[x] = 0ull;
            if (!GEO) {
              const uint32_t off = (uint32_t)(a - p);
              const uint32_t key = (off << 8) | (uint32_t)x;
              uint32_t h = fib_slot(off, lg);
              for (int t = 0; t < hs; ++t) {
                if (atomicCAS(&s_hkey[h], 0u, key) == 0u) break;
                h = (h + 1) & (uint32_t)(hs - 1);
              }
            }
          }
        }
        __syncwarp();
        int qn = 0;
        if (GEO) {
          // every pair (x, y), x < y, of R+(p) over the lanes: (a, c) is an
          // edge when the pair passes the graph's own membership test
          const int npair = k * (k - 1) / 2;
          const int k2m1 = 2 * k - 1;
          if (lane == 0) probes += (unsigned long long)npair;
          for (int t0 = 0; t0 < npair; t0 += 32) {
            const int t = t0 + lane;
            bool hit = false;
            int x = 0, y = 0;
            if (t < npair) {
              // x: the largest row with x (2k - 1 - x) / 2 <= t pairs before it
              // (exact up to kPairRowExact members, else one adjustment each way)
              x = pair_row_biased(k2m1, t);
              if (k > kPairRowExact) {
                x = max(0, min(x, k - 2));
                if ((x + 1) * (k2m1 - x - 1) / 2 <= t) ++x;
                if (x * (k2m1 - x) / 2 > t) --x;
              }
              y = t - (int)((unsigned)(x * (k2m1 - x)) >> 1) + x + 1;
              int r = T.P.f32 ? member_f32(s_pos[x], s_pos[y], T.P) : 2;
              if (r == 2) {
                int b, mf, mr;
                r = edge_f64(C.posd[s_col[x]], C.posd[s_col[y]], T.P, b, mf, mr) ? 1 : 0;
              }
              hit = r == 1;
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (hit) s_q[qn + __popc(m & lt)] = (unsigned long long)(x | (y << 16));
            qn += __popc(m);
            if (qn >= 32) {
              __syncwarp();
              const int nroot = drain_one(qn - 32 + lane, fp, op, wp, racc);
              tris += nroot > 0;
              rooted += nroot;
              qn -= 32;
              __syncwarp();
            }
          }
        } else
        // rows in batches of 32; the batch's non-empty rows are compacted
        // onto the lanes, their work items (a, c in R+(a)) flattened and
        // spread over the lanes 32 at a time.  A lane finds the row of its
        // item from the mask of rows ending inside the window (one warp OR
        // reduction) and the count of rows that ended before it.
        for (int xb = 0; xb < k; xb += 32) {
          const int x = xb + lane;
          int len = 0;
          long long rs = 0;
          if (x < k) {
            len = s_len[x];
            rs = s_rs[x];
          }
          const unsigned nz = __ballot_sync(0xffffffffu, len > 0);
          const int nrows = __popc(nz);
          const int src = lane < nrows ? (int)__fns(nz, 0, lane + 1) : 0;
          // every lane takes part in each shuffle; the select comes after
          const int slen = __shfl_sync(0xffffffffu, len, src);
          const int clen = lane < nrows ? slen : 0;
          const long long crs = __shfl_sync(0xffffffffu, rs, src);
          const int cx = xb + src;
          int incl = clen;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
          }
          const int tot = __shfl_sync(0xffffffffu, incl, 31);
          const int excl = incl - clen;
          int done = 0;  // compacted rows that ended before the window
          // two windows of 32 items per iteration: both record loads are in
          // flight before either is probed
          for (int t0 = 0; t0 < tot; t0 += 64) {
            int tw[2], ox[2];
            long long ridx[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              const int w0 = t0 + 32 * u;
              const int last = incl - 1 - w0;  // window position of the row's last item
              const unsigned bit = (lane < nrows && last >= 0 && last < 32) ? (1u << last) : 0u;
              const unsigned ends = __reduce_or_sync(0xffffffffu, bit);
              const int j = (done + __popc(ends & lt)) & 31;
              done += __popc(ends);
              const long long ors = __shfl_sync(0xffffffffu, crs, j);
              const int oex = __shfl_sync(0xffffffffu, excl, j);
              ox[u] = __shfl_sync(0xffffffffu, cx, j);
              tw[u] = w0 + lane;
              ridx[u] = ors + (tw[u] - oex);
            }
            unsigned long long rr[2] = {0ull, 0ull};
#pragma unroll
            for (int u = 0; u < 2; ++u)
              if (tw[u] < tot) rr[u] = G.rec[ridx[u]];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              bool hit = false;
              int y = 0;
              const uint32_t mac = rec_meta(rr[u]);
              // first probe for every lane; the rare collisions continue
              // in a loop that only runs while some lane is unresolved
              const int off = rec_col(rr[u]) - p;
              const bool live = tw[u] < tot && off < kMaxOffset;
              uint32_t h = fib_slot((uint32_t)off, lg);
              uint32_t e = live ? s_hkey[h] : 0u;
              hit = live && (e >> 8) == (uint32_t)off;
              bool open = live && !hit && e != 0u;
              for (int it = 1; it < hs && __any_sync(0xffffffffu, open); ++it) {
                if (open) {
                  h = (h + 1) & (uint32_t)(hs - 1);
                  e = s_hkey[h];
                  hit = (e >> 8) == (uint32_t)off;
                  open = !hit && e != 0u;
                }
              }
              if (hit) y = (int)(e & 0xffu);
              const unsigned m = __ballot_sync(0xffffffffu, hit);
              if (hit) {
                const int pos = qn + __popc(m & lt);
                s_q[pos] = ((unsigned long long)mac << 32) | (uint32_t)(ox[u] | (y << 16));
              }
              qn += __popc(m);
            }
            while (qn >= 32) {
              __syncwarp();
              const int nroot = drain_one(qn - 32 + lane, fp, op, wp, racc);
              tris += nroot > 0;
              rooted += nroot;
              qn -= 32;
              __syncwarp();
            }
          }
        }
        __syncwarp();
        if (lane < qn) {
          const int nroot = drain_one(lane, fp, op, wp, racc);
          tris += nroot > 0;
          rooted += nroot;
        }
        if (ADJ) {
          // flush the neighbours' gradient accumulators of this root
          __syncwarp();
          for (int x = lane; x < k; x += 32) {
            const unsigned long long v = s_g[x];
            if (v) fix_merge(&g_lo[s_col[x]], &g_hi[s_col[x]], v, (long long)v < 0 ? ~0ull : 0ull);
          }
        }
      } else {
        // Long row: the same enumeration reading the row from global memory.
        const unsigned long long* rowp = G.rec + b0;
        for (int x = 0; x < k - 1; ++x) {
          const unsigned long long ra_rec = rowp[x];
          const int a = rec_col(ra_rec);
          const uint32_t mpa = rec_meta(ra_rec);
          const int64_t ra = G.start[a];
          const int ka = G.len[a];
          const uint8_t fa = C.flags[a];
          const int oa = C.orig[a];
          const double wa = (WEIGHTED || ADJ) ? C.w[a] : 0.0;
          if (lane == 0) probes += (unsigned long long)ka;
          for (int j = lane; j < ka; j += 32) {
            const unsigned long long r = G.rec[ra + j];
            const int c = rec_col(r);
            const int y = x + 1 + lower_bound_g(rowp + x + 1, k - x - 1, c);
            if (y < k && rec_col(rowp[y]) == c) {
              const int nroot =
                  ADJ ? tri_grad<false>(X, fp, op, wp, fa, oa, wa, C.flags[c], C.orig[c], C.w[c], mpa,
                                 rec_meta(rowp[y]), rec_meta(r), racc, &g_lo[a], &g_hi[a], &g_lo[c],
                                 &g_hi[c])
                      : tri_bin<WEIGHTED, COUNTS>(X, fp, op, wp, fa, oa, wa, C.flags[c], C.orig[c],
                                                  WEIGHTED ? C.w[c] : 0.0, mpa, rec_meta(rowp[y]),
                                                  rec_meta(r));
              tris += nroot > 0;
              rooted += nroot;
            }
          }
        }
      }
      if (ADJ) {
        racc = fix_warp_sum(racc);
        if (lane == 0 && (racc.lo | racc.hi)) fix_merge(&g_lo[p], &g_hi[p], racc.lo, racc.hi);
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    tris += __shfl_xor_sync(0xffffffffu, tris, o);
    rooted += __shfl_xor_sync(0xffffffffu, rooted, o);
    probes += __shfl_xor_sync(0xffffffffu, probes, o);
  }
  if (lane == 0) {
    if (tris) atomicAdd(&stats[0], tris);
    if (rooted) atomicAdd(&stats[1], rooted);
    if (probes) atomicAdd(&stats[2], probes);
  }
  if (SHIST) {
    __syncthreads();
    for (int k = threadIdx.x; k < nh; k += blockDim.x) {
      if (COUNTS) {
        const unsigned long long v = X.cnt[k];
        if (v) atomicAdd(&g_cnt[k], v);
      }
      if (WEIGHTED) {
        const unsigned long long lo = X.lim[k], hi = X.lim[nh + k];
        if (lo | hi) fix_merge(&g_lim[k], &g_lim[nh + k], lo, hi);
      }
    }
  }
}

}  // namespace

// Warps per block: as many as fit in shared memory (at most 32).
static int tri3_warps(const TriParams& T, bool weighted, bool counts, bool shist, bool adj = false,
                      bool geo = false) {
  const int nh = T.ncfg * T.nmu * 4;
  int nw = kTriMaxWarps;
  while (nw > 1 &&
         tri_layout(nh, T.nmu, T.nbins, T.cap, shist, weighted, counts, nw, adj, geo).total >
             kSmemLimit)
    nw -= 1;
  return nw;
}


static bool tri3_shist(int nh, bool weighted, bool counts) {
  return (size_t)nh * 8 * ((counts ? 1 : 0) + (weighted ? 2 : 0)) <= kMaxHistSmem;
}

size_t tri3_smem_bytes(const TriParams& T, bool weighted, bool counts) {
  const int nh = T.ncfg * T.nmu * 4;
  const bool shist = tri3_shist(nh, weighted, counts);
  return tri_layout(nh, T.nmu, T.nbins, T.cap, shist, weighted, counts,
                    tri3_warps(T, weighted, counts, shist))
      .total;
}

// One launch of the triangle kernel for the roots kmin < k <= kskip of T.
static void launch_tri3_part(const DevCatalog& C, const CSRView& G, const TriParams& T,
                             bool weighted, bool counts, unsigned long long* g_cnt,
                             unsigned long long* g_lim, unsigned long long* stats, int* work,
                             cudaStream_t s) {
  const int nh = T.ncfg * T.nmu * 4;
  const bool shist = tri3_shist(nh, weighted, counts);
  const bool geo = T.geo != 0;
  const int nw = tri3_warps(T, weighted, counts, shist, false, geo);
  const size_t smem =
      tri_layout(nh, T.nmu, T.nbins, T.cap, shist, weighted, counts, nw, false, geo).total;
  if (smem > kSmemLimit) throw Error{-2, "3PCF: per-warp shared memory exceeds the SM limit"};
  GR_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int), s));
#define GR_TRI_LAUNCH(W, K, S)                                                                \
  do {                                                                                        \
    auto kfn = geo ? tri3_kernel<W, K, S, false, true> : tri3_kernel<W, K, S, false, false>;  \
    GR_CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize,        \
                                     (int)smem));                                             \
    int per_sm = 0;                                                                           \
    GR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, nw * 32, smem));   \
    if (per_sm < 1) per_sm = 1;                                                               \
    int64_t blocks = (int64_t)per_sm * sm_count();                                                   \
    const int64_t need = ((int64_t)C.n + nw * kChunk - 1) / (nw * kChunk);                    \
    if (blocks > need) blocks = need;                                                         \
    kfn<<<(unsigned)blocks, nw * 32, smem, s>>>(C, G, T, g_cnt, g_lim, stats, work, nullptr,  \
                                                nullptr, 0.0, nullptr, nullptr);              \
  } while (0)
  if (weighted && counts) {
    if (shist) GR_TRI_LAUNCH(true, true, true); else GR_TRI_LAUNCH(true, true, false);
  } else if (weighted) {
    if (shist) GR_TRI_LAUNCH(true, false, true); else GR_TRI_LAUNCH(true, false, false);
  } else {
    if (shist) GR_TRI_LAUNCH(false, true, true); else GR_TRI_LAUNCH(false, true, false);
  }
#undef GR_TRI_LAUNCH
  GR_CHECK_LAUNCH();
}

// Rows longer than the main launch's capacity (at most kTriCapShort, which
// keeps 16 to 32 warps per block) go to a second, geometric launch whose
// capacity fits them (up to kTriCapLong, fewer warps); rows beyond that take
// the global-memory path.  The two launches add into the same outputs.
constexpr int kTriCapShort = 256;
constexpr int kTriCapLong = 1024;

static void tri3_split(const TriParams& T, TriParams& A, TriParams& B, bool& two) {
  A = T;
  A.kmin = 0;
  A.kskip = 0x7fffffff;
  two = T.long_geo && T.maxdeg > T.cap && T.cap >= kTriCapShort;
  if (!two) return;
  A.kskip = T.cap;
  B = T;
  B.geo = 1;
  B.cap = (int)std::min<int64_t>(((int64_t)T.maxdeg + 31) / 32 * 32, kTriCapLong);
  B.kmin = T.cap;
  B.kskip = 0x7fffffff;
}

int launch_tri3(const DevCatalog& C, const CSRView& G, const TriParams& T, bool weighted,
                 bool counts, unsigned long long* g_cnt, unsigned long long* g_lim,
                 unsigned long long* stats, int* work, cudaStream_t s) {
  if (C.n <= 0) return 0;
  if (!weighted) counts = true;
  TriParams A, B;
  bool two = false;
  tri3_split(T, A, B, two);
  launch_tri3_part(C, G, A, weighted, counts, g_cnt, g_lim, stats, work, s);
  if (two) launch_tri3_part(C, G, B, weighted, counts, g_cnt, g_lim, stats, work, s);
  return two ? 2 : 1;
}

static void launch_adj3_part(const DevCatalog& C, const CSRView& G, const TriParams& T,
                             const double* cot2, const double* cot3, double gscale,
                             unsigned long long* g_lo, unsigned long long* g_hi,
                             unsigned long long* stats, int* work, cudaStream_t s) {
  const int nh = T.ncfg * T.nmu * 4;
  const bool geo = T.geo != 0;
  const int nw = tri3_warps(T, false, false, false, true, geo);
  const size_t smem =
      tri_layout(nh, T.nmu, T.nbins, T.cap, false, false, false, nw, true, geo).total;
  if (smem > kSmemLimit) throw Error{-2, "3PCF adjoint: shared memory exceeds the SM limit"};
  GR_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int), s));
  auto kfn = geo ? tri3_kernel<false, false, false, true, true>
                 : tri3_kernel<false, false, false, true, false>;
  GR_CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  GR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, nw * 32, smem));
  if (per_sm < 1) per_sm = 1;
  int64_t blocks = (int64_t)per_sm * sm_count();
  const int64_t need = ((int64_t)C.n + nw * kChunk - 1) / (nw * kChunk);
  if (blocks > need) blocks = need;
  kfn<<<(unsigned)blocks, nw * 32, smem, s>>>(C, G, T, nullptr, nullptr, stats, work, cot2, cot3,
                                              gscale, g_lo, g_hi);
  GR_CHECK_LAUNCH();
}

int launch_adj3(const DevCatalog& C, const CSRView& G, const TriParams& T, const double* cot2,
                 const double* cot3, double gscale, unsigned long long* g_lo,
                 unsigned long long* g_hi, unsigned long long* stats, int* work, cudaStream_t s) {
  if (C.n <= 0) return 0;
  TriParams A, B;
  bool two = false;
  tri3_split(T, A, B, two);
  launch_adj3_part(C, G, A, cot2, cot3, gscale, g_lo, g_hi, stats, work, s);
  if (two) launch_adj3_part(C, G, B, cot2, cot3, gscale, g_lo, g_hi, stats, work, s);
  return two ? 2 : 1;
}

}  // namespace gr
