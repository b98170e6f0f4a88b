// 3PCF triangle counting: replaces query_graph_3pcf_all
// (src/gramsci.F90:463-510), whose per-root double loop looks up the third
// edge with a binary search into another vertex's row (find_dist,
// :1579-1609).
//
// Every triangle is enumerated exactly once, from its smallest internal
// label p.  A warp takes a root p and stages its upper row R+(p) in shared
// memory together with the flags, catalogue ids and weights of those
// neighbours, a small open-addressing hash table (label -> row position) and
// an owner table mapping each flattened work item f to the neighbour a whose
// row it reads.  The work items (a, c) for c in R+(a) are spread over the
// lanes; each lane loads one 8-byte CSR record and probes the hash table for
// c.  Hits (triangles p < a < c) are pushed to a per-warp queue that is
// drained 32 at a time, so the binning work runs with every lane busy.
//
// A triangle contributes to the rooted histogram of each non-buffer vertex r
// with the bins of its three edges (symmetric bin table), the find_normal mu
// bin of r's two edges taken in catalogue-id order (k1 < k2 in the
// reference's id-sorted row) and the product (w_r w_first) w_second.
#include "gr_kernels.cuh"

namespace gr {

namespace {

constexpr int kTriMaxWarps = 32;  // block size is chosen at launch to fit shared memory
constexpr size_t kSmemLimit = 227 * 1024;
constexpr int kOwn = 512;    // flattened work items per owner-table chunk
constexpr int kQueue = 64;   // hit queue entries per warp
constexpr int kChunk = 4;    // roots taken per work-counter increment
constexpr int kCfgTableBins = 16;  // nbins up to which the configuration table is used

__host__ __device__ inline size_t align8(size_t x) { return (x + 7) & ~(size_t)7; }
__host__ __device__ inline int hash_size(int cap) {
  int h = 32;
  while (h < 2 * cap) h <<= 1;
  return h;
}

struct TriLayout {
  size_t off_cnt, off_fix, off_cot, off_norm, off_rank, off_cfg, off_warp, warp_bytes, total;
  // per-warp sub-offsets
  size_t o_rs, o_w, o_g, o_col, o_meta, o_orig, o_pre, o_hkey, o_qm, o_qxy, o_flag, o_hval, o_own;
};

// adj: the adjoint variant (cotangent tables, per-neighbour gradient
// accumulators) instead of histograms.
__host__ __device__ inline TriLayout tri_layout(int nh, int nmu, int nbins, int cap, bool shist,
                                                bool weighted, int nwarps, bool adj = false) {
  TriLayout L;
  size_t o = 0;
  L.off_cnt = o;
  if (shist) o += (size_t)nh * 8;
  L.off_fix = o;
  if (shist && weighted) o += (size_t)nh * 16;
  L.off_cot = o;
  if (adj) o += (size_t)nh / 4 * 2 * 8;  // cot2, cot3: ncfg * nmu doubles each
  L.off_norm = o;
  o = align8(o + (size_t)nmu * nmu);
  L.off_rank = o;
  o = align8(o + sizeof(int) * 3 * (size_t)(nbins + 2));
  L.off_cfg = o;  // configuration of every (b1, b2, b3), small nbins only
  if (nbins <= kCfgTableBins) o = align8(o + sizeof(uint16_t) * (size_t)nbins * nbins * nbins);
  L.off_warp = o;
  const int hs = hash_size(cap);
  size_t w = 0;
  L.o_rs = w;   w += (size_t)cap * 8;
  L.o_w = w;    w += (size_t)cap * 8;
  L.o_g = w;    if (adj) w += (size_t)cap * 16;  // gradient (lo, hi) per neighbour
  L.o_col = w;  w += (size_t)cap * 4;
  L.o_meta = w; w += (size_t)cap * 4;
  L.o_orig = w; w += (size_t)cap * 4;
  L.o_pre = w;  w += (size_t)(cap + 1) * 4;
  L.o_hkey = w; w += (size_t)hs * 4;
  L.o_qm = w;   w += (size_t)kQueue * 4;
  L.o_qxy = w;  w += (size_t)kQueue * 2;
  L.o_flag = w; w += (size_t)cap;
  L.o_hval = w; w += (size_t)hs;
  L.o_own = w;  w += (size_t)kOwn;
  L.warp_bytes = align8(w);
  L.total = o + L.warp_bytes * nwarps;
  return L;
}

struct TriCtx {
  const uint8_t* norm;
  const int* F;  // 3 x (nbins+2)
  const uint16_t* cfgtab;  // symmetric configuration table or NULL
  int nbins, nmu, ncfg, rsd, nh, equi;
  unsigned long long* cnt;
  unsigned long long* lo;  // fixed-point sums: lo[k], lo[nh + k] = hi[k]
  double fscale;
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

// One triangle (p, a, c) with p < a < c in labels.  Per-vertex data are
// passed in; contributions that land in the same bin are merged before the
// shared-memory atomics.  Returns the number of rooted contributions.
template <bool WEIGHTED>
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
  int m[3] = {-1, -1, -1};
  double pr[3] = {0.0, 0.0, 0.0};
  int cnt[3] = {0, 0, 0};
  if (!(fp & FLAG_BUFFER)) {  // root p: neighbours a, c
    const bool ac = oa < oc;
    m[0] = normal_bin(X, meta_muf(mpa), meta_muf(mpc), ac);
    if (WEIGHTED) pr[0] = ac ? (wp * wa) * wc : (wp * wc) * wa;
    cnt[0] = 1;
  }
  if (!(fa & FLAG_BUFFER)) {  // root a: neighbours p, c
    const bool pc = op < oc;
    m[1] = normal_bin(X, meta_mur(mpa), meta_muf(mac), pc);
    if (WEIGHTED) pr[1] = pc ? (wa * wp) * wc : (wa * wc) * wp;
    cnt[1] = 1;
  }
  if (!(fc & FLAG_BUFFER)) {  // root c: neighbours p, a
    const bool pa = op < oa;
    m[2] = normal_bin(X, meta_mur(mpc), meta_mur(mac), pa);
    if (WEIGHTED) pr[2] = pa ? (wc * wp) * wa : (wc * wa) * wp;
    cnt[2] = 1;
  }
  const int total = cnt[0] + cnt[1] + cnt[2];
  // merge equal bins
  if (m[1] >= 0 && m[1] == m[0]) { cnt[0] += cnt[1]; pr[0] += pr[1]; cnt[1] = 0; }
  if (m[2] >= 0 && m[2] == m[0]) { cnt[0] += cnt[2]; pr[0] += pr[2]; cnt[2] = 0; }
  else if (m[2] >= 0 && m[2] == m[1] && cnt[1]) { cnt[1] += cnt[2]; pr[1] += pr[2]; cnt[2] = 0; }
  const int base = (cfg - 1) + X.ncfg * X.nmu * nr;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    if (cnt[r] == 0) continue;
    const int k = base + X.ncfg * (m[r] - 1);
    atomicAdd(&X.cnt[k], (unsigned long long)cnt[r]);
    if (WEIGHTED) fix_add(&X.lo[k], &X.lo[X.nh + k], pr[r], X.fscale);
  }
  return total;
}

// Adjoint of one triangle (p, a, c): every non-buffer root r contributes
// (cot2 - [all random] cot3)[cfg, m_r] (N3 accumulates minus the product);
// with C the sum, dL/dw_p += C w_a w_c, dL/dw_a += C w_p w_c, dL/dw_c +=
// C w_p w_a.  p's term goes to the lane's register accumulator, a's and c's
// to the given fixed-point accumulators.
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
    fix_add(alo, ahi, C * (wp * wc), X.gscale);
    fix_add(clo, chi, C * (wp * wa), X.gscale);
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

__device__ __forceinline__ uint32_t hash_slot(int key, int hmask) {
  return ((uint32_t)key * 2654435761u) & (uint32_t)hmask;
}

// ADJ: accumulate the weight gradient (g_lo / g_hi, label order) of
// L = sum cot2 N2 + cot3 N3 instead of the histograms.
template <bool WEIGHTED, bool SHIST, bool ADJ>
__global__ void __launch_bounds__(kTriMaxWarps * 32) tri3_kernel(DevCatalog C, CSRView G, TriParams T,
                                                           unsigned long long* __restrict__ g_cnt,
                                                           unsigned long long* __restrict__ g_fix,
                                                           double fscale,
                                                           unsigned long long* __restrict__ stats,
                                                           int* __restrict__ work,
                                                           const double* __restrict__ cot2,
                                                           const double* __restrict__ cot3,
                                                           double gscale,
                                                           unsigned long long* __restrict__ g_lo,
                                                           unsigned long long* __restrict__ g_hi) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int nh = T.ncfg * T.nmu * 4;
  const TriLayout L = tri_layout(nh, T.nmu, T.nbins, T.cap, SHIST, WEIGHTED, blockDim.x >> 5, ADJ);
  TriCtx X;
  X.nbins = T.nbins;
  X.nmu = T.nmu;
  X.ncfg = T.ncfg;
  X.rsd = T.rsd;
  X.equi = T.equi;
  X.nh = nh;
  X.fscale = fscale;
  X.cnt = SHIST ? reinterpret_cast<unsigned long long*>(smem + L.off_cnt) : g_cnt;
  X.lo = SHIST ? reinterpret_cast<unsigned long long*>(smem + L.off_fix) : g_fix;
  uint8_t* s_norm = smem + L.off_norm;
  int* s_F = reinterpret_cast<int*>(smem + L.off_rank);
  X.norm = s_norm;
  X.F = s_F;
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
      X.cnt[k] = 0ull;
      if (WEIGHTED) {
        X.lo[k] = 0ull;
        X.lo[nh + k] = 0ull;
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
  long long* s_rs = reinterpret_cast<long long*>(wb + L.o_rs);
  double* s_w = reinterpret_cast<double*>(wb + L.o_w);
  int* s_col = reinterpret_cast<int*>(wb + L.o_col);
  uint32_t* s_meta = reinterpret_cast<uint32_t*>(wb + L.o_meta);
  int* s_orig = reinterpret_cast<int*>(wb + L.o_orig);
  int* s_pre = reinterpret_cast<int*>(wb + L.o_pre);
  int* s_hkey = reinterpret_cast<int*>(wb + L.o_hkey);
  uint32_t* s_qm = reinterpret_cast<uint32_t*>(wb + L.o_qm);
  uint16_t* s_qxy = reinterpret_cast<uint16_t*>(wb + L.o_qxy);
  uint8_t* s_flag = wb + L.o_flag;
  uint8_t* s_hval = wb + L.o_hval;
  uint8_t* s_own = wb + L.o_own;
  unsigned long long* s_glo = reinterpret_cast<unsigned long long*>(wb + L.o_g);
  unsigned long long* s_ghi = s_glo + T.cap;
  const int hs = hash_size(T.cap);
  const int hmask = hs - 1;

  unsigned long long tris = 0, rooted = 0, probes = 0;

  for (;;) {
    int base_root = 0;
    if (lane == 0) base_root = atomicAdd(work, kChunk);
    base_root = __shfl_sync(0xffffffffu, base_root, 0);
    if (base_root >= C.n) break;
    const int end_root = min(base_root + kChunk, C.n);
    for (int p = base_root; p < end_root; ++p) {
      const int64_t b0 = G.row_ptr[p];
      const int k = (int)(G.row_ptr[p + 1] - b0);
      if (k < 2) continue;
      const uint8_t fp = C.flags[p];
      const int op = C.orig[p];
      const double wp = WEIGHTED ? C.w[p] : 0.0;
      Fix128 racc = {0ull, 0ull};
      if (k <= T.cap) {
        __syncwarp();
        for (int h = lane; h < hs; h += 32) s_hkey[h] = -1;
        __syncwarp();
        // stage R+(p) and the data of its vertices; insert into the hash table
        int carry = 0;
        for (int xb = 0; xb < k; xb += 32) {
          const int x = xb + lane;
          int len = 0;
          if (x < k) {
            const unsigned long long r = G.rec[b0 + x];
            const int a = rec_col(r);
            s_col[x] = a;
            s_meta[x] = rec_meta(r);
            const long long rs = G.row_ptr[a];
            s_rs[x] = rs;
            len = (int)(G.row_ptr[a + 1] - rs);
            s_flag[x] = C.flags[a];
            s_orig[x] = C.orig[a];
            if (WEIGHTED) s_w[x] = C.w[a];
            if (ADJ) {
              s_glo[x] = 0ull;
              s_ghi[x] = 0ull;
            }
            uint32_t h = hash_slot(a, hmask);
            for (int t = 0; t < hs; ++t) {
              if (atomicCAS(&s_hkey[h], -1, a) == -1) {
                s_hval[h] = (uint8_t)x;
                break;
              }
              h = (h + 1) & hmask;
            }
          }
          int incl = len;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
          }
          if (x < k) {
            s_pre[x + 1] = carry + incl;
            // record index of work item f = s_rs[x] + f
            s_rs[x] -= (long long)(carry + incl - len);
          }
          carry += __shfl_sync(0xffffffffu, incl, 31);
        }
        if (lane == 0) s_pre[0] = 0;
        const int W = carry;
        if (lane == 0) probes += (unsigned long long)W;
        int qn = 0;
        int x0 = 0;  // first row overlapping the current owner chunk
        for (int fb = 0; fb < W; fb += kOwn) {
          const int fe = min(W, fb + kOwn);
          __syncwarp();
          // owner table for work items [fb, fe)
          while (x0 < k && s_pre[x0 + 1] <= fb) ++x0;
          for (int x = x0; x < k && s_pre[x] < fe; ++x) {
            const int lo = max(s_pre[x], fb), hi = min(s_pre[x + 1], fe);
            for (int f = lo + lane; f < hi; f += 32) s_own[f - fb] = (uint8_t)x;
          }
          __syncwarp();
          for (int f0 = fb; f0 < fe; f0 += 32) {
            const int f = f0 + lane;
            bool hit = false;
            int x = 0, y = 0;
            uint32_t mac = 0;
            if (f < fe) {
              x = s_own[f - fb];
              const unsigned long long r = G.rec[s_rs[x] + f];
              const int c = rec_col(r);
              mac = rec_meta(r);
              uint32_t h = hash_slot(c, hmask);
              for (int t = 0; t < hs; ++t) {
                const int key = s_hkey[h];
                if (key == c) {
                  hit = true;
                  y = s_hval[h];
                  break;
                }
                if (key < 0) break;
                h = (h + 1) & hmask;
              }
            }
            const unsigned m = __ballot_sync(0xffffffffu, hit);
            if (hit) {
              const int pos = qn + __popc(m & lt);
              s_qm[pos] = mac;
              s_qxy[pos] = (uint16_t)(x | (y << 8));
            }
            qn += __popc(m);
            if (qn >= 32) {
              __syncwarp();
              const int e = qn - 32 + lane;
              const uint16_t xy = s_qxy[e];
              const int qx = xy & 0xff, qy = xy >> 8;
              const int nroot =
                  ADJ ? tri_grad(X, fp, op, wp, s_flag[qx], s_orig[qx], s_w[qx], s_flag[qy],
                                 s_orig[qy], s_w[qy], s_meta[qx], s_meta[qy], s_qm[e], racc,
                                 &s_glo[qx], &s_ghi[qx], &s_glo[qy], &s_ghi[qy])
                      : tri_bin<WEIGHTED>(X, fp, op, wp, s_flag[qx], s_orig[qx],
                                          WEIGHTED ? s_w[qx] : 0.0, s_flag[qy], s_orig[qy],
                                          WEIGHTED ? s_w[qy] : 0.0, s_meta[qx], s_meta[qy], s_qm[e]);
              tris += nroot > 0;
              rooted += nroot;
              qn -= 32;
              __syncwarp();
            }
          }
        }
        __syncwarp();
        if (lane < qn) {
          const uint16_t xy = s_qxy[lane];
          const int qx = xy & 0xff, qy = xy >> 8;
          const int nroot =
              ADJ ? tri_grad(X, fp, op, wp, s_flag[qx], s_orig[qx], s_w[qx], s_flag[qy],
                             s_orig[qy], s_w[qy], s_meta[qx], s_meta[qy], s_qm[lane], racc,
                             &s_glo[qx], &s_ghi[qx], &s_glo[qy], &s_ghi[qy])
                  : tri_bin<WEIGHTED>(X, fp, op, wp, s_flag[qx], s_orig[qx],
                                      WEIGHTED ? s_w[qx] : 0.0, s_flag[qy], s_orig[qy],
                                      WEIGHTED ? s_w[qy] : 0.0, s_meta[qx], s_meta[qy], s_qm[lane]);
          tris += nroot > 0;
          rooted += nroot;
        }
        if (ADJ) {
          // flush the neighbours' gradient accumulators of this root
          __syncwarp();
          for (int x = lane; x < k; x += 32) {
            const unsigned long long lo = s_glo[x], hi = s_ghi[x];
            if (lo | hi) fix_merge(&g_lo[s_col[x]], &g_hi[s_col[x]], lo, hi);
          }
        }
      } else {
        // Long row: the same enumeration reading the row from global memory.
        const unsigned long long* rowp = G.rec + b0;
        for (int x = 0; x < k - 1; ++x) {
          const unsigned long long ra_rec = rowp[x];
          const int a = rec_col(ra_rec);
          const uint32_t mpa = rec_meta(ra_rec);
          const int64_t ra = G.row_ptr[a];
          const int ka = (int)(G.row_ptr[a + 1] - ra);
          const uint8_t fa = C.flags[a];
          const int oa = C.orig[a];
          const double wa = WEIGHTED ? C.w[a] : 0.0;
          if (lane == 0) probes += (unsigned long long)ka;
          for (int j = lane; j < ka; j += 32) {
            const unsigned long long r = G.rec[ra + j];
            const int c = rec_col(r);
            const int y = x + 1 + lower_bound_g(rowp + x + 1, k - x - 1, c);
            if (y < k && rec_col(rowp[y]) == c) {
              const int nroot =
                  ADJ ? tri_grad(X, fp, op, wp, fa, oa, wa, C.flags[c], C.orig[c], C.w[c], mpa,
                                 rec_meta(rowp[y]), rec_meta(r), racc, &g_lo[a], &g_hi[a], &g_lo[c],
                                 &g_hi[c])
                      : tri_bin<WEIGHTED>(X, fp, op, wp, fa, oa, wa, C.flags[c], C.orig[c],
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
      const unsigned long long v = X.cnt[k];
      if (v) {
        atomicAdd(&g_cnt[k], v);
        if (WEIGHTED) fix_merge(&g_fix[k], &g_fix[nh + k], X.lo[k], X.lo[nh + k]);
      }
    }
  }
}

}  // namespace

// Warps per block: as many as fit in shared memory (at most 32).
static int tri3_warps(const TriParams& T, bool weighted, bool shist, bool adj = false) {
  const int nh = T.ncfg * T.nmu * 4;
  int nw = kTriMaxWarps;
  while (nw > 1 && tri_layout(nh, T.nmu, T.nbins, T.cap, shist, weighted, nw, adj).total > kSmemLimit)
    nw -= 1;
  return nw;
}

size_t tri3_smem_bytes(const TriParams& T, bool weighted) {
  const int nh = T.ncfg * T.nmu * 4;
  const bool shist = (size_t)nh * 8 * (weighted ? 3 : 1) <= kMaxHistSmem;
  return tri_layout(nh, T.nmu, T.nbins, T.cap, shist, weighted, tri3_warps(T, weighted, shist)).total;
}

void launch_tri3(const DevCatalog& C, const CSRView& G, const TriParams& T, bool weighted,
                 unsigned long long* g_cnt, unsigned long long* g_fix, double fscale,
                 unsigned long long* stats, int* work, cudaStream_t s) {
  if (C.n <= 0) return;
  const int nh = T.ncfg * T.nmu * 4;
  const bool shist = (size_t)nh * 8 * (weighted ? 3 : 1) <= kMaxHistSmem;
  const int nw = tri3_warps(T, weighted, shist);
  const TriLayout L = tri_layout(nh, T.nmu, T.nbins, T.cap, shist, weighted, nw);
  const size_t smem = L.total;
  if (smem > kSmemLimit) throw Error{-2, "3PCF: per-warp shared memory exceeds the SM limit"};
  GR_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int), s));
#define GR_TRI_LAUNCH(W, S)                                                                   \
  do {                                                                                        \
    auto kfn = tri3_kernel<W, S, false>;                                                             \
    GR_CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize,        \
                                     (int)smem));                                             \
    int per_sm = 0;                                                                           \
    GR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, nw * 32, smem));   \
    if (per_sm < 1) per_sm = 1;                                                               \
    int64_t blocks = (int64_t)per_sm * 148;                                                   \
    const int64_t need = ((int64_t)C.n + nw * kChunk - 1) / (nw * kChunk);                    \
    if (blocks > need) blocks = need;                                                         \
    kfn<<<(unsigned)blocks, nw * 32, smem, s>>>(C, G, T, g_cnt, g_fix, fscale, stats, work,    \
                                                nullptr, nullptr, 0.0, nullptr, nullptr);     \
  } while (0)
  if (weighted) {
    if (shist) GR_TRI_LAUNCH(true, true); else GR_TRI_LAUNCH(true, false);
  } else {
    if (shist) GR_TRI_LAUNCH(false, true); else GR_TRI_LAUNCH(false, false);
  }
#undef GR_TRI_LAUNCH
  GR_CHECK_LAUNCH();
}

void launch_adj3(const DevCatalog& C, const CSRView& G, const TriParams& T, const double* cot2,
                 const double* cot3, double gscale, unsigned long long* g_lo,
                 unsigned long long* g_hi, unsigned long long* stats, int* work, cudaStream_t s) {
  if (C.n <= 0) return;
  const int nh = T.ncfg * T.nmu * 4;
  const int nw = tri3_warps(T, true, false, true);
  const size_t smem = tri_layout(nh, T.nmu, T.nbins, T.cap, false, true, nw, true).total;
  if (smem > kSmemLimit) throw Error{-2, "3PCF adjoint: shared memory exceeds the SM limit"};
  GR_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int), s));
  auto kfn = tri3_kernel<true, false, true>;
  GR_CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  GR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, nw * 32, smem));
  if (per_sm < 1) per_sm = 1;
  int64_t blocks = (int64_t)per_sm * 148;
  const int64_t need = ((int64_t)C.n + nw * kChunk - 1) / (nw * kChunk);
  if (blocks > need) blocks = need;
  kfn<<<(unsigned)blocks, nw * 32, smem, s>>>(C, G, T, nullptr, nullptr, 0.0, stats, work, cot2,
                                              cot3, gscale, g_lo, g_hi);
  GR_CHECK_LAUNCH();
}

}  // namespace gr
