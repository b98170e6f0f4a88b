// 3PCF triangle counting: replaces query_graph_3pcf_all
// (src/gramsci.F90:463-510), whose per-root double loop looks up the third
// edge with a binary search into another vertex's row (find_dist,
// :1579-1609).
//
// Here every triangle is enumerated exactly once, from its smallest internal
// label p: for each a in R+(p) and each c in R+(a), c is looked up in R+(p),
// which sits in shared memory.  The (a, c) work items of one root are
// flattened over the warp's lanes through a prefix sum of |R+(a)|, so short
// and long rows keep all lanes busy.  A found triangle contributes to the
// rooted histogram of each non-buffer vertex r, with the bins of its three
// edges, the find_normal mu bin of r's two edges taken in catalogue-id order
// (as k1 < k2 in the reference's id-sorted row), and the product
// (w_r w_first) w_second.
#include "gr_kernels.cuh"

namespace gr {

namespace {

constexpr int kTriWarps = 8;
constexpr int kTriThreads = kTriWarps * 32;

struct TriLayout {
  size_t off_cnt, off_sum, off_norm, off_rank, off_warp, warp_bytes, total;
};

__host__ __device__ inline size_t align8(size_t x) { return (x + 7) & ~(size_t)7; }

__host__ __device__ inline TriLayout tri_layout(int nh, int nmu, int nbins, int cap, bool shist,
                                                bool weighted) {
  TriLayout L;
  size_t o = 0;
  L.off_cnt = o;
  if (shist) o += (size_t)nh * 8;
  L.off_sum = o;
  if (shist && weighted) o += (size_t)nh * 8;
  L.off_norm = o;
  o = align8(o + (size_t)nmu * nmu);
  L.off_rank = o;
  o = align8(o + sizeof(int) * 3 * (size_t)(nbins + 2));
  L.off_warp = o;
  L.warp_bytes = align8((size_t)cap * (8 + 4 + 4) + (size_t)(cap + 1) * 4);
  L.total = o + L.warp_bytes * kTriWarps;
  return L;
}

struct TriCtx {
  const uint8_t* norm;
  const int* F;  // 3 x (nbins+2)
  int nbins, nmu, ncfg, rsd;
  unsigned long long* cnt;
  double* sum;
};

__device__ __forceinline__ int rank3_s(const int* F, int nb2, int a, int b, int c) {
  return 1 + (F[a] - F[1]) + (F[nb2 + b] - F[nb2 + a]) + (F[2 * nb2 + c] - F[2 * nb2 + b]);
}

template <bool WEIGHTED>
__device__ __forceinline__ void tri_add(const TriCtx& X, int cfg, int mu1, int mu2, bool first_is_1,
                                        int nr, double prod) {
  int m = 1;
  if (X.rsd) m = first_is_1 ? X.norm[(mu1 - 1) + X.nmu * (mu2 - 1)]
                            : X.norm[(mu2 - 1) + X.nmu * (mu1 - 1)];
  int k = (cfg - 1) + X.ncfg * ((m - 1) + X.nmu * nr);
  atomicAdd(&X.cnt[k], 1ull);
  if (WEIGHTED) atomicAdd(&X.sum[k], prod);
}

// Triangle (p, a, c), p < a < c in labels, with edge metadata (p,a), (p,c),
// (a,c).  Returns the number of rooted contributions.
template <bool WEIGHTED>
__device__ __forceinline__ int tri_contrib(const DevCatalog& C, const TriCtx& X, uint8_t fp, int op,
                                           double wp, int a, int c, uint32_t mpa, uint32_t mpc,
                                           uint32_t mac) {
  const uint8_t fa = C.flags[a], fc = C.flags[c];
  const int oa = C.orig[a], oc = C.orig[c];
  double wa = 0.0, wc = 0.0;
  if (WEIGHTED) {
    wa = C.w[a];
    wc = C.w[c];
  }
  int s1 = meta_bin(mpa), s2 = meta_bin(mpc), s3 = meta_bin(mac);
  sort3i(s1, s2, s3);
  const int cfg = rank3_s(X.F, X.nbins + 2, s1, s2, s3);
  const int nr = (fp & FLAG_RANDOM) + (fa & FLAG_RANDOM) + (fc & FLAG_RANDOM);
  int n = 0;
  if (!(fp & FLAG_BUFFER)) {  // root p: neighbours a, c
    bool ac = oa < oc;
    double pr = 0.0;
    if (WEIGHTED) pr = ac ? (wp * wa) * wc : (wp * wc) * wa;
    tri_add<WEIGHTED>(X, cfg, meta_muf(mpa), meta_muf(mpc), ac, nr, pr);
    n++;
  }
  if (!(fa & FLAG_BUFFER)) {  // root a: neighbours p, c
    bool pc = op < oc;
    double pr = 0.0;
    if (WEIGHTED) pr = pc ? (wa * wp) * wc : (wa * wc) * wp;
    tri_add<WEIGHTED>(X, cfg, meta_mur(mpa), meta_muf(mac), pc, nr, pr);
    n++;
  }
  if (!(fc & FLAG_BUFFER)) {  // root c: neighbours p, a
    bool pa = op < oa;
    double pr = 0.0;
    if (WEIGHTED) pr = pa ? (wc * wp) * wa : (wc * wa) * wp;
    tri_add<WEIGHTED>(X, cfg, meta_mur(mpc), meta_mur(mac), pa, nr, pr);
    n++;
  }
  return n;
}

// first index in sorted a[0..n) with a[i] >= v
__device__ __forceinline__ int lower_bound_i(const int* a, int n, int v) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

template <bool WEIGHTED, bool SHIST>
__global__ void __launch_bounds__(kTriThreads) tri3_kernel(DevCatalog C, CSRView G, TriParams T,
                                                           unsigned long long* __restrict__ g_cnt,
                                                           double* __restrict__ g_sum,
                                                           unsigned long long* __restrict__ stats) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int nh = T.ncfg * T.nmu * 4;
  const TriLayout L = tri_layout(nh, T.nmu, T.nbins, T.cap, SHIST, WEIGHTED);
  TriCtx X;
  X.nbins = T.nbins;
  X.nmu = T.nmu;
  X.ncfg = T.ncfg;
  X.rsd = T.rsd;
  X.cnt = SHIST ? reinterpret_cast<unsigned long long*>(smem + L.off_cnt) : g_cnt;
  X.sum = SHIST ? reinterpret_cast<double*>(smem + L.off_sum) : g_sum;
  uint8_t* s_norm = smem + L.off_norm;
  int* s_F = reinterpret_cast<int*>(smem + L.off_rank);
  X.norm = s_norm;
  X.F = s_F;
  if (SHIST) {
    for (int k = threadIdx.x; k < nh; k += blockDim.x) {
      X.cnt[k] = 0ull;
      if (WEIGHTED) X.sum[k] = 0.0;
    }
  }
  for (int k = threadIdx.x; k < T.nmu * T.nmu; k += blockDim.x) s_norm[k] = T.rsd ? T.normal[k] : 1;
  const int nb2 = T.nbins + 2;
  for (int k = threadIdx.x; k < 3 * nb2; k += blockDim.x) s_F[k] = T.rank.F[k / nb2][k % nb2];
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  unsigned char* wbase = smem + L.off_warp + L.warp_bytes * wib;
  long long* s_rstart = reinterpret_cast<long long*>(wbase);
  int* s_col = reinterpret_cast<int*>(wbase + (size_t)T.cap * 8);
  uint32_t* s_meta = reinterpret_cast<uint32_t*>(wbase + (size_t)T.cap * 12);
  int* s_pre = reinterpret_cast<int*>(wbase + (size_t)T.cap * 16);

  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  unsigned long long tris = 0, rooted = 0, probes = 0;

  for (int p = warp; p < C.n; p += nwarps) {
    const int64_t b0 = G.row_ptr[p];
    const int k = (int)(G.row_ptr[p + 1] - b0);
    if (k < 2) continue;
    const uint8_t fp = C.flags[p];
    const int op = C.orig[p];
    const double wp = WEIGHTED ? C.w[p] : 0.0;
    if (k <= T.cap) {
      __syncwarp();
      int carry = 0;
      for (int xb = 0; xb < k; xb += 32) {
        int x = xb + lane;
        int len = 0;
        if (x < k) {
          int a = G.col[b0 + x];
          s_col[x] = a;
          s_meta[x] = G.meta[b0 + x];
          long long rs = G.row_ptr[a];
          s_rstart[x] = rs;
          len = (int)(G.row_ptr[a + 1] - rs);
        }
        int incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          int y = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += y;
        }
        if (x < k) s_pre[x + 1] = carry + incl;
        carry += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (lane == 0) s_pre[0] = 0;
      __syncwarp();
      const int W = carry;
      probes += (lane == 0) ? (unsigned long long)W : 0ull;
      for (int base = 0; base < W; base += 32) {
        int f = base + lane;
        if (f >= W) break;
        // last x with pre[x] <= f
        int lo = 0, hi = k - 1;
        while (lo < hi) {
          int mid = (lo + hi + 1) >> 1;
          if (s_pre[mid] <= f)
            lo = mid;
          else
            hi = mid - 1;
        }
        const int x = lo;
        const int64_t e = s_rstart[x] + (f - s_pre[x]);
        const int c = G.col[e];
        const int y = lower_bound_i(s_col, k, c);
        if (y < k && s_col[y] == c) {
          int nroot = tri_contrib<WEIGHTED>(C, X, fp, op, wp, s_col[x], c, s_meta[x], s_meta[y],
                                            G.meta[e]);
          tris += nroot > 0;
          rooted += nroot;
        }
      }
    } else {
      // Long row: the same enumeration with the row read from global memory.
      const int* rowc = G.col + b0;
      for (int x = 0; x < k - 1; ++x) {
        const int a = rowc[x];
        const uint32_t mpa = G.meta[b0 + x];
        const int64_t ra = G.row_ptr[a];
        const int ka = (int)(G.row_ptr[a + 1] - ra);
        if (lane == 0) probes += (unsigned long long)ka;
        for (int j = lane; j < ka; j += 32) {
          const int c = G.col[ra + j];
          const int y = lower_bound_i(rowc, k, c);
          if (y < k && rowc[y] == c) {
            int nroot = tri_contrib<WEIGHTED>(C, X, fp, op, wp, a, c, mpa, G.meta[b0 + y],
                                              G.meta[ra + j]);
            tris += nroot > 0;
            rooted += nroot;
          }
        }
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
      unsigned long long v = X.cnt[k];
      if (v) {
        atomicAdd(&g_cnt[k], v);
        if (WEIGHTED) atomicAdd(&g_sum[k], X.sum[k]);
      }
    }
  }
}

}  // namespace

void launch_tri3(const DevCatalog& C, const CSRView& G, const TriParams& T, bool weighted,
                 unsigned long long* g_cnt, double* g_sum, unsigned long long* stats,
                 cudaStream_t s) {
  if (C.n <= 0) return;
  const int nh = T.ncfg * T.nmu * 4;
  size_t hist_bytes = (size_t)nh * 8 * (weighted ? 2 : 1);
  const bool shist = hist_bytes <= kMaxHistSmem;
  TriLayout L = tri_layout(nh, T.nmu, T.nbins, T.cap, shist, weighted);
  size_t smem = L.total;
#define GR_TRI_LAUNCH(W, S)                                                                   \
  do {                                                                                        \
    auto kfn = tri3_kernel<W, S>;                                                             \
    GR_CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize,        \
                                     (int)smem));                                             \
    int per_sm = 0;                                                                           \
    GR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kTriThreads, smem)); \
    if (per_sm < 1) per_sm = 1;                                                               \
    int64_t blocks = (int64_t)per_sm * 148;                                                   \
    int64_t need = ((int64_t)C.n + kTriWarps - 1) / kTriWarps;                                \
    if (blocks > need) blocks = need;                                                         \
    kfn<<<(unsigned)blocks, kTriThreads, smem, s>>>(C, G, T, g_cnt, g_sum, stats);            \
  } while (0)
  if (weighted) {
    if (shist) GR_TRI_LAUNCH(true, true); else GR_TRI_LAUNCH(true, false);
  } else {
    if (shist) GR_TRI_LAUNCH(false, true); else GR_TRI_LAUNCH(false, false);
  }
#undef GR_TRI_LAUNCH
  GR_CHECK_LAUNCH();
}

}  // namespace gr
