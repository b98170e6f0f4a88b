// 4PCF 4-clique counting: replaces query_4pcf_all2 (src/gramsci.F90:662-825),
// whose per-root triple loop performs three find_dist binary searches per
// candidate triple.
//
// Every 4-clique is enumerated exactly once, from its smallest label p: for
// each a in R+(p), the warp builds X = R+(a) ∩ R+(p) in shared memory
// (ballot compaction keeps it sorted), then for each b in X and each c in
// R+(b) looks c up in X.  The clique's six edge bins are known at that point;
// it then contributes, for every vertex r that is a root in the reference
// (not a buffer point, row length > 3), with the other three vertices taken
// in catalogue-id order (a < b < c of the reference's k1 < k2 < k3), if the
// perimeter r-a-b-c-r is canonical (bintable entry > 0), to N2 / N3 at
// (cfg, bin(r,b), bin(a,c)) and to the six disconnected pair terms.
#include "gr_kernels.cuh"

namespace gr {

namespace {

constexpr int kQuadWarps = 4;
constexpr int kQuadThreads = kQuadWarps * 32;

__host__ __device__ inline size_t qalign8(size_t x) { return (x + 7) & ~(size_t)7; }

struct QuadLayout {
  size_t off_rank, off_warp, warp_bytes, total;
};

__host__ __device__ inline QuadLayout quad_layout(int nbins, int cap) {
  QuadLayout L;
  size_t o = 0;
  L.off_rank = o;
  o = qalign8(o + sizeof(int) * 4 * (size_t)(nbins + 2));
  L.off_warp = o;
  // row: rstart(8) col(4) meta(4) len(4); X: xstart(8) xc(4) xy(4) xm(4) xpre(4, cap+1)
  L.warp_bytes = qalign8((size_t)cap * (8 + 4 + 4 + 4) + (size_t)cap * (8 + 4 + 4 + 4) + (size_t)(cap + 1) * 4);
  L.total = o + L.warp_bytes * kQuadWarps;
  return L;
}

__device__ __forceinline__ int qlower_bound(const int* a, int n, int v) {
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

struct QuadCtx {
  const int* F;  // 4 x (nbins+2)
  int nbins, ncfg, nbin, tetra;
  unsigned long long *cnt, *dcnt;
  unsigned long long *fix, *dfix;  // fixed-point (lo, hi) sums, hi at +5*nbin / +24*nbin
  double fscale;  // scale of the 4-point products
  double dscale;  // scale of the pair products of the disconnected terms
};

// disc term t: gate role and pair roles (0 = root i, 1 = a, 2 = b, 3 = c),
// gramsci.F90:754-818 (t = 1..6 there).
__constant__ int kGate[6] = {3, 3, 1, 0, 0, 0};
__constant__ int kPu[6] = {0, 0, 0, 1, 3, 3};
__constant__ int kPv[6] = {1, 2, 3, 2, 2, 1};

// -tetra terms (gramsci.F90:591-646): gate role, product roles, and the
// pair that must also be random for discR; roles 0 = root, 1..3 = the
// other vertices in catalogue-id order.
__constant__ int kTGate[6] = {3, 3, 1, 0, 0, 0};
__constant__ int kTPa[6] = {3, 3, 1, 0, 0, 0};
__constant__ int kTPb[6] = {0, 0, 0, 1, 3, 3};
__constant__ int kTPc[6] = {1, 2, 3, 2, 2, 1};

// query_graph_tetrahedron: a 4-clique with all six edges in bin b counts from
// each non-buffer vertex (no row-length condition).
template <bool WEIGHTED>
__device__ __forceinline__ int tetra_contrib(const DevCatalog& C, const QuadCtx& X, const int v[4],
                                             const uint32_t m[6]) {
  const int b = meta_bin(m[0]);
#pragma unroll
  for (int k = 1; k < 6; ++k)
    if (meta_bin(m[k]) != b) return 0;
  uint8_t fl[4];
  int og[4];
  double w[4];
  bool rnd[4];
  int nr = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    fl[k] = C.flags[v[k]];
    og[k] = C.orig[v[k]];
    w[k] = WEIGHTED ? C.w[v[k]] : 0.0;
    rnd[k] = fl[k] & FLAG_RANDOM;
    nr += rnd[k];
  }
  const int nb = X.nbins;
  int n = 0;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    if (fl[r] & FLAG_BUFFER) continue;
    int o[3], t = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k != r) o[t++] = k;
    int q;
    if (og[o[0]] > og[o[1]]) { q = o[0]; o[0] = o[1]; o[1] = q; }
    if (og[o[1]] > og[o[2]]) { q = o[1]; o[1] = o[2]; o[2] = q; }
    if (og[o[0]] > og[o[1]]) { q = o[0]; o[0] = o[1]; o[1] = q; }
    const int role[4] = {r, o[0], o[1], o[2]};
    atomicAdd(&X.cnt[(b - 1) + nb * nr], 1ull);
    if (WEIGHTED)
      fix_add(&X.fix[(b - 1) + nb * nr], &X.fix[(b - 1) + nb * (nr + 5)],
              ((w[r] * w[o[0]]) * w[o[1]]) * w[o[2]], X.fscale);
#pragma unroll
    for (int tt = 0; tt < 6; ++tt) {
      if (!rnd[role[kTGate[tt]]]) continue;
      const int ua = role[kTPa[tt]], ub = role[kTPb[tt]], uc = role[kTPc[tt]];
      const int nr3 = (int)rnd[ua] + (int)rnd[ub] + (int)rnd[uc];
      const int kt = (b - 1) + nb * tt;
      const double qv = WEIGHTED ? (w[ua] * w[ub]) * w[uc] : 0.0;
      atomicAdd(&X.dcnt[kt + nb * 6 * nr3], 1ull);
      if (WEIGHTED) fix_add(&X.dfix[kt + nb * 6 * nr3], &X.dfix[kt + nb * 6 * (nr3 + 5)], qv, X.dscale);
      if (rnd[ub] && rnd[uc]) {
        atomicAdd(&X.dcnt[kt + nb * 24], 1ull);
        if (WEIGHTED) fix_add(&X.dfix[kt + nb * 24], &X.dfix[kt + nb * 54], qv, X.dscale);
      }
    }
    n++;
  }
  return n;
}

template <bool WEIGHTED>
__device__ __forceinline__ int quad_contrib(const DevCatalog& C, const CSRView& G, const QuadCtx& X,
                                            const int v[4], const uint32_t m[6]) {
  // m: (0,1) (0,2) (0,3) (1,2) (1,3) (2,3)
  int B[4][4];
  B[0][1] = B[1][0] = meta_bin(m[0]);
  B[0][2] = B[2][0] = meta_bin(m[1]);
  B[0][3] = B[3][0] = meta_bin(m[2]);
  B[1][2] = B[2][1] = meta_bin(m[3]);
  B[1][3] = B[3][1] = meta_bin(m[4]);
  B[2][3] = B[3][2] = meta_bin(m[5]);
  uint8_t fl[4];
  int og[4];
  double w[4];
  bool rnd[4];
  int nr = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    fl[k] = C.flags[v[k]];
    og[k] = C.orig[v[k]];
    w[k] = WEIGHTED ? C.w[v[k]] : 0.0;
    rnd[k] = fl[k] & FLAG_RANDOM;
    nr += rnd[k];
  }
  const int nb2 = X.nbins + 2;
  int n = 0;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    if (fl[r] & FLAG_BUFFER) continue;
    if (G.deg_full[v[r]] <= 3) continue;
    int o[3], t = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k != r) o[t++] = k;
    // order the other three by catalogue id
    int q;
    if (og[o[0]] > og[o[1]]) { q = o[0]; o[0] = o[1]; o[1] = q; }
    if (og[o[1]] > og[o[2]]) { q = o[1]; o[1] = o[2]; o[2] = q; }
    if (og[o[0]] > og[o[1]]) { q = o[0]; o[0] = o[1]; o[1] = q; }
    const int b1 = B[r][o[0]], b2 = B[o[0]][o[1]], b3 = B[o[1]][o[2]], b4 = B[r][o[2]];
    if (!(b1 <= b2 && b2 <= b3 && b3 <= b4)) continue;
    const int cfg = 1 + (X.F[b1] - X.F[1]) + (X.F[nb2 + b2] - X.F[nb2 + b1]) +
                    (X.F[2 * nb2 + b3] - X.F[2 * nb2 + b2]) + (X.F[3 * nb2 + b4] - X.F[3 * nb2 + b3]);
    const int d1 = B[r][o[1]], d2 = B[o[0]][o[2]];
    const int kk = (cfg - 1) + X.ncfg * ((d1 - 1) + X.nbins * (d2 - 1));
    atomicAdd(&X.cnt[kk + X.nbin * nr], 1ull);
    if (WEIGHTED)
      fix_add(&X.fix[kk + X.nbin * nr], &X.fix[kk + X.nbin * (nr + 5)],
              ((w[r] * w[o[0]]) * w[o[1]]) * w[o[2]], X.fscale);
    const int role[4] = {r, o[0], o[1], o[2]};
#pragma unroll
    for (int tt = 0; tt < 6; ++tt) {
      if (!rnd[role[kGate[tt]]]) continue;
      const int u = role[kPu[tt]], vv = role[kPv[tt]];
      const int npr = (int)rnd[u] + (int)rnd[vv];
      const int kt = kk + X.nbin * tt;
      const double q = WEIGHTED ? w[u] * w[vv] : 0.0;
      atomicAdd(&X.dcnt[kt + X.nbin * 6 * npr], 1ull);
      if (WEIGHTED)
        fix_add(&X.dfix[kt + X.nbin * 6 * npr], &X.dfix[kt + X.nbin * (6 * npr + 24)], q, X.dscale);
      if (npr == 2) {
        atomicAdd(&X.dcnt[kt + X.nbin * 18], 1ull);
        if (WEIGHTED) fix_add(&X.dfix[kt + X.nbin * 18], &X.dfix[kt + X.nbin * 42], q, X.dscale);
      }
    }
    n++;
  }
  return n;
}

template <bool WEIGHTED>
__global__ void __launch_bounds__(kQuadThreads) quad4_kernel(DevCatalog C, CSRView G, QuadParams Q,
                                                             unsigned long long* __restrict__ g_cnt,
                                                             unsigned long long* __restrict__ g_fix,
                                                             unsigned long long* __restrict__ d_cnt,
                                                             unsigned long long* __restrict__ d_fix,
                                                             double fscale, double dscale,
                                                             unsigned long long* __restrict__ stats) {
  extern __shared__ __align__(16) unsigned char smem[];
  const QuadLayout L = quad_layout(Q.nbins, Q.cap);
  int* s_F = reinterpret_cast<int*>(smem + L.off_rank);
  const int nb2 = Q.nbins + 2;
  for (int k = threadIdx.x; k < 4 * nb2; k += blockDim.x) s_F[k] = Q.rank.F[k / nb2][k % nb2];
  __syncthreads();
  QuadCtx X;
  X.F = s_F;
  X.nbins = Q.nbins;
  X.ncfg = Q.ncfg;
  X.nbin = Q.ncfg * Q.nbins * Q.nbins;
  X.tetra = Q.tetra;
  X.cnt = g_cnt;
  X.fix = g_fix;
  X.dcnt = d_cnt;
  X.dfix = d_fix;
  X.fscale = fscale;
  X.dscale = dscale;

  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const int wib = threadIdx.x >> 5;
  unsigned char* wb = smem + L.off_warp + L.warp_bytes * wib;
  const int cap = Q.cap;
  long long* r_start = reinterpret_cast<long long*>(wb);
  long long* x_start = reinterpret_cast<long long*>(wb + (size_t)cap * 8);
  int* r_col = reinterpret_cast<int*>(wb + (size_t)cap * 16);
  uint32_t* r_meta = reinterpret_cast<uint32_t*>(wb + (size_t)cap * 20);
  int* r_len = reinterpret_cast<int*>(wb + (size_t)cap * 24);
  int* x_c = reinterpret_cast<int*>(wb + (size_t)cap * 28);
  int* x_y = reinterpret_cast<int*>(wb + (size_t)cap * 32);
  uint32_t* x_m = reinterpret_cast<uint32_t*>(wb + (size_t)cap * 36);
  int* x_pre = reinterpret_cast<int*>(wb + (size_t)cap * 40);

  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  unsigned long long quads = 0, rooted = 0, probes = 0;

  for (int p = warp; p < C.n; p += nwarps) {
    const int64_t b0 = G.start[p];
    const int k = G.len[p];
    if (k < 3 || k > cap) continue;  // rows longer than cap are rejected on the host
    __syncwarp();
    for (int x = lane; x < k; x += 32) {
      const unsigned long long rr = G.rec[b0 + x];
      int a = rec_col(rr);
      r_col[x] = a;
      r_meta[x] = rec_meta(rr);
      r_start[x] = G.start[a];
      r_len[x] = G.len[a];
    }
    __syncwarp();
    for (int x = 0; x < k - 2; ++x) {
      const int a = r_col[x];
      const int64_t ra = r_start[x];
      const int ka = r_len[x];
      // X = R+(a) ∩ R+(p), entries beyond position x of R+(p)
      int nx = 0;
      for (int j0 = 0; j0 < ka; j0 += 32) {
        int j = j0 + lane;
        bool found = false;
        int c = 0, y = 0;
        unsigned long long rr = 0;
        if (j < ka) {
          rr = G.rec[ra + j];
          c = rec_col(rr);
          y = x + 1 + qlower_bound(r_col + x + 1, k - x - 1, c);
          found = y < k && r_col[y] == c;
        }
        unsigned msk = __ballot_sync(0xffffffffu, found);
        if (found) {
          int pos = nx + __popc(msk & lt);
          x_c[pos] = c;
          x_y[pos] = y;
          x_m[pos] = rec_meta(rr);
          x_start[pos] = G.start[c];
        }
        nx += __popc(msk);
      }
      if (lane == 0) probes += (unsigned long long)ka;
      __syncwarp();
      if (nx < 2) continue;
      // prefix over |R+(b)| for b in X
      int carry = 0;
      for (int zb = 0; zb < nx; zb += 32) {
        int z = zb + lane;
        int len = 0;
        if (z < nx) len = G.len[x_c[z]];
        int incl = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          int yy = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += yy;
        }
        if (z < nx) x_pre[z + 1] = carry + incl;
        carry += __shfl_sync(0xffffffffu, incl, 31);
      }
      if (lane == 0) x_pre[0] = 0;
      __syncwarp();
      const int W = carry;
      if (lane == 0) probes += (unsigned long long)W;
      for (int base = 0; base < W; base += 32) {
        const int f = base + lane;
        if (f >= W) break;
        int lo = 0, hi = nx - 1;
        while (lo < hi) {
          int mid = (lo + hi + 1) >> 1;
          if (x_pre[mid] <= f)
            lo = mid;
          else
            hi = mid - 1;
        }
        const int z = lo;
        const int64_t e = x_start[z] + (f - x_pre[z]);
        const unsigned long long rr = G.rec[e];
        const int d = rec_col(rr);
        const int z2 = z + 1 + qlower_bound(x_c + z + 1, nx - z - 1, d);
        if (z2 < nx && x_c[z2] == d) {
          const int v[4] = {p, a, x_c[z], d};
          const uint32_t m[6] = {r_meta[x], r_meta[x_y[z]], r_meta[x_y[z2]],
                                 x_m[z],    x_m[z2],        rec_meta(rr)};
          int nroot = X.tetra ? tetra_contrib<WEIGHTED>(C, X, v, m)
                              : quad_contrib<WEIGHTED>(C, G, X, v, m);
          quads += nroot > 0;
          rooted += nroot;
        }
      }
      __syncwarp();
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
}

}  // namespace

void launch_quad4(const DevCatalog& C, const CSRView& G, const QuadParams& Q, bool weighted,
                  unsigned long long* g_cnt, unsigned long long* g_fix, unsigned long long* d_cnt,
                  unsigned long long* d_fix, double fscale, double dscale,
                  unsigned long long* stats, cudaStream_t s) {
  if (C.n <= 0) return;
  QuadLayout L = quad_layout(Q.nbins, Q.cap);
  size_t smem = L.total;
#define GR_QUAD_LAUNCH(W)                                                                     \
  do {                                                                                        \
    auto kfn = quad4_kernel<W>;                                                               \
    GR_CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize,        \
                                     (int)smem));                                             \
    int per_sm = 0;                                                                           \
    GR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, kQuadThreads, smem)); \
    if (per_sm < 1) per_sm = 1;                                                               \
    int64_t blocks = (int64_t)per_sm * 148;                                                   \
    int64_t need = ((int64_t)C.n + kQuadWarps - 1) / kQuadWarps;                              \
    if (blocks > need) blocks = need;                                                         \
    kfn<<<(unsigned)blocks, kQuadThreads, smem, s>>>(C, G, Q, g_cnt, g_fix, d_cnt, d_fix, fscale, dscale, stats); \
  } while (0)
  if (weighted) GR_QUAD_LAUNCH(true); else GR_QUAD_LAUNCH(false);
#undef GR_QUAD_LAUNCH
  GR_CHECK_LAUNCH();
}

size_t quad4_smem_bytes(int nbins, int cap) { return quad_layout(nbins, cap).total; }

}  // namespace gr
