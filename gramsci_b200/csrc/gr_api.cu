// C ABI of libgramsci_cuda.so (include/gramsci_cuda.h): context, catalogue
// and binning state, and the count entry points that chain the cell index,
// the CSR build and the counting kernels.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <map>
#include <mutex>
#include <new>
#include <sys/stat.h>
#include <string>
#include <vector>

#include "../../include/gramsci_cuda.h"
#include "gr_batch.cuh"

using namespace gr;

// The speculative rebuild of the last configuration (index and graph
// phases) as two instantiated CUDA graphs, replayed by the next 3PCF count
// whose configuration is the same: every pointer, capacity and size the two
// phases read, the binning and the previous bounding box (`key`).  A replay
// launches the phases' 18 kernels and copies at once instead of one host
// launch each.
struct SpecGraph {
  std::vector<unsigned long long> key;
  cudaGraphExec_t idx = nullptr, csr = nullptr;
  void release() {
    if (idx) cudaGraphExecDestroy(idx);
    if (csr) cudaGraphExecDestroy(csr);
    idx = csr = nullptr;
    key.clear();
  }
  ~SpecGraph() { release(); }
};

struct gr_ctx {
  int device = 0;
  cudaStream_t own = nullptr;
  cudaStream_t user = nullptr;
  std::string err;
  // catalogue, catalogue order
  DevBuf<double> xyz, w;
  DevBuf<int> buffer;
  bool has_buffer = false;
  bool cat_set = false;
  int64_t n = 0, n_data = 0, n_rand = 0;
  bool uniform = false;
  double w_gal = 0.0, w_ran = 0.0;
  // binning
  bool bins_set = false;
  double rmin = 0, rmax = 0;
  int nbins = 0, nmu = 1, logbins = 0;
  int precision = 0;
  int autotune = 1;
  int last_variant = 0;
  int64_t timeout_ms = 1000;
  // derived state
  CellIndex index;
  UpperCSR csr;
  bool csr_valid = false;
  int clique_mode = 0;  // GR_OPT_CLIQUE_MODE
  // speculative rebuilds (count_tri): catalogue generation (set_catalog),
  // generation of the last verified build, and whether speculating on a new
  // catalogue is still worth it (off after it once found a changed grid)
  uint64_t cat_gen = 0, spec_gen = ~0ull;
  bool spec_new_ok = true;
  bool keep_graph = false;    // GR_OPT_KEEP_GRAPH
  bool graph_loaded = false;  // graph read by gr_graph_load
  PairParams P{};
  DevBuf<uint8_t> normal_dev;
  int normal_nmu = 0;                     // nmu of the table in normal_dev (0: none)
  DevBuf<unsigned long long> hcnt, dcnt, stats;
  DevBuf<unsigned long long> hfix, dfix;  // fixed-point sums (lo words, then hi words)
  double wmax = 0.0;                      // max |w| over the catalogue
  double wgmax = 0.0, wrmax = 0.0;        // max |w| over galaxies / randoms
  DevBuf<unsigned char> uniform_flag;
  DevBuf<int> work;
  HostBuf<unsigned long long> stage;     // pinned read-back of a call's results
  DevBuf<double> hval;                   // fixed-point sums converted on the device
  DevBuf<int> qorder;                    // 4-clique root order (n) + its class counts
  SpecGraph spec_graph;                  // captured speculative rebuild (count_tri)
  SpecGraph spec_index;                  // captured speculative index (gr_count_2pcf)
  DevBuf<double> cot, grad;              // adjoint inputs / output
  DevBuf<unsigned long long> gfix;       // adjoint fixed-point gradients (lo[n], hi[n])
  // batched regions: 0 none, 1 nsplit^3 subcubes, 2 region ids, 3 mocks
  int region_mode = 0;
  int nsplit = 0;
  RegionLayout regions;
  DevBuf<unsigned long long> bcnt, bfix, bstats;
  DevBuf<unsigned long long> rcnt, rfix;  // per-region histograms
  DevBuf<int> bwork;
  bool batch_weighted = false;
  int batch_variant = 0;
  double batch_fscale = 1.0;
  cudaEvent_t bev[2] = {nullptr, nullptr};
  gr_stats st{};
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // [4]: query start

  cudaStream_t stream() const { return user ? user : own; }
};

namespace gr {

// ---------------------------------------------------------------- params ----
void make_pair_params(PairParams& P, double rmin, double rmax, int nbins, int nmu, int logbins,
                      double X, int force_fp64) {
  std::memset(&P, 0, sizeof(P));
  P.rmin = rmin;
  P.rmax = rmax;
  P.rmin2 = rmin * rmin;
  P.rmax2 = rmax * rmax;
  P.nbins = nbins;
  P.nmu = nmu;
  P.logbins = logbins;
  P.rsd = nmu >= 2;
  if (logbins) {
    P.inv_dr = 1.0 / ((std::log10(rmax) - std::log10(rmin)) / (double)nbins);
    P.log_rmin = std::log10(rmin);
  } else {
    P.inv_dr = 1.0 / ((rmax - rmin) / (double)nbins);
    P.log_rmin = 0.0;
  }
  P.mu_scale = (double)(0.5f * (float)nmu);
  // FP32 fast path: error bounds for coordinates rounded to float.
  //   coordinate error            <= X u            (u = 2^-24)
  //   separation component error  <= e1 = 2 X u + R u
  //   |d_f - d|                   <= sqrt(3) e1 + 8 u R
  // The 8 u R covers the squared separation (three roundings, 1.5 u R on d)
  // and a square root taken as d2 * rsqrtf(d2) (2 ulp = 4 u, plus u for the
  // product), so kernels may use either that or the rounded square root.
  // Doubled for safety.
  const double u = std::ldexp(1.0, -24);
  const double R = rmax * 1.01 + 1e-30;
  const double e1 = 2.0 * X * u + R * u;
  const double d0 = 2.0 * (std::sqrt(3.0) * e1 + 8.0 * u * R);
  P.d0 = (float)(d0 * (1.0 + 1e-6));
  double hi = rmax + 2.0 * d0;
  hi = hi * hi * (1.0 + 16.0 * u);
  P.rmax2_hi = std::nextafter((float)hi, std::numeric_limits<float>::infinity());
  double lo = rmin - 2.0 * d0;
  if (lo > 0.0) {
    lo = lo * lo * (1.0 - 16.0 * u);
    P.rmin2_lo = std::nextafter((float)lo, -std::numeric_limits<float>::infinity());
  } else {
    P.rmin2_lo = -1.0f;
  }
  // inner bounds of the certain-edge band for the membership-only test
  double in_hi = rmax - 2.0 * d0;
  if (in_hi > 0.0) {
    in_hi = in_hi * in_hi * (1.0 - 16.0 * u);
    P.rmax2_lo = std::nextafter((float)in_hi, -std::numeric_limits<float>::infinity());
  } else {
    P.rmax2_lo = -1.0f;
  }
  double in_lo = rmin + 2.0 * d0;
  in_lo = in_lo * in_lo * (1.0 + 16.0 * u);
  P.rmin2_hi = std::nextafter((float)in_lo, std::numeric_limits<float>::infinity());
  P.f_rmin = (float)rmin;
  P.f_inv_dr = (float)P.inv_dr;
  P.f_mu_scale = (float)P.mu_scale;
  P.f_nmu = (float)nmu;
  const double tmax = nbins + 1.0;
  double tg = (d0 + u * std::fabs(rmin) + u * R) * P.inv_dr + 4.0 * u * tmax;
  tg = 2.0 * tg + 1e-9 * tmax;
  P.tguard = (float)tg;
  // line-of-sight cosine: (pi/2)(|ds|/|s| + |dm|/|m|) + arithmetic, doubled.
  // The arithmetic term eC = 128 u covers the cosine evaluated with
  // approximate square roots and division (about 21 u: dot product 3 u,
  // |m| and d 6.5 u each, product u, __fdividef 4 u) with a margin of six.
  const double pi = 3.14159265358979323846;
  P.eA = (float)(pi * std::sqrt(3.0) * e1);
  P.mB = (float)(8.0 * X * u + 1e-30);
  P.eB = (float)(pi * 2.0 * std::sqrt(3.0) * X * u);
  P.eC = (float)(128.0 * u);
  P.f32 = (!force_fp64 && !logbins && std::isfinite(tg) && tg < 0.05 && std::isfinite(X)) ? 1 : 0;
}

static int64_t multiset(int64_t m, int r) {
  if (r == 0) return 1;
  if (m <= 0) return 0;
  int64_t num = 1, den = 1;
  for (int i = 0; i < r; ++i) {
    num *= (m + i);
    den *= (i + 1);
  }
  return num / den;
}

void make_rank_tables(RankTables& T, int n, int k) {
  std::memset(&T, 0, sizeof(T));
  T.n = n;
  T.k = k;
  for (int j = 0; j < k; ++j) {
    int r = k - j - 1;
    T.F[j][0] = 0;
    T.F[j][1] = 0;
    for (int v = 1; v <= n; ++v) T.F[j][v + 1] = T.F[j][v] + (int)multiset(n - v + 1, r);
  }
}

double fix_scale(double pmax) {
  // 4 * pmax * scale <= 2^62, so a sum of up to four products fits in 63 bits
  if (!(pmax > 0.0) || !std::isfinite(pmax)) return 1.0;
  int e;
  std::frexp(pmax * (1.0 + 1e-9), &e);  // pmax < 2^e
  return std::ldexp(1.0, 60 - e);
}

double fix_value(unsigned long long lo, unsigned long long hi, double scale) {
  // scale is a power of two: one rounding in the conversion, none after it
  return i128_to_double(lo, hi) / scale;
}

double fix_split_value(unsigned long long lo, unsigned long long hi, double scale) {
  // hi * 2^32 + lo as a signed 128-bit integer (exact), then one rounding
  const __int128 v = ((__int128)(long long)hi << 32) + (__int128)lo;
  const unsigned __int128 u = (unsigned __int128)v;
  return i128_to_double((unsigned long long)u, (unsigned long long)(u >> 64)) / scale;
}

}  // namespace gr

namespace {

// find_normal (src/gramsci.F90:1611-1625) for every (mu1, mu2): single
// precision, operations in source order, no contraction.  A negative
// radicand gives NaN and bin 1.
void normal_table(int nmu, std::vector<uint8_t>& out) {
  out.assign((size_t)nmu * nmu, 1);
  const double mu_scale = (double)(0.5f * (float)nmu);
  for (int b = 1; b <= nmu; ++b)
    for (int a = 1; a <= nmu; ++a) {
      volatile float m1 = (float)((double)((float)a - 0.5f) / mu_scale - 1.0);
      volatile float m2 = (float)((double)((float)b - 0.5f) / mu_scale - 1.0);
      volatile float t1 = m1 * m1;
      volatile float s1 = 0.75f - t1;
      volatile float t2 = m2 * m2;
      volatile float s2 = s1 - t2;
      volatile float t3 = m1 * m2;
      volatile float r = s2 + t3;
      volatile float sq = std::sqrt((float)r);
      volatile float v = 1.1547f * sq;
      volatile float v2 = v * (float)nmu;
      int m = 1;
      if (v2 == v2) {
        float f = std::floor((float)v2);
        m = (int)f + 1;
        if (m < 1) m = 1;
        if (m > nmu) m = nmu;
      }
      out[(size_t)(a - 1) + (size_t)nmu * (b - 1)] = (uint8_t)m;
    }
}

// The find_normal table of nmu on the device, uploaded when nmu changes.
static void ensure_normal(gr_ctx* c, int nmu, cudaStream_t s) {
  if (c->normal_nmu == nmu && c->normal_dev.p) return;
  std::vector<uint8_t> nt;
  normal_table(nmu, nt);
  c->normal_dev.reserve(nt.size());
  GR_CUDA_TRY(cudaMemcpyAsync(c->normal_dev.p, nt.data(), nt.size(), cudaMemcpyHostToDevice, s));
  GR_CUDA_TRY(cudaStreamSynchronize(s));  // nt is pageable and goes out of scope
  c->normal_nmu = nmu;
}

// ------------------------------------------------------------------ autotune --
// Kernel variant per workload class, chosen by timing the variants on the
// first workload of that class and cached in a JSON file
// ($GRAMSCI_AUTOTUNE, default ~/.cache/gramsci_b200/autotune.json; an
// unwritable path keeps the cache in memory).  The choice only affects
// speed: every variant produces identical results.
struct Tuner {
  std::mutex mu;
  bool loaded = false;
  std::map<std::string, int> choice;
  std::string path() const {
    const char* e = std::getenv("GRAMSCI_AUTOTUNE");
    if (e && e[0]) return e;
    const char* h = std::getenv("HOME");
    return std::string(h ? h : "/tmp") + "/.cache/gramsci_b200/autotune.json";
  }
  void load() {
    if (loaded) return;
    loaded = true;
    std::ifstream f(path());
    std::string line;
    while (std::getline(f, line)) {
      const size_t a = line.find('"'), b = line.find('"', a + 1), c = line.find(':', b);
      if (a == std::string::npos || b == std::string::npos || c == std::string::npos) continue;
      choice[line.substr(a + 1, b - a - 1)] = std::atoi(line.c_str() + c + 1);
    }
  }
  void save() {
    const std::string p = path();
    const size_t slash = p.rfind('/');
    if (slash != std::string::npos) {
      std::string dir = p.substr(0, slash);
      for (size_t k = 1; k <= dir.size(); ++k)
        if (k == dir.size() || dir[k] == '/') mkdir(dir.substr(0, k).c_str(), 0755);
    }
    std::ofstream f(p);
    if (!f) return;
    f << "{\n";
    size_t i = 0;
    for (const auto& kv : choice) f << "  \"" << kv.first << "\": " << kv.second << (++i < choice.size() ? ",\n" : "\n");
    f << "}\n";
  }
};

Tuner& tuner() {
  static Tuner t;
  return t;
}

int set_err(gr_ctx* c, int code, const std::string& m) {
  if (c) c->err = m;
  return code;
}

#define GR_API_BEGIN(ctx)                          \
  if (!(ctx)) return GR_E_ARG;                     \
  try {                                            \
    GR_CUDA_TRY(cudaSetDevice((ctx)->device));

#define GR_API_END(ctx)                            \
  }                                                \
  catch (const gr::Error& e) {                     \
    return set_err((ctx), e.code, e.msg);          \
  }                                                \
  catch (const std::bad_alloc&) {                  \
    return set_err((ctx), GR_E_CAPACITY, "host allocation failed"); \
  }                                                \
  catch (...) {                                    \
    return set_err((ctx), GR_E_CUDA, "unknown error"); \
  }                                                \
  return GR_OK;

// The 128-bit fixed-point sums of a histogram in FP64, on the device: value
// k of (lo[k], hi[k]) times inv_scale[k / per] (inverses of powers of two,
// so one rounding, as the host's fix_value).  split: (lo, hi) are the split
// limbs of fix_red, worth hi * 2^32 + lo (fix_split_value).  The host then
// reads n doubles instead of 2n words and converts nothing.
__global__ void fix_convert_kernel(const unsigned long long* __restrict__ lo,
                                   const unsigned long long* __restrict__ hi, int64_t n,
                                   int64_t per, double4 inv_scale, int split, int stride,
                                   double* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = i / per;
    const double is = c == 0 ? inv_scale.x : (c == 1 ? inv_scale.y : (c == 2 ? inv_scale.z : inv_scale.w));
    unsigned long long l = lo[i * stride], h = hi[i * stride];
    if (split) {
      // (signed h) << 32 as 128 bits, plus l
      const long long hs = (long long)h;
      const unsigned long long L = (unsigned long long)hs << 32;
      unsigned long long H = (unsigned long long)(hs >> 32);
      const unsigned long long L2 = L + l;
      H += L2 < L ? 1ull : 0ull;
      l = L2;
      h = H;
    }
    out[i] = fix_to_double(l, h, is);
  }
}

// Queue fix_convert_kernel: n values from (lo, lo + hi_off) entries of
// `stride` words each, categories of `per` values with scales sc[0..3].
static void enqueue_fix_convert(const unsigned long long* lo, int64_t hi_off, int64_t n,
                                int64_t per, const double sc[4], bool split, double* out,
                                cudaStream_t s, int stride = 1) {
  if (n <= 0) return;
  const double4 inv = make_double4(1.0 / sc[0], 1.0 / sc[1], 1.0 / sc[2], 1.0 / sc[3]);
  const int blocks = (int)std::min<int64_t>((n + 255) / 256, 2 * (int64_t)sm_count());
  fix_convert_kernel<<<blocks, 256, 0, s>>>(lo, lo + hi_off * stride, n, per, inv, split ? 1 : 0,
                                            stride, out);
  GR_CHECK_LAUNCH();
}

// Clears *flag unless all galaxy weights are equal and all random weights are
// equal; writes max |w| over galaxies to wmax[0] and over randoms to wmax[1]
// (as the bits of non-negative doubles) and sets *nonfinite when a weight is
// not finite (tested directly, not through the maxima).  Reduced per block
// first, so each block makes at most four global updates.
__global__ void uniform_check_kernel(const double* __restrict__ w, int64_t n_data, int64_t n,
                                     unsigned char* flag, unsigned long long* wmax,
                                     int* nonfinite) {
  __shared__ unsigned long long s_mg[32], s_mr[32];
  __shared__ int s_bad[32];
  unsigned long long mg = 0, mr = 0;
  bool bad = false, nf = false;
  const double refg = n_data > 0 ? w[0] : 0.0;
  const double refr = n > n_data ? w[n_data] : 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double v = w[i];
    nf = nf || !isfinite(v);
    const double ref = i < n_data ? refg : refr;
    bad = bad || __double_as_longlong(v) != __double_as_longlong(ref);
    const unsigned long long a = (unsigned long long)__double_as_longlong(fabs(v));
    if (i < n_data) mg = a > mg ? a : mg;
    else mr = a > mr ? a : mr;
  }
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long u = __shfl_xor_sync(0xffffffffu, mg, o);
    mg = u > mg ? u : mg;
    u = __shfl_xor_sync(0xffffffffu, mr, o);
    mr = u > mr ? u : mr;
  }
  bad = __any_sync(0xffffffffu, bad);
  if (__any_sync(0xffffffffu, nf) && (threadIdx.x & 31) == 0) atomicOr(nonfinite, 1);
  const int wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    s_mg[wid] = mg;
    s_mr[wid] = mr;
    s_bad[wid] = bad ? 1 : 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int b = 0;
    for (int k = 0; k < nw; ++k) {
      mg = s_mg[k] > mg ? s_mg[k] : mg;
      mr = s_mr[k] > mr ? s_mr[k] : mr;
      b |= s_bad[k];
    }
    if (mg) atomicMax(&wmax[0], mg);
    if (mr) atomicMax(&wmax[1], mr);
    if (b) *flag = 0;
  }
}

unsigned long long mix_host(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// 64-bit fingerprint of the coordinates in catalogue order: a wrapping sum
// of a mixed hash of (index, x, y, z), so the order of the additions does
// not matter.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  // splitmix64 finaliser
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__global__ void fingerprint_kernel(const double* __restrict__ xyz, int64_t n,
                                   unsigned long long* out) {
  unsigned long long acc = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    unsigned long long h = mix64((unsigned long long)i + 0x9e3779b97f4a7c15ull);
    for (int c = 0; c < 3; ++c)
      h = mix64(h ^ (unsigned long long)__double_as_longlong(xyz[3 * i + c]));
    acc += h;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

void require_ready(gr_ctx* c) {
  if (!c->cat_set) throw gr::Error{GR_E_ARG, "catalogue not set (gr_set_catalog)"};
  if (!c->bins_set) throw gr::Error{GR_E_ARG, "bins not set (gr_set_bins)"};
}

void ensure_events(gr_ctx* c) {
  for (int k = 0; k < 5; ++k)
    if (!c->ev[k]) GR_CUDA_TRY(cudaEventCreate(&c->ev[k]));
}

float ev_ms(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

// Index build + pair parameters (shared by every query).
// speculate: see CellIndex / UpperCSR; the caller checks the flags
// sub: cell grid of the index (1: cells at least rmax wide, 2: rmax/2,
// 0: chosen by density, see CellIndex::build)
void build_index(gr_ctx* c, bool speculate = false, int sub = 1) {
  cudaStream_t s = c->stream();
  c->index.build(c->xyz.p, c->w.p, c->has_buffer ? c->buffer.p : nullptr, c->n, c->n_data, c->rmax, s,
                 speculate, sub, kDenseCellPoints);
  make_pair_params(c->P, c->rmin, c->rmax, c->nbins, c->nmu, c->logbins, c->index.coord_max,
                   c->precision == 1);
  c->csr_valid = false;
}

void build_csr(gr_ctx* c, bool speculate = false) {
  c->csr.build(c->index.view(), c->P, c->stream(), speculate);
  c->csr_valid = !speculate;  // a speculative graph is valid once settled
}

// The index and graph of the last call (or of gr_graph_load) are current and
// may be reused by this call.
bool reuse_graph(const gr_ctx* c) { return c->csr_valid && (c->keep_graph || c->graph_loaded); }

int round_cap(int64_t maxdeg, int lo, int hi) {
  int64_t c = ((maxdeg + 31) / 32) * 32;
  if (c < lo) c = lo;
  if (c > hi) c = hi;
  return (int)c;
}

// product of `ng` galaxy weights and `nr` random weights, left to right
double uniform_product(double wg, double wr, int ng, int nr) {
  double p = 1.0;
  bool first = true;
  for (int k = 0; k < ng; ++k) {
    p = first ? wg : p * wg;
    first = false;
  }
  for (int k = 0; k < nr; ++k) {
    p = first ? wr : p * wr;
    first = false;
  }
  return p;
}

}  // namespace

// Everything the speculative index and graph phases read from the host:
// the catalogue's device pointers and sizes, the binning and precision, the
// previous bounding box, and every buffer's address and capacity.
static std::vector<unsigned long long> spec_key(const gr_ctx* c) {
  std::vector<unsigned long long> k;
  auto add = [&](auto v) {
    unsigned long long u = 0;
    std::memcpy(&u, &v, std::min(sizeof(v), sizeof(u)));
    k.push_back(u);
  };
  auto buf = [&](const auto& b) {
    add(b.p);
    add(b.n);
  };
  add(c->xyz.p);
  add(c->w.p);
  add(c->has_buffer ? c->buffer.p : nullptr);
  add(c->n);
  add(c->n_data);
  add(c->rmin);
  add(c->rmax);
  add(c->nbins);
  add(c->nmu);
  add(c->logbins);
  add(c->precision);
  const CellIndex& I = c->index;
  add(I.have_prev);
  add(I.prev_n);
  add(I.prev_rmax);
  add(I.prev_sub);
  for (int i = 0; i < 7; ++i) add(I.prev_raw[i]);
  buf(I.bbox_raw);
  buf(I.bbox_prev);
  buf(I.cell_count);
  buf(I.key_orig);
  buf(I.slot);
  buf(I.tmp_perm);
  buf(I.cell_start);
  buf(I.orig);
  buf(I.cell_key);
  buf(I.cell_start64);
  buf(I.scan_tmp);
  buf(I.pos4);
  buf(I.posd);
  buf(I.w);
  buf(I.flags);
  const UpperCSR& G = c->csr;
  buf(G.deg_up);
  buf(G.deg_full);
  buf(G.work);
  buf(G.scan_tmp);
  buf(G.rstart);
  buf(G.cbound);
  buf(G.cbase);
  buf(G.scratch);
  buf(G.stats);
  buf(G.ctl);
  return k;
}

// Capture the speculative index and graph phases of the current
// configuration (the call has just run them with success) on the context's
// own stream.  A capture that fails leaves no graph: the next call runs the
// phases eagerly.
static std::vector<unsigned long long> spec_key(const gr_ctx* c, int sub, bool with_csr) {
  std::vector<unsigned long long> k = spec_key(c);
  k.push_back((unsigned long long)sub);
  k.push_back(with_csr ? 1ull : 0ull);
  return k;
}

// Capture the speculative index phase (grid choice `sub`) and, with_csr, the
// graph phase of the current configuration into G (the call has just run
// them with success) on the context's own stream.  A capture that fails
// leaves no graph: the next call runs the phases eagerly.
static void capture_spec_graph(gr_ctx* c, SpecGraph& G, int sub, bool with_csr) {
  G.release();
  // the configuration as this call leaves it (a successful speculative build
  // changes none of it; buffers it grew have their new addresses)
  const std::vector<unsigned long long> key = spec_key(c, sub, with_csr);
  cudaStream_t user = c->user;
  c->user = nullptr;  // build_index / build_csr enqueue on c->stream()
  cudaStream_t s = c->own;
  cudaGraph_t g[2] = {nullptr, nullptr};
  cudaGraphExec_t e[2] = {nullptr, nullptr};
  bool ok = true;
  const int phases = with_csr ? 2 : 1;
  for (int phase = 0; phase < phases && ok; ++phase) {
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      ok = false;
      break;
    }
    try {
      if (phase == 0)
        build_index(c, true, sub);
      else
        build_csr(c, true);
    } catch (...) {
      ok = false;
    }
    if (cudaStreamEndCapture(s, &g[phase]) != cudaSuccess || !g[phase]) ok = false;
    if (ok && cudaGraphInstantiate(&e[phase], g[phase], 0) != cudaSuccess) ok = false;
  }
  for (int k = 0; k < 2; ++k)
    if (g[k]) cudaGraphDestroy(g[k]);
  c->user = user;
  cudaGetLastError();  // a failed capture leaves nothing behind
  if (!ok || !c->index.speculated || spec_key(c, sub, with_csr) != key) {
    for (int k = 0; k < 2; ++k)
      if (e[k]) cudaGraphExecDestroy(e[k]);
    return;
  }
  G.idx = e[0];
  G.csr = e[1];
  G.key = key;
}

extern "C" {

const char* gr_version(void) { return "gramsci_b200 0.1 (sm_100a)"; }

int gr_create(gr_ctx** out, int device) {
  if (!out) return GR_E_ARG;
  *out = nullptr;
  gr_ctx* c = nullptr;
  try {
    c = new gr_ctx();
    c->device = device;
    GR_CUDA_TRY(cudaSetDevice(device));
    GR_CUDA_TRY(cudaStreamCreateWithFlags(&c->own, cudaStreamNonBlocking));
  } catch (const gr::Error& e) {
    delete c;
    return e.code;
  } catch (...) {
    delete c;
    return GR_E_CAPACITY;
  }
  *out = c;
  return GR_OK;
}

int gr_destroy(gr_ctx* c) {
  if (!c) return GR_E_ARG;
  cudaSetDevice(c->device);
  if (c->own) cudaStreamSynchronize(c->own);
  for (int k = 0; k < 5; ++k)
    if (c->ev[k]) cudaEventDestroy(c->ev[k]);
  for (int k = 0; k < 2; ++k)
    if (c->bev[k]) cudaEventDestroy(c->bev[k]);
  c->regions.release_graph();
  c->spec_graph.release();
  c->spec_index.release();
  if (c->own) cudaStreamDestroy(c->own);
  delete c;
  return GR_OK;
}

const char* gr_last_error(const gr_ctx* c) { return c ? c->err.c_str() : "null context"; }

int gr_set_stream(gr_ctx* c, void* stream) {
  GR_API_BEGIN(c)
  c->user = reinterpret_cast<cudaStream_t>(stream);
  GR_API_END(c)
}

static int set_catalog_impl(gr_ctx* c, const double* xyz, const double* w, const int32_t* buffer,
                            int64_t n_data, int64_t n_rand, cudaMemcpyKind kind) {
  GR_API_BEGIN(c)
  if (n_data < 0 || n_rand < 0) return set_err(c, GR_E_ARG, "negative catalogue size");
  int64_t n = n_data + n_rand;
  if (n >= (int64_t)1 << 31) return set_err(c, GR_E_CAPACITY, "catalogue larger than 2^31-1 points");
  if (n > 0 && (!xyz || !w)) return set_err(c, GR_E_ARG, "null xyz or w");
  cudaStream_t s = c->stream();
  c->cat_gen++;
  c->xyz.reserve(3 * n + 1);
  c->w.reserve(n + 1);
  if (n > 0) {
    GR_CUDA_TRY(cudaMemcpyAsync(c->xyz.p, xyz, sizeof(double) * 3 * n, kind, s));
    GR_CUDA_TRY(cudaMemcpyAsync(c->w.p, w, sizeof(double) * n, kind, s));
  }
  c->has_buffer = buffer != nullptr;
  if (buffer) {
    c->buffer.reserve(n + 1);
    GR_CUDA_TRY(cudaMemcpyAsync(c->buffer.p, buffer, sizeof(int32_t) * n, kind, s));
  }
  c->n = n;
  c->n_data = n_data;
  c->n_rand = n_rand;
  // Uniform weights (all galaxies equal, all randoms equal) let the kernels
  // keep integer counts only; sums are then count x product.
  // [0] uniform flag, [4] non-finite weight flag (int), [8] max |w| galaxies,
  // [16] max |w| randoms, [24] fingerprint
  c->uniform_flag.reserve(32);
  // pinned stage: [0..3) the 24 bytes below, [3] first galaxy weight,
  // [4] first random weight
  c->stage.reserve(8);
  unsigned char* init = reinterpret_cast<unsigned char*>(c->stage.p);
  std::memset(init, 0, 24);
  init[0] = 1;
  GR_CUDA_TRY(cudaMemcpyAsync(c->uniform_flag.p, init, 24, cudaMemcpyHostToDevice, s));
  unsigned long long* d_wmax = reinterpret_cast<unsigned long long*>(c->uniform_flag.p + 8);
  if (n > 0) {
    int blocks = (int)std::min<int64_t>((n + 255) / 256, (int64_t)2 * sm_count());
    uniform_check_kernel<<<blocks, 256, 0, s>>>(c->w.p, n_data, n, c->uniform_flag.p, d_wmax,
                                                reinterpret_cast<int*>(c->uniform_flag.p + 4));
    GR_CHECK_LAUNCH();
  }
  // the read-back lands in the stage after the upload above has read it
  unsigned char* out = reinterpret_cast<unsigned char*>(c->stage.p);
  double* wgr = reinterpret_cast<double*>(c->stage.p + 3);
  wgr[0] = 0.0;
  wgr[1] = 0.0;
  GR_CUDA_TRY(cudaMemcpyAsync(out, c->uniform_flag.p, 24, cudaMemcpyDeviceToHost, s));
  if (n_data > 0) GR_CUDA_TRY(cudaMemcpyAsync(&wgr[0], c->w.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  if (n_rand > 0)
    GR_CUDA_TRY(cudaMemcpyAsync(&wgr[1], c->w.p + n_data, sizeof(double), cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaStreamSynchronize(s));
  const double wg = wgr[0], wr = wgr[1];
  unsigned char flag = out[0];
  int nonfinite = 0;
  std::memcpy(&nonfinite, out + 4, 4);
  if (nonfinite) {
    c->cat_set = false;  // nothing may be counted on a half-set catalogue
    return set_err(c, GR_E_ARG, "non-finite weights");
  }
  std::memcpy(&c->wgmax, out + 8, 8);
  std::memcpy(&c->wrmax, out + 16, 8);
  c->wmax = std::max(c->wgmax, c->wrmax);
  if (!std::isfinite(c->wmax)) {
    c->cat_set = false;
    return set_err(c, GR_E_ARG, "non-finite weights");
  }
  c->uniform = flag != 0;
  c->w_gal = wg;
  c->w_ran = wr;
  c->cat_set = true;
  c->csr_valid = false;
  c->graph_loaded = false;
  c->regions.valid = false;
  // region ids and mocks describe the points of the previous catalogue
  if (c->region_mode >= 2) {
    c->regions.set_split();
    c->regions.release_graph();
    c->region_mode = c->nsplit > 0 ? 1 : 0;
  }
  GR_API_END(c)
}

int gr_set_catalog(gr_ctx* c, const double* xyz, const double* w, const int32_t* buffer,
                   int64_t n_data, int64_t n_rand) {
  return set_catalog_impl(c, xyz, w, buffer, n_data, n_rand, cudaMemcpyHostToDevice);
}

int gr_set_catalog_dev(gr_ctx* c, const double* xyz, const double* w, const int32_t* buffer,
                       int64_t n_data, int64_t n_rand) {
  return set_catalog_impl(c, xyz, w, buffer, n_data, n_rand, cudaMemcpyDeviceToDevice);
}

int gr_set_bins(gr_ctx* c, double rmin, double rmax, int32_t nbins, int32_t nmu, int32_t logbins) {
  GR_API_BEGIN(c)
  if (nbins < 1 || nbins > kMaxBins) return set_err(c, GR_E_ARG, "nbins must be in 1..127");
  if (nmu < 1 || nmu > kMaxBins) return set_err(c, GR_E_ARG, "nmu must be in 1..127");
  if (!(rmax > rmin) || !(rmin >= 0.0) || !std::isfinite(rmax))
    return set_err(c, GR_E_ARG, "need 0 <= rmin < rmax");
  if (logbins && !(rmin > 0.0)) return set_err(c, GR_E_ARG, "log bins need rmin > 0");
  c->rmin = rmin;
  c->rmax = rmax;
  c->nbins = nbins;
  c->nmu = nmu;
  c->logbins = logbins ? 1 : 0;
  c->bins_set = true;
  c->csr_valid = false;
  c->graph_loaded = false;
  c->regions.valid = false;
  GR_API_END(c)
}

int gr_set_option(gr_ctx* c, int32_t key, int64_t value) {
  GR_API_BEGIN(c)
  if (key == GR_OPT_PRECISION) {
    if (value != 0 && value != 1) return set_err(c, GR_E_ARG, "precision must be 0 or 1");
    if (c->precision != (int)value) {
      c->csr_valid = false;
      c->graph_loaded = false;
      c->regions.valid = false;
      c->regions.release_graph();
    }
    c->precision = (int)value;
  } else if (key == GR_OPT_KEEP_GRAPH) {
    if (value != 0 && value != 1) return set_err(c, GR_E_ARG, "keep-graph must be 0 or 1");
    c->keep_graph = value != 0;
  } else if (key == GR_OPT_AUTOTUNE) {
    if (value < 0 || value > 1 + kPairVariants) return set_err(c, GR_E_ARG, "autotune must be 0, 1 or 2+variant");
    c->autotune = (int)value;
  } else if (key == GR_OPT_CLIQUE_MODE) {
    if (value < 0 || value > 2) return set_err(c, GR_E_ARG, "clique mode must be 0, 1 or 2");
    c->clique_mode = (int)value;
  } else if (key == GR_OPT_TIMEOUT_MS) {
    if (value <= 0) return set_err(c, GR_E_ARG, "timeout must be positive");
    c->timeout_ms = value;
  } else {
    return set_err(c, GR_E_UNSUPPORTED, "unknown option");
  }
  GR_API_END(c)
}

// Two timing events destroyed on every exit path (the tuners below).
struct ScopedEvents {
  cudaEvent_t a = nullptr, b = nullptr;
  ScopedEvents() {
    GR_CUDA_TRY(cudaEventCreate(&a));
    GR_CUDA_TRY(cudaEventCreate(&b));
  }
  ~ScopedEvents() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
  ScopedEvents(const ScopedEvents&) = delete;
  ScopedEvents& operator=(const ScopedEvents&) = delete;
};

// Pair-sweep variant for a catalogue layout: cached per workload class or
// timed now (histograms are reset by the caller afterwards).
static int pick_pair2_variant(gr_ctx* c, const DevCatalog& C, bool weighted, double fscale,
                              unsigned long long* hcnt, unsigned long long* hfix,
                              unsigned long long* stats, int* work, cudaStream_t s) {
  // a grid of rmax/2 cells is read by the tile sweep only
  if (C.grid.sub == 2) return kPairTile2;
  if (c->autotune == 0) return kPairWarpCell;
  if (c->autotune >= 2) {
    const int v = c->autotune - 2;
    return v == kPairTile2 ? kPairTile : v;
  }
  // the variants that read cells at least rmax wide
  const int nvar = kPairTile + 1;
  const double per_cell = C.grid.ncell > 0 ? (double)C.n / (double)C.grid.ncell : 1.0;
  int dens = 0;
  while (dens < 20 && std::ldexp(1.0, dens + 1) <= per_cell) ++dens;
  int hb = 0;
  while (hb < 20 && (2 << hb) <= c->nbins * c->nmu) ++hb;
  // number of cells in factors of 4: how well a variant fills the SMs with
  // warps or blocks per cell depends on it
  int cb = 0;
  while (cb < 20 && ((int64_t)4 << (2 * cb)) <= C.grid.ncell) ++cb;
  char key[128];
  std::snprintf(key, sizeof(key), "pair2v9|%s|%s|dens%d|hist%d|cells%d", c->P.f32 ? "f32" : "f64",
                weighted ? "w" : "u", dens, hb, cb);
  Tuner& T = tuner();
  {
    std::lock_guard<std::mutex> lock(T.mu);
    T.load();
    auto it = T.choice.find(key);
    if (it != T.choice.end()) return it->second;
  }
  const int nh = c->nbins * c->nmu * 4;
  ScopedEvents ev;
  cudaEvent_t a = ev.a, b = ev.b;
  // every variant once untimed (its first launch loads its code), then the
  // fastest of three interleaved rounds
  float t[kPairVariants];
  for (int v = 0; v < nvar; ++v) {
    t[v] = 1e30f;
    launch_pair2(C, c->P, weighted, hcnt, hfix, fscale, stats, work, s, v);
  }
  for (int round = 0; round < 3; ++round) {
    for (int v = 0; v < nvar; ++v) {
      GR_CUDA_TRY(cudaMemsetAsync(hcnt, 0, sizeof(unsigned long long) * nh, s));
      GR_CUDA_TRY(cudaMemsetAsync(hfix, 0, sizeof(unsigned long long) * 2 * nh, s));
      GR_CUDA_TRY(cudaEventRecord(a, s));
      launch_pair2(C, c->P, weighted, hcnt, hfix, fscale, stats, work, s, v);
      GR_CUDA_TRY(cudaEventRecord(b, s));
      GR_CUDA_TRY(cudaEventSynchronize(b));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      t[v] = std::min(t[v], ms);
    }
  }
  int best = kPairWarpCell;
  for (int v = 1; v < nvar; ++v)
    if (t[v] < t[best]) best = v;
  std::lock_guard<std::mutex> lock(T.mu);
  T.choice[key] = best;
  T.save();
  return best;
}

int gr_count_2pcf(gr_ctx* c, double* N2, double* N3, int64_t* counts, double* catsum) {
  GR_API_BEGIN(c)
  require_ready(c);
  ensure_events(c);
  cudaStream_t s = c->stream();
  const int nbm = c->nbins * c->nmu, nh = nbm * 4;
  const bool weighted = !c->uniform;
  const double fscale = fix_scale(c->wmax * c->wmax);
  c->hcnt.reserve(nh);
  c->hfix.reserve(2 * nh);
  c->stats.reserve(8);
  // read-back in the pinned stage: counts (nh), fixed-point sums (2 nh),
  // stats (8), the speculative grid's bounding-box flag (1)
  c->stage.reserve(3 * (size_t)nh + 9);
  unsigned long long* hc = c->stage.p;
  unsigned long long* hf = hc + nh;
  unsigned long long* st = hf + 2 * (size_t)nh;
  unsigned long long* gflag = st + 8;
  std::vector<double> hs(nh, 0.0);
  // dense catalogues: cells of rmax/2 and the tile sweep
  int sub = 1;
  if (c->autotune == 1) sub = 0;
  if (c->autotune == 2 + kPairTile2) sub = 2;
  // A catalogue seen before (or a new one while that has worked) is indexed
  // on the grid of the last bounding box without waiting for the new one;
  // a device flag read with the histograms repeats the call with waits when
  // the box changed (as for the 3PCF).
  const bool reuse = reuse_graph(c);
  const bool can_spec =
      !reuse && c->index.have_prev && (c->cat_gen == c->spec_gen || c->spec_new_ok);
  int variant = 0;
  bool replayed = false;
  for (int attempt = 0; attempt < 2; ++attempt) {
    const bool spec = can_spec && attempt == 0;
    replayed = spec && c->spec_index.idx && spec_key(c, sub, false) == c->spec_index.key;
    GR_CUDA_TRY(cudaEventRecord(c->ev[0], s));
    if (!reuse) {
      if (replayed) {
        // the host state of the last identical build stands
        GR_CUDA_TRY(cudaGraphLaunch(c->spec_index.idx, s));
        c->csr_valid = false;
      } else {
        build_index(c, spec, sub);
      }
    }
    GR_CUDA_TRY(cudaEventRecord(c->ev[1], s));
    c->work.reserve(4);
    variant = pick_pair2_variant(c, c->index.view(), weighted, fscale, c->hcnt.p, c->hfix.p,
                                 c->stats.p, c->work.p, s);
    c->last_variant = variant;
    GR_CUDA_TRY(cudaEventRecord(c->ev[1], s));
    GR_CUDA_TRY(cudaMemsetAsync(c->hcnt.p, 0, sizeof(unsigned long long) * nh, s));
    GR_CUDA_TRY(cudaMemsetAsync(c->hfix.p, 0, sizeof(unsigned long long) * 2 * nh, s));
    GR_CUDA_TRY(cudaMemsetAsync(c->stats.p, 0, sizeof(unsigned long long) * 8, s));
    launch_pair2(c->index.view(), c->P, weighted, c->hcnt.p, c->hfix.p, fscale, c->stats.p,
                 c->work.p, s, variant);
    GR_CUDA_TRY(cudaEventRecord(c->ev[2], s));
    GR_CUDA_TRY(cudaMemcpyAsync(hc, c->hcnt.p, sizeof(unsigned long long) * nh, cudaMemcpyDeviceToHost, s));
    if (weighted)
      GR_CUDA_TRY(cudaMemcpyAsync(hf, c->hfix.p, sizeof(unsigned long long) * 2 * nh, cudaMemcpyDeviceToHost, s));
    GR_CUDA_TRY(cudaMemcpyAsync(st, c->stats.p, sizeof(unsigned long long) * 8, cudaMemcpyDeviceToHost, s));
    *gflag = 0;
    const bool speculated = spec && c->index.speculated;
    if (speculated)
      GR_CUDA_TRY(cudaMemcpyAsync(gflag, c->index.mismatch_flag(), sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, s));
    GR_CUDA_TRY(cudaEventRecord(c->ev[3], s));
    GR_CUDA_TRY(cudaStreamSynchronize(s));
    if (speculated && *gflag != 0) {  // the bounding box changed: repeat with waits
      if (c->cat_gen != c->spec_gen) c->spec_new_ok = false;
      continue;
    }
    // a speculative index that held: kept as a graph for the next call of
    // the same configuration
    if (speculated && !replayed) capture_spec_graph(c, c->spec_index, sub, false);
    break;
  }
  if (!reuse) c->spec_gen = c->cat_gen;
  if (weighted)
    for (int k = 0; k < nh; ++k) hs[k] = fix_value(hf[k], hf[nh + k], fscale);
  if (!weighted) {
    for (int cat = 0; cat < 4; ++cat) {
      double prod = uniform_product(c->w_gal, c->w_ran, 2 - ((cat >> 1) + (cat & 1)),
                                    (cat >> 1) + (cat & 1));
      for (int k = 0; k < nbm; ++k) hs[k + nbm * cat] = (double)hc[k + nbm * cat] * prod;
    }
  }
  int64_t rooted = 0;
  for (int k = 0; k < nh; ++k) rooted += (int64_t)hc[k];
  for (int k = 0; k < nbm; ++k) {
    if (N2) N2[k] = ((hs[k] + hs[k + nbm]) + hs[k + 2 * nbm]) + hs[k + 3 * nbm];
    if (N3) N3[k] = hs[k + 3 * nbm];
  }
  if (counts)
    for (int k = 0; k < nh; ++k) counts[k] = (int64_t)hc[k];
  if (catsum)
    for (int k = 0; k < nh; ++k) catsum[k] = hs[k];
  std::memset(&c->st, 0, sizeof(c->st));
  c->st.ms_index = ev_ms(c->ev[0], c->ev[1]);
  c->st.ms_graph = 0.0;
  c->st.ms_query = ev_ms(c->ev[1], c->ev[2]);
  c->st.ms_total = ev_ms(c->ev[0], c->ev[2]);
  c->st.n_points = c->n;
  c->st.n_edges = 2 * (int64_t)st[2];
  c->st.tuples = (int64_t)st[2];
  c->st.rooted = rooted;
  c->st.fp64_rechecks = (int64_t)st[0];
  c->st.candidates = (int64_t)st[1];
  c->st.kernel_launches = c->index.launches + 1;
  GR_API_END(c)
}

// Longest-first root order of the current graph for the 4-clique kernels
// (rows longer than the class cap share the first class).  Measured on the
// 4PCF workload: unit weights 4.97 -> 4.34 ms, lognormal weighted sums 9.86
// -> 8.23 ms, adjoint 12.9 -> 9.3 ms (the last roots of a block no longer
// keep its other warps waiting at the final barrier, nor the launch waiting
// on one heavy root).  The triangle kernel keeps label order: on the 3PCF
// workload the order cost 0.04 ms (0.765 against 0.723 ms: the sort, and
// neighbouring roots no longer sharing their rows in L1), and the 3M-point
// adjoint catalogue gained nothing (398 against 396 ms, 852 against 849 ms).
constexpr int kRootOrderLaunches = 3;  // kernels of order_roots_by_length
static const int* root_order(gr_ctx* c, cudaStream_t s, const int** above = nullptr,
                             int* nclass = nullptr) {
  const int cap = (int)std::min<int64_t>(std::max<int64_t>(c->csr.max_deg, 1024) + 1, 1 << 16);
  c->qorder.reserve((size_t)c->n + cap + 1);
  int* scratch = c->qorder.p + c->n;
  order_roots_by_length(c->csr.view(), (int)c->n, cap, c->qorder.p, scratch, s);
  // after the ordering, scratch[b] holds the number of roots in the classes
  // above b (classes 0..cap)
  if (above) *above = scratch;
  if (nclass) *nclass = cap + 1;
  return c->qorder.p;
}

// Third-edge test of the triangle kernel: the geometric pair test unless the
// hash probes are forced.  Measured: 3PCF catalogue with 5 mu bins and upper
// degree 13.7, 0.743 ms geometric against 0.754 ms (the FP32 binning of the
// re-tested third edges with approximate square root and division; 0.78
// against 0.75 ms with correctly rounded ones); without mu bins 0.56
// against 0.64 ms; upper degree 156, 197 against 250 ms with 5 mu bins.
static int tri_geometric(const gr_ctx* c) {
  return c->clique_mode == 1 ? 0 : 1;
}

static int count_tri(gr_ctx* c, bool equi, double* N2, double* N3, int64_t* counts, double* catsum) {
  GR_API_BEGIN(c)
  require_ready(c);
  ensure_events(c);
  cudaStream_t s = c->stream();
  const int nmu = c->nmu;
  const int ncfg = equi ? c->nbins : (int)(((int64_t)c->nbins * (c->nbins + 1) * (c->nbins + 2)) / 6);
  const int nbin = ncfg * nmu, nh = nbin * 4;
  const bool weighted = !c->uniform;
  const bool want_counts = counts != nullptr || !weighted;
  double fscale[4];
  for (int nr = 0; nr < 4; ++nr)
    fscale[nr] = fix_scale(std::pow(c->wgmax, 3 - nr) * std::pow(c->wrmax, nr));
  c->hcnt.reserve(nh);
  c->hfix.reserve(2 * nh);
  c->stats.reserve(8);
  ensure_normal(c, nmu, s);
  const bool reuse = reuse_graph(c);
  // A rebuild of a catalogue seen before runs without waiting on the host:
  // the grid is taken from the last bounding box, the graph is filled in the
  // scratch area as it is, and the triangle kernel's row capacity is taken
  // from the last graph (longer rows take its global-memory path, so any
  // capacity gives the same result).  A device flag records a changed
  // bounding box and the graph build one that ran out of room; both are
  // read with the results, and the call is then repeated with waits.
  const bool can_spec =
      !reuse && c->index.have_prev && (c->cat_gen == c->spec_gen || c->spec_new_ok);
  // read-back layout in the pinned stage: counts (nh), the sums converted
  // on the device (nh doubles), kernel stats (8), graph control (4) and
  // stats (3), bbox flag (1)
  c->stage.reserve(2 * (size_t)nh + 16);
  c->hval.reserve(nh);
  unsigned long long* hc = c->stage.p;
  double* hv = reinterpret_cast<double*>(hc + nh);
  unsigned long long* st = hc + 2 * (size_t)nh;
  unsigned long long* gctl = st + 8;
  unsigned long long* gsts = gctl + 4;
  unsigned long long* gflag = gsts + 3;
  std::vector<double> hs(nh, 0.0);
  cudaEvent_t q0 = c->ev[4];  // owned by the context
  c->work.reserve(4);
  int tri_launches = 0;
  std::vector<unsigned long long> key;
  bool replayed = false;
  for (int attempt = 0; attempt < 2; ++attempt) {
    const bool spec = can_spec && attempt == 0;
    bool replay = false;
    if (spec) {
      key = spec_key(c, 1, true);
      replay = c->spec_graph.idx && c->spec_graph.csr && key == c->spec_graph.key;
    }
    replayed = replay;
    GR_CUDA_TRY(cudaEventRecord(c->ev[0], s));
    if (!reuse) {
      if (replay) {
        // the host state of the last identical build stands
        GR_CUDA_TRY(cudaGraphLaunch(c->spec_graph.idx, s));
        c->csr_valid = false;
      } else {
        build_index(c, spec);
      }
    }
    GR_CUDA_TRY(cudaEventRecord(c->ev[1], s));
    if (!reuse) {
      if (replay) {
        GR_CUDA_TRY(cudaGraphLaunch(c->spec_graph.csr, s));
        c->csr.compacted = false;
      } else {
        build_csr(c, spec);
      }
    }
    GR_CUDA_TRY(cudaEventRecord(c->ev[2], s));
    {
      ZeroList z;
      z.add(c->hcnt.p, sizeof(unsigned long long) * nh);
      z.add(c->hfix.p, sizeof(unsigned long long) * 2 * nh);
      z.add(c->stats.p, sizeof(unsigned long long) * 8);
      zero_async(z, s);
    }
    TriParams T{};
    T.nbins = c->nbins;
    T.nmu = nmu;
    T.ncfg = ncfg;
    T.rsd = nmu >= 2;
    T.equi = equi ? 1 : 0;
    T.cap = round_cap(c->csr.max_deg, 32, 256);
    T.normal = c->normal_dev.p;
    make_rank_tables(T.rank, c->nbins, 3);
    for (int nr = 0; nr < 4; ++nr) T.fscale[nr] = fscale[nr];
    T.P = c->P;
    T.geo = tri_geometric(c);
    T.maxdeg = (int)std::min<int64_t>(c->csr.max_deg, 1 << 30);
    T.long_geo = c->clique_mode != 1;
    const CSRView G = c->csr.view();
    GR_CUDA_TRY(cudaEventRecord(q0, s));
    tri_launches = 1 + launch_tri3(c->index.view(), G, T, weighted, want_counts, c->hcnt.p,
                                   c->hfix.p, c->stats.p, c->work.p, s);  // + the zero fill
    GR_CUDA_TRY(cudaEventRecord(c->ev[3], s));
    if (want_counts)
      GR_CUDA_TRY(cudaMemcpyAsync(hc, c->hcnt.p, sizeof(unsigned long long) * nh, cudaMemcpyDeviceToHost, s));
    if (weighted) {
      enqueue_fix_convert(c->hfix.p, nh, nh, nbin, fscale, false, c->hval.p, s);
      GR_CUDA_TRY(cudaMemcpyAsync(hv, c->hval.p, sizeof(double) * nh, cudaMemcpyDeviceToHost, s));
    }
    GR_CUDA_TRY(cudaMemcpyAsync(st, c->stats.p, sizeof(unsigned long long) * 8, cudaMemcpyDeviceToHost, s));
    std::memset(gctl, 0, sizeof(unsigned long long) * 8);
    if (spec) {
      GR_CUDA_TRY(cudaMemcpyAsync(gctl, c->csr.ctl.p, sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost, s));
      GR_CUDA_TRY(cudaMemcpyAsync(gsts, c->csr.stats.p, sizeof(unsigned long long) * 3, cudaMemcpyDeviceToHost, s));
      if (c->index.speculated)
        GR_CUDA_TRY(cudaMemcpyAsync(gflag, c->index.mismatch_flag(), sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, s));
    }
    GR_CUDA_TRY(cudaStreamSynchronize(s));
    if (spec) {
      if (*gflag != 0 || gctl[1] == 1) {  // repeat with waits
        if (c->cat_gen != c->spec_gen) c->spec_new_ok = false;
        continue;
      }
      c->csr.settle(gctl, gsts);
      c->csr_valid = true;
      // a speculative build that needed no second pass: keep it as graphs
      // for the next call of the same configuration
      if (!replayed) {
        capture_spec_graph(c, c->spec_graph, 1, true);
        c->csr_valid = true;
        c->csr.settle(gctl, gsts);
      }
    }
    break;
  }
  if (!reuse) c->spec_gen = c->cat_gen;
  // graph statistics are on the host after the build (or the load)
  const unsigned long long gst[3] = {(unsigned long long)c->csr.rechecks,
                                     (unsigned long long)c->csr.candidates,
                                     (unsigned long long)c->csr.max_deg};
  if (weighted)
    for (int k = 0; k < nh; ++k) hs[k] = hv[k];
  if (!weighted) {
    for (int nr = 0; nr < 4; ++nr) {
      double prod = uniform_product(c->w_gal, c->w_ran, 3 - nr, nr);
      for (int k = 0; k < nbin; ++k) hs[k + nbin * nr] = (double)hc[k + nbin * nr] * prod;
    }
  }
  for (int k = 0; k < nbin; ++k) {
    if (N2) N2[k] = ((hs[k] + hs[k + nbin]) + hs[k + 2 * nbin]) + hs[k + 3 * nbin];
    // -equi with line-of-sight bins sums N2 only (gramsci.F90:425-428)
    if (N3) N3[k] = (equi && nmu >= 2) ? 0.0 : -hs[k + 3 * nbin];
  }
  if (counts)
    for (int k = 0; k < nh; ++k) counts[k] = (int64_t)hc[k];
  if (catsum)
    for (int k = 0; k < nh; ++k) catsum[k] = hs[k];
  std::memset(&c->st, 0, sizeof(c->st));
  c->st.ms_index = ev_ms(c->ev[0], c->ev[1]);
  c->st.ms_graph = ev_ms(c->ev[1], c->ev[2]);
  c->st.ms_query = ev_ms(q0, c->ev[3]);
  c->st.ms_total = c->st.ms_index + c->st.ms_graph + c->st.ms_query;
  c->st.n_points = c->n;
  c->st.n_edges = 2 * c->csr.n_edges;
  c->st.tuples = (int64_t)st[0];
  c->st.rooted = (int64_t)st[1];
  c->st.probes = (int64_t)st[2];
  c->st.upper_edges = c->csr.n_edges;
  c->st.fp64_rechecks = (int64_t)gst[0];
  c->st.candidates = (int64_t)gst[1];
  c->st.kernel_launches =
      (reuse ? 0 : c->index.launches + c->csr.launches) + tri_launches + (weighted ? 1 : 0);
  GR_API_END(c)
}

int gr_count_3pcf(gr_ctx* c, double* N2, double* N3, int64_t* counts, double* catsum) {
  return count_tri(c, false, N2, N3, counts, catsum);
}

int gr_count_equi(gr_ctx* c, double* N2, double* N3, int64_t* counts, double* catsum) {
  return count_tri(c, true, N2, N3, counts, catsum);
}

// Edges among R+(p) in the 4-clique kernels: the geometric pair test (rows
// up to 256 members) or hash probes of the members' rows.  Measured on the
// 4PCF workload (upper degree 17.5): unit weights 5.0 ms geometric against
// 6.3 ms, lognormal weighted sums 9.8 against 10.8 ms, adjoint 13.0 against
// 15.3 ms.
static int quad_geometric(const gr_ctx* c, int cap, int nbins) {
  return (cap > 256 || nbins > 255 || c->clique_mode == 1) ? 0 : 1;
}

static int count_quad(gr_ctx* c, bool tetra, double* N2, double* N3, double* discN, double* discR,
                      int64_t* counts, double* catsum, int64_t* dcount, double* dsum) {
  GR_API_BEGIN(c)
  require_ready(c);
  ensure_events(c);
  cudaStream_t s = c->stream();
  const int nb = c->nbins;
  const int64_t ncfg64 = ((int64_t)nb * (nb + 1) * (nb + 2) * (nb + 3)) / 24;
  const int64_t nbin64 = tetra ? nb : ncfg64 * nb * nb;
  if (nbin64 * 29 > ((int64_t)1 << 31)) return set_err(c, GR_E_CAPACITY, "4PCF histogram too large");
  const int ncfg = (int)ncfg64, nbin = (int)nbin64;
  const int ndc = tetra ? 5 : 4;  // disc categories
  // the last category (discR) equals the one before it (all randoms) and is
  // copied here instead of accumulated on the device
  const int nh = nbin * 5, nd = nbin * 6 * ndc, ndv = nbin * 6 * (ndc - 1);
  const bool weighted = !c->uniform;
  // unit-weight 4PCF: the kernels fill the pattern histogram (kQuadPatterns
  // x nbin counts), expanded here into the N2 / N3 and disconnected-term counts
  const bool patterns = !weighted && !tetra;
  const int nhk = patterns ? nbin * kQuadPatterns : nh, ndk = patterns ? 0 : ndv;
  const double fscale = fix_scale(c->wmax * c->wmax * c->wmax * c->wmax);
  const double dscale = fix_scale(tetra ? c->wmax * c->wmax * c->wmax : c->wmax * c->wmax);
  c->hcnt.reserve(std::max(nh, nhk));
  c->hfix.reserve((size_t)2 * nh * kFixStride);
  c->dcnt.reserve(ndv);
  c->dfix.reserve((size_t)2 * ndv * kFixStride);
  c->stats.reserve(8);
  const bool reuse = reuse_graph(c);
  GR_CUDA_TRY(cudaEventRecord(c->ev[0], s));
  if (!reuse) build_index(c);
  GR_CUDA_TRY(cudaEventRecord(c->ev[1], s));
  if (!reuse) build_csr(c);
  GR_CUDA_TRY(cudaEventRecord(c->ev[2], s));
  const unsigned long long gst[3] = {(unsigned long long)c->csr.rechecks,
                                     (unsigned long long)c->csr.candidates,
                                     (unsigned long long)c->csr.max_deg};
  GR_CUDA_TRY(cudaMemsetAsync(c->hcnt.p, 0, sizeof(unsigned long long) * nhk, s));
  if (ndk) GR_CUDA_TRY(cudaMemsetAsync(c->dcnt.p, 0, sizeof(unsigned long long) * ndk, s));
  if (weighted) {
    GR_CUDA_TRY(cudaMemsetAsync(c->hfix.p, 0, sizeof(unsigned long long) * 2 * nh * kFixStride, s));
    GR_CUDA_TRY(cudaMemsetAsync(c->dfix.p, 0, sizeof(unsigned long long) * 2 * ndv * kFixStride, s));
  }
  GR_CUDA_TRY(cudaMemsetAsync(c->stats.p, 0, sizeof(unsigned long long) * 8, s));
  if ((int64_t)gst[2] > 1024)
    return set_err(c, GR_E_CAPACITY, "4PCF: a point has more than 1024 larger-label neighbours");
  QuadParams Q{};
  Q.nbins = nb;
  Q.ncfg = ncfg;
  Q.tetra = tetra ? 1 : 0;
  // integer counts are not part of the reference's output: kept when the
  // caller asks for them (and always for unit weights, whose sums are
  // count x product)
  Q.counts = (!weighted || counts || dcount) ? 1 : 0;
  Q.cap = round_cap((int64_t)gst[2], 32, 1024);
  make_rank_tables(Q.rank, nb, 4);
  Q.P = c->P;
  Q.geo = quad_geometric(c, Q.cap, nb);
  const CSRView G = c->csr.view();
  cudaEvent_t q0 = c->ev[4];  // owned by the context
  GR_CUDA_TRY(cudaEventRecord(q0, s));
  Q.order = root_order(c, s, &Q.above, &Q.nclass);
  c->work.reserve(4);
  std::vector<unsigned long long> hc(nh), dc(nd);
  std::vector<double> hs(nh, 0.0), ds(nd, 0.0);
  // read-back in the pinned stage: counts (nh, ndv; or the nhk pattern
  // counts, fewer), the sums converted on the device (nh, ndv doubles),
  // kernel stats (8)
  c->stage.reserve(2 * ((size_t)nh + ndv) + 8);
  c->hval.reserve((size_t)nh + ndv);
  unsigned long long* sc = c->stage.p;
  unsigned long long* sd = sc + nh;
  double* sv = reinterpret_cast<double*>(sd + ndv);
  unsigned long long* st = sd + ndv + nh + ndv;
  // First attempt: unweighted counts in block-private 32-bit counters, and
  // weighted sums as split limbs added without returned values (fix_red).
  // Both are exact while every bin receives fewer than 2^32 updates, which
  // holds when the rooted total is below 2^32 (a rooted clique updates each
  // N2 / N3 bin and each disconnected-term bin at most once); otherwise the
  // launch is repeated with 64-bit counters and carried 128-bit sums.
  for (int attempt = 0; attempt < 2; ++attempt) {
    if (attempt > 0) {
      GR_CUDA_TRY(cudaMemsetAsync(c->hcnt.p, 0, sizeof(unsigned long long) * nhk, s));
      if (ndk) GR_CUDA_TRY(cudaMemsetAsync(c->dcnt.p, 0, sizeof(unsigned long long) * ndk, s));
      if (weighted) {
        GR_CUDA_TRY(cudaMemsetAsync(c->hfix.p, 0, sizeof(unsigned long long) * 2 * nh * kFixStride, s));
        GR_CUDA_TRY(cudaMemsetAsync(c->dfix.p, 0, sizeof(unsigned long long) * 2 * ndv * kFixStride, s));
      }
      GR_CUDA_TRY(cudaMemsetAsync(c->stats.p, 0, sizeof(unsigned long long) * 8, s));
      GR_CUDA_TRY(cudaEventRecord(q0, s));
    }
    Q.split = (weighted && attempt == 0) ? 1 : 0;
    const bool shared = launch_quad4(c->index.view(), G, Q, weighted, c->hcnt.p, c->hfix.p,
                                     c->dcnt.p, c->dfix.p, nhk, ndk, fscale, dscale, attempt == 0,
                                     c->stats.p, c->work.p, s);
    GR_CUDA_TRY(cudaEventRecord(c->ev[3], s));
    if (Q.counts) {
      GR_CUDA_TRY(cudaMemcpyAsync(sc, c->hcnt.p, sizeof(unsigned long long) * nhk, cudaMemcpyDeviceToHost, s));
      if (ndk)
        GR_CUDA_TRY(cudaMemcpyAsync(sd, c->dcnt.p, sizeof(unsigned long long) * ndk, cudaMemcpyDeviceToHost, s));
    }
    if (weighted) {
      const double fs[4] = {fscale, fscale, fscale, fscale};
      const double ds4[4] = {dscale, dscale, dscale, dscale};
      enqueue_fix_convert(c->hfix.p, nh, nh, nh, fs, Q.split != 0, c->hval.p, s, kFixStride);
      enqueue_fix_convert(c->dfix.p, ndv, ndv, ndv, ds4, Q.split != 0, c->hval.p + nh, s, kFixStride);
      GR_CUDA_TRY(cudaMemcpyAsync(sv, c->hval.p, sizeof(double) * ((size_t)nh + ndv), cudaMemcpyDeviceToHost, s));
    }
    GR_CUDA_TRY(cudaMemcpyAsync(st, c->stats.p, sizeof(unsigned long long) * 8, cudaMemcpyDeviceToHost, s));
    GR_CUDA_TRY(cudaStreamSynchronize(s));
    if (!(shared || Q.split) || st[1] < (1ull << 32)) break;
  }
  if (patterns) {
    quad_expand_patterns(sc, nbin, hc.data(), dc.data());
  } else if (Q.counts) {
    std::memcpy(hc.data(), sc, sizeof(unsigned long long) * nh);
    std::memcpy(dc.data(), sd, sizeof(unsigned long long) * ndv);
  }
  if (st[3] != 0)
    return set_err(c, GR_E_CAPACITY, "4PCF: label offsets within a row exceed the hash key range");
  // discR category = the all-random category before it
  for (int k = 0; k < nbin * 6; ++k) dc[(size_t)ndv + k] = dc[(size_t)ndv - nbin * 6 + k];
  if (weighted) {
    std::memcpy(hs.data(), sv, sizeof(double) * nh);
    std::memcpy(ds.data(), sv + nh, sizeof(double) * ndv);
    for (int k = 0; k < nbin * 6; ++k) ds[(size_t)ndv + k] = ds[(size_t)ndv - nbin * 6 + k];
  }
  if (!weighted) {
    for (int nr = 0; nr < 5; ++nr) {
      double prod = uniform_product(c->w_gal, c->w_ran, 4 - nr, nr);
      for (int k = 0; k < nbin; ++k) hs[k + (size_t)nbin * nr] = (double)hc[k + (size_t)nbin * nr] * prod;
    }
    for (int cat = 0; cat < ndc; ++cat) {
      // 4PCF pair terms: cat = randoms in the pair (3 = discR, both random);
      // -tetra 3-products: cat = randoms in the product (4 = discR, all random)
      const int q = tetra ? 3 : 2;
      const int nrnd = tetra ? (cat == 4 ? 3 : cat) : (cat == 3 ? 2 : cat);
      double prod = uniform_product(c->w_gal, c->w_ran, q - nrnd, nrnd);
      for (int k = 0; k < nbin * 6; ++k)
        ds[k + (size_t)nbin * 6 * cat] = (double)dc[k + (size_t)nbin * 6 * cat] * prod;
    }
  }
  for (int k = 0; k < nbin; ++k) {
    double acc = 0.0;
    for (int nr = 0; nr < 5; ++nr) acc += hs[k + (size_t)nbin * nr];
    if (N2) N2[k] = acc;
    if (N3) N3[k] = hs[k + (size_t)nbin * 4];
  }
  for (int k = 0; k < nbin * 6; ++k) {
    double acc = 0.0;
    for (int cat = 0; cat < ndc - 1; ++cat) acc += ds[k + (size_t)nbin * 6 * cat];
    if (discN) discN[k] = acc;
    if (discR) discR[k] = ds[k + (size_t)nbin * 6 * (ndc - 1)];
  }
  if (counts)
    for (int k = 0; k < nh; ++k) counts[k] = (int64_t)hc[k];
  if (catsum)
    for (int k = 0; k < nh; ++k) catsum[k] = hs[k];
  if (dcount)
    for (int k = 0; k < nd; ++k) dcount[k] = (int64_t)dc[k];
  if (dsum)
    for (int k = 0; k < nd; ++k) dsum[k] = ds[k];
  std::memset(&c->st, 0, sizeof(c->st));
  c->st.ms_index = ev_ms(c->ev[0], c->ev[1]);
  c->st.ms_graph = ev_ms(c->ev[1], c->ev[2]);
  c->st.ms_query = ev_ms(q0, c->ev[3]);
  c->st.ms_total = c->st.ms_index + c->st.ms_graph + c->st.ms_query;
  c->st.n_points = c->n;
  c->st.n_edges = 2 * c->csr.n_edges;
  c->st.tuples = (int64_t)st[0];
  c->st.rooted = (int64_t)st[1];
  c->st.probes = (int64_t)st[2];
  c->st.upper_edges = c->csr.n_edges;
  c->st.fp64_rechecks = (int64_t)gst[0];
  c->st.candidates = (int64_t)gst[1];
  c->st.kernel_launches = c->index.launches + c->csr.launches + 1 + (Q.order ? kRootOrderLaunches : 0) +
                          (weighted ? 2 : 0);
  GR_API_END(c)
}

int gr_count_4pcf(gr_ctx* c, double* N2, double* N3, double* discN, double* discR,
                  int64_t* counts, double* catsum, int64_t* dcount, double* dsum) {
  return count_quad(c, false, N2, N3, discN, discR, counts, catsum, dcount, dsum);
}

int gr_count_tetra(gr_ctx* c, double* N2, double* N3, double* discN, double* discR,
                   int64_t* counts, double* catsum, int64_t* dcount, double* dsum) {
  return count_quad(c, true, N2, N3, discN, discR, counts, catsum, dcount, dsum);
}

int gr_graph_build(gr_ctx* c) {
  GR_API_BEGIN(c)
  require_ready(c);
  if (!reuse_graph(c)) {
    build_index(c);
    build_csr(c);
  }
  GR_CUDA_TRY(cudaStreamSynchronize(c->stream()));
  GR_API_END(c)
}

// ------------------------------------------------------ graph persistence ----
namespace {

struct GraphFileHeader {
  char magic[8];  // "GRAMSCSR"
  uint32_t version, header_bytes;
  int64_t n, n_edges, max_deg;
  double rmin, rmax;
  int32_t nbins, nmu, logbins, reserved0;
  unsigned long long fingerprint, checksum;
  int64_t rechecks, candidates;
  unsigned long long labels;  // FNV-1a of the cell labelling (label -> point)
  unsigned char pad[128 - 8 - 8 - 24 - 16 - 16 - 16 - 16 - 8];
};
static_assert(sizeof(GraphFileHeader) == 128, "graph file header is 128 bytes");

unsigned long long fnv1a(unsigned long long h, const void* p, size_t bytes) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  for (size_t k = 0; k < bytes; ++k) h = (h ^ b[k]) * 0x100000001b3ull;
  return h;
}

unsigned long long coord_fingerprint(gr_ctx* c) {
  cudaStream_t s = c->stream();
  c->uniform_flag.reserve(32);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(c->uniform_flag.p + 24);
  GR_CUDA_TRY(cudaMemsetAsync(d, 0, sizeof(unsigned long long), s));
  if (c->n > 0) {
    int blocks = (int)std::min<int64_t>((c->n + 255) / 256, (int64_t)8 * sm_count());
    fingerprint_kernel<<<blocks, 256, 0, s>>>(c->xyz.p, c->n, d);
    GR_CHECK_LAUNCH();
  }
  unsigned long long h = 0;
  GR_CUDA_TRY(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaStreamSynchronize(s));
  return h ^ mix_host((unsigned long long)c->n);
}

unsigned long long label_fingerprint(gr_ctx* c) {
  std::vector<int> orig(c->n);
  if (c->n > 0) {
    GR_CUDA_TRY(cudaMemcpyAsync(orig.data(), c->index.orig.p, sizeof(int) * c->n, cudaMemcpyDeviceToHost,
                                c->stream()));
    GR_CUDA_TRY(cudaStreamSynchronize(c->stream()));
  }
  return fnv1a(0xcbf29ce484222325ull, orig.data(), sizeof(int) * orig.size());
}

}  // namespace

int gr_graph_save(gr_ctx* c, const char* path) {
  GR_API_BEGIN(c)
  if (!path) return set_err(c, GR_E_ARG, "null path");
  require_ready(c);
  if (!c->csr_valid) {
    build_index(c);
    build_csr(c);
  }
  cudaStream_t s = c->stream();
  c->csr.compact(s);
  const int64_t n = c->n, E = c->csr.n_edges;
  std::vector<int64_t> rp(n + 1);
  std::vector<unsigned long long> rec(E);
  std::vector<int> deg(n);
  GR_CUDA_TRY(cudaMemcpyAsync(rp.data(), c->csr.row_ptr.p, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, s));
  if (E > 0)
    GR_CUDA_TRY(cudaMemcpyAsync(rec.data(), c->csr.rec.p, sizeof(unsigned long long) * E, cudaMemcpyDeviceToHost, s));
  if (n > 0)
    GR_CUDA_TRY(cudaMemcpyAsync(deg.data(), c->csr.deg_full.p, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaStreamSynchronize(s));
  GraphFileHeader H;
  std::memset(&H, 0, sizeof(H));
  std::memcpy(H.magic, "GRAMSCSR", 8);
  H.version = 1;
  H.header_bytes = sizeof(H);
  H.n = n;
  H.n_edges = E;
  H.max_deg = c->csr.max_deg;
  H.rmin = c->rmin;
  H.rmax = c->rmax;
  H.nbins = c->nbins;
  H.nmu = c->nmu;
  H.logbins = c->logbins;
  H.rechecks = c->csr.rechecks;
  H.candidates = c->csr.candidates;
  H.fingerprint = coord_fingerprint(c);
  H.labels = label_fingerprint(c);
  unsigned long long h = 0xcbf29ce484222325ull;
  h = fnv1a(h, rp.data(), sizeof(int64_t) * rp.size());
  h = fnv1a(h, rec.data(), sizeof(unsigned long long) * rec.size());
  h = fnv1a(h, deg.data(), sizeof(int) * deg.size());
  H.checksum = h;
  FILE* f = std::fopen(path, "wb");
  if (!f) return set_err(c, GR_E_ARG, std::string("cannot write ") + path);
  bool ok = std::fwrite(&H, sizeof(H), 1, f) == 1 &&
            std::fwrite(rp.data(), sizeof(int64_t), rp.size(), f) == rp.size() &&
            std::fwrite(rec.data(), sizeof(unsigned long long), rec.size(), f) == rec.size() &&
            std::fwrite(deg.data(), sizeof(int), deg.size(), f) == deg.size();
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return set_err(c, GR_E_ARG, std::string("short write to ") + path);
  GR_API_END(c)
}

int gr_graph_load(gr_ctx* c, const char* path) {
  GR_API_BEGIN(c)
  if (!path) return set_err(c, GR_E_ARG, "null path");
  require_ready(c);
  FILE* f = std::fopen(path, "rb");
  if (!f) return set_err(c, GR_E_ARG, std::string("cannot read ") + path);
  GraphFileHeader H;
  auto fail = [&](const char* why) {
    std::fclose(f);
    return set_err(c, GR_E_ARG, why);
  };
  if (std::fread(&H, sizeof(H), 1, f) != 1) return fail("graph file: short header");
  if (std::memcmp(H.magic, "GRAMSCSR", 8) != 0 || H.version != 1 || H.header_bytes != sizeof(H))
    return fail("graph file: not a version-1 graph");
  if (H.n != c->n) return fail("graph file: point count differs from the catalogue");
  if (H.rmin != c->rmin || H.rmax != c->rmax || H.nbins != c->nbins || H.nmu != c->nmu ||
      H.logbins != c->logbins)
    return fail("graph file: binning differs from gr_set_bins");
  if (H.n_edges < 0 || H.max_deg < 0 || H.max_deg > H.n) return fail("graph file: bad sizes");
  if (H.fingerprint != coord_fingerprint(c)) return fail("graph file: coordinates differ");
  const int64_t n = H.n, E = H.n_edges;
  std::vector<int64_t> rp(n + 1);
  std::vector<unsigned long long> rec(E);
  std::vector<int> deg(n);
  if (std::fread(rp.data(), sizeof(int64_t), rp.size(), f) != rp.size() ||
      std::fread(rec.data(), sizeof(unsigned long long), rec.size(), f) != rec.size() ||
      std::fread(deg.data(), sizeof(int), deg.size(), f) != deg.size())
    return fail("graph file: short payload");
  std::fclose(f);
  unsigned long long h = 0xcbf29ce484222325ull;
  h = fnv1a(h, rp.data(), sizeof(int64_t) * rp.size());
  h = fnv1a(h, rec.data(), sizeof(unsigned long long) * rec.size());
  h = fnv1a(h, deg.data(), sizeof(int) * deg.size());
  if (h != H.checksum) return set_err(c, GR_E_ARG, "graph file: checksum mismatch");
  // structural checks before anything reaches the device: rows in range,
  // labels in range and increasing within a row (the query kernels rely on it)
  // bins in range, full degrees equal to the rows' (the kernels index
  // histograms by bin and size their staging by degree)
  if (rp[0] != 0 || rp[n] != E) return set_err(c, GR_E_ARG, "graph file: bad row pointers");
  int64_t maxd = 0;
  std::vector<int> dchk(n, 0);
  for (int64_t p = 0; p < n; ++p) {
    if (rp[p + 1] < rp[p]) return set_err(c, GR_E_ARG, "graph file: bad row pointers");
    maxd = std::max(maxd, rp[p + 1] - rp[p]);
    uint32_t prev = (uint32_t)p;
    for (int64_t e = rp[p]; e < rp[p + 1]; ++e) {
      const uint32_t q = (uint32_t)rec[e];
      if (q <= prev || q >= (uint64_t)n) return set_err(c, GR_E_ARG, "graph file: bad neighbour label");
      const uint32_t m = (uint32_t)(rec[e] >> 32);
      const int b = (int)(m & 0xff), mf = (int)((m >> 8) & 0xff), mr = (int)((m >> 16) & 0xff);
      if ((m >> 24) != 0 || b < 1 || b > c->nbins || mf < 1 || mf > c->nmu || mr < 1 || mr > c->nmu)
        return set_err(c, GR_E_ARG, "graph file: bad bin");
      dchk[p]++;
      dchk[q]++;
      prev = q;
    }
  }
  if (maxd != H.max_deg) return set_err(c, GR_E_ARG, "graph file: bad degree");
  if (dchk != deg) return set_err(c, GR_E_ARG, "graph file: bad degree");
  cudaStream_t s = c->stream();
  build_index(c);
  if (label_fingerprint(c) != H.labels)
    return set_err(c, GR_E_ARG, "graph file: cell labelling differs (written by another version)");
  UpperCSR& G = c->csr;
  G.n = n;
  G.n_edges = E;
  G.max_deg = H.max_deg;
  G.rechecks = H.rechecks;
  G.candidates = H.candidates;
  // rows go to the scratch layout (rstart = row offsets, deg_up = lengths)
  std::vector<int> up(n + 1, 0);
  for (int64_t p = 0; p < n; ++p) up[p] = (int)(rp[p + 1] - rp[p]);
  G.rstart.reserve(n + 1);
  G.deg_up.reserve(n + 1);
  G.scratch.reserve(E + 1);
  G.deg_full.reserve(n + 1);
  G.stats.reserve(4);
  unsigned long long st[4] = {(unsigned long long)H.rechecks, (unsigned long long)H.candidates,
                              (unsigned long long)H.max_deg, 0ull};
  GR_CUDA_TRY(cudaMemcpyAsync(G.rstart.p, rp.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, s));
  GR_CUDA_TRY(cudaMemcpyAsync(G.deg_up.p, up.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s));
  if (E > 0)
    GR_CUDA_TRY(cudaMemcpyAsync(G.scratch.p, rec.data(), sizeof(unsigned long long) * E, cudaMemcpyHostToDevice, s));
  if (n > 0)
    GR_CUDA_TRY(cudaMemcpyAsync(G.deg_full.p, deg.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s));
  G.compacted = false;
  GR_CUDA_TRY(cudaMemcpyAsync(G.stats.p, st, sizeof(st), cudaMemcpyHostToDevice, s));
  GR_CUDA_TRY(cudaStreamSynchronize(s));
  c->csr_valid = true;
  c->graph_loaded = true;
  GR_API_END(c)
}

int gr_graph_nedges(gr_ctx* c, int64_t* n_edges) {
  GR_API_BEGIN(c)
  if (!n_edges) return set_err(c, GR_E_ARG, "null output");
  if (!c->csr_valid) {
    require_ready(c);
    build_index(c);
    build_csr(c);
  }
  *n_edges = 2 * c->csr.n_edges;
  GR_API_END(c)
}

int gr_graph_export(gr_ctx* c, int64_t* row_ptr, int32_t* col, uint8_t* bin, uint8_t* mu) {
  GR_API_BEGIN(c)
  if (!c->csr_valid) {
    require_ready(c);
    build_index(c);
    build_csr(c);
  }
  cudaStream_t s = c->stream();
  c->csr.compact(s);
  const int64_t n = c->n, E = c->csr.n_edges;
  std::vector<int64_t> rp(n + 1);
  std::vector<int> orig(n);
  std::vector<unsigned long long> rc(E);
  GR_CUDA_TRY(cudaMemcpyAsync(rp.data(), c->csr.row_ptr.p, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, s));
  if (E > 0)
    GR_CUDA_TRY(cudaMemcpyAsync(rc.data(), c->csr.rec.p, sizeof(unsigned long long) * E, cudaMemcpyDeviceToHost, s));
  if (n > 0)
    GR_CUDA_TRY(cudaMemcpyAsync(orig.data(), c->index.orig.p, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaStreamSynchronize(s));
  // expand the upper rows into the reference's symmetric, id-sorted rows
  std::vector<int64_t> deg(n + 1, 0);
  for (int64_t p = 0; p < n; ++p)
    for (int64_t e = rp[p]; e < rp[p + 1]; ++e) {
      deg[orig[p]]++;
      deg[orig[(int)(uint32_t)rc[e]]]++;
    }
  std::vector<int64_t> out_ptr(n + 1, 0);
  for (int64_t i = 0; i < n; ++i) out_ptr[i + 1] = out_ptr[i] + deg[i];
  std::vector<int64_t> fill(out_ptr.begin(), out_ptr.end() - 1);
  std::vector<uint64_t> ent(2 * E);
  for (int64_t p = 0; p < n; ++p)
    for (int64_t e = rp[p]; e < rp[p + 1]; ++e) {
      int i = orig[p], j = orig[(int)(uint32_t)rc[e]];
      uint32_t m = (uint32_t)(rc[e] >> 32);
      uint64_t b = m & 0xff, mf = (m >> 8) & 0xff, mr = (m >> 16) & 0xff;
      ent[fill[i]++] = ((uint64_t)j << 16) | (b << 8) | mf;
      ent[fill[j]++] = ((uint64_t)i << 16) | (b << 8) | mr;
    }
  for (int64_t i = 0; i < n; ++i) std::sort(ent.begin() + out_ptr[i], ent.begin() + out_ptr[i + 1]);
  if (row_ptr) std::copy(out_ptr.begin(), out_ptr.end(), row_ptr);
  for (int64_t k = 0; k < 2 * E; ++k) {
    if (col) col[k] = (int32_t)(ent[k] >> 16);
    if (bin) bin[k] = (uint8_t)((ent[k] >> 8) & 0xff);
    if (mu) mu[k] = (uint8_t)(ent[k] & 0xff);
  }
  GR_API_END(c)
}

// ---------------------------------------------------------------- adjoints --
static double max_abs(const double* a, int64_t n) {
  double m = 0.0;
  if (a)
    for (int64_t i = 0; i < n; ++i) m = std::max(m, std::fabs(a[i]));
  return m;
}

static void finish_grad(gr_ctx* c, double gscale, double* grad_w, cudaEvent_t q0) {
  cudaStream_t s = c->stream();
  const int64_t n = c->n;
  c->grad.reserve(n + 1);
  launch_grad_finish((int)n, c->index.orig.p, c->gfix.p, c->gfix.p + n, gscale, c->grad.p, s);
  GR_CUDA_TRY(cudaEventRecord(c->ev[3], s));
  if (n > 0) GR_CUDA_TRY(cudaMemcpyAsync(grad_w, c->grad.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaStreamSynchronize(s));
  c->st.ms_query = ev_ms(q0, c->ev[3]);
}

// Layout of the 2PCF adjoint sweep (warp per cell, or block per cell of 128
// or 256 threads): timed and cached like the forward sweep's variant, under
// its own key (the fastest adjoint layout is not always the forward's).
static int pick_adj2_layout(gr_ctx* c, const DevCatalog& C, const double* c2, const double* c3,
                            double gscale, unsigned long long* g_lo, unsigned long long* g_hi,
                            int* work, cudaStream_t s) {
  // a grid of rmax/2 cells is read by the tile sweep only
  if (C.grid.sub == 2) return kPairTile2;
  if (c->autotune == 0) return kPairWarpCell;
  if (c->autotune >= 2) {
    const int v = c->autotune - 2;
    if (v == kPairTile || v == kPairTile2) return kPairTile;
    return v == kPairDense128 || v == kPairDenseQ128 ? kPairDense128
           : v == kPairDense256 || v == kPairDenseQ256 ? kPairDense256 : kPairWarpCell;
  }
  const double per_cell = C.grid.ncell > 0 ? (double)C.n / (double)C.grid.ncell : 1.0;
  int dens = 0;
  while (dens < 20 && std::ldexp(1.0, dens + 1) <= per_cell) ++dens;
  int hb = 0;
  while (hb < 20 && (2 << hb) <= c->nbins * c->nmu) ++hb;
  int cb = 0;
  while (cb < 20 && ((int64_t)4 << (2 * cb)) <= C.grid.ncell) ++cb;
  char key[128];
  std::snprintf(key, sizeof(key), "adj2v2|%s|dens%d|hist%d|cells%d", c->P.f32 ? "f32" : "f64", dens,
                hb, cb);
  Tuner& T = tuner();
  {
    std::lock_guard<std::mutex> lock(T.mu);
    T.load();
    auto it = T.choice.find(key);
    if (it != T.choice.end()) return it->second;
  }
  // the tile sweep accumulates into g_lo / g_hi: the caller zeroes them
  // after the timing runs
  const int layouts[4] = {kPairWarpCell, kPairDense128, kPairDense256, kPairTile};
  c->stats.reserve(8);
  auto run = [&](int v) {
    if (layouts[v] == kPairTile)
      launch_adj2_tile(C, c->P, c2, c3, gscale, g_lo, g_hi, c->stats.p, work, s);
    else
      launch_adj2(C, c->P, c2, c3, gscale, g_lo, g_hi, work, s, layouts[v]);
  };
  ScopedEvents ev;
  cudaEvent_t a = ev.a, b = ev.b;
  float t[4] = {1e30f, 1e30f, 1e30f, 1e30f};
  for (int v = 0; v < 4; ++v) run(v);
  for (int round = 0; round < 3; ++round)
    for (int v = 0; v < 4; ++v) {
      GR_CUDA_TRY(cudaEventRecord(a, s));
      run(v);
      GR_CUDA_TRY(cudaEventRecord(b, s));
      GR_CUDA_TRY(cudaEventSynchronize(b));
      float ms = 0.f;
      cudaEventElapsedTime(&ms, a, b);
      t[v] = std::min(t[v], ms);
    }
  int best = 0;
  for (int v = 1; v < 4; ++v)
    if (t[v] < t[best]) best = v;
  std::lock_guard<std::mutex> lock(T.mu);
  T.choice[key] = layouts[best];
  T.save();
  return layouts[best];
}

int gr_adjoint_2pcf(gr_ctx* c, const double* cot2, const double* cot3, double* grad_w) {
  GR_API_BEGIN(c)
  require_ready(c);
  if (!cot2 || !grad_w) return set_err(c, GR_E_ARG, "null cot2 or grad_w");
  ensure_events(c);
  cudaStream_t s = c->stream();
  const int nbm = c->nbins * c->nmu;
  const int64_t n = c->n;
  const double cmax = max_abs(cot2, nbm) + max_abs(cot3, nbm);
  c->cot.reserve(2 * nbm);
  c->gfix.reserve(2 * n + 2);
  c->work.reserve(4);
  c->stats.reserve(8);
  GR_CUDA_TRY(cudaMemcpyAsync(c->cot.p, cot2, sizeof(double) * nbm, cudaMemcpyHostToDevice, s));
  if (cot3)
    GR_CUDA_TRY(cudaMemcpyAsync(c->cot.p + nbm, cot3, sizeof(double) * nbm, cudaMemcpyHostToDevice, s));
  else
    GR_CUDA_TRY(cudaMemsetAsync(c->cot.p + nbm, 0, sizeof(double) * nbm, s));
  GR_CUDA_TRY(cudaEventRecord(c->ev[0], s));
  if (!reuse_graph(c)) {
    // dense catalogues: cells of rmax/2 and the tile sweep
    int sub = 1;
    if (c->autotune == 1) sub = 0;
    if (c->autotune == 2 + kPairTile2) sub = 2;
    build_index(c, false, sub);
  }
  GR_CUDA_TRY(cudaEventRecord(c->ev[1], s));
  std::memset(&c->st, 0, sizeof(c->st));
  const double* dc3 = c->cot.p + nbm;
  // the tile sweep's per-warp 64-bit partials take up to 32 terms: 2^6 of
  // headroom over the largest term (2 cotangents times a weight)
  const double gscale_t = fix_scale(64.0 * 2.0 * cmax * c->wmax);
  const double gscale_c = fix_scale(2.0 * cmax * c->wmax);
  const int variant = pick_adj2_layout(c, c->index.view(), c->cot.p, dc3, gscale_t, c->gfix.p,
                                       c->gfix.p + n, c->work.p, s);
  const bool tile = variant == kPairTile || variant == kPairTile2;
  const double gscale = tile ? gscale_t : gscale_c;
  GR_CUDA_TRY(cudaEventRecord(c->ev[2], s));  // after any tuning runs
  GR_CUDA_TRY(cudaMemsetAsync(c->gfix.p, 0, sizeof(unsigned long long) * (2 * n + 2), s));
  if (tile) {
    GR_CUDA_TRY(cudaMemsetAsync(c->stats.p, 0, sizeof(unsigned long long) * 8, s));
    launch_adj2_tile(c->index.view(), c->P, c->cot.p, dc3, gscale, c->gfix.p, c->gfix.p + n,
                     c->stats.p, c->work.p, s);
  } else {
    launch_adj2(c->index.view(), c->P, c->cot.p, dc3, gscale, c->gfix.p, c->gfix.p + n, c->work.p,
                s, variant);
  }
  finish_grad(c, gscale, grad_w, c->ev[2]);
  c->st.ms_index = ev_ms(c->ev[0], c->ev[1]);
  c->st.ms_total = c->st.ms_index + c->st.ms_query;
  c->st.n_points = n;
  c->st.kernel_launches = c->index.launches + 2;
  GR_API_END(c)
}

int gr_adjoint_3pcf(gr_ctx* c, const double* cot2, const double* cot3, double* grad_w) {
  GR_API_BEGIN(c)
  require_ready(c);
  if (!cot2 || !grad_w) return set_err(c, GR_E_ARG, "null cot2 or grad_w");
  ensure_events(c);
  cudaStream_t s = c->stream();
  const int nmu = c->nmu;
  const int ncfg = (int)(((int64_t)c->nbins * (c->nbins + 1) * (c->nbins + 2)) / 6);
  const int nc = ncfg * nmu;
  const int64_t n = c->n;
  const double cmax = max_abs(cot2, nc) + max_abs(cot3, nc);
  // 2^10 below the per-term bound: the kernel sums up to 1023 terms of one
  // root per neighbour in signed 64 bits before the 128-bit totals
  const double gscale = fix_scale(3.0 * cmax * c->wmax * c->wmax * 1024.0);
  ensure_normal(c, nmu, s);
  c->cot.reserve(2 * nc);
  c->gfix.reserve(2 * n + 2);
  c->work.reserve(4);
  c->stats.reserve(8);
  GR_CUDA_TRY(cudaMemcpyAsync(c->cot.p, cot2, sizeof(double) * nc, cudaMemcpyHostToDevice, s));
  if (cot3)
    GR_CUDA_TRY(cudaMemcpyAsync(c->cot.p + nc, cot3, sizeof(double) * nc, cudaMemcpyHostToDevice, s));
  GR_CUDA_TRY(cudaEventRecord(c->ev[0], s));
  const bool rebuilt = !c->csr_valid;
  if (rebuilt) {
    build_index(c);
    build_csr(c);
  }
  GR_CUDA_TRY(cudaEventRecord(c->ev[1], s));
  GR_CUDA_TRY(cudaMemsetAsync(c->gfix.p, 0, sizeof(unsigned long long) * (2 * n + 2), s));
  GR_CUDA_TRY(cudaMemsetAsync(c->stats.p, 0, sizeof(unsigned long long) * 8, s));
  TriParams T{};
  T.nbins = c->nbins;
  T.nmu = nmu;
  T.ncfg = ncfg;
  T.rsd = nmu >= 2;
  T.cap = round_cap(c->csr.max_deg, 32, 256);
  T.normal = c->normal_dev.p;
  make_rank_tables(T.rank, c->nbins, 3);
  T.P = c->P;
  T.geo = c->clique_mode == 1 ? 0 : 1;  // faster for the adjoint at every degree measured
  T.maxdeg = (int)std::min<int64_t>(c->csr.max_deg, 1 << 30);
  T.long_geo = c->clique_mode != 1;
  const CSRView G = c->csr.view();
  std::memset(&c->st, 0, sizeof(c->st));
  launch_adj3(c->index.view(), G, T, c->cot.p, cot3 ? c->cot.p + nc : nullptr, gscale, c->gfix.p,
              c->gfix.p + n, c->stats.p, c->work.p, s);
  finish_grad(c, gscale, grad_w, c->ev[1]);
  c->st.ms_graph = rebuilt ? ev_ms(c->ev[0], c->ev[1]) : 0.0;
  c->st.ms_total = c->st.ms_graph + c->st.ms_query;
  c->st.n_points = n;
  c->st.n_edges = 2 * c->csr.n_edges;
  c->st.upper_edges = c->csr.n_edges;
  c->st.kernel_launches = (rebuilt ? c->index.launches + c->csr.launches : 0) + 2;
  GR_API_END(c)
}

int gr_adjoint_4pcf(gr_ctx* c, const double* cot2, const double* cot3, const double* cotN,
                    const double* cotR, double* grad_w) {
  GR_API_BEGIN(c)
  require_ready(c);
  if (!cot2 || !grad_w) return set_err(c, GR_E_ARG, "null cot2 or grad_w");
  ensure_events(c);
  cudaStream_t s = c->stream();
  const int nb = c->nbins;
  const int64_t ncfg64 = ((int64_t)nb * (nb + 1) * (nb + 2) * (nb + 3)) / 24;
  const int64_t nbin64 = ncfg64 * nb * nb;
  if (nbin64 * 29 > ((int64_t)1 << 31)) return set_err(c, GR_E_CAPACITY, "4PCF histogram too large");
  const int nbin = (int)nbin64;
  const int64_t n = c->n;
  // largest |gradient| one clique adds to one vertex: four roots, each with
  // a 4-product cotangent times three weights and three pair terms times one
  const double w = c->wmax;
  const double c4 = max_abs(cot2, nbin) + max_abs(cot3, nbin);
  const double cd = max_abs(cotN, 6 * (int64_t)nbin) + max_abs(cotR, 6 * (int64_t)nbin);
  const double gscale = fix_scale(4.0 * (c4 * w * w * w + 3.0 * cd * w));
  std::vector<double> cot((size_t)14 * nbin, 0.0);
  std::memcpy(cot.data(), cot2, sizeof(double) * nbin);
  if (cot3) std::memcpy(cot.data() + nbin, cot3, sizeof(double) * nbin);
  if (cotN) std::memcpy(cot.data() + 2 * (size_t)nbin, cotN, sizeof(double) * 6 * nbin);
  if (cotR) std::memcpy(cot.data() + 8 * (size_t)nbin, cotR, sizeof(double) * 6 * nbin);
  c->cot.reserve(14 * (int64_t)nbin);
  c->gfix.reserve(2 * n + 2);
  c->work.reserve(4);
  c->stats.reserve(8);
  GR_CUDA_TRY(cudaMemcpyAsync(c->cot.p, cot.data(), sizeof(double) * cot.size(),
                              cudaMemcpyHostToDevice, s));
  GR_CUDA_TRY(cudaEventRecord(c->ev[0], s));
  const bool reuse = c->csr_valid;
  if (!reuse) {
    build_index(c);
    build_csr(c);
  }
  GR_CUDA_TRY(cudaEventRecord(c->ev[1], s));
  if (c->csr.max_deg > 1024)
    return set_err(c, GR_E_CAPACITY, "4PCF: a point has more than 1024 larger-label neighbours");
  GR_CUDA_TRY(cudaMemsetAsync(c->gfix.p, 0, sizeof(unsigned long long) * (2 * n + 2), s));
  GR_CUDA_TRY(cudaMemsetAsync(c->stats.p, 0, sizeof(unsigned long long) * 8, s));
  QuadParams Q{};
  Q.nbins = nb;
  Q.ncfg = (int)ncfg64;
  Q.tetra = 0;
  Q.cap = round_cap(c->csr.max_deg, 32, 1024);
  make_rank_tables(Q.rank, nb, 4);
  Q.P = c->P;
  Q.geo = quad_geometric(c, Q.cap, nb);
  std::memset(&c->st, 0, sizeof(c->st));
  Q.order = root_order(c, s, &Q.above, &Q.nclass);
  launch_adj4(c->index.view(), c->csr.view(), Q, c->cot.p, gscale, c->gfix.p, c->gfix.p + n,
              c->stats.p, c->work.p, s);
  unsigned long long st[8];
  GR_CUDA_TRY(cudaMemcpyAsync(st, c->stats.p, sizeof(st), cudaMemcpyDeviceToHost, s));
  finish_grad(c, gscale, grad_w, c->ev[1]);
  if (st[3] != 0)
    return set_err(c, GR_E_CAPACITY, "4PCF: label offsets within a row exceed the hash key range");
  c->st.ms_graph = reuse ? 0.0 : ev_ms(c->ev[0], c->ev[1]);
  c->st.ms_total = c->st.ms_graph + c->st.ms_query;
  c->st.n_points = n;
  c->st.n_edges = 2 * c->csr.n_edges;
  c->st.upper_edges = c->csr.n_edges;
  c->st.tuples = (int64_t)st[0];
  c->st.rooted = (int64_t)st[1];
  c->st.probes = (int64_t)st[2];
  c->st.kernel_launches =
      (reuse ? 0 : c->index.launches + c->csr.launches) + 2 + (Q.order ? kRootOrderLaunches : 0);
  GR_API_END(c)
}

// ----------------------------------------------------------- batched regions --
int gr_set_regions(gr_ctx* c, int32_t nsplit) {
  GR_API_BEGIN(c)
  if (nsplit < 0 || nsplit > 64) return set_err(c, GR_E_ARG, "nsplit must be in 0..64");
  c->nsplit = nsplit;
  c->region_mode = nsplit > 0 ? 1 : 0;
  c->regions.set_split();
  c->regions.release_graph();
  GR_API_END(c)
}

int gr_set_region_ids(gr_ctx* c, const int32_t* region_of_point, int32_t nregions) {
  GR_API_BEGIN(c)
  if (!c->cat_set) return set_err(c, GR_E_ARG, "catalogue not set (gr_set_catalog)");
  if (nregions < 1 || nregions > (1 << 20)) return set_err(c, GR_E_ARG, "nregions must be in 1..2^20");
  if (c->n > 0 && !region_of_point) return set_err(c, GR_E_ARG, "null region ids");
  c->regions.set_ids(region_of_point, c->n, nregions, c->stream());
  c->region_mode = 2;
  GR_API_END(c)
}

int gr_set_mocks(gr_ctx* c, int32_t nmocks, const int64_t* n_data, const int64_t* n_rand) {
  GR_API_BEGIN(c)
  if (!c->cat_set) return set_err(c, GR_E_ARG, "catalogue not set (gr_set_catalog)");
  if (nmocks < 1 || nmocks > (1 << 20)) return set_err(c, GR_E_ARG, "nmocks must be in 1..2^20");
  if (!n_data || !n_rand) return set_err(c, GR_E_ARG, "null mock sizes");
  c->regions.set_mocks(n_data, n_rand, nmocks, c->n, c->stream());
  c->region_mode = 3;
  GR_API_END(c)
}

// The region layout of the current split, catalogue and binning, planned on
// first use (pair parameters, weight mode, grid resolution).  rmax_cells:
// the caller reads the layout with the rmax-wide cell kernels (graph
// build), so a layout of rmax/2 cells is planned again.
static void ensure_regions(gr_ctx* c, cudaStream_t s, bool rmax_cells) {
  if (c->regions.valid && (!rmax_cells || c->regions.grid_sub == 1)) return;
  // pair parameters from the catalogue's coordinate bound
  c->index.build(c->xyz.p, c->w.p, nullptr, c->n, c->n_data, c->rmax, s);
  make_pair_params(c->P, c->rmin, c->rmax, c->nbins, c->nmu, c->logbins, c->index.coord_max,
                   c->precision == 1);
  c->csr_valid = false;
  // dense regions: cells of rmax/2 and the tile sweep
  int sub = 1;
  if (!rmax_cells) {
    if (c->autotune == 1) sub = 0;
    if (c->autotune == 2 + kPairTile2) sub = 2;
  }
  c->regions.plan(c->xyz.p, c->n, c->n_data, c->rmax, c->nsplit, s, sub, kDenseCellPoints);
  // mocks carry their own galaxy / random split and normalisation: always
  // the fixed-point sums
  c->batch_weighted = !c->uniform || c->region_mode == 3;
  c->batch_fscale = fix_scale(c->wmax * c->wmax);
}

// Device work of one batched call: region layout, histogram reset, pair sweep.
static void enqueue_batched(gr_ctx* c, cudaStream_t s) {
  const int nh = c->nbins * c->nmu * 4;
  c->regions.enqueue_layout(c->xyz.p, c->w.p, s);
  GR_CUDA_TRY(cudaMemsetAsync(c->bcnt.p, 0, sizeof(unsigned long long) * nh, s));
  GR_CUDA_TRY(cudaMemsetAsync(c->bfix.p, 0, sizeof(unsigned long long) * 2 * nh, s));
  GR_CUDA_TRY(cudaMemsetAsync(c->bstats.p, 0, sizeof(unsigned long long) * 8, s));
  launch_pair2(c->regions.view(), c->P, c->batch_weighted, c->bcnt.p, c->bfix.p, c->batch_fscale,
               c->bstats.p, c->bwork.p, s, c->batch_variant);
}

// 2PCF sums of one histogram set (nh counts and 2nh fixed-point words) into
// the caller's arrays.
static void pair_outputs(const gr_ctx* c, bool weighted, double fscale,
                         const unsigned long long* hc, const unsigned long long* hf, double* N2,
                         double* N3, int64_t* counts, double* catsum) {
  const int nbm = c->nbins * c->nmu, nh = nbm * 4;
  std::vector<double> hs(nh, 0.0);
  if (weighted) {
    for (int k = 0; k < nh; ++k) hs[k] = fix_value(hf[k], hf[nh + k], fscale);
  } else {
    for (int cat = 0; cat < 4; ++cat) {
      const int nr = (cat >> 1) + (cat & 1);
      const double prod = uniform_product(c->w_gal, c->w_ran, 2 - nr, nr);
      for (int k = 0; k < nbm; ++k) hs[k + nbm * cat] = (double)hc[k + nbm * cat] * prod;
    }
  }
  for (int k = 0; k < nbm; ++k) {
    if (N2) N2[k] = ((hs[k] + hs[k + nbm]) + hs[k + 2 * nbm]) + hs[k + 3 * nbm];
    if (N3) N3[k] = hs[k + 3 * nbm];
  }
  if (counts)
    for (int k = 0; k < nh; ++k) counts[k] = (int64_t)hc[k];
  if (catsum)
    for (int k = 0; k < nh; ++k) catsum[k] = hs[k];
}

int gr_count_2pcf_batched(gr_ctx* c, double* N2, double* N3, int64_t* counts, double* catsum) {
  GR_API_BEGIN(c)
  require_ready(c);
  if (c->region_mode == 0) return set_err(c, GR_E_ARG, "regions not set (gr_set_regions, gr_set_region_ids or gr_set_mocks)");
  ensure_events(c);
  for (int k = 0; k < 2; ++k)
    if (!c->bev[k]) GR_CUDA_TRY(cudaEventCreateWithFlags(&c->bev[k], cudaEventDisableTiming));
  // the batched work runs on the context's own stream (capturable), ordered
  // after and before the caller's stream
  cudaStream_t us = c->stream(), s = c->own;
  const int nbm = c->nbins * c->nmu, nh = nbm * 4;
  GR_CUDA_TRY(cudaEventRecord(c->bev[0], us));
  GR_CUDA_TRY(cudaStreamWaitEvent(s, c->bev[0], 0));
  GR_CUDA_TRY(cudaEventRecord(c->ev[0], s));
  ensure_regions(c, s, false);
  if (!c->regions.exec) {
    c->bcnt.reserve(nh);
    c->bfix.reserve(2 * nh);
    c->bstats.reserve(8);
    c->bwork.reserve(4);
    // lay out once, pick the pair-sweep variant on this layout, then run
    // eagerly and capture the same work for replay
    c->batch_variant = kPairWarpCell;
    c->regions.enqueue_layout(c->xyz.p, c->w.p, s);
    c->batch_variant = pick_pair2_variant(c, c->regions.view(), c->batch_weighted, c->batch_fscale,
                                          c->bcnt.p, c->bfix.p, c->bstats.p, c->bwork.p, s);
    enqueue_batched(c, s);
    GR_CUDA_TRY(cudaStreamSynchronize(s));
    c->regions.release_graph();
    GR_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue_batched(c, s);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(s, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    GR_CUDA_TRY(cudaStreamEndCapture(s, &c->regions.graph));
    GR_CUDA_TRY(cudaGraphInstantiate(&c->regions.exec, c->regions.graph, 0));
    GR_CUDA_TRY(cudaEventRecord(c->ev[0], s));
  }
  GR_CUDA_TRY(cudaGraphLaunch(c->regions.exec, s));
  GR_CUDA_TRY(cudaEventRecord(c->ev[1], s));
  std::vector<unsigned long long> hc(nh), hf(2 * nh, 0ull);
  unsigned long long st[8];
  GR_CUDA_TRY(cudaMemcpyAsync(hc.data(), c->bcnt.p, sizeof(unsigned long long) * nh, cudaMemcpyDeviceToHost, s));
  if (c->batch_weighted)
    GR_CUDA_TRY(cudaMemcpyAsync(hf.data(), c->bfix.p, sizeof(unsigned long long) * 2 * nh, cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaMemcpyAsync(st, c->bstats.p, sizeof(st), cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaEventRecord(c->bev[1], s));
  GR_CUDA_TRY(cudaStreamWaitEvent(us, c->bev[1], 0));
  GR_CUDA_TRY(cudaStreamSynchronize(s));
  pair_outputs(c, c->batch_weighted, c->batch_fscale, hc.data(), hf.data(), N2, N3, counts, catsum);
  int64_t rooted = 0;
  for (int k = 0; k < nh; ++k) rooted += (int64_t)hc[k];
  std::memset(&c->st, 0, sizeof(c->st));
  c->st.ms_query = ev_ms(c->ev[0], c->ev[1]);
  c->st.ms_total = c->st.ms_query;
  c->st.n_points = c->regions.n_members;
  c->st.tuples = (int64_t)st[2];
  c->st.rooted = rooted;
  c->st.fp64_rechecks = (int64_t)st[0];
  c->st.candidates = (int64_t)st[1];
  c->st.kernel_launches = 11;
  GR_API_END(c)
}

int gr_count_2pcf_regions(gr_ctx* c, double* N2, double* N3, int64_t* counts, double* catsum) {
  GR_API_BEGIN(c)
  require_ready(c);
  if (c->region_mode == 0) return set_err(c, GR_E_ARG, "regions not set (gr_set_regions, gr_set_region_ids or gr_set_mocks)");
  ensure_events(c);
  cudaStream_t s = c->stream();
  const int nbm = c->nbins * c->nmu, nh = nbm * 4;
  GR_CUDA_TRY(cudaEventRecord(c->ev[0], s));
  ensure_regions(c, s, false);
  const int nreg = c->regions.nreg;
  const size_t tot = (size_t)nreg * nh;
  c->rcnt.reserve(tot);
  c->rfix.reserve(2 * tot);
  c->bstats.reserve(8);
  c->bwork.reserve(4);
  c->regions.enqueue_layout(c->xyz.p, c->w.p, s);
  {
    ZeroList z;
    z.add(c->rcnt.p, sizeof(unsigned long long) * tot);
    z.add(c->rfix.p, sizeof(unsigned long long) * 2 * tot);
    z.add(c->bstats.p, sizeof(unsigned long long) * 8);
    zero_async(z, s);
  }
  GR_CUDA_TRY(cudaEventRecord(c->ev[1], s));
  launch_pair2_tile(c->regions.view(), c->P, c->batch_weighted, c->rcnt.p, c->rfix.p,
                    c->batch_fscale, c->bstats.p, c->bwork.p, s, true);
  GR_CUDA_TRY(cudaEventRecord(c->ev[2], s));
  std::vector<unsigned long long> hc(tot), hf(2 * tot, 0ull);
  unsigned long long st[8];
  GR_CUDA_TRY(cudaMemcpyAsync(hc.data(), c->rcnt.p, sizeof(unsigned long long) * tot, cudaMemcpyDeviceToHost, s));
  if (c->batch_weighted)
    GR_CUDA_TRY(cudaMemcpyAsync(hf.data(), c->rfix.p, sizeof(unsigned long long) * 2 * tot, cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaMemcpyAsync(st, c->bstats.p, sizeof(st), cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaStreamSynchronize(s));
  int64_t rooted = 0;
  for (int r = 0; r < nreg; ++r) {
    const size_t o = (size_t)r * nh;
    pair_outputs(c, c->batch_weighted, c->batch_fscale, hc.data() + o, hf.data() + 2 * o,
                 N2 ? N2 + (size_t)r * nbm : nullptr, N3 ? N3 + (size_t)r * nbm : nullptr,
                 counts ? counts + o : nullptr, catsum ? catsum + o : nullptr);
  }
  for (size_t k = 0; k < tot; ++k) rooted += (int64_t)hc[k];
  std::memset(&c->st, 0, sizeof(c->st));
  c->st.ms_index = ev_ms(c->ev[0], c->ev[1]);
  c->st.ms_query = ev_ms(c->ev[1], c->ev[2]);
  c->st.ms_total = ev_ms(c->ev[0], c->ev[2]);
  c->st.n_points = c->regions.n_members;
  c->st.tuples = (int64_t)st[2];
  c->st.rooted = rooted;
  c->st.fp64_rechecks = (int64_t)st[0];
  c->st.candidates = (int64_t)st[1];
  c->st.kernel_launches = 11;
  GR_API_END(c)
}

int gr_count_3pcf_batched(gr_ctx* c, double* N2, double* N3, int64_t* counts, double* catsum) {
  GR_API_BEGIN(c)
  require_ready(c);
  if (c->region_mode == 0) return set_err(c, GR_E_ARG, "regions not set (gr_set_regions, gr_set_region_ids or gr_set_mocks)");
  ensure_events(c);
  cudaStream_t s = c->stream();
  const int nmu = c->nmu;
  const int ncfg = (int)(((int64_t)c->nbins * (c->nbins + 1) * (c->nbins + 2)) / 6);
  const int nbin = ncfg * nmu, nh = nbin * 4;
  GR_CUDA_TRY(cudaEventRecord(c->ev[0], s));
  ensure_regions(c, s, true);
  const bool weighted = c->batch_weighted;
  // mocks carry no global galaxy / random split: one scale for every product
  double fscale[4];
  for (int nr = 0; nr < 4; ++nr)
    fscale[nr] = c->region_mode == 3 ? fix_scale(c->wmax * c->wmax * c->wmax)
                                     : fix_scale(std::pow(c->wgmax, 3 - nr) * std::pow(c->wrmax, nr));
  c->hcnt.reserve(nh);
  c->hfix.reserve(2 * nh);
  c->stats.reserve(8);
  c->work.reserve(4);
  ensure_normal(c, nmu, s);
  c->regions.enqueue_layout(c->xyz.p, c->w.p, s);
  const DevCatalog RC = c->regions.view();
  GR_CUDA_TRY(cudaEventRecord(c->ev[1], s));
  c->csr.build(RC, c->P, s);
  c->csr_valid = false;  // the graph of the region members, not of the catalogue
  GR_CUDA_TRY(cudaEventRecord(c->ev[2], s));
  {
    ZeroList z;
    z.add(c->hcnt.p, sizeof(unsigned long long) * nh);
    z.add(c->hfix.p, sizeof(unsigned long long) * 2 * nh);
    z.add(c->stats.p, sizeof(unsigned long long) * 8);
    zero_async(z, s);
  }
  TriParams T{};
  T.nbins = c->nbins;
  T.nmu = nmu;
  T.ncfg = ncfg;
  T.rsd = nmu >= 2;
  T.equi = 0;
  T.cap = round_cap(c->csr.max_deg, 32, 256);
  T.normal = c->normal_dev.p;
  make_rank_tables(T.rank, c->nbins, 3);
  for (int nr = 0; nr < 4; ++nr) T.fscale[nr] = fscale[nr];
  T.P = c->P;
  T.geo = tri_geometric(c);
  T.maxdeg = (int)std::min<int64_t>(c->csr.max_deg, 1 << 30);
  T.long_geo = c->clique_mode != 1;
  const int tri_launches = 1 + launch_tri3(RC, c->csr.view(), T, weighted, true, c->hcnt.p,
                                           c->hfix.p, c->stats.p, c->work.p, s);
  GR_CUDA_TRY(cudaEventRecord(c->ev[3], s));
  std::vector<unsigned long long> hc(nh), hf(2 * nh, 0ull);
  std::vector<double> hs(nh, 0.0);
  unsigned long long st[8];
  GR_CUDA_TRY(cudaMemcpyAsync(hc.data(), c->hcnt.p, sizeof(unsigned long long) * nh, cudaMemcpyDeviceToHost, s));
  if (weighted)
    GR_CUDA_TRY(cudaMemcpyAsync(hf.data(), c->hfix.p, sizeof(unsigned long long) * 2 * nh, cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaMemcpyAsync(st, c->stats.p, sizeof(st), cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaStreamSynchronize(s));
  if (weighted) {
    for (int k = 0; k < nh; ++k) hs[k] = fix_value(hf[k], hf[nh + k], fscale[k / nbin]);
  } else {
    for (int nr = 0; nr < 4; ++nr) {
      const double prod = uniform_product(c->w_gal, c->w_ran, 3 - nr, nr);
      for (int k = 0; k < nbin; ++k) hs[k + nbin * nr] = (double)hc[k + nbin * nr] * prod;
    }
  }
  for (int k = 0; k < nbin; ++k) {
    if (N2) N2[k] = ((hs[k] + hs[k + nbin]) + hs[k + 2 * nbin]) + hs[k + 3 * nbin];
    if (N3) N3[k] = -hs[k + 3 * nbin];
  }
  if (counts)
    for (int k = 0; k < nh; ++k) counts[k] = (int64_t)hc[k];
  if (catsum)
    for (int k = 0; k < nh; ++k) catsum[k] = hs[k];
  std::memset(&c->st, 0, sizeof(c->st));
  c->st.ms_index = ev_ms(c->ev[0], c->ev[1]);
  c->st.ms_graph = ev_ms(c->ev[1], c->ev[2]);
  c->st.ms_query = ev_ms(c->ev[2], c->ev[3]);
  c->st.ms_total = ev_ms(c->ev[0], c->ev[3]);
  c->st.n_points = c->regions.n_members;
  c->st.n_edges = 2 * c->csr.n_edges;
  c->st.upper_edges = c->csr.n_edges;
  c->st.tuples = (int64_t)st[0];
  c->st.rooted = (int64_t)st[1];
  c->st.probes = (int64_t)st[2];
  c->st.fp64_rechecks = c->csr.rechecks;
  c->st.candidates = c->csr.candidates;
  c->st.kernel_launches = c->csr.launches + tri_launches + 9;
  GR_API_END(c)
}

int gr_regions_info(gr_ctx* c, int32_t* nregions, int64_t* nmembers) {
  GR_API_BEGIN(c)
  if (!c->regions.valid) return set_err(c, GR_E_ARG, "no region layout (call gr_count_2pcf_batched)");
  if (nregions) *nregions = c->regions.nreg;
  if (nmembers) *nmembers = c->regions.n_members;
  GR_API_END(c)
}

int gr_regions_export(gr_ctx* c, int64_t* member_off, int32_t* member_orig, int32_t* member_buffer) {
  GR_API_BEGIN(c)
  RegionLayout& L = c->regions;
  if (!L.valid) return set_err(c, GR_E_ARG, "no region layout (call gr_count_2pcf_batched)");
  // the laid-out members (the last batched call's layout): region r owns
  // the cells [cell_off[r], cell_off[r] + its cell count), its members the
  // labels of those cells
  cudaStream_t s = c->own;
  const int64_t M = L.n_members;
  std::vector<int> mo(M), cs(L.ncell + 1);
  std::vector<uint8_t> mf(M);
  if (M > 0) {
    GR_CUDA_TRY(cudaMemcpyAsync(mo.data(), L.orig.p, sizeof(int) * M, cudaMemcpyDeviceToHost, s));
    GR_CUDA_TRY(cudaMemcpyAsync(mf.data(), L.flags.p, M, cudaMemcpyDeviceToHost, s));
  }
  GR_CUDA_TRY(cudaMemcpyAsync(cs.data(), L.cell_start.p, sizeof(int) * (L.ncell + 1),
                              cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaStreamSynchronize(s));
  // members of each region, ordered by catalogue index
  for (int r = 0; r < L.nreg; ++r) {
    const int64_t b = L.h_mem_off[r], e = L.h_mem_off[r + 1];
    const int c0 = L.h_cell_off[r];
    const int c1 = c0 + (int)L.h_grid[r].ncell;
    const int lb = cs[c0], le = cs[c1];
    if ((int64_t)(le - lb) != e - b) return set_err(c, GR_E_CUDA, "region layout is inconsistent");
    std::vector<std::pair<int, int>> v;
    v.reserve(e - b);
    for (int k = lb; k < le; ++k) v.push_back({mo[k], (mf[k] & FLAG_BUFFER) ? 1 : 0});
    std::sort(v.begin(), v.end());
    for (int64_t k = b; k < e; ++k) {
      if (member_orig) member_orig[k] = v[k - b].first;
      if (member_buffer) member_buffer[k] = v[k - b].second;
    }
  }
  if (member_off)
    for (int r = 0; r <= L.nreg; ++r) member_off[r] = L.h_mem_off[r];
  GR_API_END(c)
}

int gr_get_stats(gr_ctx* c, gr_stats* out) {
  if (!c || !out) return GR_E_ARG;
  *out = c->st;
  return GR_OK;
}

}  // extern "C"
