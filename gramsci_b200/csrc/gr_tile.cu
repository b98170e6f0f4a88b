// Tile pair sweep for dense cells: the 2PCF pair binning of gr_pair.cu
// (create_graph + query_graph_2pcf, src/gramsci.F90:288-379) reorganised for
// cells holding tens to hundreds of points.
//
// A warp takes a cell from the work counter; its lanes hold 32 of the
// cell's points as roots.  The forward candidates (labels above the roots in
// the half stencil) are staged 32 at a time in the warp's own shared-memory
// tile, as separate x / y / z / buffer-flag arrays, and every lane tests all
// 32 against its root with packed FP32x2 arithmetic (two candidates per
// instruction) on the squared separation, without a square root, against the
// outer bounds of the guard band.  Each lane records its hits in a 32-bit
// mask; after the tile the masks are compacted into a per-warp queue and the
// hits are binned 32 at a time with every lane busy: exact classification
// (FP32 with the guard band, FP64 inside it), then the two rooted updates of
// the pair, as in the other sweeps.  No block barrier is taken.
//
// On grids of cells at least rmax/2 wide (GridParams::sub = 2) the stencil
// is two cells on every axis: 15.6 rmax^3 of candidate volume per root
// against 27 rmax^3 with cells at least rmax wide, for the same 4.2 rmax^3
// of neighbour volume.
//
// Histograms are private to each warp in shared memory when they fit (32-bit
// counts, flushed to the global 64-bit counts before any could overflow, and
// 128-bit fixed-point sums for weighted catalogues), else updated with
// global atomics.  With per-region output (batched regions) each region has
// its own histogram: a warp flushes its private copy into the region of its
// cell whenever that region changes.
//
// The FP64 form (precision mode 1) stages the candidates' FP64 positions and
// tests membership with the reference arithmetic; every hit is binned by the
// exact FP64 predicate.
#include "gr_kernels.cuh"

namespace gr {

namespace {

constexpr int kTileWarps = 8;
constexpr int kTileThreads = kTileWarps * 32;
// resident blocks per SM the register allocation is sized for: 3 (at most
// 85 registers); the adjoint on cells of rmax/2 runs best at 4 (64
// registers, no spills; measured on the 3M-point adjoint catalogue: 23.5
// against 27.8 ms, while the forward sweep is faster at 3: 19.4 against
// 20.4 ms)
#ifndef GR_TILE_MIN_BLOCKS
#define GR_TILE_MIN_BLOCKS 3
#endif
constexpr int kTileQueue = 32 * 32;  // one tile's hits at most
constexpr float kBufferPush = 1.0e30f;  // added to d2 of a pair of two buffer points

// Exact bins of a pair that passed the outer membership bounds: FP32 with
// the guard band (classify_f32), FP64 reference arithmetic inside it.
// Returns false when the pair is not an edge.
template <bool F32>
__device__ __forceinline__ bool tile_bins(const DevCatalog& C, const PairParams& P, int p, int q,
                                          const float4 pi, const float4 pj, int& bin, int& muf,
                                          int& mur, unsigned long long& rechecks) {
  if (F32) {
    const int r = classify_f32<true>(pi, pj, P, bin, muf, mur);
    if (r != 2) return r == 1;
    rechecks++;
  }
  return edge_f64(C.posd[p], C.posd[q], P, bin, muf, mur);
}

// Shared memory of one warp: candidate tile (structure of arrays), labels,
// the chunk's root positions and the hit queue.
struct TileWarp {
  float x[32], y[32], z[32], w[32];
  int q[32];
  uint8_t fq[32], fr[32];  // flags of the tile's candidates and of the chunk's roots
  double wq[32], wr[32];   // weights of the same (weighted sums and adjoint)
  float4 root[32];
  uint16_t queue[kTileQueue];
  int rb[16], rpre[16];  // candidate ranges of the current chunk: begin, prefix
  // adjoint: signed 64-bit fixed-point gradient partials of the chunk's
  // roots and of the tile's candidates (at most 32 terms each before they
  // are merged into the 128-bit totals after every tile)
  unsigned long long groot[32], gcand[32];
};

// Weight adjoint arguments (ADJ mode): cotangents of N2 / N3 (nbins*nmu
// each, cot3 may be null) and the 128-bit gradient totals in label order.
struct TileAdj {
  const double* cot2;
  const double* cot3;
  double gscale;
  unsigned long long* g_lo;
  unsigned long long* g_hi;
};
// FP64 positions of the tile (FP64 form only)
struct TileWarpD {
  double x[32], y[32], z[32];
};

// F32: FP32 membership tests and binning with the guard band (else FP64).
// WHIST: histograms private to each warp in shared memory (else global).
// SUB: 1 (cells >= rmax, 5 ranges) or 2 (cells >= rmax/2, 13 ranges).
// PERREG: one histogram per region (C.cell_region), region r's counts at
// g_cnt + r*nh and fixed-point words at g_fix + 2*r*nh.
// ADJ: the 2PCF weight adjoint instead of histograms: each edge adds
// coef * w_q to dL/dw_p and coef * w_p to dL/dw_q (pair_coef).
template <bool F32, bool WEIGHTED, bool WHIST, int SUB, bool PERREG, bool ADJ>
__global__ void __launch_bounds__(kTileThreads, (ADJ && SUB == 2) ? 4 : GR_TILE_MIN_BLOCKS)
    pair2_tile_kernel(DevCatalog C, PairParams P, unsigned long long* __restrict__ g_cnt,
                      unsigned long long* __restrict__ g_fix, double fscale,
                      unsigned long long* __restrict__ stats, int* __restrict__ work, TileAdj A) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ TileWarp s_tw[kTileWarps];
  __shared__ TileWarpD s_twd[F32 ? 1 : kTileWarps];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  TileWarp& T = s_tw[wib];
  TileWarpD& TD = s_twd[F32 ? 0 : wib];
  const int nbm = P.nbins * P.nmu;
  const int nh = nbm * 4;
  // per-warp histograms: counts (32-bit), then fixed-point lo and hi words
  const size_t wstride = WHIST ? (size_t)nh * (WEIGHTED ? 20 : 4) : 0;
  unsigned int* w_cnt = reinterpret_cast<unsigned int*>(smem + wstride * wib);
  unsigned long long* w_lo =
      reinterpret_cast<unsigned long long*>(smem + wstride * wib + (size_t)nh * 4);
  unsigned long long* w_hi = w_lo + nh;
  if (WHIST) {
    for (int k = lane; k < nh; k += 32) {
      w_cnt[k] = 0u;
      if (WEIGHTED) {
        w_lo[k] = 0ull;
        w_hi[k] = 0ull;
      }
    }
  }
  if (ADJ) {
    T.groot[lane] = 0ull;
    T.gcand[lane] = 0ull;
  }
  __syncwarp();
  const int ncell = (int)C.grid.ncell;
  constexpr int NR = SUB == 2 ? 13 : 5;
  unsigned long long rechecks = 0, cands = 0, pairs = 0;
  unsigned int pending = 0;  // edges drained since the last flush (warp-uniform)
  int region = 0;            // region whose histogram the warp holds (PERREG)
  unsigned long long* o_cnt = g_cnt;
  unsigned long long* o_fix = g_fix;

  auto flush = [&]() {
    if (!WHIST) return;
    __syncwarp();
    for (int k = lane; k < nh; k += 32) {
      if (w_cnt[k]) {
        atomicAdd(&o_cnt[k], (unsigned long long)w_cnt[k]);
        w_cnt[k] = 0u;
      }
      if (WEIGHTED && (w_lo[k] | w_hi[k])) {
        fix_merge(&o_fix[k], &o_fix[nh + k], w_lo[k], w_hi[k]);
        w_lo[k] = 0ull;
        w_hi[k] = 0ull;
      }
    }
    __syncwarp();
  };

  for (;;) {
    int cell = 0;
    if (lane == 0) cell = atomicAdd(work, 1);
    cell = __shfl_sync(0xffffffffu, cell, 0);
    if (cell >= ncell) break;
    const int cb = C.cell_start[cell], ce = C.cell_start[cell + 1];
    if (cb == ce) continue;
    if (PERREG) {
      const int r = C.cell_region[cell];
      if (r != region) {
        flush();
        region = r;
        o_cnt = g_cnt + (size_t)r * nh;
        o_fix = g_fix + (size_t)r * 2 * nh;
      }
    }
    GridParams g;
    const int* cs;
    int lkey;
    cell_grid(C, cell, g, cs, lkey);
    for (int c0 = cb; c0 < ce; c0 += 32) {
      // this chunk's candidate ranges, starting just after its first root
      int rbeg = 0, rend = 0;
      if (SUB == 2) {
        if (lane < NR) forward_range2_slot(lane, c0 + 1, lkey, g, cs, rbeg, rend);
      } else {
        Ranges R5;
        forward_ranges(c0, lkey, g, cs, R5);
#pragma unroll
        for (int k = 0; k < 5; ++k)
          if (lane == k) {
            rbeg = R5.beg[k];
            rend = R5.end[k];
          }
      }
      int len = lane < NR ? rend - rbeg : 0;
      int incl = len;
#pragma unroll
      for (int o = 1; o < 16; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      const int total = __shfl_sync(0xffffffffu, incl, NR - 1);
      if (lane < NR) {
        T.rb[lane] = rbeg;
        T.rpre[lane] = incl - len;
      }
      const int p = c0 + lane;
      const bool act = p < ce;
      // lanes without a root hold a NaN position: no candidate is ever a hit
      float4 pi = make_float4(__int_as_float(0x7fc00000), 0.f, 0.f, 0.f);
      double4 pd = make_double4(__longlong_as_double(0x7ff8000000000000ll), 0.0, 0.0, 0.0);
      if (act) {
        pi = C.pos4[p];
        if (!F32) pd = C.posd[p];
      }
      T.root[lane] = pi;
      if (act) {
        T.fr[lane] = C.flags[p];
        if (WEIGHTED || ADJ) T.wr[lane] = C.w[p];
      }
      const float pwb = (act && pi.w != 0.0f) ? kBufferPush : 0.0f;
      const float2 npx = make_float2(-pi.x, -pi.x), npy = make_float2(-pi.y, -pi.y),
                   npz = make_float2(-pi.z, -pi.z), pwb2 = make_float2(pwb, pwb);
      const float hi = P.rmax2_hi, lo = P.rmin2_lo;
      // one compare per candidate: |d2 - mid| < half, widened by far more
      // than the subtraction's rounding (2^-24 of rmax2_hi), accepts every
      // d2 in (lo, hi); the few pairs just outside the band that it also
      // accepts are rejected by the exact classification of the binning
      const float midv = 0.5f * (hi + lo);
      const float halfv = __int_as_float(__float_as_int(0.5f * (hi - lo) + 1e-6f * fabsf(hi)) + 4);
      const float2 nmid2 = make_float2(-midv, -midv);
      const double pwbd = pwb;
      __syncwarp();
      int kr = 0;  // range of the tile's first candidate (warp-uniform)
      for (int t0 = 0; t0 < total; t0 += 32) {
        // stage candidate t0 + lane
        const int f = t0 + lane;
        while (kr + 1 < NR && t0 >= T.rpre[kr + 1]) ++kr;
        int k = kr;
        while (k + 1 < NR && f >= T.rpre[k + 1]) ++k;
        const int tn = min(32, total - t0);
        if (lane < tn) {
          const int q = T.rb[k] + (f - T.rpre[k]);
          const float4 c = C.pos4[q];
          T.x[lane] = c.x;
          T.y[lane] = c.y;
          T.z[lane] = c.z;
          T.w[lane] = c.w;
          T.q[lane] = q;
          T.fq[lane] = C.flags[q];
          if (WEIGHTED || ADJ) T.wq[lane] = C.w[q];
          if (!F32) {
            const double4 cd = C.posd[q];
            TD.x[lane] = cd.x;
            TD.y[lane] = cd.y;
            TD.z[lane] = cd.z;
          }
        } else {
          T.x[lane] = __int_as_float(0x7fc00000);  // NaN: never a hit
          T.y[lane] = 0.f;
          T.z[lane] = 0.f;
          T.w[lane] = 0.f;
          T.q[lane] = 0x7fffffff;
          if (!F32) {
            TD.x[lane] = __longlong_as_double(0x7ff8000000000000ll);
            TD.y[lane] = 0.0;
            TD.z[lane] = 0.0;
          }
        }
        __syncwarp();
        unsigned m = 0u;
        if (act && !F32) {
          // the reference's squared separation, separate roundings
#pragma unroll 8
          for (int j = 0; j < 32; ++j) {
            const double dx = __dsub_rn(TD.x[j], pd.x);
            const double dy = __dsub_rn(TD.y[j], pd.y);
            const double dz = __dsub_rn(TD.z[j], pd.z);
            double sd = __dmul_rn(dx, dx);
            sd = __dadd_rn(sd, __dmul_rn(dy, dy));
            sd = __dadd_rn(sd, __dmul_rn(dz, dz));
            sd = __fma_rn((double)T.w[j], pwbd, sd);
            if (sd <= P.rmax2 && !(P.rmin > 0.0 && sd <= P.rmin2)) m |= 1u << j;
          }
          if (t0 == 0) {
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (T.q[j] <= p) m &= ~(1u << j);
          }
          cands += (unsigned long long)tn;
        } else if (act) {
#pragma unroll
          for (int j = 0; j < 32; j += 2) {
            const float2 cx = *reinterpret_cast<const float2*>(&T.x[j]);
            const float2 cy = *reinterpret_cast<const float2*>(&T.y[j]);
            const float2 cz = *reinterpret_cast<const float2*>(&T.z[j]);
            const float2 cw = *reinterpret_cast<const float2*>(&T.w[j]);
            const float2 dx = __fadd2_rn(cx, npx);
            const float2 dy = __fadd2_rn(cy, npy);
            const float2 dz = __fadd2_rn(cz, npz);
            float2 d2 = __fmul2_rn(dx, dx);
            d2 = __ffma2_rn(dy, dy, d2);
            d2 = __ffma2_rn(dz, dz, d2);
            d2 = __ffma2_rn(cw, pwb2, d2);
            const float2 dm = __fadd2_rn(d2, nmid2);
            if (fabsf(dm.x) < halfv) m |= 1u << j;
            if (fabsf(dm.y) < halfv) m |= 2u << j;
          }
          // the first tile holds own-cell candidates with labels at or
          // below some lanes' roots
          if (t0 == 0) {
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (T.q[j] <= p) m &= ~(1u << j);
          }
          cands += (unsigned long long)tn;
        }
        // compact the hits into the warp's queue, then bin them
        const int cnt = __popc(m);
        int ex = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, ex, o);
          if (lane >= o) ex += v;
        }
        const int tot = __shfl_sync(0xffffffffu, ex, 31);
        int pos = ex - cnt;
        while (m) {
          const int j = __ffs(m) - 1;
          T.queue[pos++] = (uint16_t)((lane << 5) | j);
          m &= m - 1u;
        }
        __syncwarp();
        for (int e0 = 0; e0 < tot; e0 += 32) {
          if (e0 + lane < tot) {
            const int ent = T.queue[e0 + lane];
            const int r = ent >> 5, j = ent & 31;
            const int pr = c0 + r, q = T.q[j];
            const float4 a = T.root[r];
            const float4 b = make_float4(T.x[j], T.y[j], T.z[j], T.w[j]);
            int bin = 1, mf = 1, mr = 1;
            if (ADJ) {
              if (tile_bins<F32>(C, P, pr, q, a, b, bin, mf, mr, rechecks)) {
                const uint8_t fp = T.fr[r], fq = T.fq[j];
                pairs += (!(fp & FLAG_BUFFER) || !(fq & FLAG_BUFFER)) ? 1 : 0;
                const double cf = pair_coef(A.cot2, A.cot3, P.nbins, bin, mf, mr, fp, fq);
                if (cf != 0.0) {
                  atomicAdd(&T.groot[r], (unsigned long long)__double2ll_rn(cf * T.wq[j] * A.gscale));
                  atomicAdd(&T.gcand[j], (unsigned long long)__double2ll_rn(cf * T.wr[r] * A.gscale));
                }
              }
            } else if (tile_bins<F32>(C, P, pr, q, a, b, bin, mf, mr, rechecks)) {
              const uint8_t fp = T.fr[r], fq = T.fq[j];
              const bool root_p = !(fp & FLAG_BUFFER), root_q = !(fq & FLAG_BUFFER);
              const int rp = fp & FLAG_RANDOM, rq = fq & FLAG_RANDOM;
              pairs += (root_p || root_q) ? 1 : 0;
              const double prod = WEIGHTED ? T.wr[r] * T.wq[j] : 0.0;
              if (root_p) {
                const int kh = (bin - 1) + P.nbins * (mf - 1) + nbm * (2 * rp + rq);
                if (WHIST) {
                  atomicAdd(&w_cnt[kh], 1u);
                  if (WEIGHTED) fix_add(&w_lo[kh], &w_hi[kh], prod, fscale);
                } else {
                  atomicAdd(&o_cnt[kh], 1ull);
                  if (WEIGHTED) fix_add(&o_fix[kh], &o_fix[nh + kh], prod, fscale);
                }
              }
              if (root_q) {
                const int kh = (bin - 1) + P.nbins * (mr - 1) + nbm * (2 * rq + rp);
                if (WHIST) {
                  atomicAdd(&w_cnt[kh], 1u);
                  if (WEIGHTED) fix_add(&w_lo[kh], &w_hi[kh], prod, fscale);
                } else {
                  atomicAdd(&o_cnt[kh], 1ull);
                  if (WEIGHTED) fix_add(&o_fix[kh], &o_fix[nh + kh], prod, fscale);
                }
              }
            }
          }
        }
        if (ADJ) {
          // merge the tile's gradient partials into the 128-bit totals
          __syncwarp();
          const long long vc = (long long)T.gcand[lane];
          if (vc != 0) fix_add_int(&A.g_lo[T.q[lane]], &A.g_hi[T.q[lane]], vc);
          T.gcand[lane] = 0ull;
          const long long vr = (long long)T.groot[lane];
          if (vr != 0) fix_add_int(&A.g_lo[c0 + lane], &A.g_hi[c0 + lane], vr);
          T.groot[lane] = 0ull;
        }
        // a 32-bit count grows by at most 2 per binned pair
        pending += (unsigned)tot;
        if (pending > (1u << 30)) {
          flush();
          pending = 0u;
        }
        __syncwarp();
      }
    }
  }
  flush();
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    rechecks += __shfl_xor_sync(0xffffffffu, rechecks, o);
    pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
    cands += __shfl_xor_sync(0xffffffffu, cands, o);
  }
  if (lane == 0) {
    if (rechecks) atomicAdd(&stats[0], rechecks);
    if (cands) atomicAdd(&stats[1], cands);
    if (pairs) atomicAdd(&stats[2], pairs);
  }
}

}  // namespace

size_t pair2_tile_smem_bytes(const PairParams& P, bool weighted) {
  const size_t nh = (size_t)P.nbins * P.nmu * 4;
  return nh * (weighted ? 20 : 4) * kTileWarps;
}

void launch_pair2_tile(const DevCatalog& C, const PairParams& P, bool weighted,
                       unsigned long long* g_cnt, unsigned long long* g_fix, double fscale,
                       unsigned long long* stats, int* work, cudaStream_t s, bool per_region) {
  if (C.n <= 0) return;
  if (per_region && !C.cell_region) throw Error{-1, "per-region output needs a region layout"};
  size_t smem = pair2_tile_smem_bytes(P, weighted);
  const bool whist = smem <= kMaxTileHistSmem;
  if (!whist) smem = 0;
  GR_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int), s));
  const int sub = C.grid.sub == 2 ? 2 : 1;
#define GR_TILE_LAUNCH(F, W, H, S)                                                           \
  do {                                                                                        \
    auto k = per_region ? pair2_tile_kernel<F, W, H, S, true, false>                         \
                        : pair2_tile_kernel<F, W, H, S, false, false>;                        \
    GR_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,         \
                                     (int)smem));                                             \
    int per_sm = 1;                                                                           \
    GR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kTileThreads, smem)); \
    int64_t blocks = (int64_t)std::max(1, per_sm) * sm_count();                               \
    const int64_t need = (C.grid.ncell + kTileWarps - 1) / kTileWarps;                        \
    if (blocks > need) blocks = std::max<int64_t>(1, need);                                   \
    k<<<(unsigned)blocks, kTileThreads, smem, s>>>(C, P, g_cnt, g_fix, fscale, stats, work,   \
                                                   TileAdj{});                                \
  } while (0)
#define GR_TILE_S(F, W, H)                                                                   \
  do {                                                                                        \
    if (sub == 2) GR_TILE_LAUNCH(F, W, H, 2); else GR_TILE_LAUNCH(F, W, H, 1);                \
  } while (0)
#define GR_TILE_H(F, W)                                                                      \
  do {                                                                                        \
    if (whist) GR_TILE_S(F, W, true); else GR_TILE_S(F, W, false);                            \
  } while (0)
  if (P.f32) {
    if (weighted) GR_TILE_H(true, true); else GR_TILE_H(true, false);
  } else {
    if (weighted) GR_TILE_H(false, true); else GR_TILE_H(false, false);
  }
#undef GR_TILE_H
#undef GR_TILE_S
#undef GR_TILE_LAUNCH
  GR_CHECK_LAUNCH();
}

void launch_adj2_tile(const DevCatalog& C, const PairParams& P, const double* cot2,
                      const double* cot3, double gscale, unsigned long long* g_lo,
                      unsigned long long* g_hi, unsigned long long* stats, int* work,
                      cudaStream_t s) {
  if (C.n <= 0) return;
  GR_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int), s));
  const TileAdj A{cot2, cot3, gscale, g_lo, g_hi};
  const int sub = C.grid.sub == 2 ? 2 : 1;
#define GR_ADJT_LAUNCH(F, S)                                                                  \
  do {                                                                                        \
    auto k = pair2_tile_kernel<F, true, false, S, false, true>;                               \
    int per_sm = 1;                                                                           \
    GR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kTileThreads, 0));  \
    int64_t blocks = (int64_t)std::max(1, per_sm) * sm_count();                               \
    const int64_t need = (C.grid.ncell + kTileWarps - 1) / kTileWarps;                        \
    if (blocks > need) blocks = std::max<int64_t>(1, need);                                   \
    k<<<(unsigned)blocks, kTileThreads, 0, s>>>(C, P, nullptr, nullptr, 1.0, stats, work, A); \
  } while (0)
  if (P.f32) {
    if (sub == 2) GR_ADJT_LAUNCH(true, 2); else GR_ADJT_LAUNCH(true, 1);
  } else {
    if (sub == 2) GR_ADJT_LAUNCH(false, 2); else GR_ADJT_LAUNCH(false, 1);
  }
#undef GR_ADJT_LAUNCH
  GR_CHECK_LAUNCH();
}

}  // namespace gr
