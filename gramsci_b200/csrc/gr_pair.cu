// 2PCF pair binning straight from the cell sweep: replaces create_graph +
// query_graph_2pcf (src/gramsci.F90:288-379) without materialising the
// graph.  Each unordered pair is tested once (half stencil, q > p) and
// contributes to both of its rooted directions, as the reference's symmetric
// graph does: root p with mu(p->q) if p is not a buffer point, root q with
// mu(q->p) if q is not.
//
// Histograms are privatised per block in shared memory: 64-bit counts per
// (bin, mu, category) and, for weighted catalogues, 128-bit fixed-point sums
// of w_i w_j per category (see fix_add).
#include "gr_kernels.cuh"

namespace gr {

namespace {

constexpr int kPairWarps = 8;
constexpr int kPairThreads = kPairWarps * 32;

// SHIST: histogram privatised in shared memory (false: atomics straight to
// the global histogram, for bin counts too large for shared memory).
// Warp per cell: the forward candidates of a cell are computed once and
// staged in shared memory (tiles of kCellTile), then every root of the cell
// is tested against the staged candidates with larger labels.
template <bool F32, bool WEIGHTED, bool SHIST>
__global__ void __launch_bounds__(kPairThreads) pair2_kernel(DevCatalog C, PairParams P,
                                                             unsigned long long* __restrict__ g_cnt,
                                                             unsigned long long* __restrict__ g_fix,
                                                             double fscale,
                                                             unsigned long long* __restrict__ stats,
                                                             int* __restrict__ work) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ float4 s_pos[kPairWarps][kCellTile];
  __shared__ int s_lab[kPairWarps][kCellTile];
  const int nbm = P.nbins * P.nmu;
  const int nh = nbm * 4;
  unsigned long long* s_cnt = SHIST ? reinterpret_cast<unsigned long long*>(smem) : g_cnt;
  unsigned long long* s_lo = SHIST ? s_cnt + nh : g_fix;
  unsigned long long* s_hi = s_lo + nh;
  if (SHIST) {
    for (int k = threadIdx.x; k < nh; k += blockDim.x) {
      s_cnt[k] = 0ull;
      if (WEIGHTED) {
        s_lo[k] = 0ull;
        s_hi[k] = 0ull;
      }
    }
    __syncthreads();
  }

  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int ncell = (int)C.grid.ncell;
  unsigned long long rechecks = 0, cands = 0, pairs = 0;
  for (;;) {
    int cell = 0;
    if (lane == 0) cell = atomicAdd(work, 1);
    cell = __shfl_sync(0xffffffffu, cell, 0);
    if (cell >= ncell) break;
    const int cb = C.cell_start[cell], ce = C.cell_start[cell + 1];
    if (cb == ce) continue;
    Ranges R;
    {
      GridParams g;
      const int* cs;
      int lkey;
      cell_grid(C, cell, g, cs, lkey);
      forward_ranges(cb - 1, lkey, g, cs, R);
    }
    int pre[5], total = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      pre[k] = total;
      if (k < R.n) total += R.end[k] - R.beg[k];
    }
    for (int t0 = 0; t0 < total; t0 += kCellTile) {
      const int tn = min(kCellTile, total - t0);
      __syncwarp();
      for (int f = lane; f < tn; f += 32) {
        const int q = range_label(R, pre, t0 + f);
        s_lab[wib][f] = q;
        s_pos[wib][f] = C.pos4[q];
      }
      __syncwarp();
      for (int p = cb; p < ce; ++p) {
        const int fstart = max(0, p - cb + 1 - t0);
        if (fstart >= tn) continue;
        const float4 pi = C.pos4[p];
        const uint8_t fp = C.flags[p];
        const bool root_p = !(fp & FLAG_BUFFER);
        const int rp = fp & FLAG_RANDOM;
        const double wp = WEIGHTED ? C.w[p] : 0.0;
        for (int f = fstart + lane; f < tn; f += 32) {
          const int q = s_lab[wib][f];
          if (both_buffer(pi, s_pos[wib][f])) continue;
          int b, mf, mr;
          bool e;
          if (F32) {
            const int r = classify_f32<true>(pi, s_pos[wib][f], P, b, mf, mr);
            if (r == 2) {
              rechecks++;
              e = edge_f64(C.posd[p], C.posd[q], P, b, mf, mr);
            } else {
              e = r == 1;
            }
          } else {
            e = edge_f64(C.posd[p], C.posd[q], P, b, mf, mr);
          }
          if (!e) continue;
          const uint8_t fq = C.flags[q];
          const int rq = fq & FLAG_RANDOM;
          pairs += (root_p || !(fq & FLAG_BUFFER)) ? 1 : 0;
          double prod = 0.0;
          if (WEIGHTED) prod = wp * C.w[q];
          if (root_p) {
            const int k = (b - 1) + P.nbins * (mf - 1) + nbm * (2 * rp + rq);
            atomicAdd(&s_cnt[k], 1ull);
            if (WEIGHTED) fix_add(&s_lo[k], &s_hi[k], prod, fscale);
          }
          if (!(fq & FLAG_BUFFER)) {
            const int k = (b - 1) + P.nbins * (mr - 1) + nbm * (2 * rq + rp);
            atomicAdd(&s_cnt[k], 1ull);
            if (WEIGHTED) fix_add(&s_lo[k], &s_hi[k], prod, fscale);
          }
        }
        if (lane == 0) cands += (unsigned long long)(tn - fstart);
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    rechecks += __shfl_xor_sync(0xffffffffu, rechecks, o);
    pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
  }
  if (lane == 0) {
    if (rechecks) atomicAdd(&stats[0], rechecks);
    if (cands) atomicAdd(&stats[1], cands);
    if (pairs) atomicAdd(&stats[2], pairs);
  }
  if (SHIST) {
    __syncthreads();
    for (int k = threadIdx.x; k < nh; k += blockDim.x) {
      if (s_cnt[k]) {
        atomicAdd(&g_cnt[k], s_cnt[k]);
        if (WEIGHTED) fix_merge(&g_fix[k], &g_fix[nh + k], s_lo[k], s_hi[k]);
      }
    }
  }
}


// Queued variant of the warp-per-cell sweep: the membership test (FP32
// squared separation, FP64 inside the guard band at rmin and rmax) runs for
// every candidate, the edges go to a per-warp queue, and the bins, the
// line-of-sight cosines and the histogram updates run 32 edges at a time
// with every lane busy.  Pays off where most candidates are not edges.
constexpr int kPairQueue = 64;

template <bool F32, bool WEIGHTED, bool SHIST>
__global__ void __launch_bounds__(kPairThreads) pair2_queue_kernel(
    DevCatalog C, PairParams P, unsigned long long* __restrict__ g_cnt,
    unsigned long long* __restrict__ g_fix, double fscale, unsigned long long* __restrict__ stats,
    int* __restrict__ work) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ float4 s_pos[kPairWarps][kCellTile];
  __shared__ int s_lab[kPairWarps][kCellTile];
  __shared__ int s_qi[kPairWarps][kPairQueue];      // root index in the cell
  __shared__ uint8_t s_qf[kPairWarps][kPairQueue];  // tile index of the neighbour
  const int nbm = P.nbins * P.nmu;
  const int nh = nbm * 4;
  unsigned long long* s_cnt = SHIST ? reinterpret_cast<unsigned long long*>(smem) : g_cnt;
  unsigned long long* s_lo = SHIST ? s_cnt + nh : g_fix;
  unsigned long long* s_hi = s_lo + nh;
  if (SHIST) {
    for (int k = threadIdx.x; k < nh; k += blockDim.x) {
      s_cnt[k] = 0ull;
      if (WEIGHTED) {
        s_lo[k] = 0ull;
        s_hi[k] = 0ull;
      }
    }
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int ncell = (int)C.grid.ncell;
  unsigned long long rechecks = 0, cands = 0, pairs = 0;
  int cb = 0;
  // bins and both rooted updates of one queued pair (p, q)
  auto drain_one = [&](int e) {
    const int f = s_qf[wib][e];
    const int p = cb + s_qi[wib][e];
    const int q = s_lab[wib][f];
    int b = 1, mf = 1, mr = 1;
    bool ok;
    if (F32) {
      const int r = classify_f32<true>(C.pos4[p], s_pos[wib][f], P, b, mf, mr);
      if (r == 2) {
        rechecks++;
        ok = edge_f64(C.posd[p], C.posd[q], P, b, mf, mr);
      } else {
        ok = r == 1;
      }
    } else {
      ok = edge_f64(C.posd[p], C.posd[q], P, b, mf, mr);
    }
    if (!ok) return;  // cannot happen: the membership test decided the same pair
    const uint8_t fp = C.flags[p], fq = C.flags[q];
    const bool root_p = !(fp & FLAG_BUFFER), root_q = !(fq & FLAG_BUFFER);
    const int rp = fp & FLAG_RANDOM, rq = fq & FLAG_RANDOM;
    pairs += (root_p || root_q) ? 1 : 0;
    const double prod = WEIGHTED ? C.w[p] * C.w[q] : 0.0;
    if (root_p) {
      const int k = (b - 1) + P.nbins * (mf - 1) + nbm * (2 * rp + rq);
      atomicAdd(&s_cnt[k], 1ull);
      if (WEIGHTED) fix_add(&s_lo[k], &s_hi[k], prod, fscale);
    }
    if (root_q) {
      const int k = (b - 1) + P.nbins * (mr - 1) + nbm * (2 * rq + rp);
      atomicAdd(&s_cnt[k], 1ull);
      if (WEIGHTED) fix_add(&s_lo[k], &s_hi[k], prod, fscale);
    }
  };
  for (;;) {
    int cell = 0;
    if (lane == 0) cell = atomicAdd(work, 1);
    cell = __shfl_sync(0xffffffffu, cell, 0);
    if (cell >= ncell) break;
    cb = C.cell_start[cell];
    const int ce = C.cell_start[cell + 1];
    if (cb == ce) continue;
    Ranges R;
    {
      GridParams g;
      const int* cs;
      int lkey;
      cell_grid(C, cell, g, cs, lkey);
      forward_ranges(cb - 1, lkey, g, cs, R);
    }
    int pre[5], total = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      pre[k] = total;
      if (k < R.n) total += R.end[k] - R.beg[k];
    }
    int qn = 0;
    for (int t0 = 0; t0 < total; t0 += kCellTile) {
      const int tn = min(kCellTile, total - t0);
      __syncwarp();
      for (int f = lane; f < tn; f += 32) {
        const int q = range_label(R, pre, t0 + f);
        s_lab[wib][f] = q;
        s_pos[wib][f] = C.pos4[q];
      }
      __syncwarp();
      for (int p = cb; p < ce; ++p) {
        const int i = p - cb;
        const int fstart = max(0, i + 1 - t0);
        if (fstart >= tn) continue;
        // p itself is candidate i of the flattened ranges
        const float4 pi = (i >= t0 && i - t0 < tn) ? s_pos[wib][i - t0] : C.pos4[p];
        for (int f0 = fstart; f0 < tn; f0 += 32) {
          const int f = f0 + lane;
          bool e = false;
          if (f < tn && !both_buffer(pi, s_pos[wib][f])) {
            int r = F32 ? member_f32(pi, s_pos[wib][f], P) : 2;
            if (r == 2) {
              int b, mf, mr;
              rechecks++;
              r = edge_f64(C.posd[p], C.posd[s_lab[wib][f]], P, b, mf, mr) ? 1 : 0;
            }
            e = r == 1;
          }
          const unsigned m = __ballot_sync(0xffffffffu, e);
          if (e) {
            s_qi[wib][qn + __popc(m & lt)] = i;
            s_qf[wib][qn + __popc(m & lt)] = (uint8_t)f;
          }
          qn += __popc(m);
          if (qn >= 32) {
            __syncwarp();
            drain_one(qn - 32 + lane);
            qn -= 32;
            __syncwarp();
          }
        }
        if (lane == 0) cands += (unsigned long long)(tn - fstart);
      }
      // the tile's staged candidates are about to be replaced
      __syncwarp();
      if (lane < qn) drain_one(lane);
      qn = 0;
      __syncwarp();
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    rechecks += __shfl_xor_sync(0xffffffffu, rechecks, o);
    pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
  }
  if (lane == 0) {
    if (rechecks) atomicAdd(&stats[0], rechecks);
    if (cands) atomicAdd(&stats[1], cands);
    if (pairs) atomicAdd(&stats[2], pairs);
  }
  if (SHIST) {
    __syncthreads();
    for (int k = threadIdx.x; k < nh; k += blockDim.x) {
      if (s_cnt[k]) {
        atomicAdd(&g_cnt[k], s_cnt[k]);
        if (WEIGHTED) fix_merge(&g_fix[k], &g_fix[nh + k], s_lo[k], s_hi[k]);
      }
    }
  }
}

// Dense-cell variant: one block per cell, one thread per root, the cell's
// forward candidates staged in shared memory tiles and read by all threads
// at the same address (broadcast), so each candidate costs one shared load
// per warp instead of one per lane.  Suits cells holding many points (the
// warp-per-cell variant suits sparse cells, where most threads here would
// idle).  Same contributions, same histogram layout.
template <bool F32, bool WEIGHTED, bool SHIST, int NT>
__global__ void __launch_bounds__(NT) pair2_dense_kernel(DevCatalog C, PairParams P,
                                                         unsigned long long* __restrict__ g_cnt,
                                                         unsigned long long* __restrict__ g_fix,
                                                         double fscale,
                                                         unsigned long long* __restrict__ stats,
                                                         int* __restrict__ work) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int TILE = 512;
  __shared__ float4 s_pos[TILE];
  __shared__ int s_lab[TILE];
  __shared__ uint8_t s_flag[TILE];
  __shared__ double s_w[WEIGHTED ? TILE : 1];
  __shared__ int s_cell;
  const int nbm = P.nbins * P.nmu;
  const int nh = nbm * 4;
  unsigned long long* s_cnt = SHIST ? reinterpret_cast<unsigned long long*>(smem) : g_cnt;
  unsigned long long* s_lo = SHIST ? s_cnt + nh : g_fix;
  unsigned long long* s_hi = s_lo + nh;
  if (SHIST) {
    for (int k = threadIdx.x; k < nh; k += NT) {
      s_cnt[k] = 0ull;
      if (WEIGHTED) {
        s_lo[k] = 0ull;
        s_hi[k] = 0ull;
      }
    }
  }
  const int ncell = (int)C.grid.ncell;
  unsigned long long rechecks = 0, cands = 0, pairs = 0;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_cell = atomicAdd(work, 1);
    __syncthreads();
    const int cell = s_cell;
    if (cell >= ncell) break;
    const int cb = C.cell_start[cell], ce = C.cell_start[cell + 1];
    if (cb == ce) continue;
    Ranges R;
    {
      GridParams g;
      const int* cs;
      int lkey;
      cell_grid(C, cell, g, cs, lkey);
      forward_ranges(cb - 1, lkey, g, cs, R);
    }
    int pre[5], total = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      pre[k] = total;
      if (k < R.n) total += R.end[k] - R.beg[k];
    }
    for (int rb = cb; rb < ce; rb += NT) {
      const int p = rb + threadIdx.x;
      const bool act = p < ce;
      float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
      uint8_t fp = 0;
      double wp = 0.0;
      if (act) {
        pi = C.pos4[p];
        fp = C.flags[p];
        if (WEIGHTED) wp = C.w[p];
      }
      const bool root_p = !(fp & FLAG_BUFFER);
      const int rp = fp & FLAG_RANDOM;
      for (int t0 = 0; t0 < total; t0 += TILE) {
        const int tn = min(TILE, total - t0);
        __syncthreads();
        for (int f = threadIdx.x; f < tn; f += NT) {
          const int q = range_label(R, pre, t0 + f);
          s_lab[f] = q;
          s_pos[f] = C.pos4[q];
          s_flag[f] = C.flags[q];
          if (WEIGHTED) s_w[f] = C.w[q];
        }
        __syncthreads();
        if (!act) continue;
        // candidates with label > p: own-cell candidates are the first
        // (ce - cb) flattened entries, labels cb, cb+1, ...
        const int fstart = max(0, p - cb + 1 - t0);
        if (fstart < tn) cands += (unsigned long long)(tn - fstart);
        for (int f = fstart; f < tn; ++f) {
          if (both_buffer(pi, s_pos[f])) continue;
          int b, mf, mr;
          bool e;
          if (F32) {
            const int r = classify_f32<true>(pi, s_pos[f], P, b, mf, mr);
            if (r == 2) {
              rechecks++;
              e = edge_f64(C.posd[p], C.posd[s_lab[f]], P, b, mf, mr);
            } else {
              e = r == 1;
            }
          } else {
            e = edge_f64(C.posd[p], C.posd[s_lab[f]], P, b, mf, mr);
          }
          if (!e) continue;
          const uint8_t fq = s_flag[f];
          const int rq = fq & FLAG_RANDOM;
          pairs += (root_p || !(fq & FLAG_BUFFER)) ? 1 : 0;
          const double prod = WEIGHTED ? wp * s_w[f] : 0.0;
          if (root_p) {
            const int k = (b - 1) + P.nbins * (mf - 1) + nbm * (2 * rp + rq);
            atomicAdd(&s_cnt[k], 1ull);
            if (WEIGHTED) fix_add(&s_lo[k], &s_hi[k], prod, fscale);
          }
          if (!(fq & FLAG_BUFFER)) {
            const int k = (b - 1) + P.nbins * (mr - 1) + nbm * (2 * rq + rp);
            atomicAdd(&s_cnt[k], 1ull);
            if (WEIGHTED) fix_add(&s_lo[k], &s_hi[k], prod, fscale);
          }
        }
      }
    }
  }
  const int lane = threadIdx.x & 31;
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
  if (SHIST) {
    __syncthreads();
    for (int k = threadIdx.x; k < nh; k += NT) {
      if (s_cnt[k]) {
        atomicAdd(&g_cnt[k], s_cnt[k]);
        if (WEIGHTED) fix_merge(&g_fix[k], &g_fix[nh + k], s_lo[k], s_hi[k]);
      }
    }
  }
}

// Dense-cell variant with queued binning: as pair2_dense_kernel, but the
// lanes of a warp walk the staged candidates in step (lanes whose root has
// not reached a candidate yet sit it out), test membership only, and queue
// the edges per warp; bins, cosines and histogram updates run 32 edges at a
// time with every lane busy.
template <bool F32, bool WEIGHTED, bool SHIST, int NT>
__global__ void __launch_bounds__(NT) pair2_dense_queue_kernel(
    DevCatalog C, PairParams P, unsigned long long* __restrict__ g_cnt,
    unsigned long long* __restrict__ g_fix, double fscale, unsigned long long* __restrict__ stats,
    int* __restrict__ work) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int TILE = 512;
  constexpr int NW = NT / 32;
  __shared__ float4 s_pos[TILE];
  __shared__ int s_lab[TILE];
  __shared__ uint8_t s_flag[TILE];
  __shared__ double s_w[WEIGHTED ? TILE : 1];
  __shared__ int s_qp[NW][kPairQueue];       // root label
  __shared__ uint16_t s_qf[NW][kPairQueue];  // tile index of the neighbour
  __shared__ int s_cell;
  const int nbm = P.nbins * P.nmu;
  const int nh = nbm * 4;
  unsigned long long* s_cnt = SHIST ? reinterpret_cast<unsigned long long*>(smem) : g_cnt;
  unsigned long long* s_lo = SHIST ? s_cnt + nh : g_fix;
  unsigned long long* s_hi = s_lo + nh;
  if (SHIST) {
    for (int k = threadIdx.x; k < nh; k += NT) {
      s_cnt[k] = 0ull;
      if (WEIGHTED) {
        s_lo[k] = 0ull;
        s_hi[k] = 0ull;
      }
    }
  }
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int ncell = (int)C.grid.ncell;
  unsigned long long rechecks = 0, cands = 0, pairs = 0;
  auto drain_one = [&](int e) {
    const int p = s_qp[wib][e];
    const int f = s_qf[wib][e];
    const int q = s_lab[f];
    int b = 1, mf = 1, mr = 1;
    bool ok;
    if (F32) {
      const int r = classify_f32<true>(C.pos4[p], s_pos[f], P, b, mf, mr);
      if (r == 2) {
        rechecks++;
        ok = edge_f64(C.posd[p], C.posd[q], P, b, mf, mr);
      } else {
        ok = r == 1;
      }
    } else {
      ok = edge_f64(C.posd[p], C.posd[q], P, b, mf, mr);
    }
    if (!ok) return;  // cannot happen: the membership test decided the same pair
    const uint8_t fp = C.flags[p], fq = s_flag[f];
    const bool root_p = !(fp & FLAG_BUFFER), root_q = !(fq & FLAG_BUFFER);
    const int rp = fp & FLAG_RANDOM, rq = fq & FLAG_RANDOM;
    pairs += (root_p || root_q) ? 1 : 0;
    const double prod = WEIGHTED ? C.w[p] * s_w[f] : 0.0;
    if (root_p) {
      const int k = (b - 1) + P.nbins * (mf - 1) + nbm * (2 * rp + rq);
      atomicAdd(&s_cnt[k], 1ull);
      if (WEIGHTED) fix_add(&s_lo[k], &s_hi[k], prod, fscale);
    }
    if (root_q) {
      const int k = (b - 1) + P.nbins * (mr - 1) + nbm * (2 * rq + rp);
      atomicAdd(&s_cnt[k], 1ull);
      if (WEIGHTED) fix_add(&s_lo[k], &s_hi[k], prod, fscale);
    }
  };
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_cell = atomicAdd(work, 1);
    __syncthreads();
    const int cell = s_cell;
    if (cell >= ncell) break;
    const int cb = C.cell_start[cell], ce = C.cell_start[cell + 1];
    if (cb == ce) continue;
    Ranges R;
    {
      GridParams g;
      const int* cs;
      int lkey;
      cell_grid(C, cell, g, cs, lkey);
      forward_ranges(cb - 1, lkey, g, cs, R);
    }
    int pre[5], total = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      pre[k] = total;
      if (k < R.n) total += R.end[k] - R.beg[k];
    }
    for (int rb = cb; rb < ce; rb += NT) {
      const int p = rb + threadIdx.x;
      const bool act = p < ce;
      const float4 pi = act ? C.pos4[p] : make_float4(0.f, 0.f, 0.f, 0.f);
      for (int t0 = 0; t0 < total; t0 += TILE) {
        const int tn = min(TILE, total - t0);
        __syncthreads();
        for (int f = threadIdx.x; f < tn; f += NT) {
          const int q = range_label(R, pre, t0 + f);
          s_lab[f] = q;
          s_pos[f] = C.pos4[q];
          s_flag[f] = C.flags[q];
          if (WEIGHTED) s_w[f] = C.w[q];
        }
        __syncthreads();
        // candidates with label > p: own-cell candidates are the first
        // (ce - cb) flattened entries, labels cb, cb+1, ...
        const int fstart = act ? max(0, p - cb + 1 - t0) : tn;
        if (fstart < tn) cands += (unsigned long long)(tn - fstart);
        int f0 = fstart;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) f0 = min(f0, __shfl_xor_sync(0xffffffffu, f0, o));
        int qn = 0;
        for (int f = f0; f < tn; ++f) {  // warp-uniform walk over the candidates
          bool e = false;
          if (f >= fstart && !both_buffer(pi, s_pos[f])) {
            int r = F32 ? member_f32(pi, s_pos[f], P) : 2;
            if (r == 2) {
              int b, mf, mr;
              rechecks++;
              r = edge_f64(C.posd[p], C.posd[s_lab[f]], P, b, mf, mr) ? 1 : 0;
            }
            e = r == 1;
          }
          const unsigned m = __ballot_sync(0xffffffffu, e);
          if (e) {
            s_qp[wib][qn + __popc(m & lt)] = p;
            s_qf[wib][qn + __popc(m & lt)] = (uint16_t)f;
          }
          qn += __popc(m);
          if (qn >= 32) {
            __syncwarp();
            drain_one(qn - 32 + lane);
            qn -= 32;
            __syncwarp();
          }
        }
        // the staged tile is replaced after the next block barrier
        __syncwarp();
        if (lane < qn) drain_one(lane);
        __syncwarp();
      }
    }
  }
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
  if (SHIST) {
    __syncthreads();
    for (int k = threadIdx.x; k < nh; k += NT) {
      if (s_cnt[k]) {
        atomicAdd(&g_cnt[k], s_cnt[k]);
        if (WEIGHTED) fix_merge(&g_fix[k], &g_fix[nh + k], s_lo[k], s_hi[k]);
      }
    }
  }
}

}  // namespace

size_t pair2_smem_bytes(const PairParams& P, bool weighted) {
  size_t nh = (size_t)P.nbins * P.nmu * 4;
  return nh * sizeof(unsigned long long) * (weighted ? 3 : 1);
}

void launch_pair2(const DevCatalog& C, const PairParams& P, bool weighted,
                  unsigned long long* g_cnt, unsigned long long* g_fix, double fscale,
                  unsigned long long* stats, int* work, cudaStream_t s, int variant) {
  if (C.n <= 0) return;
  if (variant == kPairTile || variant == kPairTile2 || C.grid.sub == 2) {
    launch_pair2_tile(C, P, weighted, g_cnt, g_fix, fscale, stats, work, s);
    return;
  }
  size_t smem = pair2_smem_bytes(P, weighted);
  const bool shist = smem <= kMaxHistSmem;
  if (!shist) smem = 0;
  GR_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int), s));
  if (variant == kPairDense128 || variant == kPairDense256 || variant == kPairDenseQ128 ||
      variant == kPairDenseQ256) {
    const bool q = variant == kPairDenseQ128 || variant == kPairDenseQ256;
    const bool small = variant == kPairDense128 || variant == kPairDenseQ128;
    int per_sm = 1;
#define GR_DENSE_LAUNCH(F, W, S, NT)                                                          \
  do {                                                                                        \
    auto k = q ? pair2_dense_queue_kernel<F, W, S, NT> : pair2_dense_kernel<F, W, S, NT>;      \
    GR_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,         \
                                     (int)smem));                                             \
    GR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NT, smem));         \
    int64_t blocks = (int64_t)std::max(1, per_sm) * sm_count();                                      \
    if (blocks > C.grid.ncell) blocks = std::max<int64_t>(1, C.grid.ncell);                   \
    k<<<(unsigned)blocks, NT, smem, s>>>(C, P, g_cnt, g_fix, fscale, stats, work);            \
  } while (0)
#define GR_DENSE_NT(F, W, S)                                                                  \
  do {                                                                                        \
    if (small) GR_DENSE_LAUNCH(F, W, S, 128); else GR_DENSE_LAUNCH(F, W, S, 256);             \
  } while (0)
#define GR_DENSE_W(F, S)                                                                      \
  do {                                                                                        \
    if (weighted) GR_DENSE_NT(F, true, S); else GR_DENSE_NT(F, false, S);                     \
  } while (0)
    if (P.f32) {
      if (shist) GR_DENSE_W(true, true); else GR_DENSE_W(true, false);
    } else {
      if (shist) GR_DENSE_W(false, true); else GR_DENSE_W(false, false);
    }
#undef GR_DENSE_W
#undef GR_DENSE_NT
#undef GR_DENSE_LAUNCH
    GR_CHECK_LAUNCH();
    return;
  }
  int64_t blocks = (C.grid.ncell + kPairWarps - 1) / kPairWarps;
  if (blocks > (int64_t)4 * sm_count()) blocks = (int64_t)4 * sm_count();
  if (blocks < 1) blocks = 1;
#define GR_PAIR_LAUNCH(F, W, S)                                                          \
  do {                                                                                   \
    auto k = variant == kPairWarpQueue ? pair2_queue_kernel<F, W, S> : pair2_kernel<F, W, S>; \
    GR_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                                     (int)smem));                                        \
    k<<<(unsigned)blocks, kPairThreads, smem, s>>>(C, P, g_cnt, g_fix, fscale, stats, work);           \
  } while (0)
#define GR_PAIR_LAUNCH_W(F, S)                                                           \
  do {                                                                                   \
    if (weighted) GR_PAIR_LAUNCH(F, true, S); else GR_PAIR_LAUNCH(F, false, S);          \
  } while (0)
  if (P.f32) {
    if (shist) GR_PAIR_LAUNCH_W(true, true); else GR_PAIR_LAUNCH_W(true, false);
  } else {
    if (shist) GR_PAIR_LAUNCH_W(false, true); else GR_PAIR_LAUNCH_W(false, false);
  }
#undef GR_PAIR_LAUNCH_W
#undef GR_PAIR_LAUNCH
  GR_CHECK_LAUNCH();
}

}  // namespace gr
