// Weight adjoint of the 2PCF: gradient of L = sum_b cot2_b N2_b + cot3_b N3_b
// with respect to every signed normalised weight w_k.
//
// N2_b = sum over rooted pairs (i -> j) in bin b of w_i w_j
// (src/gramsci.F90:362-379), so dN2_b/dw_k is the sum of w_j over the
// edges (k, j) in bin b counted from each non-buffer end.  The kernel sweeps
// every ordered pair (the full 27-cell neighbourhood of each root); a pair
// (p, q) with coefficient
//   c = [p root] (cot2 + [p, q random] cot3)[b, mu(p->q)]
//     + [q root] (cot2 + [p, q random] cot3)[b, mu(q->p)]
// adds c w_q to grad_p (and is seen again from q).  Gradients are summed as
// signed 128-bit fixed-point integers, so they are exact up to the
// quantisation of each term and independent of the summation order
// (deterministic).
#include "gr_kernels.cuh"

namespace gr {

namespace {

constexpr int kAdjWarps = 8;
constexpr int kAdjThreads = kAdjWarps * 32;

template <bool F32>
__device__ __forceinline__ bool adj_edge(const DevCatalog& C, const PairParams& P, int p, int q,
                                         const float4& pi, const float4& pj, int& b, int& mf,
                                         int& mr) {
  if (F32) {
    const int r = classify_f32<true>(pi, pj, P, b, mf, mr);
    if (r != 2) return r == 1;
  }
  return edge_f64(C.posd[p], C.posd[q], P, b, mf, mr);
}

// Every root visits its full 27-cell neighbourhood, so each ordered pair is
// seen from both ends and a root only accumulates its own gradient: no
// atomics, one store per root.  The pair test is symmetric (same edge, bins
// swapped mu), so both ends agree on every pair.
// Sparse cells: warp per cell, lanes over staged candidates.
template <bool F32>
__global__ void __launch_bounds__(kAdjThreads) adj2_kernel(DevCatalog C, PairParams P,
                                                           const double* __restrict__ cot2,
                                                           const double* __restrict__ cot3,
                                                           double gscale,
                                                           unsigned long long* __restrict__ g_lo,
                                                           unsigned long long* __restrict__ g_hi,
                                                           int* __restrict__ work) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ float4 s_pos[kAdjWarps][kCellTile];
  __shared__ int s_lab[kAdjWarps][kCellTile];
  const int nbm = P.nbins * P.nmu;
  double* s_c2 = reinterpret_cast<double*>(smem);
  double* s_c3 = s_c2 + nbm;
  for (int k = threadIdx.x; k < nbm; k += blockDim.x) {
    s_c2[k] = cot2[k];
    s_c3[k] = cot3 ? cot3[k] : 0.0;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const int ncell = (int)C.grid.ncell;
  for (;;) {
    int cell = 0;
    if (lane == 0) cell = atomicAdd(work, 1);
    cell = __shfl_sync(0xffffffffu, cell, 0);
    if (cell >= ncell) break;
    const int cb = C.cell_start[cell], ce = C.cell_start[cell + 1];
    if (cb == ce) continue;
    Ranges9 R;
    {
      GridParams g;
      const int* cs;
      int lkey;
      cell_grid(C, cell, g, cs, lkey);
      full_ranges(lkey, g, cs, R);
    }
    int pre[9], total = 0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      pre[k] = total;
      if (k < R.n) total += R.end[k] - R.beg[k];
    }
    for (int t0 = 0; t0 < total; t0 += kCellTile) {
      const int tn = min(kCellTile, total - t0);
      __syncwarp();
      for (int f = lane; f < tn; f += 32) {
        const int q = range9_label(R, pre, t0 + f);
        s_lab[wib][f] = q;
        s_pos[wib][f] = C.pos4[q];
      }
      __syncwarp();
      for (int p = cb; p < ce; ++p) {
        const float4 pi = C.pos4[p];
        const uint8_t fp = C.flags[p];
        Fix128 acc = {0ull, 0ull};
        for (int f = lane; f < tn; f += 32) {
          const int q = s_lab[wib][f];
          if (q == p || both_buffer(pi, s_pos[wib][f])) continue;
          int b, mf, mr;
          if (!adj_edge<F32>(C, P, p, q, pi, s_pos[wib][f], b, mf, mr)) continue;
          const uint8_t fq = C.flags[q];
          const double c = pair_coef(s_c2, s_c3, P.nbins, b, mf, mr, fp, fq);
          if (c != 0.0) fix_acc(acc, c * C.w[q], gscale);
        }
        acc = fix_warp_sum(acc);
        if (lane == 0) {
          if (t0 == 0) {
            g_lo[p] = acc.lo;
            g_hi[p] = acc.hi;
          } else {  // this warp owns p: plain 128-bit add
            const unsigned long long lo = g_lo[p] + acc.lo;
            g_hi[p] = g_hi[p] + acc.hi + (lo < acc.lo ? 1ull : 0ull);
            g_lo[p] = lo;
          }
        }
      }
    }
  }
}

// Dense cells: block per cell, thread per root, candidates broadcast from
// shared memory.
template <bool F32, int NT>
__global__ void __launch_bounds__(NT) adj2_dense_kernel(DevCatalog C, PairParams P,
                                                        const double* __restrict__ cot2,
                                                        const double* __restrict__ cot3,
                                                        double gscale,
                                                        unsigned long long* __restrict__ g_lo,
                                                        unsigned long long* __restrict__ g_hi,
                                                        int* __restrict__ work) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int TILE = 512;
  __shared__ float4 s_pos[TILE];
  __shared__ int s_lab[TILE];
  __shared__ uint8_t s_flag[TILE];
  __shared__ double s_w[TILE];
  __shared__ int s_cell;
  const int nbm = P.nbins * P.nmu;
  double* s_c2 = reinterpret_cast<double*>(smem);
  double* s_c3 = s_c2 + nbm;
  for (int k = threadIdx.x; k < nbm; k += NT) {
    s_c2[k] = cot2[k];
    s_c3[k] = cot3 ? cot3[k] : 0.0;
  }
  const int ncell = (int)C.grid.ncell;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_cell = atomicAdd(work, 1);
    __syncthreads();
    const int cell = s_cell;
    if (cell >= ncell) break;
    const int cb = C.cell_start[cell], ce = C.cell_start[cell + 1];
    if (cb == ce) continue;
    Ranges9 R;
    {
      GridParams g;
      const int* cs;
      int lkey;
      cell_grid(C, cell, g, cs, lkey);
      full_ranges(lkey, g, cs, R);
    }
    int pre[9], total = 0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      pre[k] = total;
      if (k < R.n) total += R.end[k] - R.beg[k];
    }
    for (int rb = cb; rb < ce; rb += NT) {
      const int p = rb + threadIdx.x;
      const bool act = p < ce;
      float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
      uint8_t fp = 0;
      if (act) {
        pi = C.pos4[p];
        fp = C.flags[p];
      }
      Fix128 acc = {0ull, 0ull};
      for (int t0 = 0; t0 < total; t0 += TILE) {
        const int tn = min(TILE, total - t0);
        __syncthreads();
        for (int f = threadIdx.x; f < tn; f += NT) {
          const int q = range9_label(R, pre, t0 + f);
          s_lab[f] = q;
          s_pos[f] = C.pos4[q];
          s_flag[f] = C.flags[q];
          s_w[f] = C.w[q];
        }
        __syncthreads();
        if (!act) continue;
        for (int f = 0; f < tn; ++f) {
          const int q = s_lab[f];
          if (q == p || both_buffer(pi, s_pos[f])) continue;
          int b, mf, mr;
          if (!adj_edge<F32>(C, P, p, q, pi, s_pos[f], b, mf, mr)) continue;
          const double c = pair_coef(s_c2, s_c3, P.nbins, b, mf, mr, fp, s_flag[f]);
          if (c != 0.0) fix_acc(acc, c * s_w[f], gscale);
        }
      }
      if (act) {
        g_lo[p] = acc.lo;
        g_hi[p] = acc.hi;
      }
    }
  }
}

// grad (catalogue order) = fixed-point gradients (label order) / scale
__global__ void grad_finish_kernel(int n, const int* __restrict__ orig,
                                   const unsigned long long* __restrict__ g_lo,
                                   const unsigned long long* __restrict__ g_hi, double inv_scale,
                                   double* __restrict__ grad) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x)
    grad[orig[p]] = fix_to_double(g_lo[p], g_hi[p], inv_scale);
}

}  // namespace

void launch_adj2(const DevCatalog& C, const PairParams& P, const double* cot2, const double* cot3,
                 double gscale, unsigned long long* g_lo, unsigned long long* g_hi, int* work,
                 cudaStream_t s, int variant) {
  if (C.n <= 0) return;
  const size_t smem = sizeof(double) * 2 * (size_t)P.nbins * P.nmu;
  GR_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int), s));
  // the forward sweep's choice of layout: block per cell for the dense
  // variants (plain or queued), warp per cell otherwise
  const bool dense = variant == kPairDense128 || variant == kPairDense256 ||
                     variant == kPairDenseQ128 || variant == kPairDenseQ256;
  const bool small = variant == kPairDense128 || variant == kPairDenseQ128;
  if (dense) {
#define GR_ADJ_DENSE(F, NT)                                                                    \
  do {                                                                                         \
    auto k = adj2_dense_kernel<F, NT>;                                                         \
    GR_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    int per_sm = 1;                                                                            \
    GR_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NT, smem));          \
    int64_t blocks = (int64_t)std::max(1, per_sm) * sm_count();                                       \
    if (blocks > C.grid.ncell) blocks = std::max<int64_t>(1, C.grid.ncell);                    \
    k<<<(unsigned)blocks, NT, smem, s>>>(C, P, cot2, cot3, gscale, g_lo, g_hi, work);          \
  } while (0)
    if (P.f32) {
      if (small) GR_ADJ_DENSE(true, 128); else GR_ADJ_DENSE(true, 256);
    } else {
      if (small) GR_ADJ_DENSE(false, 128); else GR_ADJ_DENSE(false, 256);
    }
#undef GR_ADJ_DENSE
    GR_CHECK_LAUNCH();
    return;
  }
  int64_t blocks = (C.grid.ncell + kAdjWarps - 1) / kAdjWarps;
  if (blocks > (int64_t)4 * sm_count()) blocks = (int64_t)4 * sm_count();
  if (blocks < 1) blocks = 1;
  if (P.f32) {
    GR_CUDA_TRY(cudaFuncSetAttribute(adj2_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
    adj2_kernel<true><<<(unsigned)blocks, kAdjThreads, smem, s>>>(C, P, cot2, cot3, gscale, g_lo,
                                                                  g_hi, work);
  } else {
    GR_CUDA_TRY(cudaFuncSetAttribute(adj2_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
    adj2_kernel<false><<<(unsigned)blocks, kAdjThreads, smem, s>>>(C, P, cot2, cot3, gscale, g_lo,
                                                                   g_hi, work);
  }
  GR_CHECK_LAUNCH();
}

void launch_grad_finish(int n, const int* orig, const unsigned long long* g_lo,
                        const unsigned long long* g_hi, double gscale, double* grad,
                        cudaStream_t s) {
  if (n <= 0) return;
  const int blocks = (int)std::min<int64_t>(((int64_t)n + 255) / 256, (int64_t)8 * sm_count());
  grad_finish_kernel<<<blocks, 256, 0, s>>>(n, orig, g_lo, g_hi, 1.0 / gscale, grad);
  GR_CHECK_LAUNCH();
}

}  // namespace gr
