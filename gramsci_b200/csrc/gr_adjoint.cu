// Weight adjoint of the 2PCF: gradient of L = sum_b cot2_b N2_b + cot3_b N3_b
// with respect to every signed normalised weight w_k.
//
// N2_b = sum over rooted pairs (i -> j) in bin b of w_i w_j
// (src/gramsci.F90:362-379), so dN2_b/dw_k is the sum of w_j over the
// edges (k, j) in bin b counted from each non-buffer end.  The kernel sweeps
// every unordered pair once (the half-stencil cell sweep of the forward
// kernel); a pair (p, q) with coefficient
//   c = [p root] (cot2 + [p, q random] cot3)[b, mu(p->q)]
//     + [q root] (cot2 + [p, q random] cot3)[b, mu(q->p)]
// adds c w_q to grad_p and c w_p to grad_q.  Gradients are summed as signed
// 128-bit fixed-point integers, so they are exact up to the quantisation of
// each term and independent of the summation order (deterministic).
#include "gr_kernels.cuh"

namespace gr {

namespace {

constexpr int kAdjWarps = 8;
constexpr int kAdjThreads = kAdjWarps * 32;

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
        const bool rp = fp & FLAG_RANDOM;
        const double wp = C.w[p];
        Fix128 acc = {0ull, 0ull};
        for (int f = fstart + lane; f < tn; f += 32) {
          const int q = s_lab[wib][f];
          int b, mf, mr;
          bool e;
          if (F32) {
            const int r = classify_f32<true>(pi, s_pos[wib][f], P, b, mf, mr);
            e = (r == 2) ? edge_f64(C.posd[p], C.posd[q], P, b, mf, mr) : (r == 1);
          } else {
            e = edge_f64(C.posd[p], C.posd[q], P, b, mf, mr);
          }
          if (!e) continue;
          const uint8_t fq = C.flags[q];
          const bool rr = rp && (fq & FLAG_RANDOM);
          double c = 0.0;
          if (root_p) {
            const int k = (b - 1) + P.nbins * (mf - 1);
            c += rr ? s_c2[k] + s_c3[k] : s_c2[k];
          }
          if (!(fq & FLAG_BUFFER)) {
            const int k = (b - 1) + P.nbins * (mr - 1);
            c += rr ? s_c2[k] + s_c3[k] : s_c2[k];
          }
          if (c == 0.0) continue;
          fix_acc(acc, c * C.w[q], gscale);
          fix_add(&g_lo[q], &g_hi[q], c * wp, gscale);
        }
        acc = fix_warp_sum(acc);
        if (lane == 0 && (acc.lo | acc.hi)) fix_merge(&g_lo[p], &g_hi[p], acc.lo, acc.hi);
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
                 cudaStream_t s) {
  if (C.n <= 0) return;
  const size_t smem = sizeof(double) * 2 * (size_t)P.nbins * P.nmu;
  GR_CUDA_TRY(cudaMemsetAsync(work, 0, sizeof(int), s));
  int64_t blocks = (C.grid.ncell + kAdjWarps - 1) / kAdjWarps;
  if (blocks > 148 * 4) blocks = 148 * 4;
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
  const int blocks = (int)std::min<int64_t>(((int64_t)n + 255) / 256, 148 * 8);
  grad_finish_kernel<<<blocks, 256, 0, s>>>(n, orig, g_lo, g_hi, 1.0 / gscale, grad);
  GR_CHECK_LAUNCH();
}

}  // namespace gr
