// 2PCF pair binning straight from the cell sweep: replaces create_graph +
// query_graph_2pcf (src/gramsci.F90:288-379) without materialising the
// graph.  Each unordered pair is tested once (half stencil, q > p) and
// contributes to both of its rooted directions, as the reference's symmetric
// graph does: root p with mu(p->q) if p is not a buffer point, root q with
// mu(q->p) if q is not.
//
// Histograms are privatised per block in shared memory: 64-bit counts per
// (bin, mu, category) and, for weighted catalogues, FP64 sums of w_i w_j per
// category (each category sum has a single sign, so it is well conditioned).
#include "gr_kernels.cuh"

namespace gr {

namespace {

constexpr int kPairThreads = 256;

// SHIST: histogram privatised in shared memory (false: atomics straight to
// the global histogram, for bin counts too large for shared memory).
template <bool F32, bool WEIGHTED, bool SHIST>
__global__ void __launch_bounds__(kPairThreads) pair2_kernel(DevCatalog C, PairParams P,
                                                             unsigned long long* __restrict__ g_cnt,
                                                             double* __restrict__ g_sum,
                                                             unsigned long long* __restrict__ stats) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int nbm = P.nbins * P.nmu;
  const int nh = nbm * 4;
  unsigned long long* s_cnt = SHIST ? reinterpret_cast<unsigned long long*>(smem) : g_cnt;
  double* s_sum = SHIST ? reinterpret_cast<double*>(smem + sizeof(unsigned long long) * nh) : g_sum;
  if (SHIST) {
    for (int k = threadIdx.x; k < nh; k += blockDim.x) {
      s_cnt[k] = 0ull;
      if (WEIGHTED) s_sum[k] = 0.0;
    }
    __syncthreads();
  }

  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  unsigned long long rechecks = 0, cands = 0, pairs = 0;
  for (int p = warp; p < C.n; p += nwarps) {
    Ranges R;
    forward_ranges(p, C.cell_key[p], C.grid, C.cell_start, R);
    int pre[5], total = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      pre[k] = total;
      if (k < R.n) total += R.end[k] - R.beg[k];
    }
    const float4 pi = C.pos4[p];
    const uint8_t fp = C.flags[p];
    const bool root_p = !(fp & FLAG_BUFFER);
    const int rp = fp & FLAG_RANDOM;
    const double wp = WEIGHTED ? C.w[p] : 0.0;
    for (int f = lane; f < total; f += 32) {
      int q = range_label(R, pre, f);
      int b, mf, mr;
      bool e;
      if (F32) {
        int r = classify_f32<true>(pi, C.pos4[q], P, b, mf, mr);
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
      pairs += (root_p || !(fq & FLAG_BUFFER)) ? 1 : 0;
      const int rq = fq & FLAG_RANDOM;
      double prod = 0.0;
      if (WEIGHTED) prod = wp * C.w[q];
      if (root_p) {
        int k = (b - 1) + P.nbins * (mf - 1) + nbm * (2 * rp + rq);
        atomicAdd(&s_cnt[k], 1ull);
        if (WEIGHTED) atomicAdd(&s_sum[k], prod);
      }
      if (!(fq & FLAG_BUFFER)) {
        int k = (b - 1) + P.nbins * (mr - 1) + nbm * (2 * rq + rp);
        atomicAdd(&s_cnt[k], 1ull);
        if (WEIGHTED) atomicAdd(&s_sum[k], prod);
      }
    }
    if (lane == 0) cands += (unsigned long long)total;
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
      if (s_cnt[k]) atomicAdd(&g_cnt[k], s_cnt[k]);
      if (WEIGHTED && s_sum[k] != 0.0) atomicAdd(&g_sum[k], s_sum[k]);
    }
  }
}

}  // namespace

size_t pair2_smem_bytes(const PairParams& P, bool weighted) {
  size_t nh = (size_t)P.nbins * P.nmu * 4;
  return nh * sizeof(unsigned long long) + (weighted ? nh * sizeof(double) : 0);
}

void launch_pair2(const DevCatalog& C, const PairParams& P, bool weighted,
                  unsigned long long* g_cnt, double* g_sum, unsigned long long* stats,
                  cudaStream_t s) {
  if (C.n <= 0) return;
  size_t smem = pair2_smem_bytes(P, weighted);
  const bool shist = smem <= kMaxHistSmem;
  if (!shist) smem = 0;
  int64_t warps = C.n;
  int64_t blocks = (warps * 32 + kPairThreads - 1) / kPairThreads;
  if (blocks > 148 * 8) blocks = 148 * 8;
  if (blocks < 1) blocks = 1;
#define GR_PAIR_LAUNCH(F, W, S)                                                          \
  do {                                                                                   \
    auto k = pair2_kernel<F, W, S>;                                                      \
    GR_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,     \
                                     (int)smem));                                        \
    k<<<(unsigned)blocks, kPairThreads, smem, s>>>(C, P, g_cnt, g_sum, stats);           \
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
