// CSR adjacency build: replaces create_graph (src/gramsci.F90:288-348) with
// its kd-tree range queries (src/kdtree2.F90:1204-1363), distance sort and
// O(k^2) id sort (src/sorting_module.F90:36-47).
//
// Two passes over the half stencil of every cell (warp per cell, candidates
// staged in shared memory, lanes over candidate labels): a count pass giving
// the upper degrees, an exclusive scan giving row offsets, and a fill pass
// writing each row.  Candidates are
// visited in increasing label order and compacted with a warp ballot, so
// rows come out sorted without a sort.  Each undirected edge is stored once,
// in the row of its smaller label, with the bins seen from both ends.
#include "gr_index.cuh"

namespace gr {

namespace {

constexpr int kGraphWarps = 8;
constexpr int kGraphThreads = kGraphWarps * 32;

// Decide one candidate pair exactly.  Returns true for an edge.
template <bool F32, bool NEED_BINS>
__device__ __forceinline__ bool pair_edge(const DevCatalog& C, const PairParams& P, int p, int q,
                                          const float4& pi, const float4& pj, int& bin, int& muf,
                                          int& mur, unsigned long long& rechecks) {
  if (F32) {
    int r = classify_f32<NEED_BINS>(pi, pj, P, bin, muf, mur);
    if (r != 2) return r == 1;
    rechecks++;
  }
  return edge_f64(C.posd[p], C.posd[q], P, bin, muf, mur);
}

// Warp-per-cell sweep shared by the count and fill passes.  A warp takes a
// cell, computes the forward candidate ranges once for all its points and
// stages the candidates (labels and float4 positions) in shared memory in
// tiles of kCellTile.  Every root p of the cell is then tested against the
// staged candidates with label > p, lanes over candidates.  FILL=false
// counts upper degrees (and full degrees); FILL=true writes the rows, with
// a per-row cursor carried across tiles in `cursor`.
template <bool F32, bool FILL>
__global__ void __launch_bounds__(kGraphThreads) csr_cells_kernel(
    DevCatalog C, PairParams P, int* __restrict__ deg_up, int* __restrict__ deg_full,
    const int64_t* __restrict__ row_ptr, unsigned long long* __restrict__ rec,
    int* __restrict__ cursor, unsigned long long* __restrict__ stats, int* __restrict__ work) {
  __shared__ float4 s_pos[kGraphWarps][kCellTile];
  __shared__ int s_lab[kGraphWarps][kCellTile];
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  unsigned long long rechecks = 0, cands = 0;
  unsigned long long maxdeg = 0;
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
      const bool last_tile = t0 + kCellTile >= total;
      __syncwarp();
      for (int f = lane; f < tn; f += 32) {
        const int q = range_label(R, pre, t0 + f);
        s_lab[wib][f] = q;
        s_pos[wib][f] = C.pos4[q];
      }
      __syncwarp();
      for (int p = cb; p < ce; ++p) {
        // flattened index p - cb is p itself (range 0 starts at cb)
        const int fstart = max(0, p - cb + 1 - t0);
        if (fstart >= tn) continue;
        const float4 pi = C.pos4[p];
        int off = 0;
        int64_t rowb = 0, rowe = 0;
        if (FILL) {
          rowb = row_ptr[p];
          rowe = row_ptr[p + 1];
          off = (t0 == 0) ? 0 : cursor[p];
        }
        int cnt = 0;
        for (int f0 = fstart; f0 < tn; f0 += 32) {
          const int f = f0 + lane;
          bool e = false;
          int q = 0, b = 0, mf = 0, mr = 0;
          if (f < tn) {
            q = s_lab[wib][f];
            e = pair_edge<F32, FILL>(C, P, p, q, pi, s_pos[wib][f], b, mf, mr, rechecks);
            if (!FILL && e) atomicAdd(&deg_full[q], 1);
          }
          const unsigned m = __ballot_sync(0xffffffffu, e);
          if (FILL && e) {
            const int64_t pos = rowb + off + __popc(m & lt);
            if (pos < rowe)  // the count pass decided the same edges
              rec[pos] = ((unsigned long long)pack_meta(b, mf, mr) << 32) | (uint32_t)q;
          }
          off += __popc(m);
          cnt += __popc(m);
        }
        if (lane == 0) {
          if (FILL) {
            if (!last_tile) cursor[p] = off;
          } else {
            const int d = deg_up[p] + cnt;
            deg_up[p] = d;
            atomicAdd(&deg_full[p], cnt);
            if (last_tile) maxdeg = maxdeg > (unsigned long long)d ? maxdeg : (unsigned long long)d;
            cands += (unsigned long long)(tn - fstart);
          }
        }
        __syncwarp();
      }
    }
  }
  if (!FILL) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) rechecks += __shfl_xor_sync(0xffffffffu, rechecks, o);
    if (lane == 0) {
      if (rechecks) atomicAdd(&stats[0], rechecks);
      if (cands) atomicAdd(&stats[1], cands);
      if (maxdeg) atomicMax(&stats[2], maxdeg);
    }
  }
}

int graph_blocks(int64_t ncell) {
  int64_t b = (ncell + kGraphWarps - 1) / kGraphWarps;
  int64_t cap = 148 * 8;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace

void UpperCSR::build(const DevCatalog& C, const PairParams& P, cudaStream_t s) {
  n = C.n;
  launches = 0;
  deg_up.reserve(n + 1);
  deg_full.reserve(n + 1);
  cursor.reserve(n + 1);
  row_ptr.reserve(n + 1);
  stats.reserve(4);
  work.reserve(2);
  GR_CUDA_TRY(cudaMemsetAsync(deg_up.p, 0, sizeof(int) * (n + 1), s));
  GR_CUDA_TRY(cudaMemsetAsync(deg_full.p, 0, sizeof(int) * (n + 1), s));
  GR_CUDA_TRY(cudaMemsetAsync(stats.p, 0, sizeof(unsigned long long) * 4, s));
  GR_CUDA_TRY(cudaMemsetAsync(work.p, 0, sizeof(int) * 2, s));
  const int blocks = graph_blocks(C.grid.ncell);
  if (n > 0) {
    if (P.f32)
      csr_cells_kernel<true, false><<<blocks, kGraphThreads, 0, s>>>(
          C, P, deg_up.p, deg_full.p, nullptr, nullptr, nullptr, stats.p, work.p);
    else
      csr_cells_kernel<false, false><<<blocks, kGraphThreads, 0, s>>>(
          C, P, deg_up.p, deg_full.p, nullptr, nullptr, nullptr, stats.p, work.p);
    launches++;
    GR_CHECK_LAUNCH();
  }
  scan_i32_to_i64(deg_up.p, row_ptr.p, n, s, scan_tmp);
  launches += 3;
  GR_CUDA_TRY(cudaMemcpyAsync(&n_edges, row_ptr.p + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  unsigned long long hs[3] = {0, 0, 0};
  GR_CUDA_TRY(cudaMemcpyAsync(hs, stats.p, sizeof(hs), cudaMemcpyDeviceToHost, s));
  GR_CUDA_TRY(cudaStreamSynchronize(s));
  rechecks = (int64_t)hs[0];
  candidates = (int64_t)hs[1];
  max_deg = (int64_t)hs[2];
  rec.reserve(n_edges);
  if (n > 0 && n_edges > 0) {
    if (P.f32)
      csr_cells_kernel<true, true><<<blocks, kGraphThreads, 0, s>>>(
          C, P, nullptr, nullptr, row_ptr.p, rec.p, cursor.p, stats.p, work.p + 1);
    else
      csr_cells_kernel<false, true><<<blocks, kGraphThreads, 0, s>>>(
          C, P, nullptr, nullptr, row_ptr.p, rec.p, cursor.p, stats.p, work.p + 1);
    launches++;
    GR_CHECK_LAUNCH();
  }
}

}  // namespace gr
