// CSR adjacency build: replaces create_graph (src/gramsci.F90:288-348) with
// its kd-tree range queries (src/kdtree2.F90:1204-1363), distance sort and
// O(k^2) id sort (src/sorting_module.F90:36-47).
//
// One pass over the half stencil of every cell (warp per cell, candidates
// staged in shared memory, lanes over candidate labels) writes each row to a
// per-cell scratch region; an exclusive scan of the upper degrees gives the
// row offsets and a compaction kernel moves the rows into place.  Candidates
// are visited in increasing label order and compacted with a warp ballot, so
// rows come out sorted without a sort.  Each undirected edge is stored once,
// in the row of its smaller label, with the bins seen from both ends.
#include <algorithm>

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

// One pass over the half stencil of every cell.  A warp takes a cell,
// computes its forward candidate ranges once for all its points and stages
// the candidates (labels and float4 positions) in shared memory in tiles of
// kCellTile.  Every root p of the cell is tested against the staged
// candidates with label > p, lanes over candidates, with the cheap
// membership test (FP32 separation, FP64 only inside the guard band at rmin
// and rmax).  Edges are compacted with a ballot into a per-warp queue in
// label order, each with its final position; the queue is drained 32 at a
// time, so the radial and mu bins (the costly part) are computed with every
// lane busy.  Rows are written to a scratch area in which each cell owns its
// candidate bound (prefix sums of cell_bound_kernel); root p (local index i)
// of a cell with T forward candidates owns the slots base + i*T - i(i+1)/2
// onward.  compact() moves the rows to CSR order when a caller needs it.
constexpr int kQueue = 64;

// Candidate bound of every cell (scratch slots its rows may need): a cell
// with n points and T forward candidates gives root i at most T - i - 1
// edges, n*T - n(n+1)/2 in all.
__global__ void cell_bound_kernel(DevCatalog C, int64_t* __restrict__ bound) {
  const int ncell = (int)C.grid.ncell;
  for (int cell = blockIdx.x * blockDim.x + threadIdx.x; cell < ncell; cell += gridDim.x * blockDim.x) {
    const int cb = C.cell_start[cell], ce = C.cell_start[cell + 1];
    int64_t b = 0;
    if (ce > cb) {
      Ranges R;
      GridParams g;
      const int* cs;
      int lkey;
      cell_grid(C, cell, g, cs, lkey);
      forward_ranges(cb - 1, lkey, g, cs, R);
      int64_t total = 0;
      for (int k = 0; k < R.n; ++k) total += R.end[k] - R.beg[k];
      const int64_t nloc = ce - cb;
      b = nloc * total - nloc * (nloc + 1) / 2;
    }
    bound[cell] = b;
  }
}

template <bool F32>
// Launch bounds without a minimum block count: the compiler's own choice
// (74-78 registers, three blocks of 8 warps per SM) measured 0.245 ms on the
// 3PCF workload, against 0.278 ms at four blocks (64 registers, spills) and
// 0.290 ms with a minimum of one block (100 registers).  Reserving each
// cell's scratch with an atomic on a cursor when a warp takes the cell
// (instead of cell_bound_kernel and a scan: three launches fewer) measured
// 0.246 against 0.234 ms: the warp then waits for the returned base.
__global__ void __launch_bounds__(kGraphThreads) csr_fill_kernel(
    DevCatalog C, PairParams P, int* __restrict__ deg_up, int* __restrict__ deg_full,
    int64_t* __restrict__ rstart, const int64_t* __restrict__ cbase,
    unsigned long long* __restrict__ scratch, int64_t cap, unsigned long long* __restrict__ ctl,
    unsigned long long* __restrict__ stats, int* __restrict__ work) {
  __shared__ float4 s_pos[kGraphWarps][kCellTile];
  __shared__ int s_lab[kGraphWarps][kCellTile];
  __shared__ uint32_t s_qa[kGraphWarps][kQueue];  // tile index | (root index in the cell << 8)
  __shared__ uint32_t s_qo[kGraphWarps][kQueue];  // position in the root's row
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  unsigned long long rechecks = 0, cands = 0, disagree = 0, edges = 0;
  unsigned long long maxdeg = 0;
  const int ncell = (int)C.grid.ncell;

  int cb = 0, total = 0;
  long long base = 0;
  bool room = true;
  // bins of one queued edge, written to its slot of the root's row
  auto drain_one = [&](int e) {
    const uint32_t a = s_qa[wib][e];
    const int f = (int)(a & 0xffu);
    const long long i = (long long)(a >> 8);
    const int p = cb + (int)i;
    const int q = s_lab[wib][f];
    int b = 1, mf = 1, mr = 1;
    if (!pair_edge<F32, true>(C, P, p, q, C.pos4[p], s_pos[wib][f], b, mf, mr, rechecks)) {
      // the membership test and the binning disagree: reported, never expected
      disagree++;
      b = 1;
      mf = 1;
      mr = 1;
    }
    if (room) {
      const long long pos = base + i * total - i * (i + 1) / 2 + (long long)s_qo[wib][e];
      scratch[pos] = ((unsigned long long)pack_meta(b, mf, mr) << 32) | (uint32_t)q;
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
    if (ce - cb >= (1 << 24)) {  // queue entries hold the root index in 24 bits
      if (lane == 0) atomicMax(&ctl[1], 2ull);
      continue;
    }
    Ranges R;
    {
      GridParams g;
      const int* cs;
      int lkey;
      cell_grid(C, cell, g, cs, lkey);
      forward_ranges(cb - 1, lkey, g, cs, R);
    }
    int pre[5];
    total = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      pre[k] = total;
      if (k < R.n) total += R.end[k] - R.beg[k];
    }
    // the cell's scratch slots: [cbase[cell], cbase[cell + 1]); root i
    // has total - i - 1 candidates
    base = cbase[cell];
    room = cbase[cell + 1] <= cap;
    if (!room && lane == 0) atomicMax(&ctl[1], 1ull);
    int qn = 0;
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
        // flattened index of p is p - cb (range 0 starts at cb)
        const int i = p - cb;
        const int fstart = max(0, i + 1 - t0);
        if (fstart >= tn) continue;
        // p itself is candidate i of the flattened ranges
        const float4 pi = (i >= t0 && i - t0 < tn) ? s_pos[wib][i - t0] : C.pos4[p];
        int off = (t0 == 0) ? 0 : deg_up[p];  // edges of p in earlier tiles
        for (int f0 = fstart; f0 < tn; f0 += 32) {
          const int f = f0 + lane;
          bool e = false;
          if (f < tn) {
            const int q = s_lab[wib][f];
            int b, mf, mr;
            int r = F32 ? member_f32(pi, s_pos[wib][f], P) : 2;
            if (r == 2) {
              rechecks++;
              r = edge_f64(C.posd[p], C.posd[q], P, b, mf, mr) ? 1 : 0;
            }
            e = r == 1;
            if (e) atomicAdd(&deg_full[q], 1);
          }
          const unsigned m = __ballot_sync(0xffffffffu, e);
          if (e) {
            const int rank = __popc(m & lt);
            s_qa[wib][qn + rank] = (uint32_t)f | ((uint32_t)i << 8);
            s_qo[wib][qn + rank] = (uint32_t)(off + rank);
          }
          off += __popc(m);
          qn += __popc(m);
          if (qn >= 32) {
            __syncwarp();
            drain_one(qn - 32 + lane);
            qn -= 32;
            __syncwarp();
          }
        }
        if (lane == 0) {
          // a cell without room keeps no rows: after its last tile its roots
          // have empty rows, so that nothing reads past the scratch area
          // (the build is repeated with room; deg_up carries the running
          // count between tiles)
          deg_up[p] = (room || !last_tile) ? off : 0;
          rstart[p] = room ? base + (long long)i * total - (long long)i * (i + 1) / 2 : 0;
          cands += (unsigned long long)(tn - fstart);
          if (last_tile) {
            atomicAdd(&deg_full[p], off);
            edges += (unsigned long long)off;
            maxdeg = maxdeg > (unsigned long long)off ? maxdeg : (unsigned long long)off;
          }
        }
        __syncwarp();
      }
      // the tile's staged candidates are about to be replaced
      if (lane < qn) drain_one(lane);
      qn = 0;
      __syncwarp();
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    rechecks += __shfl_xor_sync(0xffffffffu, rechecks, o);
    disagree += __shfl_xor_sync(0xffffffffu, disagree, o);
  }
  if (lane == 0) {
    if (rechecks) atomicAdd(&stats[0], rechecks);
    if (cands) atomicAdd(&stats[1], cands);
    if (maxdeg) atomicMax(&stats[2], maxdeg);
    if (disagree) atomicAdd(&ctl[2], disagree);
    if (edges) atomicAdd(&ctl[3], edges);
  }
}

// Rows from the scratch area to CSR order.  A warp takes 32 consecutive
// roots (their lengths and offsets in one coalesced load) and copies the
// rows one after the other, lanes over records.
__global__ void csr_compact_kernel(int64_t n, const int* __restrict__ deg_up,
                                   const int64_t* __restrict__ rstart,
                                   const int64_t* __restrict__ row_ptr,
                                   const unsigned long long* __restrict__ scratch,
                                   unsigned long long* __restrict__ rec) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t p0 = ((int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; p0 < n;
       p0 += warps * 32) {
    const int64_t p = p0 + lane;
    int d = 0;
    int64_t src = 0, dst = 0;
    if (p < n) {
      d = deg_up[p];
      src = rstart[p];
      dst = row_ptr[p];
    }
#pragma unroll 4
    for (int r = 0; r < 32; ++r) {
      const int dr = __shfl_sync(0xffffffffu, d, r);
      const int64_t sr = __shfl_sync(0xffffffffu, src, r);
      const int64_t tr = __shfl_sync(0xffffffffu, dst, r);
      for (int j = lane; j < dr; j += 32) rec[tr + j] = scratch[sr + j];
    }
  }
}

int graph_blocks(int64_t ncell) {
  int64_t b = (ncell + kGraphWarps - 1) / kGraphWarps;
  const int64_t cap = (int64_t)8 * sm_count();
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace

void UpperCSR::build(const DevCatalog& C, const PairParams& P, cudaStream_t s, bool speculate) {
  n = C.n;
  launches = 0;
  deg_up.reserve(n + 1);
  deg_full.reserve(n + 1);
  rstart.reserve(n + 1);
  stats.reserve(4);
  ctl.reserve(4);
  work.reserve(2);
  // scratch: kept from earlier builds (grown to the candidate bound when short)
  if (scratch.n < (size_t)(64 * n + 1024)) scratch.reserve((size_t)(64 * n + 1024));
  const int blocks = graph_blocks(C.grid.ncell);
  const int64_t ncell = C.grid.ncell;
  cbound.reserve(ncell + 1);
  cbase.reserve(ncell + 2);
  if (ncell > 0) {
    const int bb = (int)std::min<int64_t>((ncell + 255) / 256, (int64_t)8 * sm_count());
    cell_bound_kernel<<<bb, 256, 0, s>>>(C, cbound.p);
    GR_CHECK_LAUNCH();
    scan_i64(cbound.p, cbase.p, ncell, s, scan_tmp);
    launches += 4;
  }
  unsigned long long hc[4] = {0, 0, 0, 0}, hs[3] = {0, 0, 0};
  int64_t need = 0;
  for (int attempt = 0; attempt < 2; ++attempt) {
    ZeroList z;
    z.add(deg_up.p, sizeof(int) * (n + 1));
    z.add(rstart.p, sizeof(int64_t) * (n + 1));
    z.add(deg_full.p, sizeof(int) * (n + 1));
    z.add(stats.p, sizeof(unsigned long long) * 4);
    z.add(ctl.p, sizeof(unsigned long long) * 4);
    z.add(work.p, sizeof(int) * 2);
    zero_async(z, s);
    launches++;
    if (n > 0) {
      const int64_t cap = (int64_t)scratch.n;
      if (P.f32)
        csr_fill_kernel<true><<<blocks, kGraphThreads, 0, s>>>(C, P, deg_up.p, deg_full.p, rstart.p,
                                                               cbase.p, scratch.p, cap, ctl.p, stats.p,
                                                               work.p);
      else
        csr_fill_kernel<false><<<blocks, kGraphThreads, 0, s>>>(C, P, deg_up.p, deg_full.p, rstart.p,
                                                                cbase.p, scratch.p, cap, ctl.p, stats.p,
                                                                work.p);
      launches++;
      GR_CHECK_LAUNCH();
    }
    if (speculate) {
      // the caller reads ctl and stats with its results and calls settle()
      compacted = false;
      return;
    }
    GR_CUDA_TRY(cudaMemcpyAsync(hc, ctl.p, sizeof(hc), cudaMemcpyDeviceToHost, s));
    GR_CUDA_TRY(cudaMemcpyAsync(hs, stats.p, sizeof(hs), cudaMemcpyDeviceToHost, s));
    if (ncell > 0)
      GR_CUDA_TRY(cudaMemcpyAsync(&need, cbase.p + ncell, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    GR_CUDA_TRY(cudaStreamSynchronize(s));
    if (hc[1] == 0) break;
    if (hc[1] == 2) throw Error{-2, "CSR build: a grid cell holds 2^24 points or more"};
    // out of room: grow to the exact bound and run again
    scratch.reserve((size_t)need + 1024);
  }
  if (hc[1] != 0) throw Error{-2, "CSR build: scratch overflow after growing"};
  if (hc[2] != 0) throw Error{-3, "CSR build: FP32 membership and FP64 binning disagree"};
  n_edges = (int64_t)hc[3];
  rechecks = (int64_t)hs[0];
  candidates = (int64_t)hs[1];
  max_deg = (int64_t)hs[2];
  compacted = false;
}

void UpperCSR::settle(const unsigned long long hc[4], const unsigned long long hs[3]) {
  if (hc[1] == 2) throw Error{-2, "CSR build: a grid cell holds 2^24 points or more"};
  if (hc[2] != 0) throw Error{-3, "CSR build: FP32 membership and FP64 binning disagree"};
  n_edges = (int64_t)hc[3];
  rechecks = (int64_t)hs[0];
  candidates = (int64_t)hs[1];
  max_deg = (int64_t)hs[2];
}

void UpperCSR::compact(cudaStream_t s) {
  if (compacted) return;
  row_ptr.reserve(n + 1);
  scan_i32_to_i64(deg_up.p, row_ptr.p, n, s, scan_tmp);
  rec.reserve(n_edges + 1);
  if (n > 0 && n_edges > 0) {
    const int64_t groups = (n + 31) / 32;
    const int blocks = (int)std::min<int64_t>((groups + 7) / 8, (int64_t)16 * sm_count());
    csr_compact_kernel<<<blocks, 256, 0, s>>>(n, deg_up.p, rstart.p, row_ptr.p, scratch.p, rec.p);
    GR_CHECK_LAUNCH();
  }
  compacted = true;
}

namespace {

// scratch[0..cap]: the number of roots per length class min(len, cap), then
// the first slot of each class in longest-first order.  Privatised in shared
// memory when the classes fit (smem_hist).
__global__ void root_len_hist_kernel(const int* __restrict__ len, int n, int cap,
                                     int* __restrict__ hist, bool smem_hist) {
  extern __shared__ int s_hist[];
  if (smem_hist) {
    for (int b = threadIdx.x; b <= cap; b += blockDim.x) s_hist[b] = 0;
    __syncthreads();
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    atomicAdd(smem_hist ? &s_hist[min(len[i], cap)] : &hist[min(len[i], cap)], 1);
  if (smem_hist) {
    __syncthreads();
    for (int b = threadIdx.x; b <= cap; b += blockDim.x)
      if (s_hist[b]) atomicAdd(&hist[b], s_hist[b]);
  }
}

// exclusive scan in descending class order, one block: hist[b] = the number
// of roots in the classes above b
__global__ void root_len_scan_kernel(int* __restrict__ hist, int cap) {
  __shared__ int s_warp[32];
  __shared__ int s_carry;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int j0 = 0; j0 <= cap; j0 += blockDim.x) {
    const int j = j0 + threadIdx.x;
    const int v = j <= cap ? hist[cap - j] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int w = lane < nw ? s_warp[lane] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      s_warp[lane] = w;
    }
    __syncthreads();
    const int before = s_carry + (wid > 0 ? s_warp[wid - 1] : 0);
    if (j <= cap) hist[cap - j] = before + x - v;
    __syncthreads();
    if (threadIdx.x == 0) s_carry += s_warp[nw - 1];
    __syncthreads();
  }
}

// one slot per root; lanes of a warp with the same class share one atomic
__global__ void root_scatter_kernel(const int* __restrict__ len, int n, int cap,
                                    int* __restrict__ off, int* __restrict__ order) {
  const int lane = threadIdx.x & 31;
  for (int i0 = blockIdx.x * blockDim.x; i0 < n; i0 += gridDim.x * blockDim.x) {
    const int i = i0 + threadIdx.x;
    const bool live = i < n;
    const int b = live ? min(len[i], cap) : -1;
    const unsigned grp = __match_any_sync(0xffffffffu, b);
    const int leader = __ffs(grp) - 1;
    int base = 0;
    if (live && lane == leader) base = atomicAdd(&off[b], __popc(grp));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (live) order[base + __popc(grp & ((1u << lane) - 1u))] = i;
  }
}

}  // namespace

void order_roots_by_length(const CSRView& G, int n, int cap, int* order, int* scratch,
                           cudaStream_t s) {
  if (n <= 0) return;
  GR_CUDA_TRY(cudaMemsetAsync(scratch, 0, sizeof(int) * (size_t)(cap + 1), s));
  const int blocks = (int)std::min<int64_t>(((int64_t)n + 255) / 256, 2 * (int64_t)sm_count());
  const size_t hb = sizeof(int) * (size_t)(cap + 1);
  const bool smem_hist = hb <= 32 * 1024;
  root_len_hist_kernel<<<blocks, 256, smem_hist ? hb : 0, s>>>(G.len, n, cap, scratch, smem_hist);
  GR_CHECK_LAUNCH();
  root_len_scan_kernel<<<1, 1024, 0, s>>>(scratch, cap);
  GR_CHECK_LAUNCH();
  root_scatter_kernel<<<blocks, 256, 0, s>>>(G.len, n, cap, scratch, order);
  GR_CHECK_LAUNCH();
}

}  // namespace gr
