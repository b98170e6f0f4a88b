/*
 * gramsci_cuda.h -- C ABI of the B200 N-point correlation library
 * (libgramsci_cuda.so).
 *
 * The reference program (csabiu/Gramsci, Fortran 90) has no plugin or FFI
 * layer: its hot path is a chain of internal subroutines that share module
 * globals.  Each entry point below replaces one of those seams, so a host
 * program (the Fortran driver through iso_c_binding, the C++ `gramsci` CLI,
 * or Python through ctypes) can swap the CPU code for this library without
 * changing the program's inputs, outputs or CLI.
 *
 * Conventions
 *  - Every function returns a status: GR_OK (0) or a negative GR_E_* code;
 *    gr_last_error() gives the message.  No C++ exception crosses the ABI.
 *  - Point ids are positions in the catalogue as the reference orders it:
 *    galaxies first (0 .. n_data-1), then randoms.  Ids in exported graphs are
 *    0-based (the Fortran host adds 1).
 *  - Output arrays are caller-allocated HOST memory in Fortran (column-major)
 *    order with the shapes documented per function.  A NULL output pointer
 *    means "not wanted".
 *  - One context per host thread.  Calls are synchronous: they return after
 *    the work on the context's stream has finished.
 *  - Radial bins are 1..nbins and mu bins 1..nmu as in the reference; both
 *    must be <= 127 because the reference stores them as int8
 *    (src/node_module.F90:7).
 */
#ifndef GRAMSCI_CUDA_H
#define GRAMSCI_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GR_OK 0
#define GR_E_ARG (-1)         /* invalid argument or call order            */
#define GR_E_CAPACITY (-2)    /* a size exceeds what the library supports  */
#define GR_E_CUDA (-3)        /* CUDA runtime error                        */
#define GR_E_TIMEOUT (-4)     /* reserved: no call waits on the device     */
#define GR_E_UNSUPPORTED (-5) /* option not available                      */

typedef struct gr_ctx gr_ctx;

/* Options for gr_set_option. */
#define GR_OPT_PRECISION 1 /* 0: FP32 separations + FP64 guard band (default); 1: FP64 throughout */
#define GR_OPT_TIMEOUT_MS 2 /* accepted (> 0) and stored; no kernel of this library waits on
                               another block, a flag or another device, so nothing uses it */
#define GR_OPT_AUTOTUNE 3   /* 0: fixed kernels; 1: time the pair-sweep variants once per
                               workload class and cache the choice, and give dense
                               catalogues (64 or more points per rmax-wide cell) cells of
                               rmax/2 and the tile sweep (default); 2+v: force variant v
                               (0 warp per cell, 1/2 block per cell of 128/256, 3 warp per
                               cell with queued binning, 4/5 block per cell of 128/256 with
                               queued binning, 6 the tile sweep, 7 the tile sweep on cells
                               of rmax/2) */
#define GR_OPT_KEEP_GRAPH 4 /* 0 (default): every count call builds the index and graph;
                               1: keep the graph of the last call and reuse it until the
                               catalogue, the bins or the precision change */
#define GR_OPT_CLIQUE_MODE 5 /* how the 3PCF / 4PCF kernels find the edges among a root's
                               larger-label neighbours: 0 automatic (default: mode 2 wherever
                               the rows allow it), 1 hash probes of the neighbours' rows, 2
                               the graph's membership test on the pairs of neighbours.
                               4PCF: mode 2 takes rows up to 256
                               neighbours (longer rows use 1).  3PCF: rows longer than 256
                               neighbours take a second launch in mode 2 (up to 1024, then a
                               global-memory path) unless mode 1 is forced.  Results are
                               identical; only speed differs */

/* Run statistics of the last count call (gr_get_stats). */
typedef struct gr_stats {
  double ms_index;        /* cell index build (device time)                     */
  double ms_graph;        /* CSR adjacency build (device time), 0 for 2PCF      */
  double ms_query;        /* counting kernel(s) (device time)                   */
  double ms_total;        /* whole call on the device                           */
  int64_t n_points;
  int64_t n_edges;        /* directed edges of the (rmin, rmax) graph            */
  int64_t tuples;         /* distinct pairs / triangles / 4-cliques binned       */
  int64_t rooted;         /* rooted incidences (the reference's loop count)      */
  int64_t fp64_rechecks;  /* pairs re-evaluated in FP64 inside the guard band    */
  int64_t candidates;     /* candidate pairs tested                              */
  int64_t kernel_launches;/* kernels launched by the call                        */
  int64_t probes;         /* intersection probes (3PCF/4PCF): neighbour-row entries
                             looked up in the root's row, or in the geometric
                             clique mode the pairs of the root's neighbours tested */
  int64_t upper_edges;    /* undirected edges stored in the upper CSR            */
} gr_stats;

/* Library version string. */
const char* gr_version(void);

/* Context lifetime.  Replaces the program-global state of Ngramsci
 * (src/gramsci.F90:13-38). */
int gr_create(gr_ctx** out, int device);
int gr_destroy(gr_ctx* ctx);
const char* gr_last_error(const gr_ctx* ctx);

/* Use a caller-owned CUDA stream (cudaStream_t passed as void*); NULL
 * restores the context's own stream.  Count calls wait on the stream for
 * their results, so they cannot be captured into a caller's CUDA graph.
 * Internally, a 2PCF or 3PCF count of a catalogue of the same size, box and
 * binning as the previous one replays that call's index (and graph)
 * phases as a CUDA graph the library captured on the context's own stream;
 * the replay is launched on the stream in use. */
int gr_set_stream(gr_ctx* ctx, void* stream);

/* Catalogue.  Replaces read_files_2's result (src/gramsci.F90:1364-1396):
 *   xyz    points(3,N) in Fortran order, i.e. x,y,z interleaved, N = n_data+n_rand
 *   w      signed normalised weights exactly as after gramsci.F90:1390-1391
 *   buffer 0/1 per point (1 = buffer point, never a root; gramsci.F90:363) or NULL
 * gr_set_catalog copies from host memory; gr_set_catalog_dev takes device
 * pointers (device-resident inputs) and copies them device-to-device. */
int gr_set_catalog(gr_ctx* ctx, const double* xyz, const double* w, const int32_t* buffer,
                   int64_t n_data, int64_t n_rand);
int gr_set_catalog_dev(gr_ctx* ctx, const double* xyz, const double* w, const int32_t* buffer,
                       int64_t n_data, int64_t n_rand);

/* Binning.  Replaces the CLI values rmin/rmax/nbins/nmu/-log and the derived
 * delta_r, inv_delta_r, mu_scale (src/gramsci.F90:136-147, 1216-1223).
 * RSD (line-of-sight binning) is on when nmu >= 2. */
int gr_set_bins(gr_ctx* ctx, double rmin, double rmax, int32_t nbins, int32_t nmu, int32_t logbins);
int gr_set_option(gr_ctx* ctx, int32_t key, int64_t value);

/* 2PCF.  Replaces create_graph + query_graph_2pcf (src/gramsci.F90:288-379):
 *   N2      (nbins, nmu)     sum over rooted pairs of w_i w_j          (N2(:,:,3))
 *   N3      (nbins, nmu)     the same restricted to random-random pairs (N3(:,:,3))
 *   counts  (nbins, nmu, 4)  rooted pairs by category 2*random(root)+random(neighbour)
 *   catsum  (nbins, nmu, 4)  sum of w_i w_j per category
 * The graph is not materialised: pairs are binned straight from the cell
 * sweep. */
int gr_count_2pcf(gr_ctx* ctx, double* N2, double* N3, int64_t* counts, double* catsum);

/* 3PCF.  Replaces create_graph + query_graph_3pcf_all (src/gramsci.F90:463-510)
 * including find_dist (:1579-1609), find_normal (:1611-1625) and the symmetric
 * bin table (:1459-1474).  ncfg = nbins(nbins+1)(nbins+2)/6:
 *   N2, N3  (ncfg, nmu)      N3 as the reference forms it (minus the sum over
 *                            all-random triangles)
 *   counts  (ncfg, nmu, 4)   rooted triangles by number of randoms (0..3)
 *   catsum  (ncfg, nmu, 4)   sum of w_i w_a w_b by number of randoms */
int gr_count_3pcf(gr_ctx* ctx, double* N2, double* N3, int64_t* counts, double* catsum);

/* 4PCF.  Replaces create_graph + query_4pcf_all2 (src/gramsci.F90:662-825).
 * ncfg = nbins(nbins+1)(nbins+2)(nbins+3)/24 canonical perimeters:
 *   N2, N3        (ncfg, nbins, nbins)     indexed (cfg, bin(i,b), bin(a,c))
 *   discN, discR  (ncfg, nbins, nbins, 6)  the six disconnected pair terms
 *   counts        (ncfg, nbins, nbins, 5)  rooted 4-cliques by number of randoms
 *   catsum        (ncfg, nbins, nbins, 5)
 *   dcount, dsum  (ncfg, nbins, nbins, 6, 4) disc terms by category: 0..2 =
 *                 discN by number of randoms in the pair, 3 = discR */
int gr_count_4pcf(gr_ctx* ctx, double* N2, double* N3, double* discN, double* discR,
                  int64_t* counts, double* catsum, int64_t* dcount, double* dsum);

/* -equi: equilateral triangles (all three edges in the same radial bin).
 * Replaces query_graph_equilateral_triangle (src/gramsci.F90:402-448):
 *   N2, N3  (nbins, nmu)     N3 = minus the all-random sum without mu bins,
 *                            0 with mu bins (the reference sums only N2 then)
 *   counts, catsum (nbins, nmu, 4) by number of randoms */
int gr_count_equi(gr_ctx* ctx, double* N2, double* N3, int64_t* counts, double* catsum);

/* -tetra: regular tetrahedra (all six edges of a 4-clique in the same radial
 * bin).  Replaces query_graph_tetrahedron (src/gramsci.F90:548-646):
 *   N2, N3        (nbins)      sums of the 4-products (N3: all random)
 *   discN, discR  (nbins, 6)   the six gated 3-product terms
 *   counts, catsum (nbins, 5)  by number of randoms
 *   dcount, dsum  (nbins, 6, 5) disc terms: 0..3 = discN by randoms in the
 *                 product, 4 = discR */
int gr_count_tetra(gr_ctx* ctx, double* N2, double* N3, double* discN, double* discR,
                   int64_t* counts, double* catsum, int64_t* dcount, double* dsum);

/* Graph access (parity tests, graph reuse).  Builds the (rmin, rmax) graph
 * of create_graph (src/gramsci.F90:288-348) if needed.  Export gives the
 * reference's layout: rows in point order, each row sorted by id (as
 * sort2 leaves it, src/sorting_module.F90:36-47), with the radial bin and the
 * mu bin seen from the row's point.  row_ptr has N+1 entries. */
int gr_graph_build(gr_ctx* ctx);
int gr_graph_nedges(gr_ctx* ctx, int64_t* n_edges);
int gr_graph_export(gr_ctx* ctx, int64_t* row_ptr, int32_t* col, uint8_t* bin, uint8_t* mu);

/* Graph persistence (the "graph database" of the reference's README: build
 * the graph once, query it many times).  gr_graph_save writes the graph of
 * the current catalogue and bins (building it if needed); gr_graph_load reads
 * one back for the same catalogue positions and bins -- it checks the point
 * count, the binning and a 64-bit fingerprint of the coordinates, and returns
 * GR_E_ARG on a mismatch -- after which the 2/3/4PCF, -equi and -tetra calls
 * reuse it (no graph build) until the catalogue, bins or precision change.
 * File: a 128-byte header ("GRAMSCSR", version 1, n, upper edges, max upper
 * degree, rmin, rmax, nbins, nmu, logbins, coordinate fingerprint, payload
 * checksum, labelling fingerprint), then row_ptr int64[n+1], records uint64[edges], full degree
 * int32[n], all little-endian, in the library's internal (cell) labelling. */
int gr_graph_save(gr_ctx* ctx, const char* path);
int gr_graph_load(gr_ctx* ctx, const char* path);

/* Batched regions.  Replaces the reference's domain decomposition
 * (src/domain_decomposition.f90:39-80) followed by one program run per
 * region (`-cut`, src/gramsci.F90:1224-1231) and the hand summation of the
 * outputs.  gr_set_regions(ctx, n) splits the catalogue's bounding box into
 * n^3 equal regions (0 turns it off); each region's halo is its points'
 * bounding box grown by rmax (strict bounds); points of other regions inside
 * a halo are buffer points there.  gr_count_2pcf_batched counts the 2PCF of
 * all regions in one launch (cells of every region from one work queue,
 * largest region first), with the global galaxy/random flags and weight
 * normalisation, so the result equals gr_count_2pcf on the whole catalogue.
 * The first call for a catalogue/binning/split plans the layout and captures
 * the device work in a CUDA graph; later calls replay it.  Outputs as
 * gr_count_2pcf.  gr_regions_info / gr_regions_export describe the layout
 * (member_off: nregions+1 offsets; per member its catalogue index and 1 if it
 * is a buffer point), e.g. to run the regions one launch at a time. */
int gr_set_regions(gr_ctx* ctx, int32_t nsplit);
int gr_count_2pcf_batched(gr_ctx* ctx, double* N2, double* N3, int64_t* counts, double* catsum);

/* Regions from a region id per point (jackknife regions, or any domain
 * decomposition the caller made): region_of_point has one entry in
 * [0, nregions) per catalogue point (host memory).  Region r's halo is the
 * bounding box of its points grown by rmax (strict bounds), as in
 * src/domain_decomposition.f90:39-80; points of other regions inside it are
 * its buffer points.  Replaces the subcube split until gr_set_regions is
 * called; gr_set_catalog clears it (the ids belong to the catalogue). */
int gr_set_region_ids(gr_ctx* ctx, const int32_t* region_of_point, int32_t nregions);

/* Independent catalogues (mocks) in one launch.  The catalogue given to
 * gr_set_catalog is the mocks one after another, each with its galaxies
 * first: mock m has n_data[m] galaxies then n_rand[m] randoms, with signed
 * weights normalised within the mock (the reference's normalisation, one
 * mock at a time; the catalogue's own n_data / n_rand split is not used).
 * Each mock is a region without halo: pairs never join two mocks.  The
 * batched calls then count every mock in one launch; gr_count_2pcf_regions
 * gives each mock's histograms.  Cleared by gr_set_catalog. */
int gr_set_mocks(gr_ctx* ctx, int32_t nmocks, const int64_t* n_data, const int64_t* n_rand);

/* 2PCF of every region (or mock) separately, in one launch: the histograms
 * each region's own run of the reference would write (its own points as
 * roots, its buffer points as neighbours only).  Shapes as gr_count_2pcf
 * with a last axis over the regions: N2, N3 (nbins, nmu, nregions), counts
 * and catsum (nbins, nmu, 4, nregions).  Their sum over the regions is
 * gr_count_2pcf_batched's result. */
int gr_count_2pcf_regions(gr_ctx* ctx, double* N2, double* N3, int64_t* counts, double* catsum);

/* 3PCF over all regions (or mocks) in one pass: the neighbour graph of every
 * region's members built in one launch, every triangle rooted at each of
 * its vertices that is a region's own point.  Outputs as gr_count_3pcf
 * (summed over the regions; equal to gr_count_3pcf on the whole catalogue
 * for a split into regions, the sum of the mocks' results for mocks). */
int gr_count_3pcf_batched(gr_ctx* ctx, double* N2, double* N3, int64_t* counts, double* catsum);
int gr_regions_info(gr_ctx* ctx, int32_t* nregions, int64_t* nmembers);
int gr_regions_export(gr_ctx* ctx, int64_t* member_off, int32_t* member_orig,
                      int32_t* member_buffer);

/* Weight adjoints.  Gradient of L = sum(cot2 * N2) + sum(cot3 * N3) with
 * respect to every signed normalised weight w_k (grad_w has N entries,
 * catalogue order).  cot2/cot3 have the shapes of N2/N3 of the matching
 * count call; cot3 may be NULL.  The reference has no derivatives; these
 * differentiate the sums of query_graph_2pcf (src/gramsci.F90:362-379) and
 * query_graph_3pcf_all (:475-510): N2 and N3 are multilinear in the weights
 * (each point appears at most once per pair or triangle), so
 * dN2_b/dw_k = sum over the rooted pairs/triangles in bin b that contain k of
 * the product of the other weights.  gr_adjoint_3pcf reuses the graph of the
 * last count or graph build when the catalogue and bins are unchanged.
 * Gradients are accumulated in 128-bit fixed point: deterministic. */
int gr_adjoint_2pcf(gr_ctx* ctx, const double* cot2, const double* cot3, double* grad_w);
int gr_adjoint_3pcf(gr_ctx* ctx, const double* cot2, const double* cot3, double* grad_w);

/* 4PCF weight adjoint: gradient of L = sum(cot2 N2) + sum(cot3 N3) +
 * sum(cotN discN) + sum(cotR discR) of gr_count_4pcf (query_4pcf_all2,
 * src/gramsci.F90:662-825) with respect to every signed normalised weight.
 * cot2/cot3 have N2's shape (ncfg, nbins, nbins), cotN/cotR discN's
 * (ncfg, nbins, nbins, 6); all but cot2 may be NULL.  Every rooted 4-clique
 * adds to each of its vertices the cotangent of its bin times the product of
 * the other three weights, and each gated pair term its cotangent times the
 * partner's weight.  Reuses the graph of the last count or graph build when
 * the catalogue and bins are unchanged; 128-bit fixed-point accumulation. */
int gr_adjoint_4pcf(gr_ctx* ctx, const double* cot2, const double* cot3, const double* cotN,
                    const double* cotR, double* grad_w);

/* Statistics of the last count call. */
int gr_get_stats(gr_ctx* ctx, gr_stats* out);

/* 2PCF without any device allocation.  This entry point has no counterpart
 * in the reference; it exists for callers that cannot call cudaMalloc (code
 * running inside another framework's memory pool or under a fixed memory
 * budget, plugins limited to the buffers their host gives them).  It takes
 * DEVICE pointers: the catalogue (xyz interleaved, signed normalised w,
 * galaxies first; no buffer points) and the outputs, any of which may be
 * NULL: counts (nbins, nmu, 4) int64, catsum (nbins, nmu, 4), N2 and N3
 * (nbins, nmu), the same quantities as gr_count_2pcf.  All intermediate data
 * live in one fixed device array inside the library (about 4.3 MB per GPU,
 * held until the process exits).  At most GR_NOALLOC_MAX_POINTS points and
 * nbins*nmu <= GR_NOALLOC_MAX_BINS; larger inputs return GR_E_CAPACITY and
 * run nothing.  Work runs on `stream` (cudaStream_t, NULL = default stream)
 * on the current device.  Each call waits on `stream` once, part-way: the
 * catalogue's bounding box is read back to size the cell grid; the rest of
 * the work is queued without waiting and the outputs are ready when the
 * stream reaches them.  Non-finite coordinates or weights return GR_E_ARG
 * after that read-back.  The first call on a device (and CUDA context) looks
 * up the array's device address, so make it before any stream capture.  All
 * calls share the array: calls whose work overlaps on the GPU race and must
 * be serialised by the caller. */
#define GR_NOALLOC_MAX_POINTS 32768
#define GR_NOALLOC_MAX_BINS 4096
int gr_count_2pcf_noalloc(const double* d_xyz, const double* d_w, int64_t n_data, int64_t n_rand,
                          double rmin, double rmax, int32_t nbins, int32_t nmu, int64_t* d_counts,
                          double* d_catsum, double* d_N2, double* d_N3, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GRAMSCI_CUDA_H */
