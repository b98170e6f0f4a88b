// gramsci: command-line driver with the reference program's options and
// output files (csabiu/Gramsci src/gramsci.F90:1-285), running the hot path
// on the GPU through libgramsci_cuda.so.
//
//   gramsci -gal G [-ran R] -rmin a -rmax b -nbins n [-nmu m] [-log]
//           [-out F] [-cut region.loadnodes [-gcol]] -2pcf | -3pcf | -4pcf | -equi | -tetra
//
// Exit status follows the reference: 0 after help, after an unknown option
// (the reference prints a message and stops) and after a run; 2 for an
// unreadable option value (gfortran's runtime error status); 1 for an
// input, library or output error.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../../include/gramsci_cuda.h"
#include "../../../include/gramsci_host.h"

namespace {

void print_help() {
  std::puts(" gramsci: 2-, 3- and 4-point correlation counts of a 3D point set");
  std::puts(" ");
  std::puts(" usage: gramsci -gal galaxy_file [-ran random_file] -rmin Rmin -rmax Rmax");
  std::puts("                -nbins Nbins [-nmu Nmu] [-log] [-out out_file]");
  std::puts("                [-cut region_file [-gcol]] -2pcf | -3pcf | -4pcf | -equi | -tetra");
  std::puts(" ");
  std::puts("   galaxy_file, random_file  records of x y z w");
  std::puts("   Rmin, Rmax                range of separations counted");
  std::puts("   Nbins                     radial bins (linear; -log for log10 spacing)");
  std::puts("   Nmu                       line-of-sight bins in -1 < mu < 1 (>= 2 turns them on)");
  std::puts("   out_file                  result table (default result.txt)");
  std::puts("   -equi, -tetra             equilateral triangles / regular tetrahedra only");
  std::puts("   -gcol                     region file rows are x y z w gal buffer (gramsci-decompose)");
}

// Without a context (gr_create failed) there is no message to read: name the
// status instead.
const char* status_text(int rc) {
  switch (rc) {
    case GR_E_ARG: return "invalid argument";
    case GR_E_CAPACITY: return "out of memory or over a size limit";
    case GR_E_CUDA: return "no usable CUDA device";
    case GR_E_TIMEOUT: return "a device wait ran out";
    case GR_E_UNSUPPORTED: return "unsupported option";
    default: return "unknown status";
  }
}

int fail(gr_ctx* ctx, const char* what, int rc) {
  std::fprintf(stderr, "gramsci: %s failed (%d): %s\n", what, rc,
               ctx ? gr_last_error(ctx) : status_text(rc));
  return 1;
}

}  // namespace

int main(int argc, char** argv) {
  grh_options o;
  grh_parse_args(argc, argv, &o);
  if (o.error == 1) {
    std::printf("%s\n", o.message);
    return 0;
  }
  if (o.error == 2) {
    std::fprintf(stderr, "gramsci: %s\n", o.message);
    return 2;
  }
  if (o.help) {
    print_help();
    return 0;
  }
  if (o.nbins < 1 || o.nbins > 127 || o.nmu < 1 || o.nmu > 127) {
    std::fprintf(stderr, "gramsci: need 1 <= nbins <= 127 and 1 <= nmu <= 127\n");
    return 1;
  }

  double* xyz = nullptr;
  double* w = nullptr;
  int32_t* buffer = nullptr;
  int64_t nd = 0, nr = 0;
  if (o.cut_mode) {
    const char* region = o.mpi ? "1.loadnodes" : o.cut;
    int64_t n = 0;
    // -gcol: x y z w gal buffer files with a galaxy/random split; otherwise
    // the reference's x y z w buffer read with no split (src/gramsci.F90:1304-1317)
    const int rr = o.gcol ? grh_read_region_gal(region, &xyz, &w, &buffer, &nd, &nr)
                          : grh_read_region(region, &xyz, &w, &buffer, &n);
    if (rr != 0) {
      std::fprintf(stderr, "gramsci: cannot read %s\n", region);
      return 1;
    }
    if (!o.gcol) nd = n;
  } else {
    if (grh_read_catalogue(o.gal, o.rancat ? o.ran : nullptr, &xyz, &w, &nd, &nr) != 0) {
      std::fprintf(stderr, "gramsci: cannot read the catalogues\n");
      return 1;
    }
    grh_normalise(w, nd, nr);
  }
  std::printf(" Preparing to read %lld data points\n", (long long)nd);
  std::printf(" Preparing to read %lld random points\n", (long long)nr);

  std::vector<double> edges(o.nbins + 1);
  grh_radial_bins(o.rmin, o.rmax, o.nbins, o.logbins, edges.data());

  gr_ctx* ctx = nullptr;
  int rc = gr_create(&ctx, 0);
  if (rc) return fail(nullptr, "gr_create", rc);
  if ((rc = gr_set_catalog(ctx, xyz, w, buffer, nd, nr))) return fail(ctx, "gr_set_catalog", rc);
  if ((rc = gr_set_bins(ctx, o.rmin, o.rmax, o.nbins, o.nmu, o.logbins)))
    return fail(ctx, "gr_set_bins", rc);

  const int nb = o.nbins, nm = o.nmu;
  gr_stats st;
  if (o.two_pcf) {
    std::vector<double> N2((size_t)nb * nm), N3((size_t)nb * nm);
    if ((rc = gr_count_2pcf(ctx, N2.data(), N3.data(), nullptr, nullptr)))
      return fail(ctx, "gr_count_2pcf", rc);
    gr_get_stats(ctx, &st);
    std::printf(" writing output to: %s\n", o.out);
    if (grh_write_2pcf(o.out, edges.data(), nb, nm, N2.data(), N3.data()))
      return fail(nullptr, "writing the output", -1);
    std::printf(" 2PCF: %lld pairs, %.3f ms on the GPU\n", (long long)st.tuples, st.ms_total);
  }
  if (o.three_pcf) {
    const size_t nc = (size_t)nb * (nb + 1) * (nb + 2) / 6;
    std::vector<double> N2(nc * nm), N3(nc * nm);
    if ((rc = gr_count_3pcf(ctx, N2.data(), N3.data(), nullptr, nullptr)))
      return fail(ctx, "gr_count_3pcf", rc);
    gr_get_stats(ctx, &st);
    if (grh_write_3pcf(o.out, edges.data(), nb, nm, N2.data(), N3.data()))
      return fail(nullptr, "writing the output", -1);
    std::printf(" 3PCF: %lld triangles, %.3f ms on the GPU\n", (long long)st.tuples, st.ms_total);
  }
  if (o.equi) {
    std::vector<double> N2((size_t)nb * nm), N3((size_t)nb * nm);
    if ((rc = gr_count_equi(ctx, N2.data(), N3.data(), nullptr, nullptr)))
      return fail(ctx, "gr_count_equi", rc);
    gr_get_stats(ctx, &st);
    if (grh_write_equi(o.out, edges.data(), nb, nm, N2.data(), N3.data()))
      return fail(nullptr, "writing the output", -1);
    std::printf(" -equi: %lld triangles, %.3f ms on the GPU\n", (long long)st.tuples, st.ms_total);
  }
  if (o.four_pcf) {
    const size_t nc = (size_t)nb * (nb + 1) * (nb + 2) * (nb + 3) / 24;
    const size_t nbin = nc * nb * nb;
    std::vector<double> N2(nbin), N3(nbin), dN(nbin * 6), dR(nbin * 6);
    if ((rc = gr_count_4pcf(ctx, N2.data(), N3.data(), dN.data(), dR.data(), nullptr, nullptr,
                            nullptr, nullptr)))
      return fail(ctx, "gr_count_4pcf", rc);
    gr_get_stats(ctx, &st);
    if (grh_write_4pcf(o.out, edges.data(), nb, N2.data(), N3.data(), dN.data(), dR.data()))
      return fail(nullptr, "writing the output", -1);
    std::printf(" 4PCF: %lld 4-cliques, %.3f ms on the GPU\n", (long long)st.tuples, st.ms_total);
  }
  if (o.tetra) {
    std::vector<double> N2(nb), N3(nb), dN((size_t)nb * 6), dR((size_t)nb * 6);
    if ((rc = gr_count_tetra(ctx, N2.data(), N3.data(), dN.data(), dR.data(), nullptr, nullptr,
                             nullptr, nullptr)))
      return fail(ctx, "gr_count_tetra", rc);
    gr_get_stats(ctx, &st);
    if (grh_write_tetra(o.out, edges.data(), nb, nm, N2.data(), N3.data(), dN.data(), dR.data()))
      return fail(nullptr, "writing the output", -1);
    std::printf(" -tetra: %lld 4-cliques, %.3f ms on the GPU\n", (long long)st.tuples, st.ms_total);
  }
  gr_destroy(ctx);
  grh_free(xyz);
  grh_free(w);
  grh_free(buffer);
  std::puts(" Exit... stage left!");
  return 0;
}
