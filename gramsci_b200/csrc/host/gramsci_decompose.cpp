// gramsci-decompose: region files for `gramsci -cut`, the reference's
// domain_decomposition program (csabiu/Gramsci src/domain_decomposition.f90).
//
//   gramsci-decompose rmax                      reads ./allpoints (x y z w gal
//                                               aux region), the reference run
//   gramsci-decompose rmax -gal G [-ran R] -nsplit n [-prefix P]
//                                               labels from n^3 subcubes,
//                                               FP64, globally normalised weights
//
// Writes <P>j.loadnodes for every region j (x y z w gal buffer).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../../include/gramsci_host.h"

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: gramsci-decompose rmax [-gal G [-ran R] -nsplit n] [-prefix P]\n");
    return 2;
  }
  const double rmax = std::strtod(argv[1], nullptr);
  const char *gal = nullptr, *ran = nullptr, *prefix = "";
  int nsplit = 0;
  for (int i = 2; i < argc; i += 2) {
    if (i + 1 >= argc) {
      std::fprintf(stderr, "gramsci-decompose: %s needs a value\n", argv[i]);
      return 2;
    }
    if (!std::strcmp(argv[i], "-gal")) gal = argv[i + 1];
    else if (!std::strcmp(argv[i], "-ran")) ran = argv[i + 1];
    else if (!std::strcmp(argv[i], "-nsplit")) nsplit = std::atoi(argv[i + 1]);
    else if (!std::strcmp(argv[i], "-prefix")) prefix = argv[i + 1];
    else {
      std::fprintf(stderr, "gramsci-decompose: unknown option %s\n", argv[i]);
      return 2;
    }
  }
  int32_t nreg = 0;
  const int rc = grh_decompose(gal ? nullptr : "allpoints", gal, ran, rmax, nsplit, prefix, &nreg);
  if (rc) {
    std::fprintf(stderr, "gramsci-decompose: failed (%d)\n", rc);
    return 1;
  }
  std::printf(" creating %d regions\n", nreg);
  return 0;
}
