// gramsci-resum: sum of the region tables written by `gramsci -cut` (the
// summing step the reference's example script runs after its region runs).
//
//   gramsci-resum -2pcf|-3pcf|-4pcf|-equi|-tetra -out total.txt t1 t2 ...
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../../include/gramsci_host.h"

int main(int argc, char** argv) {
  int query = 0;
  const char* out = nullptr;
  std::vector<const char*> in;
  for (int i = 1; i < argc; ++i) {
    if (!std::strcmp(argv[i], "-2pcf")) query = 2;
    else if (!std::strcmp(argv[i], "-3pcf")) query = 3;
    else if (!std::strcmp(argv[i], "-4pcf")) query = 4;
    else if (!std::strcmp(argv[i], "-equi")) query = 5;
    else if (!std::strcmp(argv[i], "-tetra")) query = 6;
    else if (!std::strcmp(argv[i], "-out") && i + 1 < argc) out = argv[++i];
    else in.push_back(argv[i]);
  }
  if (!query || !out || in.empty()) {
    std::fprintf(stderr, "usage: gramsci-resum -2pcf|-3pcf|-4pcf|-equi|-tetra -out F tables...\n");
    return 2;
  }
  const int rc = grh_resum(query, (int)in.size(), in.data(), out);
  if (rc) {
    std::fprintf(stderr, "gramsci-resum: failed (%d)\n", rc);
    return 1;
  }
  if (query == 4 || query == 6)
    std::fprintf(stderr, "gramsci-resum: disconnected-term columns are not summable; written as NaN\n");
  return 0;
}
