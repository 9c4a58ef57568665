// temf_fetd -f ROOT [-d DEVICE] [--legacy-linux]: the reference's
// `./FETD -f ROOT` (src/FETD_MAIN.f90) on the GPU.  Reads ROOT.mesh and
// ROOT.cntl, runs the adaptive BDF2 loop, writes ROOT.field and ROOT.field2.
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/temf_b200.h"

int main(int argc, char** argv) {
  const char* root = nullptr;
  int device = 0, flags = 0;
  for (int i = 1; i < argc; ++i) {
    if (!std::strcmp(argv[i], "-f") && i + 1 < argc) root = argv[++i];
    else if (!std::strcmp(argv[i], "-d") && i + 1 < argc) device = std::atoi(argv[++i]);
    else if (!std::strcmp(argv[i], "--legacy-linux")) flags |= 1;
    else {
      std::fprintf(stderr, "usage: %s -f ROOT [-d DEVICE] [--legacy-linux]\n", argv[0]);
      return 2;
    }
  }
  if (!root) {
    std::fprintf(stderr, "usage: %s -f ROOT [-d DEVICE] [--legacy-linux]\n", argv[0]);
    return 2;
  }
  char msg[512] = {0};
  const int rc = temf_case_run(root, device, flags, msg, sizeof msg);
  if (rc != TEMF_OK) {
    std::fprintf(stderr, "temf_fetd: %s (code %d)\n", msg, rc);
    return 1;
  }
  std::printf("%s.field written\n", root);
  return 0;
}
