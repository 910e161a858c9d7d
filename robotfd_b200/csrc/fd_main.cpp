// ./fd <curve1.txt> <curve2.txt> <dim> [1]  -- drop-in for the reference CLI (src/main.cpp:13-44).
// Loads both curves with txtLoader2/3, passes the shorter one as curve 1 and prints the
// lines of Frechet::Continuous::distance_cuda.  The optional "1" (forceOversize) is
// accepted and echoed; the engine always runs the O(n+m) fused decision.
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>

#include "txtReader.hpp"
#include "wrapper.hpp"

int main(int argc, char** argv) {
  if (argc < 4) {
    std::cerr << "Usage:\n"
              << "  " << argv[0] << " <curve1.txt> <curve2.txt> [dim]\n"
              << "Example:\n"
              << "  " << argv[0] << " a.txt b.txt 2\n";
    return 1;
  }
  const std::string path1 = argv[1];
  const std::string path2 = argv[2];
  const int dim = (int)std::strtoll(argv[3], nullptr, 10);
  bool forceOversize = argc >= 5 && std::string(argv[4]) == "1";
  const int n = 1 << 30;
  std::printf("%d\n", forceOversize ? 1 : 0);
  if (dim == 2 || dim == 3) {
    Curve c1(dim == 2 ? txtLoader2(path1, 0, n) : txtLoader3(path1, 0, n), dim);
    Curve c2(dim == 2 ? txtLoader2(path2, 0, n) : txtLoader3(path2, 0, n), dim);
    if (c1.size() > c2.size()) compute_distance_parallel(c2, c1, forceOversize);
    else compute_distance_parallel(c1, c2, forceOversize);
  }
  return 0;
}
