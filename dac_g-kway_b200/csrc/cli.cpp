// g-kway <graph> <k> <out>  -- drop-in for the reference CLI (main/main.cu:5-20).
// Writes <cwd>/<out>.out with one 0-based part id per line and prints the
// reference's timing lines and "***** h_cutsize N".  Unlike the reference
// (which always exits 0 and only warns on a wrong argument count), a usage or
// runtime error exits non-zero.
#include <cstdio>
#include <exception>
#include <iostream>
#include <string>

#include "gkway.hpp"

int main(int argc, char** argv) {
  if (argc != 4) {
    std::cerr << "usage: g-kway graph_file num_partition out_name\n";
    return 2;
  }
  try {
    const std::string graph_file = argv[1];
    const int k = std::stoi(argv[2]);
    const std::string out = argv[3];
    graph_partitioner(graph_file, out, k);
  } catch (const std::exception& e) {
    std::cerr << "g-kway: " << e.what() << '\n';
    return 1;
  }
  return 0;
}
