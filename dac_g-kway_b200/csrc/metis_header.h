// The header line of a METIS .graph file, read on the host by both readers
// (graph_io.cpp on the host, parse.cu on the device).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

namespace gkw {

struct MetisHeader {
  int64_t n = 0, m = 0;
  bool vsize = false, vw = false, ew = false;   // line layout: [size] [weight] (neighbour [edge weight])*
  size_t body = 0;                              // offset of the first byte after the header line
};

// The header line of a METIS .graph text ("n m [fmt [ncon]]"; comment and
// blank lines before it skipped); false with *err set on a malformed header.
// reference_quirks: the reference's reading of fmt "11" (neighbour/weight
// pairs only, gkway/graph.hpp:93-97,125-137).
bool parse_metis_header(const char* buf, size_t size, bool reference_quirks, MetisHeader* out, std::string* err);

}  // namespace gkw
