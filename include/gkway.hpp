// gkway.hpp -- C++ API, source-compatible with G-kway's host surface.
//
//   gk::Graph            replaces gkway/graph.hpp:17-51 (METIS .graph parser,
//                        getters, dump_result)
//   graph_partitioner()  replaces gkway/graph_partitioner.hpp:222 (parse,
//                        partition, print the phase times and the cut, write
//                        <cwd>/<out>.out)
//   gk::GraphPartitioner the class named by the reference's README; the
//                        reference itself only has the free function
//
// Implemented in libgkway.so on top of the C ABI in gkway.h.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "gkway.h"

namespace gk {

// METIS / mt-metis .graph reader.
//
// The reference parser (graph.hpp:70-152) keeps neighbour ids 1-based, reads no
// vertex weights, and reads a format field of "11" as "neighbour weight" pairs
// without a leading vertex weight.  This parser reads the standard METIS
// format ("n m [fmt [ncon]]", fmt digits = vertex sizes / vertex weights /
// edge weights, '%' comment lines, ncon = 1).  Pass reference_quirks = true to
// read fmt "11" the way the reference does.
class Graph {
 public:
  explicit Graph(const std::string& input_path, bool reference_quirks = false);
  Graph(std::vector<int32_t> xadj, std::vector<int32_t> adjncy0, std::vector<int32_t> adjwgt,
        std::vector<int32_t> vwgt);
  ~Graph();

  // Reference getters (graph.hpp:26-33): adjacency with 1-based ids, as the
  // reference keeps them; get_num_edge() returns the CSR entry count 2|E|.
  const int* get_adjncy();
  const int* get_adjp();
  const int* get_adjwgt();
  const int* get_vwgt();
  size_t get_num_vertex();
  size_t get_num_edge();
  int get_total_vertex_weight();
  // Writes one part id per line to <cwd>/<file_name>.out (graph.hpp:227-240).
  void dump_result(const std::vector<int>& vertex_partition, const std::string& file_name);

  // 0-based views used by the partitioner.
  const std::vector<int32_t>& xadj() const { return xadj_; }
  const std::vector<int32_t>& adjncy0() const { return adjncy_; }
  const std::vector<int32_t>& adjwgt() const { return adjwgt_; }
  const std::vector<int32_t>& vwgt() const { return vwgt_; }
  gkw_csr csr() const;

 private:
  std::vector<int32_t> xadj_, adjncy_, adjwgt_, vwgt_;
  std::vector<int32_t> adjncy1_;   // 1-based copy, built on first get_adjncy()
};

struct PartitionResult {
  std::vector<int> part;
  int64_t cut = 0;
  gkw_stats stats{};
};

class GraphPartitioner {
 public:
  explicit GraphPartitioner(const gkw_options* opt = nullptr, int device = 0);
  ~GraphPartitioner();
  GraphPartitioner(const GraphPartitioner&) = delete;
  GraphPartitioner& operator=(const GraphPartitioner&) = delete;

  std::vector<int> partition(const Graph& g, int k);
  PartitionResult partition_with_stats(const Graph& g, int k);
  // One graph for several k, coarsened once (gkw_partition_multi_k): result q
  // equals partition_with_stats(g, ks[q]) without its statistics.
  std::vector<PartitionResult> partition_multi_k(const Graph& g, const std::vector<int>& ks);
  gkw_options& options() { return opt_; }

 private:
  gkw_handle* h_ = nullptr;
  gkw_options opt_;
};

// Loads METIS from a shared library (the reference's initial partitioner,
// gkway/metis_partition.hpp:46-47) and installs it as the initial-partition
// callback in `opt`.  Returns false if the library or its symbol is missing.
// recursive: METIS_PartGraphRecursive (metis.h:185) instead of METIS_PartGraphKway.
bool use_metis_init(gkw_options* opt, const std::string& libmetis_path, bool recursive = false);

}  // namespace gk

// Source-compatible free function (graph_partitioner.hpp:222).
void graph_partitioner(const std::string& GRAPH_FILE, const std::string& OUT_FILE, const int NUM_PARTITIONS);
