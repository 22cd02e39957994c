// v2 graph file: host-side representation and I/O (pk_format.cpp).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace pk {

struct FileLayer {
    int64_t n = 0;               // nodes present
    int64_t layer_capacity = 0;  // node slots
    int64_t cap = 0;             // adjacency slots per node
    int32_t ent = 0;             // entry id
    std::vector<int32_t> ext;          // [n]
    std::vector<int16_t> degree;       // [n]
    std::vector<int16_t> heuristic;    // [n]
    std::vector<uint8_t> has_vector;   // [n]
    std::vector<int32_t> adj;          // [layer_capacity * cap]
    std::vector<float> dist;           // [layer_capacity * cap]
};

struct FileGraph {
    int32_t metric = 0, dtype = 0;
    int64_t dim = 0, max_degree = 0, build_ef = 0, capacity = 0;
    int32_t enter_level = 0;
    std::vector<FileLayer> layers;
    std::vector<uint8_t> vectors;  // layer-0 order, n0 * dim * elem bytes
};

// Both return a PK_* status.
int write_graph_file(const std::string &path, const FileGraph &g);
int read_graph_file(const std::string &path, FileGraph &g, std::string &err);

}  // namespace pk
