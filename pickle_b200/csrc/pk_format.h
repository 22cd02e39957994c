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

// A graph file mapped into memory: the arrays are pointers into the mapping
// (possibly unaligned: read small ones with memcpy), valid while the
// MappedGraph lives.
struct MappedLayer {
    int64_t n = 0, layer_capacity = 0, cap = 0;
    int32_t ent = 0;
    const uint8_t *ext = nullptr;         // int32[n]
    const uint8_t *degree = nullptr;      // int16[n]
    const uint8_t *heuristic = nullptr;   // int16[n]
    const uint8_t *has_vector = nullptr;  // uint8[n]
    const uint8_t *adj = nullptr;         // int32[layer_capacity * cap]
    const uint8_t *dist = nullptr;        // float[layer_capacity * cap]
};

struct MappedGraph {
    const uint8_t *base = nullptr;
    uint64_t bytes = 0;
    uint32_t version = 0;
    int32_t metric = 0, dtype = 0;
    int64_t dim = 0, max_degree = 0, build_ef = 0, capacity = 0;
    int32_t enter_level = 0;
    std::vector<MappedLayer> layers;
    const uint8_t *vectors = nullptr;     // layer-0 order, n0 * dim * elem bytes
    uint64_t vector_bytes = 0;
    MappedGraph() = default;
    MappedGraph(const MappedGraph &) = delete;
    MappedGraph &operator=(const MappedGraph &) = delete;
    ~MappedGraph();
};

// Both return a PK_* status.  map_graph_file verifies the checksum (all host
// cores for version 2 files) before it returns PK_OK.
int write_graph_file(const std::string &path, const FileGraph &g);
int map_graph_file(const std::string &path, MappedGraph &g, std::string &err);

}  // namespace pk
