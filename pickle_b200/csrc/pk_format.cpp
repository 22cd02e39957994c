// The v2 HNSW graph file.
//
// The reference names Serializer::to_disk / from_disk for persistence
// (include/serializer.hpp:21-25) and writes, per layer, a record of
// num_nodes, max_degree and the ext / degree / adjacency / distance arrays
// (include/serializer.hpp:27-55), but only for its retired v0 layer; the live
// v2 layer (include/hnsw_layer.hpp:57-83) cannot be saved at all.  This file
// keeps that per-layer record style and stores everything a v2 layer holds:
//
//   magic "PKHNSW2\0", u32 version = 1, u32 flags = 0,
//   i32 metric (DistFunc), i32 dtype (DataType), i64 dim, i64 max_degree (M),
//   i64 build_ef, i64 capacity (external ids), i32 enter_level, i32 num_layers,
//   per layer: i64 n, i64 layer_capacity, i64 cap, i32 ent, i32 reserved,
//              i32 ext[n], i16 degree[n], i16 heuristic[n], u8 has_vector[n],
//              i32 adj[layer_capacity*cap], f32 dist[layer_capacity*cap],
//   vectors[n0*dim] in layer-0 internal order,
//   u64 FNV-1a checksum of all preceding bytes.
//
// has_vector[v] is 0 where the layer's copy of the node's vector was never
// written: the reference's Insert copies it only into layers up to the
// highest one it searched (include/hnsw.hpp:283-297), so nodes that open a new
// top layer keep a zero row there.  A written copy equals the layer-0 row.
#include "pk_format.h"

#include <cstdio>
#include <cstring>
#include <memory>

#include "pickle_b200.h"

namespace pk {

namespace {

constexpr char kMagic[8] = {'P', 'K', 'H', 'N', 'S', 'W', '2', '\0'};
constexpr uint64_t kFnvBasis = 1469598103934665603ULL;
constexpr uint64_t kFnvPrime = 1099511628211ULL;

int64_t esize(int32_t dtype) { return dtype == 2 ? 4 : dtype == 3 ? 2 : (dtype == 0 || dtype == 1) ? 1 : 0; }

struct Writer {
    FILE *f;
    uint64_t h = kFnvBasis;
    bool ok = true;
    void put(const void *p, size_t n) {
        if (!ok || n == 0) return;
        const unsigned char *b = static_cast<const unsigned char *>(p);
        for (size_t i = 0; i < n; i++) h = (h ^ b[i]) * kFnvPrime;
        ok = std::fwrite(p, 1, n, f) == n;
    }
    template <class T>
    void val(T v) { put(&v, sizeof(T)); }
};

struct Reader {
    FILE *f;
    uint64_t h = kFnvBasis;
    bool ok = true;
    void get(void *p, size_t n) {
        if (!ok || n == 0) return;
        if (std::fread(p, 1, n, f) != n) {
            ok = false;
            return;
        }
        const unsigned char *b = static_cast<const unsigned char *>(p);
        for (size_t i = 0; i < n; i++) h = (h ^ b[i]) * kFnvPrime;
    }
    template <class T>
    T val() {
        T v{};
        get(&v, sizeof(T));
        return v;
    }
};

struct FileCloser {
    void operator()(FILE *f) const {
        if (f) std::fclose(f);
    }
};

}  // namespace

int write_graph_file(const std::string &path, const FileGraph &g) {
    std::unique_ptr<FILE, FileCloser> fp(std::fopen(path.c_str(), "wb"));
    if (!fp) return PK_ERR_IO;
    Writer w{fp.get()};
    w.put(kMagic, 8);
    w.val<uint32_t>(1);
    w.val<uint32_t>(0);
    w.val<int32_t>(g.metric);
    w.val<int32_t>(g.dtype);
    w.val<int64_t>(g.dim);
    w.val<int64_t>(g.max_degree);
    w.val<int64_t>(g.build_ef);
    w.val<int64_t>(g.capacity);
    w.val<int32_t>(g.enter_level);
    w.val<int32_t>((int32_t)g.layers.size());
    for (const FileLayer &L : g.layers) {
        w.val<int64_t>(L.n);
        w.val<int64_t>(L.layer_capacity);
        w.val<int64_t>(L.cap);
        w.val<int32_t>(L.ent);
        w.val<int32_t>(0);
        w.put(L.ext.data(), sizeof(int32_t) * L.n);
        w.put(L.degree.data(), sizeof(int16_t) * L.n);
        w.put(L.heuristic.data(), sizeof(int16_t) * L.n);
        w.put(L.has_vector.data(), L.n);
        w.put(L.adj.data(), sizeof(int32_t) * L.layer_capacity * L.cap);
        w.put(L.dist.data(), sizeof(float) * L.layer_capacity * L.cap);
    }
    w.put(g.vectors.data(), g.vectors.size());
    uint64_t h = w.h;
    if (w.ok) w.ok = std::fwrite(&h, 1, 8, fp.get()) == 8;
    FILE *raw = fp.release();
    if (std::fclose(raw) != 0) w.ok = false;
    return w.ok ? PK_OK : PK_ERR_IO;
}

int read_graph_file(const std::string &path, FileGraph &g, std::string &err) {
    std::unique_ptr<FILE, FileCloser> fp(std::fopen(path.c_str(), "rb"));
    if (!fp) {
        err = "cannot open " + path;
        return PK_ERR_IO;
    }
    Reader r{fp.get()};
    char magic[8];
    r.get(magic, 8);
    const uint32_t version = r.val<uint32_t>();
    r.val<uint32_t>();
    if (!r.ok || std::memcmp(magic, kMagic, 8) != 0 || version != 1) {
        err = "not a v2 graph file";
        return PK_ERR_FORMAT;
    }
    g.metric = r.val<int32_t>();
    g.dtype = r.val<int32_t>();
    g.dim = r.val<int64_t>();
    g.max_degree = r.val<int64_t>();
    g.build_ef = r.val<int64_t>();
    g.capacity = r.val<int64_t>();
    g.enter_level = r.val<int32_t>();
    const int32_t nl = r.val<int32_t>();
    if (!r.ok) {
        err = "truncated header";
        return PK_ERR_FORMAT;
    }
    if ((g.metric != PK_METRIC_L2 && g.metric != PK_METRIC_IP) || esize(g.dtype) == 0 || g.dim <= 0 ||
        g.dim > 65536 || g.max_degree < 2 || g.max_degree > 16384 || g.capacity < 0 || g.capacity > (1LL << 31) ||
        nl < 0 || nl > 32 || g.enter_level < 0 || (nl > 0 && g.enter_level >= nl)) {
        err = "bad header values";
        return PK_ERR_FORMAT;
    }
    g.layers.assign(nl, FileLayer());
    for (int l = 0; l < nl; l++) {
        FileLayer &L = g.layers[l];
        L.n = r.val<int64_t>();
        L.layer_capacity = r.val<int64_t>();
        L.cap = r.val<int64_t>();
        L.ent = r.val<int32_t>();
        r.val<int32_t>();
        if (!r.ok || L.n < 0 || L.layer_capacity < L.n || L.layer_capacity > (1LL << 31) || L.cap < 1 ||
            L.cap > 32768 || L.n > g.capacity) {
            err = "bad layer header";
            return PK_ERR_FORMAT;
        }
        try {
            L.ext.resize(L.n);
            L.degree.resize(L.n);
            L.heuristic.resize(L.n);
            L.has_vector.resize(L.n);
            L.adj.resize((size_t)(L.layer_capacity * L.cap));
            L.dist.resize((size_t)(L.layer_capacity * L.cap));
        } catch (...) {
            err = "out of host memory";
            return PK_ERR_OOM;
        }
        r.get(L.ext.data(), sizeof(int32_t) * L.n);
        r.get(L.degree.data(), sizeof(int16_t) * L.n);
        r.get(L.heuristic.data(), sizeof(int16_t) * L.n);
        r.get(L.has_vector.data(), L.n);
        r.get(L.adj.data(), sizeof(int32_t) * L.layer_capacity * L.cap);
        r.get(L.dist.data(), sizeof(float) * L.layer_capacity * L.cap);
        if (!r.ok) {
            err = "truncated layer";
            return PK_ERR_FORMAT;
        }
    }
    const int64_t n0 = nl ? g.layers[0].n : 0;
    try {
        g.vectors.resize((size_t)(n0 * g.dim * esize(g.dtype)));
    } catch (...) {
        err = "out of host memory";
        return PK_ERR_OOM;
    }
    r.get(g.vectors.data(), g.vectors.size());
    const uint64_t want = r.h;
    uint64_t got = 0;
    if (!r.ok || std::fread(&got, 1, 8, fp.get()) != 8) {
        err = "truncated vectors or checksum";
        return PK_ERR_FORMAT;
    }
    if (got != want) {
        err = "checksum mismatch";
        return PK_ERR_FORMAT;
    }
    return PK_OK;
}

}  // namespace pk
