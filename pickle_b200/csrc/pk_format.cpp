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
//   u64 checksum of all preceding bytes: version 1 = FNV-1a 64 over the bytes;
//   version 2 (what this library writes) = the bytes in 4 MiB blocks, each
//   block's digest FNV-1a 64 over its little-endian 64-bit words (the last
//   one zero padded) and then its length, the checksum FNV-1a 64 over the
//   block digests and then the total length, so that a reader verifies the
//   blocks in parallel.  Both versions are read.
//
// Reading maps the file (mmap) and hands out pointers into the mapping: the
// arrays go from the mapping straight to the device, with no copy in host
// memory, while the block digests are checked by all host cores.
//
// has_vector[v] is 0 where the layer's copy of the node's vector was never
// written: the reference's Insert copies it only into layers up to the
// highest one it searched (include/hnsw.hpp:283-297), so nodes that open a new
// top layer keep a zero row there.  A written copy equals the layer-0 row.
#include "pk_format.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "pickle_b200.h"

namespace pk {

namespace {

constexpr char kMagic[8] = {'P', 'K', 'H', 'N', 'S', 'W', '2', '\0'};
constexpr uint64_t kFnvBasis = 1469598103934665603ULL;
constexpr uint64_t kFnvPrime = 1099511628211ULL;
constexpr uint64_t kBlock = 4ull << 20;
constexpr uint32_t kWriteVersion = 2;

int64_t esize(int32_t dtype) { return dtype == 2 ? 4 : dtype == 3 ? 2 : (dtype == 0 || dtype == 1) ? 1 : 0; }

// Digest of one block: FNV-1a 64 over its little-endian words, then its length.
uint64_t block_digest(const uint8_t *p, uint64_t n) {
    uint64_t h = kFnvBasis;
    uint64_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w;
        std::memcpy(&w, p + i, 8);
        h = (h ^ w) * kFnvPrime;
    }
    if (i < n) {
        uint64_t w = 0;
        std::memcpy(&w, p + i, (size_t)(n - i));
        h = (h ^ w) * kFnvPrime;
    }
    return (h ^ n) * kFnvPrime;
}

// Version 2 checksum of n bytes, the blocks digested by all host cores.
uint64_t block_checksum(const uint8_t *p, uint64_t n) {
    const uint64_t nb = (n + kBlock - 1) / kBlock;
    std::vector<uint64_t> dig((size_t)nb);
    const unsigned nt = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(nb, std::thread::hardware_concurrency()));
    std::atomic<uint64_t> next{0};
    auto work = [&]() {
        for (uint64_t b; (b = next.fetch_add(1)) < nb;)
            dig[(size_t)b] = block_digest(p + b * kBlock, std::min(kBlock, n - b * kBlock));
    };
    std::vector<std::thread> ts;
    for (unsigned t = 1; t < nt; t++) ts.emplace_back(work);
    work();
    for (auto &t : ts) t.join();
    uint64_t h = kFnvBasis;
    for (uint64_t d : dig) h = (h ^ d) * kFnvPrime;
    return (h ^ n) * kFnvPrime;
}

uint64_t byte_checksum(const uint8_t *p, uint64_t n) {
    uint64_t h = kFnvBasis;
    for (uint64_t i = 0; i < n; i++) h = (h ^ p[i]) * kFnvPrime;
    return h;
}

// The version 2 checksum over a stream of writes.
struct BlockHasher {
    uint64_t file_h = kFnvBasis, blk_h = kFnvBasis, total = 0, word = 0, blk_len = 0;
    unsigned wfill = 0;
    void close_block() {
        if (wfill) {
            blk_h = (blk_h ^ word) * kFnvPrime;
            word = 0;
            wfill = 0;
        }
        blk_h = (blk_h ^ blk_len) * kFnvPrime;
        file_h = (file_h ^ blk_h) * kFnvPrime;
        blk_h = kFnvBasis;
        blk_len = 0;
    }
    void update(const uint8_t *c, size_t n) {
        while (n) {
            const size_t take = (size_t)std::min<uint64_t>(n, kBlock - blk_len);
            size_t i = 0;
            for (; i < take && wfill; i++) {
                word |= (uint64_t)c[i] << (8 * wfill);
                if (++wfill == 8) {
                    blk_h = (blk_h ^ word) * kFnvPrime;
                    word = 0;
                    wfill = 0;
                }
            }
            for (; i + 8 <= take; i += 8) {
                uint64_t w;
                std::memcpy(&w, c + i, 8);
                blk_h = (blk_h ^ w) * kFnvPrime;
            }
            for (; i < take; i++) word |= (uint64_t)c[i] << (8 * wfill++);
            blk_len += take;
            total += take;
            c += take;
            n -= take;
            if (blk_len == kBlock) close_block();
        }
    }
    uint64_t final() {
        if (blk_len) close_block();
        return (file_h ^ total) * kFnvPrime;
    }
};

struct Writer {
    FILE *f;
    BlockHasher h;
    bool ok = true;
    void put(const void *p, size_t n) {
        if (!ok || n == 0) return;
        h.update(static_cast<const uint8_t *>(p), n);
        ok = std::fwrite(p, 1, n, f) == n;
    }
    template <class T>
    void val(T v) { put(&v, sizeof(T)); }
};

struct FileCloser {
    void operator()(FILE *f) const {
        if (f) std::fclose(f);
    }
};

// Bounds-checked cursor over the mapping.
struct Cursor {
    const uint8_t *p;
    uint64_t n, off = 0;
    bool ok = true;
    const uint8_t *take(uint64_t bytes) {
        if (!ok || bytes > n - off) {
            ok = false;
            return nullptr;
        }
        const uint8_t *q = p + off;
        off += bytes;
        return q;
    }
    template <class T>
    T val() {
        T v{};
        const uint8_t *q = take(sizeof(T));
        if (q) std::memcpy(&v, q, sizeof(T));
        return v;
    }
};

}  // namespace

int write_graph_file(const std::string &path, const FileGraph &g) {
    std::unique_ptr<FILE, FileCloser> fp(std::fopen(path.c_str(), "wb"));
    if (!fp) return PK_ERR_IO;
    Writer w{fp.get()};
    w.put(kMagic, 8);
    w.val<uint32_t>(kWriteVersion);
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
    uint64_t h = w.h.final();
    if (w.ok) w.ok = std::fwrite(&h, 1, 8, fp.get()) == 8;
    FILE *raw = fp.release();
    if (std::fclose(raw) != 0) w.ok = false;
    return w.ok ? PK_OK : PK_ERR_IO;
}

MappedGraph::~MappedGraph() {
    if (base && base != MAP_FAILED) munmap(const_cast<uint8_t *>(base), (size_t)bytes);
}

int map_graph_file(const std::string &path, MappedGraph &g, std::string &err) {
    const int fd = open(path.c_str(), O_RDONLY);
    if (fd < 0) {
        err = "cannot open " + path;
        return PK_ERR_IO;
    }
    struct stat st;
    if (fstat(fd, &st) != 0) {
        close(fd);
        err = "cannot stat " + path;
        return PK_ERR_IO;
    }
    if (st.st_size < 64 + 8) {
        close(fd);
        err = "not a v2 graph file";
        return PK_ERR_FORMAT;
    }
    void *m = mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
    close(fd);
    if (m == MAP_FAILED) {
        err = "cannot map " + path;
        return PK_ERR_IO;
    }
    g.base = static_cast<const uint8_t *>(m);
    g.bytes = (uint64_t)st.st_size;
    madvise(m, (size_t)st.st_size, MADV_SEQUENTIAL);
    Cursor r{g.base, g.bytes - 8};
    const uint8_t *magic = r.take(8);
    const uint32_t version = r.val<uint32_t>();
    r.val<uint32_t>();
    if (!r.ok || std::memcmp(magic, kMagic, 8) != 0 || (version != 1 && version != 2)) {
        err = "not a v2 graph file";
        return PK_ERR_FORMAT;
    }
    g.version = version;
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
    g.layers.assign(nl, MappedLayer());
    for (int l = 0; l < nl; l++) {
        MappedLayer &L = g.layers[l];
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
        const uint64_t e = (uint64_t)L.layer_capacity * (uint64_t)L.cap;
        L.ext = r.take(4 * (uint64_t)L.n);
        L.degree = r.take(2 * (uint64_t)L.n);
        L.heuristic = r.take(2 * (uint64_t)L.n);
        L.has_vector = r.take((uint64_t)L.n);
        L.adj = r.take(4 * e);
        L.dist = r.take(4 * e);
        if (!r.ok) {
            err = "truncated layer";
            return PK_ERR_FORMAT;
        }
    }
    const int64_t n0 = nl ? g.layers[0].n : 0;
    g.vector_bytes = (uint64_t)n0 * (uint64_t)g.dim * (uint64_t)esize(g.dtype);
    g.vectors = r.take(g.vector_bytes);
    if (!r.ok || r.off != g.bytes - 8) {
        err = r.ok ? "trailing bytes before the checksum" : "truncated vectors or checksum";
        return PK_ERR_FORMAT;
    }
    uint64_t got = 0;
    std::memcpy(&got, g.base + g.bytes - 8, 8);
    const uint64_t want = version == 2 ? block_checksum(g.base, g.bytes - 8) : byte_checksum(g.base, g.bytes - 8);
    if (got != want) {
        err = "checksum mismatch";
        return PK_ERR_FORMAT;
    }
    return PK_OK;
}

}  // namespace pk
