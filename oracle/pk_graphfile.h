/*
 * Reader/writer for the v2 HNSW graph file, oracle side.  TEST INFRASTRUCTURE:
 * used by the reference harness (ref_harness.cpp) and the C restatement
 * (pk_oracle.c) so that the reference, the restatement and the device library
 * can search one and the same graph.  The device library has its own,
 * independent implementation of the format (pickle_b200/csrc/pk_format.cpp);
 * tests cross-read files written by either side.
 *
 * The reference's serializer (include/serializer.hpp:27-55) writes, per layer,
 * a size, num_nodes, max_degree and then the ext/degree/adj/dist arrays, but
 * it targets the retired v0 layer and does not compile against the live v2
 * layer (include/hnsw_layer.hpp:57-83).  This format keeps that per-layer
 * record style and adds what the v2 layer holds:
 *
 *   char     magic[8]      "PKHNSW2\0"
 *   uint32   version       1
 *   uint32   flags         0
 *   int32    metric        DistFunc value: 1 = L2, 2 = IP   (include/common.hpp:28-33)
 *   int32    dtype         DataType value: 0 u8, 1 i8, 2 f32, 3 f16 (include/common.hpp:21-26)
 *   int64    dim
 *   int64    max_degree    M; layer 0 holds 2M slots (include/hnsw.hpp:235)
 *   int64    build_ef
 *   int64    capacity      number of external ids (m_capacity, include/hnsw.hpp:130)
 *   int32    enter_level   (include/hnsw.hpp:133)
 *   int32    num_layers
 *   per layer:
 *     int64  n             nodes present (m_next_id, include/hnsw_layer.hpp:71)
 *     int64  layer_capacity slots allocated (m_capacity)
 *     int64  cap           adjacency slots per node (m_max_degree)
 *     int32  ent_id        (m_ent_id)
 *     int32  reserved
 *     int32  ext[n]        internal -> external id (NodeMeta.m_ext_id)
 *     int16  degree[n]     (NodeMeta.m_degree)
 *     int16  heuristic[n]  (NodeMeta.m_heuristic)
 *     uint8  has_vector[n] 1 if the layer's copy of the node's vector was
 *                          written, 0 if it is still the zero row: Insert calls
 *                          AddNode (which copies the vector) only for levels up
 *                          to the highest level it searched, so a node whose
 *                          level is above the current entry level keeps zero
 *                          rows in the layers above (include/hnsw.hpp:283-297).
 *                          The first node of every new top layer, which is that
 *                          layer's entry point, is such a node.
 *     int32  adj[layer_capacity*cap]  fixed stride cap, -1 padded.  A node's
 *                          neighbours are adj[v*cap, v*cap + degree[v]); the
 *                          reference lets degree exceed cap, in which case the
 *                          list runs on into the following rows (its AddEdge
 *                          appends without a bound, include/hnsw_layer.hpp:441-447)
 *     float  dist[layer_capacity*cap] FLT_MAX padded
 *   dtype    vectors[n0*dim]  layer-0 internal order.  A layer's written copy of a
 *                          node's vector equals its layer-0 row
 *                          (include/hnsw_layer.hpp:304-307), so upper layers
 *                          store only has_vector.
 *   uint64   checksum      version 1: FNV-1a 64 over every preceding byte.
 *                          version 2 (same layout; written by the device
 *                          library): the preceding bytes in blocks of 4 MiB,
 *                          each block's digest FNV-1a 64 over its
 *                          little-endian 64-bit words (the last one zero
 *                          padded) and then its length, the checksum FNV-1a 64
 *                          over the block digests and then the total length -
 *                          the blocks can be verified in parallel.
 * Both versions are read here; pkf_write writes version 1.
 */
#ifndef PK_ORACLE_GRAPHFILE_H
#define PK_ORACLE_GRAPHFILE_H

#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#define PKF_MAGIC "PKHNSW2"

typedef struct {
    int64_t n, layer_capacity, cap;
    int32_t ent_id;
    int32_t *ext;
    int16_t *degree;
    int16_t *heuristic;
    uint8_t *has_vector;
    int32_t *adj;
    float *dist;
} pkf_layer;

typedef struct {
    int32_t metric, dtype;
    int64_t dim, max_degree, build_ef, capacity;
    int32_t enter_level, num_layers;
    pkf_layer *layers;
    void *vectors;
} pkf_graph;

static inline int pkf_elem_size(int dtype) {
    switch (dtype) {
        case 0: case 1: return 1;
        case 2: return 4;
        case 3: return 2;
        default: return 0;
    }
}

#define PKF_FNV_BASIS 1469598103934665603ULL
#define PKF_FNV_PRIME 1099511628211ULL
#define PKF_BLOCK ((uint64_t)4 << 20)

/* The version 2 checksum, computed over a stream of bytes. */
typedef struct {
    uint64_t file_h, blk_h, total, word, blk_len;
    unsigned wfill;
} pkf_bh;

static inline void pkf_bh_init(pkf_bh *b) {
    b->file_h = b->blk_h = PKF_FNV_BASIS;
    b->total = b->word = b->blk_len = 0;
    b->wfill = 0;
}
static inline void pkf_bh_close_block(pkf_bh *b) {
    if (b->wfill) {
        b->blk_h = (b->blk_h ^ b->word) * PKF_FNV_PRIME;
        b->word = 0;
        b->wfill = 0;
    }
    b->blk_h = (b->blk_h ^ b->blk_len) * PKF_FNV_PRIME;
    b->file_h = (b->file_h ^ b->blk_h) * PKF_FNV_PRIME;
    b->blk_h = PKF_FNV_BASIS;
    b->blk_len = 0;
}
static inline void pkf_bh_update(pkf_bh *b, const void *p, size_t n) {
    const unsigned char *c = (const unsigned char *)p;
    while (n) {
        uint64_t room = PKF_BLOCK - b->blk_len;
        size_t take = n < room ? n : (size_t)room, i = 0;
        for (; i < take && b->wfill; i++) {
            b->word |= (uint64_t)c[i] << (8 * b->wfill);
            if (++b->wfill == 8) {
                b->blk_h = (b->blk_h ^ b->word) * PKF_FNV_PRIME;
                b->word = 0;
                b->wfill = 0;
            }
        }
        for (; i + 8 <= take; i += 8) {
            uint64_t w;
            memcpy(&w, c + i, 8);
            b->blk_h = (b->blk_h ^ w) * PKF_FNV_PRIME;
        }
        for (; i < take; i++) b->word |= (uint64_t)c[i] << (8 * b->wfill++);
        b->blk_len += take;
        b->total += take;
        c += take;
        n -= take;
        if (b->blk_len == PKF_BLOCK) pkf_bh_close_block(b);
    }
}
static inline uint64_t pkf_bh_final(pkf_bh *b) {
    if (b->blk_len) pkf_bh_close_block(b);
    return (b->file_h ^ b->total) * PKF_FNV_PRIME;
}

typedef struct {
    FILE *f;
    uint64_t h;
    int err;
    int version;
    pkf_bh bh;
} pkf_io;

static inline void pkf_hash(pkf_io *io, const void *p, size_t n) {
    if (io->version == 2) {
        pkf_bh_update(&io->bh, p, n);
        return;
    }
    const unsigned char *b = (const unsigned char *)p;
    uint64_t h = io->h;
    for (size_t i = 0; i < n; i++) {
        h ^= b[i];
        h *= PKF_FNV_PRIME;
    }
    io->h = h;
}

static inline void pkf_w(pkf_io *io, const void *p, size_t n) {
    if (io->err || n == 0) return;
    if (fwrite(p, 1, n, io->f) != n) io->err = 1;
    pkf_hash(io, p, n);
}

static inline void pkf_r(pkf_io *io, void *p, size_t n) {
    if (io->err || n == 0) return;
    if (fread(p, 1, n, io->f) != n) { io->err = 1; return; }
    pkf_hash(io, p, n);
}

static inline void pkf_free(pkf_graph *g) {
    if (!g) return;
    if (g->layers) {
        for (int l = 0; l < g->num_layers; l++) {
            free(g->layers[l].ext);
            free(g->layers[l].degree);
            free(g->layers[l].heuristic);
            free(g->layers[l].has_vector);
            free(g->layers[l].adj);
            free(g->layers[l].dist);
        }
        free(g->layers);
    }
    free(g->vectors);
    memset(g, 0, sizeof(*g));
}

static inline int pkf_write(const char *path, const pkf_graph *g) {
    pkf_io io;
    memset(&io, 0, sizeof(io));
    io.f = fopen(path, "wb");
    io.h = PKF_FNV_BASIS;
    io.version = 1;
    if (!io.f) return -1;
    char magic[8] = PKF_MAGIC;
    uint32_t version = 1, flags = 0;
    pkf_w(&io, magic, 8);
    pkf_w(&io, &version, 4);
    pkf_w(&io, &flags, 4);
    pkf_w(&io, &g->metric, 4);
    pkf_w(&io, &g->dtype, 4);
    pkf_w(&io, &g->dim, 8);
    pkf_w(&io, &g->max_degree, 8);
    pkf_w(&io, &g->build_ef, 8);
    pkf_w(&io, &g->capacity, 8);
    pkf_w(&io, &g->enter_level, 4);
    pkf_w(&io, &g->num_layers, 4);
    for (int l = 0; l < g->num_layers; l++) {
        const pkf_layer *L = &g->layers[l];
        int32_t reserved = 0;
        pkf_w(&io, &L->n, 8);
        pkf_w(&io, &L->layer_capacity, 8);
        pkf_w(&io, &L->cap, 8);
        pkf_w(&io, &L->ent_id, 4);
        pkf_w(&io, &reserved, 4);
        pkf_w(&io, L->ext, 4 * (size_t)L->n);
        pkf_w(&io, L->degree, 2 * (size_t)L->n);
        pkf_w(&io, L->heuristic, 2 * (size_t)L->n);
        pkf_w(&io, L->has_vector, (size_t)L->n);
        pkf_w(&io, L->adj, 4 * (size_t)(L->layer_capacity * L->cap));
        pkf_w(&io, L->dist, 4 * (size_t)(L->layer_capacity * L->cap));
    }
    int64_t n0 = g->num_layers > 0 ? g->layers[0].n : 0;
    pkf_w(&io, g->vectors, (size_t)(n0 * g->dim) * (size_t)pkf_elem_size(g->dtype));
    uint64_t h = io.h;
    if (!io.err && fwrite(&h, 1, 8, io.f) != 8) io.err = 1;
    if (fclose(io.f) != 0) io.err = 1;
    return io.err ? -2 : 0;
}

/* Returns 0 on success, -1 open failure, -2 truncated, -3 bad magic/version,
 * -4 bad header values, -5 checksum mismatch, -6 out of memory. */
static inline int pkf_read(const char *path, pkf_graph *g) {
    memset(g, 0, sizeof(*g));
    pkf_io io;
    memset(&io, 0, sizeof(io));
    io.f = fopen(path, "rb");
    io.h = PKF_FNV_BASIS;
    if (!io.f) return -1;
    char head[16];
    uint32_t version, flags;
    if (fread(head, 1, 16, io.f) != 16) { fclose(io.f); return -2; }
    memcpy(&version, head + 8, 4);
    memcpy(&flags, head + 12, 4);
    if (memcmp(head, PKF_MAGIC, 8) != 0 || (version != 1 && version != 2)) { fclose(io.f); return -3; }
    io.version = (int)version;
    pkf_bh_init(&io.bh);
    pkf_hash(&io, head, 16);
    pkf_r(&io, &g->metric, 4);
    pkf_r(&io, &g->dtype, 4);
    pkf_r(&io, &g->dim, 8);
    pkf_r(&io, &g->max_degree, 8);
    pkf_r(&io, &g->build_ef, 8);
    pkf_r(&io, &g->capacity, 8);
    pkf_r(&io, &g->enter_level, 4);
    pkf_r(&io, &g->num_layers, 4);
    if (io.err) { fclose(io.f); return -2; }
    if (pkf_elem_size(g->dtype) == 0 || (g->metric != 1 && g->metric != 2) || g->dim <= 0 || g->dim > 65536 ||
        g->num_layers < 0 || g->num_layers > 64 || g->capacity < 0 || g->max_degree <= 0 ||
        g->max_degree > 16384) {
        fclose(io.f);
        return -4;
    }
    g->layers = (pkf_layer *)calloc((size_t)(g->num_layers > 0 ? g->num_layers : 1), sizeof(pkf_layer));
    if (!g->layers) { fclose(io.f); return -6; }
    for (int l = 0; l < g->num_layers; l++) {
        pkf_layer *L = &g->layers[l];
        int32_t reserved;
        pkf_r(&io, &L->n, 8);
        pkf_r(&io, &L->layer_capacity, 8);
        pkf_r(&io, &L->cap, 8);
        pkf_r(&io, &L->ent_id, 4);
        pkf_r(&io, &reserved, 4);
        if (io.err) { pkf_free(g); fclose(io.f); return -2; }
        if (L->n < 0 || L->cap <= 0 || L->cap > 32768 || L->layer_capacity > (int64_t)1 << 31 ||
            L->layer_capacity < L->n) {
            pkf_free(g); fclose(io.f); return -4;
        }
        size_t n = (size_t)L->n, e = (size_t)(L->layer_capacity * L->cap);
        L->ext = (int32_t *)malloc(4 * n + 4);
        L->degree = (int16_t *)malloc(2 * n + 2);
        L->heuristic = (int16_t *)malloc(2 * n + 2);
        L->has_vector = (uint8_t *)malloc(n + 1);
        L->adj = (int32_t *)malloc(4 * e + 4);
        L->dist = (float *)malloc(4 * e + 4);
        if (!L->ext || !L->degree || !L->heuristic || !L->has_vector || !L->adj || !L->dist) {
            pkf_free(g); fclose(io.f); return -6;
        }
        pkf_r(&io, L->ext, 4 * n);
        pkf_r(&io, L->degree, 2 * n);
        pkf_r(&io, L->heuristic, 2 * n);
        pkf_r(&io, L->has_vector, n);
        pkf_r(&io, L->adj, 4 * e);
        pkf_r(&io, L->dist, 4 * e);
        if (io.err) { pkf_free(g); fclose(io.f); return -2; }
    }
    int64_t n0 = g->num_layers > 0 ? g->layers[0].n : 0;
    size_t vb = (size_t)(n0 * g->dim) * (size_t)pkf_elem_size(g->dtype);
    g->vectors = malloc(vb ? vb : 1);
    if (!g->vectors) { pkf_free(g); fclose(io.f); return -6; }
    pkf_r(&io, g->vectors, vb);
    uint64_t want = io.version == 2 ? pkf_bh_final(&io.bh) : io.h, got = 0;
    if (io.err || fread(&got, 1, 8, io.f) != 8) { pkf_free(g); fclose(io.f); return -2; }
    fclose(io.f);
    if (got != want) { pkf_free(g); return -5; }
    return 0;
}

#endif
