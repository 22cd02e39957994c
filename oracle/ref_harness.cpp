// Harness around the reference's own, unmodified pickle::v2 headers.
//
// TEST INFRASTRUCTURE.  oracle/Makefile compiles this file against the
// reference's include/ directory with the reference's Release flags
// (CMakeLists.txt:15-17 plus CMake's -DNDEBUG) into oracle/_ref/pk_ref.
// Tests and bench.py's CPU baseline run that binary as a subprocess; nothing
// in the product links or calls it.  One graph per process, because the
// reference's per-thread visited tables are sized on first use
// (include/visited.hpp:266-269) and a second, taller graph in the same process
// would index past them.
//
// Commands (every array is a .npy file; see oracle/pk_npy.h):
//   build  --data X.npy --metric l2|ip --M m --efc e --threads t
//          [--order ids.npy(int32)] [--levels lv.npy(uint8)] --out g.pkg
//       Runs HNSWGraph::Build (include/hnsw.hpp:497-507).  --levels replaces the
//       random_device level draw of InitBuffer (include/hnsw.hpp:222-245,
//       include/util.hpp:38-64) so that a build can be reproduced; with
//       --threads 1 the build is then deterministic.
//   search --graph g.pkg --queries Q.npy --k k --ef ef --threads t
//          [--repeat r] [--dynamic] [--ids out.npy] [--dists out.npy] [--metrics]
//          [--kq k.npy(int32) --efq ef.npy(int32)]
//       Runs the batch AnnSearch (include/hnsw.hpp:528-541) timed with a
//       steady clock around the whole batch, as benchmark/hnsw_pickle.cpp:79-86
//       does, and the collect_metric pass (benchmark/hnsw_pickle.cpp:88-92).
//       By default the distance kernels are instantiated with a fixed Dim
//       for 96/100/128/200 like benchmark/hnsw_pickle.cpp:9-27 (the timed
//       path); --dynamic uses std::dynamic_extent (the metric path).
//       With --kq/--efq every query has its own k and ef: the batch loop of
//       include/hnsw.hpp:528-541 (OpenMP dynamic,20) over the single-query
//       AnnSearch (:509-525) with that query's values; --k is then the row
//       width of --ids/--dists.
//   dist   --a A.npy --b B.npy --metric l2|ip --out D.npy
//       Row-wise pickle::Distance (include/distance.hpp:10-20) for KATs.
#include <omp.h>
#include "hnsw.hpp"

#include <chrono>
#include <cstdio>
#include <map>
#include <string>
#include <vector>
#include <algorithm>
#include <numeric>

#include "pk_npy.h"
#include "pk_graphfile.h"

using namespace pickle;
using namespace pickle::v2;

// ---- access to HNSWGraph's private state (it declares no friend) ----------
template <class Tag, typename Tag::type P>
struct Rob {
    friend typename Tag::type get(Tag) { return P; }
};
#define PK_ROB(NAME, TYPE, MEMBER)                         \
    struct NAME {                                          \
        typedef TYPE HNSWGraph::*type;                     \
        friend type get(NAME);                             \
    };                                                     \
    template struct Rob<NAME, &HNSWGraph::MEMBER>;
PK_ROB(G_max_degree, size_t, m_max_degree)
PK_ROB(G_build_ef, size_t, m_build_ef)
PK_ROB(G_capacity, size_t, m_capacity)
PK_ROB(G_df, DistFunc, m_df)
PK_ROB(G_enter_level, internal_id_t, m_enter_level)
PK_ROB(G_layers, std::vector<HNSWLayerPtr>, m_hnsw_layers)
PK_ROB(G_insert_level, std::vector<uint8_t>, m_insert_level)
PK_ROB(G_layer_capacity, std::vector<size_t>, m_layer_capacity)
PK_ROB(G_data, NDArray, m_data)

// ---- access to HNSWLayer's private state through its declared friend ------
namespace pickle::v2 {
class Serializer {
public:
    static void Load(HNSWLayer &L, const pkf_layer &F, int64_t capacity, DataType dtype, int64_t dim, DistFunc df,
                     const char *vec0, const std::vector<int32_t> &ext_to_in0, size_t esz) {
        std::vector<size_t> shape = {(size_t)F.layer_capacity, (size_t)dim};
        L.Init((size_t)F.cap, (size_t)F.layer_capacity, (external_id_t)capacity, dtype, shape, df);
        L.m_next_id = (internal_id_t)F.n;
        L.m_is_empty = F.n == 0;
        L.m_ent_id = F.ent_id;
        for (int64_t i = 0; i < F.n; i++) {
            L.m_node_list[i].m_ext_id = F.ext[i];
            L.m_node_list[i].m_degree = F.degree[i];
            L.m_node_list[i].m_heuristic = F.heuristic[i];
            L.m_ext2in_table.at(F.ext[i]) = (internal_id_t)i;
            if (F.has_vector[i])
                std::memcpy(L.m_data.get_raw(i), vec0 + (size_t)ext_to_in0.at(F.ext[i]) * dim * esz, dim * esz);
        }
        std::memcpy(L.m_adj_list.data(), F.adj, sizeof(int32_t) * F.layer_capacity * F.cap);
        std::memcpy(L.m_dist_list.data(), F.dist, sizeof(float) * F.layer_capacity * F.cap);
    }
    static void Save(const HNSWLayer &L, pkf_layer &F) {
        F.n = L.m_next_id;
        F.layer_capacity = (int64_t)L.m_capacity;
        F.cap = (int64_t)L.m_max_degree;
        F.ent_id = L.m_ent_id;
        F.ext = (int32_t *)malloc(4 * F.n + 4);
        F.degree = (int16_t *)malloc(2 * F.n + 2);
        F.heuristic = (int16_t *)malloc(2 * F.n + 2);
        F.has_vector = (uint8_t *)calloc(F.n + 1, 1);
        F.adj = (int32_t *)malloc(4 * F.layer_capacity * F.cap + 4);
        F.dist = (float *)malloc(4 * F.layer_capacity * F.cap + 4);
        for (int64_t i = 0; i < F.n; i++) {
            F.ext[i] = L.m_node_list[i].m_ext_id;
            F.degree[i] = L.m_node_list[i].m_degree;
            F.heuristic[i] = L.m_node_list[i].m_heuristic;
        }
        std::memcpy(F.adj, L.m_adj_list.data(), sizeof(int32_t) * F.layer_capacity * F.cap);
        std::memcpy(F.dist, L.m_dist_list.data(), sizeof(float) * F.layer_capacity * F.cap);
    }
    static const char *Row(const HNSWLayer &L, int64_t i) { return (const char *)L.m_data.get_raw(i); }
    static int64_t Count(const HNSWLayer &L) { return L.m_next_id; }
    static int64_t Cap(const HNSWLayer &L) { return (int64_t)L.m_max_degree; }
    static int Degree(const HNSWLayer &L, int64_t i) { return L.m_node_list[i].m_degree; }
};
}  // namespace pickle::v2

// ---- small helpers ---------------------------------------------------------
static std::map<std::string, std::string> parse(int argc, char **argv, int from) {
    std::map<std::string, std::string> a;
    for (int i = from; i < argc; i++) {
        std::string k = argv[i];
        if (k.rfind("--", 0) != 0) continue;
        if (i + 1 < argc && std::string(argv[i + 1]).rfind("--", 0) != 0) {
            a[k.substr(2)] = argv[i + 1];
            i++;
        } else {
            a[k.substr(2)] = "1";
        }
    }
    return a;
}

static DataType npy_dtype(const pk_npy &a) {
    if (a.kind == 'u' && a.word == 1) return DataType::Uint8;
    if (a.kind == 'i' && a.word == 1) return DataType::Int8;
    if (a.kind == 'f' && a.word == 4) return DataType::Float32;
    if (a.kind == 'f' && a.word == 2) return DataType::Float16;
    fprintf(stderr, "unsupported npy dtype %c%d\n", a.kind, a.word);
    exit(2);
}

static DistFunc metric_of(const std::string &s) {
    if (s == "l2") return DistFunc::L2;
    if (s == "ip") return DistFunc::IP;
    fprintf(stderr, "unsupported metric %s\n", s.c_str());
    exit(2);
}

static size_t esize(DataType t) {
    return t == DataType::Float32 ? 4 : t == DataType::Float16 ? 2 : 1;
}

static NDArray to_ndarray(const pk_npy &a) {
    auto holder = std::make_shared<std::vector<char>>((char *)a.data,
                                                      (char *)a.data + a.shape[0] * a.shape[1] * a.word);
    return NDArray(holder, npy_dtype(a), {(size_t)a.shape[0], (size_t)a.shape[1]});
}

// The same Dim specialisations as benchmark/hnsw_pickle.cpp:9-27.
template <class F>
static void dim_switch(size_t dim, bool dynamic, F &&f) {
    if (dynamic) { f(std::integral_constant<size_t, std::dynamic_extent>{}); return; }
    switch (dim) {
        case 128: f(std::integral_constant<size_t, 128>{}); break;
        case 100: f(std::integral_constant<size_t, 100>{}); break;
        case 96: f(std::integral_constant<size_t, 96>{}); break;
        case 200: f(std::integral_constant<size_t, 200>{}); break;
        default: f(std::integral_constant<size_t, std::dynamic_extent>{}); break;
    }
}

template <class F>
static void type_switch(DataType t, F &&f) {
    switch (t) {
        case DataType::Uint8: f((uint8_t *)nullptr); break;
        case DataType::Int8: f((int8_t *)nullptr); break;
        case DataType::Float32: f((float *)nullptr); break;
        case DataType::Float16: f((float16_t *)nullptr); break;
    }
}

static int save_graph(HNSWGraph &g, DataType dtype, size_t dim, const char *path) {
    auto &layers = g.*get(G_layers{});
    pkf_graph F{};
    F.metric = (int32_t)(g.*get(G_df{}));
    F.dtype = (int32_t)dtype;
    F.dim = (int64_t)dim;
    F.max_degree = (int64_t)(g.*get(G_max_degree{}));
    F.build_ef = (int64_t)(g.*get(G_build_ef{}));
    F.capacity = (int64_t)(g.*get(G_capacity{}));
    F.enter_level = g.*get(G_enter_level{});
    F.num_layers = (int32_t)layers.size();
    F.layers = (pkf_layer *)calloc(F.num_layers, sizeof(pkf_layer));
    for (int l = 0; l < F.num_layers; l++) Serializer::Save(*layers[l], F.layers[l]);
    int64_t n0 = F.num_layers ? F.layers[0].n : 0;
    size_t es = esize(dtype);
    // has_vector: a layer's row is either the node's layer-0 row (written by
    // AddNode) or still zero (AddNode never ran for that level).
    std::vector<int64_t> in0(F.capacity, -1);
    for (int64_t i = 0; i < n0; i++) in0.at(F.layers[0].ext[i]) = i;
    std::vector<char> zero(dim * es, 0);
    for (int l = 0; l < F.num_layers; l++)
        for (int64_t i = 0; i < F.layers[l].n; i++) {
            const char *row = Serializer::Row(*layers[l], i);
            int64_t j = in0.at(F.layers[l].ext[i]);
            if (j >= 0 && std::memcmp(row, Serializer::Row(*layers[0], j), dim * es) == 0) {
                F.layers[l].has_vector[i] = 1;
            } else if (std::memcmp(row, zero.data(), dim * es) == 0) {
                F.layers[l].has_vector[i] = 0;
            } else {
                fprintf(stderr, "layer %d row %lld is neither the node's vector nor zero\n", l, (long long)i);
                return -9;
            }
        }
    F.vectors = malloc(n0 * dim * es + 1);
    for (int64_t i = 0; i < n0; i++) std::memcpy((char *)F.vectors + i * dim * es, Serializer::Row(*layers[0], i), dim * es);
    int rc = pkf_write(path, &F);
    pkf_free(&F);
    return rc;
}

static HNSWGraph *load_graph(const char *path, DataType *dtype_out, size_t *dim_out) {
    pkf_graph F;
    int rc = pkf_read(path, &F);
    if (rc != 0) {
        fprintf(stderr, "pkf_read(%s) failed: %d\n", path, rc);
        exit(3);
    }
    auto *g = new HNSWGraph((size_t)F.max_degree, (size_t)F.build_ef, (DistFunc)F.metric);
    DataType dtype = (DataType)F.dtype;
    size_t dim = (size_t)F.dim, es = esize(dtype);
    g->*get(G_capacity{}) = (size_t)F.capacity;
    g->*get(G_enter_level{}) = F.enter_level;
    std::vector<int32_t> ext_to_in0(F.capacity, -1);
    for (int64_t i = 0; i < (F.num_layers ? F.layers[0].n : 0); i++) ext_to_in0.at(F.layers[0].ext[i]) = (int32_t)i;
    NDArray data(dtype, {(size_t)F.capacity, dim});
    std::vector<uint8_t> levels(F.capacity, 0);
    std::vector<size_t> layer_cap(F.num_layers);
    auto &layers = g->*get(G_layers{});
    layers.clear();
    for (int l = 0; l < F.num_layers; l++) {
        auto L = std::make_shared<HNSWLayer>();
        Serializer::Load(*L, F.layers[l], F.capacity, dtype, (int64_t)dim, (DistFunc)F.metric, (const char *)F.vectors,
                         ext_to_in0, es);
        layers.push_back(L);
        layer_cap[l] = (size_t)F.layers[l].layer_capacity;
        for (int64_t i = 0; i < F.layers[l].n; i++) levels.at(F.layers[l].ext[i]) = (uint8_t)l;
    }
    for (int64_t e = 0; e < F.capacity; e++)
        if (ext_to_in0[e] >= 0)
            std::memcpy(data.get_raw(e), (const char *)F.vectors + (size_t)ext_to_in0[e] * dim * es, dim * es);
    g->*get(G_data{}) = data;
    g->*get(G_insert_level{}) = levels;
    g->*get(G_layer_capacity{}) = layer_cap;
    pkf_free(&F);
    *dtype_out = dtype;
    *dim_out = dim;
    return g;
}

// ---- commands --------------------------------------------------------------
static int cmd_build(std::map<std::string, std::string> &a) {
    pk_npy X;
    if (pk_npy_read(a["data"].c_str(), &X) != 0 || X.ndim != 2) { fprintf(stderr, "bad --data\n"); return 2; }
    DataType dtype = npy_dtype(X);
    size_t n = (size_t)X.shape[0], dim = (size_t)X.shape[1];
    DistFunc df = metric_of(a["metric"]);
    size_t M = std::stoul(a.count("M") ? a["M"] : "32");
    size_t efc = std::stoul(a.count("efc") ? a["efc"] : "100");
    int threads = a.count("threads") ? std::stoi(a["threads"]) : omp_get_max_threads();
    omp_set_num_threads(threads);

    std::vector<external_id_t> order;
    if (a.count("order")) {
        pk_npy O;
        if (pk_npy_read(a["order"].c_str(), &O) != 0 || O.word != 4 || (size_t)O.shape[0] != n) {
            fprintf(stderr, "bad --order\n");
            return 2;
        }
        order.assign((int32_t *)O.data, (int32_t *)O.data + n);
        free(O.data);
    } else {
        order = GetRandIndices<external_id_t>(n);  // as benchmark/hnsw_pickle.cpp:42
    }
    NDArray all = to_ndarray(X);
    free(X.data);

    auto *g = new HNSWGraph(M, efc, df);
    auto t0 = std::chrono::steady_clock::now();
    if (!a.count("levels")) {
        type_switch(dtype, [&](auto *tp) {
            using T = std::remove_pointer_t<decltype(tp)>;
            dim_switch(dim, false, [&](auto D) { g->Build<T, decltype(D)::value>(order, all); });
        });
    } else {
        pk_npy LV;
        if (pk_npy_read(a["levels"].c_str(), &LV) != 0 || LV.word != 1 || (size_t)LV.shape[0] != n) {
            fprintf(stderr, "bad --levels\n");
            return 2;
        }
        // Build with the given levels: the steps of HNSWGraph::Build and
        // InitBuffer (include/hnsw.hpp:222-245, :497-507) with the level draw
        // replaced, then the same parallel Insert loop.
        g->*get(G_data{}) = all;
        g->InitBuffer(n);
        std::vector<uint8_t> levels((uint8_t *)LV.data, (uint8_t *)LV.data + n);
        free(LV.data);
        int top = *std::max_element(levels.begin(), levels.end());
        std::vector<size_t> lcap(top + 1, 0);
        for (uint8_t l : levels)
            for (int j = 0; j <= l; j++) lcap[j]++;
        auto &layers = g->*get(G_layers{});
        layers.clear();
        for (int i = 0; i <= top; i++) {
            auto L = std::make_shared<HNSWLayer>();
            L->Init(i == 0 ? 2 * M : M, lcap[i], (external_id_t)n, dtype, {lcap[i], dim}, df);
            layers.push_back(L);
        }
        g->*get(G_insert_level{}) = levels;
        g->*get(G_layer_capacity{}) = lcap;
        type_switch(dtype, [&](auto *tp) {
            using T = std::remove_pointer_t<decltype(tp)>;
            dim_switch(dim, false, [&](auto D) {
                constexpr size_t Dim = decltype(D)::value;
#pragma omp parallel for schedule(static, 100)
                for (size_t i = 0; i < n; i++) {
                    auto q = all.get_span<T, Dim>((size_t)order[i]);
                    g->Insert<T, Dim>(order[i], q);
                }
            });
        });
    }
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    int over = 0;
    auto &layers = g->*get(G_layers{});
    for (auto &L : layers)
        for (int64_t i = 0; i < Serializer::Count(*L); i++) over += Serializer::Degree(*L, i) > Serializer::Cap(*L);
    int rc = save_graph(*g, dtype, dim, a["out"].c_str());
    printf("{\"build_s\": %.4f, \"threads\": %d, \"n\": %zu, \"layers\": %zu, \"degree_over_cap\": %d, \"save_rc\": %d}\n",
           secs, threads, n, layers.size(), over, rc);
    return rc == 0 ? 0 : 4;
}

static int cmd_search(std::map<std::string, std::string> &a) {
    DataType dtype;
    size_t dim;
    HNSWGraph *g = load_graph(a["graph"].c_str(), &dtype, &dim);
    pk_npy Q;
    if (pk_npy_read(a["queries"].c_str(), &Q) != 0 || Q.ndim != 2 || (size_t)Q.shape[1] != dim ||
        npy_dtype(Q) != dtype) {
        fprintf(stderr, "bad --queries\n");
        return 2;
    }
    size_t nq = (size_t)Q.shape[0];
    NDArray queries = to_ndarray(Q);
    free(Q.data);
    int k = std::stoi(a["k"]), ef = std::stoi(a["ef"]);
    int threads = a.count("threads") ? std::stoi(a["threads"]) : omp_get_max_threads();
    int repeat = a.count("repeat") ? std::stoi(a["repeat"]) : 1;
    bool dynamic = a.count("dynamic") > 0;
    omp_set_num_threads(threads);

    std::vector<int32_t> kq, efq;
    if (a.count("kq") || a.count("efq")) {
        pk_npy KQ, EQ;
        if (pk_npy_read(a["kq"].c_str(), &KQ) != 0 || pk_npy_read(a["efq"].c_str(), &EQ) != 0 || KQ.word != 4 ||
            EQ.word != 4 || (size_t)KQ.shape[0] != nq || (size_t)EQ.shape[0] != nq) {
            fprintf(stderr, "bad --kq/--efq\n");
            return 2;
        }
        kq.assign((int32_t *)KQ.data, (int32_t *)KQ.data + nq);
        efq.assign((int32_t *)EQ.data, (int32_t *)EQ.data + nq);
        free(KQ.data);
        free(EQ.data);
    }

    std::vector<std::vector<Entry>> results;
    std::vector<double> secs;
    type_switch(dtype, [&](auto *tp) {
        using T = std::remove_pointer_t<decltype(tp)>;
        dim_switch(dim, dynamic, [&](auto D) {
            constexpr size_t Dim = decltype(D)::value;
            for (int r = 0; r < repeat; r++) {
                auto t0 = std::chrono::steady_clock::now();
                if (kq.empty()) {
                    results = g->AnnSearch<T, Dim, false>(k, ef, queries);
                } else {
                    results.assign(nq, {});
#pragma omp parallel for schedule(dynamic, 20)
                    for (size_t i = 0; i < nq; i++)
                        results[i] = g->AnnSearch<T, Dim, false>(kq[i], efq[i], queries.get_span<T, Dim>(i));
                }
                secs.push_back(std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
            }
        });
    });
    std::vector<double> sorted = secs;
    std::sort(sorted.begin(), sorted.end());
    double med = sorted[sorted.size() / 2];

    double hop = 0, dist = 0, base_hop = 0, base_dist = 0, nbr = 0;
    if (a.count("metrics")) {
        Profiler::Global()->Reset();
        type_switch(dtype, [&](auto *tp) {
            using T = std::remove_pointer_t<decltype(tp)>;
            (void)g->AnnSearch<T, std::dynamic_extent, true>(k, ef, queries);
        });
        auto P = Profiler::Global();
        hop = P->GetHop();
        dist = P->GetDist();
        base_hop = P->GetHop(0);
        base_dist = P->GetDist(0);
        nbr = P->GetNeighbor();
    }
    if (a.count("ids") || a.count("dists")) {
        std::vector<int32_t> ids(nq * k, -1);
        std::vector<float> ds(nq * k, std::numeric_limits<float>::max());
        for (size_t i = 0; i < nq; i++)
            for (size_t j = 0; j < results[i].size() && j < (size_t)k; j++) {
                ids[i * k + j] = results[i][j].m_vid;
                ds[i * k + j] = results[i][j].m_dist;
            }
        int64_t shape[2] = {(int64_t)nq, (int64_t)k};
        if (a.count("ids")) pk_npy_write(a["ids"].c_str(), "<i4", 2, shape, ids.data());
        if (a.count("dists")) pk_npy_write(a["dists"].c_str(), "<f4", 2, shape, ds.data());
    }
    printf("{\"nq\": %zu, \"k\": %d, \"ef\": %d, \"threads\": %d, \"repeat\": %d, \"median_s\": %.6f, "
           "\"qps\": %.1f, \"dynamic\": %d, \"hop\": %.0f, \"dist\": %.0f, \"base_hop\": %.0f, "
           "\"base_dist\": %.0f, \"neighbor\": %.0f, \"all_s\": [",
           nq, k, ef, threads, repeat, med, nq / med, (int)dynamic, hop, dist, base_hop, base_dist, nbr);
    for (size_t i = 0; i < secs.size(); i++) printf("%s%.6f", i ? ", " : "", secs[i]);
    printf("]}\n");
    return 0;
}

static int cmd_dist(std::map<std::string, std::string> &a) {
    pk_npy A, B;
    if (pk_npy_read(a["a"].c_str(), &A) != 0 || pk_npy_read(a["b"].c_str(), &B) != 0 || A.shape[0] != B.shape[0] ||
        A.shape[1] != B.shape[1] || A.kind != B.kind || A.word != B.word) {
        fprintf(stderr, "bad --a/--b\n");
        return 2;
    }
    DistFunc df = metric_of(a["metric"]);
    DataType dtype = npy_dtype(A);
    size_t n = (size_t)A.shape[0], dim = (size_t)A.shape[1];
    bool dynamic = a.count("dynamic") > 0;
    std::vector<float> out(n);
    type_switch(dtype, [&](auto *tp) {
        using T = std::remove_pointer_t<decltype(tp)>;
        dim_switch(dim, dynamic, [&](auto D) {
            constexpr size_t Dim = decltype(D)::value;
            for (size_t i = 0; i < n; i++) {
                std::span<const T, Dim> x((const T *)A.data + i * dim, dim);
                std::span<const T, Dim> y((const T *)B.data + i * dim, dim);
                out[i] = Distance<T, Dim>(x, y, df);
            }
        });
    });
    int64_t shape[1] = {(int64_t)n};
    return pk_npy_write(a["out"].c_str(), "<f4", 1, shape, out.data()) == 0 ? 0 : 4;
}

int main(int argc, char **argv) {
    if (argc < 2) {
        fprintf(stderr, "usage: pk_ref build|search|dist ...\n");
        return 2;
    }
    auto a = parse(argc, argv, 2);
    std::string cmd = argv[1];
    if (cmd == "build") return cmd_build(a);
    if (cmd == "search") return cmd_search(a);
    if (cmd == "dist") return cmd_dist(a);
    fprintf(stderr, "unknown command %s\n", cmd.c_str());
    return 2;
}
