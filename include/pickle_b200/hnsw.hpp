// Header-only C++ front end of the B200 HNSW index, with the names and call
// shapes of the reference's pickle::v2::HNSWGraph (include/hnsw.hpp:23-220)
// and Serializer (include/serializer.hpp:21-25), implemented over the C ABI of
// pickle_b200.h (link with -lpickle_b200).
//
// Differences a caller of the reference will notice:
//  * failures throw pickle_b200::Error (status code + message) instead of
//    asserting or calling exit(-1) (include/marco.hpp:20-68);
//  * the device index is created on the first Build or Insert, when the
//    element type and dimension are known (the reference learns them from the
//    NDArray as well);
//  * Insert takes a batch (Insert of one row is the batch of one), and a
//    batch of new rows is inserted together on the GPU;
//  * AnnSearch(k, ef, NDArray) runs the whole batch in one device call.
#ifndef PICKLE_B200_HNSW_HPP
#define PICKLE_B200_HNSW_HPP

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <span>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "../pickle_b200.h"

namespace pickle_b200 {

// include/common.hpp:21-33 (same numeric values)
enum class DataType { Uint8 = 0, Int8 = 1, Float32 = 2, Float16 = 3 };
enum class DistFunc { L1 = 0, L2 = 1, IP = 2, RUNTIME = 3 };

// include/queue.hpp:17-28
struct Entry {
    float m_dist{std::numeric_limits<float>::max()};
    int32_t m_vid{-1};
};

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
    if (rc != PK_OK) throw Error(rc, std::string("pickle_b200: ") + pk_last_error());
}

// A 16-bit float storage type (the reference uses _Float16 / __fp16 via the
// float16_t macro, include/marco.hpp:11-17).
struct half_t {
    uint16_t bits;
};

template <class T>
constexpr DataType dtype_of() {
    if constexpr (std::is_same_v<T, uint8_t>) return DataType::Uint8;
    else if constexpr (std::is_same_v<T, int8_t>) return DataType::Int8;
    else if constexpr (std::is_same_v<T, float>) return DataType::Float32;
    else {
        static_assert(sizeof(T) == 2, "element type must be uint8_t, int8_t, float or a 16-bit float");
        return DataType::Float16;
    }
}

// include/ndarray.hpp:17-101: a row-major 2-D byte buffer with a dtype,
// shared (not copied) between owners.
struct NDArray {
    std::shared_ptr<std::vector<char>> m_data;
    std::vector<size_t> m_shape;
    DataType m_dtype{DataType::Float32};

    NDArray() = default;
    NDArray(std::shared_ptr<std::vector<char>> data, DataType dtype, std::vector<size_t> shape)
        : m_data(std::move(data)), m_shape(std::move(shape)), m_dtype(dtype) {}
    size_t rows() const { return m_shape.at(0); }
    size_t cols() const { return m_shape.at(1); }
    const void *raw() const { return m_data->data(); }
};

class HNSWGraph {
public:
    HNSWGraph() = default;
    HNSWGraph(size_t max_degree, size_t build_ef, DistFunc df) { Init(max_degree, build_ef, df); }
    HNSWGraph(const HNSWGraph &) = delete;
    HNSWGraph &operator=(const HNSWGraph &) = delete;
    HNSWGraph(HNSWGraph &&o) noexcept { swap(o); }
    HNSWGraph &operator=(HNSWGraph &&o) noexcept {
        swap(o);
        return *this;
    }
    ~HNSWGraph() {
        if (m_h) pk_index_destroy(m_h);
    }

    void Init(size_t max_degree, size_t build_ef, DistFunc df) {
        if (df != DistFunc::L2 && df != DistFunc::IP) throw Error(PK_ERR_ARG, "pickle_b200: DistFunc must be L2 or IP");
        m_max_degree = max_degree;
        m_build_ef = build_ef;
        m_df = df;
    }

    // Seed of the per-node level draw (the reference uses std::random_device).
    void SetSeed(uint64_t seed) { m_seed = seed; }

    // HNSWGraph::Build (include/hnsw.hpp:497-507): inserts data row ext_ids[i]
    // with external id ext_ids[i], for i = 0, 1, ...
    template <class T, size_t Dim = std::dynamic_extent>
    void Build(const std::vector<int32_t> &ext_ids, const NDArray &data, int32_t max_batch = 0) {
        ensure<T>(data.cols());
        check(pk_index_build(m_h, data.raw(), (int64_t)data.rows(), ext_ids.data(), max_batch));
    }

    // HNSWGraph::Insert (include/hnsw.hpp:247-302), one row.
    template <class T, size_t Dim = std::dynamic_extent>
    void Insert(int32_t ext_id, std::span<const T, Dim> query) {
        ensure<T>(query.size());
        check(pk_index_add(m_h, query.data(), 1, &ext_id, 1));
    }

    // Batch insertion of n rows (row i has external id ext_ids[i]).
    template <class T>
    void InsertBatch(const std::vector<int32_t> &ext_ids, const T *rows, size_t dim, int32_t max_batch = 0) {
        ensure<T>(dim);
        check(pk_index_add(m_h, rows, (int64_t)ext_ids.size(), ext_ids.data(), max_batch));
    }

    // AnnSearch for one query (include/hnsw.hpp:509-525).
    template <class T, size_t Dim = std::dynamic_extent, bool collect_metric = false>
    std::vector<Entry> AnnSearch(int top_k, int search_ef, std::span<const T, Dim> query) const {
        auto r = search_rows(top_k, search_ef, query.data(), 1);
        return r.at(0);
    }

    // AnnSearch for a batch (include/hnsw.hpp:528-541).
    template <class T, size_t Dim = std::dynamic_extent, bool collect_metric = false>
    std::vector<std::vector<Entry>> AnnSearch(int top_k, int search_ef, NDArray queries) const {
        if (queries.m_dtype != dtype_of<T>()) throw Error(PK_ERR_ARG, "pickle_b200: query dtype mismatch");
        return search_rows(top_k, search_ef, queries.raw(), queries.rows());
    }

    pk_index *handle() const { return m_h; }

    static HNSWGraph FromHandle(pk_index *h) {
        HNSWGraph g;
        g.m_h = h;
        int64_t info[12];
        check(pk_index_info(h, info));
        g.m_max_degree = (size_t)info[5];
        g.m_build_ef = (size_t)info[6];
        g.m_df = (DistFunc)info[7];
        g.m_dtype = (DataType)info[8];
        g.m_dim = (size_t)info[4];
        return g;
    }

private:
    pk_index *m_h = nullptr;
    size_t m_max_degree = 0, m_build_ef = 0, m_dim = 0;
    DistFunc m_df = DistFunc::L2;
    DataType m_dtype = DataType::Float32;
    uint64_t m_seed = 0;

    void swap(HNSWGraph &o) noexcept {
        std::swap(m_h, o.m_h);
        std::swap(m_max_degree, o.m_max_degree);
        std::swap(m_build_ef, o.m_build_ef);
        std::swap(m_dim, o.m_dim);
        std::swap(m_df, o.m_df);
        std::swap(m_dtype, o.m_dtype);
        std::swap(m_seed, o.m_seed);
    }

    template <class T>
    void ensure(size_t dim) {
        if (m_h) {
            if (dim != m_dim || dtype_of<T>() != m_dtype) throw Error(PK_ERR_ARG, "pickle_b200: dtype/dim mismatch");
            return;
        }
        check(pk_index_create(&m_h, (int)m_df, (int)dtype_of<T>(), (int64_t)dim, (int64_t)m_max_degree,
                              (int64_t)m_build_ef));
        m_dim = dim;
        m_dtype = dtype_of<T>();
        check(pk_index_set_seed(m_h, m_seed));
    }

    std::vector<std::vector<Entry>> search_rows(int k, int ef, const void *q, size_t nq) const {
        if (!m_h) throw Error(PK_ERR_STATE, "pickle_b200: search before build");
        std::vector<int32_t> ids(nq * (size_t)k);
        std::vector<float> ds(nq * (size_t)k);
        check(pk_index_search(m_h, q, (int64_t)nq, k, ef, ids.data(), ds.data()));
        std::vector<std::vector<Entry>> out(nq);
        for (size_t i = 0; i < nq; i++) {
            for (int j = 0; j < k; j++) {
                if (ids[i * k + j] < 0) break;  // the reference returns min(k, found) entries
                out[i].push_back(Entry{ds[i * k + j], ids[i * k + j]});
            }
        }
        return out;
    }
};

// The persistence pair the reference names (include/serializer.hpp:21-25),
// for the v2 graph.
struct Serializer {
    static void to_disk(const std::string &filename, const HNSWGraph &g) {
        check(pk_index_save(g.handle(), filename.c_str()));
    }
    static HNSWGraph from_disk(const std::string &filename) {
        pk_index *h = nullptr;
        check(pk_index_load(&h, filename.c_str()));
        return HNSWGraph::FromHandle(h);
    }
};

}  // namespace pickle_b200

#endif
