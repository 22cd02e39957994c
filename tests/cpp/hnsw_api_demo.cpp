// Uses the header-only C++ front end the way a caller of pickle::v2::HNSWGraph
// would: Build from an NDArray, AnnSearch a batch, Serializer round trip.
// Prints "ids <first row>" or "error <code>".  argv[1]: where to write the
// graph file (default: pk_cpp_demo.pkg in the working directory).
#include <cstdio>
#include <random>
#include <string>

#include "pickle_b200/hnsw.hpp"

using namespace pickle_b200;

int main(int argc, char **argv) {
    const std::string path = argc > 1 ? argv[1] : "pk_cpp_demo.pkg";
    const size_t n = 2000, dim = 32, nq = 16;
    std::mt19937 rng(1);
    std::uniform_int_distribution<int> u(0, 255);
    auto data = std::make_shared<std::vector<char>>(n * dim * sizeof(float));
    auto *f = reinterpret_cast<float *>(data->data());
    for (size_t i = 0; i < n * dim; i++) f[i] = (float)u(rng);
    NDArray all(data, DataType::Float32, {n, dim});
    std::vector<int32_t> ext(n);
    for (size_t i = 0; i < n; i++) ext[i] = (int32_t)i;
    auto qd = std::make_shared<std::vector<char>>(nq * dim * sizeof(float));
    std::memcpy(qd->data(), data->data(), qd->size());
    NDArray queries(qd, DataType::Float32, {nq, dim});
    try {
        HNSWGraph g(8, 64, DistFunc::L2);
        g.SetSeed(1);
        g.Build<float>(ext, all);
        auto res = g.AnnSearch<float>(5, 32, queries);
        Serializer::to_disk(path, g);
        HNSWGraph h = Serializer::from_disk(path);
        auto res2 = h.AnnSearch<float>(5, 32, queries);
        bool same = res.size() == res2.size();
        for (size_t i = 0; same && i < res.size(); i++)
            for (size_t j = 0; same && j < res[i].size(); j++)
                same = res[i][j].m_vid == res2[i][j].m_vid && res[i][j].m_dist == res2[i][j].m_dist;
        printf("ids");
        for (auto &e : res[0]) printf(" %d", e.m_vid);
        printf("\nreload %s\n", same ? "same" : "DIFFERENT");
        return same ? 0 : 1;
    } catch (const Error &e) {
        printf("error %d %s\n", e.code, e.what());
        return 3;
    }
}
