// Batched HNSW insertion on the GPU.
//
// The reference inserts one node at a time per thread (HNSWGraph::Insert,
// include/hnsw.hpp:247-302): descend the upper layers greedily, search every
// layer the node joins with ef = build_ef, keep neighbours with
// SelectHeuristic (include/hnsw.hpp:70-116), then write the node's lists
// (AddNode, include/hnsw_layer.hpp:297-332) and add the reverse edges
// (AddEdge, include/hnsw_layer.hpp:360-465).  Its parallel Build runs many
// such inserts at once against a graph that the others are changing.
//
// Here a batch of nodes is inserted in three kernels:
//   1. insert_search_kernel  one warp per new node: the descent, the per-layer
//      searches and SelectHeuristic, all against the graph as it stood before
//      the batch (the searches reuse the exact query path of pk_warp.cuh; for
//      large batches layer 0 may instead take the candidates that the
//      low-precision walk of pk_fast.cu found for the batch's nodes, with
//      their exact distances recomputed here);
//   2. add_node_kernel       one warp per (node, layer): the node's own lists;
//   3. add_edge_kernel       one warp per (layer, target node): the reverse
//      edges into that target, applied in batch order with AddEdge's
//      insert-or-re-prune logic.
// With one node per batch this is exactly the reference's one-thread build,
// except that a list never grows past its cap: where the reference's
// re-prune appends without a bound (include/hnsw_layer.hpp:441-447) and spills
// into the next nodes' rows, a kept neighbour that finds the list full is
// handled as pruned.
#include <cub/cub.cuh>

#include "pk_build.h"
#include "pk_warp.cuh"

namespace pk {

namespace {

using namespace dev;

// std::lower_bound over a float range, with libstdc++'s probe sequence (the
// reference calls it on a prefix that its own re-prune can leave unsorted, so
// the probe sequence, not just the contract, decides the answer).
__device__ __forceinline__ int lower_bound_seq(const float *a, int n, float x) {
    int first = 0, len = n;
    while (len > 0) {
        const int half = len >> 1;
        const int mid = first + half;
        if (a[mid] < x) {
            first = mid + 1;
            len = len - half - 1;
        } else {
            len = half;
        }
    }
    return first;
}

// Rows one dist_rows step covers; occlusion tests run in steps of this many
// and stop at the first step that finds an occluder, as the reference's loops
// stop at the first occluder (the outcome, occluded or not, is the same).
template <int KMAX>
__device__ __forceinline__ int step_rows(const LaneCfg &lc) {
    constexpr int U = KMAX <= 1 ? 4 : KMAX <= 2 ? 2 : 1;
    return U * (32 / lc.G);
}

// Is any of the rows[0..n) closer to the row in qr than `bound`?  (strict:
// d < bound).  Warp-uniform.
template <int DT, int KMAX>
__device__ __forceinline__ bool any_closer(const VecView &vv, const LaneCfg &lc, const uint4 (&qr)[KMAX], bool ip,
                                           const int32_t *rows, float *dd, int n, float bound, int lane) {
    const int step = step_rows<KMAX>(lc);
    for (int c0 = 0; c0 < n; c0 += step) {
        const int m = min(step, n - c0);
        dist_rows<DT, KMAX, false>(vv, lc, qr, ip, rows + c0, dd + c0, m, lane);
        __syncwarp();
        bool hit = false;
        for (int t = lane; t < m; t += 32) hit |= dd[c0 + t] < bound;
        if (__any_sync(kFull, hit)) return true;
    }
    return false;
}

// SelectHeuristic (include/hnsw.hpp:70-116) with keep_pruned = true, on the
// result heap W left in ws.wbuf by search_layer.  Writes R then Pruned to
// out[0..nR+nP) and returns nR | nP << 16.  rrow/rd: shared staging of
// top_k entries.  v1 is occluded when some kept r has d(v1, r) < d(v1, q).
template <int DT, int KMAX>
__device__ int select_heuristic(const VecView &vv, const LaneCfg &lc, uint4 (&qr)[KMAX], bool ip, const DevLayer &L,
                                bool layer0, int wl, int top_k, WarpScratch &ws, int32_t *rrow, float *rd, Ent *out,
                                int lane) {
    MinHeap Wh{ws.ctop, ws.ctail, 0, ws.ccap};
    SmallMinHeap Wd{ws.wbuf, 0};
    if (lane == 0)
        for (int i = 0; i < wl; i++) Wh.push(ws.wbuf[i]);  // for (e : candidates) W.insert(e)
    __syncwarp();
    int nR = 0;
    int whlen = wl;
    while (whlen > 0 && nR < top_k) {
        Ent v1;
        if (lane == 0) v1 = Wh.at(0);
        v1.d = __shfl_sync(kFull, v1.d, 0);
        v1.id = __shfl_sync(kFull, v1.id, 0);
        const int32_t v1row = layer0 ? v1.id : L.vrow[v1.id];
        load_regs<KMAX>(qr, vv.row(v1row), lc, lane, false);
        const bool occl = any_closer<DT, KMAX>(vv, lc, qr, ip, rrow, rd, nR, v1.d, lane);
        if (lane == 0) {
            if (!occl) {
                out[nR] = v1;
                rrow[nR] = v1row;
            } else {
                Wd.push(v1);
            }
            Wh.pop();
        }
        if (!occl) nR++;
        whlen--;
        __syncwarp();
    }
    int nP = 0;
    if (lane == 0)
        while (Wd.len > 0 && nR + nP < top_k) {
            out[nR + nP] = Wd.pop();
            nP++;
        }
    nP = __shfl_sync(kFull, nP, 0);
    __syncwarp();
    return nR | (nP << 16);
}

template <int DT, int KMAX>
__global__ void __launch_bounds__(128, 4) insert_search_kernel(const DevGraph *__restrict__ gp, const LaneCfg lc,
                                                                const InsertSearchArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int gwarp = blockIdx.x * wpb + wib;
    const int64_t row_bytes = gp->row_bytes;
    unsigned char *my = smem + (size_t)wib * insert_smem_per_warp(a.wcap, a.top_k0, row_bytes);

    WarpScratch ws;
    ws.wbuf = reinterpret_cast<Ent *>(my);
    ws.wcap = a.wcap;
    ws.ctop = ws.wbuf + a.wcap;
    ws.st = reinterpret_cast<Stage *>(my + search_stage_off(a.wcap));
    ws.rowbuf = reinterpret_cast<uint8_t *>(my + search_rowbuf_off(a.wcap));
    int32_t *rrow = reinterpret_cast<int32_t *>(ws.rowbuf + kStageRows * row_bytes);
    float *rd = reinterpret_cast<float *>(rrow + a.top_k0);
    ws.bind(a.gs, gwarp);

    const VecView vv{gp->vec0, gp->zero_row, gp->row_bytes};
    const bool ip = gp->metric == PK_METRIC_IP;
    const int L = a.enter_level;

    for (;;) {
        int bi = 0;
        if (lane == 0) bi = atomicAdd(a.work, 1);
        bi = __shfl_sync(kFull, bi, 0);
        if (bi >= a.nb) break;
        const int lvl = a.levels[bi];
        const int32_t pos = a.pos0 + bi;  // its layer-0 id = its vec0 row
        uint4 qr[KMAX];
        load_regs<KMAX>(qr, vv.row(pos), lc, lane, false);
        int32_t cnt[3] = {0, 0, 0};
        bool full = false;
        bool have_enter = false;
        int32_t enter = -1;
        if (a.graph_nonempty) {
            for (int level = L; level >= lvl + 1 && !full; --level) {
                const DevLayer Ly = gp->L[level];
                const int32_t e0 = have_enter ? enter : Ly.ent;
                const int32_t c = slide_layer<DT, KMAX, false>(vv, lc, qr, ip, Ly, e0, ws, cnt, full, lane);
                const int32_t dn = Ly.down[c];
                enter = dn >= 0 ? dn : gp->L[level - 1].ent;
                have_enter = true;
            }
            const int top_search = lvl < L ? lvl : L;
            for (int level = top_search; level >= 0 && !full; --level) {
                const DevLayer Ly = gp->L[level];
                const int32_t e0 = have_enter ? enter : Ly.ent;
                const int top_k = level == 0 ? a.top_k0 : a.top_k0 / 2;
                int wl = 0;
                if (level == 0 && a.l0_cand) {
                    // the walk's candidates with their exact distances, kept
                    // as the result heap of efc entries the search would leave
                    const int32_t *cl = a.l0_cand + (int64_t)bi * a.l0_stride;
                    MaxHeap W{ws.wbuf, 0};
                    for (int j0 = 0; j0 < a.efc; j0 += 32) {
                        const int j = j0 + lane;
                        const int32_t v = j < a.efc ? cl[j] : -1;
                        const bool ok = v >= 0 && v < a.pos0;
                        const unsigned m = __ballot_sync(kFull, ok);
                        if (ok) {
                            const int p = __popc(m & ((1u << lane) - 1));
                            ws.st->id[p] = v;
                            ws.st->row[p] = v;
                        }
                        __syncwarp();
                        const int nn = __popc(m);
                        dist_rows<DT, KMAX, false>(vv, lc, qr, ip, ws.st->row, ws.st->d, nn, lane);
                        __syncwarp();
                        if (lane == 0)
                            for (int t = 0; t < nn; t++) {
                                const float d = ws.st->d[t];
                                if (W.len < a.efc || W.a[0].d > d) {
                                    W.push(Ent{d, ws.st->id[t]});
                                    if (W.len > a.efc) W.pop();
                                }
                            }
                        __syncwarp();
                    }
                    wl = __shfl_sync(kFull, W.len, 0);
                } else {
                    wl = search_layer<DT, KMAX, false>(vv, lc, qr, ip, Ly, level == 0, e0, a.efc, ws, cnt, full, lane);
                    if (full) break;
                }
                // The batch's earlier nodes (j < bi) are not in the graph yet;
                // offer every one that joins this layer to the result set, as
                // if the search had reached it.  With one node per batch there
                // are none, and the insertion is the reference's exactly.
                {
                    MaxHeap W{ws.wbuf, wl};
                    for (int j0 = 0; j0 < bi; j0 += 32) {
                        const int j = j0 + lane;
                        const bool ok = j < bi && a.levels[j] >= level;
                        const unsigned m = __ballot_sync(kFull, ok);
                        if (ok) {
                            const int p = __popc(m & ((1u << lane) - 1));
                            ws.st->id[p] = a.node_id[(int64_t)j * a.max_levels + level];
                            ws.st->row[p] = a.pos0 + j;
                        }
                        __syncwarp();
                        const int nn = __popc(m);
                        dist_rows<DT, KMAX, false>(vv, lc, qr, ip, ws.st->row, ws.st->d, nn, lane);
                        __syncwarp();
                        if (lane == 0)
                            for (int t = 0; t < nn; t++) {
                                const float d = ws.st->d[t];
                                if (W.len < a.efc || W.a[0].d > d) {
                                    W.push(Ent{d, ws.st->id[t]});
                                    if (W.len > a.efc) W.pop();
                                }
                            }
                        __syncwarp();
                    }
                    wl = __shfl_sync(kFull, W.len, 0);
                }
                Ent *out = reinterpret_cast<Ent *>(a.out) + ((int64_t)bi * a.max_levels + level) * a.top_k0;
                const int rp = select_heuristic<DT, KMAX>(vv, lc, qr, ip, Ly, level == 0, wl, top_k, ws, rrow, rd,
                                                           out, lane);
                if (lane == 0) a.counts[(int64_t)bi * a.max_levels + level] = rp;
                // next entry: R[0] (include/hnsw.hpp:275-276), one level down
                if (level > 0) {
                    const int32_t r0 = out[0].id;
                    const int32_t dn = Ly.down[r0];
                    enter = dn >= 0 ? dn : gp->L[level - 1].ent;
                    have_enter = true;
                }
                load_regs<KMAX>(qr, vv.row(pos), lc, lane, false);
                __syncwarp();
            }
        }
        if (full && lane == 0) atomicAdd(a.work + 1, 1);
        __syncwarp();
    }
}

// AddNode (include/hnsw_layer.hpp:297-332) and the bookkeeping of NewInID
// (include/hnsw_layer.hpp:168-177), one warp per (batch node, layer).
__global__ void add_node_kernel(DevGraph *__restrict__ gp, const AddNodeArgs a) {
    const int lane = threadIdx.x & 31;
    const int64_t w = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (w >= a.nitems) return;
    const int bi = a.item_node[w];
    const int lv = a.item_level[w];
    const int32_t id = a.item_id[w];
    DevLayer &L = gp->L[lv];
    const int64_t base = (int64_t)id * L.cap;
    const bool add = lv <= a.top_inserted[bi];
    if (a.meta_only) {
        // NewInID bookkeeping, before the batch's searches: external id, the
        // id one layer down, and which row holds this layer's copy of the
        // vector (none above the highest layer the node searched,
        // include/hnsw.hpp:283-297)
        if (lane == 0) {
            L.ext[id] = a.ext_ids[bi];
            if (lv > 0) {
                L.down[id] = a.item_down[w];
                L.vrow[id] = add ? a.pos0 + bi : -1;
            }
        }
        return;
    }
    int heur = 0, deg = 0;
    if (add) {
        const int rp = a.counts[(int64_t)bi * a.max_levels + lv];
        const int nR = rp & 0xffff, nP = rp >> 16;
        const Ent *src = reinterpret_cast<const Ent *>(a.out) + ((int64_t)bi * a.max_levels + lv) * a.top_k0;
        heur = nR < L.cap ? nR : (int)L.cap;
        deg = heur + nP < L.cap ? heur + nP : (int)L.cap;
        for (int i = lane; i < deg; i += 32) {
            // R[0..heur) then Pruned[0..deg-heur): contiguous in src
            const Ent e = src[i < heur ? i : nR + (i - heur)];
            L.adj[base + i] = e.id;
            L.dist[base + i] = e.d;
        }
    }
    if (lane == 0) {
        L.deg[id] = deg;
        L.heu[id] = heur;
    }
}

// AddEdge (include/hnsw_layer.hpp:360-465) for every reverse edge of the
// batch, one warp per (layer, target), edges applied in batch order.
template <int DT, int KMAX>
__global__ void __launch_bounds__(128) add_edge_kernel(DevGraph *__restrict__ gp, const LaneCfg lc,
                                                       const AddEdgeArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int64_t seg = (int64_t)blockIdx.x * (blockDim.x >> 5) + wib;
    if (seg >= *a.nseg) return;
    const int capmax = a.capmax;
    unsigned char *my = smem + (size_t)wib * add_edge_smem_per_warp(capmax);
    Ent *hw = reinterpret_cast<Ent *>(my);
    Ent *hd = hw + capmax + 2;
    int32_t *rows = reinterpret_cast<int32_t *>(hd + capmax + 2);
    float *dd = reinterpret_cast<float *>(rows + capmax + 2);

    const VecView vv{gp->vec0, gp->zero_row, gp->row_bytes};
    const bool ip = gp->metric == PK_METRIC_IP;
    const int64_t e0 = a.seg_start[seg], e1 = a.seg_start[seg + 1];
    const uint64_t key0 = a.keys[e0];
    const int lv = (int)(key0 >> 58);
    DevLayer &L = gp->L[lv];
    const int32_t t = (int32_t)((key0 >> 27) & 0x7fffffffull);
    const int cap = (int)L.cap;
    int32_t *adj = L.adj + (int64_t)t * cap;
    float *dist = L.dist + (int64_t)t * cap;
    const bool layer0 = lv == 0;
    auto vrow_of = [&](int32_t v) -> int32_t { return layer0 ? v : L.vrow[v]; };
    uint4 qr[KMAX];

    for (int64_t e = e0; e < e1; e++) {
        const int64_t slot = (int64_t)(a.keys[e] & ((1ull << 27) - 1));
        const Ent src = reinterpret_cast<const Ent *>(a.edges)[slot];  // (distance, new node id)
        const int32_t nid = src.id;
        const float distance = src.d;
        // lists of a loaded reference graph may have spilled past cap; only
        // the node's own row is used here
        const int degree = min(L.deg[t], cap);
        const int heur = min(L.heu[t], degree);
        __syncwarp();
        int offset = 0;
        if (lane == 0) offset = lower_bound_seq(dist, heur, distance);
        offset = __shfl_sync(kFull, offset, 0);
        // occlusion test against the closer part of the heuristic prefix
        load_regs<KMAX>(qr, vv.row(vrow_of(nid)), lc, lane, false);
        for (int i = lane; i < offset; i += 32) rows[i] = vrow_of(adj[i]);
        __syncwarp();
        bool ins = !any_closer<DT, KMAX>(vv, lc, qr, ip, rows, dd, offset, distance, lane);
        if (ins && offset >= cap) ins = false;
        if (!ins) {
            // insert into the distance-sorted pruned suffix
            if (lane == 0) {
                int32_t *adj_p = adj + heur;
                float *dist_p = dist + heur;
                const int pruned = degree - heur;
                const int off = lower_bound_seq(dist_p, pruned, distance);
                if (off == pruned && degree < cap) {
                    adj_p[off] = nid;
                    dist_p[off] = distance;
                    L.deg[t] = degree + 1;
                } else if (off < pruned) {
                    const int end = degree < cap ? pruned : pruned - 1;
                    for (int i = end; i > off; i--) {
                        adj_p[i] = adj_p[i - 1];
                        dist_p[i] = dist_p[i - 1];
                    }
                    adj_p[off] = nid;
                    dist_p[off] = distance;
                    L.deg[t] = degree + (degree < cap ? 1 : 0);
                }
            }
            __syncwarp();
            continue;
        }
        // re-run the heuristic over the tail
        SmallMinHeap W{hw, 0}, Wd{hd, 0};
        if (lane == 0) {
            for (int i = offset; i < degree; i++) W.push(Ent{dist[i], adj[i]});
            adj[offset] = nid;
            dist[offset] = distance;
        }
        int cur_h = offset + 1;
        int wlen = degree - offset;
        __syncwarp();
        while (wlen > 0) {
            Ent v1;
            if (lane == 0) v1 = W.pop();
            v1.d = __shfl_sync(kFull, v1.d, 0);
            v1.id = __shfl_sync(kFull, v1.id, 0);
            wlen--;
            load_regs<KMAX>(qr, vv.row(vrow_of(v1.id)), lc, lane, false);
            for (int i = lane; i < cur_h; i += 32) rows[i] = vrow_of(adj[i]);
            __syncwarp();
            bool keep = !any_closer<DT, KMAX>(vv, lc, qr, ip, rows, dd, cur_h, v1.d, lane);
            if (keep && cur_h >= cap) keep = false;
            if (lane == 0) {
                if (keep) {
                    adj[cur_h] = v1.id;
                    dist[cur_h] = v1.d;
                } else {
                    Wd.push(v1);
                }
            }
            if (keep) cur_h++;
            __syncwarp();
        }
        if (lane == 0) {
            int cur_deg = cur_h;
            while (cur_deg < cap && Wd.len > 0) {
                const Ent x = Wd.pop();
                adj[cur_deg] = x.id;
                dist[cur_deg] = x.d;
                cur_deg++;
            }
            L.heu[t] = cur_h;
            L.deg[t] = cur_deg;
        }
        __syncwarp();
    }
}

// Reverse-edge records of the batch.  Slot s = (bi * max_levels + lv) * top_k0
// + i holds edge i of node bi's list on layer lv; its sort key orders edges by
// (layer, target, slot), i.e. by target and then by batch order.
__global__ void edge_keys_kernel(const EdgeKeyArgs a) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= a.nslots) return;
    const int64_t per_node = (int64_t)a.max_levels * a.top_k0;
    const int bi = (int)(s / per_node);
    const int lv = (int)((s / a.top_k0) % a.max_levels);
    const int i = (int)(s % a.top_k0);
    uint64_t key = ~0ull;
    Ent ed{0.f, -1};
    if (lv <= a.top_inserted[bi] && lv <= a.levels[bi]) {
        const int rp = a.counts[(int64_t)bi * a.max_levels + lv];
        const int n = (rp & 0xffff) + (rp >> 16);
        if (i < n) {
            const Ent e = reinterpret_cast<const Ent *>(a.out)[s];
            key = ((uint64_t)lv << 58) | ((uint64_t)(uint32_t)e.id << 27) | (uint64_t)s;
            ed = Ent{e.d, a.node_id[(int64_t)bi * a.max_levels + lv]};
        }
    }
    a.keys[s] = key;
    reinterpret_cast<Ent *>(a.edges)[s] = ed;
}

__global__ void seg_marks_kernel(const uint64_t *keys, int64_t n, int32_t *flags) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t k = keys[i];
    const bool valid = k != ~0ull;
    const bool start = valid && (i == 0 || (keys[i - 1] >> 27) != (k >> 27));
    flags[i] = start ? 1 : 0;
}

__global__ void seg_collect_kernel(const uint64_t *keys, const int32_t *flags, const int32_t *scan, int64_t n,
                                   int64_t *seg_start, int32_t *nseg) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (flags[i]) seg_start[scan[i]] = i;
    const bool valid = keys[i] != ~0ull;
    const bool last_valid = valid && (i == n - 1 || keys[i + 1] == ~0ull);
    if (last_valid) {
        const int ns = scan[i] + flags[i];
        *nseg = ns;
        seg_start[ns] = i + 1;
    }
}

template <int DT>
void *pick_search(int kmax) {
    switch (kmax) {
        case 1: return (void *)insert_search_kernel<DT, 1>;
        case 2: return (void *)insert_search_kernel<DT, 2>;
        case 4: return (void *)insert_search_kernel<DT, 4>;
        case 8: return (void *)insert_search_kernel<DT, 8>;
        case 16: return (void *)insert_search_kernel<DT, 16>;
        case 32: return (void *)insert_search_kernel<DT, 32>;
        default: return nullptr;
    }
}
template <int DT>
void *pick_edge(int kmax) {
    switch (kmax) {
        case 1: return (void *)add_edge_kernel<DT, 1>;
        case 2: return (void *)add_edge_kernel<DT, 2>;
        case 4: return (void *)add_edge_kernel<DT, 4>;
        case 8: return (void *)add_edge_kernel<DT, 8>;
        case 16: return (void *)add_edge_kernel<DT, 16>;
        case 32: return (void *)add_edge_kernel<DT, 32>;
        default: return nullptr;
    }
}
void *insert_search_ptr(int dtype, int kmax) {
    switch (dtype) {
        case PK_DTYPE_U8: return pick_search<PK_DTYPE_U8>(kmax);
        case PK_DTYPE_I8: return pick_search<PK_DTYPE_I8>(kmax);
        case PK_DTYPE_F32: return pick_search<PK_DTYPE_F32>(kmax);
        case PK_DTYPE_F16: return pick_search<PK_DTYPE_F16>(kmax);
        default: return nullptr;
    }
}
void *add_edge_ptr(int dtype, int kmax) {
    switch (dtype) {
        case PK_DTYPE_U8: return pick_edge<PK_DTYPE_U8>(kmax);
        case PK_DTYPE_I8: return pick_edge<PK_DTYPE_I8>(kmax);
        case PK_DTYPE_F32: return pick_edge<PK_DTYPE_F32>(kmax);
        case PK_DTYPE_F16: return pick_edge<PK_DTYPE_F16>(kmax);
        default: return nullptr;
    }
}

}  // namespace

int insert_search_blocks_per_sm(int dtype, const LaneCfg &lc, int wpb, size_t smem) {
    void *fn = insert_search_ptr(dtype, lc.KMAX);
    if (!fn) return 0;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, wpb * 32, smem) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_insert_search(const DevGraph *g, int dtype, const LaneCfg &lc, const InsertSearchArgs &a, int grid,
                                 int wpb, size_t smem, cudaStream_t s) {
    void *fn = insert_search_ptr(dtype, lc.KMAX);
    if (!fn) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    void *args[] = {(void *)&g, (void *)&lc, (void *)&a};
    return cudaLaunchKernel(fn, dim3(grid), dim3(wpb * 32), args, smem, s);
}

cudaError_t launch_add_node(DevGraph *g, const AddNodeArgs &a, cudaStream_t s) {
    if (a.nitems == 0) return cudaSuccess;
    const int wpb = 4;
    const int64_t grid = (a.nitems + wpb - 1) / wpb;
    add_node_kernel<<<(unsigned)grid, wpb * 32, 0, s>>>(g, a);
    return cudaGetLastError();
}

cudaError_t launch_add_edges(DevGraph *g, int dtype, const LaneCfg &lc, EdgeWork &w, const EdgeKeyArgs &ka,
                             int capmax, cudaStream_t s) {
    const int64_t n = ka.nslots;
    if (n == 0) return cudaSuccess;
    edge_keys_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(ka);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    size_t tmp = w.temp_bytes;
    // the key carries the slot number, so sorting keys alone keeps batch order
    e = cub::DeviceRadixSort::SortKeys(w.temp, tmp, ka.keys, w.keys_sorted, (int)n, 0, 63, s);
    if (e != cudaSuccess) return e;
    seg_marks_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(w.keys_sorted, n, w.flags);
    tmp = w.temp_bytes;
    e = cub::DeviceScan::ExclusiveSum(w.temp, tmp, w.flags, w.scan, (int)n, s);
    if (e != cudaSuccess) return e;
    cudaMemsetAsync(w.nseg, 0, sizeof(int32_t), s);
    seg_collect_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(w.keys_sorted, w.flags, w.scan, n, w.seg_start,
                                                                  w.nseg);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    void *fn = add_edge_ptr(dtype, lc.KMAX);
    if (!fn) return cudaErrorInvalidValue;
    const int wpb = 4;
    const size_t smem = (size_t)wpb * add_edge_smem_per_warp(capmax);
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    AddEdgeArgs ea;
    ea.keys = w.keys_sorted;
    ea.edges = ka.edges;
    ea.seg_start = w.seg_start;
    ea.nseg = w.nseg;
    ea.capmax = capmax;
    // one warp per segment; at most one segment per edge slot
    const int64_t grid = (n + wpb - 1) / wpb;
    void *args[] = {(void *)&g, (void *)&lc, (void *)&ea};
    return cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(wpb * 32), args, smem, s);
}

size_t edge_sort_temp_bytes(int64_t n) {
    size_t a = 0, b = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, a, (const uint64_t *)nullptr, (uint64_t *)nullptr, (int)n, 0, 63);
    cub::DeviceScan::ExclusiveSum(nullptr, b, (const int32_t *)nullptr, (int32_t *)nullptr, (int)n);
    return a > b ? a : b;
}

}  // namespace pk
