// Host-side task DAG construction.  See dag.hpp.
#include "dag.hpp"

#include <algorithm>

#include "../../include/mustard_b200.h"

namespace mtd {

namespace {
int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
}  // namespace

Dag::Dag(int kind, int64_t n, int64_t tile)
    : kind_(kind), n_(n), tile_(tile), tiles_(static_cast<int>(ceil_div(n, tile))) {}

int64_t Dag::extent(int t) const { return std::min<int64_t>(tile_, n_ - int64_t(t) * tile_); }

bool Dag::valid_tile(const TileId &t) const {
    return t.first >= 0 && t.second >= 0 && t.first < tiles_ && t.second < tiles_;
}

int Dag::add_task(int op, int wi, int wj, const int *reads, int nreads) {
    if (op < MTD_OP_POTRF || op > MTD_OP_GEMM_NN) return -MTD_ERR_INVALID_ARG;
    if (nreads < 0 || nreads > 8 || (nreads > 0 && reads == nullptr)) return -MTD_ERR_INVALID_ARG;
    HostTask t;
    t.op = op;
    t.write = {wi, wj};
    if (!valid_tile(t.write)) return -MTD_ERR_INVALID_ARG;
    for (int r = 0; r < nreads; ++r) {
        TileId id{reads[2 * r], reads[2 * r + 1]};
        if (!valid_tile(id)) return -MTD_ERR_INVALID_ARG;
        t.reads.push_back(id);
    }
    // Operands: the reads other than the written tile, in the caller's order.
    std::vector<TileId> others;
    bool reads_write = false;
    for (const auto &id : t.reads) {
        if (id == t.write) reads_write = true;
        else others.push_back(id);
    }
    // Every operation updates its output in place, so the output tile must be read.
    if (!reads_write) return -MTD_ERR_INVALID_ARG;
    switch (op) {
    case MTD_OP_POTRF:
    case MTD_OP_GETRF:
        if (wi != wj || !others.empty()) return -MTD_ERR_INVALID_ARG;
        t.a = t.write;
        break;
    case MTD_OP_TRSM_RLT:   // writes (i,k), triangular (k,k)
    case MTD_OP_TRSM_RUN:
        if (others.size() != 1) return -MTD_ERR_INVALID_ARG;
        t.a = others[0];
        if (t.a.first != t.a.second || t.a.first != wj || wi == wj) return -MTD_ERR_INVALID_ARG;
        break;
    case MTD_OP_TRSM_LLNU:  // writes (k,i), triangular (k,k)
        if (others.size() != 1) return -MTD_ERR_INVALID_ARG;
        t.a = others[0];
        if (t.a.first != t.a.second || t.a.first != wi || wi == wj) return -MTD_ERR_INVALID_ARG;
        break;
    case MTD_OP_SYRK_LN:    // writes (i,i), reads (i,k)
        if (others.size() != 1 || wi != wj) return -MTD_ERR_INVALID_ARG;
        t.a = others[0];
        if (t.a.first != wi) return -MTD_ERR_INVALID_ARG;
        break;
    case MTD_OP_GEMM_NT:    // writes (j,i), reads A=(j,k), B=(i,k)
        if (others.size() != 2) return -MTD_ERR_INVALID_ARG;
        t.a = others[0];
        t.b = others[1];
        if (t.a.first != wi || t.b.first != wj || t.a.second != t.b.second) return -MTD_ERR_INVALID_ARG;
        break;
    case MTD_OP_GEMM_NN:    // writes (i,j), reads A=(i,k), B=(k,j)
        if (others.size() != 2) return -MTD_ERR_INVALID_ARG;
        t.a = others[0];
        t.b = others[1];
        if (t.a.first != wi || t.b.second != wj || t.a.second != t.b.first) return -MTD_ERR_INVALID_ARG;
        break;
    }

    const int idx = num_tasks();
    // Last writer of every tile in reads + {write} (mustard/mustard.h:279-296) ...
    std::vector<int> dep;
    std::vector<TileId> tiles = t.reads;
    tiles.push_back(t.write);
    for (const auto &id : tiles) {
        auto it = last_writer_.find(id);
        if (it != last_writer_.end()) dep.push_back(it->second);
    }
    // ... and, so that custom graphs are safe, the readers of the tile this task
    // overwrites.  The reference's LU and Cholesky lists never produce such an edge.
    auto rit = readers_since_.find(t.write);
    if (rit != readers_since_.end())
        for (int r : rit->second) dep.push_back(r);
    std::sort(dep.begin(), dep.end());
    dep.erase(std::unique(dep.begin(), dep.end()), dep.end());

    tasks_.push_back(t);
    deps_.push_back(dep);
    last_writer_[t.write] = idx;
    readers_since_[t.write].clear();
    for (const auto &id : t.reads)
        if (id != t.write) readers_since_[id].push_back(idx);
    return idx;
}

int Dag::build_reference_order() {
    const int T = tiles_;
    auto add = [&](int op, int wi, int wj, std::initializer_list<int> r) {
        std::vector<int> v(r);
        int rc = add_task(op, wi, wj, v.data(), static_cast<int>(v.size() / 2));
        return rc < 0 ? -rc : 0;
    };
    int rc = 0;
    if (kind_ == MTD_KIND_CHOLESKY) {
        // mustard/cholesky_mustard.cu:224-395
        for (int k = 0; k < T && !rc; ++k) {
            rc |= add(MTD_OP_POTRF, k, k, {k, k});
            for (int i = k + 1; i < T; ++i) rc |= add(MTD_OP_TRSM_RLT, i, k, {k, k, i, k});
            for (int i = k + 1; i < T; ++i) {
                rc |= add(MTD_OP_SYRK_LN, i, i, {i, i, i, k});
                for (int j = i + 1; j < T; ++j) rc |= add(MTD_OP_GEMM_NT, j, i, {j, i, j, k, i, k});
            }
        }
    } else if (kind_ == MTD_KIND_LU) {
        // mustard/lu_mustard.cu:345-533
        for (int k = 0; k < T && !rc; ++k) {
            rc |= add(MTD_OP_GETRF, k, k, {k, k});
            for (int i = k + 1; i < T; ++i) rc |= add(MTD_OP_TRSM_LLNU, k, i, {k, k, k, i});
            for (int i = k + 1; i < T; ++i) {
                rc |= add(MTD_OP_TRSM_RUN, i, k, {k, k, i, k});
                for (int j = k + 1; j < T; ++j) rc |= add(MTD_OP_GEMM_NN, i, j, {i, k, k, j, i, j});
            }
        }
    } else {
        return MTD_ERR_INVALID_ARG;
    }
    return rc ? MTD_ERR_INVALID_ARG : MTD_OK;
}

int Dag::items_of(int ti) const {
    const HostTask &t = tasks_[ti];
    const int64_t m = extent(t.write.first), n = extent(t.write.second);
    switch (t.op) {
    case MTD_OP_GEMM_NT:
    case MTD_OP_GEMM_NN:
        return static_cast<int>(ceil_div(m, kGemmTile) * ceil_div(n, kGemmTile));
    case MTD_OP_SYRK_LN: {
        int64_t b = ceil_div(m, kGemmTile);
        return static_cast<int>(b * (b + 1) / 2);
    }
    case MTD_OP_TRSM_RLT:
    case MTD_OP_TRSM_RUN:
        return static_cast<int>(ceil_div(m, kPanelRows));
    case MTD_OP_TRSM_LLNU:
        return static_cast<int>(ceil_div(n, kPanelRows));
    default:
        return 1;
    }
}

// Lookahead priority: diagonal factorisations, panel solves and the updates that feed
// the next panel go to the critical-path queue.
int Dag::queue_of(int ti) const {
    const HostTask &t = tasks_[ti];
    switch (t.op) {
    case MTD_OP_POTRF:
    case MTD_OP_GETRF:
    case MTD_OP_TRSM_RLT:
    case MTD_OP_TRSM_RUN:
    case MTD_OP_TRSM_LLNU:
        return 0;
    default: {
        const int k = t.a.second;
        return std::min(t.write.first, t.write.second) == k + 1 ? 0 : 1;
    }
    }
}

int Dag::lower(std::vector<DevTask> &out, std::vector<int> &succ, std::vector<int> &pred_count,
               int64_t queue_cap[kNumQueues]) const {
    const int nt = num_tasks();
    out.assign(nt, DevTask{});
    pred_count.assign(nt, 0);
    for (int q = 0; q < kNumQueues; ++q) queue_cap[q] = 0;

    // A triangular solve reads the inverses of the diagonal blocks that the diagonal
    // factorisation of its triangular tile leaves in the workspace, so the last writer
    // of that tile must be the matching factorisation.
    std::map<TileId, int> writer;
    for (int t = 0; t < nt; ++t) {
        const HostTask &h = tasks_[t];
        if (h.op == MTD_OP_TRSM_RLT || h.op == MTD_OP_TRSM_RUN || h.op == MTD_OP_TRSM_LLNU) {
            auto it = writer.find(h.a);
            const int want = h.op == MTD_OP_TRSM_RLT ? MTD_OP_POTRF : MTD_OP_GETRF;
            if (it == writer.end() || tasks_[it->second].op != want) return MTD_ERR_BAD_DAG;
        }
        writer[h.write] = t;
    }

    std::vector<std::vector<int>> succs(nt);
    for (int t = 0; t < nt; ++t) {
        pred_count[t] = static_cast<int>(deps_[t].size());
        for (int d : deps_[t]) succs[d].push_back(t);
    }
    succ.clear();
    for (int t = 0; t < nt; ++t) {
        const HostTask &h = tasks_[t];
        DevTask &d = out[t];
        d.op = h.op;
        d.queue = queue_of(t);
        d.n_items = items_of(t);
        d.wi = h.write.first;
        d.wj = h.write.second;
        d.ai = h.a.first;
        d.aj = h.a.second;
        d.bi = h.b.first;
        d.bj = h.b.second;
        d.succ_begin = static_cast<int32_t>(succ.size());
        d.succ_count = static_cast<int32_t>(succs[t].size());
        for (int s : succs[t]) succ.push_back(s);
        queue_cap[d.queue] += d.n_items;
    }
    return MTD_OK;
}

}  // namespace mtd
