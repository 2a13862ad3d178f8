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

int64_t Dag::origin(int t) const { return edges_.empty() ? int64_t(t) * tile_ : edges_[t]; }

int64_t Dag::extent(int t) const {
    return edges_.empty() ? std::min<int64_t>(tile_, n_ - int64_t(t) * tile_) : edges_[t + 1] - edges_[t];
}

int64_t Dag::unit() const {
    if (edges_.empty()) return tile_;
    int64_t u = int64_t(1) << 30;
    for (int64_t e : edges_)
        if (e > 0) u = std::min<int64_t>(u, e & -e);  // lowest set bit
    return u;
}

int Dag::set_edges(const std::vector<int64_t> &edges) {
    if (!tasks_.empty()) return MTD_ERR_STATE;
    if (edges.size() < 2 || edges.front() != 0 || edges.back() != n_) return MTD_ERR_INVALID_ARG;
    for (size_t i = 1; i < edges.size(); ++i)
        if (edges[i] <= edges[i - 1]) return MTD_ERR_INVALID_ARG;
    edges_ = edges;
    tiles_ = static_cast<int>(edges.size()) - 1;
    tile_ = 0;
    for (size_t i = 1; i < edges.size(); ++i) tile_ = std::max(tile_, edges[i] - edges[i - 1]);
    return MTD_OK;
}

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

int64_t Dag::reference_task_count(int kind, int64_t T) {
    // Cholesky: per step with m = T-k-1 trailing tiles, m TRSM + m SYRK + m(m-1)/2 GEMM;
    // LU: m TRSM-L + m TRSM-R + m^2 GEMM; plus one diagonal factorisation per step.
    int64_t total = T;
    for (int64_t m = 0; m < T; ++m) total += kind == MTD_KIND_CHOLESKY ? 2 * m + m * (m - 1) / 2 : 2 * m + m * m;
    return total;
}

int Dag::build_reference_order() {
    const int T = tiles_;
    if (reference_task_count(kind_, T) > kMaxReferenceTasks) return MTD_ERR_INVALID_ARG;
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

int items_of(const DevTask &t) {
    switch (t.op) {
    case MTD_OP_GEMM_NT:
    case MTD_OP_GEMM_NN:
        return static_cast<int>(ceil_div(t.m, kGemmTile) * ceil_div(t.n, kGemmTile));
    case MTD_OP_SYRK_LN: {
        const int64_t b = ceil_div(t.m, kGemmTile);
        return static_cast<int>(b * (b + 1) / 2);
    }
    case MTD_OP_TRSM_RLT:
    case MTD_OP_TRSM_RUN:
        return static_cast<int>(ceil_div(t.m, kTrsmRows));
    case MTD_OP_TRSM_LLNU:
        return static_cast<int>(ceil_div(t.n, kTrsmRows));
    default:  // diagonal factorisations, and a join's one no-op item
        return 1;
    }
}

// Lookahead priority: diagonal factorisations, panel solves, every update of a diagonal
// tile and the updates that feed the next panel go to the critical-path queue; updates of
// the two columns after it to queue 1, the rest to queue 2 (each queue is FIFO, so the
// near-panel updates no longer wait behind the bulk of later columns).  The
// updates of one diagonal tile form a chain (each writes the tile the next one reads) that
// ends in its factorisation; with only the last link prioritised, the earlier links waited
// in the bulk queue behind the GEMM items (a critical-path walk of the traced TF32 factor
// at N = 32768 found 50 of its 67 ms spent that way).
int Dag::queue_of(int ti) const {
    const HostTask &t = tasks_[ti];
    switch (t.op) {
    case MTD_OP_POTRF:
    case MTD_OP_GETRF:
    case MTD_OP_TRSM_RLT:
    case MTD_OP_TRSM_RUN:
    case MTD_OP_TRSM_LLNU:
    case MTD_OP_SYRK_LN:
        return 0;
    default: {
        // how many steps before the written tile's column becomes the panel
        const int ahead = std::min(t.write.first, t.write.second) - t.a.second;
        return ahead <= 1 ? 0 : (ahead <= 3 ? 1 : 2);
    }
    }
}

namespace {

DevTask make_task(int op, int queue, int64_t cr, int64_t cc, int64_t ar, int64_t ac, int64_t br, int64_t bc,
                  int64_t m, int64_t n, int64_t k) {
    DevTask d{};
    d.op = op;
    d.queue = queue;
    d.cr = static_cast<int32_t>(cr);
    d.cc = static_cast<int32_t>(cc);
    d.ar = static_cast<int32_t>(ar);
    d.ac = static_cast<int32_t>(ac);
    d.br = static_cast<int32_t>(br);
    d.bc = static_cast<int32_t>(bc);
    d.m = static_cast<int32_t>(m);
    d.n = static_cast<int32_t>(n);
    d.k = static_cast<int32_t>(k);
    d.n_items = items_of(d);
    return d;
}

// The reference's tiled task list (cholesky_mustard.cu:224-395 / lu_mustard.cu:345-533)
// over an s x s grid of sub-tiles of edge `b` starting at element (o, o) of an e x e
// diagonal block; appends device tasks and their in-nest predecessor lists.
void nested_factorisation(bool chol, int64_t o, int64_t e, int64_t b, std::vector<DevTask> &tasks,
                          std::vector<std::vector<int>> &preds) {
    const int s = static_cast<int>(ceil_div(e, b));
    auto ext = [&](int p) { return std::min<int64_t>(b, e - int64_t(p) * b); };
    auto org = [&](int p) { return o + int64_t(p) * b; };
    std::map<TileId, int> last;
    auto add = [&](const DevTask &d, TileId w, std::initializer_list<TileId> reads) {
        std::vector<int> dep;
        std::vector<TileId> tl(reads);
        tl.push_back(w);
        for (const auto &id : tl) {
            auto it = last.find(id);
            if (it != last.end()) dep.push_back(it->second);
        }
        std::sort(dep.begin(), dep.end());
        dep.erase(std::unique(dep.begin(), dep.end()), dep.end());
        last[w] = static_cast<int>(tasks.size());
        tasks.push_back(d);
        preds.push_back(dep);
    };
    for (int p = 0; p < s; ++p) {
        const int64_t P = org(p), ep = ext(p);
        if (chol) {
            add(make_task(MTD_OP_POTRF, 0, P, P, P, P, 0, 0, ep, ep, ep), {p, p}, {{p, p}});
            for (int q = p + 1; q < s; ++q)
                add(make_task(MTD_OP_TRSM_RLT, 0, org(q), P, P, P, 0, 0, ext(q), ep, 0), {q, p}, {{p, p}, {q, p}});
            for (int q = p + 1; q < s; ++q) {
                add(make_task(MTD_OP_SYRK_LN, 0, org(q), org(q), org(q), P, 0, 0, ext(q), ext(q), ep), {q, q},
                    {{q, q}, {q, p}});
                for (int r = q + 1; r < s; ++r)
                    add(make_task(MTD_OP_GEMM_NT, 0, org(r), org(q), org(r), P, org(q), P, ext(r), ext(q), ep),
                        {r, q}, {{r, q}, {r, p}, {q, p}});
            }
        } else {
            add(make_task(MTD_OP_GETRF, 0, P, P, P, P, 0, 0, ep, ep, ep), {p, p}, {{p, p}});
            for (int q = p + 1; q < s; ++q)
                add(make_task(MTD_OP_TRSM_LLNU, 0, P, org(q), P, P, 0, 0, ep, ext(q), 0), {p, q}, {{p, p}, {p, q}});
            for (int q = p + 1; q < s; ++q) {
                add(make_task(MTD_OP_TRSM_RUN, 0, org(q), P, P, P, 0, 0, ext(q), ep, 0), {q, p}, {{p, p}, {q, p}});
                for (int r = p + 1; r < s; ++r)
                    add(make_task(MTD_OP_GEMM_NN, 0, org(q), org(r), org(q), P, P, org(r), ext(q), ext(r), ep),
                        {q, r}, {{q, p}, {p, r}, {q, r}});
            }
        }
    }
}

}  // namespace

int Dag::lower(int nest, Lowered &out) const {
    const int nt = num_tasks();
    out = Lowered{};

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

    std::vector<DevTask> &dev = out.tasks;
    std::vector<std::vector<int>> &preds = out.preds;
    std::vector<std::vector<int>> entry(nt);
    std::vector<int> exit_of(nt, -1);
    out.host_items.assign(nt, 0);
    for (int t = 0; t < nt; ++t) {
        const HostTask &h = tasks_[t];
        const int q = queue_of(t);
        const int64_t wr = origin(h.write.first), wc = origin(h.write.second);
        const int64_t em = extent(h.write.first), en = extent(h.write.second);
        const int64_t ar = origin(h.a.first), ac = origin(h.a.second), br = origin(h.b.first), bc = origin(h.b.second);
        const int first = static_cast<int>(dev.size());
        const bool diag = h.op == MTD_OP_POTRF || h.op == MTD_OP_GETRF;
        if (diag && nest > 0 && em > nest) {
            nested_factorisation(h.op == MTD_OP_POTRF, wr, em, nest, dev, preds);
            const int last = static_cast<int>(dev.size());
            std::vector<char> has_succ(last - first, 0);
            for (int d = first; d < last; ++d) {
                for (int p : preds[d]) has_succ[p - first] = 1;  // in-nest edges only so far
                if (preds[d].empty()) entry[t].push_back(d);
            }
            std::vector<int> sinks;
            for (int d = first; d < last; ++d)
                if (!has_succ[d - first]) sinks.push_back(d);
            if (sinks.size() == 1) {
                exit_of[t] = sinks[0];
            } else {
                exit_of[t] = static_cast<int>(dev.size());
                dev.push_back(make_task(kOpJoin, 0, wr, wc, 0, 0, 0, 0, em, en, 0));
                preds.push_back(sinks);
            }
        } else {
            DevTask d{};
            switch (h.op) {
            case MTD_OP_POTRF:
            case MTD_OP_GETRF:
                d = make_task(h.op, q, wr, wc, wr, wc, 0, 0, em, em, em);
                break;
            case MTD_OP_TRSM_RLT:
            case MTD_OP_TRSM_RUN:  // X = write tile (m x n), triangle = n x n at a
            case MTD_OP_TRSM_LLNU: // X = write tile (m x n), triangle = m x m at a
                d = make_task(h.op, q, wr, wc, ar, ac, 0, 0, em, en, 0);
                break;
            case MTD_OP_SYRK_LN:
                d = make_task(h.op, q, wr, wc, ar, ac, 0, 0, em, em, extent(h.a.second));
                break;
            default:  // GEMM_NT / GEMM_NN
                d = make_task(h.op, q, wr, wc, ar, ac, br, bc, em, en, extent(h.a.second));
                break;
            }
            dev.push_back(d);
            preds.emplace_back();
            entry[t].push_back(first);
            exit_of[t] = first;
        }
        for (int d = first; d < static_cast<int>(dev.size()); ++d) out.host_items[t] += dev[d].n_items;
    }
    // Host edges d -> t become exit(d) -> every entry of t.
    for (int t = 0; t < nt; ++t)
        for (int e : entry[t])
            for (int d : deps_[t]) preds[e].push_back(exit_of[d]);

    const int nd = static_cast<int>(dev.size());
    std::vector<std::vector<int>> succs(nd);
    for (int d = 0; d < nd; ++d) {
        std::sort(preds[d].begin(), preds[d].end());
        preds[d].erase(std::unique(preds[d].begin(), preds[d].end()), preds[d].end());
        for (int p : preds[d]) succs[p].push_back(d);
    }
    for (int d = 0; d < nd; ++d) {
        dev[d].succ_begin = static_cast<int32_t>(out.succ.size());
        dev[d].succ_count = static_cast<int32_t>(succs[d].size());
        for (int s : succs[d]) out.succ.push_back(s);
        out.queue_cap[dev[d].queue] += dev[d].n_items;
    }
    return MTD_OK;
}

}  // namespace mtd
