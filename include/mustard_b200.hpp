// mustard_b200.hpp -- header-only C++ host interface over the C ABI (mustard_b200.h).
//
// Mirrors the reference's mustard::TiledGraphCreator (mustard/mustard.h:132-384) so a
// driver written against the reference reads the same: the library call the reference
// captures between beginCaptureOperation and endCaptureOperation becomes one
// recordOperation(op) call.
//
//   reference (cholesky_mustard.cu:232-253)        here
//   creator->beginCaptureOperation({k,k},{{k,k}});  creator.beginCaptureOperation({k,k},{{k,k}});
//   cusolverDnDpotrf(handle, LOWER, B, ...);        creator.recordOperation(MTD_OP_POTRF);
//   creator->endCaptureOperation();                 creator.endCaptureOperation();
//   ... queue + scheduler graph set-up ...          creator.finalize();
//   cudaGraphLaunch(schedulerExec, s);              creator.run(dA, lda, s);
//
// Errors are reported by throwing mustard_b200::Error (status + LAPACK-style info); the
// reference calls exit() through checkCudaErrors (include/utils.h:9-18).
#pragma once

#include <cstdint>
#include <cstdio>
#include <initializer_list>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "mustard_b200.h"

namespace mustard_b200 {

using MatrixTile = std::pair<int, int>;  // (row tile, column tile), as mustard.h:53

class Error : public std::runtime_error {
public:
    Error(int status, int info = 0)
        : std::runtime_error(std::string(mtd_strerror(status)) + (info ? " (info=" + std::to_string(info) + ")" : "")),
          status(status), info(info) {}
    int status;
    int info;
};

inline void check(int rc, int info = 0) {
    if (rc != MTD_OK) throw Error(rc, info);
}

class TiledGraphCreator {
public:
    std::vector<std::vector<int>> subgraphDependencies;  // as mustard.h:137

    TiledGraphCreator(int kind, int64_t n, int64_t tile) { check(mtd_graph_create(&g_, kind, n, tile)); }
    ~TiledGraphCreator() {
        if (g_) mtd_graph_destroy(g_);
    }
    TiledGraphCreator(const TiledGraphCreator &) = delete;
    TiledGraphCreator &operator=(const TiledGraphCreator &) = delete;

    void beginCaptureOperation(MatrixTile tileToWrite, std::initializer_list<MatrixTile> tilesToRead) {
        if (open_) throw Error(MTD_ERR_STATE);
        open_ = true;
        op_ = -1;
        write_ = tileToWrite;
        reads_.assign(tilesToRead.begin(), tilesToRead.end());
    }
    // The operation the task performs (replaces the captured cuBLAS/cuSOLVER call).
    void recordOperation(int op) {
        if (!open_) throw Error(MTD_ERR_STATE);
        op_ = op;
    }
    int endCaptureOperation() {
        if (!open_ || op_ < 0) throw Error(MTD_ERR_STATE);
        open_ = false;
        std::vector<int> flat;
        for (const auto &t : reads_) {
            flat.push_back(t.first);
            flat.push_back(t.second);
        }
        const int idx = mtd_graph_add_task(g_, op_, write_.first, write_.second, flat.data(),
                                           static_cast<int>(reads_.size()));
        if (idx < 0) throw Error(-idx);
        subgraphDependencies.push_back(deps(idx));
        return idx;
    }
    // The reference's whole task list for the graph's kind (LU or Cholesky).
    void buildTiled() {
        check(mtd_graph_build_tiled(g_));
        for (int t = static_cast<int>(subgraphDependencies.size()); t < numTasks(); ++t)
            subgraphDependencies.push_back(deps(t));
    }
    void printDeps() const {  // mustard.h:183-195
        for (size_t i = 0; i < subgraphDependencies.size(); ++i) {
            std::printf("%zu:", i);
            for (int d : subgraphDependencies[i]) std::printf(" %d", d);
            std::printf("\n");
        }
    }
    void setTrace(bool on) { check(mtd_graph_set_trace(g_, on ? 1 : 0)); }
    void setTimeout(double seconds) { check(mtd_graph_set_timeout(g_, seconds)); }
    void finalize() { check(mtd_graph_finalize(g_)); }
    // Stream-ordered run; with sync the status is checked (throws on failure).
    int run(double *dA, int64_t lda, void *stream, bool sync = true) {
        int info = 0;
        const int rc = mtd_run(g_, dA, lda, stream, sync ? &info : nullptr);
        check(rc, info);
        return info;
    }
    int numTasks() const { return mtd_graph_num_tasks(g_); }
    mtd_graph *handle() { return g_; }

private:
    std::vector<int> deps(int t) const {
        const int c = mtd_graph_get_deps(g_, t, nullptr, 0);
        if (c < 0) throw Error(-c);
        std::vector<int> v(static_cast<size_t>(c));
        if (c) mtd_graph_get_deps(g_, t, v.data(), c);
        return v;
    }
    mtd_graph *g_ = nullptr;
    bool open_ = false;
    int op_ = -1;
    MatrixTile write_{0, 0};
    std::vector<MatrixTile> reads_;
};

}  // namespace mustard_b200
