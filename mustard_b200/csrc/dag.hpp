// Host-side task DAG: the data the reference keeps in TiledGraphCreator
// (mustard/mustard.h:132-384) -- task list, last-writer map, predecessor lists -- and its
// lowering to the device task table (element geometry, work items, priorities,
// successor lists).
#pragma once

#include <cstdint>
#include <map>
#include <utility>
#include <vector>

#include "device_types.hpp"

namespace mtd {

using TileId = std::pair<int, int>;  // (row tile, column tile), the reference's MatrixTile

struct HostTask {
    int op = 0;
    TileId write{0, 0};
    std::vector<TileId> reads;  // as given by the caller (reference order)
    TileId a{0, 0};             // first operand (triangular tile for TRSM)
    TileId b{0, 0};             // second operand (GEMM only)
};

// The device form of a graph.
struct Lowered {
    std::vector<DevTask> tasks;
    std::vector<int> succ;                 // CSR payload, indexed by DevTask::succ_begin
    std::vector<std::vector<int>> preds;   // per device task
    std::vector<int> host_items;           // work items of each host task (all its device tasks)
    int64_t queue_cap[kNumQueues] = {0, 0};
};

class Dag {
public:
    Dag(int kind, int64_t n, int64_t tile);

    int kind() const { return kind_; }
    int64_t n() const { return n_; }
    int64_t tile() const { return tile_; }
    int tiles() const { return tiles_; }
    int64_t origin(int t) const;  // first row (or column) of tile row t
    int64_t extent(int t) const;  // rows (or columns) of tile row t
    // The largest power of two dividing every tile edge (and n): the alignment every tile
    // origin and extent has.  With uniform tiles, the tile edge itself.
    int64_t unit() const;
    // Tile rows at the given element edges (edges[0] = 0 < edges[1] < ... < edges[T] = n)
    // instead of uniform `tile`-wide ones; only before any task is recorded.
    int set_edges(const std::vector<int64_t> &edges);

    // Returns the new task index, or a negative mtd_status.
    int add_task(int op, int wi, int wj, const int *reads, int nreads);
    // The reference's whole task list for this kind; MTD_ERR_INVALID_ARG when it would
    // exceed kMaxReferenceTasks (checked in closed form before anything is built).
    int build_reference_order();
    // Tasks of the reference's list for `kind` over T x T tiles (cholesky_mustard.cu:200-204,
    // lu_mustard.cu:322-326), in 64 bits.
    static int64_t reference_task_count(int kind, int64_t T);
    static constexpr int64_t kMaxReferenceTasks = int64_t(1) << 25;

    int num_tasks() const { return static_cast<int>(tasks_.size()); }
    const std::vector<int> &deps(int t) const { return deps_[t]; }
    const HostTask &task(int t) const { return tasks_[t]; }

    // Device lowering.  A diagonal factorisation of a tile larger than `nest` elements
    // (nest > 0, a multiple of kNB) becomes a nested tiled factorisation with nest-sized
    // sub-tiles -- the reference's own remedy for big diagonal tiles
    // (recordSubgraph, mustard/lu_mustard.cu:133-254, used when B > MAX_TILE) -- so the
    // critical path runs on many SMs.  Returns MTD_OK or MTD_ERR_BAD_DAG.
    int lower(int nest, Lowered &out) const;

private:
    int kind_;
    int64_t n_, tile_;
    int tiles_;
    std::vector<int64_t> edges_;  // empty: uniform tiles
    std::vector<HostTask> tasks_;
    std::vector<std::vector<int>> deps_;
    std::map<TileId, int> last_writer_;                 // tileIndexByMap (mustard.h:177)
    std::map<TileId, std::vector<int>> readers_since_;  // readers since the last write

    bool valid_tile(const TileId &t) const;
    int queue_of(int t) const;
};

int items_of(const DevTask &t);

}  // namespace mtd
