"""Partitioned LU over several GPUs: the host-side plan of the reference's p_lu_mustard
(mustard/lu_mustard_p.cu), and its B200 form on one NVSwitch node.

The reference (no pivoting, like its single-GPU LU):

- **ownership**: 1-D block-cyclic slices of tile rows.  Slice k (every tile (k, j)) lives on
  PE ``k mod P``, each PE holding ``ceil(T / P)`` slices of the full width
  (lu_mustard_p.cu:54-72);
- **step k**: the slice's owner factors the diagonal tile (GETRF) and solves the slice's
  tiles right of it, U(k, j) = L_kk^-1 A(k, j) (TRSM left, lower, unit) (:247-275,
  :300-318); the slice then travels down a **chain** of PEs: each waits for its
  predecessor's flag, forwards the flag to its neighbour while PEs further on still own
  rows below the diagonal, and fetches the slice's tiles from the owner into a receive
  buffer (:276-298, :319-348);
- every PE then solves its own tiles below the diagonal, L(i, k) = A(i, k) U_kk^-1 (TRSM
  right, upper), and updates its tiles right of them, A(i, j) -= L(i, k) U(k, j) (GEMM)
  (:350-460).  Everything is one host-launched CUDA graph per PE, no device scheduler.

The B200 form keeps the ownership and the per-step task split.  The chain becomes one
broadcast per step from the owner: NVSwitch gives every GPU full bandwidth to every peer,
so the chain's P - 1 sequential hops only add latency.  Receivers are the PEs that still
own rows below the diagonal, as in the chain.  Each GPU's share of a step is a small task
graph (its TRSM_RUN and GEMM_NN tiles) for the persistent scheduler.

``build_plan`` lists, per step, the owner's tasks, the broadcast (source, receivers in the
reference's chain order, tiles) and every rank's update tasks.  The tests execute a plan on
gloo CPU ranks with the oracle's tile arithmetic and check the distributed factor against
the single-process tiled LU, bit for bit.  The per-GPU launches are not built: every run of
this build has one GPU.
"""
from dataclasses import dataclass, field

GETRF, TRSM_LLNU, TRSM_RUN, GEMM_NN = "GETRF", "TRSM_LLNU", "TRSM_RUN", "GEMM_NN"


def owner(i, world):
    """Rank holding tile row (slice) i: i mod world (lu_mustard_p.cu:54-72)."""
    return i % world


def slices_of(rank, tiles, world):
    """Tile rows a rank holds, in order."""
    return list(range(rank, tiles, world))


def chain(k, tiles, world):
    """Receivers of slice k in the reference's chain order: the owner's neighbours o + 1,
    o + 2, ... (mod world), as long as the PE at that distance still owns a row below the
    diagonal (distance < tiles - k; lu_mustard_p.cu:276-298)."""
    o = owner(k, world)
    return [(o + d) % world for d in range(1, world) if d < tiles - k]


@dataclass
class Step:
    k: int
    owner: int
    owner_tasks: list                 # (op, write tile, read tiles) on the owner, in order
    source: int                       # rank broadcasting slice k
    receivers: list                   # ranks receiving it, in chain order
    tiles: list                       # the broadcast tiles: (k, k .. T-1)
    rank_tasks: dict = field(default_factory=dict)  # rank -> its update tasks of the step


@dataclass
class Plan:
    world: int
    tiles: int
    steps: list

    def tasks(self):
        """Every task once, in a topological order (step by step)."""
        out = []
        for s in self.steps:
            out += s.owner_tasks
            for r in range(self.world):
                out += s.rank_tasks.get(r, [])
        return out

    def broadcast_tiles(self):
        """Tiles sent in total (each to every receiver of its step)."""
        return sum(len(s.tiles) * len(s.receivers) for s in self.steps)


def build_plan(tiles, world):
    """The partitioned LU of a ``tiles`` x ``tiles`` tile grid on ``world`` GPUs."""
    if world < 1 or tiles < 1:
        raise ValueError("world and tiles must be >= 1")
    steps = []
    for k in range(tiles):
        o = owner(k, world)
        own = [(GETRF, (k, k), [(k, k)])]
        own += [(TRSM_LLNU, (k, j), [(k, k), (k, j)]) for j in range(k + 1, tiles)]
        step = Step(k, o, own, o, chain(k, tiles, world), [(k, j) for j in range(k, tiles)])
        for i in range(k + 1, tiles):
            r = owner(i, world)
            tasks = step.rank_tasks.setdefault(r, [])
            tasks.append((TRSM_RUN, (i, k), [(k, k), (i, k)]))
            tasks += [(GEMM_NN, (i, j), [(i, k), (k, j), (i, j)]) for j in range(k + 1, tiles)]
        steps.append(step)
    return Plan(world, tiles, steps)


def slice_bytes(n, tile, k, elem=8):
    """Bytes of slice k's broadcast part (tile row k, columns k*tile .. n)."""
    rows = min(tile, n - k * tile)
    return rows * (n - k * tile) * elem
