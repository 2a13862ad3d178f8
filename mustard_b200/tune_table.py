"""Persistent table of the batched autotuner's choices (JSON).

``mtd_batch_autotune`` times trial factorisations for every distinct matrix size of a batch
(seconds of GPU time for a large batch).  The choice for a size depends only on the size, the
precision and the device, so it is kept in a JSON file and reused: a later batch tunes only
the sizes the table does not hold yet.

Layout::

    {"version": 1,
     "devices": {"<device name>": {"fp64": {"512": {"tile": 384, "nest": 128}, ...},
                                   "fp32": {...}}}}

Writes go to a temporary file that replaces the table, so a reader never sees half a file.
"""
import json
import os
import tempfile

VERSION = 1
PREC_KEYS = {0: "fp64", 1: "tf32", 2: "fp32", 3: "bf16"}  # mtd_precision values


def empty():
    return {"version": VERSION, "devices": {}}


def load(path):
    """The table at ``path``, or an empty one if the file does not exist."""
    if not os.path.exists(path):
        return empty()
    with open(path) as f:
        t = json.load(f)
    if t.get("version") != VERSION or not isinstance(t.get("devices"), dict):
        raise ValueError(f"{path}: not a version-{VERSION} tuning table")
    return t


def save(table, path):
    d = os.path.dirname(os.path.abspath(path))
    fd, tmp = tempfile.mkstemp(prefix=".tune-", suffix=".json", dir=d)
    try:
        with os.fdopen(fd, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except BaseException:
        if os.path.exists(tmp):
            os.unlink(tmp)
        raise


def lookup(table, device, prec, n):
    """(tile, nest) recorded for size ``n``, or None."""
    e = table["devices"].get(device, {}).get(PREC_KEYS[prec], {}).get(str(int(n)))
    return None if e is None else (int(e["tile"]), int(e["nest"]))


def record(table, device, prec, n, tile, nest):
    table["devices"].setdefault(device, {}).setdefault(PREC_KEYS[prec], {})[str(int(n))] = {
        "tile": int(tile), "nest": int(nest)}


def missing(table, device, prec, sizes):
    """Indices of the matrices whose size the table does not hold."""
    return [i for i, n in enumerate(sizes) if lookup(table, device, prec, n) is None]
