"""Autotuned launch shapes, persisted in a JSON cache.

The native tuners (bq_autotune_query_f3 for one tree, bq_autotune_batched_knn_f3
for a batch of clouds) time every combination of leaf threshold, stack depth,
block size and queries per warp on the caller's inputs.  Their choice depends
on the workload's size and the GPU, not on the exact points, so it is cached
under the key (workload kind and k, size bucket, GPU name): the bucket is
the rounded base-2 logarithm of the prim and query counts.

The cache is a JSON file: $CUBQL_B200_TUNING_CACHE, or
~/.cache/cubql_b200/tuning.json.  A missing or unreadable file is an empty
cache; entries are written back after every new tuning run.
"""
import ctypes
import json
import math
import os

import torch


def cache_path():
    return os.environ.get("CUBQL_B200_TUNING_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "cubql_b200", "tuning.json"))


def _load(path):
    try:
        with open(path) as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def _store(path, data):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _bucket(x):
    return int(round(math.log2(max(int(x), 1))))


def cache_key(kind, k, num_prims, num_queries, gpu=None):
    """'kind|k|n2^a|q2^b|gpu name' for a workload."""
    if gpu is None:
        gpu = torch.cuda.get_device_name()
    return f"{kind}|k{k}|n2^{_bucket(num_prims)}|q2^{_bucket(num_queries)}|{gpu}"


def _tuning_dict(best):
    import cubql_b200 as bq
    return {f: getattr(best, f) for f, _ in bq.bq_tuning._fields_}


def _cached(kind, k, n, nq, run, path=None, retune=False):
    path = path or cache_path()
    key = cache_key(kind, k, n, nq)
    data = _load(path)
    if not retune and key in data:
        return dict(data[key], cached=True, key=key)
    t = run()
    data[key] = t
    _store(path, data)
    return dict(t, cached=False, key=key)


def tuned_query(boxes, points, queries, k=0, path=None, retune=False):
    """Launch shape for one tree over `boxes`/`points` queried with `queries`:
    closest point (k == 0) or kNN.  Returns a dict with makeLeafThreshold,
    stackDepth, blockSize, queriesPerWarp, buildMs, queryMs (of the tuning
    run), plus 'cached' and 'key'."""
    import cubql_b200 as bq
    boxes = bq._as_boxes(boxes)
    points, queries = bq._vec3(points, "points"), bq._vec3(queries, "queries")

    def run():
        best = bq.bq_tuning()
        bq._check(bq._lib.bq_autotune_query_f3(bq._ptr(boxes), bq._ptr(points), boxes.shape[0], bq._ptr(queries),
                                               queries.shape[0], k, ctypes.byref(best), None, bq._stream()))
        return _tuning_dict(best)
    return _cached("query", k, boxes.shape[0], queries.shape[0], run, path, retune)


def tuned_batched_knn(boxes, points, offsets, queries, queryOffsets, k, path=None, retune=False):
    """Launch shape for a batched build + kNN (bq_autotune_batched_knn_f3),
    cached per (k, size bucket, number-of-clouds bucket, GPU)."""
    import cubql_b200 as bq
    boxes = bq._as_boxes(boxes)
    nseg = offsets.numel() - 1

    def run():
        return {f: v for f, v in bq.autotune_batched_knn(boxes, points, offsets, queries, queryOffsets, k).items()}
    return _cached(f"batched{_bucket(nseg)}", k, boxes.shape[0], queries.shape[0], run, path, retune)


def query_config_of(t, tieMode=0):
    """The bq_query_config of a tuning dict."""
    import cubql_b200 as bq
    return bq.query_config(tieMode=tieMode, stackDepth=t["stackDepth"], blockSize=t["blockSize"],
                           queriesPerWarp=t["queriesPerWarp"])
