"""Data-parallel selection over several GPUs (one process per GPU).

Precursors are independent, so a library is split into contiguous ranges of its
precursor_idx-sorted order; every rank searches its range against its own copy of
the DIA run, with no exchange on the data path.  The only collective is the final
gather of the variable-length candidate columns (counts first, then the padded
columns), after which concatenating the ranks' results in rank order reproduces
the single-GPU candidate order (precursor_idx order, then rank).
"""
from __future__ import annotations

import numpy as np

PRECURSOR_KEYS = ("precursor_idx", "precursor_mz_library", "precursor_mz", "precursor_rt_library",
                  "precursor_rt", "precursor_naa", "precursor_rt_tolerance")
FRAGMENT_KEYS = ("fragment_mz_library", "fragment_mz", "fragment_intensity", "fragment_cardinality",
                 "fragment_charge", "fragment_loss_type", "fragment_number", "fragment_position",
                 "fragment_type")
CANDIDATE_COLS = ("precursor_idx", "rank", "score", "scan_center", "scan_start", "scan_stop",
                  "cycle_center", "cycle_start", "cycle_stop")


def shard_bounds(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [lo, hi) of n items for ``rank`` of ``world`` (sizes differ by <= 1)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard_library(arrays: dict, rank: int, world: int) -> dict:
    """SpecLibFlat.from_arrays keyword arrays of one shard.

    The precursor arrays are stably sorted by precursor_idx first (what
    SpecLibFlat::from_arrays does, src/speclib_flat/mod.rs:139-163), so the shards
    are contiguous in the order the search emits candidates.  Each shard carries
    only its own fragments, re-based to start at 0."""
    pidx = np.asarray(arrays["precursor_idx"])
    order = np.argsort(pidx, kind="stable")
    lo, hi = shard_bounds(len(pidx), rank, world)
    sel = order[lo:hi]
    fs = np.asarray(arrays["flat_frag_start_idx"], np.int64)[sel]
    fe = np.asarray(arrays["flat_frag_stop_idx"], np.int64)[sel]
    counts = fe - fs
    new_fe = np.cumsum(counts)
    new_fs = new_fe - counts
    fidx = (np.concatenate([np.arange(a, b) for a, b in zip(fs, fe)]) if len(sel)
            else np.zeros(0, np.int64))
    out = {}
    for k in PRECURSOR_KEYS:
        if k in arrays and arrays[k] is not None:
            out[k] = np.ascontiguousarray(np.asarray(arrays[k])[sel])
    out["flat_frag_start_idx"] = new_fs.astype(np.uint64)
    out["flat_frag_stop_idx"] = new_fe.astype(np.uint64)
    for k in FRAGMENT_KEYS:
        out[k] = np.ascontiguousarray(np.asarray(arrays[k])[fidx])
    return out


def gather_candidates(columns: tuple, group=None, device=None) -> tuple:
    """All-gathers the nine candidate columns of every rank and returns them
    concatenated in rank order (on every rank).  ``columns`` is the tuple of
    CandidateCollection.to_arrays()."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    dev = torch.device("cpu") if device is None else torch.device(device)
    n_local = torch.tensor([len(columns[0])], dtype=torch.int64, device=dev)
    counts = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(counts, n_local, group=group)
    counts = [int(c.item()) for c in counts]
    cap = max(max(counts), 1)
    out = []
    for col in columns:
        a = np.asarray(col)
        # u64 travels as int64 bits, f32 as f32
        t_dtype = torch.float32 if a.dtype == np.float32 else torch.int64
        buf = torch.zeros(cap, dtype=t_dtype, device=dev)
        if len(a):
            src = a.view(np.int64) if a.dtype == np.uint64 else a
            buf[: len(a)] = torch.from_numpy(np.ascontiguousarray(src)).to(dev)
        parts = [torch.zeros(cap, dtype=t_dtype, device=dev) for _ in range(world)]
        dist.all_gather(parts, buf, group=group)
        cat = np.concatenate([p[:n].cpu().numpy() for p, n in zip(parts, counts)])
        out.append(cat.view(np.uint64) if a.dtype == np.uint64 else cat)
    return tuple(out)


def merge_idf(lib, group=None) -> None:
    """Sharded scoring: sums the IDF histograms and fragment totals of the ranks' shards
    of one library (the exchange step scoring needs: src/idf/mod.rs counts the fragments
    of the whole library per m/z bin) and sets the sums on ``lib``.  ``lib`` is this
    rank's SpecLibFlat (or anything with idf_counts / set_idf / num_fragments); the
    counts travel as one int32 all-reduce, on the device under NCCL, on the host under
    gloo."""
    import torch
    import torch.distributed as td

    on_device = td.get_backend(group) == "nccl"
    if on_device:
        from . import _ffi

        n = int(_ffi.load().ads_idf_bins())
        counts = torch.empty(n, dtype=torch.int32, device=f"cuda:{lib.device}")
        lib.idf_counts(out=counts)
    else:
        counts = torch.from_numpy(lib.idf_counts().view(np.int32).copy())
    total = torch.tensor([lib.num_fragments], dtype=torch.int64, device=counts.device)
    td.all_reduce(counts, op=td.ReduceOp.SUM, group=group)
    td.all_reduce(total, op=td.ReduceOp.SUM, group=group)
    if on_device:
        lib.set_idf(counts, int(total.item()))
    else:
        lib.set_idf(counts.numpy().view(np.uint32), int(total.item()))
