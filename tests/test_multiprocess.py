"""Multi-process selection on CPU with the gloo backend (world size 2).

Each rank searches its contiguous library shard (the CPU oracle stands in for the
per-rank GPU search, which this container cannot run) and the ranks gather their
candidates; the gathered result must equal the single-process search of the whole
library, column for column.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from alphadia_search_rs_b200 import sharding, synth


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, name, result_path):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "tests")]
    import datetime

    import torch.distributed as dist

    from _util import COLS, oracle_search

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfg, lib, run = synth.make_workload(name, "numpy")
        la = synth.library_arrays(lib)
        shard = sharding.shard_library(la, rank, world)
        local = oracle_search(run, shard, cfg.params_dict())
        cols = tuple(local[c] for c in COLS)
        gathered = sharding.gather_candidates(cols)
        if rank == 0:
            np.savez(result_path, **dict(zip(COLS, gathered)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["tiny", "tiny_uneven"])
def test_sharded_search_equals_single_process(tmp_path, name):
    from _util import COLS, oracle_search

    out = str(tmp_path / "gathered.npz")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, name, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = dict(np.load(out))
    cfg, lib, run = synth.make_workload(name, "numpy")
    ref = oracle_search(run, synth.library_arrays(lib), cfg.params_dict())
    assert len(ref["rank"]) > 0
    for c in COLS:
        assert np.array_equal(np.asarray(got[c]).view(np.uint8), np.asarray(ref[c]).view(np.uint8)), c


def test_shard_bounds_cover():
    for n in (0, 1, 7, 100):
        for w in (1, 2, 3, 8):
            spans = [sharding.shard_bounds(n, r, w) for r in range(w)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            assert max(h - l for l, h in spans) - min(h - l for l, h in spans) <= 1


def test_shard_library_keeps_fragments():
    cfg, lib, run = synth.make_workload("tiny_uneven", "numpy")
    la = synth.library_arrays(lib)
    parts = [sharding.shard_library(la, r, 3) for r in range(3)]
    assert sum(len(p["precursor_idx"]) for p in parts) == len(la["precursor_idx"])
    assert sum(len(p["fragment_mz"]) for p in parts) == len(la["fragment_mz"])
    allp = np.concatenate([p["precursor_idx"] for p in parts])
    assert np.array_equal(allp, np.sort(la["precursor_idx"], kind="stable"))
    for p in parts:
        fs, fe = p["flat_frag_start_idx"], p["flat_frag_stop_idx"]
        assert fs[0] == 0 and fe[-1] == len(p["fragment_mz"])
        assert "precursor_rt_tolerance" in p


class _HostIdfLib:
    """Stands in for one rank's SpecLibFlat in the IDF merge: its own histogram of
    fragment_mz_library over the m/z grid (find_closest_index, src/idf/mod.rs:13-33)."""

    def __init__(self, fragment_mz_library):
        import oracle

        grid = oracle.ppm_index()
        self.counts = np.zeros(len(grid), np.uint32)
        for mz in np.asarray(fragment_mz_library, np.float32):
            self.counts[oracle.find_closest_index(grid, float(mz))] += 1
        self.num_fragments = len(fragment_mz_library)
        self.set_to = None

    def idf_counts(self):
        return self.counts.copy()

    def set_idf(self, counts, total):
        self.set_to = (np.asarray(counts, np.uint32).copy(), int(total))


def _idf_worker(rank, world, port, result_path):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "tests")]
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        cfg, lib, run = synth.make_workload("tiny", "numpy")
        shard = sharding.shard_library(synth.library_arrays(lib), rank, world)
        host = _HostIdfLib(shard["fragment_mz_library"])
        sharding.merge_idf(host)
        counts, total = host.set_to
        np.savez(f"{result_path}.{rank}.npz", counts=counts, total=total)
    finally:
        dist.destroy_process_group()


def test_sharded_idf_merge_equals_whole_library(tmp_path):
    """Sharded scoring's exchange step: after the all-reduce every rank holds the IDF
    histogram and fragment total of the whole library."""
    world, port = 2, _free_port()
    path = str(tmp_path / "idf")
    mp.start_processes(_idf_worker, args=(world, port, path), nprocs=world, join=True,
                       start_method="spawn")
    cfg, lib, run = synth.make_workload("tiny", "numpy")
    whole = _HostIdfLib(synth.library_arrays(lib)["fragment_mz_library"])
    for r in range(world):
        got = np.load(f"{path}.{r}.npz")
        assert int(got["total"]) == whole.num_fragments
        assert np.array_equal(got["counts"], whole.counts)
