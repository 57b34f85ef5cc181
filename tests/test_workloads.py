"""The synthetic workloads reach the window lengths the GPU parity tests rely on
(CPU only: RT limits from the oracle, src/rt_index/mod.rs:89-138)."""
import numpy as np
import pytest

import oracle
from alphadia_search_rs_b200 import synth

from _util import oracle_inputs



@pytest.mark.parametrize("name,longest", [("tiny_long", (2049, 2300)), ("long_rt", (4000, 4002))])
def test_long_workloads_span_past_shared_memory_plan(name, longest):
    """The long-window workloads reach the length classes they are meant to test:
    windows of cfg2/3's and cfg4's longest classes (801, 1201 cycles), up to and past
    the 2048 cycles a warp's shared-memory plan holds (those run with the working sets
    in global memory)."""
    cfg, lib, run = synth.make_workload(name, "numpy")
    la = synth.library_arrays(lib)
    od, ol, tol = oracle_inputs(run, la)
    rt, dt = od.rt, od.delta_t
    tols = la.get("precursor_rt_tolerance", np.full(len(la["precursor_rt"]), cfg.rt_half_window[1], np.float32))
    spans = []
    for prt, t in zip(la["precursor_rt"], tols):
        a, b = oracle.rt_limits(rt, dt, float(prt), float(t), float(cfg.kernel_size))
        spans.append(b - a)
    spans = np.asarray(spans)
    assert longest[0] <= spans.max() <= longest[1]
    assert (spans > 2048).mean() >= (0.9 if name == "long_rt" else 0.01)
    if name == "tiny_long":
        for bound in (801, 1201, 2048):
            assert (spans > bound).any() and (spans <= bound).any(), bound
