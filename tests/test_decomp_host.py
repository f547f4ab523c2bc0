"""The domain-decomposition driver (pyclaw_b200.decomp) with its
torch.distributed transport, run as 2 and 3 gloo ranks on CPU with the
oracle stepping each slab: the decomposed run equals the single-grid run bit
for bit (halo rows, custom internal sides, corner cells, the CFL max and the
shared step-size control)."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

import decomp_helpers as D
from pyclaw_b200 import decomp


def test_slab_rows_partition():
    for my in (7, 40, 320):
        for n in (1, 2, 3, 8):
            if my < 2 * n:
                continue
            spans = [decomp.slab_rows(my, n, r) for r in range(n)]
            assert spans[0][0] == 0 and spans[-1][1] == my
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            assert max(b - a for a, b in spans) - min(b - a for a, b in spans) <= 1


@pytest.mark.parametrize("case,world", [("euler_case", 2), ("vc_case", 2), ("vc_case", 3)])
def test_gloo_ranks_equal_single_domain(tmp_path, case, world):
    out = str(tmp_path / "result.npz")
    mp.spawn(D.gloo_worker, args=(world, D.free_port(), getattr(D, case), out), nprocs=world, join=True)
    r = np.load(out)
    p, q, aux, run = getattr(D, case)()
    ref, ctrl = D.single_domain(p, q, aux, run)
    assert np.array_equal(r["q"], ref), np.max(np.abs(r["q"] - ref))
    assert all(n == ctrl.numsteps for n in r["numsteps"])
    assert all(t == ctrl.t for t in r["t"])
