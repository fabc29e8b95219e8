"""Golden vectors produced by the reference's own CUDA kernels
(tests/golden/make_golden.py): the oracle must reproduce them bit for bit
on the CPU, and the CUDA path through the C ABI on the GPU."""
from pathlib import Path

import numpy as np
import pytest

import oracle

GOLD = Path(__file__).resolve().parent / "golden"
CASES = sorted(p.stem for p in GOLD.glob("ref_*.npz"))
# the same reference step with its rigid-wall kernel launched (consts[4]:
# that kernel's l2 as it evaluates it on the device)
RIGID = "rigid_room"


def _load(name):
    d = np.load(GOLD / f"{name}.npz")
    return {k: d[k] for k in d.files}


def _oracle_run(d, rigid=False):
    shape = tuple(int(s) for s in d["shape"])
    c = d["consts"]
    extra = dict(normals=oracle.normals(shape, d["flags_ref"]), rigid=True, l2=float(c[4])) if rigid else {}
    sc = oracle.Scene(shape, d["flags_ref"], d["bidx"], np.zeros(d["bidx"].size, np.uint8),
                      np.ones(d["bidx"].size, np.float32), d["coef"], 1, hard=np.full(10, 10.0, np.float32),
                      rcv_idx=d["rcv"], consts=(c[1], c[2], c[3]), **extra)
    n = int(np.prod(shape))
    st = (np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(d["bidx"].size * 4 + 1, np.float32))
    ir = sc.run(d["ir"].shape[1], state=st)
    return ir, st[0]


def test_golden_present():
    assert len(CASES) >= 2, "golden vectors missing: run tests/golden/make_golden.py on a GPU"


@pytest.mark.parametrize("name", CASES)
def test_oracle_classification_matches_reference_gpu(name):
    d = _load(name)
    shape = tuple(int(s) for s in d["shape"])
    flags, _, _ = oracle.classify(shape, 1, d["flags_raw"])
    assert np.array_equal(flags, d["flags_ref"])
    assert np.array_equal(oracle.boundary_list(shape, flags), d["bidx"])


@pytest.mark.parametrize("name", CASES)
def test_oracle_step_matches_reference_gpu(name):
    d = _load(name)
    ir, p = _oracle_run(d)
    assert np.abs(d["ir"]).max() > 0
    assert np.array_equal(ir.view(np.uint32), d["ir"].view(np.uint32))
    assert np.array_equal(p.view(np.uint32), d["p_final"].view(np.uint32))


def test_oracle_rigid_walls_match_reference_gpu():
    d = _load(RIGID)
    ir, p = _oracle_run(d, rigid=True)
    assert np.abs(d["ir"]).max() > 0
    assert np.array_equal(ir.view(np.uint32), d["ir"].view(np.uint32))
    assert np.array_equal(p.view(np.uint32), d["p_final"].view(np.uint32))
    plain, _ = _oracle_run(d)                  # the rigid update does change the result
    assert not np.array_equal(plain, d["ir"])


@pytest.mark.gpu
@pytest.mark.parametrize("steps_per_pass", [1, 2])
@pytest.mark.parametrize("name", CASES + [RIGID])
def test_cuda_path_matches_reference_gpu(name, steps_per_pass):
    """The reference's own kernels' outputs, one or two steps per pass."""
    from virs_b200 import capi
    d = _load(name)
    shape = tuple(int(s) for s in d["shape"])
    p = capi.default_params(boundary_k=float(d["consts"][3]), rigid_walls=int(name == RIGID))
    sim = capi.Simulation(p)
    sim.set_grid(shape, float(d["h"]), d["flags_raw"])
    sim.classify()
    assert np.array_equal(sim.flags(), d["flags_ref"])
    assert np.array_equal(sim.boundary_indices(), d["bidx"])
    sim.set_filters(d["coef"][None, None, :])
    sim.set_receivers(d["rcv"])
    steps = d["ir"].shape[1]
    sim.start(steps)
    sim.set_time_blocking(steps_per_pass)
    assert sim.time_blocking()["active"] == (steps_per_pass == 2)
    sim.run(steps)
    got = sim.ir()
    assert np.array_equal(got.view(np.uint32), d["ir"].view(np.uint32))
    assert np.array_equal(sim.pressure().view(np.uint32), d["p_final"].view(np.uint32))
    sim.close()
