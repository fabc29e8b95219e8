"""The benchmark configurations at their full sizes, against the oracle.

  furnished room  512x384x192, 4 materials x 3 sections, sponge 16, 4
                  receivers: the classified grid bit for bit (flags,
                  normals, boundary list, materials, sponge weights) and 200
                  steps of receiver samples bit for bit, 1e-5 of FP64
  batched         the 64 source positions in the 256^3 room and the 16
                  rooms of 96^3-320^3: every member of the batch equal to
                  its own run, bit for bit, over 40 steps (a 32-step graph
                  and single steps), FP32 and BF16 storage
  inverse design  128x128x96, 6 materials x 2 sections, 4 receivers, 4000
                  steps, checkpoints every 64: the loss is the MSE to the
                  IRs of the hidden coefficients; the GPU gradients against
                  the FP64 adjoint (1e-4 of the largest of each kind), and
                  four coefficient gradients against Richardson-extrapolated
                  central differences (h = 1e-3 and 5e-4) of the FP64 model
"""
import dataclasses

import numpy as np
import pytest

import oracle
from helpers import grid_parity, oracle_grid, oracle_scene, rel_l2
from virs_b200 import capi, scenes

pytestmark = pytest.mark.gpu


def test_furnished_room_full_size_bit_exact():
    sc = scenes.furnished_room(steps=200)
    g = oracle_grid(sc)
    assert tuple(g["shape"]) == (512, 384, 192)
    sim, _ = scenes.build_simulation(sc)
    grid_parity(sim, g)
    osc = oracle_scene(sc, g)
    want = osc.run(sc.steps)
    sim.run(sc.steps)
    got = sim.ir()
    sim.close()
    assert got.shape == (4, sc.steps) and np.abs(want).max() > 0
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert rel_l2(got, osc.run(sc.steps, f64=True)) <= 1e-5


@pytest.mark.parametrize("storage", [capi.STORAGE_F32, capi.STORAGE_BF16])
def test_batched_full_membership_bit_exact(storage):
    steps = 40
    scs = scenes.batched(steps=steps)
    assert len(scs) == 80
    alone = []
    for sc in scs:
        sim, _ = scenes.build_simulation(sc, storage=storage)
        sim.run(steps)
        alone.append(sim.ir())
        sim.close()
    sims = [scenes.build_simulation(sc, storage=storage)[0] for sc in scs]
    try:
        with capi.Batch(sims) as b:
            b.run(steps)
            b.synchronize()
            for k, (sim, want) in enumerate(zip(sims, alone)):
                assert np.array_equal(sim.ir().view(np.uint32), want.view(np.uint32)), scs[k].name
    finally:
        for s in sims:
            s.close()


def _loss64(osc, coef64, target):
    osc.coef64 = np.ascontiguousarray(coef64, np.float64).reshape(-1)
    ir = osc.run64(target.shape[1])
    return float(np.mean((ir - target) ** 2)), ir


def test_inverse_design_full_size_gradients():
    sc, guess = scenes.inverse_design()
    assert sc.steps == 4000 and sc.n_materials * sc.n_sections == 12
    every = 64
    g = oracle_grid(sc)
    assert tuple(g["shape"]) == (128, 128, 96)
    osc = oracle_scene(sc, g)
    target = osc.run64(sc.steps)                       # the hidden coefficients
    at = dataclasses.replace(sc, coef64=guess)
    osc = oracle_scene(at, g)
    loss, ir64 = _loss64(osc, guess, target)
    dl = 2 * (ir64 - target) / ir64.size
    gc64, gs64 = osc.adjoint64(sc.steps, dl, every=every)

    sim, _ = scenes.build_simulation(at)
    sim.forward_checkpointed(sc.steps, every)
    ir = sim.ir(0, sc.steps)
    assert rel_l2(ir, ir64) <= 1e-5
    gc, gs = sim.adjoint(dl.astype(np.float32), sc.n_materials, sc.n_sections)
    sim.close()
    err_c = np.abs(gc - gc64).max() / np.abs(gc64).max()
    err_s = np.abs(gs - gs64).max() / np.abs(gs64).max()
    print(f"loss {loss:.3e}: coef grad err {err_c:.2e}, signal grad err {err_s:.2e} vs the FP64 adjoint")
    assert err_c <= 1e-4 and err_s <= 1e-4

    # central differences of the FP64 model at four coefficients: the largest
    # gradients of b0, b1, a1 and a2 over all materials and sections
    flat = gc64.reshape(-1, 5)
    for j in (0, 1, 3, 4):
        k = int(np.argmax(np.abs(flat[:, j])))
        fd = []
        for h in (1e-3, 5e-4):
            c = guess.reshape(-1, 5).copy()
            c[k, j] += h
            lp, _ = _loss64(osc, c.reshape(guess.shape), target)
            c[k, j] -= 2 * h
            lm, _ = _loss64(osc, c.reshape(guess.shape), target)
            fd.append((lp - lm) / (2 * h))
        rich = (4 * fd[1] - fd[0]) / 3
        got = gc.reshape(-1, 5)[k, j]
        print(f"coef [{k}][{j}]: GPU {got:.6e}  FD {rich:.6e}  FP64 adjoint {flat[k, j]:.6e}")
        assert abs(got - rich) <= 1e-4 * abs(rich), (k, j, got, rich)
