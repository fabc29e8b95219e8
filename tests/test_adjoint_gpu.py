"""The GPU adjoint (virs_forward_checkpointed + virs_adjoint) against the
FP64 CPU adjoint of the oracle, and the torch.autograd binding.

The FP64 adjoint itself is checked against central finite differences in
tests/test_oracle.py; the GPU pass runs in FP32 (FP64 gradient sums), so the
bound here is 1e-4 relative to the largest gradient of each kind."""
import dataclasses

import numpy as np
import pytest

from helpers import oracle_grid, oracle_scene
from virs_b200 import capi, scenes

pytestmark = pytest.mark.gpu


def _compare(sc, every, form=None):
    g = oracle_grid(sc)
    osc = oracle_scene(sc, g)
    if form is not None:
        osc.form = form
    target = osc.run64(sc.steps) * 0.8
    ir64 = osc.run64(sc.steps)
    dl = 2 * (ir64 - target) / ir64.size
    gc64, gs64 = osc.adjoint64(sc.steps, dl, every=every)

    sim, meta = scenes.build_simulation(sc, form=form)
    sim.forward_checkpointed(sc.steps, every)
    ir = sim.ir(0, sc.steps)
    assert np.abs(ir - ir64).max() <= 1e-4 * np.abs(ir64).max()
    gc, gs = sim.adjoint(dl.astype(np.float32), sc.n_materials, sc.n_sections)
    err_c = np.abs(gc - gc64).max() / np.abs(gc64).max()
    err_s = np.abs(gs - gs64).max() / np.abs(gs64).max()
    print(f"{sc.name}: coef grad err {err_c:.2e}, signal grad err {err_s:.2e}")
    assert err_c <= 1e-4 and err_s <= 1e-4
    with pytest.raises(capi.VirsError) as e:      # the fields were consumed
        sim.run(1)
    assert e.value.status == capi.E_STATE
    sim.close()
    return gc, gs


@pytest.mark.parametrize("form", [0, 1])
def test_gpu_adjoint_matches_fp64_adjoint(form):
    sc, _ = scenes.inverse_design(steps=300, size=(40, 36, 28), h=0.04, n_materials=6)
    sc = dataclasses.replace(sc, courant=0.5 if form == 0 else 1.0)
    _compare(sc, every=32, form=form)


def test_gpu_adjoint_inverse_design_config_reduced():
    """The inverse-design configuration (6 materials x 2 sections, 4
    receivers, checkpoints every 64 steps) on a 64x64x48 room, 800 steps."""
    sc, _ = scenes.inverse_design(steps=800, size=(64, 64, 48))
    _compare(sc, every=64)


def test_torch_autograd_descends():
    import torch
    from virs_b200.autograd import ReceiverIR, attach
    sc, guess = scenes.inverse_design(steps=200, size=(32, 32, 24), h=0.05)
    sim, meta = scenes.build_simulation(sc)
    attach(sim, meta["src"], meta["rcv"])
    with torch.no_grad():
        target = ReceiverIR.apply(torch.tensor(sc.coef64), torch.tensor(sc.src_sig), sim, sc.steps, 50)
    coef = torch.tensor(guess, requires_grad=True)
    sig = torch.tensor(sc.src_sig)
    losses = []
    opt = torch.optim.Adam([coef], lr=2e-3)
    for _ in range(4):
        opt.zero_grad()
        ir = ReceiverIR.apply(coef, sig, sim, sc.steps, 50)
        loss = torch.mean((ir - target) ** 2)
        loss.backward()
        assert coef.grad is not None and torch.isfinite(coef.grad).all()
        opt.step()
        losses.append(float(loss.detach()))
    assert losses[-1] < losses[0]
    sim.close()
