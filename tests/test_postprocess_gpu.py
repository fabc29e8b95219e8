"""virs_postprocess_ir on the GPU against the oracle's post-processing of
the same raw receiver traces: bit for bit, with and without the
anti-alias cascade and the normalisation."""
import numpy as np
import pytest

import oracle
from virs_b200 import capi, scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("with_filter,normalize", [(True, True), (True, False), (False, True)])
def test_postprocess_matches_oracle(with_filter, normalize):
    sc = scenes.plain_small(steps=900)
    sim, _ = scenes.build_simulation(sc)
    sim.run(sc.steps)
    raw = sim.ir()
    dt = float(sim.info().dt)
    fs = float(np.float32(1.0) / np.float32(dt))
    band = min(fs, 48000.0)           # the lower of the two rates bounds the passband
    sos = capi.design_chebyshev_lowpass(fs, 0.40 * band, 0.48 * band) if with_filter else None
    got = sim.postprocess_ir(48000.0, sos, normalize)
    want = oracle.postprocess(raw, dt, 48000.0, sos, normalize)
    assert got.shape == want.shape and got.shape[1] == int(48000.0 * (sc.steps * dt))
    assert np.isfinite(got).all() and np.abs(got).max() > 0
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), np.abs(got - want).max()
    sim.close()


def test_postprocess_many_receivers_and_sections():
    """Hall crop, 8 receivers, an 18-section cascade: every channel matches."""
    sc = scenes.large_hall(steps=1200, size=(128, 128, 128))
    sim, _ = scenes.build_simulation(sc)
    sim.run(sc.steps)
    raw = sim.ir()
    dt = float(sim.info().dt)
    fs = float(np.float32(1.0) / np.float32(dt))
    band = min(fs, 48000.0)
    sos = capi.design_chebyshev_lowpass(fs, 0.40 * band, 0.41 * band, 0.05, 120.0)
    assert 10 <= sos.shape[0] <= 32
    got = sim.postprocess_ir(48000.0, sos, True)
    want = oracle.postprocess(raw, dt, 48000.0, sos, True)
    assert got.shape[0] == raw.shape[0] == 8
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    sim.close()


@pytest.mark.parametrize("normalize", [True, False])
def test_postprocess_sinc_matches_oracle(normalize):
    """virs_postprocess_ir_sinc against the oracle's restatement of the same
    windowed-sinc interpolation.  Both sum in FP64 with sin and sqrt of
    their own libraries, so they agree to rounding: 1e-6 of the peak."""
    sc = scenes.plain_small(steps=900)
    sim, _ = scenes.build_simulation(sc)
    sim.run(sc.steps)
    raw = sim.ir()
    dt = float(sim.info().dt)
    got = sim.postprocess_ir_sinc(48000.0, 64, 8.0, 0.9, normalize)
    n = int(48000.0 * (sc.steps * dt))
    want = np.stack([oracle.resample_sinc(r, 1.0 / dt, 48000.0, n, 64, 8.0, 0.9, normalize) for r in raw])
    assert got.shape == want.shape and np.abs(want).max() > 0
    assert np.abs(got - want).max() <= 1e-6 * np.abs(want).max()
    sim.close()
