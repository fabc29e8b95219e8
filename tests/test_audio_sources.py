"""Audio-driven sources: a signal at its own sample rate read at the
simulation times by linear interpolation.  Known answers for the oracle's
reading on CPU; on the GPU, runs driven through virs_set_*_audio equal the
oracle's runs with the same tables, bit for bit."""
import numpy as np
import pytest

import oracle
from helpers import oracle_grid, oracle_scene
from virs_b200 import capi, scenes


def test_audio_reading_known_answers():
    dt = np.float32(1.0 / 96000.0)
    # a ramp sampled at 48 kHz is read exactly at every simulation step,
    # and is zero once the sample index + 1 reaches the end (n >= 198 here)
    x = np.arange(100, dtype=np.float32)
    got = oracle.audio_to_steps(x, 48000.0, float(dt), 250)
    si = np.arange(250, dtype=np.float32) * dt * np.float32(48000.0)
    inside = si + np.float32(1.0) < np.float32(100)
    assert inside.sum() == 198
    assert np.allclose(got[inside], si[inside], rtol=0, atol=1e-4)
    assert np.all(got[~inside] == 0)
    # a constant stays constant where it is defined
    c = oracle.audio_to_steps(np.full(10, 0.25, np.float32), 48000.0, float(dt), 10)
    assert np.all(c == np.float32(0.25))


@pytest.mark.gpu
def test_hard_source_from_audio_matches_oracle():
    sc = scenes.reference_room(steps=300)
    g = oracle_grid(sc)
    rng = np.random.default_rng(3)
    audio = rng.standard_normal(2000).astype(np.float32)
    sim, _ = scenes.build_simulation(sc)
    dt = float(sim.info().dt)
    sim.set_hard_source_audio(audio, 44100.0, sc.steps)
    sim.start(sc.steps)
    sim.run(sc.steps)
    got = sim.ir()
    osc = oracle_scene(sc, g)
    osc.hard = oracle.audio_to_steps(audio, 44100.0, dt, sc.steps)
    want = osc.run(sc.steps)
    assert np.count_nonzero(g["flags"] == 3) > 0 and np.abs(want).max() > 0
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    sim.close()


@pytest.mark.gpu
def test_soft_sources_from_audio_match_oracle():
    sc = scenes.plain_small(steps=400)
    g = oracle_grid(sc)
    rng = np.random.default_rng(4)
    sim, meta = scenes.build_simulation(sc)
    dt = float(sim.info().dt)
    audio = (rng.standard_normal((len(meta["src"]), 3000)) * 0.1).astype(np.float32)
    sim.set_sources_audio(meta["src"], audio, 48000.0, sc.steps)
    sim.start(sc.steps)
    sim.run(sc.steps)
    got = sim.ir()
    osc = oracle_scene(sc, g)
    osc.src_sig = np.stack([oracle.audio_to_steps(a, 48000.0, dt, sc.steps) for a in audio])
    want = osc.run(sc.steps)
    assert np.abs(want).max() > 0
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    sim.close()
