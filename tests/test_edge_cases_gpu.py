"""Edge cases of the step through the C ABI, against the oracle bit for bit:
a grid with no boundary voxels (an empty boundary list: the pass is not
launched, alone or in a batch), the smallest grid (3 x 3 x 3: one interior
voxel), 16-bit storage on an empty list, sizes beyond the 32-bit voxel
positions rejected before any input is read, and two handles driven from
two host threads at once."""
import numpy as np
import pytest

import oracle
from virs_b200 import capi

pytestmark = pytest.mark.gpu


def _oracle_run(shape, flags, src, sig, rcv, steps, *, storage=0, scale=1.0, h=0.05):
    ref_flags, bm, bd = oracle.classify(shape, 1, flags, None)
    bidx = oracle.boundary_list(shape, ref_flags)
    _, c2dt2, inv_h2, K = oracle.step_constants(h, 343.0, 1.0)
    fs = oracle.filter_fs(h, 343.0, 1.0)
    coef = oracle.rbj_highpass_ref(fs, 440.0, 0.1)[None, None, :]
    osc = oracle.Scene(shape, ref_flags, bidx, bm[bidx], oracle.sponge_weights_for(1, bd[bidx]), coef, 1,
                       hard=np.full(10, 10.0, np.float32), src_idx=src, src_sig=sig, rcv_idx=rcv,
                       consts=(c2dt2, inv_h2, K), form=1, storage=storage, scale=scale)
    n = int(np.prod(shape))
    st = (np.zeros(n, np.float32), np.zeros(n, np.float32), np.zeros(bidx.size * 4 + 1, np.float32))
    return osc.run(steps, state=st), st[0], bidx.size


def _sim(shape, flags, src, sig, rcv, steps, **kw):
    sim = capi.Simulation(capi.default_params(courant=1.0, boundary_form=1, **kw))
    sim.set_grid(shape, 0.05, flags)
    sim.classify()
    sim.set_sources(src, sig)
    sim.set_receivers(rcv)
    sim.start(steps)
    return sim


def _air_room(shape):
    nx, ny, nz = shape
    flags = np.zeros(nx * ny * nz, np.uint8)
    c = (nz // 2 * ny + ny // 2) * nx + nx // 2
    src = np.array([c], np.uint64)
    rcv = np.array([c + 3, c + 5 * nx, c + 2 * nx * ny], np.uint64)
    t = np.arange(200, dtype=np.float64)
    sig = (-(t - 20) / 6.0 * np.exp(-0.5 * ((t - 20) / 6.0) ** 2)).astype(np.float32)[None, :]
    return flags, src, sig, rcv


@pytest.mark.parametrize("depth", [0, 2])
def test_no_boundary_voxels(depth):
    shape = (70, 36, 30)
    flags, src, sig, rcv = _air_room(shape)
    steps = 150
    want, want_p, nb = _oracle_run(shape, flags, src, sig, rcv, steps)
    assert nb == 0
    sim = _sim(shape, flags, src, sig, rcv, steps)
    assert sim.info().boundary_count == 0 and sim.boundary_indices().size == 0
    sim.set_tiling(8, 0, depth)
    sim.run(steps)
    assert np.abs(want).max() > 0
    assert np.array_equal(sim.ir().view(np.uint32), want.view(np.uint32))
    assert np.array_equal(sim.pressure().view(np.uint32), want_p.view(np.uint32))
    sim.close()


def test_no_boundary_voxels_bf16():
    shape = (70, 36, 30)
    flags, src, sig, rcv = _air_room(shape)
    steps, scale = 150, 256.0
    want, want_p, _ = _oracle_run(shape, flags, src, sig, rcv, steps, storage=capi.STORAGE_BF16, scale=scale)
    sim = _sim(shape, flags, src, sig, rcv, steps, storage=capi.STORAGE_BF16, storage_scale=scale)
    sim.run(steps)
    assert np.array_equal(sim.ir().view(np.uint32), want.view(np.uint32))
    sim.close()


def test_batch_with_a_member_without_boundary_voxels():
    """A batch of a room with walls and an all-air room: each member equals
    its run alone."""
    steps = 100
    a_shape = (70, 36, 30)
    a_flags, a_src, a_sig, a_rcv = _air_room(a_shape)
    b_shape = (50, 40, 34)
    nx, ny, nz = b_shape
    b_flags = np.zeros(nx * ny * nz, np.uint8).reshape(nz, ny, nx)
    b_flags[1, 1:-1, 1:-1] = b_flags[-2, 1:-1, 1:-1] = 1
    b_flags[1:-1, 1, 1:-1] = b_flags[1:-1, -2, 1:-1] = 1
    b_flags[1:-1, 1:-1, 1] = b_flags[1:-1, 1:-1, -2] = 1
    b_flags = b_flags.reshape(-1)
    c = (nz // 2 * ny + ny // 2) * nx + nx // 2
    b_src, b_rcv = np.array([c], np.uint64), np.array([c + 4, c + 6 * nx], np.uint64)
    alone = []
    for shape, flags, src, sig, rcv in [(a_shape, a_flags, a_src, a_sig, a_rcv), (b_shape, b_flags, b_src, a_sig, b_rcv)]:
        s = _sim(shape, flags, src, sig, rcv, steps)
        s.run(steps)
        alone.append(s.ir())
        s.close()
    members = [_sim(a_shape, a_flags, a_src, a_sig, a_rcv, steps), _sim(b_shape, b_flags, b_src, a_sig, b_rcv, steps)]
    assert members[0].info().boundary_count == 0 and members[1].info().boundary_count > 0
    batch = capi.Batch(members)
    batch.run(steps)
    batch.synchronize()
    for m, want in zip(members, alone):
        assert np.array_equal(m.ir().view(np.uint32), want.view(np.uint32))
    batch.close()
    for m in members:
        m.close()


def test_smallest_grid():
    """3 x 3 x 3: one interior voxel, a source on it, its own receiver."""
    shape = (3, 3, 3)
    flags = np.zeros(27, np.uint8)
    src = rcv = np.array([13], np.uint64)
    sig = np.linspace(-1, 1, 40, dtype=np.float32)[None, :]
    steps = 40
    want, want_p, _ = _oracle_run(shape, flags, src, sig, rcv, steps)
    sim = _sim(shape, flags, src, sig, rcv, steps)
    sim.run(steps)
    assert np.abs(want).max() > 0
    assert np.array_equal(sim.ir().view(np.uint32), want.view(np.uint32))
    assert np.array_equal(sim.pressure().view(np.uint32), want_p.view(np.uint32))
    sim.close()


def test_grid_beyond_32_bit_positions_rejected():
    """nx rounded up to 32, times ny * nz, must stay below 2^32: the call
    fails with VIRS_E_ARG before it reads the (here tiny) flag array."""
    with capi.Simulation() as sim:
        with pytest.raises(capi.VirsError) as e:
            sim.set_grid((4096, 4096, 300), 0.05, np.zeros(8, np.uint8))
        assert e.value.status == capi.E_ARG
        assert "too large" in str(e.value)


def test_two_handles_on_two_host_threads():
    """Handles share no state but the autotuner's cache (locked) and the
    tensor-map encoder (looked up once): two simulations driven from two
    host threads at the same time give the results they give one after the
    other."""
    import threading
    shape = (70, 36, 30)
    flags, src, sig, rcv = _air_room(shape)
    nx, ny, nz = shape
    walls = flags.reshape(nz, ny, nx).copy()
    walls[1:-1, 1:-1, 1] = walls[1:-1, 1:-1, -2] = 1
    steps = 120

    def run(f, out, k):
        s = _sim(shape, f, src, sig, rcv, steps)
        s.set_tiling(8, 0, 2)
        s.run(steps)
        out[k] = s.ir()
        s.close()

    alone = {}
    run(flags, alone, 0)
    run(walls.reshape(-1), alone, 1)
    both = {}
    th = [threading.Thread(target=run, args=(f, both, k)) for k, f in enumerate([flags, walls.reshape(-1)])]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for k in (0, 1):
        assert np.array_equal(both[k].view(np.uint32), alone[k].view(np.uint32))
