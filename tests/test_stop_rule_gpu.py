"""The reference's RMS stop rule evaluated on the device (virs_set_stop_rule)
for graph-launched runs.  A virs_run of more steps than needed stops after
the step at which virs_step's host form of the rule (simulator_gpu.cu:303-330)
says stop, with bit-identical receiver samples and fields; a run that the
rule does not stop equals a plain run; the per-step API refuses the device
form."""
import dataclasses

import numpy as np
import pytest

from virs_b200 import capi, scenes

pytestmark = pytest.mark.gpu


def _host_stop(sc):
    """Step through virs_step until its host rule says stop: (stop step or
    None, the simulation)."""
    sim, _ = scenes.build_simulation(sc)
    for n in range(sc.steps):
        keep, _ = sim.step(n)
        if not keep:
            return n, sim
    return None, sim


def test_device_rule_stops_where_the_host_rule_does():
    sc = scenes.reference_room(steps=3200, size=(24, 20, 16))
    stop, host = _host_stop(sc)
    assert stop is not None and stop > 3000
    dev, _ = scenes.build_simulation(sc)
    dev.set_stop_rule(True)
    dev.run(sc.steps)                                       # graphs of 32 steps
    assert dev.stop_state() == (True, stop)
    assert dev.info().steps_done == stop + 1
    assert np.array_equal(dev.ir(0, stop + 1).view(np.uint32), host.ir(0, stop + 1).view(np.uint32))
    p, pp = dev.pressure(prev=True)
    hp, hpp = host.pressure(prev=True)
    assert np.array_equal(p.view(np.uint32), hp.view(np.uint32))
    assert np.array_equal(pp.view(np.uint32), hpp.view(np.uint32))
    dev.run(64)                                             # nothing runs after the stop
    assert dev.info().steps_done == stop + 1
    assert np.array_equal(dev.pressure().view(np.uint32), hp.view(np.uint32))
    dev.start(sc.steps)                                     # a new start clears it
    assert dev.stop_state() == (False, 0)
    host.close()
    dev.close()


def test_device_rule_lets_a_loud_room_run():
    """A hard source 100 times louder keeps the RMS above the threshold: the
    rule runs its filter every step past 3000 and never stops the run."""
    sc = dataclasses.replace(scenes.reference_room(steps=3200, size=(24, 20, 16)),
                             hard=np.full(10, 1000.0, np.float32))
    stop, host = _host_stop(sc)
    assert stop is None
    dev, _ = scenes.build_simulation(sc)
    dev.set_stop_rule(True)
    dev.run(sc.steps)
    assert dev.stop_state() == (False, 0) and dev.info().steps_done == sc.steps
    assert np.array_equal(dev.ir().view(np.uint32), host.ir().view(np.uint32))
    with pytest.raises(capi.VirsError) as e:                # the per-step API keeps the host form
        dev.step(sc.steps)
    assert e.value.status == capi.E_STATE
    host.close()
    dev.close()
