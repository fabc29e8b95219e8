"""The C ABI library: loads, exports what include/virs.h declares, and its
host-only entry points agree with the oracle.  CPU only."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import oracle
from conftest import has_gpu
from virs_b200 import capi

HEADER = Path(__file__).resolve().parent.parent / "include" / "virs.h"


def declared():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(virs_[a-z0-9_]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    L = capi.lib()
    names = declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert sorted(capi.EXPORTED) == names


def test_params_struct_matches_header():
    p = capi.default_params()
    assert p.struct_size == C.sizeof(capi.Params)
    assert p.courant == 0.5 and p.sponge_width == 1 and abs(p.boundary_gain - 0.4) < 1e-7
    assert p.mix_filtered == 0.1 and p.mix_direct == 0.9 and abs(p.bbox_nudge - 0.1) < 1e-7


@pytest.mark.parametrize("h", [343 / 88200, 0.025, 1 / 64])
def test_highpass_design_matches_oracle(h):
    fs = oracle.filter_fs(float(np.float32(h)))
    a = capi.design_highpass(fs, 440.0, 0.1)
    b = oracle.rbj_highpass_ref(fs, 440.0, 0.1)
    assert a.view(np.uint32).tolist() == b.view(np.uint32).tolist()
    a = capi.design_lowpass(fs, 2000.0, 0.7)
    b = oracle.rbj_lowpass_ref(fs, 2000.0, 0.7)
    assert a.view(np.uint32).tolist() == b.view(np.uint32).tolist()


def test_fp64_designs_are_stable_filters():
    fs = 76043.95
    k = capi.design_first_order(fs, 0.8, 1000.0)
    assert k[2] == 0 and k[4] == 0 and abs(k[3]) < 1
    dc = (k[0] + k[1]) / (1 + k[3])
    assert abs(dc - (1 - 0.8) / (1 + 0.8)) < 1e-12
    c = capi.design_octave_cascade(fs, [0.1, 0.5, 0.8])
    for s in c:                                  # poles inside the unit circle
        r = np.roots([1.0, s[3], s[4]])
        assert np.all(np.abs(r) < 1)
    with pytest.raises(capi.VirsError) as e:
        capi.design_first_order(fs, 1.0, 1000.0)
    assert e.value.status == capi.E_ARG


@pytest.mark.skipif(has_gpu(), reason="checks the no-GPU failure path")
def test_create_without_gpu_fails_loudly():
    with pytest.raises(capi.VirsError) as e:
        capi.Simulation()
    assert e.value.status in (capi.E_CUDA, capi.E_ARG)
    assert capi.last_error()
