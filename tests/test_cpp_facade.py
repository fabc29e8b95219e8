"""The C++ facade (include/virs.hpp) as a C++ host uses it: the example
program tests/cpp/facade_room.cpp is compiled against the built library.
Without a GPU the library must fail loudly with a status, never fall back;
on a GPU its receiver samples equal those of the same run through the
Python binding, bit for bit."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
LIBDIR = ROOT / "virs_b200"


def _build(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    if not (LIBDIR / "libvirs_b200.so").exists():
        pytest.skip("library not built")
    exe = tmp_path / "facade_room"
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{ROOT / 'include'}",
           str(ROOT / "tests" / "cpp" / "facade_room.cpp"), f"-L{LIBDIR}", "-lvirs_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_facade_compiles_and_reports_errors_by_status(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([str(exe), "10"], capture_output=True, text=True, timeout=300)
    if r.returncode == 0:                       # a GPU is present
        assert len(r.stdout.split()) == 10
    else:                                       # no GPU: a status, not a crash or a CPU fallback
        assert r.returncode >= 10 and "virs error" in r.stderr, (r.returncode, r.stderr)


@pytest.mark.gpu
def test_facade_matches_python_binding(tmp_path):
    from virs_b200 import capi
    exe = _build(tmp_path)
    steps = 300
    r = subprocess.run([str(exe), str(steps)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = np.array([float(x) for x in r.stdout.split()], np.float32)

    sim = capi.Simulation(capi.default_params(cell_size=0.025, bbox_nudge=0.0))
    X, Y, Z = 1.0, 0.8, 0.6
    v = np.array([0, 0, 0, X, 0, 0, X, Y, 0, 0, Y, 0, 0, 0, Z, X, 0, Z, X, Y, Z, 0, Y, Z], np.float32).reshape(-1, 3)
    t = np.array([0, 1, 2, 0, 2, 3, 4, 6, 5, 4, 7, 6, 0, 4, 5, 0, 5, 1, 1, 5, 6, 1, 6, 2, 2, 6, 7, 2, 7, 3, 3, 7, 4,
                  3, 4, 0], np.uint32).reshape(-1, 3)
    sim.set_mesh(v, t, np.zeros(12, np.int32))
    sim.classify()
    g = sim.info()
    at = lambda x, y, z: (z * g.ny + y) * g.nx + x
    u = (np.arange(steps, dtype=np.float64) - 32.0) / 8.0
    sig = (-u * np.exp(-0.5 * u * u)).astype(np.float32)[None, :]
    sim.set_sources([at(g.nx // 2, g.ny // 2, g.nz // 2)], sig)
    sim.set_receivers([at(g.nx // 4, g.ny // 3, g.nz // 2)])
    sim.start(steps)
    sim.run(steps)
    want = sim.ir()[0]
    sim.close()
    assert got.size == steps and np.abs(want).max() > 0
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_slab_room_program_compiles(tmp_path):
    """The C++ slab driver (tests/cpp/slab_room.cpp) builds against the ABI."""
    if shutil.which("g++") is None or not (LIBDIR / "libvirs_b200.so").exists():
        pytest.skip("no g++ or library")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", f"-I{ROOT / 'include'}",
           str(ROOT / "tests" / "cpp" / "slab_room.cpp"), f"-L{LIBDIR}", "-lvirs_b200", f"-Wl,-rpath,{LIBDIR}",
           "-o", str(tmp_path / "slab_room")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
