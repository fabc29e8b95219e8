"""The reference-side binding (virs_b200/integration/virs_dispatch.cpp): the
reference's dispatch functions (simulator_dispatch.h:4-25) over the C ABI.

It is compiled against stand-ins of the reference's headers
(tests/cpp/ref_stub/) and driven by tests/cpp/dispatch_replay.cpp, which
makes the dispatch calls in the order Simulator::loadObj and
Simulator::simulate make them (simulator.cpp:341, 469, 474, 569, 610, 635,
955-975, 981-1027).  On a GPU that replay must reproduce the golden vectors
that the reference's own kernels produced for the same voxelised room, bit
for bit.  Where the reference tree itself is present, the binding must also
compile against its real vectorspace.h and simulator_dispatch.h."""
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle

ROOT = Path(__file__).resolve().parents[1]
LIBDIR = ROOT / "virs_b200"
BINDING = LIBDIR / "integration"
STUB = ROOT / "tests" / "cpp" / "ref_stub"
GOLD = ROOT / "tests" / "golden"
CXX = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror"]


def _need_toolchain():
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    if not (LIBDIR / "libvirs_b200.so").exists():
        pytest.skip("library not built")


def _build_replay(tmp_path):
    _need_toolchain()
    exe = tmp_path / "dispatch_replay"
    cmd = [*CXX, f"-I{STUB}", f"-I{ROOT / 'include'}", f"-I{BINDING}", str(BINDING / "virs_dispatch.cpp"),
           str(ROOT / "tests" / "cpp" / "dispatch_replay.cpp"), f"-L{LIBDIR}", "-lvirs_b200",
           f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_binding_builds_against_the_interface(tmp_path):
    assert _build_replay(tmp_path).exists()


def test_binding_compiles_against_the_reference_headers(tmp_path):
    """The real Grid and VectorSpace (vectorspace.h:46-231) and the real
    dispatch declarations; only AudioFile (an empty submodule there) comes
    from the stand-ins."""
    _need_toolchain()
    ref = oracle.reference_tree()
    if ref is None:
        pytest.skip("the reference tree is not present")
    afile = tmp_path / "inc"
    afile.mkdir()
    shutil.copy(STUB / "AudioFile.h", afile / "AudioFile.h")
    cmd = ["g++", "-std=c++20", "-O2", "-Wall", "-fsyntax-only", f"-I{ref / 'src' / 'simulator'}", f"-I{afile}",
           f"-I{ROOT / 'include'}", f"-I{BINDING}", str(BINDING / "virs_dispatch.cpp")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def _write_input(path, shape, steps, rcv_xyz, h, flags):
    with open(path, "wb") as f:
        f.write(np.array([*shape, steps, *rcv_xyz], np.uint64).tobytes())
        f.write(np.float32(h).tobytes())
        f.write(np.ascontiguousarray(flags, np.uint8).tobytes())


def _read_output(path, n, steps):
    raw = open(path, "rb").read()
    o = 0
    flags = np.frombuffer(raw, np.uint8, n, o); o += n
    nb = int(np.frombuffer(raw, np.uint64, 1, o)[0]); o += 8
    blist = np.frombuffer(raw, np.uint32, nb, o); o += 4 * nb
    ran = int(np.frombuffer(raw, np.uint64, 1, o)[0]); o += 8
    audio = np.frombuffer(raw, np.float32, steps, o); o += 4 * steps
    p = np.frombuffer(raw, np.float32, n, o); o += 4 * n
    assert o == len(raw)
    return flags, blist, ran, audio, p


@pytest.mark.gpu
def test_reference_call_order_reproduces_golden(tmp_path):
    exe = _build_replay(tmp_path)
    d = np.load(GOLD / "ref_room.npz")
    shape = tuple(int(s) for s in d["shape"])
    nx, ny, nz = shape
    n = nx * ny * nz
    steps = d["ir"].shape[1]
    r0 = int(d["rcv"][0])
    xyz = (r0 % nx, (r0 // nx) % ny, r0 // (nx * ny))
    _write_input(tmp_path / "in.bin", shape, steps, xyz, float(d["h"]), d["flags_raw"])
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True,
                       text=True, timeout=600, env=dict(os.environ))
    assert r.returncode == 0, r.stderr
    flags, blist, ran, audio, p = _read_output(tmp_path / "out.bin", n, steps)
    assert np.array_equal(flags, d["flags_ref"])
    assert np.array_equal(blist, d["bidx"])
    assert ran == steps
    assert np.abs(audio).max() > 0
    assert np.array_equal(audio.view(np.uint32), d["ir"][0].view(np.uint32))
    assert np.array_equal(p.view(np.uint32), d["p_final"].view(np.uint32))
