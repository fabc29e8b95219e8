"""The command-line caller (virs_b200/cli/virs_simulate.cpp), as the
reference's `simulate -i config.json`.  Without a GPU: usage, the
configuration's required keys and malformed JSON are reported before any
device call.  On a GPU: the WAV it writes holds the same samples as the
same run through the Python binding, bit for bit."""
import json
import struct
import subprocess
from pathlib import Path

import numpy as np
import pytest

from virs_b200 import build, capi, scenes

ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def cli():
    if not build.LIB.exists():
        pytest.skip("library not built")
    return str(build.build_cli())


def _run(cli, *args, cwd=None):
    return subprocess.run([cli, *map(str, args)], capture_output=True, text=True, timeout=600, cwd=cwd)


def _config(tmp_path, **over):
    cfg = {"files": {"meshfile": str(tmp_path / "room.obj"), "audiofile": "impulse.wav"},
           "simulation": {"num_simulation_steps": 400, "should_save_layer_images": False}}
    for k, v in over.items():
        cfg[k] = v
    p = tmp_path / "config.json"
    p.write_text(json.dumps(cfg))
    return p


def test_usage(cli):
    r = _run(cli, "--help")
    assert r.returncode == 0 and "simulate -i CONFIG.json" in r.stderr
    r = _run(cli)
    assert r.returncode == 2 and "missing command" in r.stderr
    r = _run(cli, "simulate")
    assert r.returncode == 2 and "missing -i" in r.stderr
    r = _run(cli, "simulate", "-i", "x.json", "--storage", "f64")
    assert r.returncode == 2


def test_configuration_errors(cli, tmp_path):
    r = _run(cli, "simulate", "-i", tmp_path / "none.json")
    assert r.returncode == 2 and "cannot open" in r.stderr
    (tmp_path / "bad.json").write_text('{"files": {"meshfile": "a.obj",}')
    r = _run(cli, "simulate", "-i", tmp_path / "bad.json")
    assert r.returncode == 2 and "offset" in r.stderr
    for cfg, word in [({"simulation": {"num_simulation_steps": 10}}, "'files'"),
                      ({"files": {"audiofile": "a.wav"}, "simulation": {"num_simulation_steps": 10}}, "'meshfile'"),
                      ({"files": {"meshfile": "a.obj"}, "simulation": {"num_simulation_steps": 10}}, "'audiofile'"),
                      ({"files": {"meshfile": "a.obj", "audiofile": "a.wav"}}, "'simulation'"),
                      ({"files": {"meshfile": "a.obj", "audiofile": "a.wav"}, "simulation": {}},
                       "'num_simulation_steps'"),
                      ({"files": {"meshfile": "a.obj", "audiofile": "a.wav"},
                        "simulation": {"num_simulation_steps": 2.5}}, "'num_simulation_steps'")]:
        (tmp_path / "c.json").write_text(json.dumps(cfg))
        r = _run(cli, "simulate", "-i", tmp_path / "c.json")
        assert r.returncode == 2 and word in r.stderr, (cfg, r.stderr)


def test_material_configuration_errors(cli, tmp_path):
    base = {"files": {"meshfile": "a.obj", "audiofile": "a.wav"}, "simulation": {"num_simulation_steps": 10}}
    for extra, word in [({"materials": {"index": 0}}, "array"),
                        ({"materials": [{"type": "wall"}]}, "'index'"),
                        ({"materials": [{"index": 0, "type": "glass"}]}, "unknown material type"),
                        ({"materials": [{"index": 0, "type": "wall", "absorber": 2}],
                          "absorbers": [{"reflection": 0.9, "cutoff": 500}]}, "does not define"),
                        ({"materials": [{"index": 0, "type": "wall", "absorber": 1}]}, "'absorbers' is missing"),
                        ({"absorbers": [{"reflection": 0.9}]}, "each absorber"),
                        ({"absorbers": [{"alpha": [0.1, 0.2]}]}, "each absorber"),
                        ({"source": {"audio": True}}, "cannot open"),
                        ({"sources": [{"position": [0.1, 0.2]}]}, "'position'"),
                        ({"sources": [{"position": [0.1, 0.2, 0.3], "channel": -1}]}, "'channel'"),
                        ({"sources": [{"position": [0.1, 0.2, 0.3]}]}, "cannot open")]:
        (tmp_path / "c.json").write_text(json.dumps({**base, **extra}))
        r = _run(cli, "simulate", "-i", tmp_path / "c.json", cwd=tmp_path)
        assert r.returncode == 2 and word in r.stderr, (extra, r.stderr)


def _write_wav(path, x, rate, channels=2):
    """32-bit float WAV, the signal in channel 1 and its negative in 0."""
    x = np.asarray(x, np.float32)
    frames = np.stack([-x, x] if channels == 2 else [x], axis=1).reshape(-1)
    data = frames.tobytes()
    hdr = b"RIFF" + struct.pack("<I", 4 + 24 + 8 + len(data)) + b"WAVE"
    hdr += b"fmt " + struct.pack("<IHHIIHH", 16, 3, channels, rate, rate * 4 * channels, 4 * channels, 32)
    Path(path).write_bytes(hdr + b"data" + struct.pack("<I", len(data)) + data)


def _write_room(tmp_path, sc):
    """The scene as an OBJ with an mtllib: walls (material 0) and a speaker
    box (material 1), one quad per two triangles."""
    (tmp_path / "room.mtl").write_text("newmtl Wall\nKd 0.8 0.8 0.8\n\nnewmtl Speaker\nKd 0.8 0 0\n")
    lines = ["mtllib room.mtl", "o Room"]
    lines += ["v %.6f %.6f %.6f" % tuple(v) for v in sc.verts]
    cur = None
    for t in range(0, len(sc.tris), 2):
        m = int(sc.tri_mat[t])
        if m != cur:
            lines.append("usemtl " + ("Wall" if m == 0 else "Speaker"))
            cur = m
        a, b, c = sc.tris[t] + 1
        d = sc.tris[t + 1][2] + 1
        lines.append(f"f {a} {b} {c} {d}")
    (tmp_path / "room.obj").write_text("\n".join(lines) + "\n")


def _read_wav(path):
    b = Path(path).read_bytes()
    assert b[:4] == b"RIFF" and b[8:12] == b"WAVE"
    i, fmt, data = 12, None, None
    while i + 8 <= len(b):
        tag, n = b[i:i + 4], struct.unpack("<I", b[i + 4:i + 8])[0]
        if tag == b"fmt ":
            fmt = struct.unpack("<HHIIHH", b[i + 8:i + 24])
        elif tag == b"data":
            data = np.frombuffer(b[i + 8:i + 8 + n], np.float32)
        i += 8 + n + (n & 1)
    return fmt, data


@pytest.mark.gpu
def test_cli_wav_equals_python_run(cli, tmp_path):
    sc = scenes.reference_room(size=(8, 6, 5))            # 0.4 x 0.3 x 0.25 m with a speaker box
    _write_room(tmp_path, sc)
    steps = 400
    p = capi.default_params()                              # the reference's defaults, as the CLI uses them
    sim = capi.Simulation(p)
    sim.load_obj(tmp_path / "room.obj")
    sim.classify()
    g = sim.info()
    shape = (int(g.nx), int(g.ny), int(g.nz))
    # an air voxel near the far corner of the room, away from the speaker box
    L = np.array([8, 6, 5], np.float32) * np.float32(0.05)
    idx = int(scenes.voxel_index(0.85 * L, np.array(list(g.bbox_min), np.float32), g.cell_size, shape)[0])
    assert sim.flags()[idx] == 0
    x, y, z = idx % shape[0], (idx // shape[0]) % shape[1], idx // (shape[0] * shape[1])
    sim.set_receivers([idx])
    sim.start(steps)
    sim.run(steps)
    sos = capi.design_chebyshev_lowpass(float(g.sample_rate), 0.45 * 48000, 0.5 * 48000, 0.5, 90.0)
    want = sim.postprocess_ir(48000.0, sos, True)[0]
    sim.close()

    cfg = _config(tmp_path)
    out = tmp_path / "out.wav"
    r = _run(cli, "simulate", "-i", cfg, "-o", out, "--receiver", f"{x},{y},{z}")
    assert r.returncode == 0, r.stderr
    assert f"{steps} steps" in r.stdout
    fmt, data = _read_wav(out)
    assert fmt == (3, 1, 48000, 48000 * 4, 4, 32)
    assert np.abs(want).max() == 1.0
    assert np.array_equal(data.view(np.uint32), want.view(np.uint32))
    # the reference's receiver voxel lies outside this small grid
    r = _run(cli, "simulate", "-i", cfg, "-o", out)
    assert r.returncode == 2 and "outside" in r.stderr


@pytest.mark.gpu
def test_cli_materials_absorbers_and_audio_source(cli, tmp_path):
    """Material indexing (walls with two absorbers: a first-order design and
    a three-band cascade), and the speaker voxels playing channel 1 of a WAV
    file: the same samples as the Python binding given the same roles,
    filters and audio."""
    sc = scenes.reference_room(size=(8, 6, 5))
    _write_room(tmp_path, sc)
    steps = 300
    t = np.arange(2000) / 48000.0
    sig = (np.sin(2 * np.pi * 700 * t) * np.exp(-t * 400)).astype(np.float32)
    _write_wav(tmp_path / "in.wav", sig, 48000)
    roles = np.array([1, 0xFE], np.uint8)                  # walls take absorber 1, material 1 is the speaker
    sim = capi.Simulation(capi.default_params())
    sim.set_material_roles(roles)
    sim.load_obj(tmp_path / "room.obj")
    sim.classify()
    g = sim.info()
    fs = float(g.sample_rate)
    des = [capi.design_first_order(fs, 0.85, 800.0), capi.design_octave_cascade(fs, [0.2, 0.4, 0.6])]
    coef = np.zeros((2, 3, 5), np.float32)
    coef[0, :, 0] = 1.0
    coef[0, 0] = des[0].astype(np.float32).reshape(5)
    coef[1] = des[1].astype(np.float32).reshape(3, 5)
    sim.set_filters(coef, n_sections=3)
    sim.set_hard_source_audio(sig, 48000.0, steps)
    shape = (int(g.nx), int(g.ny), int(g.nz))
    L = np.array([8, 6, 5], np.float32) * np.float32(0.05)
    idx = int(scenes.voxel_index(0.85 * L, np.array(list(g.bbox_min), np.float32), g.cell_size, shape)[0])
    x, y, z = idx % shape[0], (idx // shape[0]) % shape[1], idx // (shape[0] * shape[1])
    sim.set_receivers([idx])
    sim.start(steps)
    sim.run(steps)
    sos = capi.design_chebyshev_lowpass(fs, 0.45 * 48000, 0.5 * 48000, 0.5, 90.0)
    want = sim.postprocess_ir(48000.0, sos, True)[0]
    sim.close()

    cfg = _config(tmp_path, materials=[{"index": 0, "type": "wall", "absorber": 1}, {"index": 1, "type": "source"}],
                  absorbers=[{"reflection": 0.85, "cutoff": 800.0}, {"alpha": [0.2, 0.4, 0.6]}],
                  source={"audio": True, "channel": 1})
    cfg_d = json.loads(cfg.read_text())
    cfg_d["files"]["audiofile"] = str(tmp_path / "in.wav")
    cfg_d["simulation"]["num_simulation_steps"] = steps
    cfg.write_text(json.dumps(cfg_d))
    out = tmp_path / "out.wav"
    r = _run(cli, "simulate", "-i", cfg, "-o", out, "--receiver", f"{x},{y},{z}")
    assert r.returncode == 0, r.stderr
    _, data = _read_wav(out)
    assert np.abs(want).max() == 1.0
    assert np.array_equal(data.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
def test_cli_point_sources_play_audio_channels(cli, tmp_path):
    """Two point sources (metres), each playing one channel of a stereo WAV
    file, the speaker box left to the reference's pulse: the same samples
    as the Python binding given the same voxels and signals."""
    sc = scenes.reference_room(size=(8, 6, 5))
    _write_room(tmp_path, sc)
    steps = 300
    t = np.arange(3000) / 44100.0
    sig = (np.sin(2 * np.pi * 500 * t) * np.exp(-t * 300)).astype(np.float32)
    _write_wav(tmp_path / "in.wav", sig, 44100)               # channel 0: -sig, channel 1: sig
    pos = np.array([[0.05, 0.25, 0.05], [0.35, 0.05, 0.20]], np.float32)      # near two corners, in the air
    sim = capi.Simulation(capi.default_params())
    sim.load_obj(tmp_path / "room.obj")
    sim.classify()
    g = sim.info()
    shape = (int(g.nx), int(g.ny), int(g.nz))
    bmin = np.array(list(g.bbox_min), np.float32)
    src = scenes.voxel_index(pos, bmin, g.cell_size, shape)
    sim.set_sources_audio(src, np.stack([-sig, sig]), 44100.0, steps)
    L = np.array([8, 6, 5], np.float32) * np.float32(0.05)
    idx = int(scenes.voxel_index(0.85 * L, bmin, g.cell_size, shape)[0])
    x, y, z = idx % shape[0], (idx // shape[0]) % shape[1], idx // (shape[0] * shape[1])
    sim.set_receivers([idx])
    sim.start(steps)
    sim.run(steps)
    sos = capi.design_chebyshev_lowpass(float(g.sample_rate), 0.45 * 48000, 0.5 * 48000, 0.5, 90.0)
    want = sim.postprocess_ir(48000.0, sos, True)[0]
    sim.close()

    cfg = _config(tmp_path, sources=[{"position": pos[0].tolist(), "channel": 0},
                                     {"position": pos[1].tolist(), "channel": 1}])
    cfg_d = json.loads(cfg.read_text())
    cfg_d["files"]["audiofile"] = str(tmp_path / "in.wav")
    cfg_d["simulation"]["num_simulation_steps"] = steps
    cfg.write_text(json.dumps(cfg_d))
    out = tmp_path / "out.wav"
    r = _run(cli, "simulate", "-i", cfg, "-o", out, "--receiver", f"{x},{y},{z}")
    assert r.returncode == 0, r.stderr
    _, data = _read_wav(out)
    assert np.array_equal(data.view(np.uint32), want.view(np.uint32))
