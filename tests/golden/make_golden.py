"""Generate golden vectors from the reference's own CUDA kernels.

Runs oracle/_ref/libref_gpu.so -- the reference's fdtd_kernel,
fdtd_kernel_boundary_biquad and spongeKernel compiled from its sources with
its own CUDA flags (oracle/Makefile, target `ref`) -- on a GPU, and writes
the inputs and outputs of each case to tests/golden/<case>.npz:

  flags_raw   voxelised flags (0/1/3), input of the sponge kernel
  flags_ref   spongeKernel output
  bidx        boundary list built from flags_ref (simulator.cpp:572-605)
  coef        the filter coefficients (RBJ high-pass 440 Hz, Q 0.1)
  consts      dt, c2dt2, inv_h2 as uploaded, and the boundary scale as the
              reference kernel computes it on the device (rigid case: also
              the rigid-wall l2 as that kernel computes it)
  rcv, ir     receiver indices and their samples after every step
  p_final     the pressure field after the last step

Usage (needs a GPU and the built checkers):  python tests/golden/make_golden.py [outdir]
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import oracle  # noqa: E402
from helpers import oracle_grid  # noqa: E402
from virs_b200 import scenes  # noqa: E402


def run_case(L, name, shape, flags_raw, h, rcv, steps, out, rigid=False):
    nx, ny, nz = shape
    flags_ref = np.empty_like(flags_raw)
    rc = L.ref_gpu_sponge(nx, ny, nz, flags_raw, flags_ref)
    assert rc == 0, rc
    # boundary list as simulator.cpp:572-605 builds it
    f3 = flags_ref.reshape(nz, ny, nx)
    zz, yy, xx = np.nonzero(f3[1:-1, 1:-1, 1:-1] == 2)
    bidx = np.sort(((zz + 1) * ny + (yy + 1)) * nx + (xx + 1)).astype(np.uint32)
    fs = oracle.filter_fs(h)
    coef = oracle.rbj_highpass_ref(fs, 440.0, 0.1)
    rcv = np.asarray(rcv, np.uint64)
    ir = np.zeros((rcv.size, steps), np.float32)
    p_final = np.zeros(flags_raw.size, np.float32)
    consts = np.zeros(5, np.float32)
    b = bidx if bidx.size else np.zeros(1, np.uint32)
    if rigid:
        normals = oracle.normals(shape, flags_ref)
        rc = L.ref_gpu_run_rigid(nx, ny, nz, h, flags_ref, normals, b, bidx.size, coef, steps, rcv.size, rcv, ir,
                                 p_final, consts)
    else:
        rc = L.ref_gpu_run(nx, ny, nz, h, flags_ref, b, bidx.size, coef, steps, rcv.size, rcv, ir, p_final, consts)
        consts = consts[:4]
    assert rc == 0, rc
    np.savez_compressed(out / f"{name}.npz", shape=np.array(shape), h=np.float32(h), flags_raw=flags_raw,
                        flags_ref=flags_ref, bidx=bidx, coef=coef, consts=consts, rcv=rcv, ir=ir, p_final=p_final)
    print(name, shape, "nb", bidx.size, "ir max", np.abs(ir).max(), "K", consts[3])


def main():
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent
    out.mkdir(parents=True, exist_ok=True)
    L = oracle.ref_gpu()
    if L is None:
        raise SystemExit("oracle/_ref/libref_gpu.so is missing: make -C oracle ref")
    # 1. the reference configuration on a small room with a speaker box
    sc = scenes.reference_room(steps=400, size=(40, 34, 28), h=0.05)
    g = oracle_grid(sc)
    rcv = scenes.voxel_index(sc.rcv_pos, g["bmin"], g["h"], g["shape"])
    run_case(L, "ref_room", g["shape"], g["flags_raw"], g["h"], rcv, sc.steps, out)
    # 2. scattered walls and speakers on an odd-sized grid
    rng = np.random.default_rng(11)
    shape = (45, 31, 27)
    n = int(np.prod(shape))
    f = np.zeros(n, np.uint8)
    f[rng.random(n) < 0.04] = 1
    f[rng.random(n) < 0.002] = 3
    rcv = rng.choice(np.flatnonzero(f == 0), 5, replace=False)
    run_case(L, "ref_scatter", shape, f, float(np.float32(0.03)), rcv, 300, out)
    # 3. the reference room with the rigid-wall kernel launched (its launch is
    #    commented at simulator_gpu.cu:280); consts[4] is its device l2
    sc = scenes.reference_room(steps=400, size=(40, 34, 28), h=0.05)
    g = oracle_grid(sc)
    rcv = scenes.voxel_index(sc.rcv_pos, g["bmin"], g["h"], g["shape"])
    run_case(L, "rigid_room", g["shape"], g["flags_raw"], g["h"], rcv, sc.steps, out, rigid=True)


if __name__ == "__main__":
    main()
