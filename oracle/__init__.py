"""CPU oracle for the VIRS FDTD path -- TEST INFRASTRUCTURE ONLY.

ctypes bindings over ``oracle/libvirs_oracle.so`` (the C restatement in
``virs_oracle.c``) and over the reference-built checkers in ``oracle/_ref/``
when they exist.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` import this
package; the product (``virs_b200``) never does.

Every function names the reference source it restates (paths relative to the
Snipet/VIRS tree).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libvirs_oracle.so"
REF_DIR = HERE / "_ref"

ROLE_IGNORE = 0xFF
ROLE_SOURCE = 0xFE

_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")


def build() -> None:
    """Compile the oracle (``make -C oracle``)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def reference_tree() -> Path | None:
    """The Snipet/VIRS source tree the reference-built checkers compile from:
    $VIRS_REFERENCE_TREE when set (it must then be that tree), else a
    directory named `reference` beside this repository, else None."""
    env = os.environ.get("VIRS_REFERENCE_TREE")
    if env:
        if not Path(env, "src/simulator/biquad.cpp").exists():
            raise FileNotFoundError(f"VIRS_REFERENCE_TREE={env} is not the Snipet/VIRS source tree "
                                    "(no src/simulator/biquad.cpp)")
        return Path(env)
    sibling = HERE.parent.parent / "reference"
    return sibling if Path(sibling, "src/simulator/biquad.cpp").exists() else None


def build_ref() -> bool:
    """Compile the reference-built checkers when the reference tree exists
    (reference_tree()); False when there is none."""
    ref = reference_tree()
    if ref is None:
        return False
    subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={ref}"], check=True)
    return True


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        L.vo_sat.restype = C.c_int
        L.vo_sat.argtypes = [_f32p] * 5
        L.vo_bbox.argtypes = [_f32p, C.c_uint64, C.c_float, _f32p, _f32p]
        L.vo_dims.argtypes = [_f32p, _f32p, C.c_float, _u64p]
        L.vo_voxelize.restype = C.c_int
        L.vo_voxelize.argtypes = [_f32p, _i32p, C.c_uint64, _u8p, C.c_uint64, C.c_float, _f32p,
                                  C.c_uint64, C.c_uint64, C.c_uint64, _u8p, _u8p]
        L.vo_classify.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_int, _u8p, _u8p, _u8p, _u8p, _u16p]
        L.vo_normals.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, _u8p, _u8p]
        L.vo_boundary_list.restype = C.c_uint64
        L.vo_boundary_list.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, _u8p, C.c_void_p]
        L.vo_step_constants.argtypes = [C.c_float, C.c_float, C.c_float, _f32p]
        L.vo_filter_fs.restype = C.c_double
        L.vo_filter_fs.argtypes = [C.c_float, C.c_double, C.c_double]
        L.vo_rbj_highpass_ref.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float, _f32p]
        L.vo_rbj_lowpass_ref.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float, _f32p]
        L.vo_sponge_weight.restype = C.c_float
        L.vo_sponge_weight.argtypes = [C.c_int, C.c_int]
        L.vo_run_f32.restype = C.c_int
        L.vo_run_f32.argtypes = [C.c_void_p]
        L.vo_run_f64.restype = C.c_int
        L.vo_run_f64.argtypes = [C.c_void_p]
        L.vo_adjoint_f64.restype = C.c_int
        L.vo_adjoint_f64.argtypes = [C.c_void_p]
        L.vo_energy_f32.restype = C.c_double
        L.vo_energy_f32.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, _u8p, _f32p, _f32p, C.c_double]
        L.vo_cheby_design.restype = C.c_int
        L.vo_cheby_design.argtypes = [C.c_double] * 5 + [C.c_void_p, C.c_int]
        L.vo_sos_df2t.restype = None
        L.vo_sos_df2t.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_uint64]
        L.vo_resample_len.restype = C.c_uint64
        L.vo_resample_len.argtypes = [C.c_double, C.c_uint64, C.c_float]
        L.vo_resample.restype = None
        L.vo_resample.argtypes = [C.c_void_p, C.c_uint64, C.c_double, C.c_double, C.c_void_p, C.c_uint64, C.c_int]
        L.vo_audio_to_steps.restype = None
        L.vo_audio_to_steps.argtypes = [C.c_void_p, C.c_uint64, C.c_float, C.c_float, C.c_uint64, C.c_void_p]
        L.vo_round16.restype = None
        L.vo_round16.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32]
        L.vo_set_threads.argtypes = [C.c_int]
        L.vo_get_threads.restype = C.c_int
        _lib = L
    return _lib


def set_threads(n: int) -> None:
    lib().vo_set_threads(int(n))


def threads() -> int:
    return int(lib().vo_get_threads())


# --------------------------------------------------------------------------
# geometry
# --------------------------------------------------------------------------

def sat(v0, v1, v2, bmin, bmax) -> bool:
    """simulator.cpp:45-141 (triangleBoxOverlap3)."""
    f = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    return bool(lib().vo_sat(f(v0), f(v1), f(v2), f(bmin), f(bmax)))


def bbox(verts: np.ndarray, nudge: float):
    """simulator.cpp:288-310, including the FLT_MIN start of the max corner."""
    v = np.ascontiguousarray(verts, dtype=np.float32).reshape(-1, 3)
    lo = np.zeros(3, np.float32)
    hi = np.zeros(3, np.float32)
    lib().vo_bbox(v, v.shape[0], nudge, lo, hi)
    return lo, hi


def dims(bmin, bmax, h: float):
    """simulator.cpp:321-329."""
    out = np.zeros(3, np.uint64)
    lib().vo_dims(np.ascontiguousarray(bmin, np.float32), np.ascontiguousarray(bmax, np.float32), h, out)
    return tuple(int(x) for x in out)


def voxelize(tris: np.ndarray, tri_mat: np.ndarray, roles: np.ndarray, h: float, bmin, shape):
    """simulator.cpp:396-452.  shape = (nx, ny, nz); returns (flags, wall_mat)
    as flat arrays in the reference layout idx = (z*ny + y)*nx + x."""
    nx, ny, nz = shape
    t = np.ascontiguousarray(tris, dtype=np.float32).reshape(-1, 9)
    m = np.ascontiguousarray(tri_mat, dtype=np.int32)
    r = np.ascontiguousarray(roles, dtype=np.uint8)
    flags = np.zeros(nx * ny * nz, np.uint8)
    wmat = np.zeros(nx * ny * nz, np.uint8)
    rc = lib().vo_voxelize(t, m, t.shape[0], r, r.size, h, np.ascontiguousarray(bmin, np.float32),
                           nx, ny, nz, flags, wmat)
    if rc != 0:
        raise ValueError("voxelize: empty grid")
    return flags, wmat


def classify(shape, width: int, flags: np.ndarray, wall_mat: np.ndarray | None = None):
    """sponge_kernel.cu:8-62 generalised to width W.  Returns
    (flags_out, bmat_per_voxel, bd2_per_voxel)."""
    nx, ny, nz = shape
    fi = np.ascontiguousarray(flags, np.uint8)
    wm = np.ascontiguousarray(wall_mat if wall_mat is not None else np.zeros_like(fi), np.uint8)
    fo = np.empty_like(fi)
    bm = np.empty_like(fi)
    bd = np.empty(fi.size, np.uint16)
    lib().vo_classify(nx, ny, nz, int(width), fi, wm, fo, bm, bd)
    return fo, bm, bd


def normals(shape, flags):
    """simulator.cpp:480-531."""
    nx, ny, nz = shape
    out = np.empty(nx * ny * nz, np.uint8)
    lib().vo_normals(nx, ny, nz, np.ascontiguousarray(flags, np.uint8), out)
    return out


def boundary_list(shape, flags) -> np.ndarray:
    """simulator.cpp:572-605."""
    nx, ny, nz = shape
    f = np.ascontiguousarray(flags, np.uint8)
    n = lib().vo_boundary_list(nx, ny, nz, f, None)
    out = np.zeros(max(int(n), 1), np.uint32)
    lib().vo_boundary_list(nx, ny, nz, f, out.ctypes.data)
    return out[: int(n)]


# --------------------------------------------------------------------------
# constants and filters
# --------------------------------------------------------------------------

def step_constants(h: float, c: float = 343.0, courant: float = 0.5):
    """simulator_gpu.cu:195-198 and :147 -> (dt, c2dt2, inv_h2, K) as float32."""
    out = np.zeros(4, np.float32)
    lib().vo_step_constants(h, c, courant, out)
    return tuple(np.float32(x) for x in out)


def filter_fs(h: float, c: float = 343.0, courant: float = 0.5) -> float:
    """simulator.cpp:940-952: the sample rate handed to the filter design."""
    return float(lib().vo_filter_fs(h, c, courant))


def rbj_highpass_ref(fs: float, cutoff: float, q: float, gain: float = 1.0) -> np.ndarray:
    """biquad.cpp:24-43 -> [b0, b1, b2, a1, a2] float32."""
    out = np.zeros(5, np.float32)
    lib().vo_rbj_highpass_ref(fs, cutoff, q, gain, out)
    return out


def rbj_lowpass_ref(fs: float, cutoff: float, q: float, gain: float = 1.0) -> np.ndarray:
    """biquad.cpp:3-22 -> [b0, b1, b2, a1, a2] float32."""
    out = np.zeros(5, np.float32)
    lib().vo_rbj_lowpass_ref(fs, cutoff, q, gain, out)
    return out


def sponge_weight(width: int, d2: int) -> np.float32:
    return np.float32(lib().vo_sponge_weight(int(width), int(d2)))


def sponge_weights_for(width: int, bd2_list: np.ndarray) -> np.ndarray:
    table = np.array([sponge_weight(width, d) for d in range(width * width + 1)], np.float32)
    return table[np.asarray(bd2_list, np.int64)]


# --------------------------------------------------------------------------
# time stepping
# --------------------------------------------------------------------------

class _RunArgs(C.Structure):
    _fields_ = [
        ("nx", C.c_uint64), ("ny", C.c_uint64), ("nz", C.c_uint64),
        ("flags", C.c_void_p),
        ("nb", C.c_uint64), ("bidx", C.c_void_p), ("bmat", C.c_void_p), ("bw", C.c_void_p),
        ("n_materials", C.c_uint32), ("n_sections", C.c_uint32),
        ("coef32", C.c_void_p), ("coef64", C.c_void_p),
        ("c2dt2", C.c_float), ("inv_h2", C.c_float), ("K", C.c_float),
        ("c2dt2_d", C.c_double), ("inv_h2_d", C.c_double), ("K_d", C.c_double),
        ("mix_y", C.c_double), ("mix_d", C.c_double), ("gain", C.c_double), ("form", C.c_int32),
        ("hard", C.c_void_p), ("n_hard", C.c_uint64),
        ("n_src", C.c_uint32), ("src_idx", C.c_void_p), ("src_sig", C.c_void_p), ("sig_len", C.c_uint64),
        ("n_rcv", C.c_uint32), ("rcv_idx", C.c_void_p),
        ("steps", C.c_uint64), ("step0", C.c_uint64), ("ir_stride", C.c_uint64),
        ("ir", C.c_void_p), ("p", C.c_void_p), ("pprev", C.c_void_p), ("state", C.c_void_p),
        ("ir64", C.c_void_p),
        ("storage", C.c_int32), ("scale", C.c_float),
        ("rigid", C.c_int32), ("l2", C.c_float), ("normals", C.c_void_p),
        ("rounding", C.c_int32), ("sr_base", C.c_uint64),
    ]


class _AdjArgs(C.Structure):
    _fields_ = [("run", C.c_void_p), ("dl_dir", C.c_void_p), ("every", C.c_uint32), ("grad_coef", C.c_void_p),
                ("grad_sig", C.c_void_p)]


def _ptr(a):
    return None if a is None else a.ctypes.data


class Scene:
    """Everything one run needs, in the reference layout (flat, x fastest)."""

    def __init__(self, shape, flags, bidx, bmat, bw, coef32, n_sections, *, coef64=None,
                 hard=None, src_idx=(), src_sig=None, rcv_idx=(), consts=None, consts64=None,
                 mix_y=0.1, mix_d=0.9, gain=float(np.float32(0.4)), form=0, storage=0, scale=1.0,
                 normals=None, rigid=False, l2=0.0, rounding=0):
        self.shape = tuple(int(s) for s in shape)
        self.flags = np.ascontiguousarray(flags, np.uint8)
        self.bidx = np.ascontiguousarray(bidx, np.uint32)
        self.bmat = np.ascontiguousarray(bmat if bmat is not None else np.zeros(self.bidx.size), np.uint8)
        self.bw = None if bw is None else np.ascontiguousarray(bw, np.float32)
        self.coef32 = np.ascontiguousarray(coef32, np.float32).reshape(-1)
        self.coef64 = None if coef64 is None else np.ascontiguousarray(coef64, np.float64).reshape(-1)
        self.n_sections = int(n_sections)
        self.n_materials = self.coef32.size // (5 * self.n_sections)
        self.hard = np.ascontiguousarray(hard if hard is not None else np.zeros(0), np.float32)
        self.src_idx = np.ascontiguousarray(src_idx, np.uint64)
        if self.src_idx.size == 0 or src_sig is None:
            self.src_sig = np.zeros((self.src_idx.size, 1), np.float32)
        else:
            self.src_sig = np.ascontiguousarray(src_sig, np.float32).reshape(self.src_idx.size, -1)
        self.rcv_idx = np.ascontiguousarray(rcv_idx, np.uint64)
        self.consts = consts          # (c2dt2, inv_h2, K) float32
        self.consts64 = consts64      # (c2dt2, inv_h2, K) float64
        self.mix_y, self.mix_d, self.gain = float(mix_y), float(mix_d), float(gain)
        self.form = int(form)
        self.storage = int(storage)   # FP32 run: 0 FP32 fields, 1 FP16, 2 BF16 (rounded as the GPU stores them)
        self.scale = float(scale)     # 16-bit storage: fields hold scale * p (a power of two)
        self.normals = None if normals is None else np.ascontiguousarray(normals, np.uint8)
        self.rigid = bool(rigid)      # FP32 run: rigid-wall update of the boundary voxels
        self.l2 = float(l2)           # its (c dt / h)^2
        self.rounding = int(rounding) # 16-bit storage: 0 to nearest, 1 stochastic (the library's definition)

    def _args(self, steps, step0, ir, p, pp, st, f64):
        a = _RunArgs()
        a.nx, a.ny, a.nz = self.shape
        a.flags = _ptr(self.flags)
        a.nb = self.bidx.size
        a.bidx, a.bmat, a.bw = _ptr(self.bidx), _ptr(self.bmat), _ptr(self.bw)
        a.n_materials, a.n_sections = self.n_materials, self.n_sections
        a.coef32 = _ptr(self.coef32)
        a.coef64 = _ptr(self.coef64)
        if self.consts is not None:
            a.c2dt2, a.inv_h2, a.K = [float(x) for x in self.consts]
        if self.consts64 is not None:
            a.c2dt2_d, a.inv_h2_d, a.K_d = [float(x) for x in self.consts64]
        a.mix_y, a.mix_d, a.gain, a.form = self.mix_y, self.mix_d, self.gain, self.form
        a.hard, a.n_hard = _ptr(self.hard), self.hard.size
        a.n_src, a.src_idx, a.src_sig, a.sig_len = self.src_idx.size, _ptr(self.src_idx), _ptr(self.src_sig), self.src_sig.shape[1]
        a.n_rcv, a.rcv_idx = self.rcv_idx.size, _ptr(self.rcv_idx)
        a.steps, a.step0, a.ir_stride = steps, step0, steps
        a.ir, a.p, a.pprev, a.state = _ptr(ir), _ptr(p), _ptr(pp), _ptr(st)
        a.storage, a.scale = self.storage, self.scale
        a.rounding = self.rounding
        if self.rigid:
            if self.normals is None:
                raise ValueError("the rigid-wall update needs the normals")
            a.rigid, a.l2, a.normals = 1, self.l2, _ptr(self.normals)
        return a

    def run64(self, steps):
        """FP64 run returning the receiver samples in double [R, steps]."""
        ir = np.zeros((max(self.rcv_idx.size, 1), steps), np.float32)
        ir64 = np.zeros((max(self.rcv_idx.size, 1), steps), np.float64)
        a = self._args(steps, 0, ir, None, None, None, True)
        a.ir64 = ir64.ctypes.data
        if lib().vo_run_f64(C.byref(a)) != 0:
            raise MemoryError("oracle run: allocation failed")
        return ir64[: self.rcv_idx.size]

    def adjoint64(self, steps, dl_dir, every=64):
        """Gradients of a receiver loss through the FP64 model: returns
        (dL/dcoef [M][S][5], dL/dsignal [n_src][steps])."""
        dl = np.ascontiguousarray(dl_dir, np.float64).reshape(self.rcv_idx.size, steps)
        gc = np.zeros(self.n_materials * self.n_sections * 5, np.float64)
        gs = np.zeros((max(self.src_idx.size, 1), steps), np.float64)
        ir = np.zeros((max(self.rcv_idx.size, 1), steps), np.float32)
        a = self._args(steps, 0, ir, None, None, None, True)
        aa = _AdjArgs()
        aa.run = C.addressof(a)
        aa.dl_dir = dl.ctypes.data
        aa.every = int(every)
        aa.grad_coef = gc.ctypes.data
        aa.grad_sig = gs.ctypes.data
        if lib().vo_adjoint_f64(C.byref(aa)) != 0:
            raise MemoryError("oracle adjoint: allocation failed")
        return gc.reshape(self.n_materials, self.n_sections, 5), gs[: self.src_idx.size]

    def run(self, steps, *, f64=False, step0=0, state=None):
        """Run ``steps`` steps.  ``state`` = (p, pprev, biquad_states) to
        continue from (modified in place); returns the IRs [R, steps]."""
        ir = np.zeros((max(self.rcv_idx.size, 1), steps), np.float32)
        dt = np.float64 if f64 else np.float32
        if state is None:
            N = int(np.prod(self.shape))
            state = (np.zeros(N, dt), np.zeros(N, dt), np.zeros(max(self.bidx.size * self.n_sections * 4, 1), dt))
        p, pp, st = state
        a = self._args(steps, step0, ir, p, pp, st, f64)
        rc = (lib().vo_run_f64 if f64 else lib().vo_run_f32)(C.byref(a))
        if rc != 0:
            raise MemoryError("oracle run: allocation failed")
        return ir[: self.rcv_idx.size]


def cheby_design(fs, fc, fstop=0.0, ap_db=0.5, as_db=90.0):
    """The anti-alias Chebyshev-I sections [n][6] (ValueError for invalid specs)."""
    out = np.zeros((64, 6), np.float64)
    n = lib().vo_cheby_design(fs, fc, fstop, ap_db, as_db, out.ctypes.data, 64)
    if n < 0:
        raise ValueError("invalid Chebyshev specification")
    return out[:n].copy()


def sos_df2t(sos, x):
    """One channel through the cascade (FP64 transposed direct form II)."""
    s = np.ascontiguousarray(sos, np.float64).reshape(-1, 6)
    x = np.ascontiguousarray(x, np.float32)
    y = np.empty_like(x)
    lib().vo_sos_df2t(s.ctypes.data, s.shape[0], x.ctypes.data, y.ctypes.data, x.size)
    return y


def postprocess(ir, dt, rate=48000.0, sos=None, normalize=True):
    """The receiver traces [R][steps] filtered, resampled to `rate` and
    (optionally) peak-normalised, as virs_postprocess_ir defines it."""
    ir = np.ascontiguousarray(ir, np.float32).reshape(-1, np.shape(ir)[-1])
    steps = ir.shape[1]
    n = int(lib().vo_resample_len(rate, steps, dt))
    sim_rate = float(np.float32(1.0) / np.float32(dt))
    out = np.zeros((ir.shape[0], n), np.float32)
    for r in range(ir.shape[0]):
        x = ir[r] if sos is None or len(sos) == 0 else sos_df2t(sos, ir[r])
        lib().vo_resample(x.ctypes.data, steps, sim_rate, rate, out[r].ctypes.data, n, int(normalize))
    return out


def resample_sinc(x, fs_in: float, rate: float, out_len: int, half: int, beta: float, cutoff: float,
                  normalize: bool = False):
    """One channel through the library's windowed-sinc resampler (FP64)."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros(int(out_len), np.float32)
    lib().vo_resample_sinc(C.c_void_p(x.ctypes.data), C.c_uint64(x.size), C.c_double(fs_in), C.c_double(rate),
                           C.c_int(int(half)), C.c_double(beta), C.c_double(cutoff), C.c_void_p(out.ctypes.data),
                           C.c_uint64(out.size), C.c_int(int(normalize)))
    return out


def audio_to_steps(x, rate: float, dt: float, steps: int):
    """An audio signal at `rate` read at step * dt (linear interpolation)."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros(steps, np.float32)
    lib().vo_audio_to_steps(x.ctypes.data, x.size, rate, dt, steps, out.ctypes.data)
    return out


def round16(x, storage: int):
    """Values rounded as the 16-bit field storage stores them (1 FP16, 2 BF16)."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    lib().vo_round16(x.ctypes.data, out.ctypes.data, C.c_uint64(x.size), C.c_int32(storage))
    return out


def design_first_order(fs: float, reflection: float, fc: float) -> np.ndarray:
    """The library's first-order absorber design restated in FP64 ({b0, b1, b2, a1, a2})."""
    out = np.zeros(5, np.float64)
    lib().vo_design_first_order(C.c_double(fs), C.c_double(reflection), C.c_double(fc), C.c_void_p(out.ctypes.data))
    return out


def design_octave_cascade(fs: float, alpha) -> np.ndarray:
    """The library's three-section octave cascade restated in FP64 ([3][5])."""
    a = np.ascontiguousarray(alpha, np.float64)
    out = np.zeros(15, np.float64)
    lib().vo_design_octave_cascade(C.c_double(fs), C.c_void_p(a.ctypes.data), C.c_void_p(out.ctypes.data))
    return out.reshape(3, 5)


def init_sphere(p, shape, center, radius: int, pressure: float, zero_outside: bool = True):
    """initSphereKernel (init_sphere.cu:4-25) applied in place to the flat
    float32 field `p` of `shape` (nx, ny, nz); returns p."""
    nx, ny, nz = shape
    assert p.dtype == np.float32 and p.flags.c_contiguous and p.size == nx * ny * nz
    cx, cy, cz = (int(c) for c in center)
    lib().vo_init_sphere(C.c_void_p(p.ctypes.data), C.c_uint64(nx), C.c_uint64(ny), C.c_uint64(nz), C.c_uint64(cx),
                         C.c_uint64(cy), C.c_uint64(cz), C.c_uint64(int(radius)), C.c_float(pressure),
                         C.c_int(int(zero_outside)))
    return p


def sr16(x, storage: int, r16):
    """Values rounded stochastically as the library's 16-bit stores round
    them (1 FP16, 2 BF16), each with its 16 random bits r16."""
    x = np.ascontiguousarray(x, np.float32)
    r = np.ascontiguousarray(np.broadcast_to(np.asarray(r16, np.uint32), x.shape))
    out = np.empty_like(x)
    lib().vo_sr16_array(C.c_void_p(x.ctypes.data), C.c_void_p(out.ctypes.data), C.c_uint64(x.size),
                        C.c_int32(storage), C.c_void_p(r.ctypes.data))
    return out


def energy(shape, flags, p, pprev, lambda2: float) -> float:
    nx, ny, nz = shape
    return float(lib().vo_energy_f32(nx, ny, nz, np.ascontiguousarray(flags, np.uint8),
                                     np.ascontiguousarray(p, np.float32), np.ascontiguousarray(pprev, np.float32),
                                     lambda2))


# --------------------------------------------------------------------------
# reference-built checkers (oracle/_ref), present only where they were built
# --------------------------------------------------------------------------

def ref_host(fast: bool = False):
    """The reference's triangleBoxOverlap3 and biquad design, compiled from
    its own sources (IEEE flags, or its Release -ffast-math flags)."""
    p = REF_DIR / ("libref_host_fast.so" if fast else "libref_host.so")
    if not p.exists():
        return None
    L = C.CDLL(str(p))
    L.ref_sat.restype = C.c_int
    L.ref_sat.argtypes = [_f32p] * 5
    L.ref_sat_batch.argtypes = [_f32p, _f32p, C.c_uint64, _u8p]
    L.ref_highpass.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float, _f32p]
    L.ref_lowpass.argtypes = [C.c_float, C.c_float, C.c_float, C.c_float, _f32p]
    return L


def ref_dsp():
    """The reference's anti-alias filter design and cascade
    (src/util/downsampling_filter_iir.cpp), compiled as it is."""
    p = REF_DIR / "libref_dsp.so"
    if not p.exists():
        return None
    L = C.CDLL(str(p))
    L.ref_cheby_design.restype = C.c_int
    L.ref_cheby_design.argtypes = [C.c_double] * 5 + [C.c_void_p, C.c_int]
    L.ref_cheby_process.restype = None
    L.ref_cheby_process.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_uint64]
    return L


def ref_gpu():
    """The reference's CUDA kernels behind a host driver that follows
    fdtd_gpu_step (needs a GPU)."""
    p = REF_DIR / "libref_gpu.so"
    if not p.exists():
        return None
    L = C.CDLL(str(p))
    L.ref_gpu_sponge.restype = C.c_int
    L.ref_gpu_sponge.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, _u8p, _u8p]
    L.ref_gpu_run_rigid.restype = C.c_int
    L.ref_gpu_run_rigid.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_float, _u8p, _u8p, _u32p, C.c_uint64,
                                    _f32p, C.c_uint32, C.c_uint32, _u64p, _f32p, _f32p, _f32p]
    L.ref_gpu_run.restype = C.c_int
    L.ref_gpu_run.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_float, _u8p, _u32p, C.c_uint64, _f32p,
                              C.c_uint32, C.c_uint32, _u64p, _f32p, _f32p, _f32p]
    return L
