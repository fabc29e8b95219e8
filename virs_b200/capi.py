"""ctypes binding of include/virs.h (the library's C ABI).

Thin and literal: one method per entry point, numpy arrays for host
buffers, a VirsError carrying the status code and the library's message on
any failure.  The library must have been built (``python -m
virs_b200.build``); there is no fallback when it is missing.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libvirs_b200.so"

OK, E_ARG, E_OOM, E_CUDA, E_UNSTABLE, E_TIMEOUT, E_STATE, E_IO = range(8)
STATUS_NAMES = {0: "OK", 1: "E_ARG", 2: "E_OOM", 3: "E_CUDA", 4: "E_UNSTABLE", 5: "E_TIMEOUT", 6: "E_STATE", 7: "E_IO"}
STORAGE_F32, STORAGE_F16, STORAGE_BF16 = 0, 1, 2
ROUND_NEAREST, ROUND_STOCHASTIC = 0, 1
ROLE_IGNORE, ROLE_SOURCE = 0xFF, 0xFE
BOUNDARY_REFERENCE, BOUNDARY_CENTERED = 0, 1


class VirsError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class Params(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32), ("device", C.c_int32), ("sound_speed", C.c_float), ("courant", C.c_float),
        ("cell_size", C.c_float), ("bbox_nudge", C.c_float), ("sponge_width", C.c_int32), ("storage", C.c_int32),
        ("boundary_form", C.c_int32),
        ("storage_scale", C.c_float), ("boundary_gain", C.c_float), ("boundary_k", C.c_float),
        ("mix_filtered", C.c_double), ("mix_direct", C.c_double), ("rigid_walls", C.c_int32),
    ]


class GridInfo(C.Structure):
    _fields_ = [
        ("nx", C.c_uint64), ("ny", C.c_uint64), ("nz", C.c_uint64), ("cell_size", C.c_float),
        ("bbox_min", C.c_float * 3), ("dt", C.c_float), ("sample_rate", C.c_double),
        ("boundary_count", C.c_uint64), ("steps_done", C.c_uint64),
    ]


class Tiling(C.Structure):
    _fields_ = [("tile_rows", C.c_int32), ("planes_per_block", C.c_int32), ("pipeline_depth", C.c_int32),
                ("ms_per_step", C.c_float)]


class Timing(C.Structure):
    _fields_ = [("step_kernel_ms", C.c_double), ("boundary_kernel_ms", C.c_double), ("step_launches", C.c_uint64),
                ("kernel_launches", C.c_uint64)]


_P = C.c_void_p
_SIGS = {
    "virs_last_error": ([], C.c_char_p),
    "virs_params_default": ([_P], C.c_int),
    "virs_create": ([_P, _P], C.c_int),
    "virs_destroy": ([_P], C.c_int),
    "virs_set_material_roles": ([_P, _P, C.c_size_t], C.c_int),
    "virs_load_obj": ([_P, C.c_char_p], C.c_int),
    "virs_set_mesh": ([_P, _P, C.c_size_t, _P, _P, C.c_size_t], C.c_int),
    "virs_set_grid": ([_P, C.c_uint64, C.c_uint64, C.c_uint64, C.c_float, _P, _P], C.c_int),
    "virs_get_grid_info": ([_P, _P], C.c_int),
    "virs_set_grid_slab": ([_P, C.c_uint64, C.c_uint64, C.c_uint64, C.c_float, C.c_uint64, C.c_uint64, _P, _P,
                            C.c_uint64, C.c_uint64], C.c_int),
    "virs_slab_planes": ([_P, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                          C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)], C.c_int),
    "virs_set_mesh_slab": ([_P, _P, C.c_size_t, _P, _P, C.c_size_t, C.c_uint32, C.c_uint32], C.c_int),
    "virs_load_obj_slab": ([_P, C.c_char_p, C.c_uint32, C.c_uint32], C.c_int),
    "virs_get_slab_info": ([_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)], C.c_int),
    "virs_classify": ([_P], C.c_int),
    "virs_get_flags": ([_P, _P, C.c_size_t], C.c_int),
    "virs_get_normals": ([_P, _P, C.c_size_t], C.c_int),
    "virs_get_wall_materials": ([_P, _P, C.c_size_t], C.c_int),
    "virs_get_boundary_indices": ([_P, _P, C.c_size_t], C.c_int),
    "virs_get_boundary_materials": ([_P, _P, _P, C.c_size_t], C.c_int),
    "virs_set_filters": ([_P, C.c_uint32, C.c_uint32, _P], C.c_int),
    "virs_design_highpass": ([C.c_float, C.c_float, C.c_float, C.c_float, _P], C.c_int),
    "virs_design_lowpass": ([C.c_float, C.c_float, C.c_float, C.c_float, _P], C.c_int),
    "virs_design_first_order": ([C.c_double, C.c_double, C.c_double, _P], C.c_int),
    "virs_design_octave_cascade": ([C.c_double, _P, _P, _P], C.c_int),
    "virs_design_chebyshev_lowpass": ([C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, _P, C.c_uint32,
                                       C.POINTER(C.c_uint32)], C.c_int),
    "virs_set_hard_source_audio": ([_P, _P, C.c_size_t, C.c_float, C.c_uint64], C.c_int),
    "virs_set_sources_audio": ([_P, C.c_uint32, _P, _P, C.c_size_t, C.c_float, C.c_uint64], C.c_int),
    "virs_postprocess_ir": ([_P, C.c_double, _P, C.c_uint32, C.c_int, _P, C.c_uint64, C.POINTER(C.c_uint64)], C.c_int),
    "virs_set_hard_source": ([_P, _P, C.c_size_t], C.c_int),
    "virs_set_sources": ([_P, C.c_uint32, _P, _P, C.c_size_t], C.c_int),
    "virs_set_receivers": ([_P, C.c_uint32, _P], C.c_int),
    "virs_start_simulation": ([_P, C.c_uint64], C.c_int),
    "virs_step": ([_P, C.c_uint32, _P, _P], C.c_int),
    "virs_run": ([_P, C.c_uint64, _P], C.c_int),
    "virs_run_host": ([_P, C.c_uint64, _P, _P, _P], C.c_int),
    "virs_synchronize": ([_P], C.c_int),
    "virs_get_ir": ([_P, C.c_uint64, C.c_uint64, _P], C.c_int),
    "virs_set_stop_rule": ([_P, C.c_int], C.c_int),
    "virs_get_stop": ([_P, C.POINTER(C.c_int), C.POINTER(C.c_uint64)], C.c_int),
    "virs_get_pressure": ([_P, _P, _P, C.c_size_t], C.c_int),
    "virs_set_pressure": ([_P, _P, _P, C.c_size_t], C.c_int),
    "virs_init_pressure_sphere": ([_P, C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.c_float, C.c_int], C.c_int),
    "virs_energy": ([_P, _P], C.c_int),
    "virs_energy_noalloc": ([_P, _P, _P], C.c_int),
    "virs_set_timing": ([_P, C.c_int], C.c_int),
    "virs_get_timing": ([_P, _P], C.c_int),
    "virs_set_tiling": ([_P, C.c_int, C.c_int, C.c_int], C.c_int),
    "virs_set_time_blocking": ([_P, C.c_int, C.c_int, C.c_int], C.c_int),
    "virs_set_rounding": ([_P, C.c_int], C.c_int),
    "virs_postprocess_ir_sinc": ([_P, C.c_double, C.c_uint32, C.c_double, C.c_double, C.c_int, _P, C.c_uint64,
                                  C.POINTER(C.c_uint64)], C.c_int),
    "virs_slab_exchange": ([_P, _P], C.c_int),
    "virs_slab_run": ([_P, C.c_uint32, C.c_uint64], C.c_int),
    "virs_slab_step_begin": ([_P, _P], C.c_int),
    "virs_slab_step_end": ([_P, _P], C.c_int),
    "virs_get_time_blocking": ([_P, _P, _P, _P, _P], C.c_int),
    "virs_check_bounded_wait": ([_P, C.c_uint32], C.c_int),
    "virs_autotune": ([_P, C.c_uint32, _P], C.c_int),
    "virs_forward_checkpointed": ([_P, C.c_uint64, C.c_uint32, _P], C.c_int),
    "virs_adjoint": ([_P, _P, _P, _P], C.c_int),
    "virs_batch_create": ([_P, C.c_uint32, _P], C.c_int),
    "virs_batch_run": ([_P, C.c_uint64, _P], C.c_int),
    "virs_batch_synchronize": ([_P], C.c_int),
    "virs_batch_set_tiling": ([_P, C.c_int, C.c_int, C.c_int], C.c_int),
    "virs_batch_autotune": ([_P, C.c_uint32, _P], C.c_int),
    "virs_batch_destroy": ([_P], C.c_int),
    "virs_get_tiling": ([_P, _P], C.c_int),
}

EXPORTED = tuple(_SIGS)

# cudaStreamLegacy: the stream handle that names CUDA's legacy default stream
_LEGACY_STREAM = 1


def _stream(stream):
    """A cudaStream_t given as an int (torch's `cuda_stream`): None is the
    handle's own stream (NULL to the C API); 0, torch's default stream, is
    CUDA's legacy default stream, passed as cudaStreamLegacy because NULL
    would select the handle's stream."""
    if stream is None:
        return None
    return _LEGACY_STREAM if int(stream) == 0 else int(stream)

_lib = None


def lib() -> C.CDLL:
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m virs_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def last_error() -> str:
    return lib().virs_last_error().decode()


def check(status: int) -> None:
    if status != OK:
        raise VirsError(status, last_error())


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def default_params(**kw) -> Params:
    p = Params()
    check(lib().virs_params_default(C.byref(p)))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise AttributeError(f"no parameter {k}")
        setattr(p, k, v)
    return p


def design_highpass(fs: float, cutoff: float, q: float, gain: float = 1.0) -> np.ndarray:
    out = np.zeros(5, np.float32)
    check(lib().virs_design_highpass(fs, cutoff, q, gain, _ptr(out)))
    return out


def design_lowpass(fs: float, cutoff: float, q: float, gain: float = 1.0) -> np.ndarray:
    out = np.zeros(5, np.float32)
    check(lib().virs_design_lowpass(fs, cutoff, q, gain, _ptr(out)))
    return out


def design_first_order(fs: float, reflection: float, fc: float) -> np.ndarray:
    out = np.zeros(5, np.float64)
    check(lib().virs_design_first_order(fs, reflection, fc, _ptr(out)))
    return out


def design_octave_cascade(fs: float, alpha, freqs=None) -> np.ndarray:
    a = _c(alpha, np.float64)
    f = None if freqs is None else _c(freqs, np.float64)
    out = np.zeros(15, np.float64)
    check(lib().virs_design_octave_cascade(fs, _ptr(a), _ptr(f), _ptr(out)))
    return out.reshape(3, 5)


def design_chebyshev_lowpass(fs: float, fc: float, fstop: float = 0.0, ripple_db: float = 0.5,
                             atten_db: float = 90.0) -> np.ndarray:
    """Chebyshev-I anti-alias low-pass as second-order sections [n][6]
    {b0, b1, b2, a0, a1, a2}."""
    out = np.zeros((32, 6), np.float64)
    n = C.c_uint32(0)
    check(lib().virs_design_chebyshev_lowpass(fs, fc, fstop, ripple_db, atten_db, _ptr(out), 32, C.byref(n)))
    return out[: n.value].copy()


class Simulation:
    """One virs_sim handle."""

    def __init__(self, params: Params | None = None, **kw):
        if params is None:
            params = default_params(**kw)
        self._h = C.c_void_p()
        check(lib().virs_create(C.byref(params), C.byref(self._h)))
        self.params = params

    # lifetime ---------------------------------------------------------------
    def close(self):
        if self._h:
            lib().virs_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # geometry ---------------------------------------------------------------
    def set_material_roles(self, roles):
        r = _c(roles, np.uint8)
        check(lib().virs_set_material_roles(self._h, _ptr(r), r.size))

    def load_obj(self, path):
        check(lib().virs_load_obj(self._h, str(path).encode()))

    def set_mesh(self, verts, tris, tri_material):
        v = _c(verts, np.float32).reshape(-1, 3)
        t = _c(tris, np.uint32).reshape(-1, 3)
        m = _c(tri_material, np.int32)
        check(lib().virs_set_mesh(self._h, _ptr(v), v.shape[0], _ptr(t), _ptr(m), t.shape[0]))

    def set_grid(self, shape, cell_size, flags, wall_material=None):
        nx, ny, nz = shape
        f = _c(flags, np.uint8)
        w = None if wall_material is None else _c(wall_material, np.uint8)
        check(lib().virs_set_grid(self._h, nx, ny, nz, cell_size, _ptr(f), _ptr(w)))

    def set_grid_slab(self, shape, cell_size, z_lo, z_hi, flags, wall_material=None, z_first=0):
        """One z-slab of the grid `shape` owning global planes [z_lo, z_hi);
        flags / wall_material hold global planes z_first.. (their first axis
        is z)."""
        nx, ny, nz = shape
        f = _c(flags, np.uint8).reshape(-1)
        nz_ext = f.size // (nx * ny)
        if nz_ext * nx * ny != f.size:
            raise ValueError("flags must hold whole planes of nx*ny voxels")
        w = None if wall_material is None else _c(wall_material, np.uint8).reshape(-1)
        if w is not None and w.size != f.size:
            raise ValueError("wall_material must match flags")
        check(lib().virs_set_grid_slab(self._h, nx, ny, nz, cell_size, z_lo, z_hi, _ptr(f), _ptr(w), z_first, nz_ext))

    def set_mesh_slab(self, verts, tris, tri_material, part: int, parts: int):
        """Slab `part` of `parts` of the grid sized from the mesh; only its
        planes are voxelised."""
        v = _c(verts, np.float32).reshape(-1, 3)
        t = _c(tris, np.uint32).reshape(-1, 3)
        m = _c(tri_material, np.int32)
        check(lib().virs_set_mesh_slab(self._h, _ptr(v), v.shape[0], _ptr(t), _ptr(m), t.shape[0], part, parts))

    def load_obj_slab(self, path, part: int, parts: int):
        check(lib().virs_load_obj_slab(self._h, str(path).encode(), part, parts))

    def slab_info(self):
        """(z_lo, z_hi, nz): owned global planes and the whole grid's planes."""
        a, b, n = C.c_uint64(), C.c_uint64(), C.c_uint64()
        check(lib().virs_get_slab_info(self._h, C.byref(a), C.byref(b), C.byref(n)))
        return int(a.value), int(b.value), int(n.value)

    def slab_planes(self):
        """(first, last, ghost_lo, ghost_hi, plane_bytes): device addresses of
        the planes of p^n a slab exchanges before its next step."""
        v = [C.c_void_p() for _ in range(4)]
        nb = C.c_size_t()
        check(lib().virs_slab_planes(self._h, *[C.byref(x) for x in v], C.byref(nb)))
        return tuple(int(x.value or 0) for x in v) + (int(nb.value),)

    def info(self) -> GridInfo:
        g = GridInfo()
        check(lib().virs_get_grid_info(self._h, C.byref(g)))
        return g

    @property
    def shape(self):
        g = self.info()
        return (int(g.nx), int(g.ny), int(g.nz))

    @property
    def nvox(self):
        nx, ny, nz = self.shape
        return nx * ny * nz

    def classify(self):
        check(lib().virs_classify(self._h))

    def flags(self) -> np.ndarray:
        out = np.empty(self.nvox, np.uint8)
        check(lib().virs_get_flags(self._h, _ptr(out), out.size))
        return out

    def wall_materials(self) -> np.ndarray:
        out = np.empty(self.nvox, np.uint8)
        check(lib().virs_get_wall_materials(self._h, _ptr(out), out.size))
        return out

    def normals(self) -> np.ndarray:
        out = np.empty(self.nvox, np.uint8)
        check(lib().virs_get_normals(self._h, _ptr(out), out.size))
        return out

    def boundary_indices(self) -> np.ndarray:
        n = int(self.info().boundary_count)
        out = np.empty(max(n, 1), np.uint32)
        check(lib().virs_get_boundary_indices(self._h, _ptr(out), n))
        return out[:n]

    def boundary_materials(self):
        n = int(self.info().boundary_count)
        m = np.empty(max(n, 1), np.uint8)
        w = np.empty(max(n, 1), np.float32)
        check(lib().virs_get_boundary_materials(self._h, _ptr(m), _ptr(w), n))
        return m[:n], w[:n]

    # filters, sources, receivers ------------------------------------------------
    def set_filters(self, coeffs, n_sections=None):
        c = _c(coeffs, np.float32)
        if n_sections is None:
            n_sections = c.shape[-2] if c.ndim == 3 else 1
        c = c.reshape(-1)
        nm = c.size // (5 * n_sections)
        check(lib().virs_set_filters(self._h, nm, n_sections, _ptr(c)))

    def set_hard_source(self, values):
        v = _c(values, np.float32)
        check(lib().virs_set_hard_source(self._h, _ptr(v), v.size))

    def set_sources(self, idx, signal):
        i = _c(np.atleast_1d(idx), np.uint64)
        s = _c(signal, np.float32).reshape(i.size, -1)
        check(lib().virs_set_sources(self._h, i.size, _ptr(i), _ptr(s), s.shape[1]))
        self._nsrc = i.size

    def set_hard_source_audio(self, samples, sample_rate: float, steps: int):
        """Flag-3 voxels driven by an audio signal at its own sample rate."""
        x = _c(samples, np.float32).reshape(-1)
        check(lib().virs_set_hard_source_audio(self._h, _ptr(x), x.size, sample_rate, steps))

    def set_sources_audio(self, idx, samples, sample_rate: float, steps: int):
        """Soft sources driven by audio channels [n][len] at their own sample rate."""
        ix = _c(np.atleast_1d(idx), np.uint64)
        x = _c(samples, np.float32).reshape(ix.size, -1)
        check(lib().virs_set_sources_audio(self._h, ix.size, _ptr(ix), _ptr(x), x.shape[1], sample_rate, steps))
        self._nsrc = ix.size

    def set_receivers(self, idx):
        i = _c(np.atleast_1d(idx), np.uint64)
        check(lib().virs_set_receivers(self._h, i.size, _ptr(i)))
        self._nrcv = i.size

    # running ------------------------------------------------------------------
    def start(self, steps: int):
        check(lib().virs_start_simulation(self._h, steps))

    def step(self, step: int):
        keep = C.c_int(1)
        v = C.c_float(0)
        check(lib().virs_step(self._h, step, C.byref(keep), C.byref(v)))
        return bool(keep.value), float(v.value)

    def run(self, steps: int, stream: int | None = None):
        check(lib().virs_run(self._h, steps, _stream(stream)))

    def slab_step_begin(self, stream: int | None = None):
        """virs_slab_step_begin: the stencil over this slab's interior planes
        (no ghost plane read), on `stream` after the handle's queued work."""
        check(lib().virs_slab_step_begin(self._h, _stream(stream)))

    def slab_step_end(self, stream: int | None = None):
        """virs_slab_step_end: the edge planes, the boundary pass and the
        sources and receivers, once the ghost planes are filled."""
        check(lib().virs_slab_step_end(self._h, _stream(stream)))

    def run_host(self, steps: int, signal=None, ir_out=None, stream: int | None = None):
        s = None if signal is None else _c(signal, np.float32)
        check(lib().virs_run_host(self._h, steps, _ptr(s), _ptr(ir_out), _stream(stream)))

    def run_host_ptr(self, steps: int, signal_ptr, ir_ptr, stream: int | None = None):
        check(lib().virs_run_host(self._h, steps, signal_ptr, ir_ptr, _stream(stream)))

    def synchronize(self):
        check(lib().virs_synchronize(self._h))

    def set_stop_rule(self, enable: bool):
        """The reference's RMS stop rule evaluated on the device in run()."""
        check(lib().virs_set_stop_rule(self._h, int(bool(enable))))

    def stop_state(self):
        """(stopped, stop_step)."""
        a, b = C.c_int(), C.c_uint64()
        check(lib().virs_get_stop(self._h, C.byref(a), C.byref(b)))
        return bool(a.value), int(b.value)

    def ir(self, first: int = 0, steps: int | None = None) -> np.ndarray:
        if steps is None:
            steps = int(self.info().steps_done) - first
        n = getattr(self, "_nrcv", 0)
        out = np.zeros((max(n, 1), steps), np.float32)
        check(lib().virs_get_ir(self._h, first, steps, _ptr(out)))
        return out[:n]

    def postprocess_ir(self, rate: float = 48000.0, sos=None, normalize: bool = True) -> np.ndarray:
        """The receiver traces of the steps run so far, anti-alias filtered
        by `sos` ([n][6], None = no filter), resampled to `rate` and, if
        asked, peak-normalised: [n_receivers][samples]."""
        s6 = None if sos is None else _c(np.asarray(sos, np.float64).reshape(-1, 6), np.float64)
        ns = 0 if s6 is None else s6.shape[0]
        n = C.c_uint64(0)
        check(lib().virs_postprocess_ir(self._h, rate, _ptr(s6), ns, int(normalize), None, 0, C.byref(n)))
        nr = getattr(self, "_nrcv", 0)
        out = np.zeros((max(nr, 1), n.value), np.float32)
        check(lib().virs_postprocess_ir(self._h, rate, _ptr(s6), ns, int(normalize), _ptr(out), out.size, C.byref(n)))
        return out[:nr]

    def postprocess_ir_sinc(self, rate: float = 48000.0, half_taps: int = 245, beta: float = 10.06,
                            cutoff: float = 0.9167, normalize: bool = True) -> np.ndarray:
        """The receiver traces resampled to `rate` by the Kaiser-windowed sinc
        (virs_postprocess_ir_sinc), peak-normalised if asked."""
        n = C.c_uint64(0)
        check(lib().virs_postprocess_ir_sinc(self._h, rate, half_taps, beta, cutoff, int(normalize), None, 0,
                                             C.byref(n)))
        nr = getattr(self, "_nrcv", 0)
        out = np.zeros((max(nr, 1), n.value), np.float32)
        check(lib().virs_postprocess_ir_sinc(self._h, rate, half_taps, beta, cutoff, int(normalize), _ptr(out),
                                             out.size, C.byref(n)))
        return out[:nr]

    def pressure(self, prev: bool = False):
        cur = np.empty(self.nvox, np.float32)
        pp = np.empty(self.nvox, np.float32) if prev else None
        check(lib().virs_get_pressure(self._h, _ptr(cur), _ptr(pp), cur.size))
        return (cur, pp) if prev else cur

    def set_pressure(self, cur, prev=None):
        c = _c(cur, np.float32)
        p = None if prev is None else _c(prev, np.float32)
        check(lib().virs_set_pressure(self._h, _ptr(c), _ptr(p), c.size))

    def init_pressure_sphere(self, x, y, z, radius, pressure, init=True):
        check(lib().virs_init_pressure_sphere(self._h, x, y, z, radius, pressure, int(init)))

    def energy(self) -> float:
        e = C.c_double()
        check(lib().virs_energy(self._h, C.byref(e)))
        return float(e.value)

    def energy_noalloc(self, d_out_ptr: int, stream: int | None = None) -> None:
        """Enqueue the allocation-free energy into the device double at d_out_ptr."""
        check(lib().virs_energy_noalloc(self._h, d_out_ptr, _stream(stream)))

    def set_timing(self, enable: bool):
        check(lib().virs_set_timing(self._h, int(enable)))

    def timing(self) -> Timing:
        t = Timing()
        check(lib().virs_get_timing(self._h, C.byref(t)))
        return t

    def check_bounded_wait(self, limit: int = 1000) -> int:
        """Status of the bounded-wait self test (VIRS_E_TIMEOUT expected)."""
        return int(lib().virs_check_bounded_wait(self._h, limit))

    def forward_checkpointed(self, steps: int, every: int = 64, stream: int | None = None):
        check(lib().virs_forward_checkpointed(self._h, steps, every, _stream(stream)))
        self._adj_steps = steps

    def adjoint(self, dl_dir, n_materials: int, n_sections: int):
        """(dL/dcoef [M][S][5] float64, dL/dsignal [n_src][steps] float32)."""
        steps = self._adj_steps
        dl = _c(dl_dir, np.float32).reshape(-1, steps)
        gc = np.zeros((n_materials, n_sections, 5), np.float64)
        nsrc = getattr(self, "_nsrc", 0)
        gs = np.zeros((max(nsrc, 1), steps), np.float32)
        check(lib().virs_adjoint(self._h, _ptr(dl), _ptr(gc), _ptr(gs)))
        return gc, gs[:nsrc]

    def autotune(self, trial_steps: int = 10) -> Tiling:
        t = Tiling()
        check(lib().virs_autotune(self._h, trial_steps, C.byref(t)))
        return t

    def tiling(self) -> Tiling:
        t = Tiling()
        check(lib().virs_get_tiling(self._h, C.byref(t)))
        return t

    def set_tiling(self, rows: int = 0, planes: int = 0, depth: int = -1):
        check(lib().virs_set_tiling(self._h, rows, planes, depth))

    def set_time_blocking(self, steps_per_pass: int = 2, rows: int = 0, planes: int = 0):
        """Two steps per pass over the fields (bit-identical to single steps)."""
        check(lib().virs_set_time_blocking(self._h, steps_per_pass, rows, planes))

    def set_rounding(self, mode: int) -> None:
        """Rounding of the 16-bit stores: ROUND_NEAREST or ROUND_STOCHASTIC."""
        check(lib().virs_set_rounding(self._h, int(mode)))

    def time_blocking(self) -> dict:
        v = [C.c_int() for _ in range(4)]
        check(lib().virs_get_time_blocking(self._h, *[C.byref(x) for x in v]))
        return {"steps_per_pass": v[0].value, "rows": v[1].value, "planes": v[2].value, "active": bool(v[3].value)}


def slab_exchange(lo: "Simulation", hi: "Simulation") -> None:
    """virs_slab_exchange: adjacent slab handles pull each other's edge plane
    of p^n into their ghost planes, on their own streams."""
    check(lib().virs_slab_exchange(lo.handle, hi.handle))


def slab_run(sims, steps: int) -> None:
    """virs_slab_run: `steps` steps of the slabs sims (in order, covering the
    grid), exchanging ghost planes before every step."""
    arr = (C.c_void_p * len(sims))(*[s.handle.value for s in sims])
    check(lib().virs_slab_run(arr, len(sims), steps))


class Batch:
    """One virs_batch: many Simulations advanced together (3 launches per step)."""

    def __init__(self, sims):
        self.sims = list(sims)                       # keep the members alive
        arr = (C.c_void_p * len(self.sims))(*[s.handle.value for s in self.sims])
        self._h = C.c_void_p()
        check(lib().virs_batch_create(arr, len(self.sims), C.byref(self._h)))

    def run(self, steps: int, stream: int | None = None):
        check(lib().virs_batch_run(self._h, steps, _stream(stream)))

    def synchronize(self):
        check(lib().virs_batch_synchronize(self._h))

    def set_tiling(self, rows: int = 0, planes: int = 0, depth: int = -1):
        check(lib().virs_batch_set_tiling(self._h, rows, planes, depth))

    def autotune(self, trial_steps: int = 4) -> Tiling:
        t = Tiling()
        check(lib().virs_batch_autotune(self._h, trial_steps, C.byref(t)))
        return t

    def close(self):
        if self._h:
            lib().virs_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
