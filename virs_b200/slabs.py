"""z-slabs: one grid split along z over several GPUs, one process per GPU.

The step is a 7-point stencil, so a split along z needs one exchange per
step: every slab sends its first and last owned planes of p^n to the slabs
below and above and receives theirs into its two ghost planes
(`virs_set_grid_slab`, `virs_slab_planes` in include/virs.h).  Boundary
lists, filter states, sources and receivers partition with their voxels;
nothing else crosses between slabs.  The reference runs one grid on one GPU
(src/simulator/simulator_gpu.cu:184-332); with the ghost planes exchanged
before every step the slabs advance exactly as that grid.

Exchanges go through torch.distributed point-to-point operations
(`batch_isend_irecv`): NCCL over NVLink between GPUs, gloo between CPU
processes.  The planes are plain device buffers of the library, wrapped as
uint8 tensors without copies.
"""
from __future__ import annotations

import numpy as np


def split_planes(nz: int, parts: int) -> list[tuple[int, int]]:
    """The interior planes 1 .. nz-2 of a grid split into `parts` contiguous
    ranges [z_lo, z_hi) of sizes differing by at most one."""
    inner = nz - 2
    if parts < 1 or inner < parts:
        raise ValueError(f"cannot split {inner} interior planes into {parts} slabs")
    base, extra = divmod(inner, parts)
    out, z = [], 1
    for r in range(parts):
        n = base + (1 if r < extra else 0)
        out.append((z, z + n))
        z += n
    return out


def flag_range(nz: int, z_lo: int, z_hi: int, sponge_width: int) -> tuple[int, int]:
    """(z_first, nz_ext): the global planes of flags a slab owning
    [z_lo, z_hi) needs: its ghost planes and sponge_width + 1 planes beyond,
    for the classification of its planes."""
    h = sponge_width + 1
    lo = max(0, z_lo - 1 - h)
    hi = min(nz, z_hi + 1 + h)
    return lo, hi - lo


def local_index(idx, shape, z_lo: int, z_hi: int):
    """Global voxel indices -> (mask of those owned by the slab [z_lo, z_hi),
    their indices in the slab's own grid, whose plane 0 is z_lo - 1)."""
    nx, ny, _ = shape
    idx = np.asarray(idx, np.uint64).reshape(-1)
    z = idx // np.uint64(nx * ny)
    own = (z >= z_lo) & (z < z_hi)
    loc = idx[own] - np.uint64((z_lo - 1) * nx * ny)
    return own, loc


class _DeviceBytes:
    """`n` bytes of device memory at `ptr`, for torch.as_tensor."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False), "version": 3,
                                         "strides": None}


def device_bytes(ptr: int, n: int, device: int | None = None):
    """A uint8 CUDA tensor viewing `n` bytes at device address `ptr` on GPU
    `device` (None = the current one).  The view aliases the memory: a copy
    into it writes `ptr` (torch would otherwise copy a buffer of another GPU
    to the current one, and a write would go to that copy)."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else int(device))
    with torch.cuda.device(dev):
        t = torch.as_tensor(_DeviceBytes(ptr, n), device=dev)
    if t.data_ptr() != ptr:
        raise RuntimeError(f"device_bytes: the view of {ptr:#x} on {dev} does not alias it")
    return t


def exchange(first, last, ghost_lo, ghost_hi, rank: int, world: int, group=None) -> None:
    """One halo exchange between neighbouring slabs: `first` goes to rank-1
    (into its `ghost_hi`), `last` to rank+1 (into its `ghost_lo`); this rank's
    ghost planes are filled from theirs.  All ranks call it at every step;
    the end ranks have one neighbour.  Tensors may be CPU (gloo) or CUDA
    (NCCL); the call returns when the receives are complete (on the current
    stream for NCCL)."""
    import torch.distributed as dist
    ops = []
    if rank > 0:
        ops.append(dist.P2POp(dist.isend, first, rank - 1, group))
        ops.append(dist.P2POp(dist.irecv, ghost_lo, rank - 1, group))
    if rank < world - 1:
        ops.append(dist.P2POp(dist.isend, last, rank + 1, group))
        ops.append(dist.P2POp(dist.irecv, ghost_hi, rank + 1, group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


def exchange_local(sims) -> None:
    """The same exchange between slab handles of one process, as copies on
    the current torch stream: sims[r] owns the r-th range from the bottom.
    Each plane is viewed on its own handle's GPU, so handles may sit on
    different GPUs (a copy between two GPUs is a peer copy)."""
    planes = [s.slab_planes() for s in sims]
    dev = [int(s.params.device) for s in sims]
    for r in range(len(sims)):
        nb = planes[r][4]
        if r > 0:
            device_bytes(planes[r][2], nb, dev[r]).copy_(device_bytes(planes[r - 1][1], planes[r - 1][4], dev[r - 1]))
        if r + 1 < len(sims):
            device_bytes(planes[r][3], nb, dev[r]).copy_(device_bytes(planes[r + 1][0], planes[r + 1][4], dev[r + 1]))


class SlabRun:
    """Drives one slab of a distributed grid.  Per step: the stencil over
    the slab's interior planes (virs_slab_step_begin) on a side stream,
    meanwhile the halo exchange with the neighbouring ranks on the current
    torch stream, then, after both, the edge planes, the boundary pass and
    the sources and receivers (virs_slab_step_end) on the current stream.
    The interior launch reads no ghost plane and the exchange sends planes
    of p^n that no kernel of the step writes, so the two run side by side.

    `sim` is a capi.Simulation set up with `setup_slab`, classified,
    configured and started; every rank runs the same number of steps."""

    def __init__(self, sim, rank: int, world: int, group=None):
        self.sim, self.rank, self.world, self.group = sim, rank, world, group
        self._side = None

    def run(self, steps: int) -> None:
        import torch
        d = int(self.sim.params.device)
        if self._side is None:
            self._side = torch.cuda.Stream(device=d)
        main = torch.cuda.current_stream(d)
        for _ in range(steps):
            first, last, glo, ghi, nb = self.sim.slab_planes()
            self._side.wait_stream(main)
            self.sim.slab_step_begin(self._side.cuda_stream)
            exchange(device_bytes(first, nb, d), device_bytes(last, nb, d), device_bytes(glo, nb, d),
                     device_bytes(ghi, nb, d), self.rank, self.world, self.group)
            main.wait_stream(self._side)
            self.sim.slab_step_end(main.cuda_stream)


def setup_slab(sim, shape, cell_size: float, flags, wall_material, rank: int, world: int, sponge_width: int):
    """Install this rank's slab of the global grid `shape` from the global
    flags / wall materials ([nz][ny][nx] or flat, host arrays); returns its
    owned planes (z_lo, z_hi)."""
    nx, ny, nz = shape
    z_lo, z_hi = split_planes(nz, world)[rank]
    z_first, n_ext = flag_range(nz, z_lo, z_hi, sponge_width)
    plane = nx * ny
    f = np.ascontiguousarray(flags, np.uint8).reshape(-1)[z_first * plane:(z_first + n_ext) * plane]
    w = None
    if wall_material is not None:
        w = np.ascontiguousarray(wall_material, np.uint8).reshape(-1)[z_first * plane:(z_first + n_ext) * plane]
    sim.set_grid_slab(shape, cell_size, z_lo, z_hi, f, w, z_first)
    return z_lo, z_hi
