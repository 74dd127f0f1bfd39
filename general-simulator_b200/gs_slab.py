"""A martensite simulation split into x-slabs across devices (gs_slab_*).

The reference holds one grid on one device (src/dynamics_mart.cu:113-117: one
cuFFT plan over the whole grid), which bounds the grid by one GPU's memory.
Here rank r of R owns the x-planes [r nx/R, (r+1) nx/R) of every variant.  A
step is three local phases of the library (gs_slab_begin / _xpass / _end)
with two all-to-all transposes and one halo exchange between them:

  begin  z and y transforms of the slab; spectra packed by destination kz
         range, send = [R][V][nx/R][ny][h/R] complex (h = nz/2); the slab's
         first and last x-plane, halo_send = [2][V][ny][nz]
  a2a    piece s of send goes to rank s
  xpass  pieces unpacked into x-pencils [V][nx][ny][h/R], x transforms and
         the B contraction, packed back by destination x range
  a2a    again
  end    y inverse, the update with the neighbours' face planes, the next
         step's z transform

The exchanges belong to the caller: `DistExchange` runs them over a
torch.distributed process group (NCCL between GPUs, gloo on CPU), and
`LocalExchange` with device copies when all slabs live on one device (the
GPU tests; no kernel waits on another).  The index maps of the packing are
restated here in numpy (`pack_by_kz`, `unpack_pencil`, `pack_by_x`,
`unpack_slab`) for the host-side tests of the decomposition.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

import gs_b200 as gb


# ---------------------------------------------------------------------------
# geometry and the index maps of the transposes (numpy restatement)
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class SlabPlan:
    nx: int
    ny: int
    nkz: int      # kz slots of the spectra being transposed (h = nz/2 for the packed layout)
    nfields: int  # V
    nranks: int

    def __post_init__(self):
        if self.nranks < 1 or self.nx % self.nranks or self.nkz % self.nranks:
            raise ValueError(f"nx {self.nx} and the kz slots {self.nkz} must be multiples of {self.nranks} ranks")

    @property
    def nxl(self) -> int:
        return self.nx // self.nranks

    @property
    def nkzl(self) -> int:
        return self.nkz // self.nranks

    def x_range(self, r: int) -> range:
        return range(r * self.nxl, (r + 1) * self.nxl)

    def kz_range(self, r: int) -> range:
        return range(r * self.nkzl, (r + 1) * self.nkzl)

    def halo_sources(self, r: int):
        """(rank, plane) that fill this rank's halo planes: below = the last
        plane of rank r-1, above = the first plane of rank r+1 (periodic)."""
        R = self.nranks
        return ((r - 1) % R, 1), ((r + 1) % R, 0)


def pack_by_kz(plan: SlabPlan, spec: np.ndarray) -> np.ndarray:
    """Slab spectra [V][nx/R][ny][nkz] -> send [R][V][nx/R][ny][nkz/R]:
    piece d holds the kz slots of rank d."""
    V, xl, ny, nk = spec.shape
    return spec.reshape(V, xl, ny, plan.nranks, plan.nkzl).transpose(3, 0, 1, 2, 4).copy()


def unpack_pencil(plan: SlabPlan, recv: np.ndarray) -> np.ndarray:
    """Received pieces [R(source)][V][nx/R][ny][nkz/R] -> x-pencils
    [V][nx][ny][nkz/R], source s filling x = s nx/R .. (s+1) nx/R - 1."""
    R, V, xl, ny, kl = recv.shape
    return recv.transpose(1, 0, 2, 3, 4).reshape(V, R * xl, ny, kl).copy()


def pack_by_x(plan: SlabPlan, pencil: np.ndarray) -> np.ndarray:
    """x-pencils [V][nx][ny][nkz/R] -> send [R][V][nx/R][ny][nkz/R]: piece d
    holds the x range of rank d."""
    V, nx, ny, kl = pencil.shape
    return pencil.reshape(V, plan.nranks, plan.nxl, ny, kl).transpose(1, 0, 2, 3, 4).copy()


def unpack_slab(plan: SlabPlan, recv: np.ndarray) -> np.ndarray:
    """Received pieces [R(source)][V][nx/R][ny][nkz/R] -> slab spectra
    [V][nx/R][ny][nkz], source s filling kz = s nkz/R .. (s+1) nkz/R - 1."""
    R, V, xl, ny, kl = recv.shape
    return recv.transpose(1, 2, 3, 0, 4).reshape(V, xl, ny, R * kl).copy()


# ---------------------------------------------------------------------------
# exchanges
# ---------------------------------------------------------------------------
class DistExchange:
    """The transposes and the halo exchange over the default torch.distributed
    process group (every rank calls each method in the same order)."""

    def __init__(self, plan_halo_bytes: int):
        import torch.distributed as dist

        self.dist = dist
        self.R = dist.get_world_size()
        self.rank = dist.get_rank()

    def all_to_all(self, recv, send) -> None:
        self.dist.all_to_all_single(recv, send)

    def halo(self, halo_recv, halo_send, plan: SlabPlan) -> None:
        import torch

        n = halo_send.numel()
        gathered = torch.empty(self.R * n, dtype=halo_send.dtype, device=halo_send.device)
        self.dist.all_gather_into_tensor(gathered, halo_send.reshape(-1))
        (lo_r, lo_p), (hi_r, hi_p) = plan.halo_sources(self.rank)
        half = n // 2
        halo_recv.view(-1)[:half].copy_(gathered[lo_r * n + lo_p * half:lo_r * n + (lo_p + 1) * half])
        halo_recv.view(-1)[half:].copy_(gathered[hi_r * n + hi_p * half:hi_r * n + (hi_p + 1) * half])


class LocalExchange:
    """All R slabs in one process on one device: the exchanges are copies of
    the pieces between the slabs' device buffers."""

    @staticmethod
    def all_to_all(recvs, sends) -> None:
        R = len(sends)
        for d in range(R):
            for s in range(R):
                n = sends[s].numel() // R
                recvs[d].view(-1)[s * n:(s + 1) * n].copy_(sends[s].view(-1)[d * n:(d + 1) * n])

    @staticmethod
    def halo(halo_recvs, halo_sends, plan: SlabPlan) -> None:
        for r in range(plan.nranks):
            (lo_r, lo_p), (hi_r, hi_p) = plan.halo_sources(r)
            half = halo_sends[r].numel() // 2
            halo_recvs[r].view(-1)[:half].copy_(halo_sends[lo_r].view(-1)[lo_p * half:(lo_p + 1) * half])
            halo_recvs[r].view(-1)[half:].copy_(halo_sends[hi_r].view(-1)[hi_p * half:(hi_p + 1) * half])


# ---------------------------------------------------------------------------
# one rank's slab on its device
# ---------------------------------------------------------------------------
class Slab:
    def __init__(self, params: gb.GsParams, rank: int, nranks: int, device=None):
        import torch

        self.params = params.copy()
        h = C.c_void_p()
        gb.check(gb.lib().gs_slab_create(C.byref(self.params), rank, nranks, C.byref(h)), "gs_slab_create")
        self.h = h
        g = gb.GsSlabGeometry()
        gb.check(gb.lib().gs_slab_info(self.h, C.byref(g)), "gs_slab_info")
        self.geom = g
        p = self.params
        self.plan = SlabPlan(p.nx, p.ny, p.nz // 2, p.nvariants, nranks)
        dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        # byte buffers of the exchanges (torch's allocator: 512-byte aligned)
        mk = lambda n: torch.empty(n, dtype=torch.uint8, device=dev)  # noqa: E731
        self.send, self.recv = mk(g.a2a_bytes), mk(g.a2a_bytes)
        self.halo_send, self.halo_recv = mk(g.halo_bytes), mk(g.halo_bytes)

    def close(self) -> None:
        if self.h:
            gb.lib().gs_slab_destroy(self.h)
            self.h = C.c_void_p()

    @property
    def local_shape(self):
        p = self.params
        return (p.nvariants, self.geom.nx_local, p.ny, p.nz)

    def set_eta(self, eta_local: np.ndarray) -> None:
        a = np.ascontiguousarray(eta_local)
        code = gb.GS_DTYPE_F64 if a.dtype == np.float64 else gb.GS_DTYPE_F32
        a = np.ascontiguousarray(a, dtype=np.float64 if code == gb.GS_DTYPE_F64 else np.float32)
        gb.check(gb.lib().gs_slab_set_field(self.h, b"eta", a.ctypes.data, a.size, code), "gs_slab_set_field")

    def eta(self, dtype=np.float64) -> np.ndarray:
        out = np.empty(self.local_shape, dtype=dtype)
        code = gb.GS_DTYPE_F64 if dtype == np.float64 else gb.GS_DTYPE_F32
        gb.check(gb.lib().gs_slab_get_field(self.h, b"eta", out.ctypes.data, out.size, code), "gs_slab_get_field")
        return out

    def set_step(self, step: int) -> None:
        gb.check(gb.lib().gs_slab_set_step(self.h, step), "gs_slab_set_step")

    def begin(self, stream: int = 0) -> None:
        gb.check(gb.lib().gs_slab_begin(self.h, self.send.data_ptr(), self.halo_send.data_ptr(), C.c_void_p(stream)),
                 "gs_slab_begin")

    def xpass(self, stream: int = 0) -> None:
        gb.check(gb.lib().gs_slab_xpass(self.h, self.recv.data_ptr(), self.send.data_ptr(), C.c_void_p(stream)),
                 "gs_slab_xpass")

    def end(self, stream: int = 0) -> None:
        gb.check(gb.lib().gs_slab_end(self.h, self.recv.data_ptr(), self.halo_recv.data_ptr(), C.c_void_p(stream)),
                 "gs_slab_end")


def _current_stream(stream: int) -> int:
    """The stream the phases run on: the caller's, else torch's current one,
    which the exchanges (torch copies, collectives) are ordered on too."""
    if stream:
        return stream
    import torch

    return torch.cuda.current_stream().cuda_stream


def step_local(slabs: List[Slab], nsteps: int, stream: int = 0) -> None:
    """Advance R slabs that share this process's device by nsteps."""
    plan = slabs[0].plan
    stream = _current_stream(stream)
    for _ in range(nsteps):
        for s in slabs:
            s.begin(stream)
        LocalExchange.all_to_all([s.recv for s in slabs], [s.send for s in slabs])
        LocalExchange.halo([s.halo_recv for s in slabs], [s.halo_send for s in slabs], plan)
        for s in slabs:
            s.xpass(stream)
        LocalExchange.all_to_all([s.recv for s in slabs], [s.send for s in slabs])
        for s in slabs:
            s.end(stream)


def step_dist(slab: Slab, nsteps: int, exchange: Optional[DistExchange] = None, stream: int = 0) -> None:
    """Advance this rank's slab by nsteps over the default process group
    (every rank calls this with the same nsteps)."""
    ex = exchange or DistExchange(slab.geom.halo_bytes)
    stream = _current_stream(stream)
    for _ in range(nsteps):
        slab.begin(stream)
        ex.all_to_all(slab.recv, slab.send)
        ex.halo(slab.halo_recv, slab.halo_send, slab.plan)
        slab.xpass(stream)
        ex.all_to_all(slab.recv, slab.send)
        slab.end(stream)


def run_local(params: gb.GsParams, eta0: np.ndarray, nsteps: int, nranks: int) -> np.ndarray:
    """The whole field after nsteps, computed by nranks slabs on this device
    (eta0: [V][nx][ny][nz])."""
    slabs = [Slab(params, r, nranks) for r in range(nranks)]
    try:
        for r, s in enumerate(slabs):
            s.set_eta(eta0[:, s.plan.x_range(r)])
        import torch

        torch.cuda.synchronize()
        step_local(slabs, nsteps)
        torch.cuda.synchronize()
        return np.concatenate([s.eta(np.float64) for s in slabs], axis=1)
    finally:
        for s in slabs:
            s.close()
