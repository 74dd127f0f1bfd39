"""Host side of the slab-decomposed step, on CPU: the index maps of the two
transposes and the halo routing, and two gloo ranks that transform a field
split into x-slabs (z and y locally, all-to-all, x on the pencils, and back)
and must match the whole field's FFT."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import gs_slab


def test_pack_maps_are_inverse_transposes():
    rng = np.random.default_rng(0)
    R, V, nx, ny, nk = 4, 3, 8, 6, 12
    plan = gs_slab.SlabPlan(nx, ny, nk, V, R)
    slabs = [rng.standard_normal((V, plan.nxl, ny, nk)) for _ in range(R)]
    sends = [gs_slab.pack_by_kz(plan, s) for s in slabs]
    # piece d of rank s's send holds rank d's kz slots of rank s's x-planes
    for s in range(R):
        for d in range(R):
            assert np.array_equal(sends[s][d], slabs[s][..., plan.kz_range(d)])
    recvs = [np.stack([sends[s][d] for s in range(R)]) for d in range(R)]
    pencils = [gs_slab.unpack_pencil(plan, r) for r in recvs]
    whole = np.concatenate(slabs, axis=1)
    for d in range(R):
        assert np.array_equal(pencils[d], whole[..., plan.kz_range(d)])
    back = [gs_slab.pack_by_x(plan, p) for p in pencils]
    recvs2 = [np.stack([back[s][d] for s in range(R)]) for d in range(R)]
    for d in range(R):
        assert np.array_equal(gs_slab.unpack_slab(plan, recvs2[d]), slabs[d])


def test_halo_sources_are_the_periodic_neighbours():
    plan = gs_slab.SlabPlan(8, 4, 4, 1, 4)
    assert plan.halo_sources(0) == ((3, 1), (1, 0))
    assert plan.halo_sources(3) == ((2, 1), (0, 0))
    one = gs_slab.SlabPlan(8, 4, 4, 1, 1)
    assert one.halo_sources(0) == ((0, 1), (0, 0))


def test_plan_rejects_uneven_splits():
    with pytest.raises(ValueError):
        gs_slab.SlabPlan(10, 4, 8, 1, 4)
    with pytest.raises(ValueError):
        gs_slab.SlabPlan(8, 4, 6, 1, 4)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        V, nx, ny, nz = 2, 8, 6, 12
        rng = np.random.default_rng(42)  # the same whole field on every rank
        field = rng.standard_normal((V, nx, ny, nz)) + 1j * rng.standard_normal((V, nx, ny, nz))
        plan = gs_slab.SlabPlan(nx, ny, nz, V, world)
        mine = field[:, plan.x_range(rank)]
        spec = np.fft.fft(np.fft.fft(mine, axis=3), axis=2)  # z and y on the slab
        ex = gs_slab.DistExchange(0)

        def a2a(arr):
            send = torch.from_numpy(np.ascontiguousarray(arr)).view(torch.float64).reshape(-1)
            recv = torch.empty_like(send)
            ex.all_to_all(recv, send)
            return recv.numpy().view(np.complex128).reshape(arr.shape)

        pencil = gs_slab.unpack_pencil(plan, a2a(gs_slab.pack_by_kz(plan, spec)))
        pencil = np.fft.fft(pencil, axis=1)  # x on the pencils
        whole = np.fft.fftn(field, axes=(1, 2, 3))
        err1 = np.abs(pencil - whole[..., plan.kz_range(rank)]).max()
        back = gs_slab.unpack_slab(plan, a2a(gs_slab.pack_by_x(plan, pencil)))
        err2 = np.abs(back - whole[:, plan.x_range(rank)]).max()
        # the halo exchange: this rank's face planes, tagged by rank
        face = np.stack([np.full((V, ny, nz), 10.0 * rank + 0), np.full((V, ny, nz), 10.0 * rank + 1)])
        hs = torch.from_numpy(face.reshape(-1).copy())
        hr = torch.empty_like(hs)
        ex.halo(hr, hs, plan)
        lo, hi = hr.numpy().reshape(2, V, ny, nz)[:, 0, 0, 0]
        out.put((rank, err1, err2, lo, hi))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2])
def test_two_gloo_ranks_transform_a_split_field(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, err1, err2, lo, hi in res:
        assert err1 < 1e-10 and err2 < 1e-10
        # below: the last plane of rank - 1; above: the first plane of rank + 1
        assert lo == 10.0 * ((rank - 1) % world) + 1
        assert hi == 10.0 * ((rank + 1) % world) + 0
