"""Z-slab split of one grid over ranks: the split, the halo plan and exchange (NumPy emulation
and gloo ranks on CPU, checked against the oracle on the whole grid), and on one GPU the slab
kernel itself (one rank, and several slabs emulated in one process) against the whole-grid
z-march."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from oracle.stencil import reference_step
from pyheat3d_b200.contract import heat_stencil
from pyheat3d_b200.slab import SlabSplit


# ------------------------------------------------------------------------------ split logic
@pytest.mark.parametrize("nz,world", [(3, 1), (17, 4), (16, 4), (9, 9), (128, 3)])
def test_bounds_cover_every_plane_once(nz, world):
    for periodic in (False, True):
        sp = SlabSplit(nz, world, periodic)
        owned = [z for r in range(world) for z in range(*sp.bounds(r))]
        assert owned == list(range(nz))
        sizes = [sp.planes(r) for r in range(world)]
        assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1


def test_split_rejects_bad_sizes():
    with pytest.raises(ValueError):
        SlabSplit(4, 5, True)
    with pytest.raises(ValueError):
        SlabSplit(2, 1, True)
    with pytest.raises(ValueError):
        SlabSplit(8, 0, True)
    with pytest.raises(ValueError):
        SlabSplit(8, 2, True).bounds(2)


def test_update_range_keeps_dirichlet_ends_fixed():
    sp = SlabSplit(10, 3, False)  # planes 4 / 3 / 3
    assert [sp.update_range(r) for r in range(3)] == [(2, 5), (1, 4), (1, 3)]
    sp = SlabSplit(10, 3, True)
    assert [sp.update_range(r) for r in range(3)] == [(1, 5), (1, 4), (1, 4)]
    # a one-plane Dirichlet end slab updates nothing
    sp = SlabSplit(3, 3, False)
    assert [sp.update_range(r) for r in range(3)] == [(2, 2), (1, 2), (1, 1)]


def _emulate_exchange(bufs, sp):
    """Deliver every rank's halo plan in one process: each rank's sends to a peer, in posting
    order, pair with that peer's receives from it, in posting order."""
    world = sp.world
    if world == 1:
        if sp.periodic:
            n = sp.planes(0)
            bufs[0][0] = bufs[0][n]
            bufs[0][n + 1] = bufs[0][1]
        return
    sends = {(r, p): [] for r in range(world) for p in range(world)}
    recvs = {(r, p): [] for r in range(world) for p in range(world)}
    for r in range(world):
        for kind, peer, plane in sp.halo_plan(r):
            (sends if kind == "send" else recvs)[(r, peer)].append(plane)
    for (r, p), planes in sends.items():
        want = recvs[(p, r)]
        assert len(planes) == len(want), (r, p)
        msgs = [bufs[r][z].copy() for z in planes]
        for z, m in zip(want, msgs):
            bufs[p][z] = m


def _oracle_slab_step(buf, sp, rank, c0, c1):
    z0, z1 = sp.update_range(rank)
    new = reference_step(buf, c0, c1, "periodic" if sp.periodic else "dirichlet")
    out = buf.copy()
    out[z0:z1] = new[z0:z1]
    return out


@pytest.mark.parametrize("periodic", [False, True])
@pytest.mark.parametrize("world,nz", [(1, 9), (2, 9), (3, 10), (5, 13)])
def test_split_steps_equal_whole_grid_oracle(periodic, world, nz):
    """Slabs with emulated exchanges reproduce the whole-grid oracle bit for bit."""
    bc = "periodic" if periodic else "dirichlet"
    st = heat_stencil(3, 0.95 / 6, bc)
    c0, c1 = np.float32(st.c0), np.float32(st.c1)
    u = np.random.default_rng(3).random((nz, 7, 11), dtype=np.float32)
    sp = SlabSplit(nz, world, periodic)
    bufs = [sp.slab_of(u, r) for r in range(world)]
    want = u.copy()
    for _ in range(6):
        _emulate_exchange(bufs, sp)
        bufs = [_oracle_slab_step(bufs[r], sp, r, c0, c1) for r in range(world)]
        want = reference_step(want, c0, c1, bc)
    got = np.concatenate([b[1:-1] for b in bufs], axis=0)
    assert np.array_equal(got, want)


def test_halo_plan_pairs_two_rank_ring():
    sp = SlabSplit(8, 2, True)
    assert sp.halo_plan(0) == [("send", 1, 1), ("send", 1, 4), ("recv", 1, 5), ("recv", 1, 0)]
    assert SlabSplit(8, 2, False).halo_plan(0) == [("send", 1, 4), ("recv", 1, 5)]
    assert SlabSplit(8, 2, False).halo_plan(1) == [("send", 0, 1), ("recv", 0, 0)]


# ------------------------------------------------------------------------ gloo ranks on CPU
def _gloo_rank(rank, world, port, periodic, out):
    import torch
    import torch.distributed as dist

    from pyheat3d_b200.slab import exchange_halos, gather_planes

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bc = "periodic" if periodic else "dirichlet"
        st = heat_stencil(3, 0.15, bc)
        c0, c1 = np.float32(st.c0), np.float32(st.c1)
        u = np.random.default_rng(5).random((11, 6, 9), dtype=np.float32)
        sp = SlabSplit(11, world, periodic)
        buf = torch.from_numpy(sp.slab_of(u, rank))
        for _ in range(5):
            exchange_halos(buf, sp, rank)
            buf = torch.from_numpy(_oracle_slab_step(buf.numpy(), sp, rank, c0, c1))
        g = gather_planes(buf[1:-1].contiguous(), sp, rank)
        if rank == 0:
            want = u.copy()
            for _ in range(5):
                want = reference_step(want, c0, c1, bc)
            out.put(bool(np.array_equal(g, want)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("periodic", [False, True])
def test_exchange_over_gloo_ranks(world, periodic):
    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_rank, args=(r, world, port, periodic, q))
             for r in range(world)]
    for p in procs:
        p.start()
    ok = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert ok


def test_planes_entry_point_rejects_bad_ranges():
    from pyheat3d_b200 import _lib

    L = _lib.lib()
    # argument checks run before any device work (no GPU needed)
    for z0, z1 in ((0, 3), (2, 8), (3, 2)):
        rc = L.ph3_zmarch3d_planes(1, 2, None, 8, 8, 8, z0, z1, 0.1, 0.1, 0, 1, 0, None)
        assert rc == 1 and "planes" in _lib.last_error(), (z0, z1)  # PH3_EINVAL


# ------------------------------------------------------------------------------------- GPU
def _whole_grid(u, st, steps, storage):
    import torch

    from pyheat3d_b200 import _lib

    L = _lib.lib()
    dt = getattr(torch, storage)
    a = torch.from_numpy(u).cuda().to(dt)
    b = a.clone()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(steps):
        _lib.check(L.ph3_zmarch3d(a.data_ptr(), b.data_ptr(), None, *u.shape,
                                  float(np.float32(st.c0)), float(np.float32(st.c1)),
                                  _lib.STORAGE[storage], _lib.BC[st.bc], 0, stream))
        a, b = b, a
    return a.float().cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("storage", ["float32", "bfloat16"])
@pytest.mark.parametrize("bc", ["periodic", "dirichlet"])
def test_gpu_one_rank_equals_whole_grid(storage, bc):
    """A split over one rank (periodic halos by local copies) equals the whole-grid z-march."""
    from pyheat3d_b200.slab import SlabStepper

    st = heat_stencil(3, 0.95 / 6, bc)
    u = np.random.default_rng(8).random((40, 36, 72), dtype=np.float32)
    sp = SlabSplit(40, 1, bc == "periodic")
    s = SlabStepper(sp.slab_of(u, 0), st, sp, 0, storage=storage)
    s.step(7)
    assert np.array_equal(s.get(), _whole_grid(u, st, 7, storage))


@pytest.mark.gpu
@pytest.mark.parametrize("bc", ["periodic", "dirichlet"])
@pytest.mark.parametrize("shape", [(37, 24, 64), (29, 20, 37)])
def test_gpu_emulated_slabs_equal_whole_grid(bc, shape):
    """Several slabs on one GPU, halos delivered by plane copies in the order of the halo plan,
    each slab advanced by the z-range kernel (TMA for aligned rows, the lean march for nx = 37),
    on odd steps in the three launches of the overlapped step (halo-free planes, then the first
    and last plane): bit-identical to the whole-grid z-march."""
    import torch

    from pyheat3d_b200.slab import SlabStepper

    st = heat_stencil(3, 0.95 / 6, bc)
    u = np.random.default_rng(9).random(shape, dtype=np.float32)
    world = 4
    sp = SlabSplit(shape[0], world, bc == "periodic")
    ranks = [SlabStepper(sp.slab_of(u, r), st, sp, r, overlap=False) for r in range(world)]
    for step in range(6):
        host = [s.a.cpu().numpy() for s in ranks]
        _emulate_exchange(host, sp)
        for s, h in zip(ranks, host):
            s.a.copy_(torch.from_numpy(h))
        for s in ranks:
            stream = torch.cuda.current_stream().cuda_stream
            if step % 2 and s.z1 - s.z0 >= 3:
                s._planes(s.z0 + 1, s.z1 - 1, stream)
                s._planes(s.z0, s.z0 + 1, stream)
                s._planes(s.z1 - 1, s.z1, stream)
            else:
                s._planes(s.z0, s.z1, stream)
            s.a, s.b = s.b, s.a
    got = np.concatenate([s.get() for s in ranks], axis=0)
    assert np.array_equal(got, _whole_grid(u, st, 6, "float32"))


@pytest.mark.gpu
def test_gpu_planes_kernel_leaves_other_planes_untouched():
    import torch

    from pyheat3d_b200 import _lib

    L = _lib.lib()
    u = torch.rand((12, 16, 64), device="cuda")
    out = torch.full_like(u, -1.0)
    stream = torch.cuda.current_stream().cuda_stream
    _lib.check(L.ph3_zmarch3d_planes(u.data_ptr(), out.data_ptr(), None, 12, 16, 64, 3, 7,
                                     0.05, 0.95 / 6, 0, 1, 0, stream))
    o = out.cpu().numpy()
    assert (o[:3] == -1).all() and (o[7:] == -1).all()
    st = heat_stencil(3, 0.95 / 6, "periodic")
    # the planes 3..6 of a periodic x / y update, z neighbours from the array (no wrap)
    full = reference_step(u.cpu().numpy(), np.float32(st.c0), np.float32(st.c1), "periodic")
    assert np.array_equal(o[3:7], full[3:7])
