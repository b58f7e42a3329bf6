"""Host side of the z-slab split of one 3D run (opticrcwafdtd_b200.slab3d):
slab planes, the slabs' sims, the put-together out struct, the halo swap
between ranks and the ranks' sim check, on CPU (gloo ranks)."""
import os

import numpy as np
import pytest

from opticrcwafdtd_b200 import slab3d
from opticrcwafdtd_b200._abi import OrfError


def test_split_z_cuts_and_ghosts():
    s = slab3d.split_z(300, 2, 20)
    assert [(q.z0, q.z1, q.lo, q.hi) for q in s] == [(0, 150, 0, 151), (150, 300, 149, 300)]
    s3 = slab3d.split_z(300, 3, 20)
    assert [(q.z0, q.z1) for q in s3] == [(0, 100), (100, 200), (200, 300)]
    assert s3[1].has_below and s3[1].has_above and s3[1].n == 102
    assert not s3[0].has_below and not s3[2].has_above
    one = slab3d.split_z(50, 1, 7)
    assert [(q.lo, q.hi) for q in one] == [(0, 50)]
    # own planes cover the grid once, in order
    for n in (36, 61, 300):
        for k in (1, 2, 3):
            try:
                sl = slab3d.split_z(n, k, 7)
            except OrfError:
                continue
            own = np.concatenate([np.arange(q.z0, q.z1) for q in sl])
            assert np.array_equal(own, np.arange(n))


def test_split_z_refuses_cuts_in_the_cpml():
    with pytest.raises(OrfError, match="CPML"):
        slab3d.split_z(40, 4, 7)          # cut at 10: in reach of the 7-plane layer
    with pytest.raises(OrfError, match="fewer than"):
        slab3d.split_z(56, 4, 7)          # 14-plane slabs: under 2*7+2 planes with their ghosts
    with pytest.raises(OrfError):
        slab3d.split_z(60, 0, 7)


def _sim(n=(10, 8, 40), src_axis=3, src_index=12):
    rng = np.random.default_rng(1)
    d = 0.04
    x, y, z = (np.arange(m) * d for m in n)
    eps = {c: 1.0 + rng.random(n) for c in "xyz"}
    a, b = n[src_axis % 3], n[(src_axis + 1) % 3]
    prof = rng.random((a, b))
    src = dict(axis=src_axis, index=src_index, Ea=prof, Eb=2 * prof, Ha=3 * prof, Hb=4 * prof, neff=1.0,
               lambda0=0.6, bw=0.3)
    mons = [dict(axis=3, index=5), dict(axis=1, index=4), dict(axis=3, index=30), dict(axis=2, index=3)]
    return dict(x=x, y=y, z=z, eps=eps, npml=[3, 3, 5], periodic=[False, False, False], source=src,
                monitors=mons, lambdas=[0.5, 0.6], maxTime=1.0, shutoff=0.0, precision="double")


def test_slab_sim_slices_planes_source_and_monitors():
    sim = _sim()
    sl = slab3d.split_z(40, 2, 5)
    s0, s1 = (slab3d.slab_sim(sim, q) for q in sl)
    assert np.array_equal(s0["z"], sim["z"][0:21]) and np.array_equal(s1["z"], sim["z"][19:40])
    for c in "xyz":
        assert np.array_equal(s0["eps"][c], sim["eps"][c][:, :, 0:21])
        assert np.array_equal(s1["eps"][c], sim["eps"][c][:, :, 19:40])
    # z-normal source (1-based 12 -> plane 11): slab 0 keeps it, slab 1 gets
    # a zero source on an own plane outside the CPML
    assert s0["source"]["index"] == 12 and s0["source"]["Ea"] is sim["source"]["Ea"]
    assert s1["source"]["Ea"] == 0.0 and s1["source"]["Hb"] == 0.0
    g1 = s1["source"]["index"] - 1 + sl[1].lo
    assert sl[1].z0 <= g1 < sl[1].z1 and 5 <= g1 < 35
    # z-normal monitors only on the owner, in local 1-based indices; the
    # others on every slab unchanged
    assert s0["monitors"] == [dict(axis=3, index=5), dict(axis=1, index=4), dict(axis=2, index=3)]
    assert s1["monitors"] == [dict(axis=1, index=4), dict(axis=3, index=30 - 19), dict(axis=2, index=3)]


def test_slab_sim_source_on_the_cut_goes_to_both_slabs():
    sim = _sim(src_index=21)            # plane 20: first own plane of slab 1
    sl = slab3d.split_z(40, 2, 5)
    s0, s1 = (slab3d.slab_sim(sim, q) for q in sl)
    assert s0["source"]["index"] == 21   # the ghost plane over slab 0 (its H plane 19 is slab 0's)
    assert s1["source"]["index"] == 2    # plane 20 is local 1 of slab 1 (H plane 19 its ghost)


def test_slab_sim_cuts_x_and_y_normal_source_profiles():
    for axis in (1, 2):
        sim = _sim(src_axis=axis, src_index=5)
        sl = slab3d.split_z(40, 2, 5)
        for q in sl:
            s = slab3d.slab_sim(sim, q)
            for name in ("Ea", "Hb"):
                full = sim["source"][name]
                want = full[:, q.lo:q.hi] if axis == 1 else full[q.lo:q.hi, :]
                assert np.array_equal(s["source"][name], want)
            assert s["source"]["index"] == 5


def _fake_out(mons_shapes, nL, rng):
    mon = []
    for (na, nb) in mons_shapes:
        mon.append({k: rng.standard_normal((na, nb, nL)) + 1j * rng.standard_normal((na, nb, nL))
                    for k in ("Ea", "Eb", "Ha", "Hb")})
    return mon


def test_assemble_puts_cut_planes_together():
    sim = _sim()
    nL = 2
    rng = np.random.default_rng(5)
    nx, ny, nz = 10, 8, 40
    # the whole grid's monitor planes: z at 5 and 30 (nx x ny), x-normal (ny x nz), y-normal (nz x nx)
    full = _fake_out([(nx, ny), (ny, nz), (nx, ny), (nz, nx)], nL, rng)
    sl = slab3d.split_z(nz, 2, 5)
    outs = []
    for q in sl:
        m = []
        junk = lambda shape: rng.standard_normal(shape) * 1e3   # ghost rows: anything
        for mi, mq in enumerate(sim["monitors"]):
            ax, idx = mq["axis"], mq["index"] - 1
            if ax == 3:
                if q.z0 <= idx < q.z1:
                    m.append(full[mi])
                continue
            part = {}
            for k in ("Ea", "Eb", "Ha", "Hb"):
                f = full[mi][k]
                loc = np.zeros((ny, q.n, nL) if ax == 1 else (q.n, nx, nL), dtype=complex)
                if ax == 1:
                    loc[:] = junk(loc.shape)
                    loc[:, q.z0 - q.lo:q.z1 - q.lo] = f[:, q.z0:q.z1]
                else:
                    loc[:] = junk(loc.shape)
                    loc[q.z0 - q.lo:q.z1 - q.lo] = f[q.z0:q.z1]
                part[k] = loc
            m.append(part)
        fl = np.array([slab3d._flux(mm, 0.04) for mm in m])
        outs.append(dict(mon=m, flux=fl, steps=7, time=0.1, wallTime=1.0, lambdas=np.array([0.5, 0.6])))
    out = slab3d.assemble(sim, sl, outs)
    for mi in range(4):
        for k in ("Ea", "Eb", "Ha", "Hb"):
            assert np.array_equal(out["mon"][mi][k], full[mi][k])
        want = 0.5 * 0.04 ** 2 * np.real(full[mi]["Ea"] * np.conj(full[mi]["Hb"]) -
                                         full[mi]["Eb"] * np.conj(full[mi]["Ha"])).sum(axis=(0, 1))
        np.testing.assert_allclose(out["flux"][mi], want, rtol=1e-13)
    assert out["steps"] == 7 and out["flux"].shape == (4, nL)


def test_fixed_step_count_required():
    sim = _sim()
    sim["shutoff"] = 1e-8
    with pytest.raises(OrfError, match="shutoff"):
        slab3d._check_shutoff(sim)
    sim["periodic"] = [False, False, True]
    with pytest.raises(OrfError, match="periodic"):
        slab3d._npml_z(sim)


# ---- the swap between ranks: two gloo processes, CPU tensors for the planes

def _rank_views(rank, world, cnt):
    import torch
    v = {}
    base = 100.0 * (rank + 1)
    if rank + 1 < world:
        for f in slab3d.SEND_UP:
            v[("send_up", f)] = torch.full((cnt,), base + f)
        for f in slab3d.SEND_DOWN:
            v[("recv_above", f)] = torch.full((cnt,), -1.0)
    if rank > 0:
        for f in slab3d.SEND_DOWN:
            v[("send_down", f)] = torch.full((cnt,), base + 10 + f)
        for f in slab3d.SEND_UP:
            v[("recv_below", f)] = torch.full((cnt,), -1.0)
    return v


def _exchange_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        tr = slab3d.DistTransport()
        v = _rank_views(rank, world, 37)
        tr.exchange([v])
        got = {}
        for (kind, f), t in v.items():
            if kind.startswith("recv"):
                got[(kind, f)] = float(t[0]) if bool((t == t[0]).all()) else None
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_dist_transport_swaps_ghost_planes_between_ranks():
    import multiprocessing as mp
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_exchange_worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=100) for _ in ps)
    for p in ps:
        p.join(timeout=30)
        assert p.exitcode == 0
    for r in range(world):
        for (kind, f), val in res[r].items():
            if kind == "recv_above":     # the rank above's first own plane
                assert val == 100.0 * (r + 2) + 10 + f
            else:                        # the rank below's last own plane
                assert val == 100.0 * r + f
    assert set(res[1]) == {("recv_above", f) for f in slab3d.SEND_DOWN} | {("recv_below", f) for f in slab3d.SEND_UP}


def _same_sim_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res = {}
        sim = _sim()
        slab3d.check_same_sim(sim)           # identical sims: no error
        res["same"] = "ok"
        other = _sim()
        if rank == 1:
            other["eps"]["x"][3, 2, 17] += 1e-12   # one cell differs on one rank
        try:
            slab3d.fdtd3D_distributed(other)      # refused on the host, before any device work
            res["diff"] = "ran"
        except OrfError as e:
            res["diff"] = "refused" if "different sims" in str(e) else f"other: {e}"
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_ranks_with_different_sims_are_refused_before_device_work():
    import multiprocessing as mp
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_same_sim_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=100) for _ in ps)
    for p in ps:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert res[0] == res[1] == {"same": "ok", "diff": "refused"}


def test_sim_signature_sees_every_input():
    base = slab3d.sim_signature(_sim())
    assert slab3d.sim_signature(_sim()) == base
    for change in (lambda s: s["eps"]["z"].__setitem__((0, 0, 0), 2.0),
                   lambda s: s["source"].update(index=13),
                   lambda s: s.update(lambdas=[0.5, 0.61]),
                   lambda s: s.update(maxTime=2.0),
                   lambda s: s["monitors"].append(dict(axis=3, index=7)),
                   lambda s: s.update(precision="single")):
        s = _sim()
        change(s)
        assert slab3d.sim_signature(s) != base
