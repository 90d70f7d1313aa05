"""Ray sharding and the result gather of the multi-GPU path, run as two
gloo ranks on CPU, with the CPU oracle computing each shard."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as tmp

from conftest import PKG, REPO


def test_shard_ranges_cover_and_balance():
    from jscat import parallel
    cost = np.r_[np.full(50, 120.0), np.full(50, 400.0)]
    r = parallel.shard_ranges(cost, 4)
    assert r[0][0] == 0 and r[-1][1] == 100
    assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
    loads = [cost[s:e].sum() for s, e in r]
    assert max(loads) - min(loads) <= 400.0
    assert parallel.shard_ranges(cost, 1) == [(0, 100)]
    assert parallel.shard_ranges(np.zeros(0), 3) == [(0, 0), (0, 0), (0, 0)]


def test_los_estimate_tracks_the_reference_count():
    """The geometric estimate is within 25 % of the exact LOS
    point counts of the mixed limb/nadir fixture."""
    from jscat import parallel
    g = dict(np.load(os.path.join(REPO, "tests", "golden", "mixed_batch.npz")))
    geom = {k[5:]: v for k, v in g.items() if k.startswith("geom_")}
    est = parallel.estimate_los_points(geom)
    ratio = est / g["nlos"]
    assert np.all(ratio > 0.8) and np.all(ratio < 1.25)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, workdir, outdir):
    sys.path.insert(0, PKG)
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    from jscat import parallel, synth
    from make_golden_shim import mixed_case
    from oracle import refrun
    ctlkw, atms, ray_atm, geom = mixed_case(workdir)
    inp = synth.batch_from(atms, ray_atm, geom)
    cost = parallel.estimate_los_points(geom)
    ranges = parallel.shard_ranges(cost, world)
    s, e = ranges[rank]
    sub = parallel.select_rays(inp, s, e)
    # each rank computes its shard (the oracle stands in for the GPU here)
    atms_sub = []
    for a in range(len(sub["atm_off"]) - 1):
        lo, hi = sub["atm_off"][a], sub["atm_off"][a + 1]
        atms_sub.append({"z": sub["z"][lo:hi], "lon": sub["lon"][lo:hi], "lat": sub["lat"][lo:hi],
                         "p": sub["p"][lo:hi], "t": sub["t"][lo:hi], "q": sub["q"][:, lo:hi],
                         "k": sub["k"][:, lo:hi]})
    gsub = {k: sub[k] for k in ("time", "obsz", "obslon", "obslat", "vpz", "vplon", "vplat")}
    res = refrun.run_port(ctlkw, atms_sub, sub["ray_atm"], gsub)
    rad = parallel.gather_rows(res["rad"], ranges)
    if rank == 0:
        np.save(os.path.join(outdir, "rad.npy"), rad)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shard_and_gather(workdir, tmp_path):
    port = _free_port()
    tmp.spawn(_rank, args=(2, port, workdir, str(tmp_path)), nprocs=2, join=True)
    g = dict(np.load(os.path.join(REPO, "tests", "golden", "mixed_batch.npz")))
    rad = np.load(os.path.join(tmp_path, "rad.npy"))
    assert np.array_equal(rad, g["rad"])


def test_gather_device_follows_the_backend(monkeypatch):
    """NCCL all-gathers CUDA tensors only: the gather buffers live on the
    rank's current GPU under nccl and in host memory under gloo."""
    import torch
    import torch.distributed as dist
    from jscat import parallel
    monkeypatch.setattr(dist, "get_backend", lambda group=None: "gloo")
    assert parallel.gather_device() == torch.device("cpu")
    monkeypatch.setattr(dist, "get_backend", lambda group=None: "nccl")
    monkeypatch.setattr(torch.cuda, "current_device", lambda: 3)
    assert parallel.gather_device() == torch.device("cuda", 3)


def _rank_gather(rank, world, port, outdir):
    sys.path.insert(0, PKG)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    from jscat import parallel
    full = np.arange(7 * 3, dtype=np.float64).reshape(7, 3)
    ranges = parallel.shard_ranges(np.r_[np.ones(2), np.full(5, 0.1)], world)
    s, e = ranges[rank]
    got = parallel.gather_rows(full[s:e], ranges)
    np.save(os.path.join(outdir, "g%d.npy" % rank), got)
    dist.barrier()
    dist.destroy_process_group()


def test_gather_rows_uneven_ranges(tmp_path):
    """Ranges of unequal length (one of them possibly empty) come back in
    ray order on every rank."""
    port = _free_port()
    tmp.spawn(_rank_gather, args=(3, port, str(tmp_path)), nprocs=3, join=True)
    full = np.arange(7 * 3, dtype=np.float64).reshape(7, 3)
    for r in range(3):
        assert np.array_equal(np.load(os.path.join(tmp_path, "g%d.npy" % r)), full)
