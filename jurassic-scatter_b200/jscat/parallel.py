"""Ray sharding across ranks (one process per GPU).

Rays -- and the scattering trees rooted at them -- are independent
(src/forwardmodel.c:60-68 runs them as an OpenMP loop), so a batch is
split into contiguous ray ranges, one per rank, with no data-path
exchange.  Ranges are balanced by a cheap geometric estimate of each
ray's LOS point count, because path lengths range over an order of
magnitude (nadir ~120 points, grazing limb ~400).  The only collective
is the final gather of radiances/transmittances.
"""
import numpy as np

RE = 6367.421


def estimate_los_points(geom, zmin=0.0, zmax=120.0, rayds=10.0, raydz=1.0):
    """Approximate LOS points per ray from the straight line observer ->
    view point: the chord through the shell between the lowest altitude
    the line reaches (or the ground) and zmax, divided by the step length
    the ray tracer takes (min(rayds, raydz/|cos zenith|))."""
    def cart(z, lon, lat):
        r = RE + np.asarray(z, dtype=np.float64)
        la, lo = np.radians(lat), np.radians(lon)
        return np.stack([r * np.cos(la) * np.cos(lo), r * np.cos(la) * np.sin(lo),
                         r * np.sin(la)], axis=-1)
    xo = cart(geom["obsz"], geom["obslon"], geom["obslat"])
    xv = cart(geom["vpz"], geom["vplon"], geom["vplat"])
    d = xv - xo
    d /= np.linalg.norm(d, axis=-1, keepdims=True)
    # closest approach of the line to the Earth's centre
    tmin = -np.sum(xo * d, axis=-1)
    rmin = np.linalg.norm(xo + tmin[:, None] * d, axis=-1)
    rtop, rbot = RE + zmax, RE + zmin
    s_top = np.sqrt(np.maximum(rtop ** 2 - rmin ** 2, 0.0))
    hits = rmin < rbot
    s_lo = np.where(hits, np.sqrt(np.maximum(rbot ** 2 - rmin ** 2, 0.0)), 0.0)
    # points = integral of 1/step along the chord; step = min(rayds,
    # raydz/|cos|) with |cos| = s/r at distance s from the closest approach
    u = np.linspace(0.0, 1.0, 65)
    sgrid = s_lo[:, None] + (s_top - s_lo)[:, None] * u[None, :]
    r = np.sqrt(rmin[:, None] ** 2 + sgrid ** 2)
    inv_step = np.maximum(1.0 / rayds, sgrid / (raydz * r))
    half = np.trapezoid(inv_step, sgrid, axis=1)
    return 2.0 + np.where(hits, half, 2.0 * half)


def shard_ranges(cost, world):
    """Contiguous [start, end) ranges, one per rank, with near-equal cost."""
    cost = np.asarray(cost, dtype=np.float64)
    n = len(cost)
    if world <= 1 or n == 0:
        return [(0, n)] + [(n, n)] * max(0, world - 1)
    cum = np.concatenate([[0.0], np.cumsum(cost)])
    cuts = [0]
    for k in range(1, world):
        cuts.append(int(np.searchsorted(cum, cum[-1] * k / world)))
    cuts.append(n)
    cuts = np.maximum.accumulate(np.minimum(cuts, n))
    return [(int(cuts[i]), int(cuts[i + 1])) for i in range(world)]


def select_rays(inp, start, end):
    """Batch-input dict restricted to rays [start, end), keeping only the
    profiles they use (re-indexed)."""
    ra = np.asarray(inp["ray_atm"][start:end])
    used = np.unique(ra)
    remap = np.full(len(inp["atm_off"]) - 1, -1, dtype=np.int64)
    remap[used] = np.arange(len(used))
    off = inp["atm_off"]
    lev = np.concatenate([np.arange(off[a], off[a + 1]) for a in used]) if len(used) else \
        np.zeros(0, dtype=np.int64)
    new_off = np.concatenate([[0], np.cumsum([off[a + 1] - off[a] for a in used])]).astype(np.int32)
    out = {"atm_off": new_off, "ray_atm": remap[ra].astype(np.int32)}
    for k in ("z", "lon", "lat", "p", "t"):
        out[k] = inp[k][lev]
    for k in ("q", "k"):
        out[k] = np.ascontiguousarray(inp[k][:, lev])
    for k in ("time", "obsz", "obslon", "obslat", "vpz", "vplon", "vplat"):
        out[k] = inp[k][start:end]
    return out


def gather_device(group=None):
    """Device of the all-gather buffers: NCCL moves CUDA tensors only (the
    rank's current GPU), gloo and MPI move CPU tensors."""
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def gather_rows(local, ranges, group=None):
    """All-gather per-rank row blocks (ranges from shard_ranges) into the
    full array on every rank, over torch.distributed.  local is this rank's
    block as a numpy array; the exchange runs on gather_device(group), the
    result comes back as a numpy array."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    dev = gather_device(group)
    local = np.ascontiguousarray(local, dtype=np.float64)
    width = local.shape[1:] if local.ndim > 1 else ()
    n_max = max(e - s for s, e in ranges)
    buf = torch.zeros((n_max,) + tuple(width), dtype=torch.float64, device=dev)
    if local.shape[0]:
        buf[: local.shape[0]] = torch.from_numpy(local).to(dev)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return np.concatenate([parts[i][: e - s].cpu().numpy() for i, (s, e) in enumerate(ranges)])


def forward_sharded(ctl, inp, device, group=None, model=None, aero=None, variant=-1):
    """The multi-GPU forward model of one batch input (every rank passes the
    same inp): rays are cut into contiguous ranges balanced by the
    geometric LOS estimate, each rank runs its range on its own GPU
    through the batch C-ABI, and one all-gather returns the radiances and
    transmittances of every ray, [n_rays][nd] each, to every rank."""
    import torch.distributed as dist
    from . import api
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    geom = {k: inp[k] for k in ("obsz", "obslon", "obslat", "vpz", "vplon", "vplat")}
    ranges = shard_ranges(estimate_los_points(geom), world)
    s, e = ranges[rank]
    nd = ctl.nd
    if e > s:
        out = api.formod_batch(ctl, select_rays(inp, s, e), device=device, model=model,
                               aero=aero, variant=variant)
        rad, tau = out["rad"], out["tau"]
    else:
        rad = tau = np.zeros((0, nd))
    both = gather_rows(np.concatenate([rad, tau], axis=1), ranges, group)
    return {"rad": both[:, :nd], "tau": both[:, nd:], "ranges": ranges}
