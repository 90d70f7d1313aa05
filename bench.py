"""Benchmark: ray-channel radiances/s of the batched clear-air forward model.

Workload (per GPU): 100,000 rays, half limb (tangent heights U[5, 60] km)
and half nadir/off-nadir (zenith U[0, 60] deg) from 800 km, 2,000 profiles
(50 rays each, T sigma 5 K, VMR sigma 20 %), 8 emitters, 64 channels
700-1400 cm^-1, 40x30x300 synthetic emissivity tables per (emitter,
channel), hydrostatic balance, refraction, FP64 geometry.  A step is one
forward model over the whole batch: hydrostatic balance, ray tracing, EGA
transmittance, continua, Planck source and radiative transfer.

value: throughput with the inputs resident in HBM (device-timed).
e2e:   same, through the C-ABI with host buffers: every step copies the
       inputs from pinned host memory and the radiances back.
Inputs (5.9 GB of table intervals, ~4 GB of LOS records) exceed the 126 MB
L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "jurassic-scatter_b200"))
sys.path.insert(0, REPO)

METRIC = "ray-channel radiances/s at <=0.05 K BT err, plain vs surrogate, 1 B200"
UNIT = "ray-channel radiances/s"
WORKLOAD = "batched clear-air forward model: 100k rays (50% limb TH 5-60 km, 50% nadir/off-nadir 0-60 deg), 2000 profiles, 8 emitters, 64 channels 700-1400 cm-1"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rays", type=int, default=100_000)
    ap.add_argument("--cpu-rays", type=int, default=600,
                    help="rays of the bounded CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_workload(n_rays, seed_offset=0):
    from jscat import synth
    workdir = os.environ.get("JSC_WORKDIR", "/tmp/jsc")
    ctlkw, atms, ray_atm, geom = synth.batched_case(workdir, n_rays=n_rays,
                                                    seed=20261203 + seed_offset)
    return ctlkw, atms, ray_atm, geom


def algorithmic_bytes(n_ega, n_points, n_rays, nd, ng):
    """Bytes one ega_rt launch must touch per the roofline model: per EGA
    evaluation 4 (p,T) nodes x 2 lookups x bracketing (u,eps) pair = 128 B;
    per LOS point and channel the Planck bracket (8 B); per LOS point p, T
    and u[g] (16 + 8 G B); per ray and channel rad + tau out (8 B)."""
    return 128 * n_ega + 8 * n_points * nd + (16 + 8 * ng) * n_points + 8 * n_rays * nd


def cpu_baseline(ctlkw, atms, ray_atm, geom, n_sample):
    """The reference's OpenMP formod on a bounded sample of the workload
    (whole profiles, first n_sample rays), all host cores, after a warm-up
    call (tables and Planck data are first-call static)."""
    from oracle import refrun
    n_atm = max(1, n_sample // 50)
    sel = np.nonzero(ray_atm < n_atm)[0]
    sub_geom = {k: v[sel] for k, v in geom.items()}
    cores = os.cpu_count() or 1
    # SCA_MULT=0: the clear-air arithmetic without the reference's read of
    # the uninitialised los->aerofac (see tests/golden/make_golden.py).
    ref_kw = dict(ctlkw, sca_mult=0)
    if refrun.available():
        res = refrun.run(ref_kw, atms[:n_atm], ray_atm[sel], sub_geom,
                         threads=cores, warmup=True, timeout=3600)
        kind = "reference"
    else:
        res = refrun.run_port(ctlkw, atms[:n_atm], ray_atm[sel], sub_geom,
                              threads=cores, warmup=True, timeout=3600)
        kind = "port"
    v = len(sel) * ctlkw_nd(ctlkw) / res["seconds"]
    return {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
            "sample": "%d rays (%d profiles) of the workload, %d channels, %.1f s"
                      % (len(sel), n_atm, ctlkw_nd(ctlkw), res["seconds"])}, res, sel


def ctlkw_nd(ctlkw):
    return len(ctlkw["nus"])


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    ctlkw, atms, ray_atm, geom = make_workload(args.rays)
    from oracle import refrun
    cores = os.cpu_count() or 1
    n_atm = 4
    times = []
    for step in range(args.warmup + args.steps):
        a0 = (step * n_atm) % len(atms)
        sel_atm = list(range(a0, a0 + n_atm))
        sel = np.nonzero(np.isin(ray_atm, sel_atm))[0]
        sub = {k: v[sel] for k, v in geom.items()}
        if refrun.available():
            res = refrun.run(dict(ctlkw, sca_mult=0), [atms[i] for i in sel_atm],
                             ray_atm[sel] - a0, sub, threads=cores, warmup=True,
                             timeout=3600)
        else:
            res = refrun.run_port(ctlkw, [atms[i] for i in sel_atm], ray_atm[sel] - a0,
                                  sub, threads=cores, warmup=True, timeout=3600)
        if step >= args.warmup:
            times.append((len(sel), res["seconds"]))
    n = sum(t[0] for t in times)
    sec = sum(t[1] for t in times)
    nd = ctlkw_nd(ctlkw)
    v = n * nd / sec
    kind = "reference" if refrun.available() else "port"
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sec / max(1, len(times)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample_per_step": "%d profiles x 50 rays" % n_atm},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
                             "sample": "%d rays per step, %d channels" % (n // max(1, len(times)), nd)},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    from jscat import api, structs as S, synth, lib as L

    ctlkw, atms, ray_atm, geom = make_workload(args.rays, seed_offset=rank)
    ctl = S.make_ctl(**ctlkw)
    nd, ng = ctl.nd, ctl.ng
    inp = synth.batch_from(atms, ray_atm, geom)
    model = api.Model(ctl, device=local)
    nl = len(inp["z"])
    batch = api.Batch(model, ctl, len(atms), nl, args.rays)
    stream = torch.cuda.Stream()
    sp = stream.cuda_stream

    # Pinned host copies of every input and output (for e2e).
    def pin(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        return t.numpy()
    pinned = {k: pin(v) for k, v in inp.items()}
    out_pinned = {"rad": pin(np.empty((args.rays, nd))), "tau": pin(np.empty((args.rays, nd)))}
    h2d = sum(v.nbytes for v in pinned.values())
    d2h = sum(v.nbytes for v in out_pinned.values())

    batch.upload(pinned, stream=sp)
    batch.set_timing(True)
    tuned = batch.autotune(stream=sp)   # launch-variant autotuner (untimed)
    for _ in range(args.warmup):
        batch.run(stream=sp)
    stream.synchronize()
    res = batch.download(stream=sp)
    n_points, n_ega = batch.counters()

    # Device-resident timing.
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = api.launch_count()
    ega_ms = []
    ev0.record(stream)
    for _ in range(args.steps):
        batch.run(stream=sp)
        ega_ms.append(batch.kernel_ms("ega_rt"))
    ev1.record(stream)
    stream.synchronize()
    torch.cuda.synchronize()
    launches = api.launch_count() - l0
    t_ms = ev0.elapsed_time(ev1)
    # e2e: host buffers through the C-ABI every step.
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        batch.upload(pinned, stream=sp)
        batch.run(stream=sp)
        batch.download(stream=sp, out=out_pinned)
    e1.record(stream)
    stream.synchronize()
    e_ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    if dist:
        tt = torch.tensor([t_ms, e_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_ms, e_ms = tt.tolist()
    ms_step = t_ms / args.steps
    units = args.rays * nd * world
    value = units / (ms_step / 1e3)
    e2e = units / (e_ms / args.steps / 1e3)

    ega = float(np.mean(ega_ms))
    B = algorithmic_bytes(n_ega, n_points, args.rays, nd, ng)
    peaks_path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = json.load(open(peaks_path))["hbm_gbs"]
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    achieved = B / (ega / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(REPO, "profiles", "ega_rt_traffic.json")
    if os.path.exists(tpath):
        traffic = json.load(open(tpath)).get("bytes_per_launch")

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded generator, no dataset)",
            "config": {"workload": WORKLOAD, "rays_per_gpu": args.rays,
                       "channels": nd, "emitters": ng, "los_points": n_points,
                       "ega_evaluations": n_ega, "l2": "inputs larger than L2, no flush",
                       "parallelism": "rays sharded per GPU, no collective",
                       "ega_launch": tuned},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_source": peak_src,
                         "kernel": "ega_rt", "kernel_ms": ega,
                         "algorithmic_bytes_per_launch": B},
            "clocks": clk}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb, ref, sel = cpu_baseline(ctlkw, atms, ray_atm, geom, args.cpu_rays)
            line["cpu_baseline"] = cb
            # BT error of this run against the reference on the sample.
            sys.path.insert(0, os.path.join(REPO, "tests"))
            from helpers import bt_error
            line["bt_err_k_vs_reference"] = bt_error(res["rad"][sel], ref["rad"], ctlkw["nus"])
        except Exception as exc:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "error": str(exc)[:200]}
    if rank == 0:
        print(json.dumps(line))
    batch.close()
    model.close()
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
