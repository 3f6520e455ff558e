#!/usr/bin/env python
"""Headline benchmark: Mvis/s of the w-gridding adjoint pair (ms2dirty +
dirty2ms) at 4096^2 on ~8.1M visibilities, mixed precision (FP32 bulk, FP64
coordinates / w-phase / image accumulation / correction) at epsilon 1e-5,
with the plain FP64 GPU form (epsilon 1e-12) and the relative RMS error
against an FP64 direct Fourier transform reported beside it.

A step = one ms2dirty of the visibilities + one dirty2ms of the model image
over the whole workload.  ``value`` times steps with inputs resident in HBM
(CUDA events on the gridder's stream); ``e2e`` times the same steps through
the public API from pinned host buffers (H2D of uvw + data, D2H of the
result inside the timed region).

Workload (synthetic, seeded): 128 antennas uniform within 6 km, 8 s cadence
over 997 timesteps (8128 baselines -> 8,103,616 visibilities), one channel at
150 MHz, dec -30 deg, |w| scaled to 30% of max|uv|, 200 power-law point
sources; 4096^2 image at 5" pixels.

--impl reference times the reference's own CPU w-gridder (ducc0 as vendored
by WSClean, compiled from the reference sources into oracle/_ref) on the same
workload with all host threads.
"""
from __future__ import annotations

import argparse
import gc
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "Mvis/s ms2dirty+dirty2ms @4096²: FP32-mixed vs FP64 GPU, rel err vs FP64 DFT"
UNIT = "Mvis/s"
EPS_MIXED, EPS_FP64 = 1e-5, 1e-12
# WSClean's call pattern of the reference w-gridder (wgriddinggridder_simple.cpp:56-58)
CALL = "negate_v, no divide_by_n, sigma 1.1..2.0"
GRIDS_PATH = os.path.join(HERE, "tests", "golden", "ducc_grids.json")


def ducc_grids():
    """The grids the reference (ducc0) chooses for the benchmark workloads,
    from its verbosity-1 report on the same seeded data
    (tests/golden/make_ducc_grids.py).  The roofline charges their
    algorithmic bytes, so that it does not depend on this library's own
    (smaller, band-pruned) grid choice."""
    with open(GRIDS_PATH) as fh:
        return json.load(fh)


def grid_tuple(g):
    return (int(g["nu"]), int(g["nv"]), int(g["nplanes"]))


def peak_hbm():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def roofline(bytes_per_step, ms_per_step, kernel):
    """HBM roofline of a workload: algorithmic bytes (the reference's grid,
    the build plan's formula) over the measured time."""
    peak, src = peak_hbm()
    achieved = bytes_per_step / (ms_per_step / 1e3) / 1e9
    return {"bound": "hbm", "kernel": kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": src, "bytes_per_step": int(bytes_per_step)}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-clocks", action="store_true",
                    help="do not sample nvidia-smi during the timed region")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the config-4 batched-facets measurement")
    ap.add_argument("--legs", default="1,3,4,5",
                    help="the other configurations to measure after the headline "
                         "(comma list of 1, 3, 4, 5; empty for none)")
    ap.add_argument("--timed-only", action="store_true",
                    help="stop after the timed region (for profiler launch lists)")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="fraction of the 997 timesteps (small cases for ncu captures)")
    ap.add_argument("--launch-summary", metavar="CSV",
                    help="summarise an ncu launch list (gpu__time_duration.sum) of a "
                         "--timed-only run: per kernel launches, time and share over the "
                         "last --steps steps, then exit")
    return ap.parse_args()


def launch_summary(path, steps):
    """Per-kernel totals of the last `steps` steps (two gridder calls each,
    each starting with k_scan) of an ncu --csv launch list: launches, device
    time and share, and -- when the list holds dram__bytes_read/write.sum --
    the DRAM bytes read and written, with the total per step."""
    import collections
    import csv
    import re
    rows = list(csv.reader(open(path)))
    hi = next(i for i, r in enumerate(rows) if "Kernel Name" in r)
    h = rows[hi]
    ii, ki = h.index("ID"), h.index("Kernel Name")
    mi, vi, ui = h.index("Metric Name"), h.index("Metric Value"), h.index("Metric Unit")
    scale = {"nsecond": 1e-6, "ns": 1e-6, "usecond": 1e-3, "us": 1e-3, "msecond": 1.0, "ms": 1.0,
             "second": 1e3, "s": 1e3,
             "byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "Tbyte": 1e12}
    launches = collections.OrderedDict()  # launch id -> (kernel, {metric: value})
    for r in rows[hi + 1:]:
        if len(r) <= vi or not r[vi]:
            continue
        ent = launches.setdefault(r[ii], (r[ki], {}))
        ent[1][r[mi]] = float(r[vi].replace(",", "")) * scale.get(r[ui], 1.0)
    launches = list(launches.values())
    # each call starts with its visibility scan (k_scan or k_scan_keys; not
    # the read-back of the scan's statistics)
    starts = [i for i, (k, _) in enumerate(launches) if re.search(r"\bk_scan(_keys)?[<(]", k)]
    seg = launches[starts[-2 * steps]:] if len(starts) >= 2 * steps else launches
    tot = collections.OrderedDict()
    for k, m in seg:
        name = k.split("(")[0].replace("void ", "")
        c = tot.setdefault(name, [0, 0.0, 0.0, 0.0])
        c[0] += 1
        c[1] += m.get("gpu__time_duration.sum", 0.0)
        c[2] += m.get("dram__bytes_read.sum", 0.0)
        c[3] += m.get("dram__bytes_write.sum", 0.0)
    T = sum(v[1] for v in tot.values()) or 1.0
    dram = any(v[2] or v[3] for v in tot.values())
    print(f"{'kernel':72s} {'launches':>8s} {'ms':>8s} {'share':>6s}"
          + (f" {'read GB':>8s} {'write GB':>8s}" if dram else ""))
    for k, (n, ms, rd, wr) in sorted(tot.items(), key=lambda x: -x[1][1]):
        print(f"{k[:72]:72s} {n:8d} {ms:8.3f} {100 * ms / T:5.1f}%"
              + (f" {rd / 1e9:8.3f} {wr / 1e9:8.3f}" if dram else ""))
    print(f"total {T:.3f} ms over {sum(v[0] for v in tot.values())} launches in {steps} step(s)")
    if dram:
        b = sum(v[2] + v[3] for v in tot.values())
        print(f"total DRAM {b / 1e9:.3f} GB")
        print(f"traffic_bytes_per_step: {int(b / steps)}")


def profiled_traffic():
    """DRAM bytes per step (read + write, all kernels of one ms2dirty +
    dirty2ms) from the committed ncu summary, or None."""
    path = os.path.join(HERE, "profiles", "pipeline_traffic_config2.txt")
    try:
        with open(path) as fh:
            for line in fh:
                if line.startswith("traffic_bytes_per_step:"):
                    return int(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


def algorithmic_bytes(nvis, nrows, nx, ny, grid, s_vis, s_grid):
    """Bytes per call of one direction (ms2dirty or dirty2ms)."""
    nu, nv, npl = grid
    return (nvis * s_vis + nrows * 24 + npl * 3 * s_grid * nu * nv
            + npl * 16 * nx * ny + 2 * 8 * nx * ny)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload(scale=1.0):
    from wsclean_b200 import synth
    c = synth.config2(scale=scale)
    rng = np.random.default_rng(12)
    nx = c["npix_x"]
    ix, iy, flux = synth.point_sky(c["nsrc"], nx, nx, rng)
    return c, ix, iy, flux


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo",
                                timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def config2_dict(nvis, nx, world):
    """The workload description both arms print (the same dict)."""
    return {"workload": "config-2 adjoint pair: 8.1M vis, 4096^2 @ 5\", eps 1e-5",
            "nvis": nvis, "npix": nx, "call": CALL, "parallelism": f"replicas x{world}",
            "l2": "inputs and grids larger than L2 (uvw 194 MB, grids GBs)"}


def run_reference(args, world, rank):
    """The reference's CPU w-gridder (compiled ducc0) on the same workload."""
    if rank != 0:
        return
    import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "compiled reference (oracle/_ref) missing"}))
        return
    c, ix, iy, flux = workload(args.scale)
    from wsclean_b200 import synth
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    nvis = uvw.shape[0] * len(freq)
    # the gridder's run time does not depend on the values: seeded noise
    # stands in for the sky visibilities so no GPU is touched here
    g = np.random.default_rng(3)
    vis = (g.normal(size=(uvw.shape[0], len(freq)))
           + 1j * g.normal(size=(uvw.shape[0], len(freq)))).astype(np.complex64)
    model = synth.sky_image(nx, nx, ix, iy, flux).astype(np.float32)
    cores = os.cpu_count()
    kw = dict(prec="float", negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0,
              nthreads=cores)

    def step():
        t0 = time.perf_counter()
        O.ref_ms2dirty(uvw, freq, vis, nx, nx, px, px, EPS_MIXED, **kw)
        O.ref_dirty2ms(uvw, freq, model, px, px, EPS_MIXED, **kw)
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        step()
    ts = [step() for _ in range(args.steps)]
    tot = sum(ts)
    value = nvis * len(ts) / tot / 1e6
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": len(ts), "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(ts),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Earth-rotation observation, 200 point sources)",
        "config": config2_dict(nvis, nx, world),
        "instance": "ducc0 <float,float>",
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": "full workload per step (one ms2dirty + one dirty2ms)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


KW = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)
KW_REF = dict(KW, nthreads=0)


def device_timed(torch, dev, fns, steps, warmup):
    """Mean device time (ms) of each synchronous library call in fns, by CUDA
    events on torch's current stream (the calls are ordered on it)."""
    st = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        for f in fns:
            f()
    torch.cuda.synchronize(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(fns) + 1)]
    tot = [0.0] * len(fns)
    for _ in range(steps):
        ev[0].record(st)
        for i, f in enumerate(fns):
            f()
            ev[i + 1].record(st)
        torch.cuda.synchronize(dev)
        for i in range(len(fns)):
            tot[i] += ev[i].elapsed_time(ev[i + 1])
    return [t / steps for t in tot]


def cpu_pair(uvw, freq, vis, model, nx, px, eps, prec, wgt=None, sample=""):
    """The reference's CPU w-gridder (oracle/_ref, all host threads) on one
    ms2dirty + dirty2ms, with its grid choice from the verbosity report."""
    import oracle as O
    if not O.ref_available():
        return None, None
    t0 = time.perf_counter()
    _, rep = O.ref_ms2dirty(uvw, freq, vis, nx, nx, px, px, eps, prec=prec, wgt=wgt,
                            return_report=True, **KW_REF)
    t1 = time.perf_counter()
    O.ref_dirty2ms(uvw, freq, model, px, px, eps, prec=prec, wgt=wgt, vis_dtype=vis.dtype, **KW_REF)
    t2 = time.perf_counter()
    nvis = vis.size
    return ({"value": nvis / (t2 - t0) / 1e6, "unit": UNIT, "cores": os.cpu_count(),
             "kind": "reference", "ms2dirty_mvis_s": nvis / (t1 - t0) / 1e6,
             "dirty2ms_mvis_s": nvis / (t2 - t1) / 1e6,
             "sample": sample or "full workload, one ms2dirty + one dirty2ms"},
            O.parse_report(rep)[0])


def leg_config1(torch, dev, ctx, grids, with_cpu):
    """Config 1: plain FP64 (complex128) pair at epsilon 1e-12, 1024^2 at 10",
    2.9M visibilities -- the form of WSClean's own CPU path."""
    from wsclean_b200 import synth
    c = synth.config1()
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(1)
    ix, iy, flux = synth.point_sky(c["nsrc"], nx, nx, rng)
    vis = synth.predict_vis(uvw, freq, nx, nx, px, px, ix, iy, flux, device=dev)
    vis = vis + 0.1 * (rng.normal(size=vis.shape) + 1j * rng.normal(size=vis.shape))
    model = synth.sky_image(nx, nx, ix, iy, flux)
    nrows, nvis = uvw.shape[0], vis.size
    tu, tf = torch.as_tensor(uvw, device=dev), torch.as_tensor(freq, device=dev)
    tv, tm = torch.as_tensor(vis, device=dev), torch.as_tensor(model, device=dev)
    d = torch.zeros((nx, nx), dtype=torch.float64, device=dev)
    o = torch.zeros(vis.shape, dtype=torch.complex128, device=dev)
    eps = 1e-12
    t1, t2 = device_timed(torch, dev, [
        lambda: ctx.ms2dirty(tu, tf, tv, nx, nx, px, px, eps, precision="fp64", dirty=d, **KW),
        lambda: ctx.dirty2ms(tu, tf, tm, px, px, eps, precision="fp64", vis=o, **KW)], 5, 2)
    st = ctx.stats()
    pix = rng.integers(0, nx * nx, 16)
    acc = {"ms2dirty_rel_rms_vs_dft":
           rel_rms(d.cpu().numpy().ravel()[pix], dft_pixels(uvw, freq, vis, nx, nx, px, px, pix,
                                                            torch, dev))}
    cpu, g = cpu_pair(uvw, freq, vis, model, nx, px, eps, "double") if with_cpu else (None, None)
    g = g or grids["config1"]["fp64"]
    B = 2 * algorithmic_bytes(nvis, nrows, nx, nx, grid_tuple(g), 16, 16)
    return {"workload": "config 1: 64 antennas within 3 km, 360 x 10 s, 4 channels, 2.9M complex128 "
                        "visibilities, 1024^2 at 10\", FP64 at eps 1e-12",
            "nvis": nvis, "ms2dirty_mvis_s": nvis / t1 / 1e3, "dirty2ms_mvis_s": nvis / t2 / 1e3,
            "value": nvis / (t1 + t2) / 1e3, "ms_per_step": t1 + t2,
            "grid": {"nu": st["nu"], "nv": st["nv"], "nplanes": st["nplanes"], "W": st["supp"]},
            "reference_grid": g, "roofline": roofline(B, t1 + t2, "FP64 pair"),
            "accuracy": acc, "cpu_baseline": cpu}


def leg_config3(torch, dev, ctx, grids, with_cpu):
    """Config 3: the chi^2-gradient pair (one dirty2ms of the model, one
    ms2dirty of the weighted residuals) at 2048^2 / 8" on the config-2 array,
    Briggs robust-0 times U[0.5, 2] noise weights, mixed at eps 1e-5."""
    from wsclean_b200 import synth
    c = synth.config3()
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    rng = np.random.default_rng(3)
    ix, iy, flux = synth.point_sky(c["nsrc"], nx, nx, rng)
    vis = synth.predict_vis(uvw, freq, nx, nx, px, px, ix, iy, flux, device=dev)
    noise = rng.uniform(0.5, 2.0, vis.shape)
    w = (noise * synth.briggs_weights(uvw, freq, nx, nx, px, px, robust=0.0,
                                      noise_weights=noise)).astype(np.float32)
    model = synth.sky_image(nx, nx, ix, iy, flux)
    model = (model * (1 + 0.05 * rng.normal(size=model.shape))).astype(np.float32)
    nrows, nvis = uvw.shape[0], vis.size
    tu, tf = torch.as_tensor(uvw, device=dev), torch.as_tensor(freq, device=dev)
    tv = torch.as_tensor(vis.astype(np.complex64), device=dev)
    tw, tm = torch.as_tensor(w, device=dev), torch.as_tensor(model, device=dev)
    d = torch.zeros((nx, nx), dtype=torch.float32, device=dev)
    o = torch.zeros(vis.shape, dtype=torch.complex64, device=dev)
    eps = 1e-5
    t2, t1 = device_timed(torch, dev, [
        lambda: ctx.dirty2ms(tu, tf, tm, px, px, eps, wgt=tw, vis=o, **KW),
        lambda: ctx.ms2dirty(tu, tf, tv, nx, nx, px, px, eps, wgt=tw, dirty=d, **KW)], 10, 3)
    st = ctx.stats()
    cpu, g = (cpu_pair(uvw, freq, vis.astype(np.complex64), model, nx, px, eps, "float", wgt=w)
              if with_cpu else (None, None))
    g = g or grids["config3"]["mixed"]
    B = 2 * algorithmic_bytes(nvis, nrows, nx, nx, grid_tuple(g), 8, 8) + 2 * nvis * 4
    return {"workload": "config 3: chi^2 gradient pair, config-2 array (8.1M vis) at 2048^2 / 8\", "
                        "Briggs(0) x U[0.5,2] weights, mixed at eps 1e-5",
            "nvis": nvis, "ms2dirty_mvis_s": nvis / t1 / 1e3, "dirty2ms_mvis_s": nvis / t2 / 1e3,
            "value": nvis / (t1 + t2) / 1e3, "ms_per_step": t1 + t2,
            "grid": {"nu": st["nu"], "nv": st["nv"], "nplanes": st["nplanes"], "W": st["supp"]},
            "reference_grid": g, "roofline": roofline(B, t1 + t2, "mixed pair with weights"),
            "cpu_baseline": cpu}


def run_batched(dev, torch, ctx, args):
    """Config 4: 16 Voronoi facets x 8 output channels (8 of 64 input
    channels each) = 128 jobs over the same rows, gridded and degridded
    through one reusable plan (one persistent spread / interpolation launch
    per call, replayed as a CUDA graph), against the plain FP64 form run job
    by job over all 128 jobs, at the mixed form's epsilon (1e-5, the same
    stated accuracy) and at 1e-12."""
    from wsclean_b200 import synth
    from wsclean_b200 import gridder as G
    c = synth.config4()
    uvw, freq, px = c["uvw"], c["freq"], c["pixsize"]
    nrows = uvw.shape[0]
    jobs = [dict(npix_x=f["nx"], npix_y=f["ny"], center_x=f["dx"] * px, center_y=f["dy"] * px,
                 chan_begin=8 * oc, chan_end=8 * oc + 8)
            for oc in range(8) for f in synth.facets4()]
    kw = KW
    g = torch.Generator(device=dev).manual_seed(7)
    vis = torch.complex(torch.randn(nrows, 64, device=dev, generator=g),
                        torch.randn(nrows, 64, device=dev, generator=g))
    jv = nrows * 8 * len(jobs)
    t0 = time.perf_counter()
    plan = G.Plan(uvw, freq, px, px, EPS_MIXED, jobs=jobs, **kw)
    torch.cuda.synchronize(dev)
    t_build = time.perf_counter() - t0
    st = torch.cuda.Stream(dev)
    models = [torch.zeros((j["npix_x"], j["npix_y"]), device=dev) for j in jobs]
    for m in models:
        m[m.shape[0] // 2, m.shape[1] // 2] = 1.0
    dirty = [torch.empty((j["npix_x"], j["npix_y"]), device=dev) for j in jobs]
    pred = torch.empty_like(vis)
    n = 3
    with torch.cuda.stream(st):
        for _ in range(3):
            plan.ms2dirty(vis, dirty)
            plan.dirty2ms(models, pred)
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record(st)
        for _ in range(n):
            plan.ms2dirty(vis, dirty)
        e[1].record(st)
        for _ in range(n):
            plan.dirty2ms(models, pred)
        e[2].record(st)
        st.synchronize()
    tg, td = e[0].elapsed_time(e[1]) / n, e[1].elapsed_time(e[2]) / n
    W = plan.stats(0)["supp"]
    plan.close()
    del dirty, pred, models
    # plain FP64 form, job by job over all 128 jobs (a first pass creates the
    # FFT plans of each facet size and is not timed)
    vis64 = vis.to(torch.complex128)
    del vis
    tu = torch.as_tensor(uvw, device=dev)
    tf = torch.as_tensor(freq, device=dev)
    chans = [vis64[:, 8 * oc:8 * oc + 8].contiguous() for oc in range(8)]
    del vis64

    def per_job(eps, timed_jobs):
        for rep in range(2):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            for j in (timed_jobs if rep else timed_jobs[:16]):
                c0, c1 = j["chan_begin"], j["chan_end"]
                ctx.ms2dirty(tu, tf[c0:c1], chans[c0 // 8], j["npix_x"], j["npix_y"], px, px, eps,
                             precision="fp64", center_x=j["center_x"], center_y=j["center_y"],
                             dirty_dtype=np.float64, **kw)
            torch.cuda.synchronize(dev)
            t = (time.perf_counter() - t0) * 1e3
        return t

    t64 = per_job(EPS_FP64, jobs)
    t64e = per_job(EPS_MIXED, jobs)
    del chans
    cycles = 10
    return {"workload": "config 4: 96 antennas within 10 km, 360 x 10 s, 64 channels 120-180 MHz; "
                        "16 Voronoi facets (512^2..2048^2, phase centre at the box centre) x 8 "
                        "output channels = 128 jobs",
            "rows": nrows, "job_visibilities": jv, "plan_build_s": t_build, "W": W,
            "mixed_ms2dirty_ms": tg, "mixed_dirty2ms_ms": td,
            "mixed_ms2dirty_mvis_s": jv / tg / 1e3, "mixed_dirty2ms_mvis_s": jv / td / 1e3,
            "mixed_pair_mvis_s": jv / (tg + td) / 1e3,
            "mixed_pair_mvis_s_with_build_over_%d_cycles" % cycles:
                jv / (tg + td + t_build * 1e3 / cycles) / 1e3,
            "fp64_per_job_ms2dirty_ms": t64, "fp64_per_job_ms2dirty_mvis_s": jv / t64 / 1e3,
            "fp64_per_job_eps_1e-5_ms2dirty_ms": t64e,
            "fp64_per_job_eps_1e-5_ms2dirty_mvis_s": jv / t64e / 1e3,
            "mixed_batched_over_fp64_per_job": t64 / tg,
            "mixed_batched_over_fp64_per_job_same_eps": t64e / tg,
            "fp64_timing": "all 128 jobs timed (warm FFT plans), wall clock with a device sync "
                           "on both sides; the mixed plan time excludes its build (reported "
                           "beside it, and amortised over %d major cycles)" % cycles}


def leg_config5(torch, dev, ctx, grids, with_cpu, args):
    """Config 5: 522M visibilities (256 antennas, 1000 x 8 s, 16 channels)
    at 8192^2 / 2", streamed from page-locked host memory in 256 MiB chunks
    through wsg_stream_*: dirty2ms of the sky model (2000 point sources and 5
    Gaussians) chunk by chunk, then ms2dirty of those visibilities.  Also the
    same with the chunks resident in HBM (no host copies), the plain
    host-to-device copy time of the data, the tuned schedule against the
    plain one on a 2% time subsample, and the reference on 30% of the data."""
    from wsclean_b200 import synth
    from wsclean_b200 import gridder as G
    c = synth.config5()
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    nrows, nchan = uvw.shape[0], len(freq)
    nvis = nrows * nchan
    rng = np.random.default_rng(5)
    ix, iy, flux = synth.point_sky(c["nsrc"], nx, nx, rng)
    model = synth.sky_image(nx, nx, ix, iy, flux) + synth.gaussian_blobs(nx, nx, c["ngauss"], rng)
    model32 = model.astype(np.float32)
    rows = (256 << 20) // (24 + 8 * nchan)
    bounds = list(range(0, nrows, rows)) + [nrows]
    parts = list(zip(bounds[:-1], bounds[1:]))
    h_uvw = torch.as_tensor(uvw).pin_memory()
    h_vis = torch.empty((nrows, nchan), dtype=torch.complex64).pin_memory()
    h_model = torch.as_tensor(model32).pin_memory()
    h_dirty = torch.empty((nx, nx), dtype=torch.float32).pin_memory()
    ext = G.data_extent(uvw, freq)
    out = {"workload": "config 5: 256 antennas (log-radial to 20 km), 1000 x 8 s, 16 channels "
                       "140-190 MHz, 522M complex64 visibilities, 8192^2 at 2\", |w| up to 40% "
                       "of max|uv|, mixed at eps 1e-5, streamed in 256 MiB chunks",
           "nvis": nvis, "chunks": len(parts)}
    s = G.Stream(freq, nx, nx, px, px, EPS_MIXED, ext, nvis=nvis, context=ctx, **KW)
    try:
        def d2m(src_uvw, dst_vis, pipelined=False):
            # pipelined (wsg_ctx_set_async): each chunk's predictions are
            # copied back to page-locked memory while the next chunk is
            # computed; they are in place after the synchronisation
            ctx.set_async(pipelined)
            try:
                s.predict_begin(h_model)
                for a, b in parts:
                    s.predict(src_uvw[a:b], vis=dst_vis[a:b])
                ctx.synchronize()
            finally:
                ctx.set_async(False)

        def m2d(src_uvw, src_vis, dst):
            for a, b in parts:
                s.add(src_uvw[a:b], src_vis[a:b])
            s.finish(dst)

        def wall(f):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            f()
            torch.cuda.synchronize(dev)
            return (time.perf_counter() - t0) * 1e3

        # warm-up on the first chunks (buffers, FFT plans), then one full pass
        s.predict_begin(h_model)
        s.predict(h_uvw[:parts[0][1]], vis=h_vis[:parts[0][1]])
        for a, b in parts[:2]:
            s.add(h_uvw[a:b], h_vis[a:b])
        s.finish(h_dirty)
        t_d2m_sync = wall(lambda: d2m(h_uvw, h_vis))
        t_d2m = wall(lambda: d2m(h_uvw, h_vis, pipelined=True))
        t_m2d = wall(lambda: m2d(h_uvw, h_vis, h_dirty))
        st = s.stats()
        # accuracy: dirty2ms on 20k visibilities (1250 rows x 16 channels)
        # against the FP64 DFT of the model's pixels (torch, on the GPU)
        sel_rows = rng.choice(nrows, 1250, replace=False)
        nz = np.flatnonzero(model)
        vref = synth.predict_vis(uvw[sel_rows], freq, nx, nx, px, px, nz // nx, nz % nx,
                                 model.ravel()[nz], device=dev)
        out["accuracy"] = {"dirty2ms_rel_rms_vs_dft_20k": rel_rms(h_vis.numpy()[sel_rows], vref)}
        pix = np.concatenate([rng.choice(nz, 4, replace=False), rng.integers(0, nx * nx, 4)])
        out["accuracy"]["ms2dirty_rel_rms_vs_dft_8px"] = rel_rms(
            h_dirty.numpy().ravel()[pix],
            dft_pixels(uvw, freq, h_vis.numpy(), nx, nx, px, px, pix, torch, dev))
        # the streamed ms2dirty again with Briggs(0) imaging weights, looked
        # up on the device while each batch is scanned and recorded; the
        # weight grid is built from every chunk first, as WSClean does
        from wsclean_b200.gridder import ImageWeights
        iw = ImageWeights("briggs", 0.0, nx, nx, px, px, context=ctx)
        try:
            def build_weights():
                for a, b in parts:
                    iw.grid(h_uvw[a:b], freq)
                iw.finish()
            t_wbuild = wall(build_weights)
            s.set_imaging_weights(iw)
            t_m2d_briggs = wall(lambda: m2d(h_uvw, h_vis, h_dirty))
            s.set_imaging_weights(None)
        finally:
            iw.close()
        # the same passes with the data resident in HBM
        d_uvw = h_uvw.to(dev)
        d_vis = h_vis.to(dev)
        d_dirty = torch.empty((nx, nx), dtype=torch.float32, device=dev)
        d_out = torch.empty_like(d_vis)
        r_d2m = wall(lambda: d2m(d_uvw, d_out))
        r_m2d = wall(lambda: m2d(d_uvw, d_vis, d_dirty))
        del d_out, d_dirty
        # plain copies of what the streamed passes move to the device
        t_h2d = wall(lambda: [d_vis[a:b].copy_(h_vis[a:b], non_blocking=True) for a, b in parts]
                     + [d_uvw[a:b].copy_(h_uvw[a:b], non_blocking=True) for a, b in parts])
        del d_uvw, d_vis
    finally:
        s.close()
    torch.cuda.empty_cache()
    g = grids["config5"]["mixed"]
    B = 2 * algorithmic_bytes(nvis, nrows, nx, nx, grid_tuple(g), 8, 8)
    h2d = 2 * h_uvw.numel() * 8 + h_vis.numel() * 8 + h_model.numel() * 4
    d2h = h_vis.numel() * 8 + h_dirty.numel() * 4
    out.update({
        "ms2dirty_mvis_s": nvis / t_m2d / 1e3, "dirty2ms_mvis_s": nvis / t_d2m / 1e3,
        "dirty2ms_synchronous_chunks_mvis_s": nvis / t_d2m_sync / 1e3,
        "ms2dirty_briggs_weights_mvis_s": nvis / t_m2d_briggs / 1e3,
        "briggs_weights_build_ms": t_wbuild,
        "value": nvis / (t_m2d + t_d2m) / 1e3, "ms_per_step": t_m2d + t_d2m,
        "resident_ms2dirty_mvis_s": nvis / r_m2d / 1e3, "resident_dirty2ms_mvis_s": nvis / r_d2m / 1e3,
        "resident_value": nvis / (r_m2d + r_d2m) / 1e3,
        "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
        "h2d_copy_alone_ms": t_h2d,
        "h2d_hidden_fraction": max(0.0, min(1.0, (r_m2d + t_h2d - t_m2d) / t_h2d)),
        "grid": {"nu": st["nu"], "nv": st["nv"], "nplanes": st["nplanes"], "W": st["supp"],
                 "u_band_rows": st["band_rows"]},
        "reference_grid": g, "roofline": roofline(B, t_m2d + t_d2m, "streamed pair"),
        "timing": "wall clock around each full pass, device synchronised on both sides; "
                  "ms2dirty calls return once their chunk is on the device, dirty2ms runs "
                  "pipelined (predictions copied back to page-locked memory while the next "
                  "chunk is computed, all in place at the closing synchronisation; "
                  "dirty2ms_synchronous_chunks: each predict returns with its chunk in place)"})
    # the reference on the first 30% of the timesteps (its FFT work is fixed
    # and its gridding work follows the visibilities: a small sample would
    # understate its rate at full size)
    cpu = None
    if with_cpu:
        r30 = int(0.3 * nrows) // 32640 * 32640
        cpu, _ = cpu_pair(uvw[:r30], freq, h_vis.numpy()[:r30], model32, nx, px, EPS_MIXED,
                          "float", sample="first 300 of 1000 timesteps (156.7M visibilities) of "
                                          "the same data, one ms2dirty + one dirty2ms of ducc0 "
                                          "<float,float>")
    del h_vis, h_uvw
    # tuned against plain on a 2% time subsample
    sub = synth.config5(scale=0.02)
    su, sf = sub["uvw"], sub["freq"]
    sv = (rng.normal(size=(len(su), nchan)) + 1j * rng.normal(size=(len(su), nchan))).astype(np.complex64)
    tu, tf, tv = (torch.as_tensor(su, device=dev), torch.as_tensor(sf, device=dev),
                  torch.as_tensor(sv, device=dev))
    dd = torch.empty((nx, nx), dtype=torch.float32, device=dev)
    tp, tt = device_timed(torch, dev, [
        lambda: ctx.ms2dirty(tu, tf, tv, nx, nx, px, px, EPS_MIXED, dirty=dd, **KW),
        lambda: ctx.ms2dirty(tu, tf, tv, nx, nx, px, px, EPS_MIXED, dirty=dd, tuning=True, **KW)],
        2, 1)
    out["tuned_vs_plain_2pct"] = {"nvis": sv.size, "plain_ms2dirty_ms": tp, "tuned_ms2dirty_ms": tt,
                                  "tuned_subdivision": ctx.last_tuning()}
    del tu, tf, tv, dd
    ctx.release_buffers()
    out["cpu_baseline"] = cpu
    return out


def dft_pixels(uvw, freq, vis, nx, ny, px, py, pix, torch, dev):
    """FP64 direct sum of the ms2dirty image at flat pixel indices (GPU, torch)."""
    from wsclean_b200 import synth
    i, j = pix // ny, pix % ny
    l, m = synth.pixel_lm(i.astype(float), j.astype(float), nx, ny, px, py)
    nm1 = -(l * l + m * m) / (np.sqrt(1 - l * l - m * m) + 1)
    Lm = torch.as_tensor(np.stack([l, -m, -nm1]), dtype=torch.float64, device=dev)
    out = torch.zeros(len(pix), dtype=torch.float64, device=dev)
    U = torch.as_tensor(uvw, dtype=torch.float64, device=dev)
    V = torch.as_tensor(vis, dtype=torch.complex128, device=dev)
    for c, f in enumerate(freq):
        for r0 in range(0, U.shape[0], 1 << 20):
            ph = (U[r0:r0 + (1 << 20)] * (f / synth.C_LIGHT)) @ Lm
            ph = ph - torch.round(ph)
            out += (V[r0:r0 + (1 << 20), c:c + 1] * torch.exp(2j * math.pi * ph)).real.sum(0)
    return out.cpu().numpy()


def rel_rms(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.sqrt(np.sum(np.abs(a - b) ** 2) / np.sum(np.abs(b) ** 2)))


def run_ours(args, world, rank, local, pg):
    import torch
    from wsclean_b200 import synth
    from wsclean_b200.gridder import Context

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    c, ix, iy, flux = workload(args.scale)
    uvw, freq, nx, px = c["uvw"], c["freq"], c["npix_x"], c["pixsize"]
    nrows, nchan = uvw.shape[0], len(freq)
    nvis = nrows * nchan
    vis64 = synth.predict_vis(uvw, freq, nx, nx, px, px, ix, iy, flux, device=dev)
    noise = np.random.default_rng(3).normal(size=vis64.shape) * 0.1
    vis64 = vis64 + noise + 1j * np.random.default_rng(4).normal(size=vis64.shape) * 0.1
    model = synth.sky_image(nx, nx, ix, iy, flux)

    ctx = Context(local)
    kw = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)
    d_uvw = torch.as_tensor(uvw, device=dev)
    d_freq = torch.as_tensor(freq, device=dev)
    forms = {
        "mixed": dict(eps=EPS_MIXED, vis=torch.as_tensor(vis64.astype(np.complex64), device=dev),
                      model=torch.as_tensor(model.astype(np.float32), device=dev),
                      dirty=torch.zeros((nx, nx), dtype=torch.float32, device=dev),
                      out=torch.zeros((nrows, nchan), dtype=torch.complex64, device=dev)),
        "fp64": dict(eps=EPS_FP64, vis=torch.as_tensor(vis64, device=dev),
                     model=torch.as_tensor(model, device=dev),
                     dirty=torch.zeros((nx, nx), dtype=torch.float64, device=dev),
                     out=torch.zeros((nrows, nchan), dtype=torch.complex128, device=dev)),
    }
    # the plain FP64 form at the mixed form's accuracy (same buffers)
    forms["fp64_eps_mixed"] = dict(forms["fp64"], eps=EPS_MIXED, prec="fp64")
    stream = torch.cuda.current_stream(dev)

    def call_pair(form, f):
        ctx.ms2dirty(d_uvw, d_freq, f["vis"], nx, nx, px, px, f["eps"], precision=f.get("prec", form),
                     dirty=f["dirty"], **kw)
        st1 = ctx.stats()
        ctx.dirty2ms(d_uvw, d_freq, f["model"], px, px, f["eps"], precision=f.get("prec", form), vis=f["out"], **kw)
        st2 = ctx.stats()
        return st1, st2

    def barrier():
        torch.cuda.synchronize(dev)
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize(dev)

    def timed(form, steps, warmup):
        f = forms[form]
        for _ in range(warmup):
            call_pair(form, f)
        barrier()
        # no Python garbage-collector pauses inside the timed steps (the
        # device clock would count them as idle time)
        gc.collect()
        gc.disable()
        t_ms = t_dm = 0.0
        phases = {}
        l0 = ctx.stats()["kernel_launches"]
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        step_ms = []
        for _ in range(steps):
            # the library runs on its own stream and synchronises before
            # returning, so events on the current stream bracket each call
            ev[0].record(stream)
            st1 = None
            ctx.ms2dirty(d_uvw, d_freq, f["vis"], nx, nx, px, px, f["eps"], precision=f.get("prec", form),
                         dirty=f["dirty"], **kw)
            ev[1].record(stream)
            st1 = ctx.stats()
            ctx.dirty2ms(d_uvw, d_freq, f["model"], px, px, f["eps"], precision=f.get("prec", form),
                         vis=f["out"], **kw)
            ev[2].record(stream)
            st2 = ctx.stats()
            torch.cuda.synchronize(dev)
            t_ms += ev[0].elapsed_time(ev[1])
            t_dm += ev[1].elapsed_time(ev[2])
            step_ms.append(round(ev[0].elapsed_time(ev[2]), 3))
            for k in ("ms_prep", "ms_grid", "ms_fft", "ms_screen", "ms_total"):
                phases.setdefault("ms2dirty_" + k, []).append(st1[k])
                phases.setdefault("dirty2ms_" + k, []).append(st2[k])
        gc.enable()
        barrier()
        launches = ctx.stats()["kernel_launches"] - l0
        tt = torch.tensor([t_ms, t_dm], dtype=torch.float64, device=dev)
        if pg is not None:
            pg.all_reduce(tt, op=pg.ReduceOp.MAX)
        t_ms, t_dm = float(tt[0]), float(tt[1])
        phases = {k: statistics.median(v) for k, v in phases.items()}
        return t_ms, t_dm, phases, launches, st1, st2, step_ms

    # ---- timed region (mixed, the headline)
    sampler = ClockSampler(local)
    if not args.no_clocks:
        sampler.start()
    t_ms, t_dm, phases, launches, st1, st2, step_ms = timed("mixed", args.steps, args.warmup)
    clocks = sampler.stop()
    ms_per_step = (t_ms + t_dm) / args.steps
    value = world * nvis * args.steps / ((t_ms + t_dm) / 1e3) / 1e6
    grid_info = {"nu": st1["nu"], "nv": st1["nv"], "nplanes": st1["nplanes"], "W": st1["supp"],
                 "sigma": round(st1["sigma"], 4), "u_band_rows": st1["band_rows"]}

    if args.timed_only:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup,
                              "ms_per_step": ms_per_step, "step_ms": step_ms,
                              "timed_only": True, "scale": args.scale, "grid": grid_info,
                              "phases_ms": phases, "gpu_launches": launches}))
        ctx.close()
        return

    # ---- FP64 plain form (same workload)
    fp64 = None
    if not args.no_fp64:
        k64 = max(2, args.steps // 3)
        t64_ms, t64_dm, ph64, _, s64, _, _ = timed("fp64", k64, 1)
        fp64 = {"value": world * nvis * k64 / ((t64_ms + t64_dm) / 1e3) / 1e6,
                "ms2dirty_mvis_s": world * nvis * k64 / (t64_ms / 1e3) / 1e6,
                "dirty2ms_mvis_s": world * nvis * k64 / (t64_dm / 1e3) / 1e6,
                "ms_per_step": (t64_ms + t64_dm) / k64,
                "grid": {"nu": s64["nu"], "nplanes": s64["nplanes"], "W": s64["supp"]}}
        # the same FP64 form at the mixed form's accuracy (epsilon 1e-5)
        t5_ms, t5_dm, _, _, s5, _, _ = timed("fp64_eps_mixed", k64, 1)
        fp64["at_eps_mixed"] = {
            "eps": EPS_MIXED, "value": world * nvis * k64 / ((t5_ms + t5_dm) / 1e3) / 1e6,
            "ms_per_step": (t5_ms + t5_dm) / k64,
            "grid": {"nu": s5["nu"], "nplanes": s5["nplanes"], "W": s5["supp"]}}

    # ---- accuracy (outside the timed region): FP64 direct sums
    rng = np.random.default_rng(99)
    acc = {}
    pix = rng.integers(0, nx * nx, 64)
    vsel = rng.choice(nvis, 10000, replace=False)
    dft_img = dft_pixels(uvw, freq, vis64, nx, nx, px, px, pix, torch, dev)
    dft_vis = synth.predict_vis(uvw[vsel // nchan], freq, nx, nx, px, px, ix, iy, flux,
                                device=dev)[:, 0] if nchan == 1 else None
    for form in ("mixed",) + (() if args.no_fp64 else ("fp64",)):
        f = forms[form]
        call_pair(form, f)
        torch.cuda.synchronize(dev)
        img = f["dirty"].double().cpu().numpy().ravel()[pix]
        acc[form] = {"ms2dirty_rel_rms_vs_dft": rel_rms(img, dft_img)}
        if dft_vis is not None:
            acc[form]["dirty2ms_rel_rms_vs_dft"] = rel_rms(
                f["out"].cpu().numpy().ravel()[vsel], dft_vis)
        # adjointness: |<y, A x> - <A^H y, x>| / (|y| |A x|)
        g = torch.Generator(device="cpu").manual_seed(5)
        x = torch.randn((nx, nx), generator=g, dtype=torch.float64).to(dev)
        y = (torch.randn((nrows, nchan), generator=g, dtype=torch.float64)
             + 1j * torch.randn((nrows, nchan), generator=g, dtype=torch.float64)).to(dev)
        Ax = ctx.dirty2ms(d_uvw, d_freq, x, px, px, f["eps"], precision=f.get("prec", form),
                          vis_dtype=np.complex128, **kw)
        Aty = ctx.ms2dirty(d_uvw, d_freq, y, nx, nx, px, px, f["eps"], precision=f.get("prec", form),
                           dirty_dtype=np.float64, **kw)
        a = torch.vdot(y.ravel(), Ax.ravel()).real.item()
        b = torch.vdot(Aty.ravel().to(torch.complex128), x.ravel().to(torch.complex128)).real.item()
        acc[form]["adjoint_mismatch"] = abs(a - b) / (y.norm().item() * Ax.norm().item())
        del x, y, Ax, Aty

    # ---- end to end from pinned host buffers through the public API
    h_uvw = torch.as_tensor(uvw).pin_memory()
    h_freq = torch.as_tensor(freq)
    h_vis = forms["mixed"]["vis"].cpu().pin_memory()
    h_model = forms["mixed"]["model"].cpu().pin_memory()
    h_dirty = torch.zeros((nx, nx), dtype=torch.float32).pin_memory()
    h_out = torch.zeros((nrows, nchan), dtype=torch.complex64).pin_memory()

    def e2e_step():
        ctx.ms2dirty(h_uvw, h_freq, h_vis, nx, nx, px, px, EPS_MIXED, precision="mixed",
                     dirty=h_dirty, **kw)
        ctx.dirty2ms(h_uvw, h_freq, h_model, px, px, EPS_MIXED, precision="mixed", vis=h_out, **kw)

    def e2e_run(pipelined):
        # pipelined: the context's asynchronous mode, in which consecutive
        # calls overlap their host transfers with each other's kernels
        ctx.set_async(pipelined)
        for _ in range(max(1, args.warmup)):
            e2e_step()
        ctx.synchronize()
        barrier()
        gc.collect()
        gc.disable()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        ctx.synchronize()
        torch.cuda.synchronize(dev)
        t = time.perf_counter() - t0
        gc.enable()
        ctx.set_async(False)
        te = torch.tensor([t], dtype=torch.float64, device=dev)
        if pg is not None:
            pg.all_reduce(te, op=pg.ReduceOp.MAX)
        return world * nvis * args.steps / float(te[0]) / 1e6

    e2e_sync = e2e_run(False)
    e2e_val = e2e_run(True)
    h2d = 2 * h_uvw.numel() * 8 + h_vis.numel() * 8 + h_model.numel() * 4 + 2 * nchan * 8
    d2h = h_dirty.numel() * 4 + h_out.numel() * 8

    # ---- CPU baseline (reference, rank 0, N=1), with the reference's grid
    # choice for the roofline from its verbosity report
    grids = ducc_grids()
    cpu, ref_grid = None, None
    with_cpu = rank == 0 and world == 1 and not args.no_cpu_baseline
    if with_cpu:
        try:
            cpu, ref_grid = cpu_pair(
                uvw, freq, forms["mixed"]["vis"].cpu().numpy(), forms["mixed"]["model"].cpu().numpy(),
                nx, px, EPS_MIXED, "float",
                sample="full workload, one ms2dirty + one dirty2ms, ducc0 <float,float> at eps "
                       "1e-5 with WSClean's arguments")
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"}
    ref_grid = ref_grid or grids["config2"]["mixed"]

    # ---- roofline of the pipeline (algorithmic bytes, the reference's grid)
    B = algorithmic_bytes(nvis, nrows, nx, nx, grid_tuple(ref_grid), 8, 8) * 2
    rl = roofline(B, ms_per_step, "ms2dirty+dirty2ms pipeline")
    rl["traffic"] = profiled_traffic()
    rl["reference_grid"] = ref_grid

    # ---- the other configurations (rank 0 only: they are single-GPU legs)
    legs = {}
    want = set(x.strip() for x in args.legs.split(",") if x.strip())
    if args.no_batch:
        want.discard("4")
    del forms, h_vis, h_out, h_model, h_dirty, d_uvw, d_freq
    ctx.release_buffers()
    torch.cuda.empty_cache()
    if rank == 0:
        for name, fn in (("1", lambda: leg_config1(torch, dev, ctx, grids, with_cpu)),
                         ("3", lambda: leg_config3(torch, dev, ctx, grids, with_cpu)),
                         ("4", lambda: run_batched(dev, torch, ctx, args)),
                         ("5", lambda: leg_config5(torch, dev, ctx, grids, with_cpu, args))):
            if name not in want:
                continue
            try:
                legs["config" + name] = fn()
            except Exception as e:  # reported, not fatal
                legs["config" + name] = {"error": f"{type(e).__name__}: {e}"}
            ctx.release_buffers()
            gc.collect()
            torch.cuda.empty_cache()

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 coords/phase/accumulate)",
            "data": "synthetic (seeded Earth-rotation observation, 200 point sources)",
            "config": config2_dict(nvis, nx, world),
            "grid": grid_info,
            "ms2dirty_mvis_s": world * nvis * args.steps / (t_ms / 1e3) / 1e6,
            "dirty2ms_mvis_s": world * nvis * args.steps / (t_dm / 1e3) / 1e6,
            "fp64": fp64,
            "mixed_over_fp64": (value / fp64["value"]) if fp64 else None,
            "mixed_over_fp64_same_eps": (value / fp64["at_eps_mixed"]["value"]) if fp64 else None,
            "accuracy": acc,
            "phases_ms": phases,
            "step_ms": step_ms,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h),
                    "mode": "pipelined calls (wsg_ctx_set_async), pinned host buffers",
                    "synchronous_calls_value": e2e_sync},
            "roofline": rl,
            "cpu_baseline": cpu,
            "configs": legs,
            "clocks": clocks,
            "gpu_launches": launches,
        }
        print(json.dumps(out))
    ctx.close()


def main():
    args = parse_args()
    if args.launch_summary:
        launch_summary(args.launch_summary, args.steps)
        return
    world, rank, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
