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
# Grid chosen by the reference (ducc0) for this workload, from its verbosity-1
# report (oracle/_ref run on the same seeded data): mixed eps 1e-5 -> 7392^2 x
# 14 planes; FP64 eps 1e-12 -> 7392^2 x 22 planes.  Used only for the
# algorithmic-bytes roofline so that it does not depend on this library's
# own (smaller) grid choice.
DUCC_GRID = {"mixed": (7392, 7392, 14), "fp64": (7392, 7392, 22)}


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
        "config": {"workload": "config-2 adjoint pair: 8.1M vis, 4096^2 @ 5\", eps 1e-5",
                   "nvis": nvis, "npix": nx, "instance": "ducc0 <float,float>",
                   "wsclean_args": "negate_v, no divide_by_n, sigma 1.1..2.0"},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": "full workload per step (one ms2dirty + one dirty2ms)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def run_batched(dev, torch, ctx, args):
    """Config 4: 16 Voronoi facets x 8 output channels (8 of 64 input
    channels each) = 128 jobs over the same rows, gridded and degridded
    through one reusable plan (one persistent spread / interpolation launch
    per call, replayed as a CUDA graph), against the plain FP64 form run job
    by job (timed on the first 16 jobs and scaled to all 128)."""
    from wsclean_b200 import synth
    from wsclean_b200 import gridder as G
    c = synth.config4()
    uvw, freq, px = c["uvw"], c["freq"], c["pixsize"]
    nrows = uvw.shape[0]
    jobs = [dict(npix_x=f["nx"], npix_y=f["ny"], center_x=f["dx"] * px, center_y=f["dy"] * px,
                 chan_begin=8 * oc, chan_end=8 * oc + 8)
            for oc in range(8) for f in synth.facets4()]
    kw = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)
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
    # plain FP64 form, job by job
    vis64 = vis.to(torch.complex128)
    del vis
    tu = torch.as_tensor(uvw, device=dev)
    tf = torch.as_tensor(freq, device=dev)
    sub = jobs[:16]
    t64 = 0.0
    for rep in range(2):   # the first pass creates the FFT plans of each facet size
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for j in sub:
            c0, c1 = j["chan_begin"], j["chan_end"]
            ctx.ms2dirty(tu, tf[c0:c1], vis64[:, c0:c1].contiguous(), j["npix_x"], j["npix_y"],
                         px, px, EPS_FP64, precision="fp64", center_x=j["center_x"],
                         center_y=j["center_y"], dirty_dtype=np.float64, **kw)
        torch.cuda.synchronize(dev)
        t64 = (time.perf_counter() - t0) / len(sub) * len(jobs) * 1e3
    del vis64
    return {"workload": "config 4: 96 antennas within 10 km, 360 x 10 s, 64 channels 120-180 MHz; "
                        "16 Voronoi facets (512^2..2048^2, phase centre at the box centre) x 8 "
                        "output channels = 128 jobs",
            "rows": nrows, "job_visibilities": jv, "plan_build_s": t_build, "W": W,
            "mixed_ms2dirty_ms": tg, "mixed_dirty2ms_ms": td,
            "mixed_ms2dirty_mvis_s": jv / tg / 1e3, "mixed_dirty2ms_mvis_s": jv / td / 1e3,
            "fp64_per_job_ms2dirty_ms": t64, "fp64_per_job_ms2dirty_mvis_s": jv / t64 / 1e3,
            "mixed_batched_over_fp64_per_job": t64 / tg,
            "fp64_timing": "16 of 128 jobs timed (warm FFT plans), scaled to 128"}


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

    # ---- config 4: batched facets x output channels through one plan
    batched = None
    if not args.no_batch:
        try:
            batched = run_batched(dev, torch, ctx, args)
        except Exception as e:  # reported, not fatal
            batched = {"error": str(e)}
        torch.cuda.empty_cache()

    # ---- roofline of the pipeline (algorithmic bytes, the reference's grid)
    B = (algorithmic_bytes(nvis, nrows, nx, nx, DUCC_GRID["mixed"], 8, 8) * 2)
    achieved = B / (ms_per_step / 1e3) / 1e9
    peaks_path = os.path.join(HERE, "MEASURED_PEAKS.json")
    peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        with open(peaks_path) as fh:
            peak, peak_src = float(json.load(fh)["hbm_gbs"]), "measured"

    # ---- CPU baseline (reference, rank 0, N=1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            import oracle as O
            if O.ref_available():
                cores = os.cpu_count()
                vis32 = forms["mixed"]["vis"].cpu().numpy()
                m32 = forms["mixed"]["model"].cpu().numpy()
                rk = dict(prec="float", negate_v=True, divide_by_n=False, sigma_min=1.1,
                          sigma_max=2.0, nthreads=cores)
                t0 = time.perf_counter()
                O.ref_ms2dirty(uvw, freq, vis32, nx, nx, px, px, EPS_MIXED, **rk)
                O.ref_dirty2ms(uvw, freq, m32, px, px, EPS_MIXED, **rk)
                tc = time.perf_counter() - t0
                cpu = {"value": nvis / tc / 1e6, "unit": UNIT, "cores": cores, "kind": "reference",
                       "sample": "full workload, one ms2dirty + one dirty2ms, ducc0 <float,float> "
                                 "at eps 1e-5 with WSClean's arguments"}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 coords/phase/accumulate)",
            "data": "synthetic (seeded Earth-rotation observation, 200 point sources)",
            "config": {"workload": "config-2 adjoint pair: 8.1M vis, 4096^2 @ 5\", eps 1e-5",
                       "nvis": nvis, "npix": nx, "parallelism": f"replicas x{world}",
                       "l2": "inputs and grids larger than L2 (uvw 194 MB, grids GBs)",
                       "grid": grid_info},
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
            "roofline": {"bound": "hbm", "kernel": "ms2dirty+dirty2ms pipeline",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profiled_traffic(),
                         "peak_source": peak_src,
                         "bytes_per_step": B},
            "cpu_baseline": cpu,
            "batched_facets": batched,
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
