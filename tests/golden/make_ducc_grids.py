"""Writes tests/golden/ducc_grids.json: the grid (nu x nv x nplanes, support W)
that the reference w-gridder chooses for each benchmark configuration, from
its verbosity-1 report (ducc0 Params, wgridder.h:1535-1560), run through the
compiled reference (oracle/_ref) on the seeded synthetic data of
wsclean_b200.synth with WSClean's argument pattern.

The benchmark's roofline charges the algorithmic bytes of these grids (not of
this library's own, smaller, band-pruned grids), so that the figure does not
depend on the library's tuning.  bench.py re-derives the config-2 entry from
the report of its own CPU-baseline run when that runs; tests/test_oracle.py
checks the config-2 entries against the reference again.

Run on a machine with many cores (the config-5 run grids 522M visibilities
on the CPU, a few minutes on 16 cores):

    python tests/golden/make_ducc_grids.py [configs...]   (default: 1 2 3 5)
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from wsclean_b200 import synth  # noqa: E402

KW = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)
OUT = os.path.join(HERE, "ducc_grids.json")


def grid_of(uvw, freq, vis, nx, px, eps, prec, wgt=None):
    t0 = time.time()
    _, rep = O.ref_ms2dirty(uvw, freq, vis, nx, nx, px, px, eps, prec=prec, wgt=wgt,
                            return_report=True, **KW)
    g = O.parse_report(rep)[0]
    g["cpu_s"] = round(time.time() - t0, 2)
    return g


def noise_vis(shape, dtype, seed):
    rng = np.random.default_rng(seed)
    return (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(dtype)


def main(which):
    res = json.load(open(OUT)) if os.path.exists(OUT) else {}
    # the grid depends on the coordinates, the image and the active count,
    # not on the visibility values: seeded noise stands in for the sky
    if "1" in which:
        c = synth.config1()
        v = noise_vis((len(c["uvw"]), len(c["freq"])), np.complex128, 1)
        res["config1"] = {"fp64": grid_of(c["uvw"], c["freq"], v, c["npix_x"], c["pixsize"],
                                          1e-12, "double")}
    if "2" in which:
        c = synth.config2()
        v = noise_vis((len(c["uvw"]), 1), np.complex64, 2)
        res["config2"] = {
            "mixed": grid_of(c["uvw"], c["freq"], v, c["npix_x"], c["pixsize"], 1e-5, "float"),
            "fp64": grid_of(c["uvw"], c["freq"], v.astype(np.complex128), c["npix_x"],
                            c["pixsize"], 1e-12, "double")}
    if "3" in which:
        c = synth.config3()
        v = noise_vis((len(c["uvw"]), 1), np.complex64, 3)
        w = np.random.default_rng(3).uniform(0.5, 2.0, v.shape).astype(np.float32)
        res["config3"] = {"mixed": grid_of(c["uvw"], c["freq"], v, c["npix_x"], c["pixsize"],
                                           1e-5, "float", wgt=w)}
    if "5" in which:
        c = synth.config5()
        v = noise_vis((len(c["uvw"]), len(c["freq"])), np.complex64, 5)
        res["config5"] = {"mixed": grid_of(c["uvw"], c["freq"], v, c["npix_x"], c["pixsize"],
                                           1e-5, "float")}
    res["_note"] = ("grid chosen by the reference (compiled oracle/_ref, verbosity report) on the "
                    "seeded synthetic data; written by tests/golden/make_ducc_grids.py")
    with open(OUT, "w") as fh:
        json.dump(res, fh, indent=1, sort_keys=True)
    print(json.dumps(res, indent=1, sort_keys=True))


if __name__ == "__main__":
    main(sys.argv[1:] or ["1", "2", "3", "5"])
