"""Concurrent gridders on one GPU, as WSClean runs them with
-parallel-gridding N: each scheduler worker thread owns its own gridder
(threadedscheduler.cpp:54-58), so several contexts -- each with its own
stream, buffers and cuFFT plans -- run at the same time from different host
threads.  The results must equal those of the same calls made one after the
other (FP64: to rounding; mixed: to FP32 summation order, the spreading
atomics add in any order).
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KW = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)


def problem(seed, nrow=40000, nchan=4, nx=256, ny=192):
    rng = np.random.default_rng(seed)
    px = np.deg2rad(20.0 / 3600)
    freq = np.linspace(1.3e8, 1.6e8, nchan)
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([1500.0, 1500.0, 300.0])
    vis = rng.normal(size=(nrow, nchan)) + 1j * rng.normal(size=(nrow, nchan))
    model = rng.normal(size=(nx, ny))
    return dict(uvw=uvw, freq=freq, vis=vis, model=model, nx=nx, ny=ny, px=px)


def run(ctx, p, prec, eps):
    d = ctx.ms2dirty(p["uvw"], p["freq"], p["vis"], p["nx"], p["ny"], p["px"], p["px"], eps,
                     precision=prec, dirty_dtype=np.float64, **KW)
    v = ctx.dirty2ms(p["uvw"], p["freq"], p["model"], p["px"], p["px"], eps, precision=prec,
                     vis_dtype=np.complex128, **KW)
    return d, v


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("prec,eps,tol", [("fp64", 1e-12, 1e-12), ("mixed", 1e-5, 5e-6)])
def test_threads_with_own_contexts_match_sequential(prec, eps, tol):
    from wsclean_b200.gridder import Context
    nthreads, reps = 4, 3
    probs = [problem(100 + i) for i in range(nthreads)]
    seq_ctx = Context(0)
    expect = [run(seq_ctx, p, prec, eps) for p in probs]
    results = [[None] * reps for _ in range(nthreads)]
    errors = []
    start = threading.Barrier(nthreads)

    def worker(i):
        try:
            ctx = Context(0)
            start.wait(timeout=60)
            for r in range(reps):
                results[i][r] = run(ctx, probs[i], prec, eps)
        except Exception as e:  # reported by the main thread
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(nthreads)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads), "a gridding thread did not finish"
    assert not errors, errors
    for i in range(nthreads):
        for r in range(reps):
            d, v = results[i][r]
            assert rel(d, expect[i][0]) < tol, (i, r, rel(d, expect[i][0]))
            assert rel(v, expect[i][1]) < tol, (i, r, rel(v, expect[i][1]))


def test_threads_with_dropin_gridders():
    """The WGriddingGridder mirror, one per thread: chunked inversion and
    prediction running concurrently give the single-thread images."""
    from wsclean_b200.gridder import WGriddingGridder
    nthreads = 3
    probs = [problem(200 + i, nrow=20000, nchan=2, nx=128, ny=128) for i in range(nthreads)]

    def image_of(p):
        g = WGriddingGridder(p["nx"], p["ny"], p["nx"], p["ny"], p["px"], p["px"], 0.0, 0.0,
                             epsilon=1e-5)
        try:
            g.InitializeInversion()
            half = p["uvw"].shape[0] // 2
            g.AddInversionData(p["uvw"][:half], p["freq"], p["vis"][:half])
            g.AddInversionData(p["uvw"][half:], p["freq"], p["vis"][half:])
            g.FinalizeImage(1.0)
            img = g.RealImage().astype(np.float64)
            g.InitializePrediction(np.ascontiguousarray(p["model"].T))  # [y, x]
            vis = g.PredictVisibilities(p["uvw"], p["freq"]).astype(np.complex128)
        finally:
            g.close()
        return img, vis

    expect = [image_of(p) for p in probs]
    got = [None] * nthreads
    errors = []

    def worker(i):
        try:
            got[i] = image_of(probs[i])
        except Exception as e:
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(nthreads)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads)
    assert not errors, errors
    for i in range(nthreads):
        assert rel(got[i][0], expect[i][0]) < 1e-5
        assert rel(got[i][1], expect[i][1]) < 1e-5
