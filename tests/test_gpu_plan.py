"""Reusable plans and batched jobs (wsg_plan_*): a plan built once for fixed
coordinates and run on new visibilities / images, one job or a batch of
facets x output channels drained by a single persistent spread /
interpolation launch, replayed from a CUDA graph, and recorded inside a
torch.cuda.graph major cycle (predict -> residual -> invert).

Tolerances: a single-job plan uses the same grid as the raw call, so the two
agree to rounding (atomics reorder sums); batch jobs share the largest job's
kernel, so against the raw per-job calls and the DFT they agree to epsilon."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu
KW = dict(negate_v=True, divide_by_n=False, sigma_min=1.1, sigma_max=2.0)
DEV = torch.device("cuda", 0)


def problem(seed, nrow=6000, nchan=6):
    rng = np.random.default_rng(seed)
    px = np.deg2rad(30 / 3600)
    freq = np.linspace(1.4e8, 1.6e8, nchan)
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([800.0, 800.0, 250.0])
    vis = rng.normal(size=(nrow, nchan)) + 1j * rng.normal(size=(nrow, nchan))
    return rng, uvw, freq, vis, px


@pytest.mark.parametrize("prec,eps,tol", [("mixed", 1e-5, 1e-6), ("fp64", 1e-12, 1e-12)])
def test_single_job_plan_matches_raw_calls(prec, eps, tol):
    from wsclean_b200 import gridder as G
    rng, uvw, freq, vis, px = problem(1)
    wgt = rng.uniform(0.5, 2.0, vis.shape)
    mask = (rng.uniform(size=vis.shape) > 0.1).astype(np.uint8)
    vdt = np.complex64 if prec == "mixed" else np.complex128
    nx, ny = 96, 80
    with G.Plan(uvw, freq, px, px, eps, nx, ny, wgt=wgt, mask=mask, precision=prec,
                vis_dtype=vdt, dirty_dtype=np.float64, center_x=2 * px, center_y=-px,
                **KW) as plan:
        tv = torch.as_tensor(vis.astype(vdt), device=DEV)
        d = plan.ms2dirty(tv)[0]
        torch.cuda.synchronize()
        raw = G.ms2dirty(uvw, freq, vis.astype(vdt), nx, ny, px, px, eps, wgt=wgt, mask=mask,
                         precision=prec, dirty_dtype=np.float64, center_x=2 * px,
                         center_y=-px, **KW)
        assert O.rel_rms(d.cpu().numpy(), raw) < tol
        model = torch.as_tensor(rng.normal(size=(nx, ny)), device=DEV)
        v = plan.dirty2ms(model)
        torch.cuda.synchronize()
        rawv = G.dirty2ms(uvw, freq, model.cpu().numpy(), px, px, eps, wgt=wgt, mask=mask,
                          precision=prec, vis_dtype=vdt, center_x=2 * px, center_y=-px, **KW)
        assert O.rel_rms(v.cpu().numpy(), rawv) < tol
        st = plan.stats(0)
        assert st["nvis"] == int(np.count_nonzero(mask)) and st["nplanes"] > 1


def test_repeated_calls_replay_a_graph():
    from wsclean_b200 import gridder as G
    rng, uvw, freq, vis, px = problem(2)
    s = torch.cuda.Stream(DEV)
    with torch.cuda.stream(s), G.Plan(uvw, freq, px, px, 1e-5, 64, 64, **KW) as plan:
        tv = torch.as_tensor(vis.astype(np.complex64), device=DEV)
        out = torch.zeros((64, 64), dtype=torch.float32, device=DEV)
        first = None
        for it in range(4):   # eager, recorded + replayed, replayed, replayed
            plan.ms2dirty(tv, out)
            s.synchronize()
            if first is None:
                first = out.clone()
            else:
                assert torch.allclose(out, first, rtol=0, atol=1e-5 * first.abs().max().item())
            tv.mul_(1.0)   # same pointers, new call
        # new values through the same recorded graph
        tv.mul_(2.0)
        plan.ms2dirty(tv, out)
        s.synchronize()
        assert torch.allclose(out, 2 * first, rtol=0, atol=1e-5 * first.abs().max().item())


def facet_jobs(px):
    # three facets of different sizes and phase centres x two output channels
    facets = [dict(npix_x=64, npix_y=96, center_x=-40 * px, center_y=25 * px),
              dict(npix_x=128, npix_y=128, center_x=0.0, center_y=0.0),
              dict(npix_x=80, npix_y=48, center_x=70 * px, center_y=-60 * px)]
    jobs = []
    for c0, c1 in ((0, 3), (3, 6)):
        for f in facets:
            jobs.append(dict(f, chan_begin=c0, chan_end=c1))
    return jobs


@pytest.mark.parametrize("prec,eps", [("mixed", 1e-5), ("fp64", 1e-10)])
def test_batched_facets_against_dft_and_raw(prec, eps):
    from wsclean_b200 import gridder as G
    rng, uvw, freq, vis, px = problem(3)
    vdt = np.complex64 if prec == "mixed" else np.complex128
    tol = 1e-5 if prec == "mixed" else 1e-9
    jobs = facet_jobs(px)
    with G.Plan(uvw, freq, px, px, eps, jobs=jobs, precision=prec, vis_dtype=vdt,
                dirty_dtype=np.float64, **KW) as plan:
        imgs = plan.ms2dirty(torch.as_tensor(vis.astype(vdt), device=DEV))
        torch.cuda.synchronize()
        Ws = {plan.stats(j)["supp"] for j in range(len(jobs))}
        assert len(Ws) == 1   # one shared kernel
        for j, job in enumerate(jobs):
            fr = freq[job["chan_begin"]:job["chan_end"]]
            vj = vis[:, job["chan_begin"]:job["chan_end"]]
            d = imgs[j].cpu().numpy()
            ref = O.dft_ms2dirty(uvw, fr, vj, job["npix_x"], job["npix_y"], px, px,
                                 negate_v=True, divide_by_n=False, center_x=job["center_x"],
                                 center_y=job["center_y"])
            assert O.rel_rms(d, ref) < tol, j
            raw = G.ms2dirty(uvw, fr, vj.astype(vdt), job["npix_x"], job["npix_y"], px, px, eps,
                             precision=prec, dirty_dtype=np.float64, center_x=job["center_x"],
                             center_y=job["center_y"], **KW)
            assert O.rel_rms(d, raw) < 2 * tol, j
        # prediction: facets of the same channels add up
        models = [np.zeros((j["npix_x"], j["npix_y"])) for j in jobs]
        for m in models:
            m[rng.integers(0, m.shape[0], 5), rng.integers(0, m.shape[1], 5)] = rng.uniform(1, 2, 5)
        v = plan.dirty2ms([torch.as_tensor(m, device=DEV) for m in models])
        torch.cuda.synchronize()
        want = np.zeros(vis.shape, dtype=np.complex128)
        for j, job in enumerate(jobs):
            c0, c1 = job["chan_begin"], job["chan_end"]
            want[:, c0:c1] += O.dft_dirty2ms(uvw, freq[c0:c1], models[j], px, px, negate_v=True,
                                             divide_by_n=False, center_x=job["center_x"],
                                             center_y=job["center_y"])
        assert O.rel_rms(v.cpu().numpy(), want) < tol


def test_batched_plan_is_adjoint():
    from wsclean_b200 import gridder as G
    rng, uvw, freq, vis, px = problem(4)
    jobs = facet_jobs(px)
    with G.Plan(uvw, freq, px, px, 1e-10, jobs=jobs, precision="fp64", vis_dtype=np.complex128,
                dirty_dtype=np.float64, **KW) as plan:
        y = torch.as_tensor(vis, device=DEV)
        xs = [torch.as_tensor(rng.normal(size=(j["npix_x"], j["npix_y"])), device=DEV) for j in jobs]
        Ax = plan.dirty2ms(xs)
        Aty = plan.ms2dirty(y)
        torch.cuda.synchronize()
        a = torch.vdot(y.ravel(), Ax.ravel()).real.item()
        b = sum(torch.sum(t * x).item() for t, x in zip(Aty, xs))
        assert abs(a - b) / (y.norm().item() * Ax.norm().item()) < 1e-12


def test_major_cycle_in_torch_cuda_graph():
    from wsclean_b200 import gridder as G
    rng, uvw, freq, vis, px = problem(5)
    jobs = facet_jobs(px)[:3]
    for j in jobs:
        j["chan_begin"], j["chan_end"] = 0, len(freq)
    data = torch.as_tensor(vis.astype(np.complex64), device=DEV)
    models = [torch.as_tensor(rng.normal(size=(j["npix_x"], j["npix_y"])).astype(np.float32),
                              device=DEV) for j in jobs]
    with G.Plan(uvw, freq, px, px, 1e-5, jobs=jobs, **KW) as plan:
        pred = torch.empty_like(data)
        resid = torch.empty_like(data)
        dirty = [torch.empty((j["npix_x"], j["npix_y"]), device=DEV) for j in jobs]

        def cycle():
            plan.dirty2ms(models, pred)
            torch.sub(data, pred, out=resid)
            plan.ms2dirty(resid, dirty)

        s = torch.cuda.Stream(DEV)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            cycle()   # eager warm-up (launch attributes)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        eager = [d.clone() for d in dirty]
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            cycle()
        for d in dirty:
            d.zero_()
        g.replay()
        torch.cuda.synchronize()
        for d, e in zip(dirty, eager):
            assert torch.allclose(d, e, rtol=0, atol=1e-5 * e.abs().max().item())
        # a new model through the recorded cycle
        for m in models:
            m.mul_(0.5)
        g.replay()
        torch.cuda.synchronize()
        plan.dirty2ms(models, pred)
        torch.sub(data, pred, out=resid)
        ref = plan.ms2dirty(resid)
        torch.cuda.synchronize()
        for d, e in zip(dirty, ref):
            assert torch.allclose(d, e, rtol=0, atol=1e-5 * e.abs().max().item())
        del g


def test_plan_rejects_host_memory_and_bad_jobs():
    from wsclean_b200 import gridder as G
    from wsclean_b200 import _lib as L
    rng, uvw, freq, vis, px = problem(6)
    with G.Plan(uvw, freq, px, px, 1e-5, 64, 64, **KW) as plan:
        with pytest.raises(ValueError):
            plan.ms2dirty(vis.astype(np.complex64))
    with pytest.raises(L.InvalidArgument):
        G.Plan(uvw, freq, px, px, 1e-5, jobs=[dict(npix_x=63, npix_y=64)], **KW)
    with pytest.raises(L.InvalidArgument):
        G.Plan(uvw, freq, px, px, 1e-5, jobs=[dict(npix_x=64, npix_y=64, chan_begin=4,
                                                   chan_end=9)], **KW)


def test_plan_jobs_without_data():
    """A job whose channels are all flagged images to zero and predicts
    nothing; the shared kernel then comes from the largest job with data."""
    from wsclean_b200 import gridder as G
    rng, uvw, freq, vis, px = problem(7)
    mask = np.ones(vis.shape, np.uint8)
    mask[:, 3:] = 0   # channels 3..5 flagged
    jobs = [dict(npix_x=128, npix_y=128, chan_begin=3, chan_end=6),   # largest, no data
            dict(npix_x=64, npix_y=64, chan_begin=0, chan_end=3)]
    with G.Plan(uvw, freq, px, px, 1e-5, jobs=jobs, mask=mask, dirty_dtype=np.float64,
                **KW) as plan:
        imgs = plan.ms2dirty(torch.as_tensor(vis.astype(np.complex64), device=DEV))
        torch.cuda.synchronize()
        assert float(imgs[0].abs().max()) == 0.0
        ref = O.dft_ms2dirty(uvw, freq[:3], vis[:, :3], 64, 64, px, px, negate_v=True,
                             divide_by_n=False)
        assert O.rel_rms(imgs[1].cpu().numpy(), ref) < 1e-5
        assert plan.stats(0)["nvis"] == 0
        models = [torch.ones((128, 128), dtype=torch.float64, device=DEV),
                  torch.zeros((64, 64), dtype=torch.float64, device=DEV)]
        models[1][10, 20] = 1.0
        v = plan.dirty2ms(models).cpu().numpy()
        assert np.all(v[:, 3:] == 0)
        want = O.dft_dirty2ms(uvw, freq[:3], models[1].cpu().numpy(), px, px, negate_v=True,
                              divide_by_n=False)
        assert O.rel_rms(v[:, :3], want) < 1e-5


def test_context_outlives_its_plans():
    """The C ABI refuses to destroy a context that still has plans."""
    import ctypes
    from wsclean_b200 import gridder as G
    from wsclean_b200 import _lib as L
    rng, uvw, freq, vis, px = problem(8)
    ctx = G.Context(0)
    plan = G.Plan(uvw, freq, px, px, 1e-5, 64, 64, context=ctx, **KW)
    assert L.lib().wsg_ctx_destroy(ctx._h) == L.WSG_ERR_STATE
    plan.close()
    assert L.lib().wsg_ctx_destroy(ctx._h) == L.WSG_OK
    ctx._h = None
    # a gridder's context cannot be switched to pipelined mode
    g = G.WGriddingGridder(64, 64, 64, 64, px, px, 0.0, 0.0)
    view = L.lib().wsg_gridder_ctx(g._h)
    assert L.lib().wsg_ctx_set_async(ctypes.c_void_p(view), 1) == L.WSG_ERR_INVALID
    g.close()


@pytest.mark.parametrize("prec,tol", [("mixed", 1e-6), ("fp64", 1e-12)])
def test_plan_band_wider_than_the_pruned_transform(prec, tol):
    """A job whose u band is wider than the longest pruned column transform
    (the full-grid layout, u transform by the library FFT): plan calls equal
    the single calls."""
    from wsclean_b200 import gridder as G
    rng = np.random.default_rng(12)
    nrow, nx, ny = 4000, 6000, 32
    freq = np.array([1.40e8, 1.45e8])
    px = np.deg2rad(10 / 3600)
    umax = 0.45 / px * 299792458.0 / freq.max()
    uvw = rng.uniform(-1, 1, (nrow, 3)) * np.array([umax, umax, 0.2 * umax])
    vdt = np.complex64 if prec == "mixed" else np.complex128
    vis = (rng.normal(size=(nrow, 2)) + 1j * rng.normal(size=(nrow, 2))).astype(vdt)
    eps = 1e-5 if prec == "mixed" else 1e-12
    kw = dict(KW, sigma_min=1.5)
    with G.Plan(uvw, freq, px, px, eps, nx, ny, precision=prec, vis_dtype=vdt,
                dirty_dtype=np.float64, **kw) as plan:
        d = plan.ms2dirty(torch.as_tensor(vis, device=DEV))[0]
        model = torch.as_tensor(rng.normal(size=(nx, ny)), device=DEV)
        v = plan.dirty2ms(model)
        torch.cuda.synchronize()
        st = plan.stats(0)
        assert st["band_rows"] == st["nu"] > 8192
    raw = G.ms2dirty(uvw, freq, vis, nx, ny, px, px, eps, precision=prec,
                     dirty_dtype=np.float64, **kw)
    assert O.rel_rms(d.cpu().numpy(), raw) < tol
    rawv = G.dirty2ms(uvw, freq, model.cpu().numpy(), px, px, eps, precision=prec,
                      vis_dtype=vdt, **kw)
    assert O.rel_rms(v.cpu().numpy(), rawv) < tol
