"""Parity of the gather path (kr_bessel_sum + kr_traces) and of compute_seismogram.

Reference golden vectors: ``compute_gather`` (float64 CPU gather) on two small cases and
``compute_seismogram`` on the 6-layer model.  At the full gather size (8192 slownesses,
2047 frequencies, 100 offsets) each stage is checked against a float64 NumPy/SciPy
evaluation of that stage on the GPU's own inputs: sampled U(r, w) entries (full sum over
all 8192 slownesses with scipy's J0) and the trace FFT of the whole U.  Tolerance 1e-10.
"""

import numpy as np
import pytest
import torch

from conftest import rel_err
from oracle import kennett_oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-10


def _m(g, prefix=""):
    from seismicinversion_b200.layer_model import LayerModel

    return LayerModel(*[g[prefix + k] for k in ("alpha", "beta", "rho", "thickness", "Q_alpha", "Q_beta")])


def test_gather_small_golden(golden):
    from seismicinversion_b200 import compute_gather, compute_gather_gpu
    from seismicinversion_b200.earth_models import default_ocean_crust_model
    from seismicinversion_b200.source import ricker_10hz

    g = golden("gather_small.npz")
    t, offs, gm1 = compute_gather_gpu(_m(g, "m1_"), g["offsets"], T=64.0, nw=256, np_slow=128,
                                      p_max=1.2, source_func=ricker_10hz, free_surface=True)
    assert gm1.shape == (8, 512) and np.array_equal(t, g["time_m1"])
    assert rel_err(gm1, g["gather_m1"]) < TOL
    _, _, gd = compute_gather(default_ocean_crust_model(), g["offsets"], T=32.0, nw=128,
                              np_slow=96, p_max=1.0)
    assert rel_err(gd, g["gather_md"]) < TOL


def test_seismogram_c0(golden):
    from seismicinversion_b200 import compute_seismogram
    from seismicinversion_b200.source import ricker_10hz

    g = golden("c0_trace.npz")
    t, tr = compute_seismogram(_m(g), float(g["p"]), T=64.0, nw=2048, source_func=ricker_10hz,
                               free_surface=True)
    assert np.array_equal(t, g["time"])
    assert rel_err(tr, g["trace"]) < TOL


def test_seismogram_default_eps():
    from seismicinversion_b200 import compute_seismogram
    from seismicinversion_b200.earth_models import default_ocean_crust_model

    m = default_ocean_crust_model()
    t, tr = compute_seismogram(m, 0.3, T=32.0, nw=256, eps=0.05)
    _, tro, _ = O.seismogram(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta, 0.3,
                             T=32.0, nw=256, eps=0.05)
    assert rel_err(tr, tro) < TOL


def test_bessel_sum_random_and_ragged():
    from seismicinversion_b200 import device as D

    rng = np.random.default_rng(3)
    for n_p, n_w, n_r in [(300, 100, 7), (1, 1, 1), (65, 33, 9), (1000, 31, 3)]:
        R = rng.standard_normal((n_p, n_w)) + 1j * rng.standard_normal((n_p, n_w))
        p = np.sort(rng.uniform(0.001, 1.2, n_p))
        pw = rng.uniform(0, 1, n_p) * p
        om = np.sort(rng.uniform(0.05, 200.0, n_w))
        r = rng.uniform(0.0, 50.0, n_r)
        U = D.bessel_sum(torch.as_tensor(R, device="cuda"), p, pw, 1.3e-3, om, r).cpu().numpy()
        Uo = O.bessel_sum(R, p, om, r, 1.3e-3, taper=pw / p)
        assert rel_err(U, Uo) < TOL, (n_p, n_w, n_r)
    # no slownesses: U = 0
    U = D.bessel_sum(torch.zeros((0, 5), dtype=torch.complex128, device="cuda"), [], [], 0.1,
                     np.arange(1, 6.0), [1.0, 2.0])
    assert torch.count_nonzero(U) == 0


def test_bessel_sum_zeros_and_orderings():
    """Exact zeros (p = 0 in a uniform grid, omega = 0, offset 0: J0 = 1 and zero weights),
    a uniform grid reaching the fast Hankel path at large arguments, and the same slownesses in
    descending order (no rotation scheme: every term on the per-term path)."""
    from seismicinversion_b200 import device as D

    rng = np.random.default_rng(9)
    n_p, dp = 700, 1.2 / 700
    p = np.arange(n_p) * dp  # starts at 0
    pw = 0.5 * (1.0 + np.cos(np.pi * p / 1.2)) * p
    om = np.r_[0.0, np.linspace(0.01, 200.0, 45)]
    r = np.r_[0.0, 0.5, 7.0, 49.5]
    R = rng.standard_normal((n_p, len(om))) + 1j * rng.standard_normal((n_p, len(om)))
    taper = np.divide(pw, p, out=np.zeros_like(p), where=p > 0)
    Uo = O.bessel_sum(R, p, om, r, dp, taper=taper)
    U = D.bessel_sum(torch.as_tensor(R, device="cuda"), p, pw, dp, om, r).cpu().numpy()
    assert np.isfinite(U).all()
    assert rel_err(U, Uo) < TOL
    assert np.all(U[:, 0] == 0)  # omega = 0
    rev = slice(None, None, -1)
    Ur = D.bessel_sum(torch.as_tensor(R[rev].copy(), device="cuda"), p[rev].copy(),
                      pw[rev].copy(), dp, om, r).cpu().numpy()
    assert rel_err(Ur, Uo) < TOL


def test_traces_vs_numpy():
    from seismicinversion_b200 import device as D

    rng = np.random.default_rng(4)
    for n_r, nw in [(3, 8), (5, 256), (1, 2048)]:
        U = rng.standard_normal((n_r, nw - 1)) + 1j * rng.standard_normal((n_r, nw - 1))
        S = rng.standard_normal(nw - 1) + 1j * rng.standard_normal(nw - 1)
        decay = np.exp(-0.05 * np.arange(2 * nw))
        tr = D.traces(torch.as_tensor(U, device="cuda"), nw, S=S, decay=decay).cpu().numpy()
        assert rel_err(tr, O.hermitian_traces(U * S, nw, decay)) < 1e-13


def test_full_size_gather_stagewise():
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.kennett_gather_gpu import gather_device
    from seismicinversion_b200.source import ricker_10hz
    from scipy.special import j0

    m = random_layered_model(20, seed=1)
    offsets = np.arange(1, 101) * 0.5
    T, nw, npp, pmax = 64.0, 2048, 8192, 1.2
    time, R, U, g = gather_device(m, offsets, T, nw, npp, pmax, source_func=ricker_10hz,
                                  free_surface=True)
    assert g.shape == (100, 4096)
    Rh, Uh, gh = R.cpu().numpy(), U.cpu().numpy(), g.cpu().numpy()
    dw = 2 * np.pi / T
    om = np.arange(1, nw) * dw
    dp = pmax / npp
    p = np.arange(1, npp + 1) * dp
    taper = 0.5 * (1 + np.cos(np.pi * p / pmax))
    rng = np.random.default_rng(9)
    for _ in range(24):
        ir, iw = int(rng.integers(100)), int(rng.integers(nw - 1))
        ref = np.sum(j0((om[iw] * p) * offsets[ir]) * (Rh[:, iw] * (((taper * p) * om[iw]) * dp)))
        scale = np.max(np.abs(Uh[:, iw])) + 1e-300
        assert abs(Uh[ir, iw] - ref) / scale < TOL, (ir, iw)
    gamma = np.pi / T
    S = ricker_10hz(om, nw * dw)
    assert rel_err(gh, O.hermitian_traces(Uh * S, nw, np.exp(-gamma * time))) < 1e-12


def test_gather_returning_reflectivity_overlapped_copy():
    """The chunked, copy-overlapped path returns the same R grid as the batch call and the
    same traces as the plain call."""
    from seismicinversion_b200 import compute_gather_gpu, kennett_reflectivity_batch
    from seismicinversion_b200.earth_models import damped_gather_grid, random_layered_model

    m = random_layered_model(7, seed=12)
    offs = np.array([0.5, 3.0, 12.0, 30.0])
    t, _, g, R = compute_gather_gpu(m, offs, T=32.0, nw=512, np_slow=1031, p_max=1.1,
                                    free_surface=True, return_reflectivity=True, copy_chunks=5)
    t2, _, g2 = compute_gather_gpu(m, offs, T=32.0, nw=512, np_slow=1031, p_max=1.1,
                                   free_surface=True)
    _, omd, p, _, _, _ = damped_gather_grid(32.0, 512, 1031, 1.1)
    Rb = kennett_reflectivity_batch(m, p, omd, free_surface=True)
    assert np.array_equal(R, Rb)
    assert np.array_equal(g, g2) and np.array_equal(t, t2)


def test_cli_output_files(tmp_path, monkeypatch):
    """The command lines write the reference's file formats (.npz gather, two-column text)."""
    from seismicinversion_b200 import compute_gather_gpu, compute_seismogram
    from seismicinversion_b200.earth_models import default_ocean_crust_model
    from seismicinversion_b200.kennett_gather_gpu import main as gather_main
    from seismicinversion_b200.kennett_seismogram import main as seis_main

    monkeypatch.chdir(tmp_path)
    gather_main(["--r-min", "1", "--r-max", "3", "--dr", "1", "-n", "128", "--np", "64",
                 "-T", "32", "-o", "g.png", "--no-plot", "--free-surface"])
    z = np.load(tmp_path / "g.npz")
    t, offs, g = compute_gather_gpu(default_ocean_crust_model(), np.arange(1.0, 3.5, 1.0),
                                    T=32.0, nw=128, np_slow=64, free_surface=True)
    assert np.array_equal(z["gather"], g) and np.array_equal(z["offsets"], offs)
    seis_main(["-p", "0.25", "-n", "256", "--no-plot"])
    d = np.loadtxt(tmp_path / "seismogram_p0.2500.txt")
    t, s = compute_seismogram(default_ocean_crust_model(), 0.25, nw=256)
    assert d.shape == (512, 2) and np.allclose(d[:, 1], s, rtol=1e-7, atol=1e-7 * np.abs(s).max())


@pytest.mark.parametrize("return_reflectivity", [False, True])
def test_graph_replay_matches_eager(return_reflectivity):
    """Repeated gathers on one grid replay a captured CUDA graph: with the layer model
    changing between calls (a different layer table in the same staging slot) every result
    equals the eager path's bit for bit."""
    from seismicinversion_b200 import compute_gather_gpu
    from seismicinversion_b200 import kennett_gather_gpu as K
    from seismicinversion_b200.earth_models import random_layered_model

    models = [random_layered_model(9, seed=s) for s in (21, 22, 23)]
    offs = np.array([0.5, 2.0, 7.5, 19.0, 33.0])
    kw = dict(T=32.0, nw=512, np_slow=777, p_max=1.1, free_surface=True,
              return_reflectivity=return_reflectivity)
    eager = [[np.array(x) for x in compute_gather_gpu(m, offs, use_graph=False, **kw)]
             for m in models]
    n_graphs = len(K._GRAPHS)
    for rep in range(2):
        for m, ref in zip(models, eager):
            out = compute_gather_gpu(m, offs, **kw)
            assert len(out) == len(ref)
            for a, b in zip(out, ref):
                assert np.array_equal(a, b)
    assert len(K._GRAPHS) >= min(n_graphs + 1, K._GRAPH_MAX)


def test_consecutive_calls_return_independent_arrays():
    """Every array compute_gather_gpu returns belongs to the caller (the reference returns
    fresh arrays): a second call on the same grid, through the replayed graph, leaves the
    first call's R grid and gather untouched; copy_outputs=False returns the receive buffers
    themselves, which the next call overwrites."""
    from seismicinversion_b200 import compute_gather_gpu
    from seismicinversion_b200.earth_models import random_layered_model

    offs = np.array([1.0, 4.0, 9.0])
    kw = dict(T=32.0, nw=256, np_slow=300, p_max=1.0, free_surface=True,
              return_reflectivity=True)
    m1, m2 = random_layered_model(6, seed=31), random_layered_model(6, seed=32)
    for _ in range(3):  # eager, capture, replay
        _, _, g1, R1 = compute_gather_gpu(m1, offs, **kw)
        keep = (g1.copy(), R1.copy())
        _, _, g2, R2 = compute_gather_gpu(m2, offs, **kw)
        assert np.array_equal(g1, keep[0]) and np.array_equal(R1, keep[1])
        assert not np.array_equal(R1, R2) and not np.shares_memory(R1, R2)
    _, _, G1, V1 = compute_gather_gpu(m1, offs, copy_outputs=False, **kw)
    v1 = V1.copy()
    _, _, G2, V2 = compute_gather_gpu(m2, offs, copy_outputs=False, **kw)
    assert np.shares_memory(V1, V2) and np.array_equal(V2, R2) and not np.array_equal(V1, v1)
    assert np.shares_memory(G1, G2) and np.array_equal(G2, g2)
    # the reference's signature (gather only): a new page-locked block per call
    kw0 = {k: v for k, v in kw.items() if k != "return_reflectivity"}
    for _ in range(3):  # eager, capture, replay
        _, _, h1 = compute_gather_gpu(m1, offs, **kw0)
        k1 = h1.copy()
        _, _, h2 = compute_gather_gpu(m2, offs, **kw0)
        assert np.array_equal(h1, k1) and not np.shares_memory(h1, h2)
        assert np.array_equal(h1, g1) and np.array_equal(h2, g2)


def test_full_size_gather_end_to_end_vs_oracle():
    """The 21-layer gather workload at full size -- 8192 slownesses x 2047 damped frequencies
    x 100 offsets, free surface, Ricker 10 Hz -- through the public compute_gather_gpu call
    against the oracle's gather of the same inputs (reflectivity and float64 J0 slowness sum
    on every host core in a spawned process pool, tens of seconds): the R grid and the 100
    traces of 4096 samples to 1e-10 (and the displayed first 30 s)."""
    from oracle.cpu_baseline import GatherBaseline
    from seismicinversion_b200 import compute_gather_gpu
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.source import ricker_10hz

    m = random_layered_model(20, seed=1)
    offsets = np.arange(1, 101) * 0.5
    T, nw, npp, pmax = 64.0, 2048, 8192, 1.2
    base = GatherBaseline(m, offsets, T, nw, npp, pmax, True, n_sample=npp, chunk=16)
    try:
        _, Ro, Uo = base.step()
    finally:
        base.close()
    assert Ro.shape == (npp, nw - 1)
    dw = 2 * np.pi / T
    om = np.arange(1, nw) * dw
    time = np.arange(2 * nw) * (T / (2 * nw))
    go = O.hermitian_traces(Uo * ricker_10hz(om, nw * dw), nw, np.exp(-(np.pi / T) * time))
    t, offs, g, R = compute_gather_gpu(m, offsets, T=T, nw=nw, np_slow=npp, p_max=pmax,
                                       source_func=ricker_10hz, free_surface=True,
                                       return_reflectivity=True)
    assert np.array_equal(t, time) and g.shape == (100, 4096)
    assert rel_err(R, Ro) < 1e-10
    assert rel_err(g, go) < 1e-10
    shown = time < 30.0
    assert rel_err(g[:, shown], go[:, shown]) < 1e-10
