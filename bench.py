#!/usr/bin/env python
"""Benchmark of the Kennett reflectivity + discrete-wavenumber gather path on B200.

Workload (one "step"): the 21-layer gather model (water + 19 elastic layers + half-space,
seed 1), 2047 damped frequencies omega_k = k 2pi/64 + i pi/64 (T = 64 s, nw = 2048),
8192 slownesses p_j = j 1.2/8192, 100 offsets 0.5..50 km, Ricker 10 Hz, free surface:
(1) the full R(omega, p) grid, (2) the Bessel-weighted slowness sum U(r, omega),
(3) the 100 traces of 4096 samples.  Metric: (omega, p, interface) updates per second
(2047 x 8192 x 20 = 3.35e8 per step).

Device timing: CUDA events around each step on the launching stream, L2 flushed between
steps (256 MB write, outside the events), max over ranks.  ``e2e``: the same step through
the public ``compute_gather_gpu`` call with the reference's signature (host model and offsets
in, host traces out), wall clock; ``e2e_with_reflectivity``: the same call asked for the R
grid as well (``return_reflectivity=True``, the 268 MB grid copied back every step).

``--impl reference`` times the CPU oracle (NumPy/SciPy restatement of the reference,
organised like the reference's process-pool gather) on a bounded slowness sample with all
host cores; rank 0 only.
"""

from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = dict(workload="kennett_gather_21layer", layers=21, n_sub=20, seed=1, T=64.0,
                nw=2048, n_omega=2047, n_p=8192, p_max=1.2, n_offsets=100, dr=0.5,
                free_surface=True, source="ricker_10Hz", dtype="complex128")
FLOPS_PER_UPDATE = 340.0          # reference-literal count per (omega, p, interface) update
FLOPS_PER_PAIR_FS = 25.0          # free-surface epilogue per (omega, p)
FLOPS_PER_BESSEL_TERM = 6.0       # per (r, omega, p), J0 evaluation counted separately
# Adjoint (misfit gradient / vector-Jacobian product) update, literal count of the code with
# the same convention (cmul 6, cadd 2, reciprocal 6): forward step 340 + reverse of the step
# 920 (13 products of 2x2 complex matrices at 56, entry-wise phase / determinant terms) +
# phase-derivative terms 56 + residual 16 = 1332.  The contraction of the coefficient
# adjoints with their 10 x 6 parameter tangents happens once per (slowness, interface) after
# the frequency sum, not per update, and is not counted.
FLOPS_PER_ADJOINT_UPDATE = 1332.0
L2_FLUSH_BYTES = 256 << 20
NOMINAL_FP64_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=0, help="slownesses in the CPU sample")
    ap.add_argument("--profile", action="store_true",
                    help="device steps only (no e2e, CPU baseline or peak probe): for ncu")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the inversion / batching / serving measurements")
    ap.add_argument("--profile-kernel", choices=["inversion", "batch", "gmm", "gather512"],
                    default=None,
                    help="run only a small case of that workload (for ncu), no JSON line")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi sampler running during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().strip().splitlines() if r]
        os.unlink(self.f.name)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax.append(float(r[2]))
                for n, v in zip(names, r[5:9]):
                    if v.strip() == "Active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm)}


def _nvml_sample_loop(bus_id, conn, interval):
    """Child process: sample the SM clock and the clock event reasons until told to stop."""
    import time as _t

    import pynvml

    pynvml.nvmlInit()
    h = pynvml.nvmlDeviceGetHandleByPciBusId(bus_id)
    smax = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
    # the first queries of a process are slow (tens to hundreds of ms): make them before
    # the timed region starts
    pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
    pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
    samples = []
    conn.send("ready")
    t0 = _t.perf_counter()
    while not conn.poll(interval):
        try:
            samples.append((pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM),
                            pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)))
        except Exception:
            pass
    dt = _t.perf_counter() - t0
    conn.recv()
    conn.send((smax, samples, dt))


class NvmlClocks:
    """NVML sampler (every 5 ms, read-only queries) in a spawned child process, so that it
    keeps sampling while the timing thread holds the interpreter; the timed region of a step
    is tens of ms, too short for nvidia-smi's 200 ms interval."""

    NAMES = {"hw_slowdown": "nvmlClocksEventReasonHwSlowdown",
             "hw_thermal_slowdown": "nvmlClocksEventReasonHwThermalSlowdown",
             "sw_thermal_slowdown": "nvmlClocksEventReasonSwThermalSlowdown",
             "sw_power_cap": "nvmlClocksEventReasonSwPowerCap"}

    def __init__(self, bus_id):
        import multiprocessing as mp

        self.bus_id = bus_id
        self.ctx = mp.get_context("spawn")
        self.proc = self.conn = None

    @classmethod
    def open(cls, torch, dev):
        import pynvml

        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(dev)
        bus = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"
        pynvml.nvmlDeviceGetHandleByPciBusId(bus)  # fails here, not in the child
        return cls(bus)

    def start(self):
        self.conn, child = self.ctx.Pipe()
        self.proc = self.ctx.Process(target=_nvml_sample_loop, args=(self.bus_id, child, 0.005),
                                     daemon=True)
        self.proc.start()
        if not self.conn.poll(60) or self.conn.recv() != "ready":
            raise RuntimeError("clock sampler did not start")

    def stop(self):
        import pynvml

        self.conn.send("stop")
        smax, samples, dt = self.conn.recv() if self.conn.poll(30) else (None, [], 0.0)
        self.proc.join(10)
        sm = [x[0] for x in samples]
        reasons = sorted(k for k, attr in self.NAMES.items()
                         if any(x[1] & getattr(pynvml, attr) for x in samples))
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": reasons, "samples": len(sm),
                "sampler": f"nvml in a child process, {1e3 * dt / max(len(sm), 1):.1f} ms per "
                           f"sample over {1e3 * dt:.0f} ms"}


def clock_sampler(torch, dev, index):
    """NVML sampler when pynvml can open the device, else nvidia-smi."""
    try:
        return NvmlClocks.open(torch, dev)
    except Exception:
        return Clocks(index)


def host_info(threads: int) -> dict:
    """CPU model and thread settings of a CPU leg (the worker count it used; the oracle's
    workers pin OpenMP / BLAS to one thread each)."""
    model = None
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"cpu_model": model, "threads_used": int(threads),
            "host_cores_available": len(os.sched_getaffinity(0)),
            "worker_env": {"OMP_NUM_THREADS": "1", "OPENBLAS_NUM_THREADS": "1",
                           "MKL_NUM_THREADS": "1"}}


def fp64_peak(torch, dev):
    """Measured FP64 CUDA-core peak (DFMA probe, best of 5) in TFLOP/s."""
    from seismicinversion_b200 import _lib

    h = _lib.lib()
    blocks, iters = 148 * 8, 20000
    out = torch.empty(blocks * 256, dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream(dev)
    best = 0.0
    for _ in range(6):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        _lib.check(h.kr_bench_fp64_fma(blocks, iters, out.data_ptr(), st.cuda_stream), "probe")
        b.record(st)
        b.synchronize()
        best = max(best, h.kr_bench_fp64_fma_flops(blocks, iters) / (a.elapsed_time(b) * 1e-3))
    return best / 1e12


def _events(torch, st, fn, reps):
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fn()
    a.record(st)
    for _ in range(reps):
        fn()
    b.record(st)
    b.synchronize()
    return a.elapsed_time(b) / reps


def bench_gmm(torch, D, tab, p_t, w_t, R_kennett, reps):
    """Global Matrix Method forward (kr_gmm_reflectivity) on the gather's R grid: time per
    launch and agreement with the Kennett grid of the timed step (slownesses <= 1.0 s/km)."""
    n_p, n_w = R_kennett.shape
    Rg = torch.empty_like(R_kennett)
    D.gmm_reflectivity(tab, p_t, w_t, True, out=Rg)
    torch.cuda.synchronize()
    evs = []
    for _ in range(reps):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        e[0].record()
        D.gmm_reflectivity(tab, p_t, w_t, True, out=Rg)
        e[1].record()
        evs.append(e)
    torch.cuda.synchronize()
    ms = float(np.mean([a.elapsed_time(b) for a, b in evs]))
    sel = p_t <= 1.0
    diff = float(((Rg[sel] - R_kennett[sel]).abs().amax(1) / R_kennett[sel].abs().amax(1)).max())
    L = tab.shape[1]
    upd = n_p * n_w * (L - 2)
    return {"workload": "21-layer gather grid, 8192 p x 2047 damped omega, free surface",
            "ms": ms, "interface_updates_per_s": upd / (ms * 1e-3),
            "max_rel_diff_vs_kennett_p_le_1": diff}


def _rel(x, ref) -> float:
    """max|x - ref| / max|ref| (the reference's error metric)."""
    x, ref = np.asarray(x), np.asarray(ref)
    return float(np.max(np.abs(x - ref)) / (np.max(np.abs(ref)) + 1e-300))


def accuracy_c0():
    """The single-trace configuration (6 layers, p = 0.2, 2047 frequencies, free surface,
    Ricker 10 Hz) through the public drop-ins against the oracle: R and the 4096-sample trace."""
    from oracle import kennett_oracle as O
    from seismicinversion_b200 import compute_seismogram, kennett_reflectivity
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.source import ricker_10hz

    m = random_layered_model(5, seed=0)
    arrs = [m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta]
    _, tr = compute_seismogram(m, 0.2, T=64.0, nw=2048, source_func=ricker_10hz,
                               free_surface=True)
    om = np.arange(1, 2048) * (2 * np.pi / 64.0)
    R = kennett_reflectivity(m, 0.2, om, free_surface=True)
    _, tro, Ro = O.seismogram(*arrs, 0.2, T=64.0, nw=2048, free_surface=True,
                              source=lambda w, wm: O.ricker_spectrum(w, 100 * np.pi))
    return {"c0_R": _rel(R, Ro), "c0_trace": _rel(tr, tro)}


def taup_cpu_baseline(torch, true, start, p, w, n_grad=8):
    """CPU baseline of the tau-p derivative workload, as the reference computes it: per
    slowness, the differentiable forward on the CPU and torch.autograd.grad of the misfit
    (taup_inversion.py:153-172), torch.func.hessian of it (:177) and jacrev
    (kennett_torch.py:611-641), through the differentiable oracle with torch threads = host
    cores.  Gradients timed on n_grad of the slownesses, the Hessian and jacrev on one,
    extrapolated to all of them."""
    from oracle import torch_oracle as T
    from seismicinversion_b200.kennett_torch import _pack_params, _unpack_params

    cores = len(os.sched_getaffinity(0))
    threads = torch.get_num_threads()
    torch.set_num_threads(cores)
    n_hw = 64  # frequencies of the timed Hessian (its cost is linear in them)
    try:
        tt = {k: torch.as_tensor(getattr(true, k)) for k in
              ("alpha", "beta", "rho", "thickness", "Q_alpha", "Q_beta")}
        ts = {k: torch.as_tensor(getattr(start, k)) for k in tt}
        om = torch.as_tensor(w)
        m0 = _pack_params(ts["alpha"], ts["beta"], ts["rho"], ts["thickness"])
        sel = np.linspace(0, len(p) - 1, n_grad).round().astype(int)

        def chi_p(m, pj):
            a, b, r, h = _unpack_params(m, ts["alpha"], ts["beta"], ts["rho"], ts["thickness"])
            R = T.reflectivity(a, b, r, h, ts["Q_alpha"], ts["Q_beta"], [pj], om)
            Ro = T.reflectivity(*tt.values(), [pj], om).detach()
            return T.misfit(R, Ro)

        chi_p(m0.clone().requires_grad_(True), float(p[0]))  # warm (allocator, threads)
        t0 = time.perf_counter()
        for j in sel:
            m = m0.clone().requires_grad_(True)
            torch.autograd.grad(chi_p(m, float(p[j])), m)
        grad_s = (time.perf_counter() - t0) / len(sel) * len(p)
        j = int(sel[len(sel) // 2])
        om_full = om
        om = om_full[:n_hw]
        t0 = time.perf_counter()
        torch.func.hessian(lambda m: chi_p(m, float(p[j])))(m0)
        hess_s = (time.perf_counter() - t0) * len(p) * len(om_full) / n_hw
        om = om_full

        def f(m):
            a, b, r, h = _unpack_params(m, ts["alpha"], ts["beta"], ts["rho"], ts["thickness"])
            return T.reflectivity(a, b, r, h, ts["Q_alpha"], ts["Q_beta"], [float(p[j])], om)[0]

        t0 = time.perf_counter()
        torch.func.jacrev(lambda m: f(m).real)(m0)
        torch.func.jacrev(lambda m: f(m).imag)(m0)
        jac_s = time.perf_counter() - t0
    finally:
        torch.set_num_threads(threads)
    return {"grad_evals_per_s": 1.0 / grad_s, "seconds_per_grad_eval": grad_s,
            "seconds_per_exact_hessian": hess_s, "seconds_per_jacobian_one_slowness": jac_s,
            "seconds_per_exact_lm_iteration_est": grad_s + hess_s, "unit": "grad evals/s",
            "cores": cores, "kind": "port",
            "sample": f"autograd gradient on {len(sel)} of {len(p)} slownesses and jacrev "
                      f"(Re, Im) on 1, per slowness as the reference loops them, extrapolated "
                      f"to {len(p)}; torch.func.hessian on 1 slowness x {n_hw} of the "
                      f"{len(w)} frequencies, extrapolated linearly; differentiable torch "
                      f"restatement of the oracle, torch threads = {cores}",
            "host": host_info(cores)}


def bench_inversion(torch, dev, reps, cpu=True):
    """tau-p inversion workload: 21-layer model (79 packed parameters), 64 slownesses on
    [0.05, 0.6], omega_k = k 2pi/64 (k = 1..1024), start = true * exp(0.1 N(0,1)) (seed 2)."""
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.kennett_torch import model_to_tensors, packed_index
    from seismicinversion_b200.taup_inversion import invert_taup

    true = random_layered_model(20, seed=2)
    rng = np.random.default_rng(2)
    start = random_layered_model(20, seed=2)
    for name in ("alpha", "beta", "rho"):
        getattr(start, name)[1:] *= np.exp(0.1 * rng.standard_normal(20))
    start.thickness[1:-1] *= np.exp(0.1 * rng.standard_normal(19))
    p = np.linspace(0.05, 0.6, 64)
    w = np.arange(1, 1025) * (2 * np.pi / 64)
    st = torch.cuda.current_stream(dev)
    tab_true, tab = D.layer_table(true, dev), D.layer_table(start, dev)
    p_t, w_t = torch.as_tensor(p, device=dev), torch.as_tensor(w, device=dev).to(torch.complex128)
    R_obs = D.reflectivity(tab_true, p_t, w_t)
    # sub-millisecond calls: enough back-to-back calls that the first one's host-side issue
    # (~30 us while the device idles) does not weigh on the steady-state rate
    short = max(reps, 20)
    ms_grad = _events(torch, st, lambda: D.misfit_gradient(tab, p_t, w_t, R_obs), short)
    ms_jac = _events(torch, st, lambda: D.jacobian(tab, p_t, w_t, want_R=False), short)
    ms_fwd = _events(torch, st, lambda: D.reflectivity(tab, p_t, w_t), short)
    upd = 64 * 1024 * 20
    t = model_to_tensors(true)
    init = np.concatenate([start.alpha[1:], start.beta[1:], start.rho[1:], start.thickness[1:-1]])
    peak = fp64_peak(torch, dev)
    alg = FLOPS_PER_ADJOINT_UPDATE * upd / (ms_grad * 1e-3) / 1e12
    out = {"workload": "tau-p LM, 21 layers / 79 params, 64 p x 1024 omega",
           "grad_units": "gradient evaluations over all 64 slownesses per second",
           "grad_evals_per_s": 1e3 / ms_grad, "ms_per_grad_eval": ms_grad,
           "adjoint_updates_per_s": upd / (ms_grad * 1e-3),
           "adjoint_alg_tflops": alg, "adjoint_frac_of_fp64_peak": alg / peak,
           "ms_per_jacobian": ms_jac, "ms_per_forward": ms_fwd}
    basis = torch.eye(4 * 21, dtype=torch.float64, device=dev)[torch.as_tensor(packed_index(21))]
    ms_hvp = _events(torch, st, lambda: D.misfit_hvp(tab, p_t, w_t, R_obs, basis), reps)
    out["ms_per_exact_hessian"] = ms_hvp
    out["exact_hessian_method"] = ("79 Hessian-vector products (tangent of the adjoint, "
                                   "kr_misfit_hvp) in one launch")
    # accuracy against the reference's own jacrev / autograd at 1024 frequencies (the start
    # model above at 4 of the 64 slownesses: tests/golden/derivs_c2_1024.npz)
    from seismicinversion_b200.kennett_torch import _pack_params, jacobian, misfit_gradient_packed

    gold = ROOT / "tests" / "golden" / "derivs_c2_1024.npz"
    if gold.exists():
        with np.load(gold) as g:
            ts = model_to_tensors(start)
            om = torch.as_tensor(g["omega"])
            errs = [_rel(jacobian(ts["alpha"], ts["beta"], ts["rho"], ts["thickness"],
                                  ts["Q_alpha"], ts["Q_beta"], float(pk), om).numpy(),
                         g[f"J_{k}"]) for k, pk in enumerate(g["p"])]
            m0 = _pack_params(ts["alpha"], ts["beta"], ts["rho"], ts["thickness"]).numpy()
            _, gr = misfit_gradient_packed(m0, ts["alpha"], ts["beta"], ts["rho"],
                                           ts["thickness"], ts["Q_alpha"], ts["Q_beta"], g["p"],
                                           om, np.stack([g[f"R_obs_{k}"] for k in range(4)]))
            out["max_rel_err_vs_reference"] = {
                "jacobian_4p_1024w": max(errs), "gradient_4p_1024w": _rel(gr.cpu().numpy(),
                                                                          g["grad"]),
                "reference": "jacrev and autograd.grad of the reference's torch forward"}
    for hess in ("gauss-newton", "exact"):
        its = 10
        # one untimed iteration first: library handles, allocator pools and plans are made
        # on first use, and a cold first call would count them
        invert_taup(true, list(p), nfreq=1024, max_iter=1, hessian=hess, initial_params=init,
                    tol=0.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = invert_taup(true, list(p), nfreq=1024, max_iter=its, hessian=hess,
                          initial_params=init, tol=0.0)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        out[f"lm_{hess}"] = {"iterations": res.n_iterations, "seconds": dt,
                             "s_per_iteration": dt / max(res.n_iterations, 1),
                             "param_err_history": list(map(float, res.param_error_history)),
                             "misfit_history": list(map(float, res.misfit_history))}
    # the reference's own start (uniform +-10 %, seed 42) and its invert_taup trajectory on this
    # model at 16 slownesses x 64 frequencies (tests/golden/invert_c2.npz, the reference run on
    # the CPU; at 64 x 1024 the reference needs about a day)
    gold = ROOT / "tests" / "golden" / "invert_c2.npz"
    t0 = time.perf_counter()
    res = invert_taup(true, list(np.linspace(0.05, 0.6, 16)), nfreq=64, perturbation=0.1,
                      max_iter=10, seed=42, hessian="exact", tol=0.0)
    traj = {"workload": "21 layers, 16 p on [0.05, 0.6] x 64 omega, uniform +-10 % start "
                        "(seed 42), exact Hessian, 10 iterations",
            "seconds": time.perf_counter() - t0,
            "param_err_history": list(map(float, res.param_error_history)),
            "misfit_history": list(map(float, res.misfit_history))}
    if gold.exists():
        with np.load(gold) as g:
            n = min(len(g["param_err"]), res.n_iterations)
            traj["reference_param_err_history"] = list(map(float, g["param_err"]))
            traj["reference_misfit_history"] = list(map(float, g["misfit"]))
            traj["max_abs_diff_param_err"] = float(np.max(np.abs(
                np.array(res.param_error_history[:n]) - g["param_err"][:n])))
            traj["max_rel_diff_misfit"] = float(np.max(np.abs(
                np.array(res.misfit_history[:n]) - g["misfit"][:n]) / g["misfit"][:n]))
    out["lm_exact_reference_start"] = traj
    # K concurrent inversions (true models seeds 2..2+K-1, lognormal starts), LM state on
    # the device: one batched gradient (+ exact-Hessian) launch and one batched trial launch
    # per round for all K
    from seismicinversion_b200.taup_batch import invert_taup_batch

    K = 16
    trues, inits = [], []
    for k in range(K):
        tm = random_layered_model(20, seed=2 + k)
        r = np.random.default_rng(2 + k)
        x0 = np.concatenate([tm.alpha[1:], tm.beta[1:], tm.rho[1:], tm.thickness[1:-1]])
        x0 = x0 * np.exp(0.1 * r.standard_normal(len(x0)))
        trues.append(tm)
        inits.append(x0)
    for hess in ("gauss-newton", "exact"):
        its = 5
        invert_taup_batch(trues, list(p), nfreq=1024, max_iter=1, hessian=hess,
                          initial_params=inits, tol=0.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        res = invert_taup_batch(trues, list(p), nfreq=1024, max_iter=its, hessian=hess,
                                initial_params=inits, tol=0.0)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        n_it = sum(x.n_iterations for x in res)
        seq = out[f"lm_{hess}"]["s_per_iteration"]
        out[f"lm_batch16_{hess}"] = {
            "inversions": K, "iterations_each": its, "seconds": dt,
            "s_per_round_all_inversions": dt / its,
            "inversion_iterations_per_s": n_it / dt,
            "speedup_vs_sequential_invert_taup": (n_it * seq) / dt}
    if cpu:
        cb = taup_cpu_baseline(torch, true, start, p, np.arange(1, 1025) * (2 * np.pi / 64))
        cb["value"] = cb["grad_evals_per_s"]
        out["cpu_baseline"] = cb
        out["grad_evals_speedup_vs_cpu"] = out["grad_evals_per_s"] / cb["grad_evals_per_s"]
        out["exact_lm_iteration_speedup_vs_cpu"] = (
            cb["seconds_per_exact_lm_iteration_est"] / out["lm_exact"]["s_per_iteration"])
    return out


def uneven_cpu_baseline(specs, pool, n_models=256, max_p=8):
    """CPU rates of the uneven-batching workload on a stratified sample: every
    (4096 / n_models)-th model in order of work (smallest to largest), each on up to ``max_p``
    of its slownesses (evenly spaced) with all its frequencies and layers; even models forward
    (the NumPy oracle, as the reference's kennett_reflectivity), odd models forward + misfit
    gradient (torch autograd through the differentiable oracle, as kennett_reflectivity_torch
    and taup_misfit_grad_hessian); one model per task on a spawned pool of every host core.
    Returns (forward updates/s, gradient updates/s, description)."""
    from oracle.cpu_baseline import _grad_chunk, _layers, _refl_chunk

    order = sorted(range(len(specs)), key=lambda b: specs[b][0].n_layers * len(specs[b][1])
                   * len(specs[b][2]))
    pick = [order[int(k)] for k in np.linspace(0, len(order) - 1, n_models).round()]
    fwd, grad = [], []
    fu = gu = 0
    for b in pick:
        m, p, w = specs[b]
        ps = p[np.unique(np.linspace(0, len(p) - 1, min(max_p, len(p))).round().astype(int))]
        u = len(ps) * len(w) * (m.n_layers - 1)
        if b % 2:
            grad.append((_layers(m), ps, w, np.zeros((len(ps), len(w)), complex), False))
            gu += u
        else:
            fwd.append((_layers(m), ps, w, False))
            fu += u
    pool.warm()
    tf = pool.timed_jobs(_refl_chunk, fwd)
    tg = pool.timed_jobs(_grad_chunk, grad)
    desc = (f"{len(pick)} models stratified by work ({len(fwd)} forward, {len(grad)} forward + "
            f"gradient), <= {max_p} slownesses each with all frequencies and layers, spawned "
            f"pool of {pool.workers} processes; full-workload time extrapolated per update")
    return fu / tf, gu / tg, desc


def bench_batched(torch, dev, reps, n_models=4096, pool=None):
    """Uneven batching workload: 4096 models, total layers U{3..64}, n_omega in
    {256, 512, 1024, 2048}, n_p U{16..256} on (0, 0.8] (seed 3); odd models ask for forward +
    gradient against the R of an independently perturbed model (seed 4)."""
    from seismicinversion_b200 import device as D
    from seismicinversion_b200.batch import BatchItem, ModelBatch, autotune
    from seismicinversion_b200.earth_models import uneven_batch_specs
    from seismicinversion_b200.layer_model import LayerModel

    specs = uneven_batch_specs(n_models, seed=3)
    rng = np.random.default_rng(4)
    perturbed = []
    for m, p, w in specs:
        f = np.exp(0.03 * rng.standard_normal(m.n_layers))
        perturbed.append(LayerModel(m.alpha * f, m.beta * f, m.rho, m.thickness, m.Q_alpha, m.Q_beta))
    obs_batch = ModelBatch([BatchItem(perturbed[b], specs[b][1], specs[b][2])
                            for b in range(1, n_models, 2)], device=dev)
    obs_batch.launch()
    items = []
    for b, (m, p, w) in enumerate(specs):
        if b % 2:
            items.append(BatchItem(m, p, w, gradient=True, R_obs=obs_batch.reflectivity(b // 2)))
        else:
            items.append(BatchItem(m, p, w))
    batch = ModelBatch(items, device=dev)
    best, times = autotune(batch, candidates=[(32, 128), (64, 128), (128, 256), (128, 512),
                                              (128, 1024), (128, 2048)],
                           reps=1)
    batch.capture()
    st = torch.cuda.current_stream(dev)
    ms = _events(torch, st, batch.run, reps)
    work = batch.work()
    # plain per-call paths on samples: one call per model (all slownesses), and one call per
    # (model, slowness) as the reference's API issues them; synchronised after each call
    # odd stride: the sample alternates forward and forward+gradient models like the batch
    sample = list(range(0, n_models, 31))[:128]

    def per_model_pass():
        for b in sample:
            it = items[b]
            tab = D.layer_table(it.model, dev)
            if it.gradient:
                D.misfit_gradient(tab, it.p, it.omega, it.R_obs.reshape(len(it.p), -1))
            else:
                D.reflectivity(tab, it.p, it.omega)
            torch.cuda.synchronize()

    per_model_pass()  # untimed: first-use costs (allocator blocks of these sizes, modules)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    per_model_pass()
    per_model = (time.perf_counter() - t0) / len(sample)
    sample_p = sample[:16]  # 8 forward + 8 gradient models
    for b in sample_p[:4]:  # untimed warm calls of both kinds at this granularity
        it = items[b]
        tab = D.layer_table(it.model, dev)
        if it.gradient:
            D.misfit_gradient(tab, it.p[:1], it.omega, it.R_obs.reshape(len(it.p), -1)[:1])
        else:
            D.reflectivity(tab, it.p[:1], it.omega)
    calls = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for b in sample_p:
        it = items[b]
        tab = D.layer_table(it.model, dev)
        Ro = it.R_obs.reshape(len(it.p), -1) if it.gradient else None
        for j in range(len(it.p)):
            if it.gradient:
                D.misfit_gradient(tab, it.p[j:j + 1], it.omega, Ro[j:j + 1])
            else:
                D.reflectivity(tab, it.p[j:j + 1], it.omega)
            torch.cuda.synchronize()
            calls += 1
    per_pair_call = (time.perf_counter() - t0) / calls
    n_pairs = sum(len(it.p) for it in items)
    batched_models_per_s = n_models / (ms * 1e-3)
    alg = (FLOPS_PER_UPDATE * work["forward_updates"]
           + FLOPS_PER_ADJOINT_UPDATE * work["gradient_updates"]) / (ms * 1e-3) / 1e12
    peak = fp64_peak(torch, dev)
    extra = {}
    if pool is not None:
        # accuracy: the largest forward model and the largest gradient model of the batch at
        # full size against the oracle (reflectivity; chi and gradient by autograd)
        order = sorted(range(n_models), key=lambda b: -(specs[b][0].n_layers * len(specs[b][1])
                                                        * len(specs[b][2])))
        bf = next(b for b in order if b % 2 == 0)
        bg = next(b for b in order if b % 2 == 1)
        mf, pf, wf = specs[bf]
        Rf = pool.reflectivity(mf, pf, wf)
        mg, pg, wg = specs[bg]
        obs = items[bg].R_obs.cpu().numpy().reshape(len(pg), len(wg))
        chi_o, g_o = pool.misfit_gradient(mg, pg, wg, obs)
        chi, g = batch.misfit_gradient(bg)
        extra["max_rel_err_vs_oracle"] = {
            "forward_largest_model": _rel(batch.reflectivity(bf).cpu().numpy(), Rf),
            "gradient_largest_model": _rel(g.cpu().numpy(), g_o),
            "chi_largest_model": abs(float(chi) - chi_o) / chi_o,
            "models": f"forward: {mf.n_layers} layers x {len(pf)} p x {len(wf)} w; gradient: "
                      f"{mg.n_layers} layers x {len(pg)} p x {len(wg)} w"}
        fr, gr, desc = uneven_cpu_baseline(specs, pool)
        cpu_s = work["forward_updates"] / fr + work["gradient_updates"] / gr
        extra["cpu_baseline"] = {
            "value": n_models / cpu_s, "unit": "models/s", "cores": pool.workers, "kind": "port",
            "forward_updates_per_s": fr, "gradient_updates_per_s": gr,
            "seconds_full_batch_extrapolated": cpu_s, "sample": desc,
            "host": host_info(pool.workers)}
        extra["speedup_vs_cpu"] = (n_models / (ms * 1e-3)) / (n_models / cpu_s)
    return {"workload": "4096 uneven models, half forward+gradient", "schedule": list(best),
            "autotune_ms": {str(k): v for k, v in times.items()}, "ms_per_batch": ms,
            "models_per_s": batched_models_per_s, **work,
            "updates_per_s": (work["forward_updates"] + work["gradient_updates"]) / (ms * 1e-3),
            "alg_tflops": alg, "frac_of_fp64_peak": alg / peak,
            "plain_per_model_call_models_per_s": 1.0 / per_model,
            "plain_per_slowness_call_models_per_s": n_models / (per_pair_call * n_pairs),
            "speedup_vs_per_model_calls": batched_models_per_s * per_model,
            "speedup_vs_per_slowness_calls": batched_models_per_s * per_pair_call * n_pairs / n_models,
            "graph_captured": True, **extra}


def bench_training_data(torch, dev, n=50_000):
    """Amortized-inference training data as the reference's ``generate_training_data``: n prior
    samples of the default 6-layer model, 12 slownesses x 64 frequencies, written in the
    reference's .pt layout; wall time of the whole call (sampling, batched forward launches,
    float32 conversion, host copy, file write), after one small untimed call."""
    from seismicinversion_b200.training_data import DataGenConfig, generate_training_data

    with tempfile.TemporaryDirectory() as d:
        generate_training_data(d, DataGenConfig(n_train=2000, n_val=0, n_test=0), device=dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        generate_training_data(d, DataGenConfig(n_train=n, n_val=0, n_test=0), device=dev)
        dt = time.perf_counter() - t0
    return {"workload": f"{n} samples, default 6-layer model prior, 12 p x 64 omega, .pt output",
            "samples": n, "seconds": dt, "samples_per_s": n / dt,
            "reference_published_seconds_50k": 4747.0,
            "note": "the reference's figure (NeuralInversion/README.md, hardware not stated) "
                    "uses its global-matrix forward; this one the Kennett kernels"}


def bench_published_configs(torch, dev, reps=5):
    """The configurations the reference publishes timings for (Apple Silicon, its README
    files), run through this library's public drop-ins with host inputs and outputs; the
    reference's figures beside each (best of ``reps`` wall times after one untimed call)."""
    from seismicinversion_b200.earth_models import default_ocean_crust_model
    from seismicinversion_b200.kennett_gather_gpu import compute_gather_gpu
    from seismicinversion_b200.kennett_torch import hessian, jacobian, model_to_tensors

    m = default_ocean_crust_model()
    offs = np.arange(0.5, 50.0 + 0.25, 0.5)
    t = model_to_tensors(m)
    args = (t["alpha"], t["beta"], t["rho"], t["thickness"], t["Q_alpha"], t["Q_beta"], 0.2)

    def best(fn):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        return min(ts) * 1e3

    out = {}
    for n_p, pub in ((2048, 30.0), (4096, 60.0)):
        ms = best(lambda: compute_gather_gpu(m, offs, T=64.0, nw=2048, np_slow=n_p))
        out[f"gather_np{n_p}"] = {"ms": ms, "reference_published_s": pub,
                                  "reference_setup": "compute_gather, 10-core M-series CPU"}
    w127 = torch.as_tensor(np.arange(1, 128) * (2 * np.pi / 64))
    ms = best(lambda: jacobian(*args, w127))
    out["jacobian_5layer_nfreq127"] = {"ms": ms, "reference_published_ms": 89.0,
                                       "reference_setup": "torch.func.jacrev, Apple Silicon"}
    w31 = torch.as_tensor(np.arange(1, 32) * (2 * np.pi / 64))
    ms = best(lambda: hessian(*args, w31))
    out["hessian_5layer_nfreq31"] = {"ms": ms, "reference_published_ms": 70.0,
                                     "reference_setup": "torch.func.hessian, Apple Silicon"}
    return out


def _plain_per_request(torch, D, dev, pool, arrivals):
    """The plain per-request path at the given arrival times: one fused-kernel call and a
    device synchronisation per request, in arrival order (FIFO, one host thread)."""
    lat = []
    for k, t_arr in enumerate(arrivals):
        while time.perf_counter() < t_arr:
            pass
        m, p_t, w_t, g, obs = pool[k % len(pool)]
        tab = D.layer_table(m, dev)
        if g:
            D.misfit_gradient(tab, p_t, w_t, obs)
        else:
            D.reflectivity(tab, p_t, w_t)
        torch.cuda.synchronize()
        lat.append(time.perf_counter() - t_arr)
    lat = np.array(lat)
    span = arrivals[-1] + lat[-1] - arrivals[0]
    return {"completed": len(lat), "throughput_rps": len(lat) / span,
            "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3)}


def bench_serving(torch, dev, rates=(100, 300, 1000, 3000, 10000, 20000), duration=1.0,
                  max_requests=3000, pool=None, cpu_rates=None):
    """Serving workload: Poisson arrivals (seed 7) of requests drawn as in the batching
    workload (50/50 forward / forward+gradient), device-resident inputs, 120 GB budget; the
    client consumes results in arrival order and releases them.  At every rate the same
    arrival sequence also runs through the plain per-request path (launch + synchronise per
    request, FIFO)."""
    import gc

    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import uneven_batch_specs
    from seismicinversion_b200.serve import KennettServer

    specs = uneven_batch_specs(256, seed=5)
    poolreq = []
    for b, (m, p, w) in enumerate(specs):
        p_t = torch.as_tensor(p, device=dev)
        w_t = torch.as_tensor(w, device=dev).to(torch.complex128)
        obs = None
        if b % 2:
            obs = D.reflectivity(D.layer_table(m, dev), p_t, w_t) * 1.01
        poolreq.append((m, p_t, w_t, b % 2 == 1, obs))
    torch.cuda.synchronize()
    rng = np.random.default_rng(7)
    rng_w = np.random.default_rng(8)
    out = {"workload": "Poisson stream, uneven models as the batching workload, 50/50 fwd/grad"}
    # the application's choice: long-lived objects (models, pools, inputs) go to the permanent
    # generation so that periodic collections stay short while requests stream through
    gc.collect()
    gc.freeze()
    # one executor (streams, allocation-stream pool, pinned blocks) serves the warm-up and
    # every rate, as in a long-running server
    from seismicinversion_b200.serve import GpuBatchExecutor

    ex = GpuBatchExecutor(device=dev, n_streams=3)
    ex.prewarm(4 << 30)
    # warm-up (untimed): kernel modules, streams, allocator blocks of the batch size classes,
    # pinned staging buffers: the whole pool at once, every request alone (groups of one run
    # the single-model kernels on the execution streams), then a short stream at a high rate
    with KennettServer(executor=ex, hbm_budget_bytes=120 * 10**9, max_batch_requests=64,
                       max_inflight=2) as srv:
        warm = [srv.submit(m, p_t, w_t, gradient=g, R_obs=obs) for m, p_t, w_t, g, obs in poolreq]
        for r in warm:
            r.wait(120)
            r.release()
        for m, p_t, w_t, g, obs in poolreq:
            r = srv.submit(m, p_t, w_t, gradient=g, R_obs=obs)
            r.wait(120)
            r.release()
        warm = []
        t_next = time.perf_counter()
        for k in range(1500):
            t_next += rng_w.exponential(1.0 / 5000)
            dt = t_next - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            m, p_t, w_t, g, obs = poolreq[k % len(poolreq)]
            warm.append(srv.submit(m, p_t, w_t, gradient=g, R_obs=obs))
        for r in warm:
            r.wait(120)
            r.release()
        del warm
    _plain_per_request(torch, D, dev, poolreq, [time.perf_counter()] * 64)  # untimed warm-up
    torch.cuda.synchronize()

    for lam in rates:
        n = int(min(max_requests, lam * duration))
        gaps = rng.exponential(1.0 / lam, n)
        # the previous run's requests are garbage with reference cycles: collect them now
        # rather than in a collection that lands inside this run
        gc.collect()
        with KennettServer(executor=ex, hbm_budget_bytes=120 * 10**9, max_batch_requests=64,
                           max_inflight=2) as srv:
            t_start = time.perf_counter()
            t_next = t_start
            reqs = []
            consumed = 0  # the client consumes results in arrival order, releasing them
            for k in range(n):
                t_next += gaps[k]
                dt = t_next - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)  # releases the GIL to the scheduler thread
                m, p_t, w_t, g, obs = poolreq[k % len(poolreq)]
                reqs.append(srv.submit(m, p_t, w_t, gradient=g, R_obs=obs))
                while consumed < len(reqs) and reqs[consumed].done.is_set():
                    reqs[consumed].release()
                    consumed += 1
            for r in reqs:
                r.wait(120)
                r.release()
            stats = srv.stats(since=t_start)
        row = {k: stats[k] for k in ("completed", "throughput_rps", "p50_ms", "p99_ms",
                                     "batches", "mean_queue_ms", "mean_build_launch_ms",
                                     "mean_device_ms")}
        gc.collect()
        t0 = time.perf_counter() + 1e-3
        plain = _plain_per_request(torch, D, dev, poolreq, list(t0 + np.cumsum(gaps)))
        row["plain_per_request"] = plain
        row["throughput_vs_plain"] = row["throughput_rps"] / plain["throughput_rps"]
        out[f"rate_{lam}"] = row
    gc.unfreeze()
    if pool is not None:
        # accuracy: 4 forward and 4 forward + gradient requests served in one session, each
        # against the oracle at its full size
        sample = list(range(8))
        with KennettServer(executor=ex, max_batch_requests=64, max_inflight=2) as srv:
            reqs = [srv.submit(poolreq[k][0], poolreq[k][1], poolreq[k][2], gradient=poolreq[k][3],
                               R_obs=poolreq[k][4]) for k in sample]
            res = [r.wait(120) for r in reqs]
        ef = eg = 0.0
        for k, r in zip(sample, res):
            m, p_t, w_t, g, obs = poolreq[k]
            pn, wn = p_t.cpu().numpy(), w_t.cpu().numpy()
            if g:
                chi_o, g_o = pool.misfit_gradient(m, pn, wn, obs.cpu().numpy())
                eg = max(eg, _rel(r["grad"].cpu().numpy(), g_o), abs(float(r["chi"]) - chi_o) / chi_o)
            else:
                ef = max(ef, _rel(r["R"].cpu().numpy(), pool.reflectivity(m, pn, wn)))
        for r in reqs:
            r.release()
        out["max_rel_err_vs_oracle"] = {"forward_4_requests": ef, "gradient_4_requests": eg}
    if cpu_rates is not None:
        # per-request CPU replay of the request mix, at the CPU rates of the uneven-batching
        # sample (same model distribution): seconds per request, one request at a time on
        # every host core
        fr, gr = cpu_rates
        secs = [len(p_t) * len(w_t) * (m.n_layers - 1) / (gr if g else fr)
                for m, p_t, w_t, g, _ in poolreq]
        out["cpu_baseline"] = {"value": 1.0 / float(np.mean(secs)), "unit": "requests/s",
                               "kind": "port", "sample": "the request pool (256 requests, 50/50 "
                               "forward / forward + gradient) at the per-update CPU rates of the "
                               "uneven-batching baseline"}
    return out


def run_sharded(args, rank, world, local):
    """N > 1: one gather, slowness sum sharded over the ranks, NCCL all-reduce of U per step
    (strong scaling: total work fixed).  Timed per step with CUDA events, max over ranks."""
    import torch
    import torch.distributed as dist

    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import damped_gather_grid, random_layered_model
    from seismicinversion_b200.sharded import DeviceGatherBackend, gather_sharded, shard_range
    from seismicinversion_b200.source import ricker_10hz

    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                            device_id=torch.device("cuda", local))
    dev = D.require_cuda(torch.device("cuda", local))
    W = WORKLOAD
    model = random_layered_model(W["n_sub"], seed=W["seed"])
    T, nw, npp, pmax = W["T"], W["nw"], W["n_p"], W["p_max"]
    offsets = np.arange(1, W["n_offsets"] + 1) * W["dr"]
    om, omd, p, dp, taper, gamma = damped_gather_grid(T, nw, npp, pmax)
    S = ricker_10hz(om, nw * (2 * np.pi / T))
    decay = np.exp(-gamma * np.arange(2 * nw) * (T / (2 * nw)))
    j0, j1 = shard_range(npp, rank, world)
    tab = D.layer_table(model, dev)
    p_t = torch.as_tensor(p[j0:j1], device=dev)
    pw_t = torch.as_tensor((taper * p)[j0:j1], device=dev)
    w_t = torch.as_tensor(omd, device=dev)
    wr_t = torch.as_tensor(om, device=dev)
    off_t = torch.as_tensor(offsets, device=dev)
    S_t, dec_t = torch.as_tensor(S, device=dev), torch.as_tensor(decay, device=dev)
    R = torch.empty((j1 - j0, nw - 1), dtype=torch.complex128, device=dev)
    U = torch.empty((len(offsets), nw - 1), dtype=torch.complex128, device=dev)
    G = torch.empty((len(offsets), 2 * nw), dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream(dev)

    def step(ev):
        ev[0].record(st)
        D.reflectivity(tab, p_t, w_t, True, out=R)
        D.bessel_sum(R, p_t, pw_t, dp, wr_t, off_t, out=U)
        dist.all_reduce(torch.view_as_real(U), op=dist.ReduceOp.SUM)
        D.traces(U, nw, S=S_t, decay=dec_t, out=G)
        ev[1].record(st)

    for _ in range(args.warmup):
        flush.zero_()
        step([torch.cuda.Event(enable_timing=True) for _ in range(2)])
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    clk = clock_sampler(torch, dev, local)
    clk.start()
    evs = []
    for _ in range(args.steps):
        flush.zero_()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        step(ev)
        evs.append(ev)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = float(np.mean([e[0].elapsed_time(e[1]) for e in evs]))
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t[0])
    # end to end: host model in, the traces (and, second, also the rank's R rows) back to
    # pinned host memory
    backend = DeviceGatherBackend(dev)
    Rh = torch.empty((j1 - j0, nw - 1), dtype=torch.complex128, pin_memory=True)
    Gh = torch.empty((len(offsets), 2 * nw), dtype=torch.float64, pin_memory=True)

    def e2e_seconds(with_R):
        e2e = []
        for k in range(args.warmup + args.steps):
            torch.cuda.synchronize()
            dist.barrier()
            t0 = time.perf_counter()
            _, g, Rs, _ = gather_sharded(model, offsets, T=T, nw=nw, np_slow=npp, p_max=pmax,
                                         source_func=ricker_10hz, free_surface=True,
                                         backend=backend)
            if with_R:
                Rh.copy_(Rs, non_blocking=True)
            Gh.copy_(g, non_blocking=True)
            torch.cuda.synchronize()
            if k >= args.warmup:
                e2e.append(time.perf_counter() - t0)
        t = torch.tensor([statistics.mean(e2e)], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t[0])

    e2e_s = e2e_seconds(False)
    e2e_R_s = e2e_seconds(True)
    upd = (nw - 1) * npp * (W["layers"] - 1)
    if rank == 0:
        print(json.dumps({
            "metric": "(omega,p,interface) reflectivity updates/s, 21-layer gather workload (R grid + J0 gather + traces)",
            "value": upd / (ms * 1e-3), "unit": "updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64 (complex128)",
            "data": "synthetic (seeded random 21-layer model; no dataset exists)",
            "config": {**W, "parallelism": f"slowness-sharded x{world} + NCCL all-reduce of U",
                       "l2": "flushed between steps (256 MB write) and R grid > L2"},
            "e2e": {"value": upd / e2e_s, "unit": "updates/s", "seconds_per_step": e2e_s,
                    "h2d_bytes_per_step": int(tab.numel() * 8 + offsets.nbytes),
                    "d2h_bytes_per_step": int(Gh.numel() * 8)},
            "e2e_with_reflectivity": {
                "value": upd / e2e_R_s, "unit": "updates/s", "seconds_per_step": e2e_R_s,
                "h2d_bytes_per_step": int(tab.numel() * 8 + offsets.nbytes),
                "d2h_bytes_per_step": int(Rh.numel() * 16 + Gh.numel() * 8)},
            "gpu_launches": 5 * args.steps, "clocks": clocks,
        }))
    dist.barrier()
    dist.destroy_process_group()


def run_ours(args, rank, world, local):
    import torch

    from seismicinversion_b200 import device as D
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.kennett_gather_gpu import compute_gather_gpu
    from seismicinversion_b200.source import ricker_10hz

    dist = None  # single GPU (N > 1 runs run_sharded)
    dev = D.require_cuda(torch.device("cuda", local))
    torch.cuda.set_device(dev)
    W = WORKLOAD
    model = random_layered_model(W["n_sub"], seed=W["seed"])
    T, nw, npp, pmax = W["T"], W["nw"], W["n_p"], W["p_max"]
    offsets = np.arange(1, W["n_offsets"] + 1) * W["dr"]
    gamma = np.pi / T
    dw = 2 * np.pi / T
    om = np.arange(1, nw) * dw
    nwm = nw - 1
    dp = pmax / npp
    p = np.arange(1, npp + 1) * dp
    taper = 0.5 * (1 + np.cos(np.pi * p / pmax))
    S = ricker_10hz(om, nw * dw)
    time_axis = np.arange(2 * nw) * (T / (2 * nw))
    decay = np.exp(-gamma * time_axis)

    cpu_base = None
    if rank == 0 and world == 1 and not (args.no_cpu_baseline or args.profile):
        from oracle import kennett_oracle as O  # checker / baseline leg only
        from oracle.cpu_baseline import GatherBaseline

        # the whole workload (every slowness) in one timed sample: it also gives the error of
        # the full R grid and of every trace against the oracle
        n_sample = args.cpu_sample or npp
        cpu_base = GatherBaseline(model, offsets, T, nw, npp, pmax, True, n_sample, chunk=16)

    tab = D.layer_table(model, dev)
    p_t = torch.as_tensor(p, device=dev)
    pw_t = torch.as_tensor(taper * p, device=dev)
    w_t = torch.as_tensor(om + 1j * gamma, device=dev)
    wr_t = torch.as_tensor(om, device=dev)
    off_t = torch.as_tensor(offsets, device=dev)
    S_t = torch.as_tensor(S, device=dev)
    dec_t = torch.as_tensor(decay, device=dev)
    R = torch.empty((npp, nwm), dtype=torch.complex128, device=dev)
    U = torch.empty((len(offsets), nwm), dtype=torch.complex128, device=dev)
    G = torch.empty((len(offsets), 2 * nw), dtype=torch.float64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream(dev)

    def step(ev):
        ev[0].record(st)
        D.reflectivity(tab, p_t, w_t, True, out=R)
        ev[1].record(st)
        D.bessel_sum(R, p_t, pw_t, dp, wr_t, off_t, out=U)
        ev[2].record(st)
        D.traces(U, nw, S=S_t, decay=dec_t, out=G)
        ev[3].record(st)

    def events():
        return [torch.cuda.Event(enable_timing=True) for _ in range(4)]

    for _ in range(args.warmup):
        flush.zero_()
        step(events())
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clock_sampler(torch, dev, local)
    clk.start()
    evs = []
    for _ in range(args.steps):
        flush.zero_()
        ev = events()
        step(ev)
        evs.append(ev)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = clk.stop()
    stage = np.array([[e[i].elapsed_time(e[i + 1]) for i in range(3)] for e in evs])  # ms
    per_step = stage.sum(axis=1)
    ms = float(per_step.mean())
    st_ms = stage.mean(axis=0)
    if dist:
        t = torch.tensor([ms, *st_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, st_ms = float(t[0]), t[1:].cpu().numpy()

    upd = nwm * npp * (W["layers"] - 1)
    value = world * upd / (ms * 1e-3)
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile_run": True, "ms_per_step": ms, "stage_ms": list(map(float, st_ms))}))
        if dist:
            dist.destroy_process_group()
        return

    # end to end through the public API: host model in, host traces out (the reference's
    # call), then the same call also returning the host R grid
    def e2e_seconds(with_R):
        times = []
        for k in range(args.warmup + args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            compute_gather_gpu(model, offsets, T=T, nw=nw, np_slow=npp, p_max=pmax,
                               source_func=ricker_10hz, free_surface=True,
                               return_reflectivity=with_R, copy_outputs=not with_R)
            if k >= args.warmup:
                times.append(time.perf_counter() - t0)
        sec = statistics.mean(times)
        if dist:
            t = torch.tensor([sec], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            sec = float(t[0])
        return sec

    e2e_s = e2e_seconds(False)
    e2e_R_s = e2e_seconds(True)
    # compute_gather_gpu uploads one pinned staging buffer per call (layer-table slot, grid
    # arrays, offsets, source spectrum, decay): its size is the host-to-device traffic
    from seismicinversion_b200.kennett_gather_gpu import _grid_inputs

    h2d = 8 * int(_grid_inputs(float(T), int(nw), int(npp), float(pmax), float(np.pi / T),
                               ricker_10hz, np.ascontiguousarray(offsets, dtype=np.float64)
                               .tobytes())[2][-1])
    d2h = G.numel() * 8
    d2h_R = R.numel() * 16 + G.numel() * 8

    peak = fp64_peak(torch, dev)
    fwd_flops = FLOPS_PER_UPDATE * upd + FLOPS_PER_PAIR_FS * nwm * npp
    bes_terms = len(offsets) * nwm * npp
    kernels = {
        "reflectivity": {"ms": float(st_ms[0]), "alg_tflops": fwd_flops / (st_ms[0] * 1e-3) / 1e12,
                         "updates_per_s": upd / (st_ms[0] * 1e-3)},
        "bessel_sum": {"ms": float(st_ms[1]), "j0_terms_per_s": bes_terms / (st_ms[1] * 1e-3),
                       "alg_tflops": FLOPS_PER_BESSEL_TERM * bes_terms / (st_ms[1] * 1e-3) / 1e12},
        "traces": {"ms": float(st_ms[2])},
    }
    dom = "reflectivity" if st_ms[0] >= st_ms[1] else "bessel_sum"
    traffic = None
    tf = ROOT / "profiles" / "ncu_traffic.json"
    if tf.exists():
        try:
            traffic = json.loads(tf.read_text()).get(dom)
        except Exception:
            traffic = None
    ach = kernels[dom]["alg_tflops"]
    roofline = {"bound": "fp64", "kernel": dom, "achieved": round(ach, 3), "peak": round(peak, 3),
                "unit": "TFLOP/s", "frac": round(ach / peak, 4), "traffic": traffic,
                "traffic_source": "profiles/ncu_traffic.json: dram bytes read + written per launch "
                                  "from one ncu capture of the same kernel and workload, not "
                                  "measured in this run",
                "peak_source": "measured: DFMA probe (kr_bench_fp64_fma), best of 6",
                "nominal_peak": round(NOMINAL_FP64_TFLOPS, 2)}

    cpu = None
    accuracy = {}
    if cpu_base is not None:
        cpu_base.warm()
        dt, Rc, Uc = cpu_base.step()
        Rg = R[torch.as_tensor(cpu_base.rows, device=dev)].cpu().numpy()
        accuracy["c1_R"] = _rel(Rg, Rc)
        if len(cpu_base.rows) == npp:  # the whole workload: the traces too
            go = O.hermitian_traces(Uc * S, nw, decay)
            accuracy["c1_traces"] = _rel(G.cpu().numpy(), go)
            accuracy["c1_traces_first_30s"] = _rel(G.cpu().numpy()[:, time_axis < 30.0],
                                                   go[:, time_axis < 30.0])
        cpu = {"value": cpu_base.updates() / dt, "unit": "updates/s",
               "cores": cpu_base.workers, "kind": "port",
               "sample": f"{len(cpu_base.p)} of {npp} slownesses, all 2047 damped "
                         f"frequencies and 100 offsets: reflectivity + J0 slowness sum (the "
                         f"whole R grid and U of the workload), multiprocessing pool of "
                         f"{cpu_base.workers} (oracle port)",
               "seconds": dt, "host": host_info(cpu_base.workers)}
        cpu_base.close()

    extra = {}
    if world == 1 and not args.no_extra:
        cpu_legs = not args.no_cpu_baseline
        opool = None
        if cpu_legs:
            from oracle.cpu_baseline import ReflectivityPool  # checker / baseline legs only

            opool = ReflectivityPool()
            # the workers' start-up (spawn, imports) occupies every host core for seconds:
            # finish it here so that it does not overlap the device timings below
            opool.warm()
            accuracy.update(accuracy_c0())
        extra["gmm"] = bench_gmm(torch, D, tab, p_t, w_t, R, max(args.steps, 3))
        extra["inversion"] = bench_inversion(torch, dev, max(args.steps, 3), cpu=cpu_legs)
        extra["batched"] = bench_batched(torch, dev, max(args.steps, 2), pool=opool)
        extra["training_data"] = bench_training_data(torch, dev)
        extra["published_configs"] = bench_published_configs(torch, dev)
        b = extra["batched"].get("cpu_baseline")
        extra["serving"] = bench_serving(
            torch, dev, pool=opool,
            cpu_rates=(b["forward_updates_per_s"], b["gradient_updates_per_s"]) if b else None)
        if opool is not None:
            opool.close()
        inv = extra["inversion"].get("max_rel_err_vs_reference", {})
        accuracy.update({"c2_jacobian_vs_reference": inv.get("jacobian_4p_1024w"),
                         "c2_gradient_vs_reference": inv.get("gradient_4p_1024w")})
        for key, src in (("c3", "batched"), ("c4", "serving")):
            for k, v in extra[src].get("max_rel_err_vs_oracle", {}).items():
                if isinstance(v, float):
                    accuracy[f"{key}_{k}"] = v

    if rank == 0:
        line = {
            "metric": "(omega,p,interface) reflectivity updates/s, 21-layer gather workload (R grid + J0 gather + traces)",
            "value": value, "unit": "updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64 (complex128)",
            "data": "synthetic (seeded random 21-layer model; no dataset exists)",
            "config": {**W, "parallelism": "single",
                       "l2": "flushed between steps (256 MB write) and R grid 268 MB > L2"},
            "roofline": roofline, "cpu_baseline": cpu,
            "e2e": {"value": world * upd / e2e_s, "unit": "updates/s", "seconds_per_step": e2e_s,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "call": "compute_gather_gpu(model, offsets, ...) -> (time, offsets, traces)"},
            "e2e_with_reflectivity": {
                "value": world * upd / e2e_R_s, "unit": "updates/s", "seconds_per_step": e2e_R_s,
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h_R),
                "call": "compute_gather_gpu(..., return_reflectivity=True, copy_outputs=False): "
                        "traces and the R grid in pinned host memory"},
            "gpu_launches": 5 * args.steps, "clocks": clocks, "kernels": kernels,
            "max_rel_err_vs_oracle": accuracy,
            **extra,
        }
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle.cpu_baseline import GatherBaseline
    from seismicinversion_b200.earth_models import random_layered_model

    W = WORKLOAD
    model = random_layered_model(W["n_sub"], seed=W["seed"])
    offsets = np.arange(1, W["n_offsets"] + 1) * W["dr"]
    cores = len(os.sched_getaffinity(0))
    n_sample = args.cpu_sample or max(256, 4 * cores)
    b = GatherBaseline(model, offsets, W["T"], W["nw"], W["n_p"], W["p_max"], True, n_sample)
    for _ in range(args.warmup):
        b.step()
    ts = [b.step()[0] for _ in range(args.steps)]
    b.close()
    sec = statistics.mean(ts)
    v = b.updates() / sec
    samp = (f"{len(b.p)} of {W['n_p']} slownesses per step (evenly spaced), all 2047 damped "
            f"frequencies and 100 offsets: reflectivity + J0 slowness sum")
    line = {
        "impl": "reference",
        "metric": "(omega,p,interface) reflectivity updates/s, 21-layer gather workload (R grid + J0 gather + traces)",
        "value": v, "unit": "updates/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec * 1e3,
        "step": f"one bounded sample of the workload: {len(b.p)} of {W['n_p']} slownesses",
        "extrapolated_full_workload_ms": sec * 1e3 * W["n_p"] / len(b.p),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64 (complex128)", "data": "synthetic (seeded random 21-layer model)",
        "config": {**W, "parallelism": "host process pool"},
        "cpu_baseline": {"value": v, "unit": "updates/s", "cores": b.workers, "kind": "port",
                         "sample": samp, "host": host_info(b.workers)},
        "e2e": {"value": v, "unit": "updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "CPU oracle port (NumPy/SciPy restatement of the reference, pinned to its golden "
                "vectors) run like the reference's multiprocessing gather; the Python reference "
                "itself cannot travel to the GPU host",
    }
    print(json.dumps(line))


def profile_case(kind):
    """Small cases for ncu captures: the inversion gradient / Jacobian / Hessian-vector
    products (64 p x 1024 omega, 21 layers), a 256-model uneven batch (seed 3, half gradient),
    the GMM forward, or the 21-layer gather at 512 of its 8192 slownesses (every 16th; all 2047
    damped frequencies and 100 offsets: R grid 17 MB, Bessel sum, traces)."""
    import torch

    from seismicinversion_b200 import device as D

    dev = D.require_cuda()
    if kind == "inversion":
        from seismicinversion_b200.earth_models import random_layered_model

        true, start = random_layered_model(20, seed=2), random_layered_model(20, seed=2)
        start.alpha[1:] *= 1.05
        p = torch.as_tensor(np.linspace(0.05, 0.6, 64), device=dev)
        w = torch.as_tensor(np.arange(1, 1025) * (2 * np.pi / 64), device=dev).to(torch.complex128)
        R_obs = D.reflectivity(D.layer_table(true, dev), p, w)
        tab = D.layer_table(start, dev)
        from seismicinversion_b200.kennett_torch import packed_index

        V = torch.eye(84, dtype=torch.float64, device=dev)[torch.as_tensor(packed_index(21))]
        for _ in range(3):
            D.misfit_gradient(tab, p, w, R_obs)
            D.jacobian(tab, p, w, want_R=False)
        D.misfit_hvp(tab, p, w, R_obs, V)
    elif kind == "gather512":
        from seismicinversion_b200.earth_models import damped_gather_grid, random_layered_model

        om, omd, p, dp, taper, _ = damped_gather_grid(64.0, 2048, 8192, 1.2)
        tab = D.layer_table(random_layered_model(20, seed=1), dev)
        sel = slice(15, 8192, 16)
        p_t = torch.as_tensor(p[sel], device=dev)
        pw_t = torch.as_tensor((taper * p)[sel], device=dev)
        w_t, wr_t = torch.as_tensor(omd, device=dev), torch.as_tensor(om, device=dev)
        off_t = torch.as_tensor(np.arange(1, 101) * 0.5, device=dev)
        for _ in range(2):
            R = D.reflectivity(tab, p_t, w_t, True)
            U = D.bessel_sum(R, p_t, pw_t, 16 * dp, wr_t, off_t)
            D.traces(U, 2048)
    elif kind == "gmm":
        from seismicinversion_b200.earth_models import damped_gather_grid, random_layered_model

        _, omd, p, _, _, _ = damped_gather_grid(64.0, 2048, 8192, 1.2)
        tab = D.layer_table(random_layered_model(20, seed=1), dev)
        p_t, w_t = torch.as_tensor(p, device=dev), torch.as_tensor(omd, device=dev)
        for _ in range(2):
            D.gmm_reflectivity(tab, p_t, w_t, True)
    else:
        from seismicinversion_b200.batch import BatchItem, ModelBatch
        from seismicinversion_b200.earth_models import uneven_batch_specs

        items = []
        for b, (m, p, w) in enumerate(uneven_batch_specs(256, seed=3)):
            if b % 2:
                Ro = D.reflectivity(D.layer_table(m, dev), p, w) * 1.01
                items.append(BatchItem(m, p, w, gradient=True, R_obs=Ro))
            else:
                items.append(BatchItem(m, p, w))
        batch = ModelBatch(items, schedule=(128, 512), device=dev)
        for _ in range(2):
            batch.launch()
    torch.cuda.synchronize()


def main():
    args = parse()
    if args.profile_kernel:
        profile_case(args.profile_kernel)
        return
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif world > 1:
        run_sharded(args, rank, world, local)
    else:
        run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
