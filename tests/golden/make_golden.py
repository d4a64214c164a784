"""Generate the golden vectors in this folder by running the REFERENCE implementation.

Run from the repository root with the reference checked out read-only::

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py /path/to/SeismicInversion

It imports ``Kennett_Reflectivity`` from that checkout and stores its outputs (NumPy
reflectivity, batched reflectivity, seismogram, CPU gather, scattering matrices, torch
forward, ``jacobian`` (jacrev), ``frechet_kennett``, ``hessian`` and a small ``invert_taup``
run, and the GlobalMatrix forward) as ``.npz`` files.  The fixtures are committed; tests and the GPU box never need the
reference itself.  Models come from ``seismicinversion_b200.earth_models`` with fixed seeds.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))


def _model_arrays(m):
    return dict(alpha=m.alpha, beta=m.beta, rho=m.rho, thickness=m.thickness,
                Q_alpha=m.Q_alpha, Q_beta=m.Q_beta)


def training_data_golden(ref_root: str) -> None:
    """Reference NeuralInversion.generate_training_data on a small config (GMM forward)."""
    import tempfile

    import torch

    sys.path.insert(0, ref_root)
    from NeuralInversion.inference_config import DataGenConfig
    from NeuralInversion.inference_data import generate_training_data

    cfg = DataGenConfig(n_train=12, n_val=4, n_test=4, nfreq=32, seed=42)
    with tempfile.TemporaryDirectory() as d:
        paths = generate_training_data(d, cfg)
        out = {}
        for split, path in paths.items():
            data = torch.load(path, weights_only=True)
            out[f"{split}_log_params"] = data["log_params"].numpy()
            out[f"{split}_reflectivity"] = data["reflectivity"].numpy()
    np.savez_compressed(HERE / "training_data_small.npz", **out)


def gmm_golden(ref_root: str) -> None:
    """Reference GlobalMatrix forward (NumPy riccati and dense solvers, torch riccati)."""
    sys.path.insert(0, ref_root)
    import torch
    from GlobalMatrix.global_matrix import gmm_reflectivity
    from GlobalMatrix.gmm_torch import gmm_reflectivity_torch
    from Kennett_Reflectivity.kennett_torch import model_to_tensors
    from Kennett_Reflectivity.layer_model import LayerModel

    from seismicinversion_b200.earth_models import default_ocean_crust_model, random_layered_model

    def ref_model(m):
        return LayerModel.from_arrays(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta)

    out = {}
    w255 = np.arange(1, 256, dtype=np.float64) * (2 * np.pi / 64.0)
    cases = [("default", default_ocean_crust_model(), np.array([0.1, 0.3, 0.6, 1.0]), w255),
             ("two", random_layered_model(1, seed=3), np.array([0.1, 0.5]), w255),
             ("three", random_layered_model(2, seed=4), np.array([0.2, 0.7]), w255),
             ("c1", random_layered_model(20, seed=1), np.array([0.05, 0.3, 0.7, 1.1]),
              np.arange(1, 2048, dtype=np.float64) * (2 * np.pi / 64.0) + 1j * np.pi / 64.0)]
    for tag, m, ps, w in cases:
        out.update({f"{tag}_{k}": v for k, v in _model_arrays(m).items()})
        out[f"{tag}_p"], out[f"{tag}_omega"] = ps, w
        for fs in (False, True):
            out[f"{tag}_R_fs{int(fs)}"] = np.stack(
                [gmm_reflectivity(ref_model(m), p, w, free_surface=fs) for p in ps])
        out[f"{tag}_Rdense_fs0"] = np.stack(
            [gmm_reflectivity(ref_model(m), p, w, solver="dense") for p in ps[:2]])
    m2 = random_layered_model(20, seed=2)
    t2 = model_to_tensors(m2)
    om64 = torch.arange(1, 65, dtype=torch.float64) * (2 * np.pi / 64.0)
    out["c2_torch_R_p0.3"] = gmm_reflectivity_torch(**t2, p=0.3, omega=om64).detach().numpy()
    out["c2_torch_omega"] = om64.numpy()
    np.savez_compressed(HERE / "gmm_reflectivity.npz", **out)


def c2_derivs_golden(ref_root: str) -> None:
    """The tau-p inversion workload's derivatives at its own frequency count: 21-layer model
    (seed 2), start = true * exp(0.1 N(0, 1)) (seed 2), omega_k = k 2 pi / 64 (k = 1..1024),
    jacrev Jacobians at 4 of the 64 slownesses and the misfit gradient (autograd.grad, as
    taup_misfit_grad_hessian takes it) over those 4 slownesses."""
    sys.path.insert(0, ref_root)
    import torch
    from Kennett_Reflectivity.kennett_torch import (
        _pack_params,
        _unpack_params,
        jacobian,
        kennett_reflectivity_torch,
        model_to_tensors,
    )
    from Kennett_Reflectivity.layer_model import LayerModel

    from seismicinversion_b200.earth_models import random_layered_model

    torch.set_num_threads(max(1, os.cpu_count() or 1))
    true = random_layered_model(20, seed=2)
    start = random_layered_model(20, seed=2)
    rng = np.random.default_rng(2)
    for name in ("alpha", "beta", "rho"):
        getattr(start, name)[1:] *= np.exp(0.1 * rng.standard_normal(20))
    start.thickness[1:-1] *= np.exp(0.1 * rng.standard_normal(19))

    def tens(m):
        return model_to_tensors(LayerModel.from_arrays(m.alpha, m.beta, m.rho, m.thickness,
                                                       m.Q_alpha, m.Q_beta))

    tt, ts = tens(true), tens(start)
    om = torch.arange(1, 1025, dtype=torch.float64) * (2 * np.pi / 64.0)
    p_all = np.linspace(0.05, 0.6, 64)
    sel = np.array([0, 21, 42, 63])
    out = {f"start_{k}": v for k, v in _model_arrays(start).items()}
    out.update({f"true_{k}": v for k, v in _model_arrays(true).items()})
    out["p"], out["omega"] = p_all[sel], om.numpy()
    m0 = _pack_params(ts["alpha"], ts["beta"], ts["rho"], ts["thickness"]).detach()
    grad = torch.zeros_like(m0)
    chi = 0.0
    for k, p in enumerate(p_all[sel]):
        J = jacobian(ts["alpha"], ts["beta"], ts["rho"], ts["thickness"], ts["Q_alpha"],
                     ts["Q_beta"], float(p), om)
        out[f"J_{k}"] = J.detach().numpy()
        R_obs = kennett_reflectivity_torch(**tt, p=float(p), omega=om).detach()
        out[f"R_obs_{k}"] = R_obs.numpy()
        m = m0.clone().requires_grad_(True)
        a, b, r, h = _unpack_params(m, ts["alpha"], ts["beta"], ts["rho"], ts["thickness"])
        R = kennett_reflectivity_torch(a, b, r, h, ts["Q_alpha"], ts["Q_beta"], float(p), om)
        res = R - R_obs
        misfit = (res.real**2 + res.imag**2).sum()
        (g,) = torch.autograd.grad(misfit, m)
        grad += g
        chi += float(misfit)
    out["grad"], out["chi"] = grad.numpy(), chi
    np.savez_compressed(HERE / "derivs_c2_1024.npz", **out)


def c2_inversion_golden(ref_root: str) -> None:
    """The reference's own invert_taup on the tau-p inversion model: 21 layers (seed 2), its
    uniform +-10 % start (seed 42), exact Hessian (torch.func.hessian per slowness), 10
    iterations -- at 16 slownesses on [0.05, 0.6] and nfreq = 64: the workload's own 64 x 1024
    grid costs the reference about a day of CPU time (~11 s per slowness and iteration for
    64 frequencies, linear in them)."""
    sys.path.insert(0, ref_root)
    import torch
    from Kennett_Reflectivity.layer_model import LayerModel
    from Kennett_Reflectivity.taup_inversion import invert_taup

    from seismicinversion_b200.earth_models import random_layered_model

    torch.set_num_threads(max(1, os.cpu_count() or 1))
    m = random_layered_model(20, seed=2)
    rm = LayerModel.from_arrays(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta)
    res = invert_taup(rm, list(np.linspace(0.05, 0.6, 16)), nfreq=64, perturbation=0.1,
                      max_iter=10, seed=42, tol=0.0)
    np.savez_compressed(
        HERE / "invert_c2.npz",
        misfit=np.array(res.misfit_history), grad_norm=np.array(res.grad_norm_history),
        param_err=np.array(res.param_error_history), n_iter=res.n_iterations,
        init_alpha=res.initial_model.alpha, init_beta=res.initial_model.beta,
        init_rho=res.initial_model.rho, init_thickness=res.initial_model.thickness,
        rec_alpha=res.recovered_model.alpha, rec_beta=res.recovered_model.beta,
        rec_rho=res.recovered_model.rho, rec_thickness=res.recovered_model.thickness,
    )


def main(ref_root: str) -> None:
    sys.path.insert(0, ref_root)
    os.environ.setdefault("TQDM_DISABLE", "1")
    import torch

    from Kennett_Reflectivity.frechet_analytical import frechet_kennett
    from Kennett_Reflectivity.kennett_gather import compute_gather
    from Kennett_Reflectivity.kennett_reflectivity import kennett_reflectivity
    from Kennett_Reflectivity.kennett_reflectivity_gpu import kennett_reflectivity_batch
    from Kennett_Reflectivity.kennett_seismogram import compute_seismogram
    from Kennett_Reflectivity.kennett_torch import (
        hessian,
        jacobian,
        kennett_reflectivity_torch,
        model_to_tensors,
    )
    from Kennett_Reflectivity.layer_model import LayerModel, complex_slowness, vertical_slowness
    from Kennett_Reflectivity.scattering_matrices import (
        ocean_bottom_interface,
        solid_solid_interface,
    )
    from Kennett_Reflectivity.source import ricker_spectrum
    from Kennett_Reflectivity.taup_inversion import invert_taup

    from seismicinversion_b200.earth_models import default_ocean_crust_model, random_layered_model

    torch.set_num_threads(max(1, os.cpu_count() or 1))

    def ref_model(m):
        return LayerModel.from_arrays(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta)

    src10 = lambda w, wmax: ricker_spectrum(w, 100.0 * np.pi)  # noqa: E731

    # 1. single trace, 6-layer model (seed 0), p = 0.2, T = 64, nw = 2048, free surface, 10 Hz
    m0 = random_layered_model(5, seed=0)
    om = np.arange(1, 2048, dtype=np.float64) * (2 * np.pi / 64.0)
    R0 = kennett_reflectivity(ref_model(m0), 0.2, om, free_surface=True)
    t0, tr0 = compute_seismogram(ref_model(m0), 0.2, T=64.0, nw=2048, source_func=src10,
                                 free_surface=True)
    np.savez_compressed(HERE / "c0_trace.npz", **_model_arrays(m0), p=0.2, omega=om, R=R0,
                        time=t0, trace=tr0)

    # 2. default model, real and damped frequencies, with / without free surface
    md = default_ocean_crust_model()
    ps = np.array([0.01, 0.1, 0.2, 0.3, 0.4, 0.6, 0.8, 1.2])
    om63 = np.arange(1, 64, dtype=np.float64) * (2 * np.pi / 64.0)
    out = {}
    for tag, omg in (("real", om63), ("damped", om63 + 1j * np.pi / 64.0)):
        for fs in (False, True):
            key = f"{tag}_fs{int(fs)}"
            out["R_" + key] = np.stack(
                [kennett_reflectivity(ref_model(md), p, omg, free_surface=fs) for p in ps])
            out["Rb_" + key] = kennett_reflectivity_batch(ref_model(md), ps, omg, free_surface=fs)
            out["omega_" + key] = omg
    np.savez_compressed(HERE / "default_model_R.npz", **_model_arrays(md), p=ps, **out)

    # 3. 21-layer gather model (seed 1): a slowness subset of the 8192-point gather grid,
    #    2047 damped frequencies, free surface
    m1 = random_layered_model(20, seed=1)
    dp = 1.2 / 8192
    jsel = np.array([1, 64, 512, 1024, 2048, 3072, 4096, 5000, 6000, 6827, 7000, 7400,
                     7800, 8000, 8100, 8192])
    p1 = jsel * dp
    omd = om + 1j * np.pi / 64.0
    R1 = np.stack([kennett_reflectivity(ref_model(m1), p, omd, free_surface=True) for p in p1])
    np.savez_compressed(HERE / "c1_subset_R.npz", **_model_arrays(m1), p=p1, j=jsel, omega=omd,
                        R=R1)

    # 4. small CPU gathers (float64 reference gather)
    offs = np.arange(1, 9, dtype=np.float64) * 2.0
    tg, _, g1 = compute_gather(ref_model(m1), offs, T=64.0, nw=256, np_slow=128, p_max=1.2,
                               source_func=src10, n_workers=1, free_surface=True)
    tgd, _, gd = compute_gather(ref_model(md), offs, T=32.0, nw=128, np_slow=96, p_max=1.0,
                                n_workers=1, free_surface=False)
    np.savez_compressed(HERE / "gather_small.npz", **{f"m1_{k}": v for k, v in _model_arrays(m1).items()},
                        offsets=offs, time_m1=tg, gather_m1=g1, time_md=tgd, gather_md=gd)

    # 5. scattering matrices and slownesses for the default model's interfaces
    sc = {}
    for p in (0.1, 0.2, 0.4, 0.8):
        cp = complex(p)
        s_p = ref_model(md).complex_slowness_p()
        s_s = ref_model(md).complex_slowness_s()
        bc = ref_model(md).complex_velocity_s()
        eta = np.array([vertical_slowness(s, cp) for s in s_p])
        neta = np.array([0j] + [vertical_slowness(s, cp) for s in s_s[1:]])
        ob = ocean_bottom_interface(p, eta[0], md.rho[0], eta[1], neta[1], md.rho[1], bc[1])
        mats = [np.stack([ob.Rd, ob.Ru, ob.Tu, ob.Td])]
        for il in range(1, md.n_layers - 1):
            ss = solid_solid_interface(p, eta[il], neta[il], md.rho[il], bc[il], eta[il + 1],
                                       neta[il + 1], md.rho[il + 1], bc[il + 1])
            mats.append(np.stack([ss.Rd, ss.Ru, ss.Tu, ss.Td]))
        sc[f"eta_{p}"] = eta
        sc[f"neta_{p}"] = neta
        sc[f"scat_{p}"] = np.stack(mats)
    sc["cslow"] = np.array([complex_slowness(1.5, 20000), complex_slowness(3.0, 100)])
    np.savez_compressed(HERE / "scatter_default.npz", **sc)

    # 6. derivatives on the default model (32 frequencies), jacrev and analytical Frechet
    om32 = np.arange(1, 33, dtype=np.float64) * (2 * np.pi / 64.0)
    tens = model_to_tensors(md)
    om32_t = torch.tensor(om32, dtype=torch.float64)
    jac = {}
    for p in (0.2, 0.4):
        for fs in (False, True):
            J = jacobian(tens["alpha"], tens["beta"], tens["rho"], tens["thickness"],
                         tens["Q_alpha"], tens["Q_beta"], p, om32_t, free_surface=fs)
            jac[f"J_p{p}_fs{int(fs)}"] = J.detach().numpy()
        th = md.thickness.copy()
        th[np.isinf(th)] = 1e30
        jac[f"F_p{p}"] = frechet_kennett(md.alpha, md.beta, md.rho, th, md.Q_alpha, md.Q_beta,
                                         p, om32)
    R_obs = kennett_reflectivity_torch(**tens, p=0.2, omega=om32_t).detach()
    ap = tens["alpha"].clone()
    ap[1] = ap[1] * 1.02
    H = hessian(ap, tens["beta"], tens["rho"], tens["thickness"], tens["Q_alpha"],
                tens["Q_beta"], 0.2, om32_t, R_obs=R_obs)
    jac["H_p0.2_alpha1x1.02"] = H.detach().numpy()
    jac["R_obs_p0.2"] = R_obs.numpy()
    np.savez_compressed(HERE / "derivs_default.npz", omega=om32, **jac)

    # 7. 21-layer inversion model (seed 2): torch forward and jacrev at two slownesses,
    #    64 frequencies (k = 1..64, dw = 2 pi / 64)
    m2 = random_layered_model(20, seed=2)
    t2 = model_to_tensors(m2)
    om64 = torch.arange(1, 65, dtype=torch.float64) * (2 * np.pi / 64.0)
    d2 = {}
    for p in (0.05, 0.3):
        d2[f"R_p{p}"] = kennett_reflectivity_torch(**t2, p=p, omega=om64).detach().numpy()
        d2[f"J_p{p}"] = jacobian(t2["alpha"], t2["beta"], t2["rho"], t2["thickness"],
                                 t2["Q_alpha"], t2["Q_beta"], p, om64).detach().numpy()
    om1024 = torch.arange(1, 1025, dtype=torch.float64) * (2 * np.pi / 64.0)
    d2["R1024_p0.3"] = kennett_reflectivity_torch(**t2, p=0.3, omega=om1024).detach().numpy()
    np.savez_compressed(HERE / "derivs_c2.npz", **_model_arrays(m2), omega=om64.numpy(), **d2)

    # 8. a small Newton-LM inversion (the reference test's 5 % case)
    res = invert_taup(default_ocean_crust_model(), [0.1, 0.2, 0.3, 0.4], nfreq=32,
                      perturbation=0.05, max_iter=30)
    np.savez_compressed(
        HERE / "invert_small.npz",
        misfit=np.array(res.misfit_history), grad_norm=np.array(res.grad_norm_history),
        param_err=np.array(res.param_error_history), n_iter=res.n_iterations,
        converged=res.converged,
        init_alpha=res.initial_model.alpha, init_beta=res.initial_model.beta,
        init_rho=res.initial_model.rho, init_thickness=res.initial_model.thickness,
        rec_alpha=res.recovered_model.alpha, rec_beta=res.recovered_model.beta,
        rec_rho=res.recovered_model.rho, rec_thickness=res.recovered_model.thickness,
    )
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) < 2 or sys.argv[1].startswith("--"):
        sys.exit("usage: make_golden.py <reference checkout> [--training-data-only | --gmm-only"
                 " | --c2-derivs-only | --c2-inversion-only]")
    root = sys.argv[1]
    if "--training-data-only" in sys.argv:
        training_data_golden(root)
    elif "--gmm-only" in sys.argv:
        gmm_golden(root)
    elif "--c2-derivs-only" in sys.argv:
        c2_derivs_golden(root)
    elif "--c2-inversion-only" in sys.argv:
        c2_inversion_golden(root)
    else:
        main(root)
        training_data_golden(root)
        gmm_golden(root)
        c2_derivs_golden(root)
        c2_inversion_golden(root)
