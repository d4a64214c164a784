"""The kernels' arithmetic (csrc/kr_math.cuh), compiled for the host with g++, against the
reference's golden vectors and the oracle.  Catches math errors without a GPU; the GPU
tests then check the same code on the device."""

import ctypes
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import rel_err
from oracle import kennett_oracle as O

HERE = Path(__file__).resolve().parent


@pytest.fixture(scope="module")
def emu(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = tmp_path_factory.mktemp("emu") / "libkr_emulate.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(out),
                    str(HERE / "cpu_emulation" / "kr_emulate.cpp")], check=True)
    lib = ctypes.CDLL(str(out))

    def run(model, p, omega, fs=False):
        from seismicinversion_b200.layer_model import pack_layers

        tab = np.ascontiguousarray(pack_layers(model))
        p = np.ascontiguousarray(np.atleast_1d(p), dtype=np.float64)
        w = np.ascontiguousarray(np.asarray(omega, dtype=np.complex128))
        out = np.zeros((len(p), len(w)), dtype=np.complex128)
        lib.emu_reflectivity(ctypes.c_void_p(tab.ctypes.data), model.n_layers,
                             ctypes.c_void_p(p.ctypes.data), len(p),
                             ctypes.c_void_p(w.ctypes.data), len(w), int(fs),
                             ctypes.c_void_p(out.ctypes.data))
        return out

    return run


def _m(g):
    from seismicinversion_b200.layer_model import LayerModel

    return LayerModel(*[g[k] for k in ("alpha", "beta", "rho", "thickness", "Q_alpha", "Q_beta")])


@pytest.mark.parametrize("tag", ["real_fs0", "damped_fs1"])
def test_default_model(emu, golden, tag):
    g = golden("default_model_R.npz")
    R = emu(_m(g), g["p"], g["omega_" + tag], tag.endswith("1"))
    for i in range(len(g["p"])):
        tol = max(1e-10, 10.0 * rel_err(g["Rb_" + tag][i], g["R_" + tag][i]))
        assert rel_err(R[i], g["R_" + tag][i]) < tol


def test_c1_subset(emu, golden):
    g = golden("c1_subset_R.npz")
    R = emu(_m(g), g["p"], g["omega"], True)
    for i in range(len(g["p"])):
        assert rel_err(R[i], g["R"][i]) < 1e-10


def test_random_depths(emu):
    from seismicinversion_b200.earth_models import random_layered_model

    for n_sub in (1, 4, 40):
        m = random_layered_model(n_sub, seed=7 + n_sub)
        p = np.array([0.0, 0.2, 0.55, 1.0])
        w = np.arange(1, 64) * 0.3 + 0.05j
        R = emu(m, p, w, True)
        Ro = O.reflectivity(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta, p, w, True)
        assert rel_err(R, Ro) < 1e-10


@pytest.fixture(scope="module")
def emu_jac(emu, tmp_path_factory):
    import glob

    so = sorted(glob.glob(str(tmp_path_factory.getbasetemp() / "emu*" / "libkr_emulate.so")))[-1]
    lib = ctypes.CDLL(so)

    def run(model, p, omega, fs=False):
        from seismicinversion_b200.layer_model import pack_layers

        tab = np.ascontiguousarray(pack_layers(model))
        L = model.n_layers
        p = np.ascontiguousarray(np.atleast_1d(p), dtype=np.float64)
        w = np.ascontiguousarray(np.asarray(omega, dtype=np.complex128))
        R = np.zeros((len(p), len(w)), dtype=np.complex128)
        J = np.zeros((len(p), 4 * L, len(w)), dtype=np.complex128)
        lib.emu_jacobian(ctypes.c_void_p(tab.ctypes.data), L, ctypes.c_void_p(p.ctypes.data),
                         len(p), ctypes.c_void_p(w.ctypes.data), len(w), int(fs),
                         ctypes.c_void_p(R.ctypes.data), ctypes.c_void_p(J.ctypes.data))
        return R, J

    return run


def packed(J, L):
    """Full [4L] layer-parameter Jacobian -> the reference's packed sub-ocean order
    [alpha_1..N, beta_1..N, rho_1..N, h_1..N-1] (kennett_torch.py:552-571)."""
    idx = [0 * L + l for l in range(1, L)] + [1 * L + l for l in range(1, L)] + \
          [2 * L + l for l in range(1, L)] + [3 * L + l for l in range(1, L - 1)]
    return np.moveaxis(J[..., idx, :], -1, -2)


@pytest.mark.parametrize("p", [0.2, 0.4])
@pytest.mark.parametrize("fs", [0, 1])
def test_adjoint_vs_reference_jacrev(emu_jac, golden, p, fs):
    from seismicinversion_b200.earth_models import default_ocean_crust_model

    g = golden("derivs_default.npz")
    m = default_ocean_crust_model()
    R, J = emu_jac(m, p, g["omega"], fs)
    Jp = packed(J, m.n_layers)[0]
    assert rel_err(Jp, g[f"J_p{p}_fs{fs}"]) < 1e-10


def test_adjoint_vs_reference_jacrev_21_layers(emu_jac, golden):
    g = golden("derivs_c2.npz")
    from seismicinversion_b200.layer_model import LayerModel

    m = LayerModel(*[g[k] for k in ("alpha", "beta", "rho", "thickness", "Q_alpha", "Q_beta")])
    for p in (0.05, 0.3):
        R, J = emu_jac(m, p, g["omega"])
        assert rel_err(R[0], g[f"R_p{p}"]) < 1e-12
        assert rel_err(packed(J, m.n_layers)[0], g[f"J_p{p}"]) < 1e-10


def test_adjoint_deep_model_recomputed_segments(emu_jac):
    """101 layers: 99 steps do not fit one 64-step tape, so the reverse sweep runs over two
    checkpointed segments, the second recomputed; columns checked against central
    differences of the oracle."""
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(100, seed=31)
    L = m.n_layers
    w = np.arange(1, 17) * 0.25 + 0.04j
    p = np.array([0.1, 0.45])
    R, J = emu_jac(m, p, w, 1)
    Ro = O.reflectivity(m.alpha, m.beta, m.rho, m.thickness, m.Q_alpha, m.Q_beta, p, w, True)
    assert rel_err(R, Ro) < 1e-10
    base = [m.alpha, m.beta, m.rho, m.thickness]
    for k, l in [(0, 1), (1, 20), (2, 50), (3, 60), (0, 97), (1, 99), (2, 100), (3, 99)]:
        arrs = [b.copy() for b in base]
        d = 1e-6 * arrs[k][l]
        arrs[k][l] += d
        Rp = O.reflectivity(*arrs, m.Q_alpha, m.Q_beta, p, w, True)
        arrs[k][l] -= 2 * d
        Rm = O.reflectivity(*arrs, m.Q_alpha, m.Q_beta, p, w, True)
        fd = (Rp - Rm) / (2 * d)
        assert rel_err(J[:, k * L + l], fd) < 1e-6, (k, l, rel_err(J[:, k * L + l], fd))


def test_adjoint_vs_fd_all_parameters(emu_jac):
    """Every layer parameter incl. the ocean's alpha, rho, h, damped frequencies, free surface."""
    from seismicinversion_b200.earth_models import random_layered_model

    m = random_layered_model(4, seed=11)
    L = m.n_layers
    w = np.arange(1, 40) * 0.2 + 0.03j
    p = np.array([0.15, 0.5])
    for fs in (0, 1):
        R, J = emu_jac(m, p, w, fs)
        base = [m.alpha, m.beta, m.rho, m.thickness]
        for k in range(4):
            for l in range(L):
                if (k == 1 and l == 0) or (k == 3 and l == L - 1):
                    assert np.all(J[:, k * L + l] == 0)
                    continue
                arrs = [b.copy() for b in base]
                d = 1e-6 * arrs[k][l]
                arrs[k][l] += d
                Rp = O.reflectivity(*arrs, m.Q_alpha, m.Q_beta, p, w, bool(fs))
                arrs[k][l] -= 2 * d
                Rm = O.reflectivity(*arrs, m.Q_alpha, m.Q_beta, p, w, bool(fs))
                fd = (Rp - Rm) / (2 * d)
                assert rel_err(J[:, k * L + l], fd) < 1e-6, (fs, k, l, rel_err(J[:, k * L + l], fd))


@pytest.fixture(scope="module")
def reference_form(tmp_path_factory):
    """The reference's full-matrix recursion in 80-bit extended precision (extended=1) or in
    double (extended=0), from tests/cpu_emulation/kr_extended.cpp."""
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    out = tmp_path_factory.mktemp("ext") / "libkr_extended.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(out),
                    str(HERE / "cpu_emulation" / "kr_extended.cpp")], check=True)
    lib = ctypes.CDLL(str(out))

    def run(model, p, omega, fs, extended):
        from seismicinversion_b200.layer_model import pack_layers

        tab = np.ascontiguousarray(pack_layers(model))
        p = np.ascontiguousarray(np.atleast_1d(p), dtype=np.float64)
        w = np.ascontiguousarray(np.asarray(omega, dtype=np.complex128))
        out = np.zeros((len(p), len(w)), dtype=np.complex128)
        lib.emu_reflectivity_reference_form(ctypes.c_void_p(tab.ctypes.data), model.n_layers,
                                            ctypes.c_void_p(p.ctypes.data), len(p),
                                            ctypes.c_void_p(w.ctypes.data), len(w), int(fs),
                                            int(extended), ctypes.c_void_p(out.ctypes.data))
        return out

    return run


def test_symmetric_step_against_extended_precision(emu, reference_form):
    """The kernels' symmetric adjugate step against an 80-bit evaluation of the reference's
    full-matrix recursion, at the large slownesses where the reference's default model is
    ill-conditioned (every layer evanescent, interface determinants cancelling): the kernel
    form stays within 2.5e-10 and is several times closer than the reference's own form in
    double; on the 21-layer gather model both are at rounding level."""
    from seismicinversion_b200.earth_models import default_ocean_crust_model, random_layered_model

    w = np.arange(1, 2048, 3) * (2 * np.pi / 64) + 1j * (np.pi / 64)
    p = np.array([0.3, 0.9, 1.0, 1.012, 1.022, 1.041, 1.078, 1.087, 1.1, 1.2])
    m = default_ocean_crust_model()
    err_kernel, err_ref = [], []
    for fs in (False, True):
        x = reference_form(m, p, w, fs, extended=True)
        den = np.abs(x).max(axis=1)
        err_kernel.append(np.abs(emu(m, p, w, fs) - x).max(axis=1) / den)
        err_ref.append(np.abs(reference_form(m, p, w, fs, extended=False) - x).max(axis=1) / den)
    err_kernel, err_ref = np.concatenate(err_kernel), np.concatenate(err_ref)
    assert err_kernel.max() < 2.5e-10, err_kernel
    assert err_kernel.sum() < 0.5 * err_ref.sum(), (err_kernel.sum(), err_ref.sum())
    m21 = random_layered_model(20, seed=1)
    for fs in (False, True):
        x = reference_form(m21, p, w, fs, extended=True)
        assert rel_err(emu(m21, p, w, fs), x) < 2e-12


def test_symmetric_step_diverse_models(emu, reference_form):
    """40 random models far from the gather model (1-30 layers below the ocean, thin and thick
    layers, low-velocity zones, Q from 10 to 1e4, both surface conditions) at random
    slownesses and damped frequencies: the kernels' step stays within 5e-11 of the 80-bit
    evaluation of the reference's recursion (the reference's own double form reaches ~3e-10)."""
    from seismicinversion_b200.layer_model import LayerModel

    rng = np.random.default_rng(5)
    worst_kernel = worst_ref = 0.0
    for _ in range(40):
        n = int(rng.integers(1, 31))
        vp = rng.uniform(1.6, 7.0, n)
        if rng.random() < 0.6:
            vp = np.sort(vp)
        vs = vp / rng.uniform(1.6, 2.4, n)
        h = np.exp(rng.uniform(np.log(0.01), np.log(3.0), n))
        h[-1] = np.inf
        qa = np.exp(rng.uniform(np.log(10.0), np.log(1e4), n))
        qb = qa / rng.uniform(1.5, 3.0, n)
        m = LayerModel(np.r_[1.5, vp], np.r_[0.0, vs], np.r_[1.0, 0.31 * (1000 * vp) ** 0.25],
                       np.r_[rng.uniform(0.1, 4.0), h], np.r_[2e4, qa], np.r_[1e10, qb])
        p = np.sort(rng.uniform(0.0, 1.2, 8))
        w = np.sort(rng.uniform(0.1, 200.0, 60)) + 1j * (np.pi / 64)
        fs = bool(rng.random() < 0.5)
        x = reference_form(m, p, w, fs, extended=True)
        den = np.abs(x).max(axis=1)
        worst_kernel = max(worst_kernel, (np.abs(emu(m, p, w, fs) - x).max(axis=1) / den).max())
        worst_ref = max(worst_ref, (np.abs(reference_form(m, p, w, fs, extended=False) - x)
                                    .max(axis=1) / den).max())
    assert worst_kernel < 5e-11, (worst_kernel, worst_ref)
    assert worst_kernel <= worst_ref, (worst_kernel, worst_ref)


@pytest.fixture(scope="module")
def emu_hvp(emu, tmp_path_factory):
    import glob

    so = sorted(glob.glob(str(tmp_path_factory.getbasetemp() / "emu*" / "libkr_emulate.so")))[-1]
    lib = ctypes.CDLL(so)

    def run(tab, p, omega, fs, v, mode, R_obs=None):
        tab = np.ascontiguousarray(tab, dtype=np.float64)
        L = tab.shape[1]
        p = np.ascontiguousarray(np.atleast_1d(p), dtype=np.float64)
        w = np.ascontiguousarray(np.asarray(omega, dtype=np.complex128))
        v = np.ascontiguousarray(v, dtype=np.float64)
        Ro = np.ascontiguousarray(np.zeros((len(p), len(w)), complex) if R_obs is None else R_obs)
        hv = np.zeros(4 * L)
        jd = np.zeros((len(p), 4 * L, len(w)), dtype=np.complex128)
        lib.emu_hvp(ctypes.c_void_p(tab.ctypes.data), L, ctypes.c_void_p(p.ctypes.data), len(p),
                    ctypes.c_void_p(w.ctypes.data), len(w), int(fs), ctypes.c_void_p(v.ctypes.data),
                    int(mode), ctypes.c_void_p(Ro.ctypes.data), ctypes.c_void_p(hv.ctypes.data),
                    ctypes.c_void_p(jd.ctypes.data))
        return hv, jd

    return run


@pytest.mark.parametrize("n_sub", [4, 9, 45])
def test_tangent_of_adjoint_vs_differences(emu_jac, emu_hvp, n_sub):
    """The dual-number sweep of kr_hvp.cuh (the code the second-derivative kernels run):
    d/dv of the Jacobian and the misfit Hessian-vector product H v against central
    differences of the emulated adjoint along v, with and without free surface, for 5, 10 and
    47 layers (the last over two checkpointed tape segments).  Tolerance 1e-7 (the differences'
    own truncation and rounding)."""
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.layer_model import pack_layers

    m = random_layered_model(n_sub, seed=3)
    tab = np.ascontiguousarray(pack_layers(m))
    L = tab.shape[1]
    tab[3, -1] = 1e30
    p = np.array([0.1, 0.35, 0.7])
    w = np.arange(1, 13 if n_sub > 20 else 41) * (2 * np.pi / 64) + 1j * np.pi / 64
    rng = np.random.default_rng(n_sub)

    def jac(t, fs):
        from seismicinversion_b200.layer_model import LayerModel

        mm = LayerModel(*[t[k].copy() for k in range(6)])
        return emu_jac(mm, p, w, fs)

    for fs in (False, True):
        v = rng.standard_normal(4 * L) * np.concatenate([tab[0], tab[1], tab[2],
                                                         np.r_[tab[3, :-1], 0.0]])
        v[L] = 0.0  # the ocean's beta

        def shifted(s):
            t = tab.copy()
            t[0] += s * v[:L]
            t[1] += s * v[L:2 * L]
            t[2] += s * v[2 * L:3 * L]
            t[3, :-1] += s * v[3 * L:4 * L - 1]
            return t

        eps = 1e-6
        fd_J = (jac(shifted(eps), fs)[1] - jac(shifted(-eps), fs)[1]) / (2 * eps)
        _, jd = emu_hvp(tab, p, w, fs, v, 1)
        assert rel_err(jd, fd_J) < 1e-7
        R0 = jac(tab, fs)[0]
        Ro = R0 * 0.9 + 0.01

        def grad(t):
            R, J = jac(t, fs)
            return (2 * np.conj(R - Ro)[:, None, :] * J).real.sum((0, 2))

        fd_g = (grad(shifted(eps)) - grad(shifted(-eps))) / (2 * eps)
        hv, _ = emu_hvp(tab, p, w, fs, v, 0, Ro)
        assert rel_err(hv, fd_g) < 1e-7


@pytest.fixture(scope="module")
def emu_lib(emu, tmp_path_factory):
    import glob

    so = sorted(glob.glob(str(tmp_path_factory.getbasetemp() / "emu*" / "libkr_emulate.so")))[-1]
    return ctypes.CDLL(so)


def test_frequency_sum_adjoint_vs_jacobian_contraction(emu_jac, emu_lib):
    """adjoint_pair_sums + sums_contract_layer (the gradient and vector-Jacobian-product
    kernels: per-step adjoints summed over frequency, contracted with the coefficient tangents
    once per slowness and interface) equal the per-frequency Jacobian contracted with the seed,
    to 1e-12, for the misfit (with chi) and an arbitrary cotangent, with and without free
    surface, on a 6-layer and a 101-layer model (the latter over checkpointed segments)."""
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.layer_model import pack_layers

    lib = emu_lib
    rng = np.random.default_rng(3)
    for n_sub, fs in ((5, False), (5, True), (100, True)):
        m = random_layered_model(n_sub, seed=21 + n_sub)
        L = m.n_layers
        tab = np.ascontiguousarray(pack_layers(m))
        p = np.array([0.1, 0.45, 0.8])
        w = np.ascontiguousarray(np.arange(1, 23) * 0.3 + 0.02j)
        R, J = emu_jac(m, p, w, fs)
        for vjp in (0, 1):
            obs = (0.8 * R + 0.05) if vjp == 0 else (rng.standard_normal(R.shape)
                                                     + 1j * rng.standard_normal(R.shape))
            obs = np.ascontiguousarray(obs)
            out = np.zeros(4 * L + 1)
            lib.emu_gradient_sums(ctypes.c_void_p(tab.ctypes.data), L,
                                  ctypes.c_void_p(p.ctypes.data), len(p),
                                  ctypes.c_void_p(w.ctypes.data), len(w), int(fs), vjp,
                                  ctypes.c_void_p(obs.ctypes.data), ctypes.c_void_p(out.ctypes.data))
            seed = np.conj(obs) if vjp else 2 * np.conj(R - obs)
            want = (seed[:, None, :] * J).real.sum((0, 2))
            assert rel_err(out[:4 * L], want) < 1e-12, (n_sub, fs, vjp)
            if not vjp:
                assert abs(out[4 * L] - np.sum(np.abs(R - obs) ** 2)) < 1e-12 * out[4 * L]


def test_frequency_sum_hvp_vs_per_step_dual(emu_hvp, emu_lib):
    """hvp_pair_sums + hvp_sums_contract_layer (the Hessian-vector-product kernel: dual
    adjoints summed over frequency, contracted once per slowness and interface) equal the
    per-step dual contraction of hvp_pair to 1e-12, with and without free surface, for 6 and
    47 layers (the latter over checkpointed segments)."""
    from seismicinversion_b200.earth_models import random_layered_model
    from seismicinversion_b200.layer_model import pack_layers

    rng = np.random.default_rng(8)
    for n_sub, fs in ((5, False), (5, True), (45, True)):
        m = random_layered_model(n_sub, seed=50 + n_sub)
        tab = np.ascontiguousarray(pack_layers(m))
        L = tab.shape[1]
        tab[3, -1] = 1e30
        p = np.array([0.12, 0.4, 0.75])
        w = np.ascontiguousarray(np.arange(1, 15) * 0.35 + 0.03j)
        v = rng.standard_normal(4 * L) * np.concatenate([tab[0], tab[1], tab[2],
                                                         np.r_[tab[3, :-1], 0.0]])
        v[L] = 0.0
        v = np.ascontiguousarray(v)
        Ro = np.ascontiguousarray((rng.standard_normal((3, len(w)))
                                   + 1j * rng.standard_normal((3, len(w)))) * 0.1)
        want, _ = emu_hvp(tab, p, w, fs, v, 0, Ro)
        got = np.zeros(4 * L)
        emu_lib.emu_hvp_sums(ctypes.c_void_p(tab.ctypes.data), L,
                             ctypes.c_void_p(p.ctypes.data), len(p),
                             ctypes.c_void_p(w.ctypes.data), len(w), int(fs),
                             ctypes.c_void_p(v.ctypes.data), ctypes.c_void_p(Ro.ctypes.data),
                             ctypes.c_void_p(got.ctypes.data))
        assert rel_err(got, want) < 1e-12, (n_sub, fs, rel_err(got, want))
