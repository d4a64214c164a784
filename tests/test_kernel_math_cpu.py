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
