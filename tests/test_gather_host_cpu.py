"""Host logic of compute_gather_gpu that needs no GPU: the grid-only part of the pinned staging
buffer (_grid_inputs): 16-byte aligned sections after a 6 x 256 layer-table slot, contents equal
to the reference's grid (kennett_gather_gpu.py:198-225 conventions), and a bounded cache."""

import numpy as np

from seismicinversion_b200 import kennett_gather_gpu as K
from seismicinversion_b200.earth_models import damped_gather_grid, seismogram_omega
from seismicinversion_b200.source import ricker_spectrum


def test_grid_inputs_layout_and_contents():
    T, nw, n_p, pmax = 64.0, 256, 300, 1.2
    gamma = np.pi / T
    offs = np.array([0.5, 1.0, 7.25])
    time, dp, off, sizes, static = K._grid_inputs(T, nw, n_p, pmax, gamma, None, offs.tobytes())
    assert all(int(o) % 2 == 0 for o in off)  # float64 offsets: 16-byte aligned sections
    assert sizes[0] == 6 * 256 and off[1] >= 6 * 256
    om, omd, p, dp_ref, taper, _ = damped_gather_grid(T, nw, n_p, pmax)
    assert dp == dp_ref
    sec = [static[a - off[1]:a - off[1] + n] for a, n in zip(off[1:-1], sizes[1:])]
    assert np.array_equal(sec[0], p)
    assert np.array_equal(sec[1], taper * p)
    assert np.array_equal(sec[2], om) and np.array_equal(sec[3], omd.real)
    assert np.all(sec[4] == gamma)
    assert np.array_equal(sec[5], offs)
    S = ricker_spectrum(seismogram_omega(T, nw), nw * 2 * np.pi / T)
    assert np.array_equal(sec[6], np.asarray(S, dtype=np.complex128).view(np.float64))
    assert np.array_equal(sec[7], np.exp(-gamma * time))
    assert len(time) == 2 * nw and time[1] == T / (2 * nw)


def test_grid_inputs_cache():
    K._GRID_CACHE.clear()
    args = (64.0, 128, 64, 1.2, np.pi / 64, None)
    a = K._grid_inputs(*args, np.array([1.0]).tobytes())
    assert K._grid_inputs(*args, np.array([1.0]).tobytes()) is a
    for k in range(12):
        K._grid_inputs(*args, np.array([2.0 + k]).tobytes())
    assert len(K._GRID_CACHE) <= 8


def test_output_file_formats(tmp_path):
    """The reference CLIs' file formats: a .npz gather with keys time / offsets / gather
    (kennett_gather_gpu.py:429-436) and a two-column %.8e text seismogram
    (kennett_seismogram.py:294-296)."""
    from seismicinversion_b200.kennett_seismogram import save_seismogram_txt

    rng = np.random.default_rng(1)
    t = np.arange(16) * 0.25
    offs = np.array([0.5, 1.0, 1.5])
    g = rng.standard_normal((3, 16))
    out = K.save_gather_npz(tmp_path / "gather.png", t, offs, g)
    assert out.suffix == ".npz"
    z = np.load(out)
    assert sorted(z.files) == ["gather", "offsets", "time"]
    assert np.array_equal(z["gather"], g) and np.array_equal(z["offsets"], offs)
    s = rng.standard_normal(16)
    save_seismogram_txt(tmp_path / "s.txt", t, s)
    lines = (tmp_path / "s.txt").read_text().splitlines()
    assert len(lines) == 16 and lines[1] == f"{t[1]:.8e} {s[1]:.8e}"
