"""CPU-side checks of the C ABI: the library loads, exports every symbol the header
declares, and the host-only entry points (status strings, model validation) behave."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADERS = sorted((ROOT / "include").glob("*.h"))


def declared_functions():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names.update(re.findall(r"\b(kr_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


@pytest.fixture(scope="module")
def so():
    from seismicinversion_b200 import _lib

    if not _lib.LIB_PATH.exists():
        from seismicinversion_b200 import build

        build.build()
    return _lib.lib()


def test_header_symbols_exported(so):
    names = declared_functions()
    assert len(names) >= 8
    for n in names:
        assert hasattr(so, n), f"{n} declared in include/ but not exported"


def test_binding_table_matches_header():
    from seismicinversion_b200 import _lib

    assert sorted(_lib.exported_symbols()) == declared_functions()


def test_status_strings(so):
    assert so.kr_status_string(0) == b"KR_OK"
    assert so.kr_status_string(2) == b"KR_ERR_INVALID_MODEL"
    assert so.kr_status_string(99) == b"KR_ERR_UNKNOWN"
    assert so.kr_version() >= 10000


def _tab(model):
    from seismicinversion_b200.layer_model import pack_layers

    return np.ascontiguousarray(pack_layers(model))


def test_validate_layers_host(so):
    from seismicinversion_b200.earth_models import default_ocean_crust_model, random_layered_model

    for m in (default_ocean_crust_model(), random_layered_model(20, 1)):
        t = _tab(m)
        assert so.kr_validate_layers(t.ctypes.data, t.shape[1]) == 0
    t = _tab(random_layered_model(5, 0))
    bad = t.copy()
    bad[0, 3] = -1.0  # alpha <= 0
    assert so.kr_validate_layers(bad.ctypes.data, bad.shape[1]) == 2
    assert b"alpha" in so.kr_last_error()
    bad = t.copy()
    bad[1, 0] = 0.5  # elastic ocean
    assert so.kr_validate_layers(bad.ctypes.data, bad.shape[1]) == 2
    bad = t.copy()
    bad[4, 2] = np.nan
    assert so.kr_validate_layers(bad.ctypes.data, bad.shape[1]) == 2
    one = t[:, :1].copy()
    assert so.kr_validate_layers(one.ctypes.data, 1) == 2
    assert so.kr_validate_layers(None, 3) == 1


def test_layer_model_errors_match_reference():
    from seismicinversion_b200.layer_model import LayerModel

    with pytest.raises(ValueError, match="All alpha must be positive"):
        LayerModel([1.5, -1], [0, 1], [1, 2], [1, np.inf], [100, 100], [50, 50])
    with pytest.raises(ValueError, match="All beta must be non-negative"):
        LayerModel([1.5, 2], [0, -1], [1, 2], [1, np.inf], [100, 100], [50, 50])
    with pytest.raises(ValueError, match="length mismatch"):
        LayerModel([1.5, 2], [0], [1, 2], [1, np.inf], [100, 100], [50, 50])


def test_no_cpu_fallback_without_gpu():
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from seismicinversion_b200 import kennett_reflectivity
    from seismicinversion_b200.earth_models import default_ocean_crust_model

    with pytest.raises(RuntimeError, match="CUDA"):
        kennett_reflectivity(default_ocean_crust_model(), 0.2, np.array([1.0, 2.0]))


def test_misaligned_complex_pointers_rejected(so):
    """Every complex array must start on a 16-byte boundary; the checks run on the host
    before anything is enqueued (fake addresses are never dereferenced)."""
    i32, u32 = ctypes.c_int32, ctypes.c_uint32
    vp = ctypes.c_void_p
    tab, pp = vp(0x1000), vp(0x2000)
    for fn in (so.kr_reflectivity, so.kr_gmm_reflectivity):
        # omega misaligned by 8 bytes, then R misaligned
        assert fn(tab, i32(3), pp, i32(2), vp(0x3008), i32(4), u32(0), vp(0x4000), None) == 1
        assert fn(tab, i32(3), pp, i32(2), vp(0x3000), i32(4), u32(0), vp(0x4008), None) == 1
    ws = vp(0x8000)
    assert so.kr_bessel_sum(vp(0x3008), pp, pp, i32(2), ctypes.c_double(0.1), vp(0x5000),
                            i32(4), vp(0x6000), i32(2), vp(0x7000), ws, ctypes.c_size_t(1 << 20),
                            None) == 1
