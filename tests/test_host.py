"""Host logic without a GPU: the parameter rows and presets, the workload generators, the C-ABI library's
exports against include/ballasim_b200.h, and the calls that need no device."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from ballasim_b200 import fields as F
from ballasim_b200 import workloads as W
from ballasim_b200.params import SensorParams, preset_names, resolve

HEADER = Path(__file__).resolve().parents[1] / "include" / "ballasim_b200.h"


def test_presets_and_validation():
    assert preset_names() == ["prophesee_gen3", "samsung_gen3", "ideal"]
    p = SensorParams.preset("ideal")
    assert p.photoreceptor == "instantaneous" and p.reset_mode == "ideal" and p.theta_on == 0.2
    assert p.illuminance_scale == 1.0 and p.eps_ci == 0.0 and p.theta_floor == 0.01
    p.validate()
    with pytest.raises(ValueError):
        SensorParams().validate()  # no family, no prior
    with pytest.raises(ValueError):
        SensorParams.preset("nope")
    with pytest.raises(ValueError):
        resolve("ideal", {"theta_on": 0.005})  # below theta_floor
    with pytest.raises(ValueError):
        resolve("ideal", {"eps_ci": 0.01})  # |eps_ci| >= theta_floor / 2
    with pytest.raises(AttributeError):
        resolve("ideal", {"no_such_row": 1})
    with pytest.raises(ValueError):
        setattr(SensorParams.preset("ideal"), "reset_mode", "soft")


def test_fields_are_deterministic_and_float32():
    a, b = F.blobs(346, 260, 2, 16), F.blobs(346, 260, 2, 16)
    assert a.blobs.dtype == np.float32 and np.array_equal(a.blobs, b.blobs)
    assert not np.array_equal(a.blobs, F.blobs(346, 260, 3, 16).blobs)
    e = F.tanh_edge(64, 48, 3)
    assert abs(e.nx * e.nx + e.ny * e.ny - 1) < 1e-6 and 0 <= e.c <= 64


def test_workload_sizes():
    assert W.windows_for(1.0) == 120 and W.windows_for(2.0) == 239 and W.windows_for(0.5) == 60
    assert W.six_sensors().pixels == 4_621_160
    assert W.blobs_346x260().pixels == 89_960


def test_library_exports_every_declared_symbol():
    from ballasim_b200 import _lib
    from ballasim_b200.build import build

    build()
    declared = set(re.findall(r"^\s*(?:bs_status|const char\*|int32_t)\s+(bs_\w+)\(", HEADER.read_text(), re.M))
    assert len(declared) >= 30
    lib = C.CDLL(str(_lib.LIB_PATH))
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert declared == set(_lib.exported_symbols())


def test_calls_without_device_fail_loudly():
    from ballasim_b200 import _lib
    from ballasim_b200.sensor import SensorModel

    if _lib.cuda_available():
        pytest.skip("a B200 is visible")
    with pytest.raises(RuntimeError, match="CUDA device"):
        SensorModel("ideal", 8, 8, 1, [{"type": "constant"}], 0)


def test_level_cap_on_host():
    from ballasim_b200.sampling import level_cap

    assert level_cap([1, 1, 2], 100, 0) is None
    assert level_cap([3, 3, 3, 3], 20, 0) == 2  # 4 x (2^2 + 1) = 20 <= 20 < 4 x 9
    assert level_cap([3, 3, 3, 3], 19, 0) == 1
    with pytest.raises(ValueError):
        level_cap([5, 5], 2, 1)


def test_sensor_model_argument_checks():
    from ballasim_b200.sensor import SensorModel

    with pytest.raises(ValueError):
        SensorModel("ideal", 8, 8, 1, [{"type": "constant"}], 0, device="cpu")
    with pytest.raises(ValueError):
        SensorModel("ideal", 8, 8, 1, [{"type": "fourier", "f0_hz": 100, "a": [0.1], "phi": [0]}], 0)

