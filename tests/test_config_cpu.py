"""The linear_system/* scene settings of the host mirror (no GPU needed)."""
import pytest

from libuipc_b200 import _abi
from libuipc_b200.linear_system import B200PCG, SCENE_CONFIG_DEFAULTS, linear_system_config


def test_defaults_are_the_reference_defaults():
    c = linear_system_config()
    assert c["linear_system/tol_rate"] == 1e-3
    assert c["linear_system/solver"] == "fused_pcg"
    assert c["linear_system/fem_preconditioner"] == "diag"
    assert c["linear_system/use_cuda_graph"] == 1
    assert c["linear_system/check_interval"] == 5
    assert set(c) == set(SCENE_CONFIG_DEFAULTS)


@pytest.mark.parametrize("key,value", [
    ("linear_system/tol_rate", 0.0), ("linear_system/tol_rate", 1.0), ("linear_system/solver", "cg"),
    ("linear_system/fem_preconditioner", "amg"), ("linear_system/use_cuda_graph", 3),
    ("linear_system/check_interval", 0), ("linear_system/b200/warm_start", "random"),
    ("linear_system/unknown", 1)])
def test_invalid_settings_are_rejected(key, value):
    with pytest.raises(ValueError):
        linear_system_config({key: value})


def test_from_config_maps_the_settings():
    p = B200PCG.from_config({"linear_system/tol_rate": 1e-4, "linear_system/solver": "linear_pcg",
                             "linear_system/use_cuda_graph": 0, "linear_system/b200/precision": "mixed",
                             "linear_system/b200/warm_start": "learned"})
    assert p.kw["tol"] == 1e-4 and p.kw["check_interval"] == 1 and p.kw["use_graph"] is False
    assert p.kw["stop_rule"] == _abi.B2S_STOP_RZ and p.kw["precision"] == _abi.B2S_PRECISION_MIXED
    assert p.warm_start == "learned"
    q = B200PCG.from_config({"other/key": 3})
    assert q.kw["check_interval"] == 5 and q.kw["use_graph"] is True and q.warm_start == "zero"
