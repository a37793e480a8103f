"""Host-side configuration: the run configuration module importable without the CUDA
library, the footprint value type checked and mapped to torch dtypes, and the runtime's
default launch shape chosen from the SM count."""

from __future__ import annotations

import subprocess
import sys

import pytest
import torch

from glide_b200.config import FootprintSpec


def test_footprint_value_dtype():
    f = FootprintSpec((0.0, 1.0), (0.0, 1.0), 4, 4, (0.0, 100.0), 2, 1)
    assert f.value_dtype == "f32" and f.torch_dtype == torch.float32
    g = FootprintSpec((0.0, 1.0), (0.0, 1.0), 4, 4, (0.0, 100.0), 2, 1, ring=2, value_dtype="f64")
    assert g.torch_dtype == torch.float64 and g.device_shape == (1, 2, 1, 4, 4)
    with pytest.raises(ValueError):
        FootprintSpec((0.0, 1.0), (0.0, 1.0), 4, 4, (0.0, 100.0), 2, 1, value_dtype="f16")


def test_config_loads_no_cuda_library():
    """The CPU baselines build their configuration from this module alone."""
    code = ("import sys; import glide_b200.config, glide_b200.synthetic; "
            "print(any(m.endswith('_abi') for m in sys.modules))")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True)
    assert out.stdout.strip() == "False"


def test_runtime_reexports_the_config_types():
    from glide_b200 import config, runtime

    assert runtime.FootprintSpec is config.FootprintSpec and runtime.HannaConfig is config.HannaConfig


def test_default_launch_shape_follows_the_sm_count(monkeypatch):
    """The runtime's default step-kernel shape (host logic over the library's shape
    table, no kernel launched): one 768-thread block per SM from a batch of
    SMs x 768 particles up, 128-thread blocks below, for any SM count."""
    from types import SimpleNamespace

    from glide_b200 import runtime
    from glide_b200.autotune import launch_variants

    shapes = {v: (t, b) for v, t, b in launch_variants()}
    for sms in (148, 132, 20):
        monkeypatch.setattr(torch.cuda, "get_device_properties",
                            lambda dev, sms=sms: SimpleNamespace(multi_processor_count=sms))
        assert shapes[runtime.default_launch_variant(sms * 768, "cuda:0")] == (768, 1)
        assert shapes[runtime.default_launch_variant(sms * 768 - 1, "cuda:0")] == (128, 6)
        assert shapes[runtime.default_launch_variant(0, "cuda:0")] == (128, 6)
