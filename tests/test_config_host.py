"""The run configuration module: importable without the CUDA library, and the
footprint value type checked and mapped to torch dtypes."""

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
