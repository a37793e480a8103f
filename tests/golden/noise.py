"""Injected-noise streams shared by the golden generator, the oracle tests and
the CUDA parity tests.

``step_noise(seed, step, max_substeps, n)`` → ``(substep [max_substeps, 3, n],
meander [2, n])`` standard normals (float32) for one outer step;
``conv_uniforms(seed, step, n)`` → the two ``[n]`` uniform draws of one
convection event. Each step has its own numpy PCG64 stream, so any step can be
regenerated on its own.
"""

from __future__ import annotations

import numpy as np


def step_noise(seed: int, step: int, max_substeps: int, n: int) -> tuple[np.ndarray, np.ndarray]:
    rng = np.random.default_rng([int(seed), int(step)])
    sub = rng.standard_normal((max_substeps, 3, n), dtype=np.float32)
    mea = rng.standard_normal((2, n), dtype=np.float32)
    return sub, mea


def conv_uniforms(seed: int, step: int, n: int) -> tuple[np.ndarray, np.ndarray]:
    rng = np.random.default_rng([int(seed), 1_000_000 + int(step)])
    return rng.random(n, dtype=np.float32), rng.random(n, dtype=np.float32)


def noise_block(seed: int, steps: range | list, max_substeps: int, n: int) -> tuple[np.ndarray, np.ndarray]:
    """Noise of several consecutive steps stacked: ``[S, max_substeps, 3, n]`` and ``[S, 2, n]``."""
    subs, meas = zip(*(step_noise(seed, s, max_substeps, n) for s in steps))
    return np.stack(subs), np.stack(meas)
