"""Met-window containers: the input format of the particle step.

These mirror the reference's ``MetFieldMetadata`` / ``HourlyMetTensors``
(``src/lpdm/met_reader.py:85-153``) field for field, so a window produced by
the reference's own readers (or by ``glide_b200.synthetic``) can be handed to
the B200 schemes unchanged:

* ``hour_start`` / ``hour_end``: ``[C, Z, Y, X]`` float tensors, channel order
  given by ``channel_names``; 2-D fields (blh, sp, ustar, shf) are broadcast
  over Z (``met_reader.py:502-525``). Broadcast views (stride 0 over Z) are
  accepted.
* ``metadata.level``: AGL height of each level, ``[Z]`` (ascending for the
  terrain-following grid); ``metadata.pressure_level_hpa``: bbox-mean pressure
  per level ``[Z]``; ``metadata.lon`` ``[X]`` / ``metadata.lat`` ``[Y]``: cell
  centres; ``time_start`` / ``time_end``: the bracketing hours.
* ``height_agl_m``: ``[Z, Y, X]`` per-column AGL heights.

The B200 schemes only read attributes, so any object with the same attribute
names (the reference's dataclasses included) works.
"""

from __future__ import annotations

from collections.abc import Mapping
from dataclasses import dataclass, field
from datetime import datetime

import numpy as np
import torch


@dataclass(frozen=True)
class MetFieldMetadata:
    """Grid coordinates and time bracket of a met window (``met_reader.py:85-98``)."""

    lon: np.ndarray
    lat: np.ndarray
    level: np.ndarray
    pressure_level_hpa: np.ndarray
    time_start: datetime
    time_end: datetime
    variable_units: Mapping[str, str] = field(default_factory=dict)


@dataclass(frozen=True)
class HourlyMetTensors:
    """Hour-bracketing met snapshots (``met_reader.py:101-153``)."""

    hour_start: torch.Tensor
    hour_end: torch.Tensor
    metadata: MetFieldMetadata
    channel_names: tuple[str, ...]
    height_agl_m: torch.Tensor | None = None

    def _channel_index(self, name: str) -> int:
        try:
            return self.channel_names.index(name)
        except ValueError as exc:
            available = ", ".join(self.channel_names) or "<none>"
            raise KeyError(
                f"Channel {name!r} not present in met window. Available: {available}"
            ) from exc

    def channel(self, name: str) -> tuple[torch.Tensor, torch.Tensor]:
        """``(hour_start, hour_end)`` slices ``[Z, Y, X]`` of one named channel."""
        idx = self._channel_index(name)
        return self.hour_start[idx], self.hour_end[idx]

    def channels(self, *names: str) -> tuple[torch.Tensor, torch.Tensor]:
        """Stacked ``[len(names), Z, Y, X]`` start/end slices in the order of ``names``."""
        indices = [self._channel_index(name) for name in names]
        return self.hour_start[indices], self.hour_end[indices]


def surface_slice(window: HourlyMetTensors, name: str, level_index: int = 0):
    """``(start, end)`` ``[Y, X]`` slices of a channel at one level (no copy)."""
    s, e = window.channel(name)
    return s[level_index], e[level_index]
