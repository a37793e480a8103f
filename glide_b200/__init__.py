"""glide_b200 — a B200-native engine for GLIDE's per-timestep particle body.

Submodules: ``runtime`` (fused batch runtime), ``schemes`` (the reference's
plug-in interface: ``hanna_1982_b200``, ``emanuel_reduced_b200``,
``FootprintGridderB200``), ``serving`` (continuous-batching footprint server),
``window`` (met windows, packing, host streaming), ``sparse`` (footprint slices
compacted on the device and streamed to the host, reassembled per release for the
region writer), ``regrid`` (pressure-level -> terrain-following met regrid),
``engine`` (``GPUEngine`` primitives), ``autotune``, ``replicas``, ``synthetic``
(seeded synthetic met), ``met`` (``HourlyMetTensors``). The CUDA
library is ``libglide_b200.so`` next to this file (``python -m glide_b200.build``);
importing a module that needs it raises ``ImportError`` when it is missing.
"""

__version__ = "0.1.0"
