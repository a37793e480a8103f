"""CPU oracle for the GLIDE per-timestep particle body — TEST INFRASTRUCTURE ONLY.

A numpy restatement of the reference's algorithm for the hot path (mrghg/glide,
``src/lpdm``), each function citing the reference file:line it follows. It is
the checker for the CUDA path and the CPU baseline of ``bench.py``; nothing in
the shipped package (``glide_b200``) imports it.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference legs may import it.

Parity is pinned: ``tests/golden/make_golden.py`` runs the reference itself
(imported read-only, eager static path, injected noise) and stores its outputs
under ``tests/golden/``; ``tests/test_oracle_golden.py`` checks this oracle
against them.

``dtype`` selects the arithmetic: ``np.float32`` mirrors the reference (float32
torch on CPU, same operation order, FMA where torch's CPU kernels use it);
``np.float64`` is the FP64 oracle used to score reduced-precision met storage.
"""

from oracle.hanna import HannaParams, StepNoise, step_core  # noqa: F401
from oracle.runtime import run_batch  # noqa: F401
