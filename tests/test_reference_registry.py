"""The B200 schemes registered in the reference's own scheme registries
(``register_with_reference``): built by name through the reference's ``get_scheme``
/ ``get_convection_scheme``, listed beside its stock schemes. Runs where the
reference is installed as a package directory (``baseline/_ref``, the reference arm's
install); the end-to-end run of ``lpdm.main._run`` with them needs a GPU and is
``tests/golden/reference_runtime_dropin.py``."""

from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = ROOT / "baseline" / "_ref"


@pytest.mark.skipif(not (REF / "lpdm").is_dir(), reason="the reference is not installed in baseline/_ref")
def test_registered_in_the_reference_registries():
    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    import make_golden

    make_golden._import_reference(REF)
    import lpdm.convection.base as cb
    import lpdm.turbulence.base as tb

    from glide_b200.schemes import EmanuelB200Convection, HannaB200Scheme, register_with_reference

    register_with_reference(tb, cb)
    register_with_reference(tb, cb)  # registering the same classes again is allowed
    assert "hanna_1982_b200" in tb.list_schemes() and "hanna_1982" in tb.list_schemes()
    assert "emanuel_reduced_b200" in cb.list_schemes() and "emanuel_reduced" in cb.list_schemes()
    s = tb.get_scheme("hanna_1982_b200", meander_enabled=True, max_substeps=6)
    c = cb.get_scheme("emanuel_reduced_b200", closure_c=0.03)
    assert isinstance(s, HannaB200Scheme) and isinstance(c, EmanuelB200Convection)
    assert s.meander_enabled and s.max_substeps == 6 and s.step_includes_advection(None)
    assert set(s.required_met_keys()) == {"t", "ustar", "shf"} and set(c.required_met_keys()) == {"t", "q"}
