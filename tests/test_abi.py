"""CPU checks of the C ABI: the library loads and exports every entry point
that include/qv.h declares.  No device call is made."""
import ctypes
import re
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    text = (ROOT / "include" / "qv.h").read_text()
    return sorted(set(re.findall(r"\b(qv_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = _declared()
    for must in ("qv_create", "qv_set_points", "qv_build_tree", "qv_velocity", "qv_step_ab",
                 "qv_step_rk3", "qv_closest", "qv_enforce_periodic", "qv_ghosts", "qv_step"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from qvort_b200 import build

    so = build.build()
    lib = ctypes.CDLL(str(so))
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from qvort_b200 import lib as L

    assert set(_declared()) <= set(L.EXPORTED)


def test_default_params_are_run_in_defaults():
    from qvort_b200 import lib as L

    p = L.default_params()
    assert p.quant_circ == 9.97e-4 and p.corea == 8.244023e-9
    assert p.deriv_order == 2 and p.tree_extra_correction == 1 and p.recon_shots == 1


def test_fortran_shim_binds_declared_entry_points():
    """Every bind(C, name=...) of the Fortran interface module names an entry
    point that include/qv.h declares (and the library exports, above)."""
    text = (ROOT / "shim" / "qv_iface.f90").read_text()
    bound = set(re.findall(r"bind\(C,\s*name='(qv_[a-z0-9_]+)'\)", text))
    assert "qv_step_exchange" in bound and "qv_step" in bound
    missing = sorted(bound - set(_declared()))
    assert not missing, missing
