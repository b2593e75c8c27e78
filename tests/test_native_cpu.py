"""CPU checks of the C ABI library: it loads, and it exports every entry point
that include/invdft_force.h declares (no GPU calls)."""
import re
from pathlib import Path

from invdft_b200 import native

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    text = (ROOT / "include" / "invdft_force.h").read_text()
    return sorted(set(re.findall(r"\b(invdft_[a-z_0-9]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_functions() == sorted(native.EXPORTED)


def test_library_exports_every_declared_symbol():
    native.load()
    assert sorted(native.exported_symbols()) == declared_functions()


def test_default_params_match_reference_defaults():
    p = native.default_params()
    assert p.cheb_degree == 50 and p.max_cheb_passes == 100
    assert p.adjoint_initial_tol == 1e-11 and p.adjoint_max_iter == 5000
    assert p.adaptive_factor_adjoint == 1000.0 and p.adaptive_factor_cheb == 100.0
    assert p.degeneracy_tol == 0.002 and p.frac_occ_tol == 1e-8 and p.inter_block_size == 10


def test_create_rejects_bad_descriptor_without_gpu_work():
    import ctypes as C
    lib = native.load()
    ctx = C.c_void_p()
    rc = lib.invdft_force_create(None, None, C.byref(ctx))
    assert rc == 5 and not ctx.value
    assert b"null problem" in lib.invdft_last_error(None)
