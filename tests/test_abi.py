"""The C-ABI library loads and exports every entry point include/feab200.h declares (no GPU)."""
import ctypes
import os
import re

from conftest import ROOT


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "feab200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(feab_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_entry_points():
    syms = declared_symbols()
    for must in ("feab_hex8_element_stiffness", "feab_csr_pattern", "feab_assemble_csr", "feab_pcg_solve",
                 "feab_hex8_simp_vjp"):
        assert must in syms


def test_library_exports_every_declared_symbol():
    from feab200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    # the ctypes signature table covers the header too
    assert sorted(_lib.SIGNATURES) == declared_symbols()


def test_status_strings_and_version():
    from feab200 import _lib
    assert _lib.lib.feab_abi_version() >= 1
    assert "SPD" in _lib.status_string(_lib.FEAB_NOT_SPD)
    assert _lib.status_string(99) == "unknown status"


def test_workspace_queries_do_not_need_a_gpu():
    from feab200 import _lib
    assert _lib.lib.feab_pcg_workspace_bytes(1000, _lib.PREC_FP64) >= 3 * 8 * 1000
    assert _lib.lib.feab_pcg_workspace_bytes(1000, _lib.PREC_MIXED) >= 3 * 8 * 1000 + 4 * 4 * 1000
    assert _lib.lib.feab_pcg_workspace_bytes(10, 7) == 0
    assert _lib.lib.feab_topology_scratch_bytes(100, 50) > 0
    # banded Cholesky: 256-byte header + n_tiles * (bands + 1) band tiles + n_tiles inverse
    # diagonal tiles, each 64 x 64 doubles
    assert _lib.lib.feab_band_bytes(100, 130) == 256 + 2 * 5 * 64 * 64 * 8
    assert _lib.lib.feab_band_bytes(64, 0) == 256 + 2 * 64 * 64 * 8
    assert _lib.lib.feab_band_bytes(0, 10) == 0


def test_product_never_imports_the_oracle():
    pkg = os.path.join(ROOT, "computation-suite_b200", "feab200")
    for fn in os.listdir(pkg):
        if fn.endswith(".py"):
            src = open(os.path.join(pkg, fn)).read()
            assert "oracle" not in re.findall(r"^\s*(?:from|import)\s+(\w+)", src, flags=re.M), fn
