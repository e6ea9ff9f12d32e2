"""The C ABI: the CUDA library loads without a GPU and exports every entry point that include/*.h declares, and the
ctypes binding covers all of them; no compute calls (those need a GPU)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(dfx_\w+)\s*\(", text))
    return names


def test_header_declares_entry_points():
    names = declared()
    assert {"dfx_radon_forward", "dfx_radon_backward", "dfx_spmm_pf_forward", "dfx_spmm_pf_adjoint",
            "dfx_pf_csr_count", "dfx_pf_csr_fill", "dfx_spdhg_dual_update", "dfx_spdhg_primal_update",
            "dfx_poisson_value_grad"} <= names


def test_library_exports_every_declared_symbol():
    from diffractom_b200 import _lib
    from diffractom_b200.build import LIB, build
    if not LIB.exists():
        build()
    h = ctypes.CDLL(str(LIB))
    missing = [n for n in sorted(declared()) if not hasattr(h, n)]
    assert not missing, missing
    assert set(_lib.SIGNATURES) == declared()
    lib = _lib.lib()
    assert lib.dfx_abi_version() == _lib.ABI_VERSION


def test_status_codes_map_to_exceptions():
    from diffractom_b200 import _lib
    lib = _lib.lib()
    # argument checks run on the host before any launch: a null pointer is rejected without touching a GPU
    st = lib.dfx_radon_forward(None, None, None, 1, 4, 4, 4, 8, 8, 1, 1.0, None)
    assert st == _lib.DFX_EINVAL
    with pytest.raises(ValueError, match="null pointer"):
        _lib.check(st)
    assert lib.dfx_scan_scratch_bytes(10) >= 8


def test_lines_fastest_buffer_sizes():
    """The transpose buffers of the lines-fastest PF products, host-side queries: angles x columns x lines rounded up
    to 32; a bad size gives -1. The entry points reject null pointers on the host, before any launch."""
    from diffractom_b200 import _lib
    lib = _lib.lib()
    assert lib.dfx_spmm_pf_forward_zt_floats(18, 263, 1012) == 18 * 1012 * 288
    assert lib.dfx_spmm_pf_forward_zt_floats(1, 32, 5) == 5 * 32
    assert lib.dfx_spmm_pf_adjoint_zt_floats(360, 263, 2880) == 360 * 2880 * 288
    assert lib.dfx_spmm_pf_adjoint_zt_floats(2, 33, 7) == 2 * 7 * 64
    for f in (lib.dfx_spmm_pf_forward_zt_floats, lib.dfx_spmm_pf_adjoint_zt_floats):
        assert f(0, 10, 10) == -1 and f(1, 0, 10) == -1 and f(1, 10, 0) == -1
    st = lib.dfx_spmm_pf_forward_blocked_zt(None, None, 0, None, None, None, None, None, None, 1, 8, 8, 4, 8, 8, 0,
                                            None)
    assert st == _lib.DFX_EINVAL
    st = lib.dfx_spmm_pf_adjoint_zt(None, None, 0, None, None, None, None, None, 1, 8, 8, 8, 8, 1.0, 0, 0, None)
    assert st == _lib.DFX_EINVAL
