"""The C-ABI library loads, exports every entry point include/ppmg.h declares,
and reports argument errors with the reference's info/errno (no GPU needed:
these paths return before any CUDA call)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import ppm_legacy_b200 as ppmg
from ppm_legacy_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "ppmg.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ppmg_[a-z0-9_]+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    L = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 40
    for n in names:
        assert hasattr(L, n), n
    # and the ctypes table covers them all (so the Python mirror can call each)
    assert set(names) <= set(_lib.SIGNATURES)


def test_version_and_precision_switch():
    assert _lib.lib().ppmg_version() >= 10000
    assert ppmg.set_precision(7) == -2
    info, errno, msg = ppmg.last_error()
    assert (info, errno) == (-2, 503) and "mode" in msg
    old = _lib.lib().ppmg_get_precision()
    assert ppmg.set_precision(1) == 0 and _lib.lib().ppmg_get_precision() == 1
    assert ppmg.set_precision(old) == 0


def _p2m_call(Np, topo_id=99, kernel=2, lda=3):
    xp = np.zeros((3, 4), order="F")
    up = np.zeros((3, 4), order="F")
    f = np.zeros((3, 8, 8, 8, 1), order="F")
    return ppmg.ppm_interp_p2m(xp, Np, up, lda, topo_id, 1, kernel, [2, 2, 2], f)


def test_negative_np_is_an_argument_error():
    assert _p2m_call(-1) == -2
    assert ppmg.last_error()[:2] == (-2, 503)


def test_unknown_topology_is_an_argument_error():
    assert _p2m_call(4, topo_id=12345) == -2
    info, errno, msg = ppmg.last_error()
    assert errno == 503 and "invalid" in msg


@pytest.mark.parametrize("kernel", [0, 3, 4])
def test_unsupported_kernel_is_refused(kernel):
    assert _p2m_call(4, kernel=kernel) == -2
    assert ppmg.last_error()[1] == 503


def test_scalar_and_vector_dispatch_by_rank():
    # scalar variant: up of rank 1, no lda argument
    xp = np.zeros((3, 4), order="F")
    f = np.zeros((8, 8, 8, 1), order="F")
    info = ppmg.ppm_interp_p2m(xp, -1, np.zeros(4), 77, 1, 2, [2, 2, 2], f)
    assert info == -2
    with pytest.raises(TypeError):
        ppmg.ppm_interp_p2m(xp, 4, np.zeros(4), 1, 2)


def test_rank_argument_checks():
    xp = np.zeros((3, 2), order="F")
    info, _, _ = ppmg.ppm_util_rank(xp, -3, [0, 0, 0], [1, 1, 1], [2, 2, 2], [1] * 6)
    assert info == -2


def test_library_refuses_missing_build(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(_lib.LibraryMissing):
        _lib.lib()
