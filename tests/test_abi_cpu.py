"""The C-ABI library loads and exports every declared symbol (no GPU)."""
import ctypes

from mgcm_rt import abi


def test_library_exports_every_declared_symbol():
    L = abi.lib()
    names = abi.exported_symbols()
    assert "mgcm_rt_run" in names and "mgcm_rt_create" in names
    for n in names:
        assert hasattr(L, n), n


def test_strerror_and_version():
    L = abi.lib()
    assert L.mgcm_rt_strerror(0) == b"ok"
    assert b"Planck" in L.mgcm_rt_strerror(-3)
    assert b"unknown" in L.mgcm_rt_strerror(-999)
    assert b"Mars" in L.mgcm_rt_version()


def test_tables_host_bad_dir():
    import numpy as np
    D = ctypes.POINTER(ctypes.c_double)
    z = np.zeros(51)
    assert abi.lib().mgcm_rt_tables_host(b"/nonexistent-dir", None, None, None,
                                         z.ctypes.data_as(D)) == -6
