"""CPU: the C-ABI library loads and exports every entry point that
include/*.h declares (no compute call: there is no GPU here)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from asd2_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\*?\s*(asd2g_[a-z0-9_]+)\s*\(", src, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "asd2g_create" in names and "asd2g_droplet_step" in names
    assert len(names) >= 30


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(api.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header():
    assert set(declared_symbols()) <= set(api.EXPORTS)


def test_version():
    assert api.load().asd2g_version() == 1


def test_missing_library_fails_loudly(tmp_path):
    api_mod = api
    with pytest.raises(ImportError):
        api_mod._lib_saved = api_mod._lib
        try:
            api_mod._lib = None
            api_mod.load(str(tmp_path / "nope.so"))
        finally:
            api_mod._lib = api_mod._lib_saved


def test_params_struct_matches_header():
    # asd2g_params: 4 int32, 4 double, 12 int32, 12 double, 6 double, 4 int32, 2 double, 2 int32, 3 double
    assert ctypes.sizeof(api._Params) == 4 * 4 + 4 * 8 + 12 * 4 + 12 * 8 + 6 * 8 + 4 * 4 + 2 * 8 + 2 * 4 + 3 * 8


def test_mixed_precision_needs_producer_side_pressure_fill():
    """The FP32 level-set kernels write their own ghost mirrors, so a mixed
    session with periodic pressure sides is refused when it is created
    (before any device work)."""
    p = api.Params(32, 32, 1 / 32, 1 / 32, bc_p=("periodic",) * 4, precision=api.PRECISION_MIXED)
    with pytest.raises(api.Asd2gError) as e:
        api.Session(p)
    assert e.value.code == -4
    p = api.Params(32, 32, 1 / 32, 1 / 32, precision=7)
    with pytest.raises(api.Asd2gError) as e:
        api.Session(p)
    assert e.value.code == -1


def test_batch_refuses_periodic_pressure_before_device_work():
    ok = api.Params(32, 32, 1 / 32, 1 / 32)
    bad = api.Params(40, 24, 1 / 40, 1 / 40, bc_p=("periodic",) * 4)
    with pytest.raises(api.Asd2gError) as e:
        api.Batch([ok, bad])
    assert e.value.code == -4


def test_axisymmetric_entry_points_check_arguments_first():
    """The asd2g_axi_* functions refuse a null session or a bad component
    with ASD2G_E_ARG before any device work."""
    L = api.load()
    d = ctypes.c_double(1e-3)
    assert L.asd2g_axi_kappa(None) == -1
    assert L.asd2g_axi_rhs_u(None, 1e-3, 0, 1, 2, 7, 13) == -1
    assert L.asd2g_axi_rhs_v(None, 1e-3, 0, 1, 9, 2, 7, 13) == -1
    assert L.asd2g_axi_viscosity(None, 0, 1, 9, 2, 7, 13, 14) == -1
    assert L.asd2g_axi_hat(None, 2, 1e-3, 0, 13, 7, 9) == -1
    assert L.asd2g_axi_divergence(None, 9, 10, 8, 1) == -1
    assert L.asd2g_axi_assemble(None, 1e-3, 1) == -1
    assert L.asd2g_axi_update_dt(None, ctypes.byref(d)) == -1
    it, res = ctypes.c_int(), ctypes.c_double()
    assert L.asd2g_axi_step(None, ctypes.byref(d), 2, None, None, 0, 1e-10, 100, ctypes.byref(it),
                            ctypes.byref(res)) == -1
    assert b"null" in L.asd2g_last_error()


# Entry points for which null / zero arguments are a valid call: destroying
# nothing succeeds (like free(NULL)), sizes of nothing are 0.
NULL_OK = {"asd2g_version": 1, "asd2g_destroy": 0, "asd2g_batch_destroy": 0, "asd2g_unet_destroy": 0,
           "asd2g_conv_wpack_bytes": 0, "asd2g_unet_nparams": 0}


def _zero_args(fn):
    args = []
    for t in fn.argtypes or []:
        if hasattr(t, "_dtype_"):  # an ndpointer: a one-element array
            args.append(np.zeros(1, dtype=t._dtype_))
        elif t in (ctypes.c_int, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint, ctypes.c_longlong, ctypes.c_size_t,
                   ctypes.c_ulonglong):
            args.append(0)
        elif t in (ctypes.c_double, ctypes.c_float):
            args.append(0.0)
        elif t is ctypes.c_char:
            args.append(b"P")
        else:
            args.append(None)
    return args


def test_every_entry_point_refuses_null_arguments():
    """Every exported function called with null pointers, zero sizes and zero
    scalars returns an error status (or the documented value for a null
    destroy / an empty size); none dereferences a null pointer or launches
    device work."""
    L = api.load()
    for name in api.EXPORTS:
        fn = getattr(L, name)
        if name == "asd2g_last_error":
            assert isinstance(fn(), bytes)
            continue
        r = fn(*_zero_args(fn))
        if name in NULL_OK:
            assert r == NULL_OK[name], (name, r)
        else:
            assert r < 0, (name, r)
