"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares; host-side argument parsing matches the reference
binding's behaviour (no GPU call is made here)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from dream_b200 import _lib, beamformer, das, das_f

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b(dream_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("dream_das_plan_create", "dream_das_run", "dream_das_run_device", "dream_das_uni_run",
              "dream_das_plan_destroy"):
        assert n in names


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports_declared_symbol(name):
    L = ctypes.CDLL(_lib.LIB_PATH)
    assert hasattr(L, name), f"{name} declared in include/ but not exported"


def test_python_signatures_cover_header():
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_version_and_last_error_without_gpu():
    L = _lib.load()
    assert b"sm_100a" in L.dream_das_version()
    assert isinstance(L.dream_das_last_error(), bytes)


def test_plan_create_rejects_bad_arguments_before_device():
    h = ctypes.c_void_p()
    L = _lib.load()
    assert L.dream_das_plan_create(ctypes.byref(h), 7, 10, 10, 1, 1, 0, 0) == _lib.ERR_ARGUMENT
    assert L.dream_das_plan_create(ctypes.byref(h), 1, -1, 10, 1, 1, 0, 0) == _lib.ERR_ARGUMENT
    assert L.dream_das_plan_create(ctypes.byref(h), 1, 10, 10, 1, 1, 9, 0) == _lib.ERR_ARGUMENT
    assert L.dream_das_plan_create(None, 1, 10, 10, 1, 1, 0, 0) == _lib.ERR_ARGUMENT
    L.dream_das_plan_create(ctypes.byref(h), 7, 1, 1, 1, 1, 0, 0)
    assert b"method" in L.dream_das_last_error()


def _args():
    Y = np.zeros((100, 4))
    G = np.zeros((2, 3))
    Ro = np.zeros((5, 3))
    return Y, G, G, Ro


@pytest.mark.parametrize("mod", [das, das_f])
def test_reference_argument_errors(mod):
    Y, Gt, Gr, Ro = _args()
    with pytest.raises(RuntimeError, match="Argument 2"):
        mod.das(Y, np.zeros((2, 2)), Gr, Ro, 0.04, 0.0, 1500.0, "tfm", "ignore", "cuda")
    with pytest.raises(RuntimeError, match="Argument 3"):
        mod.das(Y, Gt, np.zeros((2, 4)), Ro, 0.04, 0.0, 1500.0, "tfm", "ignore", "cuda")
    with pytest.raises(RuntimeError, match="Obs point"):
        mod.das(Y, Gt, Gr, np.zeros((5, 2)), 0.04, 0.0, 1500.0, "tfm", "ignore", "cuda")
    with pytest.raises(RuntimeError, match="Error in das"):
        mod.das(Y, Gt, Gr, Ro, 0.04, np.zeros(3), 1500.0, "tfm", "ignore", "cuda")
    with pytest.raises(RuntimeError, match="Error in das"):
        mod.das(Y, Gt, Gr, Ro, 0.04, 0.0, 1500.0, "bogus", "ignore", "cuda")
    with pytest.raises(RuntimeError, match="Error in das"):
        mod.das(Y, Gt, Gr, Ro, 0.04, 0.0, 1500.0, "tfm", "loud", "cuda")
    with pytest.raises(RuntimeError, match="device"):
        mod.das(Y, Gt, Gr, Ro, 0.04, 0.0, 1500.0, "tfm", "ignore", "tpu")
    with pytest.raises(RuntimeError, match="cpu"):
        mod.das(Y, Gt, Gr, Ro, 0.04, 0.0, 1500.0, "tfm", "ignore", "cpu")
    with pytest.raises(RuntimeError, match="A-scans"):
        mod.das(np.zeros((100, 3)), Gt, Gr, Ro, 0.04, 0.0, 1500.0, "tfm", "ignore", "cuda")


def test_method_aliases_and_saft_ignores_gr():
    assert beamformer.parse_method("rca") == beamformer.parse_method("rca_coltx")
    K, No, Nt, Nr, multi = beamformer._check_shapes(np.zeros((10, 2)), np.zeros((2, 3)), None,
                                                    np.zeros((4, 3)), np.zeros((4, 1)), _lib.SAFT)
    assert (K, No, Nt, Nr, multi) == (10, 4, 2, 0, True)
    assert beamformer.parse_device("cuda:3") == 3 and beamformer.parse_device("gpu") == 0


def test_plan_cache_reuses_plans_per_key():
    """Bindings keep one plan per kind and thread while calls bring the same
    setup (das_setup_has_changed, include/das.h:77-94): a plan is created once
    per key, not on every call, and replaced when the setup changes."""
    import threading

    from dream_b200 import beamformer

    class FakePlan:
        created = 0

        def __init__(self):
            FakePlan.created += 1

    def run():
        beamformer._tls.__dict__.pop("plans", None)
        k1 = ("fast", 1, 3000, 262144, 64, 64, 2, 0)
        k2 = ("fast", 1, 3000, 262144, 64, 64, 3, 0)
        a = beamformer._plan(k1, FakePlan)
        assert beamformer._plan(k1, FakePlan) is a and FakePlan.created == 1
        b = beamformer._plan(k2, FakePlan)
        assert b is not a and FakePlan.created == 2
        assert beamformer._plan(k2, FakePlan) is b and FakePlan.created == 2
        c = beamformer._plan(("das",) + k1[1:], FakePlan)  # another kind keeps its own slot
        assert beamformer._plan(k2, FakePlan) is b and c is not b and FakePlan.created == 3

    errors = []

    def guarded():
        try:
            run()
        except Exception as e:  # surfaced below: assertions in a thread do not fail the test
            errors.append(e)

    t = threading.Thread(target=guarded)  # a fresh thread-local cache
    t.start()
    t.join()
    if errors:
        raise errors[0]
    assert FakePlan.created == 3
