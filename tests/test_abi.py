"""CPU checks of the C-ABI library: it loads, exports every entry point that
include/kifmm2d.h declares, and rejects bad arguments before touching CUDA."""
import ctypes
import os
import re

import pytest

from pykifmm2d_b200 import _lib as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "kifmm2d.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(kifmm_[a-z_0-9]+)\s*\(", src)))


def test_header_functions_all_exported():
    lib = B.load()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/kifmm2d.h but not exported"


def test_binding_covers_header():
    assert set(declared_functions()) <= set(B._SIGS)


def test_version_and_defaults():
    lib = B.load()
    assert lib.kifmm_version() >= 100
    o = B.Options()
    o.precision = 7
    lib.kifmm_default_options(ctypes.byref(o))
    assert o.precision == B.PREC_FP64 and o.fix_bbox == 0 and o.radii == 0


@pytest.mark.parametrize("neq,cut,kind,k,msg", [
    (2, 64, 0, 0.0, "Nequiv"),
    (65, 64, 0, 0.0, "Nequiv"),
    (32, 0, 0, 0.0, "Ncutoff"),
    (32, 64, 5, 0.0, "kernel kind"),
    (32, 64, 1, 0.0, "k > 0"),
])
def test_plan_create_rejects_bad_arguments(neq, cut, kind, k, msg):
    lib = B.load()
    h = ctypes.c_void_p()
    kd = B.KernelDesc(kind, 0, k)
    rc = lib.kifmm_plan_create(ctypes.byref(kd), neq, cut, None, ctypes.byref(h))
    assert rc == B.ERR_ARG
    assert msg in lib.kifmm_last_error().decode()
    assert not h.value


def test_null_plan_calls_return_status():
    lib = B.load()
    assert lib.kifmm_precompute(None) == B.ERR_ARG
    assert lib.kifmm_build_expansions(None, None, 0) == B.ERR_ARG
    assert lib.kifmm_plan_destroy(None) == B.OK


def test_python_layer_rejects_foreign_kernels():
    import pykifmm2d_b200 as P
    with pytest.raises(TypeError):
        P.Get_Kernel_Functions(lambda sx, sy, tx, ty: 0.0)
    with pytest.raises(ValueError):
        P.ModifiedHelmholtzKernel(0.0)
