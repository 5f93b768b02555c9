"""The C-ABI library loads without a GPU and exports every entry point include/*.h declares."""
import ctypes
import glob
import os
import re

from conftest import ROOT, load_package


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(rsd_[a-z_0-9]+)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ["rsd_ctx_create", "rsd_spmv", "rsd_solve", "rsd_heat_create", "rsd_assemble_matrix",
                 "rsd_heat_be_step", "rsd_heat_newton", "rsd_csr_autotune"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    rsd = load_package()
    assert os.path.exists(rsd.LIB_PATH), "librsd_cuda.so missing: build() first"
    lib = ctypes.CDLL(rsd.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the same set
    assert set(declared_functions()) <= set(rsd.SIGNATURES)


def test_no_device_fails_loudly():
    # without a GPU the context constructor must raise, never fall back to the CPU
    rsd = load_package()
    try:
        import torch
        if torch.cuda.is_available():
            return
    except Exception:
        pass
    try:
        rsd.Context(0)
    except rsd.RsdError as e:
        assert e.code in (-1, -3)
    else:
        raise AssertionError("context creation succeeded without a CUDA device")


def nested(depth):
    """1 + (1 + (... (1 + 1))): a right-nested sum whose postfix program needs `depth` stack entries."""
    e = "1"
    for _ in range(depth - 1):
        e = f"1 + ({e})"
    return e


def test_expression_stack_depth_is_bounded_at_compile_time():
    # the device evaluates expressions on a 16-entry stack: a deeper program is rejected when it is
    # compiled (RSD_EPARSE), never evaluated to a silent value
    rsd = load_package()
    assert rsd.expr_check(nested(16)) == 16
    try:
        rsd.expr_check(nested(17))
    except rsd.RsdError as e:
        assert e.code == -7 and "stack" in str(e)
    else:
        raise AssertionError("a 17-deep expression was accepted")
    assert rsd.expr_check("1 + 0.5*T") == 3
    assert rsd.expr_check("sin(pi*x)*sin(pi*y) + t^2") >= 2
    try:
        rsd.expr_check("1 + q")
    except rsd.RsdError as e:
        assert e.code == -7
    else:
        raise AssertionError("an unknown symbol was accepted")
