"""C ABI checks that need no GPU: the library loads, exports every entry
point include/samrai_fac_b200.h declares, rejects bad arguments with status
codes, and builds and bounds-checks its device tables for every benchmark
hierarchy in host-only mode (device -1)."""
import ctypes
import os
import re

import numpy as np
import pytest

from samrai_b200 import configs, fac

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "samrai_fac_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(fac_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = fac.load_library()
    names = declared_symbols()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n


def test_bad_arguments_return_status_codes():
    lib = fac.load_library()
    h = ctypes.c_void_p()
    assert lib.fac_ctx_create(ctypes.byref(h), 4, -1) == 1  # FAC_ERR_ARG
    assert b"dim" in lib.fac_last_error()
    assert lib.fac_ctx_create(ctypes.byref(h), 2, -1) == 0
    # operations before fac_initialize are out of order
    assert lib.fac_initialize(h) == 2  # no problems yet: FAC_ERR_STATE
    assert lib.fac_ctx_destroy(h) == 0


def test_host_only_context_refuses_operations():
    ctx = fac.FacContext([configs.config1()], device=-1)
    with pytest.raises(fac.FacError) as ei:
        ctx.smooth(fac.E, fac.R, 0, 1)
    assert ei.value.code == 2
    ctx.close()


@pytest.mark.parametrize("mk", [configs.config1, configs.config3, configs.small_3d,
                                configs.config2])
def test_tables_validate(mk):
    ctx = fac.FacContext([mk()], device=-1)
    p = ctx.problems[0]
    for ln in range(p.nlev):
        assert ctx.size(fac.U, 0, ln) == configs.field_size(p, ln, 1)
        assert ctx.size(fac.F, 0, ln) == configs.field_size(p, ln, 0)
    ctx.close()


def test_batched_tables_validate():
    probs = [configs.small_3d(seed=s) for s in range(3)]
    ctx = fac.FacContext(probs, device=-1)
    for i, p in enumerate(probs):
        assert ctx.size(fac.U, i, 2) == configs.field_size(p, 2, 1)
    ctx.close()


def test_improper_nesting_is_rejected():
    lev0 = configs.Level((1, 1, 1), np.array([[0, 0, 0, 7, 7, 0]], dtype=np.int32))
    # level-2 box outside level 1 (not nested)
    lev1 = configs.Level((2, 2, 1), np.array([[4, 4, 0, 7, 7, 0]], dtype=np.int32))
    lev2 = configs.Level((2, 2, 1), np.array([[20, 20, 0, 23, 23, 0]], dtype=np.int32))
    p = configs.Problem(dim=2, n0=(8, 8, 1), xlo=(0, 0, 0), xup=(1, 1, 1),
                        levels=[lev0, lev1, lev2])
    with pytest.raises(fac.FacError) as ei:
        fac.FacContext([p], device=-1)
    assert ei.value.code == 4
