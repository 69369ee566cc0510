"""C ABI checks that need no GPU: the library builds, loads, exports every
symbol declared in include/tm_b200.h, and rejects bad arguments before
touching the device."""
import os
import re

import numpy as np
import pytest

from cistem_downstream_bah_b200 import core

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "tm_b200.h")).read()
    return sorted(set(re.findall(r"^TM_API\s+(?:const\s+)?(?:int|long long|char)\s*\*?\s*(tm_\w+)\s*\(", text, re.M)))


def test_header_declares_the_bound_symbols():
    assert sorted(core.EXPORTED) == declared_symbols()


def test_library_loads_and_exports_all_symbols():
    L = core.load()
    for name in declared_symbols():
        assert hasattr(L, name), name
    assert b"sm_100a" in L.tm_version()


def test_unsupported_geometry_rejected_without_gpu():
    # 302 = 2 x 151: no compiled kernels and no radix plan (a prime factor above 13);
    # a box of 50 has no slice kernels
    for x, y, t in ((302, 302, 48), (512, 512, 50), (16384, 512, 64)):
        with pytest.raises(core.TmError) as e:
            core.SearchCore(x, y, t, histogram_min_scaled=-0.1, histogram_step_scaled=0.001)
        assert e.value.code == core.TM_ERR_UNSUPPORTED


def test_bad_histogram_rejected_without_gpu():
    with pytest.raises(core.TmError) as e:
        core.SearchCore(256, 256, 32, histogram_min_scaled=-0.1, histogram_step_scaled=0.0)
    assert e.value.code == core.TM_ERR_INVALID


def test_null_arguments_rejected():
    L = core.load()
    assert L.tm_create(None, None) == core.TM_ERR_INVALID
    assert L.tm_destroy(None) == core.TM_ERR_INVALID
    assert L.tm_last_error(None) == b"null context"


def test_orientation_order_matches_oracle():
    from oracle import oracle as O
    grid = O.search_grid(15.0)
    ours = core.orientation_list(grid, 0.0, 15.0, 360.0)
    ref = O.orientation_list(grid, O.psi_list(0.0, 15.0, 360.0))
    assert np.array_equal(ours, ref)
    for step in (1.5, 2.0, 5.0, 7.3):
        assert len(core.orientation_list(grid[:1], 0.0, step, 360.0)) == len(O.psi_list(0.0, step, 360.0))
