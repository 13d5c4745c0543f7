"""kc_implicit_batch_noalloc, the allocation-free variant of kc_implicit_batch
(its arrays are staged through the library's fixed device array), against the
allocating entry point through the C ABI: bit for bit, as every engine-vs-oracle
comparison here, on two different calls in a row, and at the size limit."""
import numpy as np
import pytest

from tests.engine import koralcuda
from tests.kgold import load_kgld

pytestmark = pytest.mark.gpu


def _records():
    i, _ = load_kgld("rad/rad_implicit")
    return i[:, :23].copy(), i[:, 23].copy(), i[:, 24:37].copy()


def _same(kc, opt, geom, dt, pp):
    ref_pp, ref_res = kc.implicit_batch(opt, geom, dt, pp)
    got_pp, got_res = kc.implicit_batch_noalloc(opt, geom, dt, pp)
    assert np.array_equal(got_res, ref_res)
    assert np.array_equal(got_pp.view(np.uint64), ref_pp.view(np.uint64))
    return got_res


def test_noalloc_matches_allocating_batch_on_two_calls_in_a_row():
    kc = koralcuda()
    kc.lib()
    opt = kc.puffy_options()
    geom, dt, pp = _records()
    res1 = _same(kc, opt, geom, dt, pp)
    assert res1[:, 0].sum() > 0.8 * len(res1)  # most golden records converge (297 of 336)
    # second call: fewer cells, another order; the array still holds the first call's data
    idx = np.arange(len(dt))[::-1][:200]
    _same(kc, opt, geom[idx], dt[idx], pp[idx])


def test_noalloc_at_the_size_limit_and_beyond():
    kc = koralcuda()
    lib = kc.lib()
    opt = kc.puffy_options()
    geom, dt, pp = _records()
    n = kc.KC_NOALLOC_MAX_CELLS
    rep = np.resize(np.arange(len(dt)), n)
    _same(kc, opt, geom[rep], dt[rep], pp[rep])
    import ctypes

    st = lib.kc_implicit_batch_noalloc(ctypes.byref(opt), n + 1, None, None, None, None, 0)
    assert st == kc.KC_ERR_TOO_MANY_CELLS


def test_noalloc_accepts_only_the_per_cell_form():
    import ctypes

    kc = koralcuda()
    lib = kc.lib()
    opt = kc.puffy_options()
    geom, dt, pp = _records()
    res = np.zeros((len(dt), 6), dtype=np.int32)
    pw = pp.copy()
    for mode in (kc.KC_IMPLICIT_COMPACTING, kc.KC_IMPLICIT_SORTED):
        st = lib.kc_implicit_batch_noalloc(ctypes.byref(opt), len(dt), geom.ctypes.data, dt.ctypes.data,
                                           pw.ctypes.data, res.ctypes.data, mode)
        assert st == kc.KC_ERR_INVALID_CONFIG
