"""Optional device allocations that fail (the split implicit form's list, the
learned guess's buffers, the harvest records) leave the engine usable: the call
returns KC_ERR_OOM, nothing half-allocated is published, and the following
steps still reproduce the CPU oracle bit for bit. The failures are injected on
the host (kc_debug_fail_allocs), so no GPU memory is exhausted."""
import numpy as np
import pytest

from tests.test_gpu_parity import _assert_same_state, _kc, _start

pytestmark = pytest.mark.gpu


def _oom(fn):
    kc = _kc()
    with pytest.raises(kc.KoralError) as e:
        fn()
    assert e.value.status == kc.KC_ERR_OOM


@pytest.mark.parametrize("fail_at", [1, 2, 3])
def test_split_form_oom_leaves_form_and_state(fail_at):
    kc = _kc()
    z, gpu, orc = _start("puffy_fast")
    gpu.debug_fail_allocs(fail_at)  # fail_at - 1 of the three buffers succeed, then one fails
    _oom(lambda: gpu.set_implicit_mode(kc.KC_IMPLICIT_SPLIT))
    gpu.debug_fail_allocs(0)
    gpu.step()
    orc.step()
    _assert_same_state(gpu, orc)
    # selecting the form again allocates it and runs it
    gpu.set_implicit_mode(kc.KC_IMPLICIT_SPLIT)
    gpu.step()
    orc.step()
    _assert_same_state(gpu, orc)
    for k in ["t", "dt", "n_radimp_iters", "n_radimp_solves", "n_radimp_failures"]:
        assert gpu.counters()[k] == orc.counters()[k], k


def test_harvest_oom_keeps_harvest_off_then_grows():
    z, gpu, orc = _start("puffy_fast")
    gpu.debug_fail_allocs(3)  # counters and feature buffer allocated, the target buffer fails
    _oom(lambda: gpu.harvest_implicit(4096))
    gpu.debug_fail_allocs(0)
    gpu.step()
    orc.step()
    _assert_same_state(gpu, orc)
    x, t = gpu.get_harvest(16)
    assert len(x) == 0
    gpu.harvest_implicit(4096)
    gpu.step()
    orc.step()
    _assert_same_state(gpu, orc)
    x, t = gpu.get_harvest(4096)
    assert len(x) > 0 and np.all(np.isfinite(x)) and np.all(np.isfinite(t))
    # growing the harvest keeps the old buffers when a new one fails
    for at in (1, 2):
        gpu.debug_fail_allocs(at)
        _oom(lambda: gpu.harvest_implicit(1 << 16))
        gpu.debug_fail_allocs(0)
        gpu.step()
        orc.step()
        _assert_same_state(gpu, orc)
        x2, t2 = gpu.get_harvest(4096)
        assert len(x2) > 0


@pytest.mark.parametrize("fail_at", [1, 3, 5])
def test_guess_oom_keeps_plain_guess(fail_at):
    kc = _kc()
    from oracle import mlp_ref

    z, gpu, orc = _start("puffy_fast")
    w = mlp_ref.random_blob(3)
    gpu.debug_fail_allocs(fail_at + 1)  # the counter block first, then the five guess buffers
    _oom(lambda: gpu.set_guess(w))
    gpu.debug_fail_allocs(0)
    gpu.step()
    orc.step()
    _assert_same_state(gpu, orc)
