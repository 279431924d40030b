"""Bounded device waits (failure detection without a GPU fault): the wait of
the pipelined kernels, given a short limit on an mbarrier that nothing
arrives on, gives up, records its code in the device error word, and
r2m_check_device_error reports R2M_ETIMEOUT once; the word is then clear and
the context stays usable."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc
from rotormap._lib import R2M_ETIMEOUT, check, lib

from test_gpu_search import int_e4m3, run_engine

pytestmark = pytest.mark.gpu


def test_wait_that_runs_out_is_reported_once():
    torch.zeros(1, device="cuda")
    torch.cuda.synchronize()
    check(lib().r2m_check_device_error(None))
    check(lib().r2m_selftest_bounded_wait(2_000_000, 0, None))  # ~1 ms of SM clocks
    assert lib().r2m_check_device_error(None) == R2M_ETIMEOUT
    assert "code 6" in lib().r2m_last_error().decode()
    assert lib().r2m_check_device_error(None) == 0


def test_completed_phase_is_not_an_error():
    torch.zeros(1, device="cuda")
    check(lib().r2m_selftest_bounded_wait(2_000_000, 1, None))
    assert lib().r2m_check_device_error(None) == 0


def test_context_usable_after_a_timeout():
    torch.zeros(1, device="cuda")
    check(lib().r2m_selftest_bounded_wait(1_000_000, 0, None))
    assert lib().r2m_check_device_error(None) == R2M_ETIMEOUT
    rng = np.random.default_rng(12)
    A8, _ = int_e4m3(rng, (300, 256), -1, 1)
    B8, _ = int_e4m3(rng, (5000, 256), -1, 1)
    v, l = run_engine(A8, B8, 20)
    rv, rl = orc.topk_e4m3(A8, B8, 20, 0)
    assert np.array_equal(v, rv) and np.array_equal(l, rl)


def test_selftest_rejects_bad_limit():
    assert lib().r2m_selftest_bounded_wait(-1, 0, None) != 0
    assert lib().r2m_selftest_bounded_wait(5_000_000_000, 0, None) != 0
