"""Step-count and delay rules of MGSimulator (mgsim.cpp) in the oracle and
in the library's exported helper (no GPU needed)."""
import numpy as np

import mgb_testlib as T
import mgbrain_b200 as mgb


def test_effective_steps_drops_remainder():
    L = T.oracle()
    # 1 s at 0.1 ms with a 15-step minimum delay runs 9990 steps
    assert L.mgbo_effective_steps(10000, 15) == 9990
    assert L.mgbo_effective_steps(10000, 16) == 10000
    assert L.mgbo_effective_steps(7, 1) == 7
    for steps in (0, 1, 14, 15, 16, 29, 30, 9999):
        for md in (1, 2, 15, 16, 50):
            assert mgb.effective_steps(steps, md) == L.mgbo_effective_steps(steps, md)
    assert mgb.effective_steps(10, 0) == -1


def test_steps_for_time():
    L = T.oracle()
    assert L.mgbo_steps_for_time(np.float32(1.0), np.float32(0.0001)) == 10000
    assert L.mgbo_steps_for_time(np.float32(0.2), np.float32(0.0001)) == 2000


def test_delay_quantisation_rounds_in_fp32():
    d = np.array([0.0016, 0.0015, 0.00014, 0.00015, 0.00016], np.float32)
    q, lo, hi = T.quantize_delays(d, np.float32(0.0001))
    expect = np.round(d / np.float32(0.0001)).astype(np.int32)
    # std::round rounds halves away from zero, np.round to even: compare on
    # values that are not exact halves
    assert q[0] == 16 and q[1] == 15 and q[4] == 2
    assert lo == q.min() and hi == q.max()
    assert np.all(np.abs(q - expect) <= 1)
