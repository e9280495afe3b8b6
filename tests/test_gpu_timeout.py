"""The bounded-wait failure path of the 2D stream kernel, exercised without a
fault: a context whose wait limit is 0 polls makes the first wait of every
CTA on its staged copies give up at once.  Each such CTA records the time-out,
waits (with the default bound) until the copies it issued have landed, and
exits; the batch then reports FSM_ERR_TIMEOUT, and the same context computes
correct results again once the limit is back to its default."""
import numpy as np
import pytest

import fsm_b200 as F
import workloads as W

pytestmark = pytest.mark.gpu

DEFAULT_POLLS = 1 << 20


def test_zero_poll_wait_reports_timeout_and_context_recovers():
    c = F.Context(0)
    try:
        p, e, _ = W.lumpy2d(seed=9, side=101, dx=0.08, nphip=64, dtau=0.7, eos=1, radius=3.0)
        want = c.run_event(p, e)
        c.set_wait_limit(0)
        b = F.Batch(c, [p])
        with pytest.raises(F.FsmError) as ei:
            b.run_host([(e, None)])
        assert ei.value.status == 10  # FSM_ERR_TIMEOUT
        b.close()
        # the one-event path of the same context also times out, without a fault
        with pytest.raises(F.FsmError) as ei:
            c.run_event(p, e)
        assert ei.value.status == 10
        c.set_wait_limit(DEFAULT_POLLS)
        b = F.Batch(c, [p])
        got = b.run_host([(e, None)])[0]
        b.close()
        for k in ("T", "e", "u", "pi"):
            np.testing.assert_array_equal(got[k], want[k], err_msg=k)
        again = c.run_event(p, e)
        for k in ("T", "e", "u", "pi"):
            np.testing.assert_array_equal(again[k], want[k], err_msg=k)
    finally:
        c.close()


def test_wait_limit_rejects_negative_polls():
    c = F.Context(0)
    try:
        with pytest.raises(F.FsmError) as ei:
            c.set_wait_limit(-1)
        assert ei.value.status == 1  # FSM_ERR_INVALID_ARG
    finally:
        c.close()
