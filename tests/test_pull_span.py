"""The bitmap span of the windowed group's pull steps, restated on the CPU:
over random runs that mix pull-step groups of the windowed group with the
other step forms (which write no spike bitmaps) and with checkpoint
restores (whose state holds no bitmaps), every pulled arrival step reads
only bitmaps that a pull-step group wrote for exactly the steps it reads.
The kernel's rule (kernels.cuh, k_window with PULL): a group starting at
step s0 continues the recorded span [from, end) if end == s0, else starts a
new one at s0; an arrival step x may be pulled only if x - max_delay >=
from; the group records [from, its last step + 1).  A restore forgets the
span.  Without the span check (pull whenever x - max_delay >= 0) the same
runs read stale bitmaps, which the last test shows."""
import random

import pytest

MAX_WINDOW = 8


class Device:
    def __init__(self, dmin, dmax, check_span=True):
        self.dmin, self.dmax = dmin, dmax
        self.H = dmax + max(4, min(MAX_WINDOW, dmin))
        self.tag = [None] * self.H   # (timeline, step) whose bitmap each history slot holds
        self.timeline = 0
        self.span = (0, -1)          # bits_span: no step has its bitmap yet
        self.step = 0
        self.check_span = check_span
        self.pulls = 0

    def pull_group(self, n, window):
        s0, s_end = self.step, self.step + n
        bits_from = self.span[0] if self.span[1] == s0 else s0
        if not self.check_span:
            bits_from = 0

        def deliver(x):  # arrivals of step x, from spikes of steps x - d (all before the window)
            if x - self.dmax >= bits_from:
                self.pulls += 1
                for d in range(self.dmin, self.dmax + 1):
                    y = x - d
                    if y < 0:
                        continue
                    if self.tag[y % self.H] != (self.timeline, y):
                        return False
            return True

        ok = True
        w0 = s0
        for x in range(s0 + 1, min(s0 + window, s_end)):  # the first window's later steps
            ok &= deliver(x)
        while w0 < s_end:
            wl = min(window, s_end - w0)
            for s in range(w0, w0 + wl):  # the window's updates write their bitmaps
                self.tag[s % self.H] = (self.timeline, s)
            nxt = w0 + wl
            # the next window's arrivals; after the last window, those of
            # step s_end (the next group's first step)
            for x in range(nxt, min(nxt + window, s_end) if nxt < s_end else s_end + 1):
                ok &= deliver(x)
            w0 = nxt
        self.span = (bits_from, s_end)
        self.step = s_end
        return ok

    def other_form(self, n):
        self.step += n  # its updates write no bitmaps

    def restore(self, back):
        # a checkpoint of an earlier step of this run: the state rewinds, the
        # history slots' bitmaps stay those of the run that went on
        self.step = max(0, self.step - back)
        self.timeline += 1
        self.span = (0, -1)


def random_run(rng, check_span):
    dmin = rng.randint(2, 12)
    dmax = dmin + rng.randint(0, 40)
    dev = Device(dmin, dmax, check_span)
    ok = True
    for _ in range(rng.randint(5, 40)):
        r = rng.random()
        if r < 0.55:
            ok &= dev.pull_group(rng.randint(1, 300), rng.randint(1, min(MAX_WINDOW, dmin)))
        elif r < 0.9:
            dev.other_form(rng.randint(1, 200))
        else:
            dev.restore(rng.randint(0, 400))
    return ok, dev.pulls


@pytest.mark.parametrize("seed", range(100))
def test_pulls_read_only_written_bitmaps(seed):
    ok, _ = random_run(random.Random(seed), check_span=True)
    assert ok


def test_pulls_happen():
    assert sum(random_run(random.Random(s), True)[1] for s in range(100)) > 5_000


def test_without_the_span_stale_bitmaps_are_read():
    assert sum(not random_run(random.Random(s), check_span=False)[0] for s in range(100)) > 25
