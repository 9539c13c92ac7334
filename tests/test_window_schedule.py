"""The phase schedule of the windowed step group (k_window), restated on the
CPU and checked for the orderings the kernel relies on, over random minimum
and maximum delays, windows and group lengths, mixed with single-step
launches (k_fused) between groups:

- every arrival step is delivered exactly once, in a phase after every phase
  that updated one of its source steps (sa - d, min delay <= d <= max delay)
  and before the phase that updates it;
- an accumulator buffer (step & 3, or step & 7 while windows of more than 4
  steps run) is written only after the step that used it before was updated
  (its input consumed and cleared), and between groups only the buffer of the
  current step holds input, so switching the cycle moves that one buffer;
- a history slot (step % H, H = max delay + max(4, min(8, min delay))) is
  cleared in a phase that reads
  no step sharing that slot, after every read of its old step, and before its
  new step's update writes it; the raster copy of a step reads its slot after
  the update and before the slot is cleared again.

Phases are what the grid barriers separate: work in one phase may run in any
order across blocks, so a read and a write of the same data in one phase
would race."""
import random

import pytest

ACC_BUFFERS = 4
ACC_BUFFERS_WIDE = 8
MAX_WINDOW = 8


class Schedule:
    def __init__(self, dmin, dmax):
        self.dmin, self.dmax = dmin, dmax
        self.H = dmax + max(4, min(MAX_WINDOW, dmin))
        self.mask = ACC_BUFFERS - 1
        self.buf = {}          # buffer -> [step it holds, phase of the update that consumed it]
        self.phase = 0
        self.updated = {}      # step -> phase of its update
        self.delivered = {}    # step -> phase of its delivery
        self.cleared = {}      # slot -> list of (phase, new step)
        self.reads = []        # (phase, step) history reads
        self.step = 0
        # start state: arrivals of step 0 delivered (nothing to deliver), slot 0 clear
        self.delivered[0] = -1
        self.buf[0] = [0, None]
        self.cleared.setdefault(0, []).append((-1, 0))

    # ---- actions inside a phase ------------------------------------------
    def deliver(self, sa):
        assert sa not in self.delivered, f"step {sa} delivered twice"
        for d in range(self.dmin, self.dmax + 1):
            x = sa - d
            if x >= 0:
                assert self.updated.get(x, 1 << 30) < self.phase, f"step {sa} reads unfinished step {x}"
                self.reads.append((self.phase, x))
        held = self.buf.get(sa & self.mask)  # the buffer's previous step: input consumed before the write
        if held is not None:
            assert held[1] is not None and held[1] < self.phase, f"buffer of {sa} still holds {held[0]}"
        self.buf[sa & self.mask] = [sa, None]
        self.delivered[sa] = self.phase

    def update(self, x):
        assert self.delivered.get(x, 1 << 30) < self.phase, f"step {x} updated before its arrivals"
        assert x not in self.updated
        slot_clears = [p for p, y in self.cleared.get(x % self.H, []) if y == x]
        assert slot_clears and slot_clears[-1] < self.phase, f"slot of step {x} not cleared before its update"
        held = self.buf.get(x & self.mask)
        assert held is not None and held[0] == x and held[1] is None, f"step {x} reads another step's buffer"
        held[1] = self.phase
        self.updated[x] = self.phase

    def clear(self, y):
        self.cleared.setdefault(y % self.H, []).append((self.phase, y))

    def raster(self, x):
        assert self.updated[x] < self.phase
        self.reads.append((self.phase, x))

    def barrier(self):
        self.phase += 1

    # ---- the kernels ------------------------------------------------------
    def set_cycle(self, mask):
        """The host's switch between runs (k_acc_move): only the current
        step's buffer holds input; it moves to its place in the new cycle and
        its old buffer is left zero."""
        for x, used in self.buf.values():
            assert x == self.step or used is not None, f"buffer of step {x} in use at a switch"
        old, cur = self.step & self.mask, self.buf.get(self.step & self.mask)
        if cur is not None and cur[0] == self.step and (self.step & mask) != old:
            self.buf[old] = [None, -1]
            self.buf[self.step & mask] = cur
        self.mask = mask
        self.barrier()

    def fused_step(self):
        """k_fused: update step s, deliver step s+1, the epilogue clears slot s+1."""
        s = self.step
        self.update(s)      # (its raster ids are written by the update itself)
        self.deliver(s + 1)
        self.barrier()
        self.clear(s + 1)   # last block, after every block finished
        self.barrier()
        self.step = s + 1

    def window_group(self, nsteps, W):
        assert W <= self.mask + 1, "a window's steps need distinct buffers"
        s0, s_end = self.step, self.step + nsteps
        n = nsteps - 1 if nsteps < W else W - 1
        for k in range(1, n + 1):
            self.clear(s0 + k)
        for k in range(1, n + 1):
            self.deliver(s0 + k)
        self.barrier()
        w0 = s0
        while w0 < s_end:
            wl = min(W, s_end - w0)
            for k in range(wl):
                self.update(w0 + k)
            self.barrier()
            for k in range(wl):
                self.raster(w0 + k)
            nxt = w0 + wl
            nn = min(W, s_end - nxt) if nxt < s_end else 1
            for k in range(nn):
                self.clear(nxt + k)
            for k in range(nn):
                self.deliver(nxt + k)
            self.barrier()
            w0 = nxt
        self.step = s_end

    # ---- the history slots ------------------------------------------------
    def check_slots(self):
        H = self.H
        by_slot = {}
        for rp, z in self.reads:
            by_slot.setdefault(z % H, []).append((rp, z))
        for slot, clears in self.cleared.items():
            for p, y in clears:
                for rp, z in by_slot.get(slot, []):
                    if z < y:   # the slot's old steps: every read before the clear
                        assert rp < p, f"step {z} read in phase {rp}, its slot cleared for {y} in phase {p}"
        # every read of a step happens after the clear that made the slot its
        # own, and no update writes a slot that the same phase reads
        own = {y: p for clears in self.cleared.values() for p, y in clears}
        for rp, z in self.reads:
            assert z in own and own[z] < rp
        for x, up in self.updated.items():
            for rp, z in by_slot.get(x % H, []):
                assert not (rp == up and z != x), f"update of {x} races a read of {z}"


@pytest.mark.parametrize("seed", range(40))
def test_window_schedule_orderings(seed):
    rng = random.Random(seed)
    dmin = rng.randint(2, 12)
    dmax = dmin + rng.randint(0, 40)
    sch = Schedule(dmin, dmax)
    # the single-step kernels need arrivals of the current step delivered: true at start
    for _ in range(30):
        if rng.random() < 0.25:
            sch.set_cycle(ACC_BUFFERS - 1)
            for _ in range(rng.randint(1, 5)):
                sch.fused_step()
        else:
            W = rng.randint(1, min(MAX_WINDOW, dmin))
            # the host's choice of cycle (wanted_acc_mask): 8 buffers for W > 4
            sch.set_cycle(ACC_BUFFERS_WIDE - 1 if W > ACC_BUFFERS else ACC_BUFFERS - 1)
            sch.window_group(rng.randint(1, 40), W)
    # every step up to the clock was updated once; arrivals of the clock's step are in
    assert sorted(sch.updated) == list(range(sch.step))
    assert sorted(sch.delivered) == list(range(sch.step + 1))
    sch.check_slots()


@pytest.mark.parametrize("W", [4, 8])
def test_window_schedule_catches_a_short_history(W):
    """The check has teeth, and H = max delay + W is the least history a window
    of W needs: with max delay + W - 1 slots it clears the next window's last
    slot while a delivery of the same phase still reads the step it held."""
    sch = Schedule(W, W + 2)
    sch.H = W + 2 + W - 1
    if W > ACC_BUFFERS:
        sch.set_cycle(ACC_BUFFERS_WIDE - 1)
    sch.window_group(4 * W, W)
    with pytest.raises(AssertionError, match="cleared"):
        sch.check_slots()


def test_window_schedule_catches_a_wide_window_in_four_buffers():
    """A window of 5 steps or more in the 4-buffer cycle: window_group
    refuses it, and without that guard the buffer check catches the fifth
    step's delivery into the buffer of a step the window has not updated."""
    sch = Schedule(8, 20)
    with pytest.raises(AssertionError, match="distinct buffers"):
        sch.window_group(16, 8)
    sch = Schedule(8, 20)
    for k in range(1, 8):
        sch.clear(k)
    with pytest.raises(AssertionError, match="still holds"):
        for k in range(1, 8):
            sch.deliver(k)


def test_window_schedule_catches_a_long_window():
    """A window longer than the minimum delay delivers a step whose source
    step is updated in the same window."""
    sch = Schedule(3, 9)
    with pytest.raises(AssertionError):
        sch.window_group(12, 4)
