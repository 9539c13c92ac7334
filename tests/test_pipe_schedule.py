"""The arrive/wait protocol of the pipelined step group (k_pipe), restated on
the CPU: blocks run their programs in random interleavings, and each wait
passes only when the kernel's condition holds (counter phase % 4 has counted
gridDim x (phase / 4 + 1) arrivals).  Checked for every interleaving drawn:

- a wait on phase p passes only after every block arrived on phase p (the four
  counters used round-robin never let arrivals of phase p + 4 stand in for p);
- iteration i of a block (update of step s0 + i, delivery of step s0 + i + 2)
  starts only after every block finished iteration i - 2 (for i = 1: the
  prologue's delivery of step s0 + 1), which is what its reads need: the
  arrivals of step s0 + i, the spikes of steps <= s0 + i - 2, and the
  accumulator buffer step s0 + i - 2 consumed;
- no block is more than two phases ahead of another when it arrives, and no
  interleaving deadlocks."""
import random

import pytest

PHASE_COUNTERS = 4


def program(nsteps):
    """One block's sequence of k_pipe: prologue delivery, arrive 0; per
    iteration i: wait i-1 (i >= 1), work i, arrive i+1; wait n-1, wait n."""
    ops = [("work", -1), ("arrive", 0)]
    for i in range(nsteps):
        if i >= 1:
            ops.append(("wait", i - 1))
        ops.append(("work", i))
        ops.append(("arrive", i + 1))
    if nsteps >= 1:
        ops.append(("wait", nsteps - 1))
    ops.append(("wait", nsteps))
    return ops


def run_group(nb, nsteps, rng):
    counters = [0] * PHASE_COUNTERS
    arrived = [set() for _ in range(nb)]
    done_work = [set() for _ in range(nb)]
    progs = [program(nsteps) for _ in range(nb)]
    pc = [0] * nb
    while any(pc[b] < len(progs[b]) for b in range(nb)):
        runnable = []
        for b in range(nb):
            if pc[b] >= len(progs[b]):
                continue
            op, p = progs[b][pc[b]]
            if op == "wait" and counters[p % PHASE_COUNTERS] < nb * (p // PHASE_COUNTERS + 1):
                continue
            runnable.append(b)
        assert runnable, "deadlock"
        b = rng.choice(runnable)
        op, p = progs[b][pc[b]]
        if op == "wait":
            assert all(p in arrived[o] for o in range(nb)), f"wait on phase {p} passed early"
        elif op == "arrive":
            # every other block has arrived on phase p - 2 (it cannot fall further behind)
            assert all(p - 2 < 0 or p - 2 in arrived[o] for o in range(nb))
            counters[p % PHASE_COUNTERS] += 1
            arrived[b].add(p)
        else:  # work of iteration p (p = -1: the prologue)
            if p >= 1:
                assert all(p - 2 in done_work[o] for o in range(nb)), f"iteration {p} before {p - 2} finished"
            done_work[b].add(p)
        pc[b] += 1
    # at the end every block finished every iteration
    for b in range(nb):
        assert done_work[b] == set(range(-1, nsteps))


@pytest.mark.parametrize("seed", range(60))
def test_pipe_protocol_random_interleavings(seed):
    rng = random.Random(seed)
    for _ in range(5):
        run_group(rng.randint(1, 6), rng.randint(0, 24), rng)


def _fails_with(counters, seeds=200):
    global PHASE_COUNTERS
    saved = PHASE_COUNTERS
    PHASE_COUNTERS = counters
    try:
        for seed in range(seeds):
            try:
                run_group(3, 16, random.Random(seed))
            except AssertionError:
                return True
        return False
    finally:
        PHASE_COUNTERS = saved


def test_pipe_protocol_counter_margin():
    """The check has teeth: with one counter for all phases, arrivals of phase
    p + 1 (a block needs only phase p - 1 complete to make them) let a wait on
    phase p pass early.  Two counters already keep the phases apart (arriving
    on phase p + 2 needs phase p complete); the kernel's four leave a margin."""
    assert _fails_with(1)
    assert not _fails_with(2)
