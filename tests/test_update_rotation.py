"""The windowed update's rotation of neuron groups over lane positions,
restated on the CPU.  The rule (run.cu, update_rotation; kernels.cuh,
neuron_window): a launch of `lanes` lanes updates `groups` groups of four
neurons in passes, the lane at position p of a pass taking group
(p + rot) mod groups; lanes [0, groups mod lanes) run one pass more than the
others.  When the POISSON neurons form one range starting on a group, the
host picks rot (a multiple of 32 before it is taken modulo the groups) so
that their groups fall in the last pass of the lanes without the extra pass
(their Philox draws make those passes the costliest); else rot = 0.  Checked here over random network shapes:
every group is updated exactly once per window, a warp's 32 positions stay
32 consecutive groups (apart from one wrap), and whenever a rotation is
chosen the POISSON groups land where the rule puts them, and on the
benchmark network's sizes it is chosen for both instantiations."""
import random


def update_rotation(groups, lanes, first, last, count):
    if count == 0 or groups < 1 or lanes < 1:
        return 0
    if last - first + 1 != count or first % 4 != 0:
        return 0
    ga, gb = first // 4, (last + 4) // 4
    passes, extra = groups // lanes, groups % lanes
    if passes < 1 or extra == 0:
        return 0
    t0 = (passes - 1) * lanes + extra
    rot0 = ga - t0
    rot = rot0 - (rot0 % 32)
    if (gb - ga) + 31 > passes * lanes - t0:
        return 0
    return rot % groups


def positions(groups, lanes, rot):
    """group -> (pass, lane) as the kernel walks the positions."""
    where = {}
    for p in range(groups):
        g = p + rot
        if g >= groups:
            g -= groups
        assert g not in where
        where[g] = (p // lanes, p % lanes)
    return where


def check(n, pois_first, pois_count, lanes):
    ns = (n + 3) & ~3
    groups = ns >> 2
    last = pois_first + pois_count - 1
    rot = update_rotation(groups, lanes, pois_first, last, pois_count)
    assert 0 <= rot < max(groups, 1)
    where = positions(groups, lanes, rot)
    assert sorted(where) == list(range(groups))  # each group once
    # a warp's positions 32w..32w+31 map to consecutive groups but at the wrap
    for w0 in range(0, groups, 32):
        gs = [(p + rot) % groups for p in range(w0, min(w0 + 32, groups))]
        breaks = sum(1 for a, b in zip(gs, gs[1:]) if b != a + 1)
        assert breaks <= 1
    if rot:
        passes, extra = groups // lanes, groups % lanes
        for g in range(pois_first // 4, (last + 4) // 4):
            pas, lane = where[g]
            assert pas == passes - 1 and lane >= extra, (g, pas, lane)
    return rot


def test_random_shapes():
    rng = random.Random(7)
    chosen = 0
    for _ in range(300):
        lanes = 32 * rng.randint(1, 40)
        n = rng.randint(1, 12 * lanes)
        first = 4 * rng.randint(0, max(0, n // 4 - 1))
        count = rng.randint(1, n - first)
        if check(n, first, count, lanes):
            chosen += 1
    assert chosen > 20


def test_benchmark_network_sizes():
    # 1M LIFB then 100k POISSON; 296 or 444 blocks of 256 threads
    for lanes in (296 * 256, 444 * 256):
        assert check(1_100_000, 1_000_000, 100_000, lanes) != 0


def test_no_rotation_without_one_range():
    assert update_rotation(1000, 256, 8, 100, 50) == 0     # not one range
    assert update_rotation(1000, 256, 2, 101, 100) == 0    # does not start on a group
    assert update_rotation(1024, 256, 0, 99, 100) == 0     # every lane runs as many passes
