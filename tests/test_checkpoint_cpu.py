"""Store / recompute planning on the host: segment boundaries of a checkpointed
shot and the largest segment a memory budget allows."""
import pytest

from konglong_b200.propagator import checkpoint_plan, checkpoint_slots_for_budget


def test_plan_covers_the_forward_steps_once():
    for nts, interval, s in [(5000, 8, 155), (120, 4, 7), (90, 4, 23), (17, 1, 17), (1, 3, 1)]:
        seg = checkpoint_plan(nts, interval, s)
        assert seg[0][0] == 0 and seg[-1][1] == nts
        assert all(b == a2 for (_, b), (a2, _) in zip(seg, seg[1:]))
        # every segment but the last holds exactly s snapshots, starting on a snapshot step
        for a, b in seg:
            assert a % interval == 0
        for a, b in seg[:-1]:
            assert len(range(a, b, interval)) == s
        assert 0 < len(range(seg[-1][0], nts, interval)) <= s


def test_plan_rejects_bad_arguments():
    for args in [(0, 4, 2), (10, 0, 2), (10, 4, 0)]:
        with pytest.raises(ValueError):
            checkpoint_plan(*args)


def test_budget_picks_the_largest_fitting_segment():
    gb = 1 << 30
    # all 625 snapshots of 1 GB fit: one segment, no checkpoint
    assert checkpoint_slots_for_budget(5000, 8, gb, 10 * gb, 700 * gb) == 625
    # 160 GB for 1 GB slots and 10 GB checkpoints
    s = checkpoint_slots_for_budget(5000, 8, gb, 10 * gb, 160 * gb)
    nseg = -(-625 // s)
    assert s * gb + nseg * 10 * gb <= 160 * gb
    s1 = s + 1
    assert s1 * gb + -(-625 // s1) * 10 * gb > 160 * gb
    # nothing fits
    assert checkpoint_slots_for_budget(5000, 8, gb, 10 * gb, gb // 2) == 0
