"""Host logic of the grouped NUTS runner (no GPU): how many rounds NutsGroup.run
queues before it reads the draw counts back.  The count read-back is due when
the first running instance is expected to reach its target, estimated from
the draws per round its slowest chain made so far; the block size stays the
upper bound."""
import types

from augurv2_b200.hlrb import NutsGroup


def _group(active, hist_caps):
    g = object.__new__(NutsGroup)
    g.active = list(active)
    g.samplers = [types.SimpleNamespace(hist_cap=c) for c in hist_caps]
    return g


def test_rounds_to_first_finish_uses_each_instance_rate():
    g = _group([True, True, True], [128, 128, 128])
    ran = {0: 100, 1: 100, 2: 100}.get
    # 10, 20 and 40 draws after 100 rounds: 48 draws come after 380, 140 and 20 more rounds
    assert g._rounds_to_first_finish([10, 20, 40], ran, 48) == 20


def test_rounds_to_first_finish_rounds_up_and_is_at_least_one():
    g = _group([True], [128])
    assert g._rounds_to_first_finish([7], lambda i: 30, 48) == -(-(48 - 7) * 30 // 7)   # ceil(175.7) = 176
    assert g._rounds_to_first_finish([48], lambda i: 30, 48) == 1                       # due now
    assert g._rounds_to_first_finish([60], lambda i: 30, 48) == 1


def test_rounds_to_first_finish_skips_inactive_and_undrawn_instances():
    g = _group([False, True, True], [128, 128, 128])
    ran = lambda i: 50
    # instance 0 has left the launches, instance 1 has no draw yet
    assert g._rounds_to_first_finish([47, 0, 24], ran, 48) == 50
    g = _group([True, True], [128, 128])
    assert g._rounds_to_first_finish([0, 0], ran, 48) is None
    assert g._rounds_to_first_finish([5, 5], lambda i: 0, 48) is None


def test_rounds_to_first_finish_caps_the_target_at_the_history():
    g = _group([True], [16])
    # the history holds 16 draws: 8 after 40 rounds means 40 more
    assert g._rounds_to_first_finish([8], lambda i: 40, 48) == 40
