"""Host logic of the launch-shape autotuner and of the multi-instance NUTS
scheduler (no GPU): candidate shapes, selection, the on-disk cache, and the
longest-processing-time stream assignment."""
import json

from augurv2_b200 import autotune as T
from augurv2_b200.hlrb import lpt_assign


def test_candidates_are_valid_launch_shapes():
    for N, D, C in [(2_000_000, 512, 256), (1498, 256, 512), (1000, 16, 512), (64, 8, 1), (9238, 64, 512)]:
        cands = T.hlrb_candidates(N, D, C, 148)
        assert cands, (N, D, C)
        kb = (N + 63) // 64
        for c in cands:
            assert c["fwd_warps"] in (4, 8, 16) and c["fwd_bn"] in (128, 256)
            assert not (c["fwd_warps"] == 4 and c["fwd_bn"] == 256)
            assert c["bwd_bn"] in (32, 64, 128)
            assert 1 <= c["bwd_splits"] <= kb
        # the built-in shape is among them
        bn0 = 32 if D <= 32 else (64 if D <= 64 else 128)
        sp0 = T.default_splits(N, D, C, bn0, 148)
        assert {"fwd_warps": 8, "bwd_bn": bn0, "bwd_splits": sp0, "fwd_bn": 256} in cands
        assert len({json.dumps(c, sort_keys=True) for c in cands}) == len(cands)


def test_default_splits_matches_kernel_arithmetic():
    # whole 64-row K steps per split, every split non-empty
    for N, D, C in [(2_000_000, 512, 256), (1000, 16, 512), (130, 40, 3)]:
        for bn in (32, 64, 128):
            sp = T.default_splits(N, D, C, bn, 148)
            kb = (N + 63) // 64
            per = -(-kb // sp)
            assert (sp - 1) * per < kb <= sp * per


def test_select_best_picks_the_fastest():
    cands = [{"a": i} for i in range(5)]
    best, times = T.select_best(cands, lambda c: [3.0, 1.5, 2.0, 1.5, 9.0][c["a"]])
    assert best == {"a": 1}                      # ties go to the earlier one
    assert times == {0: 3.0, 1: 1.5, 2: 2.0, 3: 1.5, 4: 9.0}


def test_cache_round_trip_skips_timing(tmp_path):
    path = str(tmp_path / "tune.json")
    calls = []
    timer = lambda c: (calls.append(c), c["bwd_splits"])[1]
    cands = [{"fwd_warps": 8, "bwd_bn": 64, "bwd_splits": s} for s in (4, 2, 8)]
    t1 = T.Autotuner(cache_path=path)
    assert t1.lookup_or_tune("gpu|hlrb|k", cands, timer) == cands[1]
    assert len(calls) == 3 and t1.timed == 3
    t2 = T.Autotuner(cache_path=path)            # a later process reads the file
    assert t2.lookup_or_tune("gpu|hlrb|k", cands, timer) == cands[1]
    assert len(calls) == 3 and t2.timed == 0
    assert json.load(open(path))["gpu|hlrb|k"]["config"] == cands[1]


def test_config_struct_round_trip():
    c = T.HlrbConfigC.of({"fwd_warps": 4, "bwd_bn": 32, "bwd_splits": 7, "fwd_bn": 128})
    assert c.as_dict() == {"fwd_warps": 4, "bwd_bn": 32, "bwd_splits": 7, "fwd_bn": 128}
    assert T.HlrbConfigC.of({}).as_dict() == {"fwd_warps": 0, "bwd_bn": 0, "bwd_splits": 0, "fwd_bn": 0}
    # the ctypes layout is the C struct's (four ints, in declaration order)
    import ctypes
    assert ctypes.sizeof(T.HlrbConfigC) == 16 and T.HlrbConfigC.fwd_bn.offset == 12


def test_lpt_assignment_balances_streams():
    costs = [10, 9, 8, 1, 1, 1, 7, 2]
    a = lpt_assign(costs, 3)
    assert sorted(a) == list(range(len(costs)))
    load = [0] * 3
    for i, q in a.items():
        load[q] += costs[i]
    # Graham's bound for LPT: at most 4/3 of the optimum (here >= sum / 3)
    assert max(load) <= 4.0 / 3.0 * sum(costs) / 3 + 1e-9
    assert lpt_assign([5.0, 1.0], 4, keys=[7, 3]) == {7: 0, 3: 1}
