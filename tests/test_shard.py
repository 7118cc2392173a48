"""Tuple sharding across ranks and the one all-reduce (gloo, world size 2-3, CPU)."""
import multiprocessing as mp
import socket

import numpy as np
import pytest

from libcc_b200 import shard
from libcc_b200 import synthetic as S


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _launch(world, no, nu, seed, want_v1, tmp_path):
    import shard_worker
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=shard_worker.run, args=(r, world, port, no, nu, seed, want_v1, str(tmp_path)))
             for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    return [dict(np.load(tmp_path / f"rank{r}.npz")) for r in range(world)]


@pytest.mark.parametrize("no", [1, 2, 3, 5, 9, 24])
@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_shards_partition_the_tuple_list(no, world):
    costs = shard.tuple_costs(no)
    n_ijk = no * (no - 1) * (no - 2) // 6
    assert len(costs) == n_ijk + no * (no - 1)
    b = shard.shard_bounds(costs, world)
    assert len(b) == world + 1 and b[0] == 0 and b[-1] == len(costs)
    assert all(b[r] <= b[r + 1] for r in range(world))
    ranges = [shard.shard_of(no, r, world) for r in range(world)]
    assert ranges == [(b[r], b[r + 1]) for r in range(world)]
    # near-equal cost: no shard exceeds its fair share by more than one tuple
    total = sum(costs)
    for r in range(world):
        assert sum(costs[b[r]:b[r + 1]]) <= total / world + 1.0 + 1e-12


def test_shard_of_rejects_bad_rank():
    with pytest.raises(ValueError):
        shard.shard_of(5, 2, 2)
    with pytest.raises(ValueError):
        shard.shard_bounds([1.0], 0)


def test_single_process_forward_is_the_whole_list():
    seen = []

    def fwd(b, e):
        seen.append((b, e))
        return 1.0, 2.0, np.ones(12)
    ets, etd, v1 = shard.sharded_forward(fwd, 3, 4)
    assert seen == [(0, len(shard.tuple_costs(3)))] and (ets, etd) == (1.0, 2.0)


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_sharded_energies_match_whole_system(world, tmp_path):
    """Every rank runs only its shard; the all-reduced (ets, etd, v1) equal the
    oracle's single-process (T) and every tuple ran exactly once."""
    from oracle import oracle as O
    no, nu, seed = 5, 10, 31
    outs = _launch(world, no, nu, seed, True, tmp_path)
    inp = S.generate(no, nu, seed)
    ets_o, etd_o, v1_o = O.c_cc_triples(inp)
    covered = []
    for o in outs:
        covered += [t for b, e in o["calls"] for t in range(b, e)]
        assert abs(float(o["etd"]) - etd_o) <= 1e-12 * abs(etd_o)
        assert abs(float(o["ets"]) - ets_o) <= 1e-12 * abs(ets_o) + 1e-15
        assert np.abs(o["v1"] - v1_o).max() <= 1e-12 * np.abs(v1_o).max()
    assert sorted(covered) == list(range(len(O.all_tuples(no))))
    # every rank holds the same reduced values
    assert all(float(o["etd"]) == float(outs[0]["etd"]) for o in outs)


def test_gloo_energies_only_and_empty_shard(tmp_path):
    """no=2 has two (degenerate) tuples; with three ranks one shard is empty and
    still joins the all-reduce."""
    from oracle import oracle as O
    no, nu, seed = 2, 7, 4
    outs = _launch(3, no, nu, seed, False, tmp_path)
    inp = S.generate(no, nu, seed)
    ets_o, etd_o, _ = O.c_cc_triples(inp)
    assert sum(len(o["calls"]) for o in outs) == 2
    assert any(len(o["calls"]) == 0 for o in outs)
    for o in outs:
        assert abs(float(o["etd"]) - etd_o) <= 1e-12 * abs(etd_o)
        assert o["v1"].size == 0
