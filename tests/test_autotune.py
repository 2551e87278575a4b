"""CPU checks of the autotuner's bookkeeping (invariantq_b200/autotune.py) with
an injected timer: it picks the fastest candidate (grid search over every
combination, or coordinate search one setting at a time), records the choice
and every candidate's time in the JSON cache, and reads the cache next time;
the key follows the circuit's structure, not its angles."""
import json

import pytest

from invariantq_b200.autotune import Autotuner, choice_id, circuit_key, prefix
from invariantq_b200.circuits import brickwall

SMALL = {"k": (2, 3, 4), "tile_bits": (11, 12), "budget": (80, 120, 160), "reg_slots": (4,)}


def fake_timer(circuit, cand):
    # separable, fastest at k = 3, tile bits 12, chunk bits 3, budget 200, 3 CTAs per SM
    return (10.0 + abs(cand["k"] - 3) + abs(cand["tile_bits"] - 12) + abs(cand["chunk_bits"] - 3) / 2.0
            + abs(cand["budget"] - 200) / 40.0 + abs(cand["ctas_per_sm"] - 3) / 4.0)


def test_grid_search_measures_once_and_caches(tmp_path):
    cache = tmp_path / "tune.json"
    c = brickwall(8, 6, seed=0)
    t = Autotuner(cache, candidates=SMALL, timer=fake_timer, search="grid")
    ch = t.choose(c, device="test-gpu")
    assert (ch["k"], ch["tile_bits"], ch["budget"]) == (3, 12, 160) and not ch["cached"]
    assert ch["choice_id"] == choice_id(ch)
    assert t.measured == len(t.grid()) == 18
    data = json.loads(cache.read_text())
    assert len(data) == 1 and len(next(iter(data.values()))["candidates_ms"]) == 18
    t2 = Autotuner(cache, candidates=SMALL, timer=fake_timer, search="grid")
    ch2 = t2.choose(c, device="test-gpu")
    assert ch2["cached"] and t2.measured == 0 and ch2["choice_id"] == ch["choice_id"]
    # other angles, same structure: same key; another device or size: another key
    assert circuit_key(brickwall(8, 6, seed=5), "test-gpu") == circuit_key(c, "test-gpu")
    assert circuit_key(c, "other-gpu") != circuit_key(c, "test-gpu")
    assert circuit_key(brickwall(9, 6, seed=0), "test-gpu") != circuit_key(c, "test-gpu")


def test_coordinate_search_over_the_full_space(tmp_path):
    """The default space (k, tile bits, chunk bits, budget, register slots,
    CTAs per SM) by coordinate search: the separable optimum is found with far
    fewer measurements than the grid's."""
    t = Autotuner(tmp_path / "tune.json", timer=fake_timer)
    ch = t.choose(brickwall(8, 6, seed=0), device="test-gpu")
    assert (ch["k"], ch["tile_bits"], ch["chunk_bits"], ch["budget"], ch["ctas_per_sm"]) == (3, 12, 3, 200, 3)
    assert t.measured < len(t.grid()) / 4
    assert ch["search"] == "coordinate" and ch["probe_ms"] == min(v for v in ch["candidates_ms"].values() if v)


def test_rejected_candidates_are_recorded_as_infinite(tmp_path):
    def timer(circuit, cand):
        if cand["tile_bits"] == 11:
            raise ValueError("rejected")
        return fake_timer(circuit, cand)
    t = Autotuner(tmp_path / "tune.json", timer=timer, start={"tile_bits": 11})
    ch = t.choose(brickwall(6, 4, seed=0), device="test-gpu")
    assert ch["tile_bits"] == 12
    assert any(v is None for v in ch["candidates_ms"].values())


def test_probe_is_a_prefix():
    c = brickwall(6, 4, seed=1)
    p = prefix(c, 0.25)
    assert 0 < len(p.ops) < len(c.ops)
    assert [id(o) for o in p.ops] == [id(o) for o in c.ops[:len(p.ops)]]


def test_adjoint_tuner_search_and_settings(tmp_path, monkeypatch):
    """Adjoint executor settings: coordinate search over tile bits, chunk bits,
    budget and CTA schedule with an injected timer; the choice becomes the
    environment the executor reads, and only inside the context."""
    import os

    from invariantq_b200.autotune import AdjointAutotuner, adjoint_env, adjoint_settings
    from invariantq_b200.gradients import Ansatz, PauliHamiltonian
    import numpy as np

    def timer(jobs, cand):
        return 5.0 + abs(cand["budget"] - 200) / 40 + (cand["chunk_bits"] != 3) + (cand["schedule"] != (4, 1))

    jobs = [(Ansatz.hardware_efficient(n, 2), PauliHamiltonian.tfim(n, 1.0), np.zeros((2, 4 * n)))
            for n in (4, 5, 6, 7)]
    t = AdjointAutotuner(tmp_path / "tune.json", stride=2, timer=timer)
    ch = t.choose(jobs, device="test-gpu")
    assert (ch["chunk_bits"], ch["budget"], ch["schedule"]) == (3, 200, (4, 1)) and not ch["cached"]
    again = AdjointAutotuner(tmp_path / "tune.json", stride=2, timer=timer).choose(jobs, device="test-gpu")
    assert again["cached"] and again["choice_id"] == ch["choice_id"] and again["schedule"] == (4, 1)
    monkeypatch.delenv("IQ_ADJOINT_BUDGET", raising=False)
    with adjoint_settings(ch):
        assert os.environ["IQ_ADJOINT_BUDGET"] == "200.0" and os.environ["IQ_NBUF"] == "1"
    assert "IQ_ADJOINT_BUDGET" not in os.environ
    assert adjoint_env(ch)["IQ_CTAS_PER_SM"] == "4"
