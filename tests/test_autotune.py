"""CPU checks of the autotuner's bookkeeping (invariantq_b200/autotune.py) with
an injected timer: it measures every candidate once, picks the fastest,
records the choice in the JSON cache, and reads the cache next time; the key
follows the circuit's structure, not its angles."""
import json

import pytest

from invariantq_b200.autotune import Autotuner, choice_id, circuit_key, prefix
from invariantq_b200.circuits import brickwall


def fake_timer(circuit, cand):
    # fastest at k = 3, tile bits 12, budget 80
    return 10.0 + abs(cand["k"] - 3) + abs(cand["tile_bits"] - 12) + abs(cand["budget"] - 80) / 40.0


def test_choose_measures_once_and_caches(tmp_path):
    cache = tmp_path / "tune.json"
    c = brickwall(8, 6, seed=0)
    t = Autotuner(cache, timer=fake_timer)
    ch = t.choose(c, device="test-gpu")
    assert (ch["k"], ch["tile_bits"], ch["budget"]) == (3, 12, 80) and not ch["cached"]
    assert ch["choice_id"] == choice_id(ch) == "k3-m12-b80-r4"
    assert t.measured == len(t.grid()) == 18
    data = json.loads(cache.read_text())
    assert len(data) == 1 and len(next(iter(data.values()))["candidates_ms"]) == 18
    t2 = Autotuner(cache, timer=fake_timer)
    ch2 = t2.choose(c, device="test-gpu")
    assert ch2["cached"] and t2.measured == 0 and ch2["choice_id"] == ch["choice_id"]
    # other angles, same structure: same key; another device or size: another key
    assert circuit_key(brickwall(8, 6, seed=5), "test-gpu") == circuit_key(c, "test-gpu")
    assert circuit_key(c, "other-gpu") != circuit_key(c, "test-gpu")
    assert circuit_key(brickwall(9, 6, seed=0), "test-gpu") != circuit_key(c, "test-gpu")


def test_probe_is_a_prefix():
    c = brickwall(6, 4, seed=1)
    p = prefix(c, 0.25)
    assert 0 < len(p.ops) < len(c.ops)
    assert [id(o) for o in p.ops] == [id(o) for o in c.ops[:len(p.ops)]]
