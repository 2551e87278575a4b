"""The autotuner on a B200: it times real candidates on a 16-qubit brick-wall,
and the simulator run with the chosen settings gives the same amplitudes as
the default run (1e-12) and reports passes, bytes, kernel time and the choice."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotuned_run_matches_default(tmp_path):
    from invariantq_b200.autotune import Autotuner
    from invariantq_b200.circuits import brickwall
    from invariantq_b200.simulator import StateVectorSimulator
    c = brickwall(16, 12, seed=4)
    tuner = Autotuner(tmp_path / "tune.json", candidates={"k": (2, 3), "tile_bits": (11, 12), "budget": (48, 80),
                                                           "reg_slots": (4,)}, search="grid")
    r = StateVectorSimulator(autotune=tuner).run(c, shots=128, seed=1)
    base = StateVectorSimulator().run(c, shots=128, seed=1)
    assert np.max(np.abs(r.statevector - base.statevector)) < 1e-12
    meta = r.metadata
    assert meta["autotune"]["choice_id"] in tuner._load()[next(iter(tuner._load()))]["candidates_ms"]
    assert tuner.measured == 8 and not meta["autotune"]["cached"]
    assert meta["gate_passes"] > 0 and meta["bytes_moved"] > 0 and meta["kernel_ms"] > 0
    assert meta["achieved_GBps"] > 0
    assert meta["autotune"]["chunk_bits"] == 4 and meta["autotune"]["ctas_per_sm"] == 3
    r2 = StateVectorSimulator(autotune=tuner).run(c, shots=16, seed=2)
    assert r2.metadata["autotune"]["cached"] and tuner.measured == 8
