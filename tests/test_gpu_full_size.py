"""The benchmark workloads at full size against Cellato itself: GoL 65536^2
(Bernoulli(0.35), 1000 generations), WireWorld and Greenberg-Hastings 32768^2
(2000 generations), seeded on the device.  The expected 16-tile checksums and
SHA-256 digests of the bit-plane bytes come from the reference's own CPU
traverser run at these sizes (tests/golden/make_golden_full.py), for the
input, after 32 generations and at the end; so every cell of the GPU result
is compared with the reference, under several temporal-block depths."""
import hashlib
import json
import os

import numpy as np
import pytest

import cellato_b200 as cb

pytestmark = pytest.mark.gpu

FULL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "full")
PLANS = {"gol-65536": [dict(), dict(temporal_steps=1), dict(temporal_steps=2), dict(temporal_steps=4),
                       dict(temporal_steps=8)],
         "wire-32768": [dict(), dict(temporal_steps=4)],
         "excitable-32768": [dict(), dict(temporal_steps=8, words_per_lane=1)]}


def _case(name):
    with open(os.path.join(FULL, f"{name}.json")) as f:
        return json.load(f)


def _digest(g) -> str:
    img = g.download("bit_planes", 64)
    return hashlib.sha256(np.ascontiguousarray(img.data).data).hexdigest()


@pytest.mark.parametrize("name", sorted(PLANS))
def test_full_size_equals_the_reference(cuda, name):
    c = _case(name)
    states = {int(k): v for k, v in c["states"].items()}
    thr = np.array(c["thresholds"], dtype=np.uint64)
    for plan in PLANS[name]:
        with cb.DeviceGrid(c["automaton"], c["x"], c["y"]) as g:
            g.fill_random(c["seed"], thr=thr)
            done = 0
            for gen in sorted(states):
                g.run(gen - done, **plan)
                done = gen
                assert g.checksum_str() == states[gen]["checksum"], (name, plan, gen)
                assert _digest(g) == states[gen]["sha256"], (name, plan, gen)
            assert g.time_step == c["generations"]
