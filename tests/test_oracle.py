"""The oracle (oracle/cellato_oracle.c) pinned against Cellato itself: the
golden fixtures produced by the reference build, and -- where the reference
build is present -- direct runs of the reference CPU traverser."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.golden.make_golden import unpack_cells


def test_generator_matches_golden(golden):
    cases, arrays = golden
    for c in cases:
        cells = O.init_cells(c["x"], c["y"], c["seed"], np.array(c["thresholds"], dtype=np.uint64))
        assert O.checksum_str(cells) == c["initial_checksum"]
        if "cells" in c:
            want = unpack_cells(arrays[c["cells"] + "_init"], c["automaton"], c["x"], c["y"])
            assert (cells == want).all()


def test_thresholds_are_exact():
    assert list(O.thresholds([0.5, 0.5])) == [1 << 52]
    assert list(O.thresholds([0.125] * 8)) == [i << 50 for i in range(1, 8)]
    with pytest.raises(ValueError):
        O.thresholds([0.5, 0.6])


@pytest.mark.parametrize("stepper", ["standard", "bit_planes"])
def test_oracle_matches_golden(golden, stepper):
    cases, arrays = golden
    for c in cases:
        if stepper == "standard" and c["x"] * c["y"] * c["steps"] > 2e7:
            continue
        a, x, y = c["automaton"], c["x"], c["y"]
        cells = O.init_cells(x, y, c["seed"], np.array(c["thresholds"], dtype=np.uint64))
        if stepper == "standard":
            out = O.run_standard(a, cells, c["steps"])
        else:
            P = O.PLANES[a]
            planes = O.pack("bit_planes", cells, P, 32).view(np.uint32)
            out = O.unpack("bit_planes", O.run_bit_planes(a, planes, x, y, c["steps"]), x, y, P, 32)
        assert O.checksum_str(out) == c["checksum"], (c, stepper)
        if "cells" in c:
            assert (out == unpack_cells(arrays[c["cells"] + "_out"], a, x, y)).all()


def test_checksum_tiles_ragged():
    # 4x4 tiles of ceil(X/4) x ceil(Y/4); the last tile row/column may be short or empty.
    cells = np.ones((5, 32), dtype=np.uint8)
    ck = O.checksum(cells)
    assert ck == [16, 16, 16, 16] * 2 + [8, 8, 8, 8] + [0, 0, 0, 0]
    vals = np.arange(256, dtype=np.int64) * 3
    assert O.checksum(cells, vals) == [3 * v for v in ck]


@pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("automaton", [0, 1, 2])
def test_oracle_matches_reference_all_layouts(automaton):
    P = O.PLANES[automaton]
    probs = {0: [0.5, 0.5], 1: [0.6, 0.05, 0.05, 0.3], 2: [0.125] * 8}[automaton]
    for (x, y, steps, seed) in [(64, 32, 7, 1), (128, 40, 13, 42), (320, 24, 9, 5)]:
        cells = O.init_cells(x, y, seed, O.thresholds(probs))
        ref_cells, ref_ck = O.ref_run(automaton, cells, steps)
        assert (O.run_standard(automaton, cells, steps) == ref_cells).all()
        for layout in ("bit_planes", "bit_array", "tiled_bit_planes"):
            for W in (32, 64):
                if (layout == "bit_array" and x % (W // P)) or (layout == "bit_planes" and x % W) or \
                        (layout == "tiled_bit_planes" and y % (W // 8)):
                    continue
                packed = O.pack(layout, cells, P, W)
                assert packed.tobytes() == O.ref_pack(automaton, layout, cells, W).tobytes(), (layout, W)
                assert (O.unpack(layout, packed, x, y, P, W) == cells).all()
                rc, rck = O.ref_run(automaton, cells, steps, layout, W)
                assert rck == ref_ck and (rc == ref_cells).all(), (layout, W)


def test_thresholds_accept_decimal_probabilities_that_sum_to_one_within_rounding():
    import cellato_b200 as cb
    from fractions import Fraction
    third = [1.0 / 3] * 3
    assert (O.thresholds(third) == cb.thresholds(third)).all()
    exact = O.thresholds([Fraction(1, 3)] * 3)
    assert (exact == cb.thresholds([Fraction(1, 3)] * 3)).all()
    assert list(exact) == [(1 << 53) // 3, (2 << 53) // 3]
    with pytest.raises(ValueError):
        O.thresholds([0.5, 0.4])


def test_sample_ratio_matches_the_reference_known_answers():
    # The scripted-word known answers of the reference's own tests
    # (tests/probability.hpp:69-110), run through the oracle's restatement of
    # sample_dyadic / sample_ratio (core/probability.hpp:27-87).
    S = O.sample_ratio
    assert S(0, 3, [], lane_bits=8) == (0, 0)            # probability zero clears every lane
    assert S(3, 3, [], lane_bits=8) == (0xFF, 0)         # probability one sets every lane
    assert S(3, 3, [], active=0x25, lane_bits=8) == (0x25, 0)
    assert S(1, 3, [], active=0, lane_bits=8) == (0, 0)  # no active lanes need no random bits
    # lane k represents k/8, most significant digit drawn first
    assert S(1, 2, [0xF0], lane_bits=8) == (0x0F, 1)
    assert S(1, 4, [0xF0, 0xCC], lane_bits=8) == (0x03, 2)
    assert S(3, 8, [0xF0, 0xCC, 0xAA], lane_bits=8) == (0x07, 3)
    assert S(1, 3, [0xF0, 0xCC, 0xAA, 0, 0], lane_bits=8)[0] == 0x07
    assert S(2, 3, [0xF0, 0xCC, 0xAA, 0, 0], lane_bits=8)[0] == 0x3F
    assert S(3, 8, [0xF0, 0xCC, 0xAA], active=0x55, lane_bits=8)[0] == 0x05  # never sets inactive lanes
    # 1/3 = 0.010101...: 101 matching digits, then a smaller one; no truncation at 64 digits
    ones = (1 << 64) - 1
    prefix = [ones if d % 2 == 0 else 0 for d in range(1, 102)] + [0]
    assert S(1, 3, prefix) == (ones, 102)
    # extreme numerators and denominators do not overflow
    assert S(1, ones, [0] * 64)[0] == ones
    assert S(ones - 1, ones, [ones] * 64)[0] == 0


def test_sample_ratio_frequencies_and_reduction():
    # Reduced and unreduced ratios agree word for word, and the lanes set by
    # random words approach the probability (the reference's frequency check,
    # tests/probability.hpp:112-140, on the restatement).
    rng = np.random.default_rng(3)
    words = [int(w) for w in rng.integers(0, np.iinfo(np.uint64).max, 4000, dtype=np.uint64, endpoint=True)]
    for num, den in [(1, 3), (3, 100), (1, 1000), (3, 4), (5, 8)]:
        assert O.sample_ratio(num, den, words[:200]) == O.sample_ratio(num * 7, den * 7, words[:200])
        hits, pos = 0, 0
        for _ in range(200):
            r, used = O.sample_ratio(num, den, words[pos:pos + 80])
            assert used > 0
            hits += bin(r).count("1")
            pos = (pos + used) % 3900
        freq = hits / (200 * 64)
        sd = (num / den * (1 - num / den) / (200 * 64)) ** 0.5
        assert abs(freq - num / den) < 6 * sd + 1e-4, (num, den, freq)
