"""The C-ABI library loads, exports every symbol the public header declares,
and its host-only entry points behave; no compute call needs a GPU here."""
import ctypes

import pytest

import cellato_b200 as cb
from cellato_b200 import _abi


def test_every_declared_symbol_is_exported():
    names = _abi.declared_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(_abi.lib, n), n


def test_header_constants_match_binding():
    text = open(_abi.HEADER_PATH).read()
    for name in ("CB2_OK", "CB2_EINVAL", "CB2_ECUDA", "CB2_ENOMEM", "CB2_ESTATE", "CB2_ETIMEOUT", "CB2_ENOTFOUND",
                 "LAYOUT_STANDARD", "LAYOUT_BIT_ARRAY", "LAYOUT_BIT_PLANES", "LAYOUT_TILED_BIT_PLANES"):
        cname = name if name.startswith("CB2_") else "CB2_" + name
        line = [l for l in text.splitlines() if l.startswith(f"#define {cname} ")][0]
        assert int(line.split()[2].strip("()")) == getattr(_abi, name)


def test_abi_version():
    assert _abi.lib.cb2_abi_version() == 4


def test_automaton_registry():
    assert cb.automaton_info("game-of-life") == ("game-of-life", 1, 2)
    assert cb.automaton_info("wire") == ("wire", 2, 4)
    assert cb.automaton_info("excitable") == ("excitable", 3, 8)
    with pytest.raises(LookupError, match="unknown automaton 'typo'"):
        cb.automaton_id("typo")


def test_layout_bytes_and_validation():
    assert cb.layout_bytes("game-of-life", "bit_planes", 64, 128, 4) == 64
    assert cb.layout_bytes("wire", "bit_planes", 32, 64, 4) == 64
    assert cb.layout_bytes("excitable", "bit_array", 32, 60, 2) == 48   # 10 cells per u32
    assert cb.layout_bytes("excitable", "bit_array", 64, 63, 1) == 24   # 21 cells per u64
    assert cb.layout_bytes("game-of-life", "tiled_bit_planes", 64, 16, 16) == 32
    assert cb.layout_bytes("game-of-life", "standard", 32, 4, 4) == 64
    with pytest.raises(ValueError, match="multiple of `word store bits`"):
        cb.layout_bytes("game-of-life", "bit_planes", 64, 96, 4)
    with pytest.raises(ValueError, match="divisible by cells_per_word"):
        cb.layout_bytes("excitable", "bit_array", 32, 64, 2)
    with pytest.raises(ValueError, match="multiples of `x_word_tile_size`"):
        cb.layout_bytes("game-of-life", "tiled_bit_planes", 64, 16, 4)


def test_grid_create_rejects_bad_sizes_without_touching_the_gpu():
    h = ctypes.c_void_p()
    assert _abi.lib.cb2_grid_create(0, 48, 16, ctypes.byref(h)) == _abi.CB2_EINVAL
    assert "multiple of 32" in _abi.last_error()
    unknown = _abi.lib.cb2_automaton_count()
    assert _abi.lib.cb2_grid_create(unknown, 64, 16, ctypes.byref(h)) == _abi.CB2_ENOTFOUND


def test_tuning_file_round_trip(tmp_path):
    p = tmp_path / "tune.txt"
    p.write_text("# comment\ngame-of-life 65536 65536 8 950 2 4\nwire 32768 32768 16 512 2 2\n")
    assert cb.tuning_load(str(p)) == 2
    out = tmp_path / "out.txt"
    assert cb.tuning_save(str(out)) >= 2
    assert "game-of-life 65536 65536 8 950 2 4" in out.read_text()
    bad = tmp_path / "bad.txt"
    bad.write_text("game-of-life 64 64 3 10 2 1\n")
    with pytest.raises(ValueError, match="invalid tuning"):
        cb.tuning_load(str(bad))


def test_network_op_counts():
    # logic + funnel-shift ops per word and generation with rows evaluated in
    # pairs (game of life 9 + 2, wire 8 + 2), and greenberg-hastings' shift
    # register (5 + 2); one shuffle per word at two words per lane
    for name, ops in (("game-of-life", 11), ("wire", 10), ("excitable", 7)):
        alu, shf = cb.network_ops(name)
        assert alu == ops and shf == 1, name


def test_server_rejects_unsupported_chunk_lengths():
    # checked before any device call: the batch kernel has pipelines of 1, 2, 4, 8, 16 and 32 generations only
    opts = _abi.ServerOpts(0, 0, 0, 12, 0, 0, 0, 0, 0, 0.0, 0)
    h = ctypes.c_void_p()
    assert _abi.lib.cb2_server_create(ctypes.byref(opts), ctypes.byref(h)) == _abi.CB2_EINVAL
    assert "temporal_steps" in _abi.last_error()
