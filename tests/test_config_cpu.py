"""TOML pipeline configurations (Pipeline::loadConfig / saveConfig,
src/pipeline/config.cpp): the reference's keys, defaults and type names,
its connection rule (``inputs`` tables) and its error messages, parsed
without a GPU; a save / load round trip keeps every stage parameter."""
import math

import pytest

from fzgpumodules_b200 import config as CF
from fzgpumodules_b200 import pipeline as P

PFPL_LIKE = """
[pipeline]
memory_strategy = "PREALLOCATE"
dims = [512, 512, 64]

[[stage]]
name = "q"
type = "Quantizer"
code_type = "uint32"
error_bound = 1e-3
error_bound_mode = "REL"
outlier_capacity = 0.1

[[stage]]
name = "d"
type = "Difference"
input_type = "int32"
output_type = "uint32"
chunk_size = 16384
inputs = [{from = "q", port = "codes"}]

[[stage]]
name = "b"
type = "Bitshuffle"
element_width = 2
inputs = [{from = "d"}]

[[stage]]
name = "r"
type = "RZE"
inputs = [{from = "b", port = "output"}]
"""


def test_parse_pfpl_like():
    cfg = CF.parse_config(PFPL_LIKE)
    assert cfg["pipeline"]["memory_strategy"] == "PREALLOCATE" and cfg["pipeline"]["dims"] == [512, 512, 64]
    (_, q), (_, d), (_, b), (_, r) = cfg["stages"]
    assert isinstance(q, P.QuantizerStage) and q.code_bytes == 4 and q.eb_mode == P.REL
    assert q.zigzag_codes is True and q.quant_radius == 32768 and q.outlier_capacity == 0.1  # loader defaults
    assert math.isinf(q.outlier_threshold) and q.inplace_outliers is False
    assert isinstance(d, P.DifferenceStage) and (d.input_type, d.output_type, d.chunk_size) == (P.INT32, P.UINT32, 16384)
    assert isinstance(b, P.BitshuffleStage) and (b.block_size, b.element_width) == (16384, 2)
    assert isinstance(r, P.RZEStage) and (r.chunk_size, r.levels) == (16384, 4)
    assert [(x.getName(), y.getName(), port) for x, y, port in cfg["connections"]] == [
        ("Difference", "Quantizer", "codes"), ("Bitshuffle", "Difference", "output"), ("RZE", "Bitshuffle", "output")]


def test_defaults_per_type():
    text = "\n".join(f'[[stage]]\nname = "s{i}"\ntype = "{t}"\n' for i, t in enumerate(
        ["LorenzoQuant", "Lorenzo", "RLE", "Bitpack", "Huffman", "Zigzag", "Negabinary", "Bitshuffle"]))
    st = [s for _, s in CF.parse_config(text)["stages"]]
    assert (st[0].error_bound, st[0].eb_mode, st[0].quant_radius, st[0].outlier_capacity, st[0].zigzag_codes) == (
        1e-3, P.ABS, 32768, 0.2, False)
    assert st[1].data_type == P.INT32 and st[2].elem == 2 and (st[3].elem, st[3].nbits) == (2, 16)
    assert st[4].bklen == 1024 and st[4].encode_mode == P.HuffmanEncodeMode.Coarse
    assert st[5].input_type == P.INT32 and st[6].input_type == P.INT32
    assert st[7].element_width == 4  # the reference's Bitshuffle default


@pytest.mark.parametrize("text,msg", [
    ('[pipeline]\ndims = [1, 1, 1]\n', "no \\[\\[stage\\]\\] entries"),
    ('[[stage]]\ntype = "RZE"\n', "must have 'name' and 'type'"),
    ('[[stage]]\nname = "a"\ntype = "RZE"\n[[stage]]\nname = "a"\ntype = "RLE"\n', "duplicate stage name"),
    ('[[stage]]\nname = "a"\ntype = "Fancy"\n', "unknown stage type"),
    ('[[stage]]\nname = "a"\ntype = "RZE"\ninputs = [{port = "x"}]\n', "missing 'from'"),
    ('[[stage]]\nname = "a"\ntype = "RZE"\ninputs = [{from = "zz"}]\n', "unknown stage"),
    ('[[stage]]\nname = "a"\ntype = "Bitpack"\ninput_type = "uint32"\nnbits = 12\n', "power of two"),
])
def test_errors(text, msg):
    with pytest.raises(CF.ConfigError, match=msg):
        CF.parse_config(text)


def test_dump_round_trip():
    cfg = CF.parse_config(PFPL_LIKE)
    stages = [s for _, s in cfg["stages"]]
    text = CF.dump_config({"input_size": 4096, "memory_strategy": "PREALLOCATE", "pool_multiplier": 3.0,
                           "num_streams": 1, "dims": [512, 512, 64]}, stages, cfg["connections"])
    again = CF.parse_config(text)
    for (_, a), (_, b) in zip(cfg["stages"], again["stages"]):
        assert type(a) is type(b) and CF._stage_table(a) == CF._stage_table(b)
    assert len(again["connections"]) == 3 and again["pipeline"]["input_size"] == 4096


BAD_VALUES = [
    ('[[stage]]\nname = "a"\ntype = "LorenzoQuant"\nerror_bound_mode = "rel"\n', 'unknown error_bound_mode "rel"'),
    ('[[stage]]\nname = "a"\ntype = "Quantizer"\nerror_bound_mode = "Absolute"\n',
     'unknown error_bound_mode "Absolute"'),
    ('[pipeline]\nmemory_strategy = "prealloc"\n[[stage]]\nname = "a"\ntype = "RZE"\n',
     'unknown memory_strategy "prealloc"'),
    ('[[stage]]\nname = "a"\ntype = "Huffman"\nencode_mode = "fine"\n', 'unknown Huffman encode_mode "fine"'),
]


@pytest.mark.parametrize("text,msg", BAD_VALUES)
def test_unknown_enum_names_are_rejected(text, msg):
    # the reference throws on names it does not know (config.cpp:60-98)
    # rather than falling back to a default mode
    with pytest.raises(CF.ConfigError, match=msg):
        CF.parse_config(text)


@pytest.mark.parametrize("text,msg", BAD_VALUES + [
    ('[[stage]]\nname = "a"\ntype = "RZE"\nlevels = 4abc\n', 'bad value "4abc"'),
    ('[[stage]]\nname = "a"\ntype = "RZE"\nlevels = 0x4\n', 'bad value "0x4"'),
    ('[[stage]]\nname = "a"\ntype = "LorenzoQuant"\nerror_bound = 1e-3x\n', 'bad number "1e-3x"'),
    ('[[stage]]\nname = "a"\ntype = "RZE" levels = 4\n', "end of the line after the value of 'type'"),
])
def test_native_loader_rejects_what_the_reference_rejects(tmp_path, text, msg):
    # the C++ loader parses and fails before anything touches the device
    import ctypes as C

    from fzgpumodules_b200._lib import lib
    path = tmp_path / "bad.toml"
    path.write_text(text)
    h = lib().fzb_pipeline_create(0, 0, 3.0)
    assert h
    try:
        rc = lib().fzb_pipeline_load_config(C.c_void_p(h), str(path).encode())
        assert rc < 0
        assert msg in lib().fzb_last_error().decode()
    finally:
        lib().fzb_pipeline_destroy(C.c_void_p(h))


def test_dump_matches_the_reference_layout():
    cfg = CF.parse_config(PFPL_LIKE)
    stages = [s for _, s in cfg["stages"]]
    text = CF.dump_config({"input_size": 4096, "memory_strategy": "PREALLOCATE", "pool_multiplier": 2.5,
                           "num_streams": 1, "dims": [512, 512, 64]}, stages, cfg["connections"])
    lines = text.split("\n")
    assert lines[:9] == ["# FZGPUModules pipeline config",
                         "# Generated by Pipeline::saveConfig(). Load with Pipeline::loadConfig().", "",
                         "[pipeline]", "input_size = 4096", 'memory_strategy = "PREALLOCATE"', "pool_multiplier = 2.5",
                         "num_streams = 1", "dims = [512, 512, 64]"]
    q = text[text.index('name = "Quantizer"'):]
    assert "error_bound = 0.0010000000474974513\n" in q and "outlier_threshold" not in q
    assert 'inputs = [{ from = "Quantizer", port = "codes" }]' in text
    assert 'inputs = [{ from = "Difference" }]' in text
