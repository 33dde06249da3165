"""Loader for libfzb.so, the sm_100a kernels behind the C ABI in include/fzb.h.

The library is built in-tree (``python -m fzgpumodules_b200.build`` or
``__graft_entry__.build()``).  There is no CPU fallback: a missing library is
an ImportError-level failure, not a silent downgrade.
"""
from __future__ import annotations

import ctypes as C
import os
import re

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libfzb.so")
HEADER = os.path.join(os.path.dirname(PKG_DIR), "include", "fzb.h")

_lib = None


class FzbError(RuntimeError):
    """A non-zero status from the C ABI."""

    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = lib().fzb_status_string(status).decode() if _lib is not None else str(status)
        super().__init__(f"{what}: {msg} (status {status})" if what else msg)


def header_symbols() -> list[str]:
    """Names of the functions include/fzb.h declares."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(fzb_[a-z0-9_]+)\s*\(", text)))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is missing; build it with __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        p, u64, sz, i32, u32, f32 = C.c_void_p, C.c_uint64, C.c_size_t, C.c_int, C.c_uint32, C.c_float
        L.fzb_version.restype = i32
        L.fzb_status_string.restype = C.c_char_p
        L.fzb_status_string.argtypes = [i32]
        L.fzb_workspace_bytes.restype = sz
        L.fzb_workspace_bytes.argtypes = [u64, u64]
        L.fzb_workspace_status.restype = i32
        L.fzb_workspace_status.argtypes = [p, p]
        L.fzb_lq_forward.restype = i32
        L.fzb_lq_forward.argtypes = [p, u64, p, f32, i32, f32, u32, i32, p, p, p, u64, p, p, p, sz, p]
        L.fzb_lq_inverse.restype = i32
        L.fzb_lq_inverse.argtypes = [p, p, p, p, u64, u64, p, f32, i32, p, p, sz, p]
        L.fzb_bitshuffle.restype = i32
        L.fzb_bitshuffle.argtypes = [p, u64, u32, i32, i32, p, p]
        L.fzb_rze_max_bytes.restype = u64
        L.fzb_rze_max_bytes.argtypes = [u64]
        L.fzb_rze_encode.restype = i32
        L.fzb_rze_encode.argtypes = [p, u64, p, p, p, sz, p]
        L.fzb_rze_decode.restype = i32
        L.fzb_rze_decode.argtypes = [p, u64, u64, p, p, sz, p]
        L.fzb_lq_bs_rze_compress.restype = i32
        L.fzb_lq_bs_rze_compress.argtypes = [p, u64, p, f32, i32, f32, u32, i32, p, p, u64, p, p, p, p, p, sz, p]
        L.fzb_lq_bs_rze_decompress.restype = i32
        L.fzb_lq_bs_rze_decompress.argtypes = [p, u64, p, p, p, u64, u64, p, f32, i32, p, C.c_uint, p, sz, p]
        L.fzb_lq_bs_rze_decompress_dev.restype = i32
        L.fzb_lq_bs_rze_decompress_dev.argtypes = [p, u64, p, p, p, u64, u64, p, p, i32, p, p, sz, p]
        L.fzb_lq_inverse_dev.restype = i32
        L.fzb_lq_inverse_dev.argtypes = [p, p, p, p, u64, u64, p, p, i32, p, p, sz, p]
        L.fzb_concat_split.restype = i32
        L.fzb_concat_split.argtypes = [p, u64, p, p, i32, p, p]
        L.fzb_rle_max_bytes.restype = u64
        L.fzb_rle_max_bytes.argtypes = [u64, i32]
        L.fzb_rle_encode.restype = i32
        L.fzb_rle_encode.argtypes = [p, u64, i32, p, p, p, sz, p]
        L.fzb_rle_decode.restype = i32
        L.fzb_rle_decode.argtypes = [p, u64, i32, p, p, sz, p]
        L.fzb_bitpack_encode.restype = i32
        L.fzb_bitpack_encode.argtypes = [p, u64, i32, i32, p, p, p, p, sz, p]
        L.fzb_bitpack_decode.restype = i32
        L.fzb_bitpack_decode.argtypes = [p, u64, i32, i32, p, p]
        L.fzb_concat_bytes.restype = u64
        L.fzb_concat_bytes.argtypes = [p, i32]
        L.fzb_concat.restype = i32
        L.fzb_concat.argtypes = [p, p, i32, p, p]
        L.fzb_concat_dev.restype = i32
        L.fzb_concat_dev.argtypes = [p, p, p, p, p, p, i32, p, p]
        L.fzb_gather_words.restype = i32
        L.fzb_gather_words.argtypes = [p, p, p, i32, p, p]
        L.fzb_status_from_bits.restype = i32
        L.fzb_status_from_bits.argtypes = [u32, p]
        L.fzb_batch_workspace_bytes.restype = sz
        L.fzb_batch_workspace_bytes.argtypes = [p, i32]
        L.fzb_batch_create.restype = p
        L.fzb_batch_create.argtypes = [p, i32, p, p, sz, p]
        L.fzb_batch_launch.argtypes = [p, p]
        L.fzb_batch_destroy.restype = None
        L.fzb_batch_destroy.argtypes = [p]
        L.fzb_batch_autotune.argtypes = [p, i32, p, sz, p, p, p]
        L.fzb_sel_chunks.restype = u64
        L.fzb_sel_chunks.argtypes = [u64]
        L.fzb_sel_workspace_bytes.restype = sz
        L.fzb_sel_workspace_bytes.argtypes = [u64]
        L.fzb_sel_max_bytes.restype = u64
        L.fzb_sel_max_bytes.argtypes = [u64]
        L.fzb_sel_features.argtypes = [p, u64, p, p]
        L.fzb_sel_trial.argtypes = [p, u64, p, p, sz, p]
        L.fzb_sel_encode.argtypes = [p, u64, i32, p, p, p, p, p, sz, p]
        L.fzb_sel_decode.argtypes = [p, u64, p, u64, p, sz, p]
        L.fzb_mlp_forward.argtypes = [p, p, p, u32, p]
        L.fzb_mlp_grad.argtypes = [p, p, p, u32, i32, p, p, p]
        L.fzb_mlp_adam.argtypes = [p, p, p, p, f32, i32, p]
        L.fzb_last_error.restype = C.c_char_p
        L.fzb_last_error.argtypes = []
        L.fzb_pipeline_create.restype = p
        L.fzb_pipeline_create.argtypes = [u64, i32, f32]
        L.fzb_pipeline_destroy.restype = None
        L.fzb_pipeline_destroy.argtypes = [p]
        L.fzb_pipeline_set_dims.argtypes = [p, u64, u64, u64]
        L.fzb_pipeline_add_lorenzo_quant.argtypes = [p, f32, i32, i32, f32, i32, f32]
        L.fzb_pipeline_add_bitshuffle.argtypes = [p, u32, i32]
        L.fzb_pipeline_add_rze.argtypes = [p, u32, i32]
        L.fzb_pipeline_add_rle.argtypes = [p, i32]
        L.fzb_pipeline_add_huffman.argtypes = [p, u32]
        L.fzb_pipeline_add_huffman_mode.argtypes = [p, u32, i32]
        L.fzb_pipeline_add_bitpack.argtypes = [p, i32, i32]
        L.fzb_pfpl_workspace_bytes.restype = sz
        L.fzb_pfpl_workspace_bytes.argtypes = [u64, u64]
        L.fzb_pfpl_compress.restype = i32
        L.fzb_pfpl_compress.argtypes = [p, u64, f32, i32, f32, u32, i32, f32, p, p, u64, p, p, p, p, p, sz, p]
        L.fzb_pfpl_decompress_workspace_bytes.restype = sz
        L.fzb_pfpl_decompress_workspace_bytes.argtypes = [u64]
        L.fzb_pfpl_decompress.restype = i32
        L.fzb_pfpl_decompress.argtypes = [p, u64, p, p, p, u64, u64, f32, i32, f32, i32, p, p, sz, p]
        L.fzb_pipeline_add_quantizer.argtypes = [p, i32, f32, i32, i32, f32, i32, i32, f32, f32]
        L.fzb_pipeline_add_difference.argtypes = [p, i32, i32, u32]
        L.fzb_pipeline_add_lorenzo.argtypes = [p, i32]
        L.fzb_pipeline_add_zigzag.argtypes = [p, i32]
        L.fzb_pipeline_add_negabinary.argtypes = [p, i32]
        L.fzb_pipeline_connect.argtypes = [p, i32, i32, C.c_char_p]
        L.fzb_pipeline_load_config.argtypes = [p, C.c_char_p]
        L.fzb_pipeline_save_config.argtypes = [p, C.c_char_p]
        L.fzb_pipeline_set_fusion.argtypes = [p, i32]
        L.fzb_pipeline_enable_graph_mode.argtypes = [p, i32]
        L.fzb_pipeline_set_num_streams.argtypes = [p, i32]
        L.fzb_pipeline_decompress_graph_captured.argtypes = [p]
        L.fzb_pipeline_check_decompress.argtypes = [p, p]
        L.fzb_pipeline_num_streams.argtypes = [p]
        L.fzb_pipeline_enable_bounds_check.argtypes = [p, i32]
        L.fzb_pipeline_enable_profiling.argtypes = [p, i32]
        L.fzb_pipeline_finalize.argtypes = [p]
        L.fzb_pipeline_is_fused.argtypes = [p]
        L.fzb_pipeline_capture_graph.argtypes = [p, p]
        L.fzb_pipeline_compress.argtypes = [p, p, u64, p, p, p]
        L.fzb_pipeline_decompress.argtypes = [p, p, u64, p, p, p]
        L.fzb_pipeline_decompress_into.argtypes = [p, p, u64, p, u64, p, p]
        L.fzb_pipeline_stage_timings.argtypes = [p, p, i32]
        L.fzb_pipeline_write_file.argtypes = [p, C.c_char_p, p]
        L.fzb_decompress_file.argtypes = [C.c_char_p, p, p, p]
        L.fzb_free.argtypes = [p]
        L.fzb_trace_enable.restype = i32
        L.fzb_trace_enable.argtypes = [i32]
        L.fzb_trace_collect.restype = i32
        L.fzb_trace_collect.argtypes = []
        L.fzb_trace_get.restype = i32
        L.fzb_trace_get.argtypes = [i32, C.c_char_p, sz, p, p]
        L.fzb_trace_reset.restype = None
        L.fzb_trace_reset.argtypes = []
        L.fzb_huff_workspace_bytes.restype = sz
        L.fzb_huff_workspace_bytes.argtypes = [u64, u32]
        L.fzb_huff_max_bytes.restype = u64
        L.fzb_huff_max_bytes.argtypes = [u64, u32]
        L.fzb_huff_histogram.restype = i32
        L.fzb_huff_histogram.argtypes = [p, u64, u32, p, p]
        L.fzb_huff_book.restype = i32
        L.fzb_huff_book.argtypes = [p, u32, p, p]
        L.fzb_huff_encode.restype = i32
        L.fzb_huff_encode.argtypes = [p, u64, u32, p, p, p, p, p, sz, p]
        L.fzb_huff_compress.restype = i32
        L.fzb_huff_compress.argtypes = [p, u64, u32, p, p, p, sz, p]
        L.fzb_crc32_workspace_bytes.restype = sz
        L.fzb_crc32_workspace_bytes.argtypes = [u64]
        L.fzb_crc32.restype = i32
        L.fzb_crc32.argtypes = [p, u64, p, p, sz, p]
        for name in ("fzb_zigzag", "fzb_negabinary"):
            getattr(L, name).restype = i32
            getattr(L, name).argtypes = [p, u64, i32, i32, p, p]
        L.fzb_scan_workspace_bytes.restype = sz
        L.fzb_scan_workspace_bytes.argtypes = [u64, i32]
        L.fzb_diff.restype = i32
        L.fzb_diff.argtypes = [p, u64, i32, u64, i32, i32, p, p, sz, p]
        L.fzb_lorenzo_int.restype = i32
        L.fzb_lorenzo_int.argtypes = [p, p, u64, i32, i32, p, p, sz, p]
        L.fzb_quantizer_workspace_bytes.restype = sz
        L.fzb_quantizer_workspace_bytes.argtypes = [u64]
        L.fzb_quantizer_forward.restype = i32
        L.fzb_quantizer_forward.argtypes = [p, u64, i32, f32, i32, f32, u32, i32, f32, i32, p, p, p, p, u64, p, p,
                                            sz, p]
        L.fzb_quantizer_inverse.restype = i32
        L.fzb_quantizer_inverse.argtypes = [p, u64, i32, f32, i32, f32, u32, i32, i32, p, p, p, u64, p, p]
        L.fzb_huff_encode_fine.restype = i32
        L.fzb_huff_encode_fine.argtypes = [p, u64, u32, p, p, p, p, p, sz, p]
        L.fzb_huff_compress_fine.restype = i32
        L.fzb_huff_compress_fine.argtypes = [p, u64, u32, p, p, p, sz, p]
        L.fzb_huff_decode.restype = i32
        L.fzb_huff_decode.argtypes = [p, u64, u64, u32, p, p, sz, p]
        L.fzb_rze_encode_noalloc.restype = i32
        L.fzb_rze_encode_noalloc.argtypes = [p, u64, p, p, p]
        _lib = L
    return _lib


def check(status: int, what: str = "") -> None:
    if status != 0:
        raise FzbError(status, what)
