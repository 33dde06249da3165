/*
 * fzb.h -- C ABI of the B200 (sm_100a) FZGPUModules hot path.
 *
 * Every entry point takes caller-owned device pointers, sizes, a caller-owned
 * device workspace (size from the matching *_workspace_bytes query) and a
 * CUDA stream passed as void*.  Nothing here allocates device memory.
 * Return value: FZB_OK (0) or a negative FZB_E_* status.  Unless a function
 * says otherwise it only enqueues work; device-side faults (malformed
 * streams, look-back timeouts) are latched in the workspace and reported by
 * fzb_workspace_status().
 *
 * Each declaration names the reference interface it replaces (paths within
 * the FZGPUModules source tree).
 */
#ifndef FZB_H
#define FZB_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FZB_OK 0
#define FZB_E_INVALID (-1)     /* bad argument / unsupported configuration   */
#define FZB_E_CUDA (-2)        /* a CUDA runtime call failed                 */
#define FZB_E_WORKSPACE (-3)   /* workspace too small                        */
#define FZB_E_CAPACITY (-4)    /* output buffer too small                    */
#define FZB_E_MALFORMED (-5)   /* compressed input is inconsistent           */
#define FZB_E_TIMEOUT (-6)     /* a bounded device wait gave up              */
#define FZB_E_RANGE (-7)       /* an input symbol is outside the codebook     */

/* Error-bound modes (modules/fused/lorenzo_quant/lorenzo_quant.h:30-34). */
#define FZB_ABS 0
#define FZB_REL 1
#define FZB_NOA 2

/* fzb_*_decompress flags */
#define FZB_NO_SYNC 1u        /* do not wait for / check the device status */
#define FZB_FORCE_EXACT 2u    /* skip the fused inverse, run the exact kernels */
#define FZB_DEVICE_FALLBACK 4u /* no host wait: the exact kernels follow the fused
                                  pass and run only if it flagged a case it leaves
                                  to them; the status is read later with
                                  fzb_workspace_status() */

int fzb_version(void);
const char* fzb_status_string(int status);

/* Per-kernel timing with CUDA events, the library side of the reference's
 * per-node profiling (Pipeline::enableProfiling / collectTimings,
 * src/pipeline/dag.cpp:107-116,418-420, include/perf.h:70).  While enabled,
 * each traced launch records an event pair on its stream.
 * fzb_trace_collect() waits for them and returns the number of distinct
 * kernel names accumulated so far (or a negative status); fzb_trace_get()
 * reads entry i (name, launches, total milliseconds). */
int fzb_trace_enable(int on);
int fzb_trace_collect(void);
int fzb_trace_get(int i, char* name, size_t name_cap, uint64_t* launches, double* total_ms);
void fzb_trace_reset(void);

/* Workspace for any entry point over n_total Lorenzo elements (or
 * 2*n_total bytes for the byte-stream coders) with room to stage up to
 * `cap` outliers (the forward entry points' outlier capacity; 0 otherwise). */
size_t fzb_workspace_bytes(uint64_t n_total, uint64_t cap);

/* Synchronises `stream` and returns the status latched in the workspace
 * (FZB_OK, FZB_E_MALFORMED or FZB_E_TIMEOUT), then clears it. */
int fzb_workspace_status(void* d_work, void* stream);

/* Device scalar block written by the forward entry points:
 * eb_state[0] value_base, [1] abs_eb, [2] ebx2_r, [3] ebx2
 * (lorenzo_quant.cu:612-644, predictor_utils.cuh:74-117). */

/* LorenzoQuantStage<float,uint16_t>::execute, forward
 * (modules/fused/lorenzo_quant/lorenzo_quant.cu:583-719; kernels
 * lorenzo_quant.cu:262-364, lorenzo_quant_nd.cu:29-105,199-274).
 * dims = {nx, ny, nz} (x fastest); ndim follows LorenzoQuantStage::ndim().
 * value_base > 0 skips the REL/NOA scan (setValueBase).  Outliers are
 * written sorted by index; *d_count receives the total found (may exceed
 * cap; only cap are stored, and on such an overflow which ones are kept
 * depends on execution order, as in the reference).  The workspace must be
 * sized with fzb_workspace_bytes(n_total, cap). */
int fzb_lq_forward(const float* d_in, uint64_t n_total, const uint32_t dims[3],
                   float eb, int eb_mode, float value_base, uint32_t radius, int zigzag,
                   uint16_t* d_codes, float* d_err, uint32_t* d_idx, uint64_t cap,
                   uint32_t* d_count, float* d_eb_state,
                   void* d_work, size_t work_bytes, void* stream);

/* LorenzoQuantStage inverse (lorenzo_quant.cu:494-581, scatter
 * lorenzo_quant_kernels.cuh:23-40, dequantize lorenzo_quant.cu:155-244,
 * lorenzo_quant_nd.cu:112-190,281-364).  abs_eb is the header's error_bound. */
int fzb_lq_inverse(const uint16_t* d_codes, const float* d_err, const uint32_t* d_idx,
                   const uint32_t* d_count, uint64_t cap, uint64_t n_total,
                   const uint32_t dims[3], float abs_eb, int zigzag, float* d_out,
                   void* d_work, size_t work_bytes, void* stream);
/* The same with the error bound read on the device from d_abs_eb (the
 * second float of the compressor's eb state), so that no host value from
 * the compression is needed: what a captured decompression graph uses.  No
 * counterpart in the reference, which reads the bound on the host. */
int fzb_lq_inverse_dev(const uint16_t* d_codes, const float* d_err, const uint32_t* d_idx,
                       const uint32_t* d_count, uint64_t cap, uint64_t n_total,
                       const uint32_t dims[3], const float* d_abs_eb, int zigzag, float* d_out,
                       void* d_work, size_t work_bytes, void* stream);

/* BitshuffleStage::execute (modules/shufflers/bitshuffle/bitshuffle_stage.cu
 * :355-475).  ew = 1, 2, 4 or 8; block a positive multiple of 1024*ew;
 * for ew 4 / 8 the buffers are ew-byte aligned.  Widths 1-2 use the ballot
 * layout (:299-349), widths 4-8 the butterfly layout (:66-278). */
int fzb_bitshuffle(const void* d_in, uint64_t bytes, uint32_t block, int ew, int inverse,
                   void* d_out, void* stream);

/* RZEStage::execute forward (modules/coders/rze/rze_stage.cu:774-843).
 * d_out must hold fzb_rze_max_bytes(bytes); *d_out_size (device u64)
 * receives the stream size (padded to 4 bytes). */
uint64_t fzb_rze_max_bytes(uint64_t bytes);
int fzb_rze_encode(const void* d_in, uint64_t bytes, void* d_out, uint64_t* d_out_size,
                   void* d_work, size_t work_bytes, void* stream);

/* RZE encode for callers that cannot allocate device memory (a plugin behind
 * a fixed-signature filter interface that only receives its input and
 * output buffers, work issued inside a stream capture that must not
 * allocate, a host callback barred from allocation calls).  No counterpart
 * in the reference: same output bytes as fzb_rze_encode, but its scratch is
 * one static device array of fixed size, resident on every device that uses
 * it until the process exits.  Inputs above FZB_RZE_NOALLOC_MAX_BYTES are
 * rejected with FZB_E_CAPACITY.  All calls on a device share that array, so
 * calls whose GPU work overlaps race and must be serialised.  The first call
 * on each device resolves the array's address; make it before any stream
 * capture.  That address is kept for the process's life and does not
 * survive cudaDeviceReset: do not call this again after a reset.  Allocates
 * nothing; d_out must hold fzb_rze_max_bytes(bytes). */
#define FZB_RZE_NOALLOC_MAX_BYTES (8ull << 20)
int fzb_rze_encode_noalloc(const void* d_in, uint64_t bytes, void* d_out, uint64_t* d_out_size,
                           void* stream);

/* RZEStage::execute inverse (rze_stage.cu:846-994) without host round
 * trips: orig_bytes is the size recorded at compression (RZE header
 * cached_orig_bytes, rze_stage.h:175-184). */
int fzb_rze_decode(const void* d_in, uint64_t in_bytes, uint64_t orig_bytes, void* d_out,
                   void* d_work, size_t work_bytes, void* stream);

/* Fused LorenzoQuant -> Bitshuffle(16384 B, ew 2) -> RZE(16384 B, 4 levels)
 * compression in one pass (the chain lorenzo_quant.cu:583-719 ->
 * bitshuffle_stage.cu:355-475 -> rze_stage.cu:774-843).  Outputs are the
 * pipeline's sinks: the outlier buffers and the RZE stream. */
int fzb_lq_bs_rze_compress(const float* d_in, uint64_t n_total, const uint32_t dims[3],
                           float eb, int eb_mode, float value_base, uint32_t radius, int zigzag,
                           float* d_err, uint32_t* d_idx, uint64_t cap, uint32_t* d_count,
                           void* d_rze, uint64_t* d_rze_size, float* d_eb_state,
                           void* d_work, size_t work_bytes, void* stream);

/* Inverse of the chain (rze_stage.cu:846-994 -> bitshuffle_stage.cu:325-349
 * -> lorenzo_quant.cu:494-581).  Single pass for 3-D fields whose rows tile
 * a 16 KiB chunk exactly; otherwise decode-to-codes + exact inverse.
 * Unless FZB_NO_SYNC is given it synchronises, verifies the device status
 * and reruns the exact kernels when the fused pass reported it left the
 * exact-integer regime. */
int fzb_lq_bs_rze_decompress(const void* d_rze, uint64_t rze_bytes, const float* d_err,
                             const uint32_t* d_idx, const uint32_t* d_count, uint64_t cap,
                             uint64_t n_total, const uint32_t dims[3], float abs_eb, int zigzag,
                             float* d_out, unsigned flags,
                             void* d_work, size_t work_bytes, void* stream);
/* The same without any host wait (FZB_DEVICE_FALLBACK) and with the error
 * bound read on the device from d_abs_eb; rze_capacity bounds the stream
 * reads (the stream's own header gives its chunk sizes).  Used by the
 * pipeline's captured decompression graph; no counterpart in the reference,
 * whose RZE and LorenzoQuant inverses read sizes and the bound on the host
 * (rze_stage.cu:853-989, lorenzo_quant.cu:494-581). */
int fzb_lq_bs_rze_decompress_dev(const void* d_rze, uint64_t rze_capacity, const float* d_err,
                                 const uint32_t* d_idx, const uint32_t* d_count, uint64_t cap,
                                 uint64_t n_total, const uint32_t dims[3], const float* d_abs_eb,
                                 int zigzag, float* d_out, void* d_work, size_t work_bytes,
                                 void* stream);

/* RLEStage<T>::execute forward (modules/coders/rle/rle.cu:261-384), element
 * width elem = 1, 2 or 4 bytes.  Wire format [u32 runs][values, padded to 4
 * bytes with zeros][u32 lengths] (rle.h:22).  d_out must hold
 * fzb_rle_max_bytes(n, elem); *d_out_size (device u64) receives the size. */
uint64_t fzb_rle_max_bytes(uint64_t n, int elem);
int fzb_rle_encode(const void* d_in, uint64_t n, int elem, void* d_out, uint64_t* d_out_size,
                   void* d_work, size_t work_bytes, void* stream);

/* RLEStage<T> inverse (rle.cu:196-259) into n elements (the element count the
 * stage header records, rle.h:123-131).  Run lengths that do not add up to n
 * are reported as FZB_E_MALFORMED by fzb_workspace_status(). */
int fzb_rle_decode(const void* d_in, uint64_t n, int elem, void* d_out, void* d_work,
                   size_t work_bytes, void* stream);

/* BitpackStage<T>::execute (modules/coders/bitpack/bitpack_stage.cu:169-244):
 * nbits a power of two <= 8*elem, or 0 to detect it from the maximum
 * (setAutoDetect, :118-124); the nbits used is written to *d_nbits (device
 * byte, optional) and the packed size to *d_out_size (device u64, optional). */
int fzb_bitpack_encode(const void* d_in, uint64_t n, int elem, int nbits, void* d_out,
                       uint8_t* d_nbits, uint64_t* d_out_size, void* d_work, size_t work_bytes,
                       void* stream);
int fzb_bitpack_decode(const void* d_in, uint64_t n, int elem, int nbits, void* d_out, void* stream);

/* PHF Huffman, HuffmanStage<uint16_t> (coarse mode; fine mode below)
 * (modules/coders/huffman/huffman_stage.cu:111-205, phf/hf_hl.cc:25-160).
 * Blob layout (phf/hf.h:38-44): [128-byte header slot][revbook = int first[32],
 * int entry[32], u16 keys[bklen]][u32 par_nbit x pardeg][u32 par_entry x
 * pardeg][u32 bitstream x total_ncell], pardeg = ceil(n / 768).  Header bytes
 * 64..127 and the upper 16 bits of the first word are written as zero (the
 * reference leaves encoder scratch there).  bklen is even, 2..65534, so every
 * u32 table of the blob stays 4-byte aligned. */
size_t fzb_huff_workspace_bytes(uint64_t n, uint32_t bklen);
uint64_t fzb_huff_max_bytes(uint64_t n, uint32_t bklen);

/* GPU_histogram_generic (util/histogram/histogram.cu): d_freq[bklen] counts
 * the symbols of d_in below bklen (larger symbols are skipped). */
int fzb_huff_histogram(const uint16_t* d_in, uint64_t n, uint32_t bklen, uint32_t* d_freq,
                       void* stream);

/* phf_CPU_build_canonized_codebook_v2 (phf/hf_bk.cc:84-140), host memory:
 * h_bk4[bklen] (bits 31..27 length, low 27 canonical code, 0xffffffff for an
 * absent symbol) and h_revbook[256 + 2*bklen]. */
int fzb_huff_book(const uint32_t* h_freq, uint32_t bklen, uint32_t* h_bk4, uint8_t* h_revbook);

/* GPU_coarse_encode + memcpy_merge (phf/hf_kernels.cu:59-140,
 * hf_buf.cc:152-176) with a device codebook: writes the blob to d_out (4-byte
 * aligned, fzb_huff_max_bytes) and its size to *d_out_size (device u64).
 * Enqueue only. */
int fzb_huff_encode(const uint16_t* d_in, uint64_t n, uint32_t bklen, const uint32_t* d_bk4,
                    const uint8_t* d_revbook, void* d_out, uint64_t* d_out_size, void* d_work,
                    size_t work_bytes, void* stream);

/* HuffmanStage<uint16_t>::execute forward: histogram, one stream
 * synchronisation to read it (as the reference does), host codebook, encode.
 * Returns FZB_E_RANGE when a symbol is >= bklen (huffman_stage.cu:151-164). */
int fzb_huff_compress(const uint16_t* d_in, uint64_t n, uint32_t bklen, void* d_out,
                      uint64_t* d_out_size, void* d_work, size_t work_bytes, void* stream);

/* HuffmanStage<uint16_t> in fine mode (setEncodeMode(Fine)): Buf with use_HFR
 * (phf/hf_buf.cc:46-58) partitions 1024 symbols; GPU_fine_encode
 * (phf/hf_kernels.cu:145-250, 486-514) when the longest code is at most 8
 * bits, else GPU_coarse_encode at sublen 1024 (phf/hf_hl.cc:69-103).  Same
 * blob layout as coarse mode with sublen 1024 and pardeg = ceil(n / 1024);
 * the bits after par_nbit in a partition's last cell are zero (the
 * reference's ReVISIT-lite kernel leaves stale shared memory there for a
 * partial last partition).  Same workspace and output bounds as coarse mode;
 * fzb_huff_decode reads the partition length from the blob. */
int fzb_huff_encode_fine(const uint16_t* d_in, uint64_t n, uint32_t bklen, const uint32_t* d_bk4,
                         const uint8_t* d_revbook, void* d_out, uint64_t* d_out_size, void* d_work,
                         size_t work_bytes, void* stream);
int fzb_huff_compress_fine(const uint16_t* d_in, uint64_t n, uint32_t bklen, void* d_out,
                           uint64_t* d_out_size, void* d_work, size_t work_bytes, void* stream);

/* HuffmanStage<uint16_t> inverse (phf/hf_kernels.cu:267-298): decodes the blob
 * (4-byte aligned, coarse or fine: sublen 768 or 1024) into n symbols.  A header that disagrees with n / bklen or a
 * bitstream that does not decode to exactly n symbols is reported as
 * FZB_E_MALFORMED by fzb_workspace_status(); work_bytes >= 256. */
int fzb_huff_decode(const void* d_in, uint64_t in_bytes, uint64_t n, uint32_t bklen, uint16_t* d_out,
                    void* d_work, size_t work_bytes, void* stream);

/* CRC-32 of device memory: the FZM data checksum (IEEE polynomial
 * 0xEDB88320, initial register and final inversion 0xFFFFFFFF;
 * src/pipeline/compressor_io.cpp:25-52, computed on the host there at
 * :218-228).  Writes the checksum to *d_crc (device u32); enqueue only.
 * Any byte alignment; up to 128 GiB. */
size_t fzb_crc32_workspace_bytes(uint64_t bytes);
int fzb_crc32(const void* d_data, uint64_t bytes, uint32_t* d_crc, void* d_work, size_t work_bytes,
              void* stream);

/* ---- Stages around the codes (enqueue only; elem_bytes 1, 2, 4 or 8;
 * arithmetic on the element bit pattern modulo 2^(8*elem_bytes)). */

/* ZigzagStage<S, U> (modules/transforms/zigzag/zigzag_stage.cu:19-96, codec
 * zigzag.h:33-57): encode signed -> unsigned, inverse decodes.  d_in may
 * equal d_out. */
int fzb_zigzag(const void* d_in, uint64_t n, int elem_bytes, int inverse, void* d_out, void* stream);
/* NegabinaryStage<S, U> (modules/transforms/negabinary/negabinary_stage.cu,
 * codec negabinary.h:30-56).  d_in may equal d_out. */
int fzb_negabinary(const void* d_in, uint64_t n, int elem_bytes, int inverse, void* d_out, void* stream);
/* Workspace of fzb_diff / fzb_lorenzo_int inverses for n elements. */
size_t fzb_scan_workspace_bytes(uint64_t n, int elem_bytes);
/* DifferenceStage<T> / DifferenceStage<S, U> (modules/predictors/diff/
 * diff.cu:26-220) for integer T: forward first differences restarting at
 * multiples of chunk_elems (a power of two; 0 = one chunk), negabinary-coded
 * when `negabinary`; inverse = the chunked prefix sum.  The forward needs
 * d_in != d_out and no workspace. */
int fzb_diff(const void* d_in, uint64_t n, int elem_bytes, uint64_t chunk_elems, int negabinary, int inverse,
             void* d_out, void* d_work, size_t work_bytes, void* stream);
/* LorenzoStage<T> (modules/predictors/lorenzo/lorenzo_stage.cu:18-400):
 * lossless integer Lorenzo.  dims {x, y, z} (0 -> x = n, y = z = 1); 1-D
 * works on all n elements in 256-element blocks, 2-D / 3-D on the
 * x*y*z field (elements past it are copied).  Forward needs d_in != d_out;
 * the 2-D / 3-D inverse needs fzb_scan_workspace_bytes(n) of workspace. */
int fzb_lorenzo_int(const void* d_in, const uint64_t dims[3], uint64_t n, int elem_bytes, int inverse, void* d_out,
                    void* d_work, size_t work_bytes, void* stream);

/* QuantizerStage<float, TCode> forward (modules/quantizers/quantizer/
 * quantizer.cu:388-649), code_bytes 2 (u16) or 4 (u32); eb_mode FZB_ABS /
 * FZB_REL / FZB_NOA; value_base > 0 skips the NOA data scan
 * (setValueBase); threshold = setOutlierThreshold (INFINITY: off); inplace =
 * setInplaceOutliers (ABS/NOA, u32 codes, zigzag required: no outlier
 * lists).  Outliers are listed in ascending index order; *d_count receives
 * min(outliers, cap).  d_eb_state (4 floats): value_base, abs_eb,
 * 1/(2 abs_eb), 2 abs_eb as resolved on the device.  Device status
 * (look-back timeout) through fzb_workspace_status(d_work). */
size_t fzb_quantizer_workspace_bytes(uint64_t n);
int fzb_quantizer_forward(const float* d_in, uint64_t n, int code_bytes, float eb, int eb_mode, float value_base,
                          uint32_t radius, int zigzag, float threshold, int inplace, void* d_codes, float* d_ovals,
                          uint32_t* d_oidx, uint32_t* d_count, uint64_t cap, float* d_eb_state, void* d_work,
                          size_t work_bytes, void* stream);
/* Inverse (quantizer.cu:398-484): abs_eb as the header stores it (ignored
 * for REL); scatters min(*d_count, cap) outliers. */
int fzb_quantizer_inverse(const void* d_codes, uint64_t n, int code_bytes, float eb, int eb_mode, float abs_eb,
                          uint32_t radius, int zigzag, int inplace, const float* d_ovals, const uint32_t* d_oidx,
                          const uint32_t* d_count, uint64_t cap, float* d_out, void* stream);

/* The pfpl preset's chain in one pass (examples/presets/pfpl.toml):
 * QuantizerStage<float, uint32_t> -> DifferenceStage<int32_t, uint32_t>
 * (16 KiB chunks) -> Bitshuffle(16384, ew 2) -> RZE(16384, 4), the chain of
 * quantizer.cu:388-649, diff.cu:26-220, bitshuffle_stage.cu:355-475 and
 * rze_stage.cu:774-843.  The RZE stream and the outliers equal those of
 * the four stages run one after another (outliers in index order unless
 * more than cap occur; then which ones are kept depends on execution
 * order); *d_count receives min(outliers, cap).  n < 2^30. */
size_t fzb_pfpl_workspace_bytes(uint64_t n, uint64_t cap);
int fzb_pfpl_compress(const float* d_in, uint64_t n, float eb, int eb_mode, float value_base, uint32_t radius,
                      int zigzag, float threshold, float* d_ovals, uint32_t* d_oidx, uint64_t cap,
                      uint32_t* d_count, void* d_rze, uint64_t* d_rze_size, float* d_eb_state, void* d_work,
                      size_t work_bytes, void* stream);
/* Its inverse: RZE decode, Bitshuffle inverse, the chunks' prefix sums and
 * dequantisation in one kernel, then the outlier scatter.  abs_eb as the
 * Quantizer header stores it (ignored for REL).  Malformed streams are
 * reported by fzb_workspace_status(d_work). */
size_t fzb_pfpl_decompress_workspace_bytes(uint64_t n);
int fzb_pfpl_decompress(const void* d_rze, uint64_t rze_bytes, const float* d_ovals, const uint32_t* d_oidx,
                        const uint32_t* d_count, uint64_t cap, uint64_t n, float eb, int eb_mode, float abs_eb,
                        int zigzag, float* d_out, void* d_work, size_t work_bytes, void* stream);

/* Pipeline output concatenation (the reference's Pipeline::concatOutputs,
 * src/pipeline/compressor.cpp:760-875; layout pipeline_utils.h:35-46):
 * [u32 n][u64 size_i x n] padded to 16 bytes, then segment i padded to 16
 * bytes, pad bytes zero.  d_out 16-byte aligned, fzb_concat_bytes() long;
 * d_srcs and sizes are host arrays of n <= FZB_CONCAT_MAX_SEGMENTS. */
#define FZB_CONCAT_MAX_SEGMENTS 32
uint64_t fzb_concat_bytes(const uint64_t* sizes, int n);
int fzb_concat(const void* const* d_srcs, const uint64_t* sizes, int n, void* d_out, void* stream);
/* The inverse of fzb_concat with the sizes read on the device: the n
 * segments of the container at d_in (in_capacity readable bytes, 16-byte
 * aligned) are copied, in whole 16-byte words, to d_dsts[i] (16-byte aligned,
 * capacities[i] bytes, a multiple of 16).  A header whose count is not n,
 * or a segment larger than its capacity or past in_capacity, sets the
 * malformed bit in *d_err (a workspace status word) and copies nothing.
 * No host wait; what the pipeline's decompression graph starts with.  The
 * reference's decompress splits the container on the host
 * (src/pipeline/compressor_exec.cpp:198-355). */
int fzb_concat_split(const void* d_in, uint64_t in_capacity, void* const* d_dsts, const uint64_t* capacities,
                     int n, uint32_t* d_err, void* stream);
/* fzb_concat enqueued before the segment sizes reach the host: segment i
 * is min(w, size_max[i]) * size_scale[i] bytes, w the u32 (size_word_bytes
 * 4) or u64 (8) at d_size_words[i], or caps[i] bytes when d_size_words[i] is
 * null; a length above caps[i] is cut to caps[i].  d_out holds
 * fzb_concat_bytes(caps, n) bytes.  The header carries the device lengths,
 * so the output equals fzb_concat of the same segments.  No counterpart in
 * the reference, whose Pipeline::compress waits for the sizes before
 * concatOutputs (src/pipeline/compressor_exec.cpp:119-152,
 * compressor.cpp:853). */
int fzb_concat_dev(const void* const* d_srcs, const uint64_t* caps, const void* const* d_size_words,
                   const uint32_t* size_word_bytes, const uint64_t* size_scale, const uint64_t* size_max,
                   int n, void* d_out, void* stream);

/* Small device results gathered for one host wait: word i (bytes[i], a
 * multiple of 4 up to 256, from a 4-byte aligned d_srcs[i]) is copied to
 * dst + offset_i, offset_i the sum of the previous lengths rounded up to 8
 * bytes each, and the source is zeroed afterwards when clear[i] (status
 * words).  dst is memory the device can store to: mapped pinned host memory
 * (cudaHostAlloc with cudaHostAllocMapped) read after the stream has been
 * synchronised.  n <= FZB_GATHER_MAX; one launch.  The reference reads each
 * such value with its own blocking copy (lorenzo_quant.cu:728-731,
 * rze_stage.cu:853,868, rle.cu:202-204). */
#define FZB_GATHER_MAX 32
int fzb_gather_words(const void* const* d_srcs, const uint32_t* bytes, const uint8_t* clear, int n, void* dst,
                     void* stream);
/* The status fzb_workspace_status() returns for a status word read without
 * it (through fzb_gather_words).  *rerun_exact (may be null) is set to 1
 * when a decompression issued with FZB_NO_SYNC left a case to the exact
 * kernels: the call is then repeated with FZB_FORCE_EXACT. */
int fzb_status_from_bits(uint32_t bits, int* rerun_exact);

/* ------------------------------------------------------------------------
 * Batched compression of many fields (no reference counterpart: it runs the
 * chain of fzb_lq_bs_rze_compress for every field in five launches --
 * reset, one value-base scan over all fields, one persistent chunk kernel
 * over every (field, chunk) unit, two assembly kernels -- plus one slab
 * kernel launch per field the single-field call codes with a slab kernel
 * (3-D, nx a power of two in [32, 1024], whole-row chunks), so a batch is one
 * CUDA graph node group).  Each field's outputs are
 * byte-identical to its own fzb_lq_bs_rze_compress call.
 *
 * fzb_batch_create validates the fields, writes the descriptors into
 * d_work (synchronous copy) and returns a handle; fzb_batch_launch only
 * enqueues (capturable; the buffers named at create time are reused on
 * every launch).  Tuning: CTAs per SM of the persistent kernel, and the
 * order fields are dispensed in (0 as given, 1 largest first); neither
 * changes any output byte.  fzb_batch_autotune times the candidates on the
 * given fields and returns the fastest.
 * ------------------------------------------------------------------------ */
typedef struct fzb_batch_field {
    const float* d_in;
    uint64_t n_total;
    uint32_t dims[3];
    float eb;
    int eb_mode;
    float value_base;
    uint32_t radius;
    int zigzag;
    float* d_err;
    uint32_t* d_idx;
    uint64_t cap;
    uint32_t* d_count;
    void* d_rze;
    uint64_t* d_rze_size;
    float* d_eb_state;
} fzb_batch_field;

/* Launch shape of a batch (zero fields take the defaults):
 * ctas_per_sm  CTAs per SM of the persistent chunk kernel (default 2);
 * order        1: the chunk kernel dispenses the largest fields first;
 * flat_tiles   1: slab-shaped 3-D fields go through the chunk kernel's flat
 *              8192-element chunks instead of the slab kernel's R-row x
 *              8-plane units (the tile shape);
 * scan_parts   value-base scan granularity, blocks per SM per field (default
 *              4; the scan of a field has at most scan_parts x SMs blocks). */
typedef struct fzb_batch_tuning {
    int ctas_per_sm;
    int order;
    int flat_tiles;
    int scan_parts;
} fzb_batch_tuning;

size_t fzb_batch_workspace_bytes(const fzb_batch_field* fields, int nfields);
void* fzb_batch_create(const fzb_batch_field* fields, int nfields, const fzb_batch_tuning* tuning, void* d_work,
                       size_t work_bytes, int* status);
int fzb_batch_launch(void* batch, void* stream);
void fzb_batch_destroy(void* batch);
/* Times launch shapes with CUDA events and returns the fastest: every CTAs
 * per SM (1-3) x dispatch order, then, from the best of those, the other
 * tile shape and scan granularities 1, 2 and 8. */
int fzb_batch_autotune(const fzb_batch_field* fields, int nfields, void* d_work, size_t work_bytes, void* stream,
                       fzb_batch_tuning* best, float* best_ms);

/* ------------------------------------------------------------------------
 * Per-chunk lossless coding with a learned coder selector (no reference
 * counterpart; every coder's bytes are its stage's bytes on that chunk).
 * Codes are cut into 64 KiB chunks (FZB_SEL_CHUNK_CODES); each chunk is
 * coded by one of: 0 Bitshuffle(16 KiB, ew 2) -> RZE, 1 RLE<u16>,
 * 2 Bitpack<u16> (detected nbits), 3 Huffman<u16> (bklen 1024, coarse).
 * Container: [u32 "FZSC"][u32 nchunks][u32 n][u32 chunk codes]
 *            [u8 tag x nchunks, pad 4][u8 param x nchunks, pad 4]
 *            [u32 size x nchunks][payloads, each padded to 4].
 * Modes: exhaustive trial (smallest output; also the labeller), learned
 * (features -> MLP -> predicted smallest; a pick that does not fit falls
 * back to trying the other coders), or one fixed coder.
 * MLP: 16 -> 64 -> 64 -> 4 FP32 with ReLU, FZB_MLP_PARAMS floats packed as
 * W1[16][64] b1[64] W2[64][64] b2[64] W3[64][4] b3[4]; it regresses the
 * four coders' costs; a chunk is coded with the coder of the smallest
 * output.  fzb_mlp_grad computes the batch gradient and loss of either the
 * mean squared error against targets T (FZB_MLP_MSE, T = log2(size/65536))
 * or the cross-entropy of softmax(-y) against the soft labels
 * softmax(-T / 0.02) (FZB_MLP_REGRET, T_k = log2(size_k / smallest size));
 * fzb_mlp_adam applies one Adam step.
 * ------------------------------------------------------------------------ */
#define FZB_SEL_CHUNK_CODES 32768
#define FZB_SEL_FEATURES 16
#define FZB_SEL_CODERS 4
#define FZB_MLP_PARAMS 5508
#define FZB_SEL_EXHAUSTIVE 0
#define FZB_SEL_LEARNED 1
#define FZB_SEL_FIXED(k) (2 + (k))
uint64_t fzb_sel_chunks(uint64_t n);
size_t fzb_sel_workspace_bytes(uint64_t n);
uint64_t fzb_sel_max_bytes(uint64_t n);
/* d_feats[nchunks][16] */
int fzb_sel_features(const uint16_t* d_codes, uint64_t n, float* d_feats, void* stream);
/* every coder's output size per chunk (d_sizes[nchunks][4], 0xFFFFFFFF =
 * does not fit / not applicable): the exhaustive-trial labels */
int fzb_sel_trial(const uint16_t* d_codes, uint64_t n, uint32_t* d_sizes, void* d_work, size_t work_bytes,
                  void* stream);
/* container into d_out (fzb_sel_max_bytes), size to *d_out_size (device
 * u64), chosen coder per chunk to d_tags (optional); d_params for LEARNED */
int fzb_sel_encode(const uint16_t* d_codes, uint64_t n, int mode, const float* d_params, void* d_out,
                   uint64_t* d_out_size, uint8_t* d_tags, void* d_work, size_t work_bytes, void* stream);
/* synchronous; work_bytes >= fzb_workspace_bytes(32768, 0) + 131328 */
int fzb_sel_decode(const void* d_in, uint64_t in_bytes, uint16_t* d_codes, uint64_t n, void* d_work,
                   size_t work_bytes, void* stream);
int fzb_mlp_forward(const float* d_params, const float* d_x, float* d_y, uint32_t batch, void* stream);
#define FZB_MLP_MSE 0
#define FZB_MLP_REGRET 1
int fzb_mlp_grad(const float* d_params, const float* d_x, const float* d_t, uint32_t batch, int loss_kind,
                 float* d_grad, float* d_loss, void* stream);
int fzb_mlp_adam(float* d_params, const float* d_grad, float* d_m, float* d_v, float lr, int step, void* stream);

/* ------------------------------------------------------------------------
 * Pipelines: C view of fz::Pipeline (include/fz/pipeline.h), the reference's
 * Pipeline API (include/pipeline/compressor.h:34-386) for bindings without
 * C++ interop.  A pipeline is an opaque handle; stages are the indices the
 * fzb_pipeline_add_* calls return (>= 0).  Errors raised inside the
 * pipeline return FZB_E_PIPELINE, with the message from fzb_last_error() on
 * the same thread.  Unlike the kernel entry points these may allocate
 * (from the pipeline's memory pool) and synchronise, as the reference's do.
 * ------------------------------------------------------------------------ */
#define FZB_E_PIPELINE (-8)    /* a pipeline call failed; see fzb_last_error() */
#define FZB_MINIMAL 0          /* MemoryStrategy::MINIMAL */
#define FZB_PREALLOCATE 1      /* MemoryStrategy::PREALLOCATE */
const char* fzb_last_error(void);
void* fzb_pipeline_create(uint64_t input_hint, int strategy, float pool_multiplier);
void fzb_pipeline_destroy(void* pipeline);
int fzb_pipeline_set_dims(void* pipeline, uint64_t x, uint64_t y, uint64_t z);
/* addStage<LorenzoQuantStage<float,uint16_t>> with Config fields. */
int fzb_pipeline_add_lorenzo_quant(void* pipeline, float eb, int eb_mode, int radius, float outlier_capacity,
                                   int zigzag, float value_base);
int fzb_pipeline_add_bitshuffle(void* pipeline, uint32_t block_size, int element_width);
int fzb_pipeline_add_rze(void* pipeline, uint32_t chunk_size, int levels);
int fzb_pipeline_add_rle(void* pipeline, int elem);
int fzb_pipeline_add_huffman(void* pipeline, uint32_t bklen);
/* HuffmanStage with setEncodeMode: 0 Coarse, 1 Fine (huffman_stage.h). */
int fzb_pipeline_add_huffman_mode(void* pipeline, uint32_t bklen, int encode_mode);
int fzb_pipeline_add_bitpack(void* pipeline, int elem, int nbits);   /* nbits 0 = setAutoDetect */
/* addStage<QuantizerStage<float, u16|u32>> with Config fields
 * (modules/quantizers/quantizer/quantizer.h:96-118); threshold INFINITY = off. */
int fzb_pipeline_add_quantizer(void* pipeline, int code_bytes, float eb, int eb_mode, int radius,
                               float outlier_capacity, int zigzag, int inplace, float threshold, float value_base);
/* addStage<DifferenceStage<T, TOut>> (modules/predictors/diff/diff.h); types
 * are FZM DataType codes (0 u8, 1 u16, 2 u32, 3 u64, 4 i8, 5 i16, 6 i32,
 * 7 i64): out_type == in_type, or the unsigned type of a signed in_type
 * (negabinary-fused).  chunk_size in bytes (setChunkSize; 0 = one chunk). */
int fzb_pipeline_add_difference(void* pipeline, int in_type, int out_type, uint32_t chunk_size);
/* addStage<LorenzoStage<T>> (modules/predictors/lorenzo/lorenzo_stage.h), T
 * signed (DataType code 4..7); dims come from fzb_pipeline_set_dims. */
int fzb_pipeline_add_lorenzo(void* pipeline, int data_type);
/* addStage<ZigzagStage<S, U>> / <NegabinaryStage<S, U>> (modules/transforms/
 * zigzag/zigzag_stage.h, negabinary/negabinary_stage.h), S signed (4..7). */
int fzb_pipeline_add_zigzag(void* pipeline, int in_type);
int fzb_pipeline_add_negabinary(void* pipeline, int in_type);
/* Pipeline::loadConfig / saveConfig (src/pipeline/config.cpp:515-640): a
 * TOML file's [pipeline] settings and [[stage]] tables, connected by their
 * `inputs` and finalized; saveConfig writes a finalized pipeline. */
int fzb_pipeline_load_config(void* pipeline, const char* path);
int fzb_pipeline_save_config(void* pipeline, const char* path);
/* connect(dependent, producer, output_name); returns the buffer id. */
int fzb_pipeline_connect(void* pipeline, int dependent, int producer, const char* output_name);
/* Fusion of LorenzoQuant -> Bitshuffle -> RZE into one pass (default on). */
int fzb_pipeline_set_fusion(void* pipeline, int on);
int fzb_pipeline_enable_graph_mode(void* pipeline, int on);
/* Pipeline::setNumStreams (include/pipeline/compressor.h:64): side streams
 * for DAG levels with several stages; before finalize.  fzb_pipeline_num_streams
 * returns the count in use after finalize (1 = the caller's stream only). */
int fzb_pipeline_set_num_streams(void* pipeline, int num_streams);
int fzb_pipeline_num_streams(void* pipeline);
/* Pipeline::enableBoundsCheck (include/pipeline/compressor.h:306): after each
 * stage, compare its actual output sizes with the reserved bytes and fail
 * with "Buffer overwrite detected" (dag.cpp:438-462). */
int fzb_pipeline_enable_bounds_check(void* pipeline, int on);
int fzb_pipeline_enable_profiling(void* pipeline, int on);
int fzb_pipeline_finalize(void* pipeline);
int fzb_pipeline_is_fused(void* pipeline);
int fzb_pipeline_capture_graph(void* pipeline, void* stream);
/* 1 when captureGraph also captured the decompression (then decompress
 * replays it with no host wait), else 0. */
int fzb_pipeline_decompress_graph_captured(void* pipeline);
/* Waits for the last decompress and fails (-8, message in fzb_last_error)
 * if the device found its input malformed. */
int fzb_pipeline_check_decompress(void* pipeline, void* stream);
/* compress (pool-owned output, valid until the next compress). */
int fzb_pipeline_compress(void* pipeline, const void* d_in, uint64_t bytes, void** d_out, uint64_t* out_bytes,
                          void* stream);
/* decompress (pool-owned output; d_in NULL = the pipeline's last outputs). */
int fzb_pipeline_decompress(void* pipeline, const void* d_in, uint64_t bytes, void** d_out, uint64_t* out_bytes,
                            void* stream);
int fzb_pipeline_decompress_into(void* pipeline, const void* d_in, uint64_t bytes, void* d_out, uint64_t capacity,
                                 uint64_t* out_bytes, void* stream);
/* Per-stage milliseconds of the last profiled compress (enableProfiling);
 * returns the number of entries written. */
int fzb_pipeline_stage_timings(void* pipeline, double* ms, int max_entries);
/* writeToFile: FZM v3.1 with CRC32 checksums (src/pipeline/compressor_io.cpp:178-265). */
int fzb_pipeline_write_file(void* pipeline, const char* path, void* stream);
/* Pipeline::decompressFromFile: *d_out is cudaMalloc'd; release it with fzb_free. */
int fzb_decompress_file(const char* path, void** d_out, uint64_t* out_bytes, void* stream);
int fzb_free(void* d_ptr);

#ifdef __cplusplus
}
#endif
#endif
