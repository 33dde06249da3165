/*
 * fzoracle.h -- CPU restatement of the FZGPUModules hot-path stage math.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * sm_100a kernels in fzgpumodules_b200/csrc.  Only tests/, the smoke()
 * entry point and bench.py's cpu_baseline / reference leg may load it; the
 * product path never calls it and has no CPU fallback.
 *
 * Every function restates one reference routine (file:line given beside
 * each declaration, paths relative to the FZGPUModules source tree) in plain
 * C11 with the reference's FP32 operation order and no FMA contraction.
 *
 * Conventions shared with the GPU build:
 *   - Lorenzo outliers are emitted sorted by element index (the reference
 *     emits them in atomicAdd order; the sorted list is one valid
 *     permutation of it).  When the capacity overflows, the first `cap`
 *     outliers by index are kept.
 *   - Codes of elements outside the logical field (pipeline padding) are 0.
 */
#ifndef FZORACLE_H
#define FZORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ErrorBoundMode (modules/fused/lorenzo_quant/lorenzo_quant.h:30-34). */
enum { ORC_ABS = 0, ORC_REL = 1, ORC_NOA = 2 };

/* Round half away from zero (the float overload of CUDA's round, used at
 * lorenzo_quant.cu:292 and lorenzo_quant_nd.cu:59,230). */
float orc_round_half_away(float v);

/* computeValueBase (modules/predictors/predictor_utils.cuh:74-117):
 * REL -> max(|min|,|max|), NOA -> max-min.  Finite inputs assumed. */
float orc_value_base(const float* x, size_t n, int mode);

/* abs_eb and ebx2_r exactly as LorenzoQuantStage::execute computes them on
 * the host (lorenzo_quant.cu:612-644).  Returns 0 on success. */
int orc_resolve_eb(float user_eb, int mode, float value_base,
                   float* abs_eb, float* ebx2_r, float* ebx2);

/* Forward fused Lorenzo predict+quantize.
 *   ndim 1: lorenzo_quantize_1d_kernel (lorenzo_quant.cu:262-364), 1024 tiles
 *   ndim 2: lorenzo_quantize_2d_kernel (lorenzo_quant_nd.cu:29-105), 32x32
 *   ndim 3: lorenzo_quantize_3d_kernel (lorenzo_quant_nd.cu:199-274), 8x8x8
 * n_total >= nx*ny*nz is the element count of the codes buffer (the pipeline
 * may pad the input); codes past the field are written as 0.
 * Returns the total outlier count (may exceed cap; only cap are stored). */
uint32_t orc_lq_fwd(const float* in, size_t n_total,
                    uint32_t nx, uint32_t ny, uint32_t nz, int ndim,
                    float ebx2_r, uint32_t radius, int zigzag,
                    uint16_t* codes, float* out_err, uint32_t* out_idx,
                    size_t cap);

/* Inverse: scatter_outliers_kernel (lorenzo_quant_kernels.cuh:23-40) then
 * lorenzo_dequantize_{1d,2d,3d}_kernel (lorenzo_quant.cu:155-244,
 * lorenzo_quant_nd.cu:112-190,281-364), reproducing their add trees. */
void orc_lq_inv(const uint16_t* codes, size_t n_total,
                const float* out_err, const uint32_t* out_idx, uint32_t n_out,
                uint32_t nx, uint32_t ny, uint32_t nz, int ndim,
                float ebx2, int zigzag, float* out);

/* Bitshuffle (modules/shufflers/bitshuffle/bitshuffle_stage.cu:299-349 for
 * ew 1/2 and the butterfly kernels at :66-293 for ew 4/8): every full
 * block of `block` bytes becomes an MSB-plane-first bit matrix; the tail
 * (< block bytes) is copied unchanged (:460-469). */
void orc_bitshuffle(const uint8_t* in, size_t bytes, uint32_t block, int ew,
                    int inverse, uint8_t* out);

/* RZE stream (modules/coders/rze/rze_stage.cu:324-445, :774-843, rze_stage.h
 * :12-23): [u32 orig][u32 n_chunks][u32 size|raw<<31 ...][chunks] padded to
 * 4 bytes with zeros.  out must hold rze_max_bytes(bytes).  Returns size. */
size_t orc_rze_max_bytes(size_t bytes);
size_t orc_rze_encode(const uint8_t* in, size_t bytes, uint8_t* out);
/* Decode (rze_stage.cu:457-551, :846-994).  Returns decoded size or
 * (size_t)-1 on a malformed stream. */
size_t orc_rze_decode(const uint8_t* in, size_t in_bytes, uint8_t* out,
                      size_t out_cap);
/* Encode one chunk (<= 16384 bytes) into dst; returns the size word with the
 * raw flag (bit 31) as the reference stores it in the stream header. */
uint32_t orc_rze_encode_chunk(const uint8_t* in, int in_size, uint8_t* dst);

/* RLE (modules/coders/rle/rle.cu:45-148, rle.h:22): elem = 1, 2 or 4 bytes.
 * [u32 runs][values, pad 4 zeroed][u32 lengths].  Returns size. */
size_t orc_rle_max_bytes(size_t n, int elem);
size_t orc_rle_encode(const void* in, size_t n, int elem, uint8_t* out);
/* Returns element count decoded, (size_t)-1 on error. */
size_t orc_rle_decode(const uint8_t* in, size_t in_bytes, int elem,
                      void* out, size_t out_cap);

/* Bitpack (modules/coders/bitpack/bitpack_stage.cu:30-124). */
int orc_bitpack_nbits_for_max(uint32_t max_val, int elem);
size_t orc_bitpack_encode(const void* in, size_t n, int elem, int nbits,
                          uint8_t* out);
void orc_bitpack_decode(const uint8_t* in, size_t n, int elem, int nbits,
                        void* out);

/* Histogram (modules/util/histogram/histogram.cu:26-60); symbols >= bklen
 * are skipped.  Returns the number of counted symbols. */
uint64_t orc_histogram(const uint16_t* in, size_t n, uint32_t bklen,
                       uint32_t* freq);

/* Canonical codebook (phf/hf_bk.cc:84-140 v2 path, phf/hf_bk_impl1.cc
 * :73-163, phf/hf_bk_internal.cc:59-101, phf/hf_canon.cc:86-131).
 * bk4: bklen u32 words (bits 31..27 = length, low 27 = code, 0xffffffff =
 * unused).  revbook: first[32] int | entry[32] int | keys u16[bklen].
 * Returns 0, or -1 when the tree is deeper than the traversal stack. */
int orc_huff_book(const uint32_t* freq, uint32_t bklen, uint32_t* bk4,
                  uint8_t* revbook);
size_t orc_huff_revbook_bytes(uint32_t bklen);
/* Coarse encode to the PHF blob (phf/hf_kernels.cu:59-132, phf/hf_hl.cc
 * :43-120, phf/hf_buf.cc:152-176).  Bytes 64..127 of the blob (encoder
 * scratch in the reference) are written as 0.  Returns blob size. */
size_t orc_huff_max_bytes(size_t n, uint32_t bklen);
size_t orc_huff_encode(const uint16_t* in, size_t n, uint32_t bklen,
                       const uint32_t* bk4, const uint8_t* revbook,
                       uint8_t* out);
/* Same blob with partitions of `sublen` symbols (1024: fine mode). */
size_t orc_huff_encode_sub(const uint16_t* in, size_t n, uint32_t bklen,
                           const uint32_t* bk4, const uint8_t* revbook,
                           uint32_t sublen, uint8_t* out);
/* Decode (phf/hf_kernels.cu:258-312).  Returns symbols written. */
size_t orc_huff_decode(const uint8_t* blob, size_t blob_bytes, uint16_t* out,
                       size_t out_cap);

/* CRC32 IEEE (src/pipeline/compressor_io.cpp:25-52). */
uint32_t orc_crc32(const void* data, size_t len);

/* Stages around the codes; ew = element bytes 1/2/4/8, arithmetic on the
 * bit pattern modulo 2^(8*ew).
 *   Zigzag (transforms/zigzag/zigzag.h:33-57), Negabinary
 *   (transforms/negabinary/negabinary.h:30-56), Difference
 *   (predictors/diff/diff.cu:26-205; chunk = elements, 0 = one chunk),
 *   integer Lorenzo (predictors/lorenzo/lorenzo_stage.cu:18-375). */
void orc_zigzag(const void* in, size_t n, int ew, int inverse, void* out);
void orc_negabinary(const void* in, size_t n, int ew, int inverse, void* out);
void orc_diff(const void* in, size_t n, int ew, size_t chunk, int nb, int inverse, void* out);
void orc_lorenzo_int(const void* in, size_t n, size_t nx, size_t ny, size_t nz, int ew, int inverse, void* out);
/* Direct quantizer ABS/NOA (quantizers/quantizer/quantizer.cu:30-167);
 * code_bytes 2 or 4; returns the outlier total, the first cap by index
 * stored.  The REL path calls CUDA's __log2f / exp2f and is checked against
 * the reference's own kernels instead. */
size_t orc_quantizer_abs(const float* in, size_t n, int code_bytes, float ebx2_r, float threshold, uint32_t radius,
                         int zigzag, void* codes, float* ovals, uint32_t* oidx, size_t cap);
void orc_quantizer_abs_inv(const void* codes, size_t n, int code_bytes, float ebx2, int zigzag, const float* ovals,
                           const uint32_t* oidx, size_t nout, float* out);
void orc_quantizer_inplace(const float* in, size_t n, float ebx2_r, float threshold, uint32_t radius,
                           uint32_t* codes);
void orc_quantizer_inplace_inv(const uint32_t* codes, size_t n, float ebx2, uint32_t radius, float* out);

#ifdef __cplusplus
}
#endif
#endif
