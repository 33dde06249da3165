/*
 * fzoracle.c -- CPU restatement of the FZGPUModules hot path (parity oracle).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the sm_100a kernels; see
 * fzoracle.h.  Built with -O2 -ffp-contract=off (no FMA) -fopenmp.
 */
#include "fzoracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* rounding, value base, error bound                                   */
/* ------------------------------------------------------------------ */

float orc_round_half_away(float v) {
    float t = truncf(v);
    float d = v - t; /* exact: fractional part of a float */
    if (fabsf(d) >= 0.5f) t += (v < 0.0f) ? -1.0f : 1.0f;
    return t;
}

/* predictor_utils.cuh:27-62,104-116: min/max with `<` / `>` comparisons. */
float orc_value_base(const float* x, size_t n, int mode) {
    if (n == 0) return 0.0f;
    float gmin = x[0], gmax = x[0];
    for (size_t i = 1; i < n; i++) {
        float v = x[i];
        if (v < gmin) gmin = v;
        if (v > gmax) gmax = v;
    }
    if (mode == ORC_NOA) return gmax - gmin;
    float amin = (gmin < 0.0f) ? -gmin : gmin;
    float amax = (gmax < 0.0f) ? -gmax : gmax;
    return amin > amax ? amin : amax;
}

/* lorenzo_quant.cu:612-644 (abs_eb, ebx2_r) and :511 (ebx2). */
int orc_resolve_eb(float user_eb, int mode, float value_base, float* abs_eb,
                   float* ebx2_r, float* ebx2) {
    float a;
    if (mode == ORC_ABS || value_base <= 0.0f)
        a = user_eb;
    else
        a = user_eb * value_base;
    *abs_eb = a;
    *ebx2_r = 1.0f / (2.0f * a);
    *ebx2 = 2.0f * a;
    return 0;
}

static inline uint16_t lq_code(float c, int zigzag) {
    int iv = (int)c;
    if (zigzag) {
        int16_t s = (int16_t)iv;
        uint16_t u = (uint16_t)s;
        return (uint16_t)((uint16_t)(u << 1) ^ (uint16_t)(s >> 15));
    }
    return (uint16_t)iv;
}

static inline float lq_decode(uint16_t u, int zigzag) {
    if (zigzag) {
        int16_t s = (int16_t)((u >> 1) ^ (uint16_t)(-(int16_t)(u & 1u)));
        return (float)s;
    }
    return (float)(int16_t)u;
}

/* ------------------------------------------------------------------ */
/* Lorenzo forward                                                     */
/* ------------------------------------------------------------------ */

/* Per-element Lorenzo delta in the reference operation order.  q() reads
 * the pre-quantized value of an in-field neighbour. */
#define QV(X, Y, Z) qbuf[((size_t)(Z) * ny + (Y)) * nx + (X)]

uint32_t orc_lq_fwd(const float* in, size_t n_total, uint32_t nx,
                    uint32_t ny, uint32_t nz, int ndim, float ebx2_r,
                    uint32_t radius, int zigzag, uint16_t* codes,
                    float* out_err, uint32_t* out_idx, size_t cap) {
    const size_t nfield = (size_t)nx * ny * nz;
    float* qbuf = (float*)malloc(sizeof(float) * (nfield ? nfield : 1));
    const float rad = (float)(uint16_t)radius; /* TCode radius, :251 */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < nfield; i++) qbuf[i] = orc_round_half_away(in[i] * ebx2_r);

    float* delta = (float*)malloc(sizeof(float) * (nfield ? nfield : 1));
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < nfield; i++) {
        uint32_t x = (uint32_t)(i % nx);
        uint32_t y = (uint32_t)((i / nx) % ny);
        uint32_t z = (uint32_t)(i / ((size_t)nx * ny));
        float c;
        if (ndim == 3) {
            /* z first (delta[z] -= delta[z-1], :236), then x within an
             * 8-wide segment (:239-241), then y via shared memory (:244-246) */
            int tx = x % 8, ty = y % 8, tz = z % 8;
            float a00 = QV(x, y, z) - (tz ? QV(x, y, z - 1) : 0.0f);
            float b0 = a00;
            if (tx) {
                float a10 = QV(x - 1, y, z) - (tz ? QV(x - 1, y, z - 1) : 0.0f);
                b0 = a00 - a10;
            }
            c = b0;
            if (ty) {
                float a01 = QV(x, y - 1, z) - (tz ? QV(x, y - 1, z - 1) : 0.0f);
                float b1 = a01;
                if (tx) {
                    float a11 = QV(x - 1, y - 1, z) -
                                (tz ? QV(x - 1, y - 1, z - 1) : 0.0f);
                    b1 = a01 - a11;
                }
                c = b0 - b1;
            }
        } else if (ndim == 2) {
            /* y first (center[i] -= center[i-1], :74), then x via a 32-wide
             * shuffle (:76-77) */
            int tx = x % 32, ty = y % 32;
            float v0 = QV(x, y, 0) - (ty ? QV(x, y - 1, 0) : 0.0f);
            c = v0;
            if (tx) {
                float v1 = QV(x - 1, y, 0) - (ty ? QV(x - 1, y - 1, 0) : 0.0f);
                c = v0 - v1;
            }
        } else {
            /* 1024-element tiles restart at 0 (:308-312) */
            size_t t = i % 1024;
            c = qbuf[i] - (t ? qbuf[i - 1] : 0.0f);
        }
        delta[i] = c;
    }

    uint32_t count = 0;
    for (size_t i = 0; i < nfield; i++) {
        float c = delta[i];
        if (fabsf(c) < rad) {
            codes[i] = lq_code(c, zigzag);
        } else {
            codes[i] = 0;
            if (count < cap) {
                out_err[count] = c;
                out_idx[count] = (uint32_t)i;
            }
            count++;
        }
    }
    for (size_t i = nfield; i < n_total; i++) codes[i] = 0;
    free(delta);
    free(qbuf);
    return count;
}

/* ------------------------------------------------------------------ */
/* Lorenzo inverse                                                     */
/* ------------------------------------------------------------------ */

/* In-place Hillis-Steele inclusive scan over v[0..n), n a power of two:
 * the add tree of a __shfl_up_sync loop `if (lane >= d) v += up(v, d)`. */
static void hs_scan(float* v, int n) {
    float tmp[1024];
    for (int d = 1; d < n; d *= 2) {
        memcpy(tmp, v, sizeof(float) * n);
        for (int i = d; i < n; i++) v[i] = tmp[i] + tmp[i - d];
    }
}

void orc_lq_inv(const uint16_t* codes, size_t n_total, const float* out_err,
                const uint32_t* out_idx, uint32_t n_out, uint32_t nx,
                uint32_t ny, uint32_t nz, int ndim, float ebx2, int zigzag,
                float* out) {
    const size_t nfield = (size_t)nx * ny * nz;
    /* memset + scatter (lorenzo_quant.cu:427-441) */
    memset(out, 0, sizeof(float) * n_total);
    for (uint32_t k = 0; k < n_out; k++)
        if (out_idx[k] < n_total) out[out_idx[k]] = out_err[k];

    if (ndim == 3) {
        const uint32_t tnx = (nx + 7) / 8, tny = (ny + 7) / 8, tnz = (nz + 7) / 8;
        const size_t ntiles = (size_t)tnx * tny * tnz;
#pragma omp parallel for schedule(static)
        for (size_t t = 0; t < ntiles; t++) {
            uint32_t bx = (uint32_t)(t % tnx), by = (uint32_t)((t / tnx) % tny),
                     bz = (uint32_t)(t / ((size_t)tnx * tny));
            float v[8][8][8]; /* [z][y][x] */
            for (int lz = 0; lz < 8; lz++)
                for (int ly = 0; ly < 8; ly++)
                    for (int lx = 0; lx < 8; lx++) {
                        uint32_t x = bx * 8 + lx, y = by * 8 + ly, z = bz * 8 + lz;
                        float d = 0.0f;
                        if (x < nx && y < ny && z < nz) {
                            size_t g = ((size_t)z * ny + y) * nx + x;
                            d = out[g] + lq_decode(codes[g], zigzag);
                        }
                        v[lz][ly][lx] = d;
                    }
            /* y sequential (:325), x HS in 8-lane segments (:333-336),
             * z HS after the smem transpose (:345-348) */
            for (int lz = 0; lz < 8; lz++)
                for (int lx = 0; lx < 8; lx++)
                    for (int ly = 1; ly < 8; ly++) v[lz][ly][lx] += v[lz][ly - 1][lx];
            for (int lz = 0; lz < 8; lz++)
                for (int ly = 0; ly < 8; ly++) hs_scan(v[lz][ly], 8);
            for (int ly = 0; ly < 8; ly++)
                for (int lx = 0; lx < 8; lx++) {
                    float col[8];
                    for (int lz = 0; lz < 8; lz++) col[lz] = v[lz][ly][lx];
                    hs_scan(col, 8);
                    for (int lz = 0; lz < 8; lz++) v[lz][ly][lx] = col[lz];
                }
            for (int lz = 0; lz < 8; lz++)
                for (int ly = 0; ly < 8; ly++)
                    for (int lx = 0; lx < 8; lx++) {
                        uint32_t x = bx * 8 + lx, y = by * 8 + ly, z = bz * 8 + lz;
                        if (x < nx && y < ny && z < nz)
                            out[((size_t)z * ny + y) * nx + x] = v[lz][ly][lx] * ebx2;
                    }
        }
    } else if (ndim == 2) {
        const uint32_t tnx = (nx + 31) / 32, tny = (ny + 31) / 32;
        const size_t ntiles = (size_t)tnx * tny;
#pragma omp parallel for schedule(static)
        for (size_t t = 0; t < ntiles; t++) {
            uint32_t bx = (uint32_t)(t % tnx), by = (uint32_t)(t / tnx);
            float v[32][32]; /* [y][x] */
            for (int ly = 0; ly < 32; ly++)
                for (int lx = 0; lx < 32; lx++) {
                    uint32_t x = bx * 32 + lx, y = by * 32 + ly;
                    float d = 0.0f;
                    if (x < nx && y < ny) {
                        size_t g = (size_t)y * nx + x;
                        d = out[g] + lq_decode(codes[g], zigzag);
                    }
                    v[ly][lx] = d;
                }
            /* each of 4 warps scans its 8 rows (:148), then the exclusive
             * prefix of warp totals computed sequentially by warp 0
             * (:151-170), then a 32-lane HS along x (:175-181) */
            for (int lx = 0; lx < 32; lx++) {
                for (int w = 0; w < 4; w++)
                    for (int i = 1; i < 8; i++) v[w * 8 + i][lx] += v[w * 8 + i - 1][lx];
                float acc[3];
                for (int w = 0; w < 3; w++) acc[w] = v[w * 8 + 7][lx];
                acc[1] += acc[0];
                acc[2] += acc[1];
                for (int w = 1; w < 4; w++)
                    for (int i = 0; i < 8; i++) v[w * 8 + i][lx] += acc[w - 1];
            }
            for (int ly = 0; ly < 32; ly++) hs_scan(v[ly], 32);
            for (int ly = 0; ly < 32; ly++)
                for (int lx = 0; lx < 32; lx++) {
                    uint32_t x = bx * 32 + lx, y = by * 32 + ly;
                    if (x < nx && y < ny) out[(size_t)y * nx + x] = v[ly][lx] * ebx2;
                }
        }
    } else {
        /* 1024-element tiles, 256 threads x Seq=4 (lorenzo_quant.cu:155-244) */
        const size_t ntiles = (nfield + 1023) / 1024;
#pragma omp parallel for schedule(static)
        for (size_t t = 0; t < ntiles; t++) {
            float v[1024];
            for (int j = 0; j < 1024; j++) {
                size_t g = t * 1024 + j;
                v[j] = (g < nfield) ? out[g] + lq_decode(codes[g], zigzag) : 0.0f;
            }
            float tsum[256];
            for (int th = 0; th < 256; th++) {
                float* p = v + th * 4;
                for (int i = 1; i < 4; i++) p[i] += p[i - 1];
                tsum[th] = p[3];
            }
            /* warp_inclusive_scan: HS of thread sums, then each thread adds
             * the inclusive value of the lane before it (:27-49) */
            for (int w = 0; w < 8; w++) {
                float s[32];
                memcpy(s, tsum + w * 32, sizeof(s));
                hs_scan(s, 32);
                for (int l = 1; l < 32; l++) {
                    float* p = v + (w * 32 + l) * 4;
                    for (int i = 0; i < 4; i++) p[i] += s[l - 1];
                }
            }
            /* block_exclusive_scan: HS over the 8 warp totals (:52-87) */
            float wt[8];
            for (int w = 0; w < 8; w++) wt[w] = v[(w * 32 + 31) * 4 + 3];
            hs_scan(wt, 8);
            for (int w = 1; w < 8; w++)
                for (int j = w * 128; j < w * 128 + 128; j++) v[j] += wt[w - 1];
            for (int j = 0; j < 1024; j++) {
                size_t g = t * 1024 + j;
                if (g < nfield) out[g] = v[j] * ebx2;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* Bitshuffle                                                          */
/* ------------------------------------------------------------------ */

/* Plane p holds bit W-1-p of every element of the block.  Element widths 1
 * and 2 (bitshuffle_stage.cu:299-349, ballot kernels): plane words are u32,
 * element 32g+e at bit e of word g.  Widths 4 and 8 (the butterfly kernels,
 * :66-110 and :175-278): plane words are u32 / u64 and element e of a group
 * sits at the word's bit W'-1-e (W' = 32 / 64), i.e. the group order is
 * reversed inside the word. */
static inline size_t bs_slot(uint32_t ew, uint32_t W, uint32_t nchunk, uint32_t i, uint32_t bit, int* pos) {
    if (ew <= 2) {
        *pos = (int)(i % 32);
        return (size_t)(W - 1 - bit) * (nchunk / 32) * 4 + (size_t)(i / 32) * 4;  /* byte offset of the u32 word */
    }
    const uint32_t gw = ew == 4 ? 32u : 64u;  /* elements per plane word */
    *pos = (int)(gw - 1 - i % gw);
    return (size_t)(W - 1 - bit) * (nchunk / gw) * (gw / 8) + (size_t)(i / gw) * (gw / 8);
}

void orc_bitshuffle(const uint8_t* in, size_t bytes, uint32_t block, int ew,
                    int inverse, uint8_t* out) {
    const size_t nfull = bytes / block;
    const uint32_t W = (uint32_t)ew * 8u;
    const uint32_t nchunk = block / (uint32_t)ew; /* elements per block */
#pragma omp parallel for schedule(static)
    for (size_t b = 0; b < nfull; b++) {
        const uint8_t* src = in + b * block;
        uint8_t* dst = out + b * block;
        if (!inverse) {
            memset(dst, 0, block);
            for (uint32_t i = 0; i < nchunk; i++) {
                uint64_t val = 0;
                memcpy(&val, src + (size_t)i * ew, (size_t)ew);
                for (uint32_t bit = 0; bit < W; bit++)
                    if ((val >> bit) & 1u) {
                        int pos;
                        const size_t off = bs_slot((uint32_t)ew, W, nchunk, i, bit, &pos);
                        dst[off + (size_t)(pos / 8)] |= (uint8_t)(1u << (pos % 8));
                    }
            }
        } else {
            for (uint32_t i = 0; i < nchunk; i++) {
                uint64_t val = 0;
                for (uint32_t bit = 0; bit < W; bit++) {
                    int pos;
                    const size_t off = bs_slot((uint32_t)ew, W, nchunk, i, bit, &pos);
                    if ((src[off + (size_t)(pos / 8)] >> (pos % 8)) & 1u) val |= (uint64_t)1 << bit;
                }
                memcpy(dst + (size_t)i * ew, &val, (size_t)ew);
            }
        }
    }
    if (bytes > nfull * block)
        memcpy(out + nfull * block, in + nfull * block, bytes - nfull * block);
}

/* ------------------------------------------------------------------ */
/* RZE                                                                 */
/* ------------------------------------------------------------------ */

#define RZE_CS 16384
#define RZE_BM4 4

/* RE level: bytes differing from their predecessor (position 0 vs 0), and
 * the bitmap of those positions (rze_stage.cu:184-224). */
static int re_level(const uint8_t* src, int n, uint8_t* dst, uint8_t* bm, int bm_bytes) {
    memset(bm, 0, (size_t)bm_bytes);
    int k = 0;
    for (int i = 0; i < n; i++) {
        uint8_t p = i ? src[i - 1] : 0;
        if (src[i] != p) {
            dst[k++] = src[i];
            bm[i >> 3] |= (uint8_t)(1u << (i & 7));
        }
    }
    return k;
}

uint32_t orc_rze_encode_chunk(const uint8_t* in, int in_size, uint8_t* out) {
    uint8_t bm1[RZE_CS / 8], bm2[RZE_CS / 64], bm3[RZE_CS / 512], bm4[RZE_BM4];
    memset(bm1, 0, sizeof(bm1));
    /* L1 zero elimination (:135-176) */
    int wpos = 0;
    for (int i = 0; i < in_size; i++)
        if (in[i]) {
            out[wpos++] = in[i];
            bm1[i >> 3] |= (uint8_t)(1u << (i & 7));
        }
    if (wpos == 0) { /* all zero: only the size tag (:359-367) */
        out[0] = (uint8_t)(in_size & 0xFF);
        out[1] = (uint8_t)((in_size >> 8) & 0xFF);
        return 2;
    }
    const int avail = RZE_CS - 2;
    const uint32_t raw = (1u << 31) | (uint32_t)in_size;
    const int b1 = (in_size + 7) / 8;
    if (wpos >= avail || wpos > avail - b1) goto store_raw;
    wpos += re_level(bm1, b1, out + wpos, bm2, (int)sizeof(bm2));
    if (wpos >= avail) goto store_raw;
    const int b2 = (b1 + 7) / 8;
    if (wpos >= avail || wpos > avail - b2) goto store_raw;
    wpos += re_level(bm2, b2, out + wpos, bm3, (int)sizeof(bm3));
    if (wpos >= avail) goto store_raw;
    const int b3 = (b2 + 7) / 8;
    if (wpos >= avail - RZE_BM4 || wpos > (avail - RZE_BM4) - b3) goto store_raw;
    wpos += re_level(bm3, b3, out + wpos, bm4, RZE_BM4);
    if (wpos >= avail - RZE_BM4) goto store_raw;
    memcpy(out + wpos, bm4, RZE_BM4);
    wpos += RZE_BM4;
    out[wpos] = (uint8_t)(in_size & 0xFF);
    out[wpos + 1] = (uint8_t)((in_size >> 8) & 0xFF);
    return (uint32_t)(wpos + 2);
store_raw:
    memcpy(out, in, (size_t)in_size);
    return raw;
}

size_t orc_rze_max_bytes(size_t bytes) {
    size_t nch = (bytes + RZE_CS - 1) / RZE_CS;
    return 8 + 4 * nch + nch * (size_t)RZE_CS + 4;
}

size_t orc_rze_encode(const uint8_t* in, size_t bytes, uint8_t* out) {
    if (bytes == 0) return 0;
    const size_t nch = (bytes + RZE_CS - 1) / RZE_CS;
    uint8_t* scratch = (uint8_t*)malloc(nch * RZE_CS);
    uint32_t* sizes = (uint32_t*)malloc(nch * sizeof(uint32_t));
#pragma omp parallel for schedule(static)
    for (size_t c = 0; c < nch; c++) {
        size_t off = c * RZE_CS;
        int sz = (int)((bytes - off) < RZE_CS ? (bytes - off) : RZE_CS);
        sizes[c] = orc_rze_encode_chunk(in + off, sz, scratch + off);
    }
    uint32_t hdr[2] = {(uint32_t)bytes, (uint32_t)nch};
    memcpy(out, hdr, 8);
    memcpy(out + 8, sizes, 4 * nch);
    size_t pos = 8 + 4 * nch;
    for (size_t c = 0; c < nch; c++) {
        uint32_t s = sizes[c] & 0x7FFFFFFFu;
        memcpy(out + pos, scratch + c * RZE_CS, s);
        pos += s;
    }
    size_t total = (pos + 3) & ~(size_t)3; /* :617-624 */
    memset(out + pos, 0, total - pos);
    free(scratch);
    free(sizes);
    return total;
}

/* Sequential RE decode (rze_stage.cu:283-298). */
static void re_decode(int dec, const uint8_t* data, const uint8_t* bm, uint8_t* outb) {
    int pos = 0;
    uint8_t cur = 0;
    for (int i = 0; i < dec; i++) {
        if ((bm[i >> 3] >> (i & 7)) & 1) cur = data[pos++];
        outb[i] = cur;
    }
}

static int popcount_bytes(const uint8_t* a, int n) {
    int c = 0;
    for (int i = 0; i < n; i++) c += __builtin_popcount(a[i]);
    return c;
}

size_t orc_rze_decode(const uint8_t* in, size_t in_bytes, uint8_t* out, size_t out_cap) {
    if (in_bytes < 8) return (size_t)-1;
    uint32_t orig, nch;
    memcpy(&orig, in, 4);
    memcpy(&nch, in + 4, 4);
    if (orig == 0 || nch == 0) return 0;
    if (orig > out_cap || 8 + 4 * (size_t)nch > in_bytes) return (size_t)-1;
    if ((size_t)nch != ((size_t)orig + RZE_CS - 1) / RZE_CS) return (size_t)-1;
    const uint32_t* entries = (const uint32_t*)(in + 8);
    size_t* in_off = (size_t*)malloc(sizeof(size_t) * nch);
    size_t cur = 8 + 4 * (size_t)nch;
    for (uint32_t c = 0; c < nch; c++) {
        in_off[c] = cur;
        cur += entries[c] & 0x7FFFFFFFu;
    }
    int bad = cur > in_bytes;
    if (!bad) {
#pragma omp parallel for schedule(static)
        for (uint32_t c = 0; c < nch; c++) {
            const uint32_t e = entries[c];
            const uint32_t comp = e & 0x7FFFFFFFu;
            const size_t ooff = (size_t)c * RZE_CS;
            const int osz = (int)((c + 1 < nch) ? RZE_CS : orig - ooff);
            const uint8_t* src = in + in_off[c];
            uint8_t* dst = out + ooff;
            if (e & 0x80000000u) {
                memcpy(dst, src, (size_t)osz);
                continue;
            }
            if (comp <= 2) {
                memset(dst, 0, (size_t)osz);
                continue;
            }
            uint8_t bm1[RZE_CS / 8], bm2[RZE_CS / 64], bm3[RZE_CS / 512], bm4[RZE_BM4];
            const int b1 = (osz + 7) / 8, b2 = (b1 + 7) / 8, b3 = (b2 + 7) / 8;
            const int bm4_start = (int)comp - 2 - RZE_BM4;
            memcpy(bm4, src + bm4_start, RZE_BM4);
            const int n4 = popcount_bytes(bm4, RZE_BM4);
            const int s3 = bm4_start - n4;
            re_decode(b3, src + s3, bm4, bm3);
            const int n3 = popcount_bytes(bm3, b3);
            const int s2 = s3 - n3;
            re_decode(b2, src + s2, bm3, bm2);
            const int n2 = popcount_bytes(bm2, b2);
            const int s1 = s2 - n2;
            re_decode(b1, src + s1, bm2, bm1);
            int pos = 0;
            for (int i = 0; i < osz; i++)
                dst[i] = ((bm1[i >> 3] >> (i & 7)) & 1) ? src[pos++] : 0;
        }
    }
    free(in_off);
    return bad ? (size_t)-1 : orig;
}

/* ------------------------------------------------------------------ */
/* RLE                                                                 */
/* ------------------------------------------------------------------ */

static inline uint32_t ld_elem(const void* p, size_t i, int elem) {
    if (elem == 1) return ((const uint8_t*)p)[i];
    if (elem == 2) return ((const uint16_t*)p)[i];
    return ((const uint32_t*)p)[i];
}

size_t orc_rle_max_bytes(size_t n, int elem) {
    return 4 + ((n * (size_t)elem + 3) & ~(size_t)3) + 4 * n;
}

size_t orc_rle_encode(const void* in, size_t n, int elem, uint8_t* out) {
    if (n == 0) {
        memset(out, 0, 4);
        return 4;
    }
    uint32_t runs = 0;
    for (size_t i = 0; i < n; i++)
        if (i == 0 || ld_elem(in, i, elem) != ld_elem(in, i - 1, elem)) runs++;
    const size_t vbytes = (size_t)runs * elem, valigned = (vbytes + 3) & ~(size_t)3;
    memcpy(out, &runs, 4);
    uint8_t* vals = out + 4;
    uint32_t* lens = (uint32_t*)(out + 4 + valigned);
    memset(vals + vbytes, 0, valigned - vbytes);
    uint32_t r = 0;
    size_t start = 0;
    for (size_t i = 1; i <= n; i++) {
        if (i == n || ld_elem(in, i, elem) != ld_elem(in, i - 1, elem)) {
            uint32_t v = ld_elem(in, start, elem);
            memcpy(vals + (size_t)r * elem, &v, (size_t)elem);
            lens[r] = (uint32_t)(i - start);
            r++;
            start = i;
        }
    }
    return 4 + valigned + 4 * (size_t)runs;
}

size_t orc_rle_decode(const uint8_t* in, size_t in_bytes, int elem, void* out,
                      size_t out_cap) {
    if (in_bytes < 4) return (size_t)-1;
    uint32_t runs;
    memcpy(&runs, in, 4);
    const size_t vbytes = (size_t)runs * elem, valigned = (vbytes + 3) & ~(size_t)3;
    if (4 + valigned + 4 * (size_t)runs > in_bytes) return (size_t)-1;
    const uint8_t* vals = in + 4;
    const uint32_t* lens = (const uint32_t*)(in + 4 + valigned);
    size_t pos = 0;
    for (uint32_t r = 0; r < runs; r++) {
        uint32_t v = 0;
        memcpy(&v, vals + (size_t)r * elem, (size_t)elem);
        if (pos + lens[r] > out_cap) return (size_t)-1;
        for (uint32_t k = 0; k < lens[r]; k++, pos++) {
            if (elem == 1) ((uint8_t*)out)[pos] = (uint8_t)v;
            else if (elem == 2) ((uint16_t*)out)[pos] = (uint16_t)v;
            else ((uint32_t*)out)[pos] = v;
        }
    }
    return pos;
}

/* ------------------------------------------------------------------ */
/* Bitpack                                                             */
/* ------------------------------------------------------------------ */

int orc_bitpack_nbits_for_max(uint32_t max_val, int elem) {
    const int full = 8 * elem;
    for (int b = 1; b < full; b *= 2)
        if ((uint64_t)max_val < ((uint64_t)1 << b)) return b;
    return full;
}

size_t orc_bitpack_encode(const void* in, size_t n, int elem, int nbits, uint8_t* out) {
    const size_t nout = (n * (size_t)nbits + 7) / 8;
    if (nbits < 8) {
        const int per = 8 / nbits;
        const uint32_t mask = (1u << nbits) - 1u;
        for (size_t b = 0; b < nout; b++) {
            uint8_t packed = 0;
            for (int k = 0; k < per; k++) {
                size_t e = b * per + k;
                if (e < n) packed |= (uint8_t)((ld_elem(in, e, elem) & mask) << (k * nbits));
            }
            out[b] = packed;
        }
    } else {
        const int bytes = nbits / 8;
        for (size_t i = 0; i < n; i++) {
            uint32_t v = ld_elem(in, i, elem);
            if (nbits < 32) v &= (1u << nbits) - 1u;
            for (int b = 0; b < bytes; b++) out[i * bytes + b] = (uint8_t)(v >> (8 * b));
        }
    }
    return nout;
}

void orc_bitpack_decode(const uint8_t* in, size_t n, int elem, int nbits, void* out) {
    for (size_t i = 0; i < n; i++) {
        uint32_t v = 0;
        if (nbits < 8) {
            const int per = 8 / nbits;
            v = (in[i / per] >> ((i % per) * nbits)) & ((1u << nbits) - 1u);
        } else {
            for (int b = 0; b < nbits / 8; b++) v |= (uint32_t)in[i * (nbits / 8) + b] << (8 * b);
        }
        if (elem == 1) ((uint8_t*)out)[i] = (uint8_t)v;
        else if (elem == 2) ((uint16_t*)out)[i] = (uint16_t)v;
        else ((uint32_t*)out)[i] = v;
    }
}

/* ------------------------------------------------------------------ */
/* Huffman: histogram, codebook, coarse encode, decode                 */
/* ------------------------------------------------------------------ */

uint64_t orc_histogram(const uint16_t* in, size_t n, uint32_t bklen, uint32_t* freq) {
    memset(freq, 0, sizeof(uint32_t) * bklen);
    uint64_t counted = 0;
    for (size_t i = 0; i < n; i++)
        if (in[i] < bklen) {
            freq[in[i]]++;
            counted++;
        }
    return counted;
}

/* Tree node of the serial Huffman builder (hf_impl.hh:77-86). */
typedef struct hnode {
    struct hnode *left, *right;
    uint64_t freq;
    uint32_t sym;
} hnode;

/* 1-indexed binary min-heap with the reference's tie rules:
 * insert stops at a parent with freq <= new (hf_bk_impl1.cc:73-81); remove
 * moves the last node to the root and sinks it, preferring the right child
 * only when strictly smaller, swapping only when strictly larger (:83-106). */
typedef struct {
    hnode** q; /* q[1..end-1] */
    int end;
} hheap;

static void heap_insert(hheap* h, hnode* n) {
    int i = h->end++, j;
    while ((j = i >> 1)) {
        if (h->q[j]->freq <= n->freq) break;
        h->q[i] = h->q[j];
        i = j;
    }
    h->q[i] = n;
}

static hnode* heap_remove(hheap* h) {
    int i = 1, l;
    hnode* n = h->q[1];
    if (h->end < 2) return NULL;
    h->end--;
    h->q[1] = h->q[h->end];
    while ((l = i << 1) < h->end) {
        if (l + 1 < h->end && h->q[l + 1]->freq < h->q[l]->freq) l++;
        if (h->q[i]->freq > h->q[l]->freq) {
            hnode* p = h->q[i];
            h->q[i] = h->q[l];
            h->q[l] = p;
            i = l;
        } else
            break;
    }
    return n;
}

size_t orc_huff_revbook_bytes(uint32_t bklen) { return 4 * 32 * 2 + 2 * (size_t)bklen; }

int orc_huff_book(const uint32_t* freq, uint32_t bklen, uint32_t* bk4, uint8_t* revbook) {
    /* phf_CPU_build_codebook_v1<uint64_t> (hf_bk_impl1.cc:142-163) */
    hnode* pool = (hnode*)calloc(4 * (size_t)bklen + 2, sizeof(hnode));
    hheap h;
    h.q = (hnode**)calloc(4 * (size_t)bklen + 2, sizeof(hnode*));
    h.end = 1;
    int nn = 0;
    for (uint32_t i = 0; i < bklen; i++)
        if (freq[i]) {
            hnode* n = &pool[nn++];
            n->freq = freq[i];
            n->sym = i;
            heap_insert(&h, n);
        }
    while (h.end > 2) {
        /* new_node(tree, 0, 0, qremove(tree), qremove(tree)): with the
         * host compiler's right-to-left argument evaluation the first
         * removal (smallest) becomes the right child. */
        hnode* r = heap_remove(&h);
        hnode* l = heap_remove(&h);
        hnode* n = &pool[nn++];
        n->left = l;
        n->right = r;
        n->freq = l->freq + r->freq;
        heap_insert(&h, n);
    }
    uint64_t* bk8 = (uint64_t*)malloc(sizeof(uint64_t) * bklen);
    memset(bk8, 0xff, sizeof(uint64_t) * bklen);
    int rc = 0;
    if (h.end == 2) {
        /* iterative in-order traversal: left = 0, right = 1; depth limited
         * to 58 (hf_bk_internal.cc:59-101, hf_impl.hh:126) */
        hnode* stack[64];
        uint64_t spath[64], slen[64];
        int depth = 0;
        hnode* p = h.q[1];
        uint64_t code = 0, len = 0;
        for (;;) {
            if (p->left || p->right) {
                if (depth + 1 > 58) { rc = -1; break; }
                stack[depth] = p; spath[depth] = code; slen[depth] = len; depth++;
                p = p->left;
                code <<= 1;
                len += 1;
                if (len > 58) { rc = -1; break; }
            } else {
                /* book[sym] = code; bitcount field (bits 58..63) = len */
                uint64_t w = code;
                w = (w & ((1ull << 58) - 1)) | ((len & 63ull) << 58);
                bk8[p->sym] = w;
                if (depth == 0) break;
                depth--;
                p = stack[depth]->right;
                code = (spath[depth] << 1) | 1u;
                len = slen[depth] + 1;
                if (len > 58) { rc = -1; break; }
            }
        }
    }
    free(h.q);
    free(pool);
    if (rc) { free(bk8); return rc; }

    /* 64 -> 32-bit truncation (hf_bk.cc:104-122): length > 27 becomes the
     * outlier cutoff 28 with code 0 */
    for (uint32_t i = 0; i < bklen; i++) {
        if (bk8[i] == ~0ull) { bk4[i] = 0xffffffffu; continue; }
        uint32_t bits = (uint32_t)(bk8[i] >> 58);
        uint32_t code = (uint32_t)(bk8[i] & 0x7ffffffu);
        if (bits > 27) { bits = 28; code = 0; }
        bk4[i] = (bits << 27) | code;
    }
    free(bk8);

    /* canonize (hf_canon.cc:86-131) */
    int numl[32] = {0}, iterby[32] = {0}, first[32] = {0}, entry[32] = {0};
    uint16_t* keys = (uint16_t*)calloc(bklen, sizeof(uint16_t));
    uint32_t* canon = (uint32_t*)malloc(sizeof(uint32_t) * bklen);
    int max_l = 0;
    for (uint32_t i = 0; i < bklen; i++)
        if (bk4[i] != 0xffffffffu) {
            int l = (int)(bk4[i] >> 27);
            if (l > max_l) max_l = l;
            numl[l]++;
        }
    for (int i = 1; i < 32; i++) entry[i] = numl[i - 1];
    for (int i = 1; i < 32; i++) entry[i] += entry[i - 1];
    for (int i = 0; i < 32; i++) iterby[i] = entry[i];
    first[max_l] = 0;
    for (int l = max_l - 1; l >= 1; l--)
        first[l] = (int)((first[l + 1] + numl[l + 1]) / 2.0 + 0.5);
    first[0] = 0xff;
    for (uint32_t i = 0; i < bklen; i++) canon[i] = 0xffffffffu;
    uint32_t* obk = (uint32_t*)malloc(sizeof(uint32_t) * bklen);
    for (uint32_t i = 0; i < bklen; i++) obk[i] = 0xffffffffu;
    for (uint32_t i = 0; i < bklen; i++) {
        uint32_t c = bk4[i];
        uint32_t l = c >> 27;
        if (c != 0xffffffffu) {
            uint32_t v = (uint32_t)(first[l] + iterby[l] - entry[l]);
            canon[iterby[l]] = (v & 0x7ffffffu) | (l << 27);
            keys[iterby[l]] = (uint16_t)i;
            iterby[l]++;
        }
    }
    for (uint32_t i = 0; i < bklen; i++)
        if (canon[i] != 0xffffffffu) obk[keys[i]] = canon[i];
    memcpy(bk4, obk, sizeof(uint32_t) * bklen);
    memcpy(revbook, first, sizeof(first));
    memcpy(revbook + sizeof(first), entry, sizeof(entry));
    memcpy(revbook + 2 * sizeof(first), keys, sizeof(uint16_t) * bklen);
    free(keys);
    free(canon);
    free(obk);
    return 0;
}

#define HUFF_SUBLEN 768

size_t orc_huff_max_bytes(size_t n, uint32_t bklen) {
    size_t pardeg = n ? (n - 1) / HUFF_SUBLEN + 1 : 0;
    return 128 + orc_huff_revbook_bytes(bklen) + 8 * pardeg + 4 * (n + pardeg) + 16;
}

static inline uint32_t shl32(uint32_t x, uint32_t s) { return s >= 32 ? 0u : x << s; }
static inline uint32_t shr32(uint32_t x, uint32_t s) { return s >= 32 ? 0u : x >> s; }

/* Coarse mode partitions 768 symbols (hf_bk.cc:28-37).  Fine mode
 * (encode_mode = Fine, hf_buf.cc:46-49) partitions 1024: its ReVISIT-lite
 * kernel (hf_kernels.cu:145-250) packs each partition MSB-first into the same
 * cells the coarse deflate below produces, and when the longest code is over
 * 8 bits it runs this coarse deflate at sublen 1024 (hf_hl.cc:69-103). */
size_t orc_huff_encode(const uint16_t* in, size_t n, uint32_t bklen, const uint32_t* bk4,
                       const uint8_t* revbook, uint8_t* out) {
    return orc_huff_encode_sub(in, n, bklen, bk4, revbook, HUFF_SUBLEN, out);
}

size_t orc_huff_encode_sub(const uint16_t* in, size_t n, uint32_t bklen, const uint32_t* bk4,
                           const uint8_t* revbook, uint32_t sublen_, uint8_t* out) {
    const size_t SUB = sublen_;
    const size_t pardeg = (n - 1) / SUB + 1;
    uint32_t* nbit = (uint32_t*)malloc(4 * pardeg);
    uint32_t* ncell = (uint32_t*)malloc(4 * pardeg);
    uint32_t* entry = (uint32_t*)malloc(4 * pardeg);
    uint32_t* cells = (uint32_t*)calloc(n + 1, 4);
    /* phase 1 fill + phase 2 deflate per partition (hf_kernels.cu:59-122) */
#pragma omp parallel for schedule(static)
    for (size_t p = 0; p < pardeg; p++) {
        uint32_t* ptr = cells + p * SUB;
        int residue = 32, total = 0;
        uint32_t bufr = 0;
        size_t did = p * SUB;
        for (size_t i = 0; i < SUB && did < n; i++, did++) {
            uint32_t word = bk4[in[did]];
            uint32_t w = word >> 27;
            uint32_t code = word & 0x7ffffffu;
            if (residue == 32) bufr = 0;
            if ((int)w <= residue) {
                residue -= (int)w;
                bufr |= shl32(code, (uint32_t)residue);
                if (residue == 0) {
                    residue = 32;
                    *ptr++ = bufr;
                }
            } else {
                uint32_t lb = w - (uint32_t)residue, rb = 32 - lb;
                bufr |= shr32(code, lb);
                *ptr++ = bufr;
                bufr = shl32(code, rb);
                residue = (int)rb;
            }
            total += (int)w;
        }
        *ptr = bufr;
        nbit[p] = (uint32_t)total;
        ncell[p] = (uint32_t)((total + 31) / 32);
    }
    uint64_t total_nbit = 0, total_ncell = 0;
    for (size_t p = 0; p < pardeg; p++) {
        entry[p] = (uint32_t)total_ncell;
        total_nbit += nbit[p];
        total_ncell += ncell[p];
    }
    /* phf_header + layout (hf.h:38-44, hf_hl.cc:50-67) */
    const uint32_t rb = (uint32_t)orc_huff_revbook_bytes(bklen);
    uint32_t ent[6];
    ent[0] = 0;
    ent[1] = 128;
    ent[2] = ent[1] + rb;
    ent[3] = ent[2] + 4 * (uint32_t)pardeg;
    ent[4] = ent[3] + 4 * (uint32_t)pardeg;
    ent[5] = ent[4] + 4 * (uint32_t)total_ncell;
    memset(out, 0, 128);
    int32_t bkl = (int32_t)(bklen & 0xffff), sublen = (int32_t)SUB, pd = (int32_t)pardeg;
    uint64_t olen = n;
    memcpy(out + 0, &bkl, 4);
    memcpy(out + 4, &sublen, 4);
    memcpy(out + 8, &pd, 4);
    memcpy(out + 16, &olen, 8);
    memcpy(out + 24, &total_nbit, 8);
    memcpy(out + 32, &total_ncell, 8);
    memcpy(out + 40, ent, sizeof(ent));
    memcpy(out + ent[1], revbook, rb);
    memcpy(out + ent[2], nbit, 4 * pardeg);
    memcpy(out + ent[3], entry, 4 * pardeg);
    for (size_t p = 0; p < pardeg; p++)
        memcpy(out + ent[4] + 4 * (size_t)entry[p], cells + p * SUB, 4 * (size_t)ncell[p]);
    free(nbit);
    free(ncell);
    free(entry);
    free(cells);
    return ent[5];
}

size_t orc_huff_decode(const uint8_t* blob, size_t blob_bytes, uint16_t* out, size_t out_cap) {
    if (blob_bytes < 128) return 0;
    int32_t sublen, pardeg;
    uint64_t olen;
    uint32_t ent[6];
    memcpy(&sublen, blob + 4, 4);
    memcpy(&pardeg, blob + 8, 4);
    memcpy(&olen, blob + 16, 8);
    memcpy(ent, blob + 40, sizeof(ent));
    if (ent[5] > blob_bytes || olen > out_cap) return 0;
    const int32_t* first = (const int32_t*)(blob + ent[1]);
    const int32_t* entry = first + 32;
    const uint16_t* keys = (const uint16_t*)(blob + ent[1] + 256);
    const uint32_t* nbit = (const uint32_t*)(blob + ent[2]);
    const uint32_t* pent = (const uint32_t*)(blob + ent[3]);
    const uint32_t* bits = (const uint32_t*)(blob + ent[4]);
    const size_t ncells = (ent[5] - ent[4]) / 4;
    /* KERNEL_CUHIP_HF_decode single_thread_inflate (hf_kernels.cu:267-298) */
#pragma omp parallel for schedule(static)
    for (int32_t p = 0; p < pardeg; p++) {
        const uint32_t* input = bits + pent[p];
        size_t limit = ncells > pent[p] ? ncells - pent[p] : 0;
        uint16_t* o = out + (size_t)sublen * p;
        size_t ocap = out_cap > (size_t)sublen * p ? out_cap - (size_t)sublen * p : 0;
        uint32_t total = nbit[p];
        uint32_t i = 0, l = 1, idx_out = 0;
        uint32_t bufr = limit ? input[0] : 0;
        uint32_t v = (bufr >> 31) & 1u;
        while (i < total) {
            while (l < 32 && v < (uint32_t)first[l]) {
                ++i;
                uint32_t ib = i / 32, bi = i % 32;
                if (bi == 0) bufr = ib < limit ? input[ib] : 0;
                v = (v << 1) | ((bufr >> (31 - bi)) & 1u);
                ++l;
            }
            if (idx_out < ocap && l < 32) {
                int32_t k = entry[l] + (int32_t)v - first[l];
                o[idx_out] = keys[k];
            }
            idx_out++;
            ++i;
            uint32_t ib = i / 32, bi = i % 32;
            if (bi == 0) bufr = ib < limit ? input[ib] : 0;
            v = (bufr >> (31 - bi)) & 1u;
            l = 1;
        }
    }
    return (size_t)olen;
}

/* ------------------------------------------------------------------ */
/* CRC32                                                               */
/* ------------------------------------------------------------------ */

uint32_t orc_crc32(const void* data, size_t len) {
    static uint32_t table[256];
    static int init = 0;
    if (!init) {
        for (uint32_t i = 0; i < 256; i++) {
            uint32_t c = i;
            for (int k = 0; k < 8; k++) c = (c & 1u) ? (0xEDB88320u ^ (c >> 1)) : (c >> 1);
            table[i] = c;
        }
        init = 1;
    }
    const uint8_t* p = (const uint8_t*)data;
    uint32_t crc = 0xFFFFFFFFu;
    for (size_t i = 0; i < len; i++) crc = table[(crc ^ p[i]) & 0xFFu] ^ (crc >> 8);
    return crc ^ 0xFFFFFFFFu;
}

/* ------------------------------------------------------------------ */
/* Stages around the codes: Zigzag, Negabinary, Difference, integer    */
/* Lorenzo, the direct Quantizer (ABS / NOA)                           */
/* ------------------------------------------------------------------ */

static uint64_t ew_mask(int ew) { return ew == 8 ? ~0ull : ((1ull << (8 * ew)) - 1ull); }

static uint64_t ld_w(const void* p, size_t i, int ew) {
    switch (ew) {
        case 1: return ((const uint8_t*)p)[i];
        case 2: return ((const uint16_t*)p)[i];
        case 4: return ((const uint32_t*)p)[i];
        default: return ((const uint64_t*)p)[i];
    }
}

static void st_w(void* p, size_t i, int ew, uint64_t v) {
    switch (ew) {
        case 1: ((uint8_t*)p)[i] = (uint8_t)v; break;
        case 2: ((uint16_t*)p)[i] = (uint16_t)v; break;
        case 4: ((uint32_t*)p)[i] = (uint32_t)v; break;
        default: ((uint64_t*)p)[i] = v; break;
    }
}

/* zigzag.h:41-48: (x << 1) ^ (x >> (W-1)); decode (u >> 1) ^ -(u & 1). */
static uint64_t zz_enc(uint64_t u, int ew) {
    const uint64_t m = ew_mask(ew);
    const int sign = (int)((u >> (8 * ew - 1)) & 1u);
    return ((u << 1) ^ (sign ? m : 0)) & m;
}
static uint64_t zz_dec(uint64_t u, int ew) {
    const uint64_t m = ew_mask(ew);
    return ((u >> 1) ^ ((u & 1u) ? m : 0)) & m;
}
/* negabinary.h:43-52: (n + M) ^ M, decode (u ^ M) - M, M = 0xAA..AA. */
static uint64_t nb_enc(uint64_t u, int ew) {
    const uint64_t m = ew_mask(ew), M = 0xAAAAAAAAAAAAAAAAull & m;
    return ((u + M) & m) ^ M;
}
static uint64_t nb_dec(uint64_t u, int ew) {
    const uint64_t m = ew_mask(ew), M = 0xAAAAAAAAAAAAAAAAull & m;
    return ((u ^ M) - M) & m;
}

void orc_zigzag(const void* in, size_t n, int ew, int inverse, void* out) {
    for (size_t i = 0; i < n; i++) {
        const uint64_t u = ld_w(in, i, ew);
        st_w(out, i, ew, inverse ? zz_dec(u, ew) : zz_enc(u, ew));
    }
}

void orc_negabinary(const void* in, size_t n, int ew, int inverse, void* out) {
    for (size_t i = 0; i < n; i++) {
        const uint64_t u = ld_w(in, i, ew);
        st_w(out, i, ew, inverse ? nb_dec(u, ew) : nb_enc(u, ew));
    }
}

/* diff.cu:26-48 (forward) and :83-104 + :166-205 (chunked prefix sum). */
void orc_diff(const void* in, size_t n, int ew, size_t chunk, int nb, int inverse, void* out) {
    const uint64_t m = ew_mask(ew);
    uint64_t acc = 0;
    for (size_t i = 0; i < n; i++) {
        const int start = (i == 0) || (chunk && i % chunk == 0);
        const uint64_t x = ld_w(in, i, ew);
        if (!inverse) {
            const uint64_t d = start ? x : ((x - ld_w(in, i - 1, ew)) & m);
            st_w(out, i, ew, nb ? nb_enc(d, ew) : d);
        } else {
            const uint64_t v = nb ? nb_dec(x, ew) : x;
            acc = start ? v : ((acc + v) & m);
            st_w(out, i, ew, acc);
        }
    }
}

/* lorenzo_stage.cu: 1-D deltas inside 256-element blocks (:18-33) and their
 * block prefix sums (:38-58); 2-D / 3-D inclusion-exclusion over the field
 * (:100-118, :215-243) and prefix sums along x, y, z (:120-200, :245-375).
 * Elements past the 2-D / 3-D field are copied. */
void orc_lorenzo_int(const void* in, size_t n, size_t nx, size_t ny, size_t nz, int ew, int inverse, void* out) {
    const uint64_t m = ew_mask(ew);
    if (ny <= 1 && nz <= 1) {
        uint64_t acc = 0;
        for (size_t i = 0; i < n; i++) {
            const uint64_t x = ld_w(in, i, ew);
            if (!inverse) {
                st_w(out, i, ew, (i & 255) ? ((x - ld_w(in, i - 1, ew)) & m) : x);
            } else {
                acc = (i & 255) ? ((acc + x) & m) : x;
                st_w(out, i, ew, acc);
            }
        }
        return;
    }
    const size_t nf = nx * ny * nz, sy = nx, sz = nx * ny;
    for (size_t i = nf; i < n; i++) st_w(out, i, ew, ld_w(in, i, ew));
    if (!inverse) {
        for (size_t z = 0; z < nz; z++)
            for (size_t y = 0; y < ny; y++)
                for (size_t x = 0; x < nx; x++) {
                    const size_t i = z * sz + y * sy + x;
                    uint64_t v = ld_w(in, i, ew);
                    if (x) v -= ld_w(in, i - 1, ew);
                    if (y) v -= ld_w(in, i - sy, ew);
                    if (x && y) v += ld_w(in, i - sy - 1, ew);
                    if (z) {
                        v -= ld_w(in, i - sz, ew);
                        if (x) v += ld_w(in, i - sz - 1, ew);
                        if (y) v += ld_w(in, i - sz - sy, ew);
                        if (x && y) v -= ld_w(in, i - sz - sy - 1, ew);
                    }
                    st_w(out, i, ew, v & m);
                }
        return;
    }
    for (size_t i = 0; i < nf; i++) st_w(out, i, ew, ld_w(in, i, ew));
    for (size_t i = 0; i < nf; i++)
        if (i % nx) st_w(out, i, ew, (ld_w(out, i, ew) + ld_w(out, i - 1, ew)) & m);
    for (size_t i = 0; i < nf; i++)
        if ((i / nx) % ny) st_w(out, i, ew, (ld_w(out, i, ew) + ld_w(out, i - sy, ew)) & m);
    for (size_t i = sz; i < nf; i++) st_w(out, i, ew, (ld_w(out, i, ew) + ld_w(out, i - sz, ew)) & m);
}

/* __float2int_rn: round half to even, saturating, NaN -> 0. */
static int f2i_rn(float v) {
    if (isnan(v)) return 0;
    const float r = nearbyintf(v);
    if (r >= 2147483648.0f) return 2147483647;
    if (r < -2147483648.0f) return (-2147483647 - 1);
    return (int)r;
}

/* quantizer.cu:30-70 (forward ABS/NOA) with the outliers listed in index
 * order; returns the outlier total (only cap stored). */
size_t orc_quantizer_abs(const float* in, size_t n, int code_bytes, float ebx2_r, float threshold, uint32_t radius,
                         int zigzag, void* codes, float* ovals, uint32_t* oidx, size_t cap) {
    const int R = (int)(code_bytes == 2 ? (uint32_t)(uint16_t)radius : radius);
    size_t k = 0;
    for (size_t i = 0; i < n; i++) {
        const float x = in[i];
        const float p = x * ebx2_r;
        const int q = f2i_rn(p);
        uint64_t c = 0;
        if (q > -R && q < R && fabsf(x) < threshold) {
            const uint64_t u = (uint64_t)(int64_t)q & ew_mask(code_bytes);
            c = zigzag ? zz_enc(u, code_bytes) : u;
        } else {
            if (k < cap) {
                ovals[k] = x;
                oidx[k] = (uint32_t)i;
            }
            k++;
        }
        st_w(codes, i, code_bytes, c);
    }
    return k;
}

/* quantizer.cu:117-138 (inverse ABS/NOA) and the scatter
 * (predictor_utils.cuh:149-160). */
void orc_quantizer_abs_inv(const void* codes, size_t n, int code_bytes, float ebx2, int zigzag, const float* ovals,
                           const uint32_t* oidx, size_t nout, float* out) {
    for (size_t i = 0; i < n; i++) {
        uint64_t u = ld_w(codes, i, code_bytes);
        if (zigzag) u = zz_dec(u, code_bytes);
        const int q = code_bytes == 2 ? (int)(int16_t)(uint16_t)u : (int)(int32_t)(uint32_t)u;
        out[i] = (float)q * ebx2;
    }
    for (size_t k = 0; k < nout; k++)
        if (oidx[k] < n) out[oidx[k]] = ovals[k];
}

/* quantizer.cu:83-107 / :147-167: in-place outliers, u32 codes. */
void orc_quantizer_inplace(const float* in, size_t n, float ebx2_r, float threshold, uint32_t radius,
                           uint32_t* codes) {
    const int R = (int)radius;
    for (size_t i = 0; i < n; i++) {
        const float x = in[i];
        const int q = f2i_rn(x * ebx2_r);
        if (q > -R && q < R && fabsf(x) < threshold) {
            codes[i] = ((uint32_t)q << 1) ^ (uint32_t)(q >> 31);
        } else {
            memcpy(&codes[i], &x, 4);
        }
    }
}

void orc_quantizer_inplace_inv(const uint32_t* codes, size_t n, float ebx2, uint32_t radius, float* out) {
    for (size_t i = 0; i < n; i++) {
        const uint32_t c = codes[i];
        if ((c >> 1) >= radius) {
            memcpy(&out[i], &c, 4);
        } else {
            const int32_t ci = (int32_t)c;
            const int q = (ci & 1) ? -((ci + 1) >> 1) : (ci >> 1);
            out[i] = (float)q * ebx2;
        }
    }
}
