// Test infrastructure: exposes the reference's own host Huffman codebook
// builder (phf_CPU_build_canonized_codebook_v2, modules/coders/huffman/phf/
// hf_bk.cc:84-140) through a C symbol so the oracle's restatement can be
// checked against it.  Linked only into oracle/_ref/libref_hfbook.so.
#include <cstdint>
#include <cstring>
#include <vector>
#include "hf_impl.hh"

extern "C" int ref_huff_book(const uint32_t* freq, int bklen, uint32_t* bk4,
                             uint8_t* revbook) {
    std::vector<uint32_t> f(freq, freq + bklen);
    try {
        phf_CPU_build_canonized_codebook_v2<uint16_t, uint32_t>(
            f.data(), bklen, bk4, revbook, nullptr);
    } catch (...) {
        return -1;
    }
    return 0;
}
