// fzm.cpp -- FZM helpers: CRC32 and the type-name tables.
#include <array>
#include <stdexcept>

#include "fz/fzm_format.h"

namespace fz {

namespace {

const std::array<uint32_t, 256>& crc_table() {
    static const std::array<uint32_t, 256> t = [] {
        std::array<uint32_t, 256> tab{};
        for (uint32_t i = 0; i < 256; i++) {
            uint32_t c = i;
            for (int k = 0; k < 8; k++) c = (c >> 1) ^ ((c & 1u) ? 0xEDB88320u : 0u);
            tab[i] = c;
        }
        return tab;
    }();
    return t;
}

}  // namespace

uint32_t crc32Update(uint32_t crc, const void* data, size_t len) {
    const auto& t = crc_table();
    const uint8_t* p = static_cast<const uint8_t*>(data);
    for (size_t i = 0; i < len; i++) crc = t[(crc ^ p[i]) & 0xFFu] ^ (crc >> 8);
    return crc;
}

size_t getDataTypeSize(DataType t) {
    switch (t) {
        case DataType::UINT8:
        case DataType::INT8: return 1;
        case DataType::UINT16:
        case DataType::INT16: return 2;
        case DataType::UINT32:
        case DataType::INT32:
        case DataType::FLOAT32: return 4;
        case DataType::UINT64:
        case DataType::INT64:
        case DataType::FLOAT64: return 8;
        default: throw std::runtime_error("Unknown data type");
    }
}

std::string dataTypeToString(DataType t) {
    static const char* names[] = {"uint8", "uint16", "uint32", "uint64", "int8",
                                  "int16", "int32",  "int64",  "float32", "float64"};
    const unsigned i = (unsigned)t;
    return i < 10 ? names[i] : "unknown";
}

std::string stageTypeToString(StageType t) {
    switch (t) {
        case StageType::LORENZO_QUANT: return "LorenzoQuant";
        case StageType::DIFFERENCE: return "Difference";
        case StageType::SCALE: return "Scale";
        case StageType::PASSTHROUGH: return "PassThrough";
        case StageType::RLE: return "RLE";
        case StageType::HUFFMAN: return "Huffman";
        case StageType::BITPACK: return "BitPack";
        case StageType::SPLIT: return "Split";
        case StageType::MERGE: return "Merge";
        case StageType::QUANTIZER: return "Quantizer";
        case StageType::ZIGZAG: return "Zigzag";
        case StageType::NEGABINARY: return "Negabinary";
        case StageType::BITSHUFFLE: return "Bitshuffle";
        case StageType::RZE: return "RZE";
        case StageType::LORENZO: return "Lorenzo";
        default: return "Unknown";
    }
}

}  // namespace fz
