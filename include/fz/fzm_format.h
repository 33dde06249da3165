// fz/fzm_format.h -- FZM v3.1 container layout (the reference's on-disk
// format, include/fzm_format.h:22-262, reproduced field for field so files
// written here and there are interchangeable).
//
//   [FZMHeaderCore, 80 B][FZMStageInfo x num_stages, 256 B each]
//   [FZMBufferEntry x num_buffers, 256 B each][payload segments, unpadded]
//
// All integers little-endian, structs naturally aligned (the static_asserts
// pin the sizes).  data_checksum = CRC32 (IEEE, reflected 0xEDB88320) of the
// payload; header_checksum = CRC32 of core + stage + buffer records with the
// header_checksum field zeroed.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <string>

namespace fz {

constexpr uint32_t FZM_MAGIC = 0x464D5A32u;  // "2ZMF" in memory order
constexpr uint8_t FZM_VERSION_MAJOR = 3;
constexpr uint8_t FZM_VERSION_MINOR = 1;
constexpr uint16_t FZM_VERSION = (uint16_t)((FZM_VERSION_MAJOR << 8) | FZM_VERSION_MINOR);
constexpr size_t FZM_LEGACY_HEADER_CORE_SIZE = 72;  // v3.0 core (no checksums)
constexpr uint16_t FZM_FLAG_HAS_DATA_CHECKSUM = 0x0001u;
constexpr uint16_t FZM_FLAG_HAS_HEADER_CHECKSUM = 0x0002u;

constexpr size_t FZM_MAX_BUFFERS = 32;
constexpr size_t FZM_MAX_NAME_LEN = 64;
constexpr size_t FZM_STAGE_CONFIG_SIZE = 128;
constexpr size_t FZM_MAX_SOURCES = 4;
constexpr size_t FZM_MAX_STAGE_INPUTS = 8;
constexpr size_t FZM_MAX_STAGE_OUTPUTS = 8;

// Pre-3.0 files stored a bare major number.
constexpr uint8_t fzmVersionMajor(uint16_t v) { return v <= 0xFF ? (uint8_t)v : (uint8_t)(v >> 8); }
constexpr uint8_t fzmVersionMinor(uint16_t v) { return v <= 0xFF ? 0 : (uint8_t)(v & 0xFF); }

// Stage type ids written into the container (fzm_format.h:71-88).
enum class StageType : uint16_t {
    UNKNOWN = 0,
    LORENZO_QUANT = 1,
    DIFFERENCE = 2,
    SCALE = 3,
    PASSTHROUGH = 4,
    RLE = 5,
    HUFFMAN = 6,
    BITPACK = 7,
    SPLIT = 10,
    MERGE = 11,
    LORENZO = 12,
    QUANTIZER = 14,
    ZIGZAG = 15,
    NEGABINARY = 16,
    BITSHUFFLE = 17,
    RZE = 18,
};

enum class DataType : uint8_t {
    UINT8 = 0,
    UINT16 = 1,
    UINT32 = 2,
    UINT64 = 3,
    INT8 = 4,
    INT16 = 5,
    INT32 = 6,
    INT64 = 7,
    FLOAT32 = 8,
    FLOAT64 = 9,
    UNKNOWN = 0xFF,  // byte-transparent stages: no type check at finalize()
};


struct FZMStageInfo {
    StageType stage_type;
    uint16_t stage_version;
    uint8_t num_inputs;
    uint8_t num_outputs;
    uint16_t reserved1;
    uint16_t input_buffer_ids[FZM_MAX_STAGE_INPUTS];    // 0xFFFF = unused
    uint16_t output_buffer_ids[FZM_MAX_STAGE_OUTPUTS];  // 0xFFFF = unused
    uint8_t stage_config[FZM_STAGE_CONFIG_SIZE];
    uint32_t config_size;
    uint8_t reserved2[84];

    FZMStageInfo() {
        std::memset(static_cast<void*>(this), 0, sizeof(*this));
        std::memset(input_buffer_ids, 0xFF, sizeof(input_buffer_ids));
        std::memset(output_buffer_ids, 0xFF, sizeof(output_buffer_ids));
    }
};
static_assert(sizeof(FZMStageInfo) == 256, "FZMStageInfo is 256 bytes");

struct FZMBufferEntry {
    StageType stage_type;
    uint16_t stage_version;
    DataType data_type;
    uint8_t producer_output_idx;
    uint16_t dag_buffer_id;  // 0xFFFF = unassigned
    char name[FZM_MAX_NAME_LEN];
    uint64_t data_size;
    uint64_t allocated_size;
    uint64_t uncompressed_size;
    uint64_t byte_offset;
    uint8_t stage_config[FZM_STAGE_CONFIG_SIZE];
    uint32_t config_size;
    uint8_t reserved2[14];

    FZMBufferEntry() {
        std::memset(static_cast<void*>(this), 0, sizeof(*this));
        dag_buffer_id = 0xFFFF;
    }
};
static_assert(sizeof(FZMBufferEntry) == 256, "FZMBufferEntry is 256 bytes");

struct FZMHeaderCore {
    uint32_t magic;
    uint16_t version;
    uint16_t num_buffers;
    uint64_t uncompressed_size;
    uint64_t compressed_size;
    uint64_t header_size;
    uint32_t num_stages;
    uint16_t num_sources;
    uint16_t flags;
    uint64_t source_uncompressed_sizes[FZM_MAX_SOURCES];
    uint32_t data_checksum;
    uint32_t header_checksum;

    FZMHeaderCore() {
        std::memset(static_cast<void*>(this), 0, sizeof(*this));
        magic = FZM_MAGIC;
        version = FZM_VERSION;
        header_size = sizeof(FZMHeaderCore);
    }
    uint64_t computeHeaderSize() const {
        return sizeof(FZMHeaderCore) + (uint64_t)num_stages * sizeof(FZMStageInfo) +
               (uint64_t)num_buffers * sizeof(FZMBufferEntry);
    }
};
static_assert(sizeof(FZMHeaderCore) == 80, "FZMHeaderCore is 80 bytes");

size_t getDataTypeSize(DataType t);  // throws on UNKNOWN
std::string dataTypeToString(DataType t);
std::string stageTypeToString(StageType t);

// CRC32 (IEEE 802.3, reflected polynomial 0xEDB88320), incremental form:
// crc = crc32Update(0xFFFFFFFF, ...) ... ^ 0xFFFFFFFF.
uint32_t crc32Update(uint32_t crc, const void* data, size_t len);
inline uint32_t crc32(const void* data, size_t len) { return crc32Update(0xFFFFFFFFu, data, len) ^ 0xFFFFFFFFu; }

}  // namespace fz
