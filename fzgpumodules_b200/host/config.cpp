// config.cpp -- Pipeline::loadConfig / saveConfig (src/pipeline/config.cpp:
// 515-640 and the per-stage readers and writers above them): TOML files with
// a [pipeline] table and one [[stage]] table per stage, connected by
// `inputs = [{from = "...", port = "..."}]`; the reference's keys, defaults,
// type names and error messages.  The parser reads the part of TOML these
// files use: comments, [table], [[array of tables]], key = value with basic
// strings, integers, floats (inf / nan included), booleans, arrays (possibly
// over several lines) and inline tables.
#include <cctype>
#include <cmath>
#include <cstring>
#include <cstdint>
#include <fstream>
#include <iomanip>
#include <limits>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "fz/pipeline.h"
#include "fz/stages.h"

namespace fz {
namespace {

struct TVal {
    enum Kind { None, Str, Int, Flt, Bool, Arr, Tab } kind = None;
    std::string s;
    int64_t i = 0;
    double f = 0;
    bool b = false;
    std::vector<TVal> arr;
    std::map<std::string, TVal> tab;
    const TVal* get(const std::string& k) const {
        auto it = tab.find(k);
        return it == tab.end() ? nullptr : &it->second;
    }
};

[[noreturn]] void fail(const std::string& m) { throw std::runtime_error(m); }

struct Parser {
    std::string t;
    size_t p = 0;
    std::string path;
    void ws(bool nl) {
        for (;;) {
            while (p < t.size() && (t[p] == ' ' || t[p] == '\t' || t[p] == '\r' || (nl && t[p] == '\n'))) p++;
            if (p < t.size() && t[p] == '#') {
                while (p < t.size() && t[p] != '\n') p++;
                continue;
            }
            return;
        }
    }
    [[noreturn]] void err(const std::string& m) {
        size_t line = 1;
        for (size_t k = 0; k < p && k < t.size(); k++) line += t[k] == '\n';
        fail("loadConfig: failed to parse \"" + path + "\": " + m + " (line " + std::to_string(line) + ")");
    }
    std::string key() {
        ws(false);
        if (p < t.size() && t[p] == '"') return str();
        size_t b = p;
        while (p < t.size() && (isalnum((unsigned char)t[p]) || t[p] == '_' || t[p] == '-')) p++;
        if (b == p) err("expected a key");
        return t.substr(b, p - b);
    }
    std::string str() {
        p++;  // opening quote
        std::string r;
        while (p < t.size() && t[p] != '"') {
            if (t[p] == '\\' && p + 1 < t.size()) {
                const char c = t[++p];
                r += c == 'n' ? '\n' : c == 't' ? '\t' : c;
            } else {
                r += t[p];
            }
            p++;
        }
        if (p >= t.size()) err("unterminated string");
        p++;
        return r;
    }
    TVal value() {
        ws(false);
        TVal v;
        if (p >= t.size()) err("expected a value");
        const char c = t[p];
        if (c == '"') {
            v.kind = TVal::Str;
            v.s = str();
        } else if (c == '[') {
            v.kind = TVal::Arr;
            p++;
            for (;;) {
                ws(true);
                if (p < t.size() && t[p] == ']') { p++; break; }
                v.arr.push_back(value());
                ws(true);
                if (p < t.size() && t[p] == ',') { p++; continue; }
                if (p < t.size() && t[p] == ']') { p++; break; }
                err("expected ',' or ']'");
            }
        } else if (c == '{') {
            v.kind = TVal::Tab;
            p++;
            for (;;) {
                ws(false);
                if (p < t.size() && t[p] == '}') { p++; break; }
                const std::string k = key();
                ws(false);
                if (p >= t.size() || t[p] != '=') err("expected '='");
                p++;
                v.tab[k] = value();
                ws(false);
                if (p < t.size() && t[p] == ',') { p++; continue; }
                if (p < t.size() && t[p] == '}') { p++; break; }
                err("expected ',' or '}'");
            }
        } else {
            size_t b = p;
            while (p < t.size() && !strchr(",]}\n#\r \t", t[p])) p++;
            std::string w = t.substr(b, p - b);
            std::string d;
            for (char ch : w) if (ch != '_') d += ch;
            if (d == "true" || d == "false") {
                v.kind = TVal::Bool;
                v.b = d == "true";
            } else if (d == "inf" || d == "+inf" || d == "-inf" || d == "nan" || d == "+nan" || d == "-nan") {
                v.kind = TVal::Flt;
                v.f = d.find("nan") != std::string::npos ? std::numeric_limits<double>::quiet_NaN()
                                                          : (d[0] == '-' ? -1.0 : 1.0) * INFINITY;
            } else if (d.find_first_of(".eE") != std::string::npos) {
                v.kind = TVal::Flt;
                size_t used = 0;
                try { v.f = std::stod(d, &used); } catch (...) { used = 0; }
                if (d.empty() || used != d.size()) err("bad number \"" + w + "\"");
            } else {
                v.kind = TVal::Int;
                size_t used = 0;
                try { v.i = std::stoll(d, &used, 10); } catch (...) { used = 0; }
                if (d.empty() || used != d.size()) err("bad value \"" + w + "\"");
            }
        }
        return v;
    }
    TVal document() {
        TVal root;
        root.kind = TVal::Tab;
        TVal* cur = &root;
        for (;;) {
            ws(true);
            if (p >= t.size()) break;
            if (t[p] == '[') {
                const bool aot = p + 1 < t.size() && t[p + 1] == '[';
                p += aot ? 2 : 1;
                const std::string k = key();
                ws(false);
                if (t.compare(p, aot ? 2 : 1, aot ? "]]" : "]") != 0) err("expected ']'");
                p += aot ? 2 : 1;
                TVal& slot = root.tab[k];
                if (aot) {
                    slot.kind = TVal::Arr;
                    slot.arr.emplace_back();
                    slot.arr.back().kind = TVal::Tab;
                    cur = &slot.arr.back();
                } else {
                    slot.kind = TVal::Tab;
                    cur = &slot;
                }
                continue;
            }
            const std::string k = key();
            ws(false);
            if (p >= t.size() || t[p] != '=') err("expected '='");
            p++;
            cur->tab[k] = value();
            ws(false);  // a value ends its line (a comment may follow)
            if (p < t.size() && t[p] != '\n') err("expected the end of the line after the value of '" + k + "'");
        }
        return root;
    }
};

std::string opt_str(const TVal& t, const char* k, const char* d) {
    const TVal* v = t.get(k);
    return v && v->kind == TVal::Str ? v->s : d;
}
int64_t opt_int(const TVal& t, const char* k, int64_t d) {
    const TVal* v = t.get(k);
    return v && v->kind == TVal::Int ? v->i : v && v->kind == TVal::Flt ? (int64_t)v->f : d;
}
double opt_dbl(const TVal& t, const char* k, double d) {
    const TVal* v = t.get(k);
    return v && v->kind == TVal::Flt ? v->f : v && v->kind == TVal::Int ? (double)v->i : d;
}
bool opt_bool(const TVal& t, const char* k, bool d) {
    const TVal* v = t.get(k);
    return v && v->kind == TVal::Bool ? v->b : d;
}

DataType dtype_of(const std::string& s) {
    static const std::map<std::string, DataType> m = {
        {"uint8", DataType::UINT8}, {"uint16", DataType::UINT16}, {"uint32", DataType::UINT32},
        {"uint64", DataType::UINT64}, {"int8", DataType::INT8}, {"int16", DataType::INT16},
        {"int32", DataType::INT32}, {"int64", DataType::INT64}, {"float32", DataType::FLOAT32},
        {"float64", DataType::FLOAT64}};
    auto it = m.find(s);
    if (it == m.end()) fail("loadConfig: unknown data type \"" + s + "\"");
    return it->second;
}

const char* dtype_name(uint8_t d) {
    switch ((DataType)d) {
        case DataType::UINT8: return "uint8";
        case DataType::UINT16: return "uint16";
        case DataType::UINT32: return "uint32";
        case DataType::UINT64: return "uint64";
        case DataType::INT8: return "int8";
        case DataType::INT16: return "int16";
        case DataType::INT32: return "int32";
        case DataType::INT64: return "int64";
        case DataType::FLOAT32: return "float32";
        case DataType::FLOAT64: return "float64";
        default: return "uint8";
    }
}

ErrorBoundMode eb_mode_of(const std::string& s) {
    if (s == "ABS") return ErrorBoundMode::ABS;
    if (s == "REL") return ErrorBoundMode::REL;
    if (s == "NOA") return ErrorBoundMode::NOA;
    fail("loadConfig: unknown error_bound_mode \"" + s + "\"");
}

MemoryStrategy strategy_of(const std::string& s) {
    if (s == "PREALLOCATE") return MemoryStrategy::PREALLOCATE;
    if (s == "MINIMAL") return MemoryStrategy::MINIMAL;
    fail("loadConfig: unknown memory_strategy \"" + s + "\"");
}

HuffmanEncodeMode huffman_mode_of(const std::string& s) {
    if (s == "Fine") return HuffmanEncodeMode::Fine;
    if (s == "Coarse") return HuffmanEncodeMode::Coarse;
    fail("loadConfig: unknown Huffman encode_mode \"" + s + "\"");
}

std::string toml_escape(const std::string& s) {
    std::string o;
    for (char c : s) {
        if (c == '\\' || c == '"') o += '\\';
        o += c;
    }
    return o;
}
const char* eb_mode_name(ErrorBoundMode m) {
    return m == ErrorBoundMode::REL ? "REL" : m == ErrorBoundMode::NOA ? "NOA" : "ABS";
}

template <typename S>
S* add_quant(Pipeline& p, const TVal& t) {
    typename S::Config c;
    c.error_bound = (float)opt_dbl(t, "error_bound", 1e-3);
    c.eb_mode = eb_mode_of(opt_str(t, "error_bound_mode", "REL"));
    c.quant_radius = (int)opt_int(t, "quant_radius", 32768);
    c.outlier_capacity = (float)opt_dbl(t, "outlier_capacity", 0.05);
    c.zigzag_codes = opt_bool(t, "zigzag_codes", true);
    c.inplace_outliers = opt_bool(t, "inplace_outliers", false);
    c.outlier_threshold = (float)opt_dbl(t, "outlier_threshold", INFINITY);
    return p.addStage<S>(c);
}

Stage* add_stage(Pipeline& p, const TVal& t, const std::string& type) {
    if (type == "LorenzoQuant") {
        if (opt_str(t, "input_type", "float32") != "float32" || opt_str(t, "code_type", "uint16") != "uint16")
            fail("loadConfig: unsupported Lorenzo type combination input_type=\"" + opt_str(t, "input_type", "float32") +
                 "\" code_type=\"" + opt_str(t, "code_type", "uint16") + "\"");
        LorenzoQuantStage<float, uint16_t>::Config c;
        c.error_bound = (float)opt_dbl(t, "error_bound", 1e-3);
        c.quant_radius = (int)opt_int(t, "quant_radius", 32768);
        c.outlier_capacity = (float)opt_dbl(t, "outlier_capacity", 0.2);
        c.eb_mode = eb_mode_of(opt_str(t, "error_bound_mode", "ABS"));
        c.zigzag_codes = opt_bool(t, "zigzag_codes", false);
        return p.addStage<LorenzoQuantStage<float, uint16_t>>(c);
    }
    if (type == "Quantizer") {
        const std::string code = opt_str(t, "code_type", "uint32");
        if (opt_str(t, "input_type", "float32") != "float32" || (code != "uint16" && code != "uint32"))
            fail("loadConfig: unsupported Quantizer type combination input_type=\"" +
                 opt_str(t, "input_type", "float32") + "\" code_type=\"" + code + "\"");
        if (code == "uint16") return add_quant<QuantizerStage<float, uint16_t>>(p, t);
        return add_quant<QuantizerStage<float, uint32_t>>(p, t);
    }
    if (type == "Lorenzo") {
        switch (dtype_of(opt_str(t, "data_type", "int32"))) {
            case DataType::INT8: return p.addStage<LorenzoStage<int8_t>>();
            case DataType::INT16: return p.addStage<LorenzoStage<int16_t>>();
            case DataType::INT32: return p.addStage<LorenzoStage<int32_t>>();
            case DataType::INT64: return p.addStage<LorenzoStage<int64_t>>();
            default: fail("loadConfig: unsupported Lorenzo data_type \"" + opt_str(t, "data_type", "int32") + "\"");
        }
    }
    if (type == "Bitshuffle") {
        auto* s = p.addStage<BitshuffleStage>();
        s->setBlockSize((size_t)opt_int(t, "block_size", 16384));
        s->setElementWidth((size_t)opt_int(t, "element_width", 4));
        return s;
    }
    if (type == "RZE") {
        auto* s = p.addStage<RZEStage>();
        s->setChunkSize((size_t)opt_int(t, "chunk_size", 16384));
        s->setLevels((int)opt_int(t, "levels", 4));
        return s;
    }
    if (type == "RLE") {
        switch (dtype_of(opt_str(t, "data_type", "uint16"))) {
            case DataType::UINT8: return p.addStage<RLEStage<uint8_t>>();
            case DataType::UINT16: return p.addStage<RLEStage<uint16_t>>();
            case DataType::UINT32: return p.addStage<RLEStage<uint32_t>>();
            case DataType::INT32: return p.addStage<RLEStage<int32_t>>();
            default: fail("loadConfig: unsupported RLE data_type \"" + opt_str(t, "data_type", "uint16") + "\"");
        }
    }
    if (type == "Difference") {
        const DataType a = dtype_of(opt_str(t, "input_type", "float32"));
        const std::string os = opt_str(t, "output_type", "");
        const DataType b = os.empty() ? a : dtype_of(os);
        const size_t cs = (size_t)opt_int(t, "chunk_size", 0);
        auto mk = [&](auto* s) -> Stage* {
            s->setChunkSize(cs);
            return s;
        };
        if (a == DataType::INT8 && b == DataType::UINT8) return mk(p.addStage<DifferenceStage<int8_t, uint8_t>>());
        if (a == DataType::INT16 && b == DataType::UINT16) return mk(p.addStage<DifferenceStage<int16_t, uint16_t>>());
        if (a == DataType::INT32 && b == DataType::UINT32) return mk(p.addStage<DifferenceStage<int32_t, uint32_t>>());
        if (a == DataType::INT64 && b == DataType::UINT64) return mk(p.addStage<DifferenceStage<int64_t, uint64_t>>());
        if (a == b) {
            switch (a) {
                case DataType::UINT8: return mk(p.addStage<DifferenceStage<uint8_t>>());
                case DataType::UINT16: return mk(p.addStage<DifferenceStage<uint16_t>>());
                case DataType::UINT32: return mk(p.addStage<DifferenceStage<uint32_t>>());
                case DataType::INT32: return mk(p.addStage<DifferenceStage<int32_t>>());
                case DataType::INT64: return mk(p.addStage<DifferenceStage<int64_t>>());
                default: break;
            }
        }
        fail("loadConfig: unsupported Difference type combination");
    }
    if (type == "Zigzag" || type == "Negabinary") {
        const bool nb = type == "Negabinary";
        switch (dtype_of(opt_str(t, "input_type", "int32"))) {
            case DataType::INT8:
                return nb ? (Stage*)p.addStage<NegabinaryStage<int8_t, uint8_t>>() : p.addStage<ZigzagStage<int8_t, uint8_t>>();
            case DataType::INT16:
                return nb ? (Stage*)p.addStage<NegabinaryStage<int16_t, uint16_t>>()
                          : p.addStage<ZigzagStage<int16_t, uint16_t>>();
            case DataType::INT32:
                return nb ? (Stage*)p.addStage<NegabinaryStage<int32_t, uint32_t>>()
                          : p.addStage<ZigzagStage<int32_t, uint32_t>>();
            case DataType::INT64:
                return nb ? (Stage*)p.addStage<NegabinaryStage<int64_t, uint64_t>>()
                          : p.addStage<ZigzagStage<int64_t, uint64_t>>();
            default: fail("loadConfig: unsupported " + type + " input_type");
        }
    }
    if (type == "Bitpack") {
        const uint8_t nb = (uint8_t)opt_int(t, "nbits", 16);
        switch (dtype_of(opt_str(t, "input_type", "uint16"))) {
            case DataType::UINT8: { auto* s = p.addStage<BitpackStage<uint8_t>>(); s->setNBits(nb); return s; }
            case DataType::UINT16: { auto* s = p.addStage<BitpackStage<uint16_t>>(); s->setNBits(nb); return s; }
            case DataType::UINT32: { auto* s = p.addStage<BitpackStage<uint32_t>>(); s->setNBits(nb); return s; }
            default: fail("loadConfig: unsupported Bitpack input_type");
        }
    }
    if (type == "Huffman") {
        auto* s = p.addStage<HuffmanStage<uint16_t>>();
        s->setBklen((uint32_t)opt_int(t, "bklen", 1024));
        s->setEncodeMode(huffman_mode_of(opt_str(t, "encode_mode", "Coarse")));
        return s;
    }
    fail("loadConfig: unknown stage type \"" + type + "\"");
}

template <typename S>
bool save_quant(Stage* st, std::ostringstream& o, const char* code) {
    auto* s = dynamic_cast<S*>(st);
    if (!s) return false;
    o << "input_type = \"float32\"\ncode_type = \"" << code << "\"\n"
      << "error_bound = " << (double)s->getErrorBound() << "\nerror_bound_mode = \"" << eb_mode_name(s->getErrorBoundMode())
      << "\"\nquant_radius = " << (int64_t)s->getQuantRadius() << "\noutlier_capacity = " << (double)s->getOutlierCapacity()
      << "\nzigzag_codes = " << (s->getZigzagCodes() ? "true" : "false") << "\n";
    const float th = s->getOutlierThreshold();
    if (std::isfinite(th)) o << "outlier_threshold = " << th << "\n";  // only a finite threshold is written
    if (s->getInplaceOutliers()) o << "inplace_outliers = true\n";
    return true;
}

// The fields of one [[stage]] table after its name and type, in the order and
// number format of the reference's writers (src/pipeline/config.cpp:250-395):
// types from the stage's own header or data types, optional keys only when
// they differ from the loader's defaults.
void save_stage_fields(Stage* st, std::ostringstream& o) {
    const auto type = (StageType)st->getStageTypeId();
    auto in_t = [&] { return dtype_name(st->getInputDataType(0)); };
    auto out_t = [&] { return dtype_name(st->getOutputDataType(0)); };
    switch (type) {
        case StageType::LORENZO_QUANT: {
            auto* s = dynamic_cast<LorenzoQuantStage<float, uint16_t>*>(st);
            if (!s) fail("saveConfig: no TOML form for stage " + st->getName());
            o << "input_type = \"float32\"\ncode_type = \"uint16\"\nerror_bound = " << (double)s->getErrorBound()
              << "\nerror_bound_mode = \"" << eb_mode_name(s->getErrorBoundMode())
              << "\"\nquant_radius = " << (int64_t)s->getQuantRadius() << "\noutlier_capacity = "
              << (double)s->getOutlierCapacity() << "\nzigzag_codes = " << (s->getZigzagCodes() ? "true" : "false")
              << "\n";
            return;
        }
        case StageType::QUANTIZER:
            if (save_quant<QuantizerStage<float, uint16_t>>(st, o, "uint16")) return;
            if (save_quant<QuantizerStage<float, uint32_t>>(st, o, "uint32")) return;
            fail("saveConfig: no TOML form for stage " + st->getName());
        case StageType::BITSHUFFLE: {
            auto* s = static_cast<BitshuffleStage*>(st);
            o << "block_size = " << (int64_t)s->getBlockSize() << "\nelement_width = " << (int64_t)s->getElementWidth()
              << "\n";
            return;
        }
        case StageType::RZE: {
            auto* s = static_cast<RZEStage*>(st);
            o << "chunk_size = " << (int64_t)s->getChunkSize() << "\nlevels = " << (int64_t)s->getLevels() << "\n";
            return;
        }
        case StageType::RLE: o << "data_type = \"" << out_t() << "\"\n"; return;
        case StageType::LORENZO: o << "data_type = \"" << out_t() << "\"\n"; return;
        case StageType::ZIGZAG:
        case StageType::NEGABINARY:
            o << "input_type = \"" << in_t() << "\"\noutput_type = \"" << out_t() << "\"\n";
            return;
        case StageType::DIFFERENCE: {
            o << "input_type = \"" << in_t() << "\"\noutput_type = \"" << out_t() << "\"\n";
            uint8_t hdr[8] = {};
            if (st->serializeHeader(0, hdr, sizeof(hdr)) >= 6) {
                uint32_t v;
                std::memcpy(&v, hdr + 2, 4);
                o << "chunk_size = " << (int64_t)v << "\n";
            }
            return;
        }
        case StageType::BITPACK: {
            uint8_t hdr[10] = {};
            const size_t n = st->serializeHeader(0, hdr, sizeof(hdr));
            o << "input_type = \"" << dtype_name(n >= 1 ? hdr[0] : (uint8_t)DataType::UINT16) << "\"\nnbits = "
              << (int64_t)(n >= 2 ? hdr[1] : 16) << "\n";
            return;
        }
        case StageType::HUFFMAN: {
            uint8_t hdr[16] = {};
            const size_t n = st->serializeHeader(0, hdr, sizeof(hdr));
            uint16_t bklen = 1024;
            if (n >= 3) std::memcpy(&bklen, hdr + 1, 2);
            o << "input_type = \"" << dtype_name(n >= 1 ? hdr[0] : (uint8_t)DataType::UINT16) << "\"\nbklen = "
              << (int64_t)bklen << "\n";
            auto* s = dynamic_cast<HuffmanStage<uint16_t>*>(st);
            if (s && s->getEncodeMode() == HuffmanEncodeMode::Fine) o << "encode_mode = \"Fine\"\n";
            return;
        }
        default: fail("saveConfig: no TOML form for stage " + st->getName());
    }
}

const char* stage_type_name(StageType t) {
    switch (t) {
        case StageType::LORENZO: return "Lorenzo";
        case StageType::LORENZO_QUANT: return "LorenzoQuant";
        case StageType::QUANTIZER: return "Quantizer";
        case StageType::BITSHUFFLE: return "Bitshuffle";
        case StageType::RZE: return "RZE";
        case StageType::RLE: return "RLE";
        case StageType::DIFFERENCE: return "Difference";
        case StageType::ZIGZAG: return "Zigzag";
        case StageType::NEGABINARY: return "Negabinary";
        case StageType::BITPACK: return "Bitpack";
        case StageType::HUFFMAN: return "Huffman";
        default: return "Unknown";
    }
}

}  // namespace

void Pipeline::loadConfig(const std::string& path) {
    if (finalized_) fail("loadConfig: pipeline is already finalized");
    std::ifstream f(path);
    if (!f) fail("loadConfig: failed to parse \"" + path + "\": cannot open file");
    std::stringstream ss;
    ss << f.rdbuf();
    Parser ps;
    ps.t = ss.str();
    ps.path = path;
    const TVal doc = ps.document();
    if (const TVal* pl = doc.get("pipeline")) {
        if (const TVal* v = pl->get("input_size"); v && v->kind == TVal::Int) input_size_hint_ = (size_t)v->i;
        if (const TVal* v = pl->get("dims"); v && v->kind == TVal::Arr) {
            std::array<size_t, 3> d = {0, 1, 1};
            for (size_t k = 0; k < 3 && k < v->arr.size(); k++)
                if (v->arr[k].kind == TVal::Int) d[k] = (size_t)v->arr[k].i;
            setDims(d);
        }
        if (const TVal* v = pl->get("memory_strategy"); v && v->kind == TVal::Str)
            setMemoryStrategy(strategy_of(v->s));
        if (const TVal* v = pl->get("pool_multiplier"); v && (v->kind == TVal::Flt || v->kind == TVal::Int))
            pool_multiplier_ = v->kind == TVal::Flt ? (float)v->f : (float)v->i;
        if (const TVal* v = pl->get("num_streams"); v && v->kind == TVal::Int) setNumStreams((int)v->i);
    }
    const TVal* arr = doc.get("stage");
    if (!arr || arr->kind != TVal::Arr || arr->arr.empty())
        fail("loadConfig: no [[stage]] entries found in \"" + path + "\"");
    std::map<std::string, Stage*> by_name;
    std::vector<std::pair<Stage*, const TVal*>> entries;
    for (const TVal& t : arr->arr) {
        const TVal* n = t.get("name");
        const TVal* ty = t.get("type");
        if (!n || !ty || n->kind != TVal::Str || ty->kind != TVal::Str)
            fail("loadConfig: each [[stage]] must have 'name' and 'type'");
        if (by_name.count(n->s)) fail("loadConfig: duplicate stage name \"" + n->s + "\"");
        Stage* s = add_stage(*this, t, ty->s);
        by_name[n->s] = s;
        entries.push_back({s, &t});
    }
    for (const auto& e : entries) {
        const TVal* ins = e.second->get("inputs");
        if (!ins || ins->kind != TVal::Arr || ins->arr.empty()) continue;  // a source stage
        const std::string name = e.second->get("name")->s;
        for (const TVal& in : ins->arr) {
            const TVal* from = in.get("from");
            if (!from || from->kind != TVal::Str)
                fail("loadConfig: stage \"" + name + "\" input missing 'from' key");
            auto it = by_name.find(from->s);
            if (it == by_name.end())
                fail("loadConfig: stage \"" + name + "\" references unknown stage \"" + from->s + "\"");
            const TVal* port = in.get("port");
            connect(e.first, it->second, port && port->kind == TVal::Str ? port->s : "output");
        }
    }
    finalize();
}

void Pipeline::saveConfig(const std::string& path) const {
    if (!finalized_) fail("saveConfig: pipeline must be finalized first");
    std::map<const Stage*, std::string> names;
    std::map<std::string, int> counts;
    for (const auto& s : stages_) {
        const std::string base = s->getName();
        const int k = counts[base]++;
        names[s.get()] = k == 0 ? base : base + std::to_string(k);
    }
    std::ostringstream o;
    o << "# FZGPUModules pipeline config\n"
      << "# Generated by Pipeline::saveConfig(). Load with Pipeline::loadConfig().\n\n";
    o << "[pipeline]\ninput_size = " << (int64_t)input_size_hint_ << "\nmemory_strategy = \""
      << (strategy_ == MemoryStrategy::PREALLOCATE ? "PREALLOCATE" : "MINIMAL") << "\"\n";
    o << std::setprecision(std::numeric_limits<double>::max_digits10);
    o << "pool_multiplier = " << (double)pool_multiplier_ << "\nnum_streams = " << (int64_t)num_streams_
      << "\ndims = [" << (int64_t)dims_[0] << ", " << (int64_t)dims_[1] << ", " << (int64_t)dims_[2] << "]\n\n";
    for (const auto& s : stages_) {
        o << "[[stage]]\nname = \"" << toml_escape(names[s.get()]) << "\"\ntype = \""
          << stage_type_name((StageType)s->getStageTypeId()) << "\"\n";
        save_stage_fields(s.get(), o);
        bool any = false;
        for (const auto& c : connections_) {
            if (c.dependent != s.get()) continue;
            o << (any ? ", " : "inputs = [") << "{ from = \"" << toml_escape(names[c.producer]) << "\"";
            if (c.output_name != "output") o << ", port = \"" << toml_escape(c.output_name) << "\"";
            o << " }";
            any = true;
        }
        if (any) o << "]\n";
        o << "\n";
    }
    std::ofstream f(path);
    if (!f) fail("saveConfig: cannot open \"" + path + "\" for writing");
    f << o.str();
    if (!f) fail("saveConfig: write error on \"" + path + "\"");
}

}  // namespace fz
