// Alenka on-disk segment format: reader and writer.
//
// Byte layout (little endian, packed), per column per segment, file
// "<table>.<column>.<segment>" (char columns: "<table>.<column>.<segment>.idx"):
//   u32 cnt | i64 lower | i64 upper | u32 comp_type | payload[cnt] |
//   u32 cnt | u32 rec_count | u32 bits | i64 orig_lower | u32 fit_count | i64 start_val
// Writer follows pfor_compress (compress.cu:413-527) and pfor_delta_compress
// (compress.cu:271-408); reader follows pfor_decompress (compress.cu:180-190).
// Column header "<table>.<column>.header": u64 total | u32 segs | u32 max_recs |
// u32 max_cnt (CudaSet::writeHeader, cm.cu:1251-1263).
// Char columns: dictionary file "<table>.<column>" (fixed width strings in code
// order), "<seg>.idx" (FOR-encoded codes) and "<seg>.hash" (u32 n + n x i64
// MurmurHash64A(value)/2), per CudaSet::compress_char (cm.cu:1765-1844).
// Catalog "data.dictionary": save_col_data / load_col_data (cm.cu:4057-4114).
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace alk {

struct SegMeta {
  uint32_t cnt = 0;        // payload bytes
  int64_t lower = 0;       // header min (FOR) or first value (delta)
  int64_t upper = 0;       // header max (FOR) or last value (delta)
  uint32_t comp_type = 0;  // 0 = FOR, 1 = FOR-delta
  uint32_t rec_count = 0;
  uint32_t bits = 0;       // FOR: 8/16/32/64; delta: packed width 1..64
  int64_t orig_lower = 0;  // value added back on decode
  uint32_t fit_count = 0;  // values per u64 word
  int64_t start_val = 0;   // delta: first value
};

constexpr size_t kSegHeadBytes = 24;   // cnt, lower, upper, comp_type
constexpr size_t kSegTailBytes = 32;   // cnt, rec_count, bits, orig_lower, fit_count, start_val

// Parse an in-memory segment file image. Returns false with err on malformed input.
bool parse_segment(const uint8_t* buf, size_t len, SegMeta& m, const uint8_t** payload,
                   std::string& err);
bool read_file(const std::string& path, std::vector<uint8_t>& out, std::string& err);
bool write_file(const std::string& path, const void* data, size_t len, bool append = false);

// Encoders (host). encode_for: min-subtract and byte-aligned width (compress.cu:413-527).
// encode_delta: adjacent difference, min-subtract, MSB-first bit packing (compress.cu:271-408).
void encode_for(const int64_t* v, uint32_t n, SegMeta& m, std::vector<uint8_t>& payload);
void encode_delta(const int64_t* v, uint32_t n, SegMeta& m, std::vector<uint8_t>& payload);
std::vector<uint8_t> segment_image(const SegMeta& m, const std::vector<uint8_t>& payload);
// Packed width of a value range as the reference computes it (double-precision log2);
// shared by the host and the device segment writers so both pick the same width.
uint32_t range_bits(int64_t lo, int64_t hi);

struct ColHeader {
  uint64_t total = 0;
  uint32_t segs = 0, max_recs = 0, max_cnt = 0;
};
bool read_col_header(const std::string& path, ColHeader& h, std::string& err);
bool write_col_header(const std::string& path, const ColHeader& h);

// MurmurHash64A (64-bit MurmurHash2 by Austin Appleby), as used at
// MurmurHash2_64.cu:201-242 with seed hash_seed=100 (bison.y:304).
uint64_t murmur64a(const void* key, int len, uint32_t seed);
constexpr uint32_t kHashSeed = 100;

struct ColData {
  uint32_t col_type = 0;    // 0 int/decimal/timestamp, 1 float, 2 char
  uint32_t col_length = 0;  // decimal: implied digits; char: width; timestamp: UINT32_MAX
};
using DataDict = std::map<std::string, std::map<std::string, ColData>>;
bool load_data_dict(const std::string& path, DataDict& dd, std::string& err);
bool save_data_dict(const std::string& path, const DataDict& dd);

// Table writer: writes one table in the reference's layout (numeric FOR or delta, char
// dictionary columns) and registers it in the catalog. Used by the generators.
struct ColumnSpec {
  std::string name;
  int kind = 0;             // 0 int, 1 decimal, 2 char
  uint32_t decimals = 0;    // for decimal
  uint32_t width = 0;       // for char
  bool delta = false;       // write FOR-delta when the segment is sorted (the -delta flag)
};
class TableWriter {
 public:
  TableWriter(std::string dir, std::string table, std::vector<ColumnSpec> cols);
  // numeric: one int64 vector per numeric column; chars: one fixed-width buffer per char column
  // (rows x width bytes), given in column order over all columns (unused entries empty).
  bool write_segment(const std::vector<const int64_t*>& ints,
                     const std::vector<const char*>& chars, uint32_t rows, std::string& err);
  bool finish(DataDict& dd, std::string& err);

 private:
  std::string dir_, table_;
  std::vector<ColumnSpec> cols_;
  uint32_t segs_ = 0, max_recs_ = 0;
  uint64_t total_ = 0;
  std::vector<uint32_t> max_cnt_;
  std::vector<std::map<uint64_t, int64_t>> dict_;  // per char column: hash/2 -> code
};

}  // namespace alk
