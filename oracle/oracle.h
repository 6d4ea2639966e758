// ORACLE — test infrastructure only. A CPU restatement of Alenka's scan -> filter
// -> join -> group-by -> order operators (operators.cu, filter.cu, zone_map.cu,
// select.cu, merge.cu, sorts.cu, cm.cu, compress.cu of antonmks/Alenka), used as the
// parity checker by tests/, __graft_entry__.smoke() and bench.py's CPU baseline.
// Nothing in the product links or calls this code.
//
// Parity pin: the codec and hash functions are pinned against the reference's own
// compress.cu / MurmurHash2_64.cu compiled from source (oracle/build_ref.sh ->
// oracle/_ref); the operator semantics follow the reference's source line by line
// (cited per function) and are cross-checked by the golden fixtures under
// tests/golden/. The reference has no tests or golden outputs of its own.
#pragma once
#include <cstddef>
#include <cstdint>

extern "C" {
// Run a script against the tables in dir (data.dictionary + segment files). STORE
// output files are written relative to dir. Returns 0 on success.
int oracle_execute(const char* dir, const char* script, int threads, char* err, int err_len);
// Decode one segment file image into int64 values (pfor_decompress, compress.cu:180-267).
// Returns the row count, or -1 on a malformed image.
int64_t oracle_decode_segment(const uint8_t* image, size_t len, int64_t* out, size_t out_cap);
/* 1 when the fixed-width entry matches the NUL-terminated LIKE pattern (gpu_regex,
 * filter.cu:67-129). */
int oracle_like(const char* entry, uint32_t width, const char* pattern);
uint64_t oracle_murmur64a(const void* key, int len, uint32_t seed);
// Rows scanned by the last oracle_execute (fact rows of every segment visited).
uint64_t oracle_rows_scanned(void);
}
