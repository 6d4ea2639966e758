/*
 * alenka_b200 — C ABI of the B200 (sm_100a) engine for Alenka's columnar
 * scan -> filter -> join -> group-by -> order path.
 *
 * Two layers, both plain C (pointers, sizes, status codes):
 *   1. The embedding API a host program binds, with the reference's names and
 *      meaning (alenka.h:30-35): alenkaInit / alenkaExecute / alenkaClose /
 *      execute_file, plus explicit-session variants (alk_session_*).
 *   2. Operator-level entry points, one per reference operator on the path. The
 *      engine behind layer 1 reaches the GPU only through these.
 * Every call is asynchronous on the given stream unless it returns a host value;
 * status 0 = OK. Device pointers are device memory the caller owns unless noted.
 */
#ifndef ALENKA_B200_H
#define ALENKA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* alk_stream; /* a cudaStream_t; NULL = legacy default stream */

/* ---------------------------------------------------------------- status */
#define ALK_OK 0
#define ALK_ERR_ARG 1         /* invalid argument */
#define ALK_ERR_CUDA 2        /* CUDA runtime error (context still usable) */
#define ALK_ERR_OVERFLOW 3    /* output capacity too small; the required size is returned */
#define ALK_ERR_TIMEOUT 4     /* a bounded device wait expired */
#define ALK_ERR_UNSUPPORTED 5 /* script form outside the supported surface */
#define ALK_ERR_IO 6          /* missing or malformed segment / catalog file */
#define ALK_ERR_PARSE 7       /* script syntax error */
#define ALK_ERR_NOMEM 8       /* device allocation failed */
#define ALK_ERR_TOO_LARGE 9   /* input exceeds a fixed-size entry point's stated maximum */

/* ------------------------------------------------- 1. embedding (alenka.h) */
/* alenkaInit (alenka.h:30): reads the flags of execute_file (bison.y:306-331) from
 * av (NULL-terminated); the data directory is the current directory. */
void alenkaInit(char** av);
/* alenkaExecute (alenka.h:31, bison.y:469-515): runs one script; 0 = success. */
int alenkaExecute(char* s);
/* alenkaClose (alenka.h:32): releases the engine. */
void alenkaClose(void);
/* execute_file (alenka.h:35, bison.y:295-455): alenka [-l MB] [-v] script.sql */
int execute_file(int ac, char** av);

/* Explicit sessions: the same engine with a chosen data directory. */
typedef struct alk_session alk_session;
/* flags: ALK_SESSION_RESIDENT keeps every loaded column segment in device memory
 * across scripts (the reference's -i buffers, cm.cu:616-656, one level further). */
#define ALK_SESSION_RESIDENT 1u
#define ALK_SESSION_PLAIN 2u    /* operator-at-a-time plan only (no fused pipelines) */
#define ALK_SESSION_NOGRAPH 4u  /* fused queries are never captured into CUDA graphs */
#define ALK_SESSION_DELTA 8u    /* STORE BINARY writes sorted columns FOR-delta (the
                                   reference's delta switch, compress.cu:428-444) */
int alk_session_open(const char* data_dir, uint32_t flags, alk_session** out);
int alk_session_execute(alk_session* s, const char* script);
const char* alk_session_error(alk_session* s);
alk_stream alk_session_stream(alk_session* s);
/* Pre-load (and pin in device memory) every column of a catalog table. */
int alk_session_preload(alk_session* s, const char* table);
/* Statistics of the last script: fact rows scanned, device kernels launched, bytes
 * copied host->device and device->host, and the plan used (0 plain, 1 fused, 2 fused and
 * replayed from the CUDA graph captured on an earlier run of the same script). */
typedef struct alk_stats {
  uint64_t rows_scanned;
  uint64_t kernels;
  uint64_t h2d_bytes;
  uint64_t d2h_bytes;
  uint32_t plan;
  uint32_t segments_skipped;
  double hot_kernel_ms;      /* device time of the dominant kernel (CUDA events) */
  uint64_t hot_kernel_bytes; /* algorithmic bytes that kernel moves */
  uint64_t hot_kernel_launches;
  double query_device_ms;    /* device time of the fused query (events around its device work) */
  uint64_t reserved_bytes;   /* survivor-list and hash-table bytes the fused stages reserved */
  uint32_t card_estimates;   /* fused stages sized by the learned estimator */
  uint32_t card_reruns;      /* fused query runs repeated because a size was too small */
  double batch_host_ms[3];   /* batches: wall time of planning, the batched launch, the rest */
  uint32_t sort_groupbys;    /* group-bys that took the sort-based form */
  uint32_t hash_groupbys;    /* group-bys fused with their filter into one hashed pass */
} alk_stats;
int alk_session_stats(alk_session* s, alk_stats* out);
/* Enable CUDA-event timing of the dominant kernel (adds two event records per launch). */
int alk_session_set_timing(alk_session* s, int on);
void alk_session_close(alk_session* s);

/* ------------------------------------------------- 2. operator entry points */

/* One column of one segment as it sits in device memory. FOR columns keep the
 * on-disk width (bits 8/16/32/64, value = stored + lower); delta columns are first
 * expanded with alk_decode_segment and then described with bits=64, lower=0.
 * Kernels read whole 16-byte units: data must stay readable up to the next multiple
 * of 16 bytes past rows * bits / 8 (the session loaders pad every payload by 256
 * bytes), and the fused stages stage 16-byte aligned columns through shared memory
 * with bulk copies (unaligned columns take a direct-load kernel instead). */
typedef struct alk_colseg {
  const void* data;
  int64_t lower;
  uint32_t rows;
  uint32_t bits;
} alk_colseg;

/* Arrays of device pointers (const int64_t* const* d_cols and the like) are HOST
 * arrays holding device addresses. */

/* Segment decode, replaces pfor_decompress (compress.cu:180-267): FOR (comp_type 0)
 * widening and FOR-delta (comp_type 1) MSB-first bit unpacking + prefix sum. d_payload
 * must be 16-byte aligned and readable up to a multiple of 16 bytes. */
int alk_decode_segment(const void* d_payload, uint32_t comp_type, uint32_t bits,
                       uint32_t fit_count, int64_t lower, int64_t start_val, uint32_t rows,
                       int64_t* d_out, alk_stream stream);

/* Segment decode that allocates nothing. No counterpart in the reference: this entry point
 * exists for callers that cannot call cudaMalloc, for example a host that has committed
 * all device memory to its own pools or a decode path that must never fail or stall on
 * an allocation.
 * Same arguments and results as alk_decode_segment. FOR segments need no scratch; a
 * FOR-delta segment keeps its scan state in one fixed device array of the library
 * (about 0.6 MB per device, held until the process exits), so at most 67,108,864 rows
 * (32768 tiles of 2048 rows) per call: larger segments return ALK_ERR_TOO_LARGE without
 * touching the device. The first call on each device looks up that array's device
 * address (cudaGetSymbolAddress) and keeps it, so make that first call before any stream
 * capture, and do not reset the device (cudaDeviceReset) after it.
 * Every call on a device shares the array: calls that overlap on the GPU (concurrent
 * streams, or threads sharing a device) race and must be serialized by the caller. */
int alk_decode_segment_noalloc(const void* d_payload, uint32_t comp_type, uint32_t bits,
                               uint32_t fit_count, int64_t lower, int64_t start_val, uint32_t rows,
                               int64_t* d_out, alk_stream stream);

/* Segment writer (host): one segment file image for n int64 values, FOR or (delta != 0
 * and sorted values) FOR-delta, laid out as pfor_compress / pfor_delta_compress write it
 * (compress.cu:271-527). ALK_ERR_OVERFLOW with *out_len set when cap is too small. */
int alk_encode_segment(const int64_t* values, uint32_t n, int delta, uint8_t* out, size_t cap,
                       size_t* out_len);
/* Segment writer (device): the same image as alk_encode_segment, built on the device
 * from n int64 values in device memory into d_image (device memory, 8-byte aligned):
 * the GPU form of pfor_compress / pfor_delta_compress (compress.cu:271-527) behind
 * CudaSet::Store's binary branch (cm.cu:1040-1240). mode 0 FOR, 1 FOR-delta, 2 FOR-delta
 * when the values are sorted (the reference's delta switch, compress.cu:428-444), else
 * FOR. *h_len = the image size; ALK_ERR_OVERFLOW when cap is too small (with *h_len a
 * size that suffices). d_image holds working statistics until the header is written;
 * nothing is allocated. Returns after the image is complete (stream synchronized). */
int alk_encode_segment_device(const int64_t* d_values, uint32_t n, int mode, void* d_image, size_t cap,
                              size_t* h_len, alk_stream stream);
/* Segment writer (device), many segments per call: segment i is n[i] values at
 * d_values[i] written into d_images[i] (device memory, 8-byte aligned, caps[i] bytes, at
 * least 24 + 8 n[i] + 32: the image is written before its size is known). The same images
 * as alk_encode_segment_device, for all segments with four launches and one stream
 * synchronisation; h_lens[i] = the image size. Host arrays of count entries. Used by
 * STORE ... BINARY for all columns of a result at once (cm.cu:1040-1240). */
int alk_encode_segments_device(const int64_t* const* d_values, const uint32_t* n, uint32_t count, int mode,
                               void* const* d_images, const size_t* caps, size_t* h_lens, alk_stream stream);

/* MurmurHash64A of n tuples of k int64 keys (row-major tuples built from k column
 * pointers), seed as given (hash_seed 100, bison.y:304). Replaces the host loop of
 * add() (merge.cu:118-141) and MurmurHash64A (MurmurHash2_64.cu:201-242). */
int alk_hash_tuples(const int64_t* const* d_cols, uint32_t k, uint64_t n, uint32_t seed,
                    uint64_t* d_out, alk_stream stream);

/* Predicate / expression program: a register machine over int64 values that the host
 * compiles from the reference's postfix queues (filter.cu:133-643, select.cu:359-800,
 * cm.cu:2250-2655). Operands are registers, columns (slots) or constants. */
#define ALK_MAX_INSTR 48
#define ALK_MAX_CONST 48
#define ALK_MAX_REGS 8
enum {
  ALK_OP_ADD = 1, ALK_OP_SUB, ALK_OP_MUL, ALK_OP_DIV,
  ALK_OP_LT, ALK_OP_GT, ALK_OP_LE, ALK_OP_GE, ALK_OP_EQ, ALK_OP_NE,
  ALK_OP_AND, ALK_OP_OR, ALK_OP_MOV,
  /* a in a set of codes: b is a constant holding a device pointer to uint32 words, word 0
   * the set's size n in bits, then the bits; 1 when 0 <= a < n and bit a is set. The
   * LIKE of a char column compiles to it (filter.cu:454-500: the dictionary entries
   * that match, then each row's code looked up). */
  ALK_OP_INSET
};
enum { ALK_K_REG = 0, ALK_K_COL = 1, ALK_K_CONST = 2 };
typedef struct alk_instr {
  uint8_t op, dst, ka, kb;
  uint16_t a, b;
  uint32_t pad;
} alk_instr;
typedef struct alk_program {
  uint32_t n_instr;
  uint32_t result; /* register holding the result */
  alk_instr ins[ALK_MAX_INSTR];
  int64_t consts[ALK_MAX_CONST];
} alk_program;

/* LIKE over a char column's dictionary (gpu_regex, filter.cu:67-129, run over the
 * dictionary file as filter.cu:454-500 does): entry k of `count` fixed-width entries at
 * d_dict (device) matches the pattern ('%' any run, '?' any character but '.', others
 * themselves; pattern_len < 256). d_bits (device, 1 + ceil(count / 32) words) receives
 * count in word 0 and bit k set for each match: the set ALK_OP_INSET tests. */
int alk_like_dictionary(const char* d_dict, uint32_t width, uint64_t count, const char* pattern,
                        uint32_t pattern_len, uint32_t* d_bits, alk_stream stream);
/* d_out[i] = d_table[d_codes[i]] for codes in [0, table_n), else -1: a char column's
 * dictionary codes mapped to their entries' ranks in byte order, which ORDER BY sorts
 * (update_char_permutation cm.cu:4218 sorts the strings themselves; the order is the
 * same). */
int alk_code_lookup(const int64_t* d_codes, uint64_t n, const int64_t* d_table, uint64_t table_n, int64_t* d_out,
                    alk_stream stream);

/* Fused segment scan, replaces filter_op + filter + copyColumns/mygather
 * (cm.cu:3609-3666, filter.cu:133-643, cm.cu:3305-3478): for every segment whose
 * zone-map verdict (seg_mode: 0 skip 'N', 1 all rows 'A', 2 evaluate 'R',
 * zone_map.cu:720) asks for it, decode the predicate columns, run the predicate and
 * write the surviving rows' out_cols (decoded to int64) in segment/row order.
 * cols is a host array [ncols][nseg]; out_cols lists column slots to emit; out_rowid
 * (optional) receives the row's index within its segment and out_seg (optional) its
 * segment. seg_counts (optional, device, nseg) receives the per-segment survivors.
 * Returns the survivor count in *h_count; if it exceeds cap nothing past cap is written
 * and ALK_ERR_OVERFLOW is returned. Synchronizes the stream. */
int alk_scan_filter(const alk_colseg* cols, uint32_t ncols, uint32_t nseg,
                    const uint8_t* seg_mode, const alk_program* pred,
                    const uint32_t* out_cols, uint32_t nout, int64_t* const* d_out,
                    uint32_t* d_out_rowid, uint32_t* d_out_seg, uint64_t* d_seg_counts,
                    uint64_t cap, uint64_t* h_count, alk_stream stream);

/* Expression evaluation over materialized columns, replaces CudaSet::op chains
 * (cm.cu:2440-2773) as driven by select() (select.cu:700-800). Asynchronous on the
 * stream (d_cols is read before the call returns). */
int alk_eval(const int64_t* const* d_cols, uint32_t ncols, uint64_t n, const alk_program* prog,
             int64_t* d_out, alk_stream stream);

/* Hash group-by with exact int64 aggregates, replaces order_inplace + GroupBy +
 * segreduce (operators.cu:367-406, cm.cu:910-956, select.cu:499-675).
 * aggs: per value column ALK_AGG_*; COUNT ignores its column (may be NULL).
 * Outputs (device, capacity n): group keys [nkeys][G], aggregates [nvals][G], and the
 * first input row of each group (smallest row index). Group order is unspecified;
 * *h_groups receives G. Synchronizes the stream. */
enum { ALK_AGG_SUM = 0, ALK_AGG_COUNT = 1, ALK_AGG_MIN = 2, ALK_AGG_MAX = 3 };
/* Sort-based group-by, the reference's own form (stable sort on the keys, head flags,
 * segmented reduction: operators.cu:367-406, select.cu:499-675), for key spaces too large
 * for a hash table sized by the rows to pay: the input is first checked for key order
 * (lexicographic, signed) and sorted (stable LSD radix) only when it is not; groups come
 * out in key order. Same arguments and outputs as alk_groupby_hash; *h_was_sorted (may be
 * NULL) = 1 when no sort was needed. Synchronizes the stream. */
int alk_groupby_sort(const int64_t* const* d_keys, uint32_t nkeys, const int64_t* const* d_vals,
                     const uint8_t* aggs, uint32_t nvals, uint64_t n, int64_t* const* d_out_keys,
                     int64_t* const* d_out_vals, uint32_t* d_out_first, uint64_t* h_groups, int* h_was_sorted,
                     alk_stream stream);
int alk_groupby_hash(const int64_t* const* d_keys, uint32_t nkeys, const int64_t* const* d_vals,
                     const uint8_t* aggs, uint32_t nvals, uint64_t n, int64_t* const* d_out_keys,
                     int64_t* const* d_out_vals, uint32_t* d_out_first, uint64_t* h_groups,
                     alk_stream stream);

/* Stable multi-key sort permutation, replaces update_permutation (sorts.cu:18-70) as
 * used by emit_order (operators.cu:1754-1763) and order_inplace: keys[0] is the most
 * significant; desc[i] != 0 sorts key i descending; ties keep input order. Writes the
 * permutation (input row index per output position) to d_perm. Synchronizes. */
int alk_sort_perm(const int64_t* const* d_keys, const uint8_t* desc, uint32_t nkeys, uint64_t n,
                  uint32_t* d_perm, alk_stream stream);
/* Same for unsigned 64-bit keys (hash order of merge.cu:147-149). */
int alk_sort_perm_u64(const uint64_t* d_key, uint64_t n, uint32_t* d_perm, alk_stream stream);

/* Gather, replaces thrust::gather in mygather / apply_permutation (cm.cu:3350,
 * sorts.cu:87): d_out[i] = d_src[d_idx[i]]. */
int alk_gather(const int64_t* d_src, const uint32_t* d_idx, uint64_t n, int64_t* d_out,
               alk_stream stream);
/* Join forms of emit_multijoin beyond the single-key inner join (operators.cu:1288-1399):
 * d_flags[i] = lcol[pl[i]] == rcol[pr[i]] (!= when neq), the AND-ed key pair test on the
 * pairs a join found; d_flags[rows[i]] = value, the left or right rows a semi or anti
 * join keeps; and, per segment g of a concatenation (rows [h_start[g], h_start[g+1]) of
 * d_keys), the least and greatest key into h_out[2g], h_out[2g+1] (INT64_MAX /
 * INT64_MIN for an empty segment), for the anti join's per-segment range test
 * (operators.cu:1215-1220). The last synchronises. alk_gather_u32 is alk_gather for u32
 * row indices (pairs compacted by an AND-ed pair test). */
int alk_gather_u32(const uint32_t* d_src, const uint32_t* d_idx, uint64_t n, uint32_t* d_out, alk_stream stream);
/* The indices i < n with d_flags[i] != 0, ascending, into d_out (room for n); the count
 * into *h_count. Synchronises. (alk_live_compact gives the same set in no set order.) */
int alk_flags_compact(const uint64_t* d_flags, uint64_t n, uint32_t* d_out, uint64_t* h_count, alk_stream stream);
int alk_pair_match(const uint32_t* d_pl, const uint32_t* d_pr, uint64_t n, const int64_t* d_lcol,
                   const int64_t* d_rcol, int neq, uint64_t* d_flags, alk_stream stream);
int alk_rows_mark(const uint32_t* d_rows, uint64_t n, uint64_t* d_flags, uint64_t value, alk_stream stream);
int alk_seg_minmax(const int64_t* d_keys, const uint64_t* h_start, uint32_t nseg, int64_t* h_out, alk_stream stream);
/* Per column segment (nseg <= 65535 descriptors): 1 when its values are in ascending
 * order (ties allowed), else 0, into h_sorted[g]. Synchronises. */
int alk_seg_sorted(const alk_colseg* segs, uint32_t nseg, uint8_t* h_sorted, alk_stream stream);

/* Width conversions used by the host engine between index and value columns. */
int alk_widen_u32(const uint32_t* d_in, uint64_t n, int64_t* d_out, alk_stream stream);
int alk_narrow_u32(const int64_t* d_in, uint64_t n, uint32_t* d_out, alk_stream stream);
/* Text loader (LOAD 'file' USING (sep) AS (...), CudaSet::LoadBigFile, cm.cu:1852-2080):
 * the records are the text's newline-terminated lines; declared column i reads the i-th
 * smallest of the declared field numbers (1-based), as the reference maps them. A field
 * ends at the separator outside double quotes (the quotes stay in it, NUL bytes are
 * dropped) and is cut to 23 bytes; it is parsed as an integer (ALK_TEXT_INT: leading
 * spaces, a sign, digits), a decimal of `scale` <= 9 fraction digits (ALK_TEXT_DECIMAL:
 * value x 10^scale, digits past the scale ignored), or, when the first record's field
 * has '-' at offset 4, as a yyyy-mm-dd date (yyyymmdd; *h_date_mask bit i); a char
 * column (ALK_TEXT_CHAR) keeps the field's bytes, NUL bytes dropped, cut or zero-padded
 * to its width. d_out[i]: device column of out_cap int64 values, or of out_cap x width
 * bytes for a char column; *h_rows gets the record count (ALK_ERR_OVERFLOW when above
 * out_cap). h_text is host memory; synchronises. */
typedef struct alk_text_col {
  uint32_t field;  /* 1-based field number as declared */
  uint32_t kind;   /* ALK_TEXT_INT, ALK_TEXT_DECIMAL or ALK_TEXT_CHAR */
  uint32_t scale;  /* decimal: digits after the point */
  uint32_t width;  /* char: bytes a value (the field, NUL bytes dropped, zero-padded) */
} alk_text_col;
#define ALK_TEXT_INT 0
#define ALK_TEXT_DECIMAL 1
#define ALK_TEXT_CHAR 2
int alk_text_load(const char* h_text, uint64_t nbytes, char sep, const alk_text_col* cols, uint32_t ncols,
                  void* const* d_out, uint64_t out_cap, uint64_t* h_rows, uint32_t* h_date_mask, alk_stream stream);
/* MurmurHash64A(value, width, seed) / 2 of n fixed-width values (the .hash file of a char
 * column, compress_char cm.cu:1765-1844; the reference hashes with seed 100). */
int alk_hash_strings(const uint8_t* d_chars, uint64_t n, uint32_t width, uint32_t seed, uint64_t* d_out,
                     alk_stream stream);
/* Frame-of-reference re-encoding of n int64 values: the exact minimum goes to *h_lower,
 * the narrowest of 8/16/32/64 bits that holds every value less it to *h_bits, and the
 * values less the minimum at that width to d_out (out_cap bytes; ALK_ERR_OVERFLOW when
 * too small). The engine keeps FOR-delta segments resident in this form: decoded once
 * at upload, then read like FOR segments (value = stored + lower). Synchronises. */
int alk_for_reencode(const int64_t* d_in, uint64_t n, void* d_out, size_t out_cap, int64_t* h_lower, uint32_t* h_bits,
                     alk_stream stream);

/* Linear-probing hash join on MurmurHash64A keys, replaces the sort-merge join of
 * emit_multijoin (operators.cu:1117-1283, moderngpu inner_join). Build indexes the
 * right rows; probe emits every (left row, right row) pair with equal keys. */
typedef struct alk_join_table alk_join_table;
int alk_join_build(const int64_t* d_keys, uint64_t n, alk_join_table** out, alk_stream stream);
/* Writes up to cap pairs; *h_pairs receives the total; ALK_ERR_OVERFLOW if total > cap. */
int alk_join_probe(const alk_join_table* t, const int64_t* d_keys, uint64_t n, uint32_t* d_left,
                   uint32_t* d_right, uint64_t cap, uint64_t* h_pairs, alk_stream stream);
void alk_join_free(alk_join_table* t, alk_stream stream);

/* ------------------------------------------------- fused pipeline stages
 * The filter -> join -> join -> group-by chain of emit_filter / emit_multijoin /
 * emit_select (operators.cu:797-1582, 1801-2084) as device stages over resident
 * segments: build stages insert a unique join key with payload columns into a
 * MurmurHash64A linear-probing table (optionally probing the previous stage's table),
 * and the probe-aggregate stage accumulates exact int64 aggregates per build row. */
typedef struct alk_ht alk_ht;
/* max_keys bounds the inserted keys; npay payload columns (<= 8) per key. */
int alk_ht_create(uint64_t max_keys, uint32_t npay, alk_ht** out, alk_stream stream);
/* Widest key range (values) that gets an exact key bitmap: bit offsets stay below 2^32,
 * and the bitmap takes at most 512 MB. */
#define ALK_DENSE_MAX_SPAN 0xFFFFFFFFull
/* Same, for keys known to lie in [key_min, key_max] (the build column's zone maps): the
 * table then also keeps an exact membership bitmap of the inserted keys (when the range
 * spans at most ALK_DENSE_MAX_SPAN values) that probes test before hashing. A key
 * inserted outside the range sets flag 8. */
int alk_ht_create_range(uint64_t max_keys, uint32_t npay, int64_t key_min, int64_t key_max, alk_ht** out,
                        alk_stream stream);
/* Dense (rank-addressed) build table for keys known to lie in [key_min, key_max], a
 * range of at most ALK_DENSE_MAX_SPAN values (from the build column's zone maps): a build
 * stage sets the
 * keys' bits in an exact bitmap, a prefix pass ranks them, and a key's slot is its rank
 * among the keys present, so keys, payload and per-key accumulators are dense over
 * [0, inserted) with no hashing. max_keys is the slot capacity (more distinct keys set
 * flag 2, capacity exceeded). ALK_ERR_UNSUPPORTED for a wider range. */
int alk_ht_create_dense(uint64_t max_keys, uint32_t npay, int64_t key_min, int64_t key_max, alk_ht** out,
                        alk_stream stream);
/* What a dense table keeps. FULL: keys and payload at their slots (the build writes one
 * record per surviving row and scatters it to its rank). RANKS: the bitmap and the rank
 * prefix only (slots for per-key accumulators; keys and payload are fetched later for a
 * few slots by alk_ht_late_rows; alk_ht_keys and alk_ht_payload return NULL). BITS: the
 * bitmap only (membership probes; a stage that asks this table for slots is refused).
 * In RANKS and BITS a build detects duplicate keys from the bitmap itself. */
#define ALK_DENSE_FULL 0
#define ALK_DENSE_RANKS 1
#define ALK_DENSE_BITS 2
/* alk_ht_create_dense with a mode; npay must be 0 unless the mode is ALK_DENSE_FULL. */
int alk_ht_create_dense_mode(uint64_t max_keys, uint32_t npay, int64_t key_min, int64_t key_max, int mode,
                             alk_ht** out, alk_stream stream);
/* Keys and payload of a few slots of an ALK_DENSE_RANKS table, after the fact. d_cand
 * holds candidate slots, their number in device memory d_count (at most cap of them are
 * handled). Each candidate's key is selected back from the bitmap and rank prefix and
 * written to d_out[0][slot]; the key's rows are then found by binary search in the build
 * table's scanned segments (seg_mode != 0) whose key range [seg_lo, seg_hi] (the key
 * column's zone maps) holds it, and payload p of the one row found is written to
 * d_out[1 + p][slot]. cols: [1 + npay][nseg] descriptors, the key column first, then the
 * payload columns; the key column of every scanned segment must be in ascending order
 * (alk_seg_sorted). A candidate whose key is found in no row or in more than one sets
 * *d_status to 1 (the rows cannot name the surviving one: build the table FULL). d_out is
 * a host array of 1 + npay device addresses of slot-indexed columns of alk_ht_slots(h)
 * values. Asynchronous; no host synchronisation, capturable in a CUDA graph. */
int alk_ht_late_rows(const alk_ht* h, const uint32_t* d_cand, const uint64_t* d_count, uint32_t cap,
                     const alk_colseg* cols, uint32_t npay, uint32_t nseg, const uint8_t* seg_mode,
                     const int64_t* seg_lo, const int64_t* seg_hi, int64_t* const* d_out, int32_t* d_status,
                     alk_stream stream);
void alk_ht_free(alk_ht* h, alk_stream stream);
/* Inserted keys and flags (1 duplicate key, 2 capacity exceeded, 4 wait expired,
 * 8 key outside the declared range). */
int alk_ht_info(const alk_ht* h, uint64_t* nslots, int* flags, alk_stream stream);
/* Slot range of a table: payload columns and per-key accumulators are indexed by the
 * key's table position, 0 <= slot < alk_ht_slots(h). */
uint64_t alk_ht_slots(const alk_ht* h);
/* Device bytes the table holds (keys, payload, bitmap, rank). */
uint64_t alk_ht_bytes(const alk_ht* h);
/* Device address of the key column (slot-indexed; free slots of a hash table hold the
 * byte pattern 0x80 repeated, 0x8080808080808080; a dense table's slots at and beyond
 * its key count are undefined). */
const int64_t* alk_ht_keys(const alk_ht* h);
/* Device address of payload column p (slot-indexed). */
const int64_t* alk_ht_payload(const alk_ht* h, uint32_t p);
/* Filter + hash GROUP BY in one pass over resident segments (emit_select's group-by,
 * select.cu:359-952, over the rows emit_filter keeps, filter.cu:133-643). pred (NULL =
 * every row) and the aggregate input programs read scan columns (slots < ncols) at their
 * stored widths; nkeys (1-4) group key columns at key_slots; nagg (<= 7) aggregates of
 * agg_kind. key_min / key_max (host arrays, or NULL) bound the key columns over the
 * scanned segments (zone maps): when the product of their spans is small (at most 2^32
 * and 16 per scanned row) the key space itself indexes the accumulators (no hashing, a
 * presence bit per slot); otherwise max_groups sizes a hash table (at most 0.7 full). The
 * groups, in no particular order, go to the device columns d_out_keys[j] /
 * d_out_vals[v] (host arrays of device addresses, out_cap values each); *h_groups is
 * the group count. Surviving rows per
 * segment go to h_seg_rows[nseg] and rows scanned to *h_rows_in (either may be NULL).
 * Synchronises. ALK_ERR_OVERFLOW: more groups than out_cap (*h_groups tells how many) or
 * a full table (more groups than the table holds: call again with a larger max_groups);
 * ALK_ERR_UNSUPPORTED: a one-column key equal to 0x8080808080808080 (the hash table's
 * free-slot marker), or a key outside the stated ranges. */
int alk_pipeline_groupby(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                         const alk_program* pred, const int32_t* key_slots, uint32_t nkeys,
                         const alk_program* agg_progs, const uint8_t* agg_kind, uint32_t nagg, uint64_t max_groups,
                         const int64_t* key_min, const int64_t* key_max, int64_t* const* d_out_keys,
                         int64_t* const* d_out_vals, uint64_t out_cap, uint64_t* h_groups, uint64_t* h_seg_rows,
                         uint64_t* h_rows_in, alk_stream stream);
/* Optional CUDA-event timing of the probe-aggregate kernel (cudaEvent_t handles). */
typedef struct alk_event_timer {
  int on;
  void* ev0;
  void* ev1;
  double ms;
  uint64_t launches;
} alk_event_timer;
/* Build stage. The predicate reads scan slots only; payload sources pay_src[p] name scan
 * slots (< 32) or, when probing, payload columns of the probed table (32 + p).
 *
 * Both stages run as a streaming scan that appends the positions of surviving rows
 * (predicate true and, when probing, the key present in the probed table's key bitmap)
 * to a device hit list sized for hit_cap survivors (8 bytes each, plus a fixed slack for
 * the scan warps' partly filled chunks; 0 = the rows scanned, which cannot overflow),
 * followed by one kernel that does the per-survivor work. If more rows survive than the
 * list holds, nothing is applied, ALK_ERR_OVERFLOW is returned and *h_hits holds the
 * exact survivor count for a rerun. h_rows_in receives the rows scanned. Synchronizes. */
int alk_pipeline_build(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                       const alk_program* pred, const alk_ht* probe, int32_t probe_slot, alk_ht* build,
                       int32_t build_slot, const int32_t* pay_src, uint64_t hit_cap, uint64_t* h_rows_in,
                       uint64_t* h_hits, alk_stream stream);
/* Probe-aggregate stage: for every surviving row whose probe key hits, aggregate
 * agg_progs[g] (ALK_AGG_SUM / MIN / MAX, or COUNT; column operands: scan slots or probed
 * payload 32 + p) into d_acc[g * acc_stride + slot] and count rows into d_cnt[slot].
 * Accumulators must be initialised by the caller. Hit list as for the build stage; the
 * timer, when on, brackets the scan and hit kernels. */
int alk_pipeline_probe_agg(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                           const alk_program* pred, const alk_ht* probe, int32_t probe_slot,
                           const alk_program* agg_progs, const uint8_t* agg_kind, uint32_t nagg, int64_t* d_acc,
                           uint64_t acc_stride, uint64_t* d_cnt, uint64_t hit_cap, uint64_t* h_rows_in,
                           uint64_t* h_hits, alk_stream stream, alk_event_timer* timer);
/* Asynchronous stages: the same work, with no host synchronisation. The counters arrive
 * in *h_status (host memory; pinned for the copy to be asynchronous) once the stream
 * reaches the end of the stage: err is ALK_OK, ALK_ERR_OVERFLOW (nothing applied; hits is
 * the exact survivor count) or ALK_ERR_TIMEOUT. Argument errors are returned at once. */
typedef struct alk_stage_status {
  uint64_t rows_in;  /* rows scanned */
  uint64_t reserved; /* hit-list entries reserved */
  int32_t err;
  int32_t pad;
  uint64_t hits;     /* survivors of the scan */
} alk_stage_status;
int alk_pipeline_build_async(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                             const alk_program* pred, const alk_ht* probe, int32_t probe_slot, alk_ht* build,
                             int32_t build_slot, const int32_t* pay_src, uint64_t hit_cap,
                             alk_stage_status* h_status, alk_stream stream);
int alk_pipeline_probe_agg_async(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                                 const alk_program* pred, const alk_ht* probe, int32_t probe_slot,
                                 const alk_program* agg_progs, const uint8_t* agg_kind, uint32_t nagg,
                                 int64_t* d_acc, uint64_t acc_stride, uint64_t* d_cnt, uint64_t hit_cap,
                                 alk_stage_status* h_status, alk_stream stream, alk_event_timer* timer);
/* alk_ht_info without synchronising: inserted keys and the four flags (duplicate key,
 * capacity exceeded, wait expired, key outside the declared range; non-zero = set) land
 * in *h_out when the stream reaches this point. */
typedef struct alk_ht_status {
  uint64_t inserted;
  int32_t flags[4];
} alk_ht_status;
int alk_ht_info_async(const alk_ht* h, alk_ht_status* h_out, alk_stream stream);
int alk_fill_i64(int64_t* d, uint64_t n, int64_t v, alk_stream stream);
/* Top-k candidates for ORDER BY ... LIMIT k (emit_order + Store LIMIT, operators.cu:1641,
 * cm.cu:1493): every live slot whose ranking value is >= the k-th largest ranking value
 * (ties included); the caller orders the few candidates with the full key list. */
int alk_topk_candidates(const int64_t* d_rank, const uint64_t* d_live, uint64_t n, uint32_t k, uint32_t* d_out,
                        uint64_t cap, uint64_t* h_count, alk_stream stream);
/* The same selection without a host round trip (k <= 16): the threshold is computed on
 * the device and the candidate count is written to device memory d_count (candidates
 * beyond cap are counted, not written). Asynchronous on the stream. */
int alk_topk_select(const int64_t* d_rank, const uint64_t* d_live, uint64_t n, uint32_t k, uint32_t* d_out,
                    uint64_t cap, uint64_t* d_count, alk_stream stream);
/* d_out[c * cap + r] = d_cols[c][d_idx[r]] for r < min(*d_count, cap) and c < ncols (<= 32);
 * the row count is read on the device. Asynchronous on the stream. */
int alk_gather_rows(const int64_t* const* d_cols, uint32_t ncols, const uint32_t* d_idx, const uint64_t* d_count,
                    uint64_t cap, int64_t* d_out, alk_stream stream);
/* Indices of live (non-zero) slots, unordered. */
int alk_live_compact(const uint64_t* d_live, uint64_t n, uint32_t* d_out, uint64_t* h_count, alk_stream stream);

/* Front end: renders the statements and postfix queues the parser produces for a script
 * (the argument queues of the reference's grammar actions, bison.y:127-287). */
int alk_parse_dump(const char* script, char* out, int out_len);

/* Seeded synthetic tables in the reference's on-disk format (no counterpart in the
 * reference, which loads text files): the single-table lineitem shape and the
 * customer/orders/lineitem shape of the three-way pipeline, in segments of seg_rows
 * rows (0: one segment), FOR or (delta != 0) FOR-delta for sorted integer columns.
 * 0 on success; a message is written into err (err_len bytes) otherwise. */
int alk_gen_lineitem_flat(const char* dir, uint64_t rows, uint32_t seg_rows, uint64_t seed, int delta,
                          char* err, int err_len);
int alk_gen_three_way(const char* dir, uint64_t customers, uint64_t orders, uint64_t lineitems,
                      uint32_t seg_rows, uint64_t seed, int delta, char* err, int err_len);
/* The same tables with skewed join keys: lineitem's orderkeys follow Zipf(zipf_s) over
 * the orders, in key order (order i gets round(N F(i)) - round(N F(i - 1)) of the N
 * rows, F the Zipf distribution function over the orders). */
int alk_gen_three_way_zipf(const char* dir, uint64_t customers, uint64_t orders, uint64_t lineitems,
                           uint32_t seg_rows, uint64_t seed, int delta, double zipf_s, char* err, int err_len);
/* Table "names" for string predicates: n_key 1..rows and n_name char(12) drawn from
 * `distinct` generated strings over A, B, X, '.', '%', '_' (lengths 0-12). */
int alk_gen_names(const char* dir, uint64_t rows, uint32_t distinct, uint32_t seg_rows, uint64_t seed, char* err,
                  int err_len);
/* The single-table lineitem shape generated in device memory, segment by segment, as a
 * function of (seed, column, row_base + row): l_orderkey (4 rows per key), l_quantity
 * U[1,50], l_extendedprice U[90000,10500000], l_discount U[0,10], l_shipdate uniform
 * over 1992-01-02..1998-12-01, l_returnflag codes of {A,N,R}, l_linestatus codes of
 * {F,O}. minmax: per segment and column (7) the [min, max] pair; write: the stored
 * values into cols [7][nseg] (data, lower = the minimum, bits set by the caller). */
int alk_gen_flat_minmax(uint64_t seed, uint64_t row_base, const uint32_t* seg_rows, uint32_t nseg, int64_t* h_minmax,
                        alk_stream stream);
int alk_gen_flat_write(uint64_t seed, uint64_t row_base, const uint32_t* seg_rows, uint32_t nseg,
                       const alk_colseg* cols, alk_stream stream);
/* One generated value (host side, for checks). */
int64_t alk_gen_flat_value(uint64_t seed, int col, uint64_t row);
/* Registers such a table in the session's catalog with every segment resident (no
 * files; exact per-segment zone maps; the file encoder's widths). */
int alk_session_gen_flat_resident(alk_session* s, const char* table, const uint32_t* seg_rows, uint32_t nseg,
                                  uint64_t seed, uint64_t row_base);

/* A yyyymmdd date value moved by a number of days (proleptic Gregorian). */
int64_t alk_date_add_days(int64_t yyyymmdd_value, int64_t days);

/* ------------------------------------------ batched filter + group-by
 * Many queries of the single-table shape FILTER t BY <conjunction> -> SELECT keys,
 * aggregates FROM it GROUP BY keys (each of which the reference runs as emit_filter +
 * emit_select, operators.cu:2306 and :1801) in one persistent launch over a work list of
 * (query, segment) items. Group keys are at most two columns whose value ranges (from the
 * zone maps) give a dense slot space; every aggregate input is a product of two affine
 * column terms, value = (am * A + ac) * (bm * B + bc) in wrapping int64 arithmetic (b < 0:
 * the second factor is 1), which covers columns and the decimal forms such as
 * price * (1 - discount). */
typedef struct alk_gb_agg {
  int64_t am, ac, bm, bc;
  int32_t a, b;   /* query column indexes (b < 0: no second factor) */
  uint32_t kind;  /* ALK_AGG_SUM / COUNT / MIN / MAX */
  uint32_t pad;
} alk_gb_agg;
typedef struct alk_gb_query {
  const alk_colseg* cols;  /* [ncols][nseg]; 16-byte aligned, readable to the next 16 bytes */
  uint32_t ncols, nseg;    /* ncols <= 8 */
  const uint8_t* seg_mode; /* per segment: 0 skip, 1 every row passes, 2 evaluate (NULL: 2) */
  const alk_program* pred; /* a conjunction of column comparisons, or NULL */
  uint32_t nkeys;          /* 0..2 */
  int32_t key_col[2];
  int64_t key_min[2], key_max[2]; /* key value ranges; slots = product of the spans */
  uint32_t nagg;                  /* <= 8 */
  alk_gb_agg agg[8];
  int64_t* d_acc;       /* device [nagg + 1][slots]: the aggregates, then the row count */
  uint64_t* h_seg_rows; /* optional host [nseg]: rows passing the filter per segment */
} alk_gb_query;
/* timer (optional): events around the group-by kernel; its time and launch count are
 * added to it. */
/* Launch shape: consumer warps per block (4 or 8; a tile is 256 rows per warp), tiles in
 * flight per block (2..4), blocks per SM (capped by shared memory); 0 = default. */
typedef struct alk_gb_tuning {
  uint32_t consumer_warps, stages, blocks_per_sm;
} alk_gb_tuning;
/* Runs the queries (accumulators initialised here) and synchronizes the stream. slots *
 * (nagg + 1) <= 64 per query (accumulators private to each thread); a larger slot space or
 * a filter that is not a conjunction returns ALK_ERR_UNSUPPORTED. *used = the shape run. */
int alk_batch_groupby(const alk_gb_query* queries, uint32_t nq, const alk_gb_tuning* tune, alk_gb_tuning* used,
                      alk_event_timer* timer, alk_stream stream);
/* Runs n scripts with one batched launch for their group-bys: every script runs up to
 * its first SELECT ... GROUP BY of the dense form, those run together, then every script
 * continues. Results are those of running the scripts one at a time. Returns the first
 * failing script's status (alk_session_error names it); the others still run. */
int alk_session_execute_batch(alk_session* s, const char* const* scripts, uint32_t n);
/* Group-by form of the operator path: 0 chosen by the expected group count (the learned
 * estimator's when it is on, else the zone maps' bound; above 2^22 groups the sort-based
 * form), 1 always hash, 2 always sort. */
int alk_session_set_groupby(alk_session* s, int mode);
/* Switches the session between the operator-at-a-time plan (on) and the fused plans. */
int alk_session_set_plain(alk_session* s, int on);
/* *out = the launch shape of the last batched group-by; autotune 0/1 turns the per-
 * workload autotuner off/on (-1 leaves it). */
int alk_session_tuning(alk_session* s, alk_gb_tuning* out, int autotune);
/* Fixes the launch shape of later batched group-bys (*shape with consumer_warps 0, or
 * NULL, returns to the autotuner or the default); a shape that shared memory cannot hold
 * is reduced as the launch reports in alk_session_tuning. */
int alk_session_set_tuning(alk_session* s, const alk_gb_tuning* shape);

/* ------------------------------------------ 4. learned cardinality estimator
 * No counterpart in the reference, which sizes every buffer from the free device memory
 * (getFreeMem, cm.cu:3184) and the rows scanned. A small MLP, 64 -> 128 -> 128 -> 3 with
 * ReLU, BF16 weights and FP32 accumulation, predicts per (stage, segment) three log
 * fractions: the rows passing the filter (of the rows), the rows passing the join probe
 * (of those) and the distinct key values (of those). The fused plan sizes its survivor
 * lists and hash tables from them on a query's first run; a size that proves too small
 * makes the query run again with the exact counts (the estimate steers the plan, never
 * the answer). */
#define ALK_CARD_FEATURES 64
#define ALK_CARD_HIDDEN 128
#define ALK_CARD_OUTPUTS 3
typedef struct alk_mlp alk_mlp;
/* Parameters in order W1[128][64], b1[128], W2[128][128], b2[128], W3[3][128], b3[3]. */
uint32_t alk_mlp_param_count(void);
/* Seeded initialisation (uniform, fan-in scaled; zero biases). Synchronizes the stream. */
int alk_mlp_create(uint64_t seed, alk_mlp** out, alk_stream stream);
void alk_mlp_free(alk_mlp* m, alk_stream stream);
/* Replace the FP32 master parameters (h_master, alk_mlp_param_count() floats); the BF16
 * weights are their round-to-nearest-even copies. Synchronizes the stream. */
int alk_mlp_set_params(alk_mlp* m, const float* h_master, alk_stream stream);
/* Copies of the FP32 master parameters and of their BF16 copies (either may be NULL). */
int alk_mlp_params(const alk_mlp* m, float* h_master, uint16_t* h_bf16, alk_stream stream);
/* d_y[n][3] = MLP(d_x[n][64]) with the BF16 weights. Asynchronous. */
int alk_mlp_forward(alk_mlp* m, const float* d_x, uint64_t n, float* d_y, alk_stream stream);
/* Gradient of the masked mean squared error sum((y - t)^2 * mask) / n with respect to the
 * parameters (layout above; bias gradients included), into d_grad; *h_loss = the loss.
 * The forward pass uses the BF16 weights. Synchronizes the stream. */
int alk_mlp_gradients(alk_mlp* m, const float* d_x, const float* d_t, const float* d_mask, uint64_t n,
                      float* d_grad, float* h_loss, alk_stream stream);
/* Adam (beta 0.9 / 0.999, eps 1e-8) over mini-batches of `batch` rows in order, for
 * `epochs` passes; *h_loss = mean loss of the last pass. Synchronizes the stream. */
int alk_mlp_train(alk_mlp* m, const float* d_x, const float* d_t, const float* d_mask, uint64_t n, uint32_t epochs,
                  uint32_t batch, float lr, float* h_loss, alk_stream stream);
/* 16 equal-width bins of a column segment's values over [lo, hi] (values outside go to
 * the end bins) into d_hist16[16]. Asynchronous. */
int alk_card_hist16(const alk_colseg* seg, int64_t lo, int64_t hi, uint32_t* d_hist16, alk_stream stream);
/* Exact per-segment counts of a stage (the estimator's labels and the exact counting
 * pass): h_counts[3 * g] rows of segment g passing pred, [3 * g + 1] of those whose
 * probe_slot value is a key of probe (all of them without a probe), [3 * g + 2] distinct
 * key_slot values among those (UINT64_MAX when key_slot < 0 or the range [key_min,
 * key_max] is wider than 2^30). Segments with seg_mode 0 count 0. Synchronizes. */
int alk_card_count(const alk_colseg* cols, uint32_t ncols, uint32_t nseg, const uint8_t* seg_mode,
                   const alk_program* pred, const alk_ht* probe, int32_t probe_slot, int32_t key_slot,
                   int64_t key_min, int64_t key_max, uint64_t* h_counts, alk_stream stream);

/* Session side. record: every fused query also runs the exact counting pass of each stage
 * and keeps one record (features, log-fraction targets, target mask) per scanned segment;
 * such runs are not captured into CUDA graphs. use: stages without recorded counts are
 * sized by the estimator (when one is trained). */
int alk_session_card_mode(alk_session* s, int record, int use);
/* Records kept so far: *h_n = their number; up to cap of them are copied (features
 * [cap][64], targets [cap][3], masks [cap][3]; NULL pointers skip a copy). */
int alk_session_card_records(alk_session* s, float* h_x, float* h_y, float* h_mask, uint64_t cap, uint64_t* h_n);
/* Train the session's estimator (created from seed on first use) on records
 * [first, first + count), shuffled by seed, with alk_mlp_train. */
int alk_session_card_train(alk_session* s, uint64_t first, uint64_t count, uint32_t epochs, uint32_t batch,
                           float lr, uint64_t seed, float* h_loss);
/* Estimator outputs for n feature rows (host arrays). */
int alk_session_card_predict(alk_session* s, const float* h_x, uint64_t n, float* h_y);
/* The trained estimator to a file and back (FP32 master parameters), so that a session
 * can use a network trained in another one. */
int alk_session_card_save(alk_session* s, const char* path);
int alk_session_card_load(alk_session* s, const char* path);
/* Forget the exact counts recorded by earlier runs and the captured graphs, so that the
 * next run of a query is a first run again. */
int alk_session_card_forget(alk_session* s);

/* Star join with bitmap join indexes (CREATE INDEX ... ON fact(dim.col) FROM fact, dim
 * WHERE fact.fk = dim.key, then a join of the fact table with a filtered dimension).
 *
 * alk_bitmap_index_build: one index segment, replaces the per-segment body of
 * emit_create_bitmap_index (operators.cu:2225-2264) and compress_int (cm.cu:4271-4336).
 * Value i < n is d_vals[lower_bound(d_keys[0..m), d_fk[i])]; the ntail values of d_tail
 * follow (the char form appends the dimension's row hashes past the fact segment's row
 * count when the dimension has more rows). Writes the sorted distinct values (h_dict, room
 * for n + ntail), the codes bit-packed MSB first, 64 / bits a word (h_words, room for
 * n + ntail words), and bits = ceil(log2(distinct + 1)). ALK_ERR_UNSUPPORTED when a
 * foreign key lies past the last dimension key (the reference gathers past its key
 * column there). All pointers but the h_* ones are device memory. Synchronises. */
int alk_bitmap_index_build(const int64_t* d_fk, uint32_t n, const int64_t* d_keys, uint32_t m, const int64_t* d_vals,
                           const int64_t* d_tail, uint32_t ntail, int64_t* h_dict, uint32_t* h_dict_n,
                           uint64_t* h_words, uint32_t* h_words_n, uint32_t* h_bits, alk_stream stream);
/* The packed codes of an index segment (as loadIndex keeps them, cm.cu:2775-2845, and
 * cmp_functor_dict reads them, filter.cu:21-65) decoded to one code a row at out_bits
 * (8, 16 or 32, at least bits) into d_out. Asynchronous. */
int alk_bitmap_index_decode(const uint64_t* d_words, uint32_t rows, uint32_t bits, uint32_t fit_count, void* d_out,
                            uint32_t out_bits, alk_stream stream);
/* The star join's row lists (star_join operators.cu:541-552): d_rowid holds, segment after
 * segment (h_seg_counts survivors of h_seg_rows rows each), the surviving rows' positions
 * in their segments. The reference fills each segment's list with copy_if over rows
 * [0, rows - 1) into a list kept from the previous segment, so a surviving last row keeps
 * the previous list's entry at that position (0 past its end); this rewrites those
 * entries the same way. Synchronises. */
int alk_star_rows_fixup(uint32_t* d_rowid, const uint64_t* h_seg_counts, const uint32_t* h_seg_rows, uint32_t nseg,
                        alk_stream stream);
/* One output column of a star join (star_join operators.cu:558-766): for row i, the
 * value at position d_rowid[i] of segment d_seg[i] of the stored FOR column segs (host
 * array of nseg descriptors: payload, header lower, rows, bits), read as the reference
 * reads the segment file (8-bit values through a signed char) plus lower. With dim_key
 * and dim_val (host pointers to one descriptor each: the dimension's key column and the
 * column wanted, stored FOR over the same rows) the column is a dimension's foreign key:
 * t = (uint32)value, plus (uint32)(lower - 1) when lower != 1, and d_out[i] = dim_val at
 * lower_bound(dim_key, t). ALK_ERR_UNSUPPORTED when a row lies past its segment or a key
 * past the last dimension key. Synchronises. */
int alk_star_gather(const alk_colseg* segs, uint32_t nseg, const uint32_t* d_rowid, const uint32_t* d_seg, uint64_t n,
                    const alk_colseg* dim_key, const alk_colseg* dim_val, int64_t* d_out, alk_stream stream);

/* Device properties of the current device. */
int alk_device_info(int* sm_count, int* cc_major, int* cc_minor);

#ifdef __cplusplus
}
#endif
#endif /* ALENKA_B200_H */
