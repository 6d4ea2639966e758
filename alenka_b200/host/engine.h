// Host engine: executes Alenka scripts on the B200 through the operator-level C ABI
// (include/alenka_b200.h). It mirrors the reference's operator layer
// (emit_filter / emit_select / emit_join / emit_order / emit_store, operators.cu) and
// its CudaSet column model (cm.h:681-789): base tables backed by segment files,
// lazily filtered views, and materialized results.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <functional>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/alenka_b200.h"
#include "format.h"
#include "script.h"

namespace alk {

struct EngineError : std::runtime_error {
  int code;
  EngineError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Device buffer owned by the engine stream (stream-ordered allocation).
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(size_t bytes, cudaStream_t s);
  ~DevBuf();
  DevBuf(DevBuf&& o) noexcept;
  DevBuf& operator=(DevBuf&& o) noexcept;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  template <class T>
  T* as() const { return (T*)p_; }
  size_t bytes() const { return n_; }
  void reset();

 private:
  void* p_ = nullptr;
  size_t n_ = 0;
  cudaStream_t s_ = nullptr;
};
using DevBufP = std::shared_ptr<DevBuf>;

struct ColMeta {
  int type = 0;        // 0 int/decimal/date/dictionary code, 2 char (codes on device)
  uint32_t dz = 0;     // decimal_zeroes
  uint32_t width = 0;  // char width
  std::string string_map;  // "<table>.<column>" dictionary the codes refer to
  bool raw = false;          // a LOAD's char column: width bytes a row, no dictionary yet
  bool no_encoding = false;  // ... declared NO ENCODING
};

struct SegInfo {
  SegMeta m;
  size_t file_off = 0;  // payload offset within the cached file image
};

// One column of a base table: per segment header metadata (zone maps) and the cached
// images (pinned host) / device residency.
struct BaseCol {
  ColMeta meta;
  std::vector<SegInfo> segs;
  std::vector<uint8_t*> host_img;     // pinned host copies of the segment files
  std::vector<size_t> host_len;
  std::vector<DevBufP> dev;           // device payload: FOR as stored; FOR-delta re-encoded as FOR
  // per segment, the resident encoding: value = stored + res_lower at res_bits (for FOR
  // segments the file's own; for FOR-delta ones the re-encoding's exact minimum and width)
  std::vector<int64_t> res_lower;
  std::vector<uint32_t> res_bits;
  // per segment: its values in ascending order (1) or not (0), as checked on the device
  // buffer recorded beside it (a segment uploaded again is checked again)
  std::vector<std::weak_ptr<DevBuf>> order_buf;
  std::vector<int8_t> ascending;
  bool headers_read = false;
  bool device_only = false;  // generated in device memory: no files, never released
  // char dictionaries
  std::vector<std::string> dict;
  std::unordered_map<uint64_t, int64_t> hash_to_code;
  bool dict_loaded = false;
  std::map<std::string, DevBufP> like_sets;  // LIKE pattern -> its matching codes [n, bits]
  DevBufP ranks;                             // entry -> dense rank in byte order (ORDER BY)
  // a bitmap join index column ("<dimension>.<column>" of a fact table): per segment its
  // dictionary (ascending values) and the offset of its codes in the index's code space
  std::vector<std::vector<int64_t>> idx_dict;
  std::vector<uint64_t> idx_off;
};

struct Var {
  enum Kind { Base, Filtered, Mat } kind = Mat;
  std::string name;
  std::vector<std::string> columnNames;
  std::map<std::string, ColMeta> meta;
  // Base
  std::string table, load_file_name;
  uint32_t segCount = 1, maxRecs = 0;
  uint64_t total = 0;
  // Filtered (fil_* queues of CudaSet, cm.h:692-698)
  std::string source;
  std::vector<std::string> fil_type, fil_value;
  std::vector<int64_t> fil_nums;
  std::vector<uint32_t> fil_prec;
  // Mat
  uint64_t n = 0;
  std::map<std::string, DevBufP> data;
  // host copies of small results (dense group-by); data gets a column on first use
  std::map<std::string, std::vector<int64_t>> host;
  std::map<std::string, int> grp_type;
  bool scanned = false;  // Filtered: an operator has read it (its row list exists)
  bool has(const std::string& c) const;
};

// A scan of a base table (or of a filtered view of one): zone-map verdict per segment,
// the compiled predicate, and the column slots the device code reads.
struct ScanPlan {
  Var* src = nullptr;
  std::vector<std::string> slots;
  alk_program pred{};
  bool has_pred = false;
  std::vector<uint8_t> mode;  // 0 skip, 1 all rows, 2 evaluate
  uint32_t slot(const std::string& c);
};

// Materialized rows of a variable for a set of fields.
struct Rows {
  uint64_t n = 0;
  std::map<std::string, DevBufP> col;
  std::vector<uint64_t> seg_counts;  // surviving rows per source segment (base/filtered)
  DevBufP seg_of_row;                // u32 source segment of every row (when requested)
};

// A fused stage whose counters are checked after the query's synchronisation.
struct FusedPending {
  std::string sig;  // stage signature (table, compiled predicate, zone-map verdicts, key)
  int st, ht;       // index of its alk_stage_status / alk_ht_status (ht -1: none)
  uint64_t upper;   // exact upper bound of its key count (rows scanned)
};

// What the fused plan needs after the device work: counters to check, the ORDER keys
// and the STORE. A captured graph keeps one, so that a replay skips the planning.
struct FusedTail {
  std::vector<FusedPending> pending;
  bool timed = false;                           // the probe-aggregate stage carries timing events
  uint64_t streamed_bytes = 0, hit_bytes = 0;   // its algorithmic bytes: all rows, per survivor
  size_t nouts = 0, ngroups = 0;                // F's columns, then the group keys, come back
  std::vector<int> okey;
  std::vector<bool> odesc;
  std::vector<ColMeta> fmeta;
  uint32_t limit = 0;
  uint64_t small = 0, cand_cap = 0;             // rows returned with the first copy; candidate cap
  std::string first_key, path, sep;
  uint64_t kernels = 0, d2h = 0, rows = 0;      // statistics of one execution
  std::string late_sig;  // the last build stage fetched its payload late (status to check)
};
struct FusedGraph;
struct SelectCtx;

// One fused stage as the cardinality estimator sees it: the scan, what it probes, and the
// key column whose distinct values it counts (the build key, or the probe-aggregate
// stage's group key).
struct CardStage {
  const ScanPlan* p = nullptr;
  const std::vector<alk_colseg>* cs = nullptr;
  int kind = 0;  // 0 build, 1 build probing another table, 2 probe-aggregate
  int32_t probe_slot = -1;
  const alk_ht* probe = nullptr;
  double probe_fill = 0;  // fraction of the probed table's key range present
  std::pair<int64_t, int64_t> probe_range{0, -1};
  int32_t key_slot = -1;
  std::pair<int64_t, int64_t> key_range{0, -1};
  const ScanPlan* up = nullptr;  // the scan that built the probed table
};

// The embedding API's implementation (alenka.h:30-35), behind both its C entry points
// (include/alenka_b200.h) and the C++-linkage ones the reference's own callers bind.
void embed_init(char** av);
int embed_execute(char* s);
void embed_close();
int embed_file(int ac, char** av);

class Engine {
 public:
  Engine(std::string dir, uint32_t flags);
  ~Engine();
  int execute(const std::string& script);
  int execute_statements(std::vector<Statement> sts, const std::string& key);
  int execute_batch(const std::vector<std::string>& scripts);
  // A lineitem-shaped table generated in device memory (segments of the given sizes).
  int gen_resident_flat(const std::string& table, const std::vector<uint32_t>& seg_rows, uint64_t seed,
                        uint64_t row_base);
  const alk_gb_tuning& last_tuning() const { return last_tuning_; }
  void set_autotune(bool on) { autotune_ = on; }
  void set_tuning(const alk_gb_tuning& t) { fixed_tuning_ = t; }
  // group-by form: 0 chosen by the expected group count, 1 hash, 2 sort
  void set_groupby_mode(int m) { groupby_mode_ = m; }
  void set_plain(bool on) { flags_ = on ? (flags_ | ALK_SESSION_PLAIN) : (flags_ & ~ALK_SESSION_PLAIN); }
  const std::string& error() const { return err_; }
  cudaStream_t stream() const { return stream_; }
  int preload(const std::string& table);
  alk_stats stats() const { return stats_; }
  void set_timing(bool on) { timing_ = on; }
  // learned cardinality estimator (session side)
  int card_mode(bool record, bool use);
  uint64_t card_records(float* x, float* y, float* m, uint64_t cap) const;
  int card_train(uint64_t first, uint64_t count, uint32_t epochs, uint32_t batch, float lr, uint64_t seed,
                 float* loss);
  void card_forward(const float* h_x, uint64_t n, float* h_y);
  void card_forget();
  int card_save(const std::string& path);
  int card_load(const std::string& path);

  // ---- used by the planner / operators ----
  Var* var(const std::string& n);
  void ensure_base_col(Var* base, const std::string& col, bool device);
  Rows materialize(Var* v, const std::vector<std::string>& fields, bool want_seg = false);
  ScanPlan plan_scan(Var* v);
  // Device descriptors [slots][segments] of a scan (uploads columns on demand).
  std::vector<alk_colseg> colsegs(const ScanPlan& p);
  // Bytes one scan reads at the resident widths (segments not skipped).
  uint64_t scan_bytes(const ScanPlan& p, const std::vector<uint32_t>& used_slots);
  size_t cycle_count(Var* v);
  uint64_t free_mem() const { return kFreeMem; }
  // getFreeMem() (cm.cu:3184) pinned to a B200's 180 GB so that segmentation is deterministic.
  static constexpr uint64_t kFreeMem = 180ull * 1000 * 1000 * 1000;

 private:
  std::string dir_, err_;
  uint32_t flags_;
  cudaStream_t stream_ = nullptr;
  DataDict dd_;
  std::map<std::string, std::unique_ptr<Var>> vars_;
  std::map<std::string, std::shared_ptr<Var>> bases_;  // catalog tables (persist across scripts)
  std::map<std::string, std::map<std::string, BaseCol>> basecols_;
  alk_stats stats_{};
  // Exact build-side key counts recorded by previous runs of the same fused stage; they
  // size the next run's hash table (overflow reruns the stage at the upper bound).
  std::map<std::string, uint64_t> card_feedback_;
  bool timing_ = false;
  cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
  cudaEvent_t evq0_ = nullptr, evq1_ = nullptr;  // around a fused query's device work
  // Pinned host staging for device->host results (a pageable destination would make
  // every copy wait for the stream).
  void* pin_ = nullptr;
  size_t pin_n_ = 0;
  void* pinned(size_t bytes);

  void reset_script_state();
  void begin_script(const std::vector<Statement>& sts, std::map<std::string, size_t>& last);
  void drop_dead(const std::map<std::string, size_t>& last, size_t i);
  Var* base_table(const std::string& t);
  BaseCol& basecol(Var* base, const std::string& col);
  void read_headers(Var* base, const std::string& col, BaseCol& bc);
  // Every segment with mode[g] != 0 holds the column's values in ascending order (one
  // device pass per segment not checked before; none when may_sync is false: unknown
  // segments then count as unsorted).
  bool segs_ascending(BaseCol& bc, const std::vector<alk_colseg>& segs, const std::vector<uint8_t>& mode,
                      bool may_sync);
  void load_dict(Var* base, const std::string& col, BaseCol& bc);
  std::vector<char> zone_maps(Var* f, Var* src);
  alk_program compile_filter(Var* f, Var* src, std::vector<std::string>& slots);

  void exec(Statement& st);
  uint64_t filter_pairs(DevBufP& pl, DevBufP& pr, uint64_t pairs, const DevBufP& lcol, const DevBufP& rcol,
                        unsigned jac, const std::vector<char>& eq_type);
  void semi_anti_join(Var* c, Rows& L, Rows& R, const std::string& lkey, const std::string& rkey,
                      const std::string& f3, const std::string& f4, unsigned jac, const std::vector<char>& eq_type,
                      char kind);
  void emit_filter(Statement& st);
  void emit_select(Statement& st);
  void select_output(SelectCtx& c);
  // Dense group-by of a FILTER -> SELECT ... GROUP BY over a base table (small key
  // domains, conjunctive filter, affine-product aggregates): false when the SELECT has
  // another form. Batches run many prepared selects in one launch.
  bool dense_select_prepare(Statement& st, SelectCtx& c);
  bool hash_select(Statement& st);  // the fused filter + hash GROUP BY
  void dense_select_run(const std::vector<SelectCtx*>& cs);
  void dense_select_finish(SelectCtx& c);
  void emit_join(Statement& st);
  void multijoin(Statement& st, const std::string& s, const std::string& j1, const std::string& j2, unsigned tab);
  void emit_order(Statement& st);
  void emit_store(Statement& st);
  void emit_store_binary(Statement& st);
  void emit_load(Statement& st);
  // star join with bitmap join indexes (host/star.cpp)
  std::string star_table(Var* v);
  void emit_create_bitmap_index(Statement& st);
  void load_star_index(Var* base, const std::string& col, BaseCol& bc);
  std::vector<uint32_t> star_set(Var* base, const std::string& col, bool eq, int64_t key);
  DevBufP star_upload(const std::vector<uint32_t>& words);
  int64_t star_string_key(const std::string& col, const std::string& lit);
  bool star_join_applies(Statement& st);
  void star_join(Statement& st);
  std::vector<DevBufP> star_sets_;         // the code sets of this script's index comparisons
  std::set<std::string> star_consumed_;    // variables whose filters a star join has moved
  DevBufP like_set(Var* base, const std::string& col, const std::string& pattern);
  const DevBufP& dict_ranks(const ColMeta& m);
  DevBufP dict_hashes(const ColMeta& m, uint32_t width);
  std::map<std::string, uint32_t> cnt_counts_;  // largest payload written per column file prefix
  // codes of a LOAD's char values per column name: hash -> code (key 0: NO ENCODING's
  // running count), kept for the session as the reference keeps its char_hash
  std::map<std::string, std::unordered_map<uint64_t, int64_t>> char_codes_;
  bool try_fused(std::vector<Statement>& sts, size_t& i);
  void run_fused(Statement& J, Statement& F, Statement& O, Statement& S, const std::string& gkey);
  // After the synchronisation: check the stages, record their counts, store the rows.
  void finish_fused(const FusedTail& t);
  void store_fused_rows(const FusedTail& t, std::vector<std::vector<int64_t>>& hf,
                        std::vector<std::vector<int64_t>>& hg, uint64_t ncand);
  // Fused queries captured as CUDA graphs, by script text and statement (resident
  // sessions; captured on a query's second successful run, replayed from the third).
  std::map<std::string, std::shared_ptr<FusedGraph>> fused_graphs_;
  std::set<std::string> fused_seen_;
  std::set<std::string> fused_nograph_;  // queries whose capture failed
  std::set<std::string> late_off_;       // build stages whose rows could not name a late candidate
  std::string cur_script_;
  std::unordered_map<std::string, std::vector<Statement>> parsed_;  // script text -> statements
  // a batch's final STOREs: formatted at once, written together after the batch (the
  // file creations dominate a small result's store) on several threads
  struct PendingWrite {
    std::string path, data;
    size_t run;
  };
  std::vector<PendingWrite>* deferred_writes_ = nullptr;
  size_t deferred_run_ = 0;
  void write_files(const std::vector<PendingWrite>& writes,
                   const std::function<void(size_t, const std::string&)>& failed);
  bool big_fetch_ = false;  // bring every candidate back (ties beyond the first copy)
  // batched group-by launch shapes by workload signature (autotuned), and the last used
  std::map<std::string, alk_gb_tuning> gb_tune_;
  alk_gb_tuning last_tuning_{};
  bool autotune_ = true;
  alk_gb_tuning fixed_tuning_{};  // consumer_warps 0: not fixed
  int groupby_mode_ = 0;
  static constexpr uint64_t kHashGroupsMax = 1ull << 22;
  uint64_t expected_groups(Var* a, const std::vector<std::string>& group_cols, uint64_t n);

  // ---- learned cardinality estimator
  bool card_record_ = false, card_use_ = false;
  alk_mlp* card_mlp_ = nullptr;
  std::vector<float> card_x_, card_y_, card_m_;  // records: features, targets, target masks
  std::map<std::string, std::vector<std::array<float, 16>>> card_hist_;  // "table.column" -> per segment
  const std::vector<std::array<float, 16>>& card_hist(const ScanPlan& p, const std::vector<alk_colseg>& cs,
                                                      uint32_t slot);
  std::vector<float> card_features(const CardStage& st);
  void card_record(const CardStage& st);
  // Estimated survivors (after the probe) and distinct keys of a stage; false when the
  // estimator is off or untrained.
  bool card_estimate(const CardStage& st, uint64_t* hits, uint64_t* keys);

  friend struct Planner;
};

}  // namespace alk
