// C entry points of the embedding layer: alenkaInit / alenkaExecute / alenkaClose /
// execute_file (alenka.h:30-35, bison.y:295-515) and the explicit session API.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "engine.h"

struct alk_session {
  std::unique_ptr<alk::Engine> eng;
  std::string err;
};

namespace {
alk_session* g_session = nullptr;
bool g_verbose = false;

int open_session(const char* dir, uint32_t flags, alk_session** out) {
  try {
    auto* s = new alk_session();
    s->eng = std::make_unique<alk::Engine>(dir ? dir : ".", flags);
    *out = s;
    return ALK_OK;
  } catch (const alk::EngineError& e) {
    std::fprintf(stderr, "alenka_b200: %s\n", e.what());
    return e.code;
  }
}
}  // namespace

extern "C" {

int alk_session_open(const char* data_dir, uint32_t flags, alk_session** out) {
  if (!out) return ALK_ERR_ARG;
  *out = nullptr;
  return open_session(data_dir, flags, out);
}

int alk_session_execute(alk_session* s, const char* script) {
  if (!s || !script) return ALK_ERR_ARG;
  int rc = s->eng->execute(script);
  s->err = s->eng->error();
  return rc;
}

const char* alk_session_error(alk_session* s) { return s ? s->err.c_str() : "no session"; }

alk_stream alk_session_stream(alk_session* s) { return s ? (alk_stream)s->eng->stream() : nullptr; }

int alk_session_preload(alk_session* s, const char* table) {
  if (!s || !table) return ALK_ERR_ARG;
  int rc = s->eng->preload(table);
  s->err = s->eng->error();
  return rc;
}

int alk_session_stats(alk_session* s, alk_stats* out) {
  if (!s || !out) return ALK_ERR_ARG;
  *out = s->eng->stats();
  return ALK_OK;
}

int alk_session_set_timing(alk_session* s, int on) {
  if (!s) return ALK_ERR_ARG;
  s->eng->set_timing(on != 0);
  return ALK_OK;
}

int alk_session_execute_batch(alk_session* s, const char* const* scripts, uint32_t n) {
  if (!s || (n && !scripts)) return ALK_ERR_ARG;
  std::vector<std::string> v;
  for (uint32_t i = 0; i < n; i++) {
    if (!scripts[i]) return ALK_ERR_ARG;
    v.emplace_back(scripts[i]);
  }
  int rc = s->eng->execute_batch(v);
  s->err = s->eng->error();
  return rc;
}

int alk_session_gen_flat_resident(alk_session* s, const char* table, const uint32_t* seg_rows, uint32_t nseg,
                                  uint64_t seed, uint64_t row_base) {
  if (!s || !table || !seg_rows || nseg == 0) return ALK_ERR_ARG;
  int rc = s->eng->gen_resident_flat(table, std::vector<uint32_t>(seg_rows, seg_rows + nseg), seed, row_base);
  s->err = s->eng->error();
  return rc;
}

int alk_session_set_groupby(alk_session* s, int mode) {
  if (!s || mode < 0 || mode > 2) return ALK_ERR_ARG;
  s->eng->set_groupby_mode(mode);
  return ALK_OK;
}

int alk_session_set_plain(alk_session* s, int on) {
  if (!s) return ALK_ERR_ARG;
  s->eng->set_plain(on != 0);
  return ALK_OK;
}

int alk_session_tuning(alk_session* s, alk_gb_tuning* out, int autotune) {
  if (!s) return ALK_ERR_ARG;
  if (out) *out = s->eng->last_tuning();
  if (autotune >= 0) s->eng->set_autotune(autotune != 0);
  return ALK_OK;
}

int alk_session_set_tuning(alk_session* s, const alk_gb_tuning* shape) {
  if (!s) return ALK_ERR_ARG;
  if (shape && shape->consumer_warps && shape->consumer_warps != 4 && shape->consumer_warps != 8) return ALK_ERR_ARG;
  s->eng->set_tuning(shape ? *shape : alk_gb_tuning{});
  return ALK_OK;
}

int alk_session_card_mode(alk_session* s, int record, int use) {
  if (!s) return ALK_ERR_ARG;
  return s->eng->card_mode(record != 0, use != 0);
}

int alk_session_card_records(alk_session* s, float* h_x, float* h_y, float* h_mask, uint64_t cap, uint64_t* h_n) {
  if (!s || !h_n) return ALK_ERR_ARG;
  *h_n = s->eng->card_records(h_x, h_y, h_mask, cap);
  return ALK_OK;
}

int alk_session_card_train(alk_session* s, uint64_t first, uint64_t count, uint32_t epochs, uint32_t batch,
                           float lr, uint64_t seed, float* h_loss) {
  if (!s || batch == 0) return ALK_ERR_ARG;
  return s->eng->card_train(first, count, epochs, batch, lr, seed, h_loss);
}

int alk_session_card_predict(alk_session* s, const float* h_x, uint64_t n, float* h_y) {
  if (!s || (n && (!h_x || !h_y))) return ALK_ERR_ARG;
  try {
    s->eng->card_forward(h_x, n, h_y);
  } catch (const alk::EngineError& e) {
    return e.code;
  }
  return ALK_OK;
}

int alk_session_card_save(alk_session* s, const char* path) {
  if (!s || !path) return ALK_ERR_ARG;
  int rc = s->eng->card_save(path);
  s->err = s->eng->error();
  return rc;
}

int alk_session_card_load(alk_session* s, const char* path) {
  if (!s || !path) return ALK_ERR_ARG;
  int rc = s->eng->card_load(path);
  s->err = s->eng->error();
  return rc;
}

int alk_session_card_forget(alk_session* s) {
  if (!s) return ALK_ERR_ARG;
  s->eng->card_forget();
  return ALK_OK;
}

void alk_session_close(alk_session* s) { delete s; }

// The reference's flags (bison.y:306-331): -l MB (segment size for stores), -v,
// -delta, -ssd, -precision N, -i. Only -v changes this engine's behaviour; the data
// directory is the current directory as in the reference.
void alenkaInit(char** av) { alk::embed_init(av); }
int alenkaExecute(char* s) { return alk::embed_execute(s); }
void alenkaClose(void) { alk::embed_close(); }
int execute_file(int ac, char** av) { return alk::embed_file(ac, av); }
}  // extern "C"

namespace alk {
void embed_init(char** av) {
  if (av)
    for (int i = 0; av[i]; i++)
      if (std::strcmp(av[i], "-v") == 0) g_verbose = true;
  if (!g_session) open_session(".", ALK_SESSION_RESIDENT, &g_session);
}

int embed_execute(char* s) {
  if (!g_session) embed_init(nullptr);
  if (!g_session || !s) return 1;
  int rc = g_session->eng->execute(s);
  if (rc != ALK_OK) std::fprintf(stderr, "alenka_b200: %s\n", g_session->eng->error().c_str());
  return rc == ALK_OK ? 0 : 1;
}

void embed_close() {
  delete g_session;
  g_session = nullptr;
}

// The engine behind the embedding API (alenkaInit's session over the current directory,
// opened on first use). The reference front end's emit_* boundary runs its scripts here.
Engine* embedding_engine() {
  if (!g_session) embed_init(nullptr);
  return g_session ? g_session->eng.get() : nullptr;
}

int embed_file(int ac, char** av) {
  if (ac < 2) return 1;
  std::ifstream f(av[ac - 1]);
  if (!f) {
    std::perror(av[ac - 1]);
    return 1;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  std::string script = ss.str();
  for (int i = 1; i < ac - 1; i++)
    if (std::strcmp(av[i], "-v") == 0) g_verbose = true;
  alk_session* s = nullptr;
  if (open_session(".", 0, &s) != ALK_OK) return 1;
  int rc = s->eng->execute(script);
  if (rc != ALK_OK) std::fprintf(stderr, "alenka_b200: %s\n", s->eng->error().c_str());
  delete s;
  return rc == ALK_OK ? 0 : 1;
}
}  // namespace alk

// Text rendering of the parsed statements and their queues (front-end tests).
extern "C" int alk_parse_dump(const char* script, char* out, int out_len) {
  std::vector<alk::Statement> sts;
  std::string err;
  if (!alk::parse_script(script ? script : "", sts, err)) {
    if (out && out_len > 0) std::snprintf(out, (size_t)out_len, "ERROR %s", err.c_str());
    return ALK_ERR_PARSE;
  }
  static const char* kinds[] = {"FILTER", "SELECT", "JOIN", "ORDER", "STORE", "STORE_BINARY", "DISPLAY", "LOAD", "OTHER", "CREATE_BITMAP_INDEX"};
  std::string s;
  for (auto& st : sts) {
    s += kinds[(int)st.kind];
    s += " s=" + st.s + " f=" + st.f + " grp=" + std::to_string(st.grp_cnt) + " sep=" + st.sep + "\n type:";
    for (auto& x : st.op_type) s += " " + x;
    s += "\n value:";
    for (auto& x : st.op_value) s += " " + x;
    s += "\n nums:";
    for (auto x : st.op_nums) s += " " + std::to_string(x);
    s += "\n prec:";
    for (auto x : st.op_nums_precision) s += " " + std::to_string(x);
    s += "\n join:";
    for (size_t i = 0; i < st.op_join.size(); i++) s += " " + st.op_join[i] + "/" + std::string(1, st.join_type[i]);
    s += " sel=" + std::to_string(st.sel_count) + " tabs=" + std::to_string(st.join_tab_cnt) + " and:";
    for (auto& kv : st.join_and_cnt) s += " " + std::to_string(kv.first) + "=" + std::to_string(kv.second);
    if (!st.index_args.empty()) {
      s += "\n index:";
      for (auto& x : st.index_args) s += " " + x;
    }
    s += "\n";
  }
  if (out && out_len > 0) std::snprintf(out, (size_t)out_len, "%s", s.c_str());
  return (int)s.size() < out_len ? ALK_OK : ALK_ERR_OVERFLOW;
}

// Segment writer (the store side of the format): FOR, or FOR-delta when delta is set and
// the values are sorted, exactly as pfor_compress / pfor_delta_compress lay them out
// (compress.cu:271-527). Writes the whole segment file image to out.
extern "C" int alk_encode_segment(const int64_t* values, uint32_t n, int delta, uint8_t* out, size_t cap,
                                  size_t* out_len) {
  if (!values || !out_len || n == 0) return ALK_ERR_ARG;
  alk::SegMeta m;
  std::vector<uint8_t> payload;
  bool sorted = true;
  for (uint32_t i = 1; i < n && sorted; i++) sorted = values[i - 1] <= values[i];
  if (delta && sorted) alk::encode_delta(values, n, m, payload);
  else alk::encode_for(values, n, m, payload);
  std::vector<uint8_t> img = alk::segment_image(m, payload);
  *out_len = img.size();
  if (img.size() > cap || !out) return ALK_ERR_OVERFLOW;
  std::memcpy(out, img.data(), img.size());
  return ALK_OK;
}
