// The reference's operator-level boundary, kept as it is so that the reference's own
// script front end drives this engine unchanged: the emit_* functions its grammar actions
// call (declared at operators.h:9-72, called from bison.y:127-287) with the same C++
// signatures, the global argument queues they fill (cm.h:66-78, operators.cu:24-41), and
// the globals the generated parser and its drivers (execute_file / alenkaExecute,
// bison.y:295-515) read or reset. Linking the reference's bison.cu + lex.yy.c + main.cu
// (and callbacks.c) against libalenka_b200.so gives its CLI and embedding API on this
// engine; include/alenka_b200_operators.h restates the declarations.
//
// Execution follows the reference's two passes. In the first pass (the parser's
// scan_state == 0) every statement-level emitter captures the queues into a statement;
// load_vars(), which both drivers call between the passes, then runs the whole script
// through the engine (so that the fused plans see the statement chain), and the second
// pass's emitters (scan_state == 1) only clear the queues. Linked without the reference's
// parser (no scan_state symbol), statements are collected and load_vars() runs them.
// Errors go through process_error -> error_cb as in the reference (operators.cu:2751).
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <map>
#include <queue>
#include <string>
#include <vector>

#include "engine.h"
#include "script.h"

using std::map;
using std::queue;
using std::string;

typedef long long int int_type;  // cm.h:56
typedef double float_type;       // cm.h:57

// Catalog entry (cm.h:661-664) and the reference's column-set class, of which this
// boundary only needs the name: the engine keeps its own variables, so varNames stays
// empty and free() is never reached through it.
struct col_data {
  unsigned int col_type;
  unsigned int col_length;
};
class CudaSet {
 public:
  void free();
};
void CudaSet::free() {}

// ---- argument queues of the grammar actions (cm.h:66-78, operators.cu:24-41) ----
queue<string> op_type;
queue<string> op_sort;
queue<string> op_presort;
queue<string> op_value;
queue<int_type> op_nums;
queue<float_type> op_nums_f;
queue<unsigned int> op_nums_precision;
queue<string> col_aliases;
string grp_val;
bool op_case = 0;
queue<string> namevars;
queue<string> typevars;
queue<int> sizevars;
queue<int> cols;
queue<char> encvars;  // emit_varchar's encoding ('N': NO ENCODING), beside the other var queues
queue<unsigned int> j_col_count;
unsigned int sel_count = 0;
unsigned int join_cnt = 0;
unsigned int distinct_cnt = 0;
unsigned int join_col_cnt = 0;
unsigned int join_tab_cnt = 0;
unsigned int tab_cnt = 0;
queue<string> op_join;
queue<char> join_type;
queue<char> join_eq_type;
unsigned int partition_count;
map<string, unsigned int> mystat;
map<unsigned int, unsigned int> join_and_cnt;
map<string, map<string, bool> > used_vars;

// ---- state the generated parser and its drivers read or reset (cm.cu:44-79,
// operators.cu:42-47, merge.cu:29) ----
size_t process_count;
size_t alloced_sz = 0;
bool verbose;
bool interactive, ssd, delta, star;
unsigned int prs;
unsigned int hash_seed;
map<string, map<string, col_data> > data_dict;
map<string, char*> index_buffers;
map<string, unsigned long long int*> idx_vals;
map<string, char*> buffers;
map<string, size_t> buffer_sizes;
size_t total_buffer_size;
queue<string> buffer_names;
void* alloced_tmp;
map<string, CudaSet*> varNames;
std::clock_t tot_disk;
bool save_dict = 0;
map<string, string> filter_var;

// Defined by the reference's parser when it is linked in (bison.y:291) and by its error
// callback file (callbacks.c:57); weak, so the library also loads on its own.
extern bool scan_state __attribute__((weak));
extern "C" void error_cb(int severity, const char* err) __attribute__((weak));

namespace alk {
Engine* embedding_engine();
}

namespace {
std::vector<alk::Statement> g_pending;  // statements of the first pass
unsigned int g_misses = 0;              // operators.cu:146, process-wide, never reset

bool second_pass() { return &scan_state != nullptr && scan_state; }

template <class T, class U>
void drain(queue<T>& q, std::vector<U>& out) {
  while (!q.empty()) {
    out.push_back((U)q.front());
    q.pop();
  }
}
}  // namespace

void clean_queues();

void process_error(const int severity, const string err) {
  string e = severity == 1 ? "(Warning) " + err : severity == 2 ? "(Fatal) " + err : "(Aborting) " + err;
  if (&error_cb != nullptr) error_cb(severity, e.c_str());
  else std::fprintf(stderr, "%s\n", e.c_str());
}

void yyerror(char* s, ...) {
  std::fprintf(stderr, "error: %s\n", s ? s : "");
  process_error(1, s ? s : "syntax error");
}

void emit(const char* s, ...) {}

namespace {
// A statement-level emitter: in the first pass the queues become a statement of the
// script; in either pass they are then cleared.
void capture(alk::StmtKind kind, const char* s, const char* f, const char* sep, int grp_cnt, bool append = false,
             bool store_sort = false) {
  if (!second_pass()) {
    alk::Statement st;
    st.kind = kind;
    st.s = s ? s : "";
    st.f = f ? f : "";
    st.sep = sep ? sep : "";
    st.grp_cnt = grp_cnt;
    st.append = append;
    st.store_sort = store_sort;
    drain(op_type, st.op_type);
    drain(op_value, st.op_value);
    drain(op_nums, st.op_nums);
    drain(op_nums_f, st.op_nums_f);
    drain(op_nums_precision, st.op_nums_precision);
    drain(op_join, st.op_join);
    drain(join_type, st.join_type);
    drain(join_eq_type, st.join_eq_type);
    st.sel_count = sel_count;
    st.join_tab_cnt = join_tab_cnt;
    st.join_and_cnt = join_and_cnt;
    st.op_case = op_case;
    if (kind == alk::StmtKind::Load)  // the AS list: emit_var / emit_varchar / emit_vardecimal
      while (!namevars.empty() && !typevars.empty() && !sizevars.empty() && !cols.empty()) {
        const bool no_enc = !encvars.empty() && encvars.front() == 'N';
        st.load_cols.push_back({namevars.front(), cols.front(), typevars.front(), sizevars.front(), no_enc});
        if (!encvars.empty()) encvars.pop();
        namevars.pop();
        typevars.pop();
        sizevars.pop();
        cols.pop();
      }
    g_pending.push_back(std::move(st));
  }
  clean_queues();
}

// A key for the engine's per-script caches: the statements' queues in text.
string script_key(const std::vector<alk::Statement>& sts) {
  string k = "frontend:";
  for (auto& st : sts) {
    k += std::to_string((int)st.kind) + "|" + st.s + "|" + st.f + "|" + st.sep + "|" + std::to_string(st.grp_cnt);
    for (auto& x : st.op_type) k += "," + x;
    for (auto& x : st.op_value) k += "," + x;
    for (auto x : st.op_nums) k += "," + std::to_string(x);
    for (auto x : st.op_nums_precision) k += "," + std::to_string(x);
    for (auto& x : st.op_join) k += "," + x;
    for (auto& c : st.load_cols) k += "," + c.name + "{" + std::to_string(c.field) + "}" + c.type + std::to_string(c.size);
    k += ";";
  }
  return k;
}
}  // namespace

// ---- expression and argument emitters (operators.cu:62-360) ----
void emit_name(const char* name) {
  op_type.push("NAME");
  op_value.push(name);
}
void emit_limit(const int val) { op_nums.push(val); }
void emit_string(const char* str) {  // the quotes of a string literal are dropped
  if (str[0] == '"') op_value.push(string(str, 1, std::strlen(str) - 2));
  else op_value.push(str);
  op_type.push("STRING");
}
void emit_string_grp(const char* str, const char* str_grp) {
  emit_string(str);
  grp_val = str_grp;
}
void emit_fieldname(const char* name1, const char* name2) {
  op_type.push("FIELD");
  op_value.push(string(name1) + "." + string(name2));
}
void emit_number(const int_type val) {
  op_type.push("NUMBER");
  op_nums.push(val);
  op_nums_precision.push(0);
}
void emit_float(const float_type val) {
  op_type.push("FLOAT");
  op_nums_f.push(val);
}
void emit_decimal(const char* str) {  // digits without the point, as a 32-bit stoi
  op_type.push("NUMBER");
  string s1(str);
  unsigned int precision = 0;
  auto pos = s1.find('.');
  if (pos != string::npos) {
    precision = (unsigned int)(s1.length() - pos - 1);
    s1.erase(pos, 1);
  }
  op_nums.push(std::stoi(s1));
  op_nums_precision.push(precision);
}
void emit_mul() { op_type.push("MUL"); }
void emit_add() { op_type.push("ADD"); }
void emit_div() { op_type.push("DIV"); }
void emit_minus() { op_type.push("MINUS"); }
void emit_and() {
  op_type.push("AND");
  join_col_cnt++;
}
void emit_or() { op_type.push("OR"); }
namespace {
void join_eq(char kind) {  // operators.cu:153-184
  op_type.push("JOIN");
  join_eq_type.push(kind);
  if (g_misses == 0) {
    join_and_cnt[tab_cnt] = join_col_cnt;
    g_misses = join_col_cnt;
    join_col_cnt = 0;
    tab_cnt++;
  } else {
    g_misses--;
  }
}
}  // namespace
void emit_eq() { join_eq('E'); }
void emit_neq() { join_eq('N'); }
void emit_distinct() {
  op_type.push("DISTINCT");
  distinct_cnt++;
}
void emit_year() { op_type.push("YEAR"); }
void emit_month() { op_type.push("MONTH"); }
void emit_day() { op_type.push("DAY"); }
void emit_cast() { op_type.push("CAST"); }
void emit_case() { op_case = 1; }  // operators.cu:2142: a flag, no queue entry
void emit_cmp(const int val) {
  op_type.push("CMP");
  op_nums.push(val);
}
void emit_count() { op_type.push("COUNT"); }
void emit_sum() { op_type.push("SUM"); }
void emit_average() { op_type.push("AVG"); }
void emit_min() { op_type.push("MIN"); }
void emit_max() { op_type.push("MAX"); }
void emit_sel_name(const char* name) {
  op_type.push("emit sel_name");
  op_value.push(name);
  sel_count++;
}
void emit_join_tab(const char* s, const char tp) {
  op_join.push(s);
  join_tab_cnt++;
  join_type.push(tp);
}
void emit_var(const char* s, const int c, const char* f, const char* ref, const char* ref_name) {
  namevars.push(s);
  typevars.push(f);
  sizevars.push(0);
  cols.push(c);
  encvars.push(0);
}
void emit_var_asc(const char* s) {
  op_type.push(s);
  op_value.push("ASC");
}
void emit_var_desc(const char* s) {
  op_type.push(s);
  op_value.push("DESC");
}
void emit_varchar(const char* s, const int c, const char* f, const int d, const char* ref, const char* ref_name,
                  const char* encoding) {
  namevars.push(s);
  typevars.push(f);
  sizevars.push(d);
  cols.push(c);
  encvars.push(encoding ? encoding[0] : 0);
}
void emit_vardecimal(const char* s, const int c, const char* f, const int scale, const int precision) {
  namevars.push(s);
  typevars.push(f);
  sizevars.push(precision);
  cols.push(c);
  encvars.push(0);
}
namespace {
bool g_store_sort = false;  // SORT SEGMENTS BY / PRESORTED BY seen for the current STORE
}
void emit_sort(const char* s, const int p) {
  op_sort.push(s);
  partition_count = p;
  g_store_sort = true;
}
void emit_presort(const char* s) {
  op_presort.push(s);
  g_store_sort = true;
}

// ---- statement emitters (operators.cu:797, 1641, 1801, 2306, 2410-2552) ----
void emit_select(const char* s, const char* f, const int grp_cnt) { capture(alk::StmtKind::Select, s, f, "", grp_cnt); }
void emit_filter(char* s, char* f) { capture(alk::StmtKind::Filter, s, f, "", 0); }
void emit_join(const char* s, const char* j1, const int grp, const int start_seg, const int end_seg) {
  capture(alk::StmtKind::Join, s, j1, "", grp);
}
void emit_order(const char* s, const char* f, const int e, const int ll) { capture(alk::StmtKind::Order, s, f, "", e); }
void emit_store(const char* s, const char* f, const char* sep) { capture(alk::StmtKind::Store, s, f, sep, 0); }
void emit_store_binary(const char* s, const char* f, const bool append) {
  const bool sorted = g_store_sort;
  g_store_sort = false;
  capture(alk::StmtKind::StoreBinary, s, f, "", 0, append, sorted);
}
void emit_display(const char* s, const char* sep) { capture(alk::StmtKind::Display, s, "", sep, 0); }
void emit_load(const char* s, const char* f, const int d, const char* sep) { capture(alk::StmtKind::Load, s, f, sep, 0); }
void emit_load_binary(const char* s, const char* f, const int d) {}  // tables load on first use
void emit_group(const char* s, const char* f, const int e) { capture(alk::StmtKind::Other, s, f, "", e); }
void emit_union(const char* s, const char* f1, const char* f2) { capture(alk::StmtKind::Other, s, f1, "", 0); }
void emit_delete(const char* f) { capture(alk::StmtKind::Other, "", f, "", 0); }
void emit_insert(const char* f, const char* s) { capture(alk::StmtKind::Other, s, f, "", 0); }
void emit_show_tables() { capture(alk::StmtKind::Other, "", "", "", 0); }
void emit_describe_table(const char* table_name) { capture(alk::StmtKind::Other, table_name, "", "", 0); }
void emit_drop_table(const char* table_name) { capture(alk::StmtKind::Other, table_name, "", "", 0); }
void emit_create_bitmap_index(const char* index_name, const char* ltable, const char* rtable, const char* rcolumn,
                              const char* lid, const char* rid) {
  capture(alk::StmtKind::CreateBitmapIndex, index_name, ltable, "", 0);
  if (!second_pass() && !g_pending.empty())
    g_pending.back().index_args = {rtable ? rtable : "", rcolumn ? rcolumn : "", lid ? lid : "", rid ? rid : ""};
}
void emit_create_index(const char* index_name, const char* table, const char* column) {
  capture(alk::StmtKind::Other, index_name, table, "", 0);
}
void emit_create_interval(const char* interval_name, const char* table, const char* lcolumn, const char* rcolumn) {
  capture(alk::StmtKind::Other, interval_name, table, "", 0);
}

// operators.cu:2680-2706
void clean_queues() {
  while (!op_type.empty()) op_type.pop();
  while (!op_value.empty()) op_value.pop();
  while (!op_join.empty()) op_join.pop();
  while (!op_nums.empty()) op_nums.pop();
  while (!op_nums_f.empty()) op_nums_f.pop();
  while (!op_nums_precision.empty()) op_nums_precision.pop();
  while (!j_col_count.empty()) j_col_count.pop();
  while (!namevars.empty()) namevars.pop();
  while (!typevars.empty()) typevars.pop();
  while (!sizevars.empty()) sizevars.pop();
  while (!encvars.empty()) encvars.pop();
  while (!cols.empty()) cols.pop();
  while (!op_sort.empty()) op_sort.pop();
  while (!op_presort.empty()) op_presort.pop();
  while (!join_type.empty()) join_type.pop();
  while (!join_eq_type.empty()) join_eq_type.pop();
  op_case = 0;
  sel_count = 0;
  join_cnt = 0;
  join_col_cnt = 0;
  distinct_cnt = 0;
  join_tab_cnt = 0;
  tab_cnt = 0;
  join_and_cnt.clear();
}

// Between the two passes (operators.cu:2708): the script the first pass captured runs on
// the engine of the embedding API. A failed script reports its error as a fatal one.
void load_vars() {
  std::vector<alk::Statement> sts;
  sts.swap(g_pending);
  if (sts.empty()) return;
  alk::Engine* eng = alk::embedding_engine();
  if (!eng) {
    process_error(2, "no device session");
    return;
  }
  const string key = script_key(sts);
  if (eng->execute_statements(std::move(sts), key) != ALK_OK) process_error(2, eng->error());
}

// cm.cu:3184: the memory the reference sizes its segments to; this engine keeps whole
// tables resident and reports the device total it plans against.
size_t getFreeMem() { return (size_t)alk::Engine::kFreeMem; }

// The catalog "data.dictionary" (cm.cu:4057-4114): same file format as the engine's.
void load_col_data(map<string, map<string, col_data> >& dd, string file_name) {
  alk::DataDict d;
  string e;
  if (!alk::load_data_dict(file_name, d, e)) return;
  for (auto& t : d)
    for (auto& c : t.second) dd[t.first][c.first] = col_data{c.second.col_type, c.second.col_length};
}
void save_col_data(map<string, map<string, col_data> >& dd, string file_name) {
  alk::DataDict d;
  for (auto& t : dd)
    for (auto& c : t.second) d[t.first][c.first] = alk::ColData{c.second.col_type, c.second.col_length};
  alk::save_data_dict(file_name, d);
}

// Statements captured by the first pass, rendered as alk_parse_dump renders the engine
// parser's (front-end tests compare the two). Returns the bytes written (0 when none).
extern "C" int alk_frontend_dump(char* out, int out_len) {
  string s;
  static const char* kinds[] = {"FILTER", "SELECT", "JOIN", "ORDER", "STORE", "STORE_BINARY", "DISPLAY", "LOAD", "OTHER", "CREATE_BITMAP_INDEX"};
  for (auto& st : g_pending) {
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
    for (size_t i = 0; i < st.op_join.size(); i++) s += " " + st.op_join[i] + "/" + string(1, st.join_type[i]);
    s += " sel=" + std::to_string(st.sel_count) + " tabs=" + std::to_string(st.join_tab_cnt) + " and:";
    for (auto& kv : st.join_and_cnt) s += " " + std::to_string(kv.first) + "=" + std::to_string(kv.second);
    if (!st.index_args.empty()) {
      s += "\n index:";
      for (auto& x : st.index_args) s += " " + x;
    }
    s += "\n";
  }
  if (out && out_len > 0) std::snprintf(out, (size_t)out_len, "%s", s.c_str());
  return (int)s.size();
}

// Drops the statements captured so far (front-end tests that only render them).
extern "C" void alk_frontend_reset(void) {
  g_pending.clear();
  clean_queues();
}
