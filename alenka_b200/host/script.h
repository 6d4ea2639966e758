// Alenka script front end: lexer + parser producing, per statement, the postfix
// argument queues that the reference's grammar actions fill before calling an
// emit_* operator (bison.y:127-287, fl.l:38-133, emit helpers operators.cu:62-360).
// The queues keep the reference's names and meaning:
//   op_type / op_value / op_nums / op_nums_f / op_nums_precision  (cm.h:69-77)
//   op_join / join_type / join_eq_type / sel_count / join_tab_cnt / join_and_cnt
//   (operators.cu:27-41)
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace alk {

enum class StmtKind {
  Filter,       // emit_filter(s, f)              bison.y:140
  Select,       // emit_select(s, f, grp_cnt)     bison.y:136
  Join,         // emit_join(s, f, ...)           bison.y:144
  Order,        // emit_order(s, f, e)            bison.y:142
  Store,        // emit_store(s, file, sep)       bison.y:146
  StoreBinary,  // emit_store_binary(s, file, append)  bison.y:148-150
  Display,      // emit_display(s, sep)           bison.y:156
  Load,         // emit_load (CSV)                bison.y:138
  Other,        // DESCRIBE / SHOW / DROP / INSERT / DELETE / CREATE INDEX name ON t(c)
  CreateBitmapIndex  // emit_create_bitmap_index(s, f, rtable, rcolumn, lid, rid)  bison.y:164-165
};

// A column of a LOAD's AS list (NAME{field}:type[(size[, decimals])], bison.y:182-185):
// what emit_var / emit_varchar / emit_vardecimal queue for the text-source CudaSet
// (operators.cu:239-286, cm.cu:2965-3015). size: a char column's width, a decimal
// column's digits after the point (the second number), else 0.
struct LoadCol {
  std::string name;
  int field = 0;
  std::string type;
  int size = 0;
  bool no_encoding = false;  // varchar(n) NO ENCODING: every value its own code
};

struct Statement {
  StmtKind kind = StmtKind::Other;
  std::string s;      // target variable (Store/Display: variable to write)
  std::string f;      // source variable (Store: output file)
  std::string sep;    // Store/Display separator
  int grp_cnt = 0;    // number of GROUP BY columns
  bool append = false;
  bool store_sort = false;  // STORE ... BINARY with SORT SEGMENTS BY / PRESORTED BY
  bool op_case = false;     // a CASE expression was emitted (emit_case, operators.cu:2142)
  std::vector<std::string> op_type, op_value;
  std::vector<int64_t> op_nums;
  std::vector<double> op_nums_f;
  std::vector<uint32_t> op_nums_precision;
  std::vector<std::string> op_join;
  std::vector<char> join_type, join_eq_type;
  unsigned sel_count = 0, join_tab_cnt = 0;
  std::map<unsigned, unsigned> join_and_cnt;
  std::vector<LoadCol> load_cols;  // LOAD: the AS list
  // CREATE INDEX s ON f(rtable.rcolumn) FROM f, rtable WHERE f.lid = rtable.rid:
  // {rtable, rcolumn, lid, rid}
  std::vector<std::string> index_args;
  int line = 0;
};

// Parse a whole script. Returns false and sets err ("line N: message") on a syntax error.
bool parse_script(const std::string& text, std::vector<Statement>& out, std::string& err);

}  // namespace alk
