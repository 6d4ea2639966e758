// Alenka script front end. The token rules follow fl.l:38-133 (case-insensitive
// keywords, longest match, signed numeric literals), the grammar and operator
// precedence follow bison.y:39-287, and each grammar action pushes onto the
// statement's queues exactly what the matching emit_* helper pushes
// (operators.cu:62-360).
#include "script.h"

#include <cctype>
#include <cstdlib>
#include <stdexcept>

namespace alk {
namespace {

enum class T {
  End, Name, String, Filename, IntNum, Decimal, Approx, Bool, Assign, Equal, NonEqual,
  Comparison, And, Or, Kw, Punct
};

struct Tok {
  T t = T::End;
  std::string text;  // name / keyword (upper) / literal text
  int64_t ival = 0;
  int sub = 0;       // COMPARISON subtoken, punct char
  int line = 1;
};

const char* kKeywords[] = {
    "LOAD", "FILTER", "DESC", "ASC", "ORDER", "BY", "JOIN", "STORE", "INTO", "GROUP", "AS",
    "SELECT", "USING", "COUNT", "SUM", "AVG", "MIN", "MAX", "LIMIT", "ON", "BINARY", "DISTINCT",
    "LEFT", "RIGHT", "OUTER", "SEMI", "ANTI", "SORT", "SEGMENTS", "PRESORTED", "INSERT", "WHERE",
    "DISPLAY", "CASE", "WHEN", "THEN", "ELSE", "END", "SHOW", "TABLES", "TABLE", "DESCRIBE",
    "DROP", "DELETE", "FROM", "LIKE", "CREATE", "INDEX", "YEAR", "MONTH", "DAY", "CAST_TO_INT",
    "APPEND", "NO", "ENCODING", "PARTITION"};  // no INTERVAL: fl.l has no such token

struct SyntaxError : std::runtime_error {
  int line;
  SyntaxError(int l, const std::string& m) : std::runtime_error(m), line(l) {}
};

class Lexer {
 public:
  explicit Lexer(const std::string& s) : s_(s) {}
  std::vector<Tok> run() {
    std::vector<Tok> out;
    while (true) {
      Tok t = next();
      out.push_back(t);
      if (t.t == T::End) break;
    }
    return out;
  }

 private:
  const std::string& s_;
  size_t p_ = 0;
  int line_ = 1;

  static std::string upper(std::string x) {
    for (auto& c : x) c = (char)std::toupper((unsigned char)c);
    return x;
  }
  bool digit(size_t i) const { return i < s_.size() && std::isdigit((unsigned char)s_[i]); }

  // Longest numeric match at p_ among the INTNUM / DECIMAL1 / APPROXNUM rules (fl.l:96-103).
  bool number(Tok& t) {
    size_t i = p_;
    if (i < s_.size() && s_[i] == '-') i++;
    size_t start_digits = i;
    while (digit(i)) i++;
    bool int_digits = i > start_digits;
    bool dec = false;
    if (i < s_.size() && s_[i] == '.') {
      size_t j = i + 1;
      while (digit(j)) j++;
      if (int_digits || j > i + 1) {
        dec = true;
        i = j;
      }
    }
    if (!int_digits && !dec) return false;
    bool approx = false;
    if (i < s_.size() && (s_[i] == 'E' || s_[i] == 'e')) {
      size_t j = i + 1;
      if (j < s_.size() && (s_[j] == '+' || s_[j] == '-')) j++;
      size_t k = j;
      while (digit(k)) k++;
      if (k > j) {
        approx = true;
        i = k;
      }
    }
    std::string txt = s_.substr(p_, i - p_);
    // [0-9]+(HOUR|MINUTE|...) is a STRING token (fl.l:104)
    if (!approx && !dec && txt[0] != '-') {
      static const char* units[] = {"MSECOND", "SECOND", "MINUTE", "HOUR", "DAY", "MONTH", "YEAR"};
      for (const char* u : units) {
        size_t L = std::char_traits<char>::length(u);
        if (upper(s_.substr(i, L)) == u) {
          t.t = T::String;
          t.text = s_.substr(p_, i - p_ + L);
          p_ = i + L;
          return true;
        }
      }
    }
    p_ = i;
    t.text = txt;
    if (approx) {
      t.t = T::Approx;
    } else if (dec) {
      t.t = T::Decimal;
    } else {
      t.t = T::IntNum;
      t.ival = std::atoll(txt.c_str());
    }
    return true;
  }

  Tok next() {
    Tok t;
    while (p_ < s_.size()) {
      char c = s_[p_];
      if (c == '\n') { line_++; p_++; continue; }
      if (c == ' ' || c == '\t' || c == '\r') { p_++; continue; }
      break;
    }
    t.line = line_;
    if (p_ >= s_.size()) return t;
    char c = s_[p_];
    if (std::isalpha((unsigned char)c)) {
      size_t i = p_;
      while (i < s_.size() && (std::isalnum((unsigned char)s_[i]) || s_[i] == '_')) i++;
      std::string w = s_.substr(p_, i - p_);
      std::string u = upper(w);
      p_ = i;
      if (u == "DATE" && s_.compare(p_, 2, "()") == 0) {  // date() is a STRING (fl.l:105)
        p_ += 2;
        t.t = T::String;
        t.text = "date()";
        return t;
      }
      if (u == "AND") { t.t = T::And; return t; }
      if (u == "OR") { t.t = T::Or; return t; }
      if (u == "TRUE" || u == "FALSE" || u == "UNKNOWN") {
        t.t = T::Bool;
        t.ival = u == "TRUE" ? 1 : (u == "FALSE" ? 0 : -1);
        return t;
      }
      for (const char* k : kKeywords)
        if (u == k) {
          t.t = T::Kw;
          t.text = u;
          return t;
        }
      t.t = T::Name;
      t.text = w;
      return t;
    }
    if (std::isdigit((unsigned char)c) || c == '.' || (c == '-' && (digit(p_ + 1) || (p_ + 2 < s_.size() && s_[p_ + 1] == '.' && digit(p_ + 2))))) {
      if (number(t)) return t;
    }
    if (c == '"') {  // \"(\\.|\"\"|[^"\n])*\" (fl.l:111)
      size_t i = p_ + 1;
      while (i < s_.size()) {
        if (s_[i] == '\\' && i + 1 < s_.size()) { i += 2; continue; }
        if (s_[i] == '"' && i + 1 < s_.size() && s_[i + 1] == '"') { i += 2; continue; }
        if (s_[i] == '"') break;
        if (s_[i] == '\n') throw SyntaxError(line_, "unterminated string");
        i++;
      }
      if (i >= s_.size()) throw SyntaxError(line_, "unterminated string");
      t.t = T::String;
      t.text = s_.substr(p_, i + 1 - p_);
      p_ = i + 1;
      return t;
    }
    if (c == '\'') {  // FILENAME (fl.l:127,131)
      size_t i = p_ + 1;
      while (i < s_.size() && s_[i] != '\'' && s_[i] != '\n') i++;
      if (i >= s_.size() || s_[i] != '\'') throw SyntaxError(line_, "unterminated file name");
      t.t = T::Filename;
      t.text = s_.substr(p_ + 1, i - p_ - 1);
      p_ = i + 1;
      return t;
    }
    auto two = s_.substr(p_, 3);
    struct Op { const char* s; T t; int sub; };
    static const Op ops[] = {{"<=>", T::Comparison, 12}, {"&&", T::And, 0}, {"||", T::Or, 0},
                             {":=", T::Assign, 0},      {"==", T::Comparison, 4},
                             {">=", T::Comparison, 6},  {"<=", T::Comparison, 5},
                             {"!=", T::Comparison, 3},  {"<>", T::NonEqual, 0},
                             {">", T::Comparison, 2},   {"<", T::Comparison, 1},
                             {"=", T::Equal, 0}};
    for (const Op& o : ops) {
      size_t L = std::char_traits<char>::length(o.s);
      if (s_.compare(p_, L, o.s) == 0) {
        t.t = o.t;
        t.sub = o.sub;
        p_ += L;
        return t;
      }
    }
    static const std::string punct = "-+&~|^/%*(),.;:!{}";
    if (punct.find(c) != std::string::npos) {
      t.t = T::Punct;
      t.sub = c;
      p_++;
      return t;
    }
    p_++;  // unknown characters are skipped (fl.l:133)
    return next();
  }
};

class Parser {
 public:
  Parser(std::vector<Tok> toks) : t_(std::move(toks)) {}

  void run(std::vector<Statement>& out) {
    while (peek().t != T::End) {
      Statement st;
      st.line = peek().line;
      cur_ = &st;
      join_col_cnt_ = 0;
      tab_cnt_ = 0;
      statement();
      expect_punct(';');
      out.push_back(std::move(st));
    }
  }

 private:
  std::vector<Tok> t_;
  size_t i_ = 0;
  Statement* cur_ = nullptr;
  unsigned join_col_cnt_ = 0, tab_cnt_ = 0;
  unsigned misses_ = 0;  // process-wide in the reference (operators.cu:146), never reset

  const Tok& peek(size_t k = 0) const { return t_[std::min(i_ + k, t_.size() - 1)]; }
  Tok take() { return t_[i_ < t_.size() - 1 ? i_++ : i_]; }
  [[noreturn]] void fail(const std::string& m) { throw SyntaxError(peek().line, m); }
  bool is_kw(const char* k, size_t off = 0) const { return peek(off).t == T::Kw && peek(off).text == k; }
  bool is_punct(char c, size_t off = 0) const { return peek(off).t == T::Punct && peek(off).sub == c; }
  void expect_kw(const char* k) {
    if (!is_kw(k)) fail(std::string("expected ") + k);
    take();
  }
  void expect_punct(char c) {
    if (!is_punct(c)) fail(std::string("expected '") + c + "'");
    take();
  }
  std::string expect(T ty, const char* what) {
    if (peek().t != ty) fail(std::string("expected ") + what);
    return take().text;
  }
  int64_t expect_int() {
    if (peek().t != T::IntNum) fail("expected integer");
    return take().ival;
  }

  // ---- emit_* queue helpers (operators.cu:62-360) ----
  void ty(const std::string& s) { cur_->op_type.push_back(s); }
  void val(const std::string& s) { cur_->op_value.push_back(s); }
  void emit_name(const std::string& n) { ty("NAME"); val(n); }
  void emit_number(int64_t v) {
    ty("NUMBER");
    cur_->op_nums.push_back(v);
    cur_->op_nums_precision.push_back(0);
  }
  void emit_decimal(const std::string& s) {  // operators.cu:112-127 (stoi of the digits)
    std::string d = s;
    uint32_t prec = 0;
    auto pos = d.find('.');
    if (pos != std::string::npos) {
      prec = (uint32_t)(d.size() - pos - 1);
      d.erase(pos, 1);
    }
    long v;
    try {
      v = std::stoi(d);
    } catch (...) {
      fail("decimal literal out of 32-bit range: " + s);
    }
    ty("NUMBER");
    cur_->op_nums.push_back(v);
    cur_->op_nums_precision.push_back(prec);
  }
  void emit_string(const std::string& s) {  // operators.cu:78-90
    if (!s.empty() && s[0] == '"') val(s.substr(1, s.size() - 2));
    else val(s);
    ty("STRING");
  }
  void emit_and() { ty("AND"); join_col_cnt_++; }
  void emit_eq(char kind) {  // operators.cu:153-184
    ty("JOIN");
    cur_->join_eq_type.push_back(kind);
    if (misses_ == 0) {
      cur_->join_and_cnt[tab_cnt_] = join_col_cnt_;
      misses_ = join_col_cnt_;
      join_col_cnt_ = 0;
      tab_cnt_++;
    } else {
      misses_--;
    }
  }
  void emit_cmp(int v) { ty("CMP"); cur_->op_nums.push_back(v); }
  void emit_sel_name(const std::string& s) { ty("emit sel_name"); val(s); cur_->sel_count++; }
  void emit_join_tab(const std::string& s, char tp) {
    cur_->op_join.push_back(s);
    cur_->join_tab_cnt++;
    cur_->join_type.push_back(tp);
  }

  // ---- expressions: precedence from bison.y:39-56, lowest first ----
  enum Prec { P_EQUAL = 1, P_NONEQUAL, P_OR, P_XOR, P_AND, P_DISTINCT, P_LIKE, P_NOT, P_BETWEEN,
              P_CMP, P_PIPE, P_AMP, P_SHIFT, P_ADD, P_MUL, P_POW };

  int binop_prec(const Tok& t, bool& right_assoc) const {
    right_assoc = false;
    switch (t.t) {
      case T::Equal: right_assoc = true; return P_EQUAL;
      case T::NonEqual: right_assoc = true; return P_NONEQUAL;
      case T::Or: return P_OR;
      case T::And: return P_AND;
      case T::Comparison: return P_CMP;
      case T::Kw: if (t.text == "LIKE") return P_LIKE; return 0;
      case T::Punct:
        if (t.sub == '+' || t.sub == '-') return P_ADD;
        if (t.sub == '*' || t.sub == '/' || t.sub == '%') return P_MUL;
        return 0;
      default: return 0;
    }
  }

  void expr(int min_prec = 1) {
    unary();
    while (true) {
      bool ra;
      const Tok& op = peek();
      int p = binop_prec(op, ra);
      if (p == 0 || p < min_prec) break;
      Tok o = take();
      expr(ra ? p : p + 1);
      switch (o.t) {
        case T::Equal: emit_eq('E'); break;
        case T::NonEqual: emit_eq('N'); break;
        case T::Or: ty("OR"); break;
        case T::And: emit_and(); break;
        case T::Comparison: emit_cmp(o.sub); break;
        case T::Kw: emit_cmp(7); break;  // LIKE
        case T::Punct:
          if (o.sub == '+') ty("ADD");
          else if (o.sub == '-') ty("MINUS");
          else if (o.sub == '*') ty("MUL");
          else if (o.sub == '/') ty("DIV");
          else ty("MOD");
          break;
        default: break;
      }
    }
  }

  void func(const char* opname) {
    take();
    expect_punct('(');
    expr();
    expect_punct(')');
    ty(opname);
  }

  void unary() {
    const Tok& t = peek();
    if (is_punct('!')) {
      take();
      expr(P_NOT + 1);
      ty("NOT");
      return;
    }
    if (is_kw("DISTINCT")) {
      take();
      expr(P_DISTINCT + 1);
      ty("DISTINCT");
      return;
    }
    switch (t.t) {
      case T::Name: {
        std::string n = take().text;
        if (is_punct('.') && peek(1).t == T::Name) {  // NAME '.' NAME -> FIELD
          take();
          std::string n2 = take().text;
          ty("FIELD");
          val(n + "." + n2);
        } else if (is_punct('(') && peek(1).t == T::String && peek(2).t == T::Punct && peek(2).sub == ')') {
          take();
          take();
          take();
          // emit_string_grp(NAME, STRING) (bison.y:219, operators.cu:92-96) pushes the
          // NAME as a string value; the literal goes to grp_val, unused on this path
          emit_string(n);
        } else if (is_punct('{')) {
          var_decl(n);
        } else if (is_kw("ASC")) {
          take();
          ty(n);
          val("ASC");
        } else if (is_kw("DESC")) {
          take();
          ty(n);
          val("DESC");
        } else {
          emit_name(n);
        }
        return;
      }
      case T::String: emit_string(take().text); return;
      case T::IntNum: emit_number(take().ival); return;
      case T::Decimal: emit_decimal(take().text); return;
      case T::Approx:
        ty("FLOAT");
        cur_->op_nums_f.push_back(std::atof(take().text.c_str()));
        return;
      case T::Bool: take(); return;  // emit("BOOL %d") records nothing
      case T::Punct:
        if (t.sub == '(') {
          take();
          expr();
          expect_punct(')');
          return;  // emit("EXPR") records nothing
        }
        break;
      case T::Kw:
        if (t.text == "COUNT") return func("COUNT");
        if (t.text == "SUM") return func("SUM");
        if (t.text == "AVG") return func("AVG");
        if (t.text == "MIN") return func("MIN");
        if (t.text == "MAX") return func("MAX");
        if (t.text == "YEAR") return func("YEAR");
        if (t.text == "MONTH") return func("MONTH");
        if (t.text == "DAY") return func("DAY");
        if (t.text == "CAST_TO_INT") return func("CAST");
        if (t.text == "CASE") {
          take();
          expect_kw("WHEN");
          expr();
          expect_kw("THEN");
          expr();
          expect_kw("ELSE");
          expr();
          expect_kw("END");
          cur_->op_case = true;  // emit_case sets a flag and queues nothing
          return;
        }
        break;
      default: break;
    }
    fail("unexpected token in expression");
  }

  // NAME '{' INTNUM '}' ':' NAME ['(' INTNUM [',' INTNUM] ')'] [NO ENCODING] (bison.y:182-185)
  void var_decl(const std::string& n) {
    LoadCol lc;
    lc.name = n;
    expect_punct('{');
    lc.field = (int)expect_int();
    expect_punct('}');
    expect_punct(':');
    lc.type = expect(T::Name, "type name");
    if (is_punct('(')) {
      take();
      lc.size = (int)expect_int();  // emit_varchar: the width
      if (is_punct(',')) {
        take();
        lc.size = (int)expect_int();  // emit_vardecimal: the digits after the point
      }
      expect_punct(')');
    }
    if (is_kw("NO")) {
      take();
      expect_kw("ENCODING");
      lc.no_encoding = true;
    }
    cur_->load_cols.push_back(lc);
  }

  int expr_list() {  // bison.y:223-228
    if (is_punct('*')) {
      take();
      emit_sel_name("*");
      return 1;
    }
    int n = 0;
    while (true) {
      expr();
      expect_kw("AS");
      emit_sel_name(expect(T::Name, "column alias"));
      n++;
      if (!is_punct(',')) break;
      take();
    }
    return n;
  }

  int val_list() {
    int n = 0;
    while (true) {
      expr();
      n++;
      if (!is_punct(',')) break;
      take();
    }
    return n;
  }

  int opt_group() {
    if (!is_kw("GROUP")) return 0;
    take();
    expect_kw("BY");
    return val_list();
  }

  void opt_limit() {
    if (is_kw("LIMIT")) {
      take();
      cur_->op_nums.push_back(expect_int());  // emit_limit (operators.cu:73-76)
    }
  }

  // join_list (bison.y:247-264): the innermost JOIN is recorded first.
  void join_list() {
    char tp = 'I';
    int toks = 0;
    if (is_kw("JOIN")) { toks = 1; tp = 'I'; }
    else if (is_kw("LEFT") && is_kw("ANTI", 1)) { toks = 3; tp = '3'; }
    else if (is_kw("RIGHT") && is_kw("ANTI", 1)) { toks = 3; tp = '4'; }
    else if (is_kw("LEFT") && is_kw("SEMI", 1)) { toks = 3; tp = '1'; }
    else if (is_kw("RIGHT") && is_kw("SEMI", 1)) { toks = 3; tp = '2'; }
    else if (is_kw("LEFT")) { toks = 2; tp = 'S'; }
    else if (is_kw("RIGHT")) { toks = 2; tp = 'R'; }
    else if (is_kw("OUTER")) { toks = 2; tp = 'O'; }
    else fail("expected JOIN");
    for (int k = 0; k < toks - 1; k++) take();
    expect_kw("JOIN");
    std::string name = expect(T::Name, "table name");
    expect_kw("ON");
    expr();
    bool more = is_kw("JOIN") || is_kw("LEFT") || is_kw("RIGHT") || is_kw("OUTER");
    if (more) {
      join_list();
      // nested forms map LEFT JOIN -> 'L' and RIGHT SEMI JOIN -> 'R' (bison.y:258-263)
      if (tp == 'S') tp = 'L';
      if (tp == '2') tp = 'R';
    }
    emit_join_tab(name, tp);
  }

  void sort_def() {
    if (is_kw("SORT")) {
      cur_->store_sort = true;
      take();
      expect_kw("SEGMENTS");
      expect_kw("BY");
      expect(T::Name, "column");
      if (is_kw("PARTITION")) {
        take();
        expect_kw("BY");
        expect_int();
      }
    } else if (is_kw("PRESORTED")) {
      cur_->store_sort = true;
      take();
      expect_kw("BY");
      expect(T::Name, "column");
    }
  }

  void statement() {
    Statement& st = *cur_;
    if (peek().t == T::Name && peek(1).t == T::Assign) {
      st.s = take().text;
      take();
      if (is_kw("SELECT")) {
        take();
        expr_list();
        expect_kw("FROM");
        st.f = expect(T::Name, "source name");
        if (is_kw("JOIN") || is_kw("LEFT") || is_kw("RIGHT") || is_kw("OUTER")) {
          join_list();
          // the grammar passes join_list's value (always 1) as emit_join's third argument,
          // not the GROUP BY count (bison.y:144-145, 268-275); the group names stay queued
          opt_group();
          st.grp_cnt = 1;
          st.kind = StmtKind::Join;
        } else {
          st.grp_cnt = opt_group();
          st.kind = StmtKind::Select;
        }
        return;
      }
      if (is_kw("FILTER")) {
        take();
        st.f = expect(T::Name, "source name");
        expect_kw("BY");
        expr();
        st.kind = StmtKind::Filter;
        return;
      }
      if (is_kw("ORDER")) {
        take();
        st.f = expect(T::Name, "source name");
        expect_kw("BY");
        if (!is_punct(';')) st.grp_cnt = val_list();
        st.kind = StmtKind::Order;
        return;
      }
      if (is_kw("LOAD")) {
        take();
        st.f = expect(T::Filename, "file name");
        expect_kw("USING");
        expect_punct('(');
        st.sep = expect(T::Filename, "separator");
        expect_punct(')');
        expect_kw("AS");
        expect_punct('(');
        val_list();
        expect_punct(')');
        st.kind = StmtKind::Load;
        return;
      }
      fail("expected SELECT, FILTER, ORDER or LOAD");
    }
    if (is_kw("STORE")) {
      take();
      st.s = expect(T::Name, "variable");
      expect_kw("INTO");
      st.f = expect(T::Filename, "file name");
      if (is_kw("USING")) {
        take();
        expect_punct('(');
        st.sep = expect(T::Filename, "separator");
        expect_punct(')');
        opt_limit();
        st.kind = StmtKind::Store;
        return;
      }
      if (is_kw("APPEND")) {
        take();
        st.append = true;
      }
      opt_limit();
      expect_kw("BINARY");
      sort_def();
      st.kind = StmtKind::StoreBinary;
      return;
    }
    if (is_kw("DISPLAY")) {
      take();
      st.s = expect(T::Name, "variable");
      expect_kw("USING");
      expect_punct('(');
      st.sep = expect(T::Filename, "separator");
      expect_punct(')');
      opt_limit();
      st.kind = StmtKind::Display;
      return;
    }
    // DESCRIBE / SHOW / DROP / INSERT / DELETE / CREATE: recorded with the names and
    // queues their emitters receive (bison.y:150-169), not executed here.
    st.kind = StmtKind::Other;
    if (is_kw("DESCRIBE")) {  // emit_describe_table($2)
      take();
      st.s = expect(T::Name, "table name");
      return;
    }
    if (is_kw("DROP") && is_kw("TABLE", 1)) {  // emit_drop_table($3)
      take();
      take();
      st.s = expect(T::Name, "table name");
      return;
    }
    if (is_kw("INSERT")) {  // INSERT INTO t SELECT expr_list FROM s: emit_insert($3, $7)
      take();
      expect_kw("INTO");
      st.f = expect(T::Name, "table name");
      expect_kw("SELECT");
      expr_list();
      expect_kw("FROM");
      st.s = expect(T::Name, "source name");
      return;
    }
    if (is_kw("DELETE")) {  // DELETE FROM t WHERE expr: emit_delete($3)
      take();
      expect_kw("FROM");
      st.f = expect(T::Name, "table name");
      expect_kw("WHERE");
      expr();
      return;
    }
    if (is_kw("CREATE")) {
      // CREATE INDEX name ON table ...: the emitters take (name, table, ...). The grammar's
      // CREATE INTERVAL form (bison.y:168) never parses: the lexer (fl.l) has no INTERVAL
      take();
      expect_kw("INDEX");
      st.s = expect(T::Name, "index name");
      expect_kw("ON");
      st.f = expect(T::Name, "table name");
      // the bitmap join index form (bison.y:164-165): CREATE INDEX s ON f(rtable.rcolumn)
      // FROM t1, t2 WHERE t3.lid = t4.rid; the FROM and WHERE table names are not passed on
      if (is_punct('(') && peek(1).t == T::Name && is_punct('.', 2)) {
        take();
        std::string rtable = expect(T::Name, "table name");
        expect_punct('.');
        std::string rcolumn = expect(T::Name, "column name");
        expect_punct(')');
        expect_kw("FROM");
        expect(T::Name, "table name");
        expect_punct(',');
        expect(T::Name, "table name");
        expect_kw("WHERE");
        expect(T::Name, "table name");
        expect_punct('.');
        std::string lid = expect(T::Name, "column name");
        if (peek().t != T::Equal) fail("expected =");
        take();
        expect(T::Name, "table name");
        expect_punct('.');
        std::string rid = expect(T::Name, "column name");
        st.kind = StmtKind::CreateBitmapIndex;
        st.index_args = {rtable, rcolumn, lid, rid};
      }
    }
    while (!is_punct(';') && peek().t != T::End) take();
  }
};

}  // namespace

bool parse_script(const std::string& text, std::vector<Statement>& out, std::string& err) {
  try {
    Lexer lx(text);
    Parser p(lx.run());
    p.run(out);
  } catch (const SyntaxError& e) {
    err = "line " + std::to_string(e.line) + ": " + e.what();
    return false;
  }
  return true;
}

}  // namespace alk
