// Operator execution of the host engine: emit_filter / emit_select / emit_join /
// emit_order / emit_store semantics on top of the operator-level C ABI.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <thread>
#include <string_view>
#include <charconv>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <numeric>

#include "../csrc/internal.h"
#include "engine.h"

namespace alk {

namespace {
void check(int rc, const char* what) {
  if (rc == ALK_OK) return;
  std::string m = std::string(what) + " failed (status " + std::to_string(rc) + ")";
  if (rc == ALK_ERR_CUDA || rc == ALK_ERR_NOMEM) m += std::string(": ") + alk::last_cuda_error();
  throw EngineError(rc, m);
}
void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw EngineError(e == cudaErrorMemoryAllocation ? ALK_ERR_NOMEM : ALK_ERR_CUDA,
                      std::string(what) + ": " + cudaGetErrorString(e));
}
[[noreturn]] void unsupported(const std::string& m) { throw EngineError(ALK_ERR_UNSUPPORTED, m); }
int64_t pow10u(uint32_t p) { return (int64_t)(unsigned int)std::pow(10.0, (double)p); }
int64_t wmul(int64_t a, int64_t b) { return (int64_t)((uint64_t)a * (uint64_t)b); }
int64_t wadd(int64_t a, int64_t b) { return (int64_t)((uint64_t)a + (uint64_t)b); }
int64_t wsub(int64_t a, int64_t b) { return (int64_t)((uint64_t)a - (uint64_t)b); }
int64_t sdiv(int64_t a, int64_t b) { return b == 0 ? 0 : (b == -1 ? (int64_t)(0 - (uint64_t)a) : a / b); }
int64_t arith(const std::string& op, int64_t a, int64_t b) {
  if (op == "MUL") return wmul(a, b);
  if (op == "ADD") return wadd(a, b);
  if (op == "MINUS") return wsub(a, b);
  return sdiv(a, b);
}
uint32_t precision_func(uint32_t& p1, uint32_t& p2, const std::string& op) {  // zone_map.cu:668-712
  if (op != "DIV") {
    if (op != "MUL") {
      uint32_t res = p1;
      if (p1 > p2) {
        p2 = p1 - p2;
        p1 = 0;
      } else {
        p1 = p2 - p1;
        p2 = 0;
      }
      return res;
    }
    uint32_t res = p1 + p2;
    p1 = p2 = 0;
    return res;
  }
  if (p1 == p2) {
    p1 = p1 + 4;
    p2 = 0;
    return p1;
  }
  if (p1 > p2) {
    p1 = p1 + (p1 - p2) + 4;
    p2 = 0;
    return p1;
  }
  p2 = p2 + (p2 - p1) + 4;
  p1 = 0;
  return p2;
}
template <class S>
auto pop(S& s) {
  if (s.empty()) throw EngineError(ALK_ERR_UNSUPPORTED, "malformed postfix program (stack underflow)");
  auto x = s.back();
  s.pop_back();
  return x;
}
DevBufP mkbuf(size_t bytes, cudaStream_t s) { return std::make_shared<DevBuf>(bytes, s); }

// Expression tree built by the symbolic select(): columns, constants, binary
// arithmetic, and aggregate results (Agg leaves refer to an aggregate slot).
struct Ast;
using AstP = std::shared_ptr<Ast>;
struct Ast {
  enum K { Col, Const, Bin, Agg } k = Const;
  std::string col;
  int64_t v = 0;
  uint8_t op = 0;
  AstP l, r;
  int agg = -1;
};
AstP mk_col(const std::string& c) {
  auto a = std::make_shared<Ast>();
  a->k = Ast::Col;
  a->col = c;
  return a;
}
AstP mk_const(int64_t v) {
  auto a = std::make_shared<Ast>();
  a->k = Ast::Const;
  a->v = v;
  return a;
}
AstP mk_bin(uint8_t op, AstP l, AstP r) {
  auto a = std::make_shared<Ast>();
  a->k = Ast::Bin;
  a->op = op;
  a->l = std::move(l);
  a->r = std::move(r);
  return a;
}
uint8_t vm_op(const std::string& op) {
  if (op == "MUL") return ALK_OP_MUL;
  if (op == "ADD") return ALK_OP_ADD;
  if (op == "MINUS") return ALK_OP_SUB;
  return ALK_OP_DIV;
}
bool has_agg(const AstP& a) {
  if (!a) return false;
  if (a->k == Ast::Agg) return true;
  return has_agg(a->l) || has_agg(a->r);
}
bool has_col(const AstP& a) {
  if (!a) return false;
  if (a->k == Ast::Col) return true;
  return has_col(a->l) || has_col(a->r);
}
// CudaSet::op(int_type* column1, int_type d, ...) (cm.cu:2480-2556) as a tree.
AstP ast_op_const(AstP c, int64_t d, const std::string& op, bool reverse, uint32_t p1, uint32_t p2) {
  int64_t d1 = (int64_t)(unsigned int)d;
  if (p2) d = wmul(d, pow10u(p2));
  if (!reverse) {
    if (op == "MUL") return mk_bin(ALK_OP_MUL, c, mk_const(d1));
    if (!p1) return mk_bin(vm_op(op), c, mk_const(wmul(d, pow10u(p2))));
    return mk_bin(vm_op(op), mk_bin(ALK_OP_MUL, c, mk_const(pow10u(p1))), mk_const(d));
  }
  AstP x = p1 ? mk_bin(ALK_OP_MUL, c, mk_const(pow10u(p1))) : c;
  return mk_bin(vm_op(op), mk_const(d), x);
}
// CudaSet::op(int_type* column1, int_type* column2, op, 0, p1, p2) (cm.cu:2559-2600)
AstP ast_op_vec(AstP c1, AstP c2, const std::string& op, uint32_t p1, uint32_t p2) {
  if (op == "MUL") return mk_bin(ALK_OP_MUL, c1, c2);
  AstP x = p1 ? mk_bin(ALK_OP_MUL, c1, mk_const(pow10u(p1))) : c1;
  AstP y = p2 ? mk_bin(ALK_OP_MUL, c2, mk_const(pow10u(p2))) : c2;
  return mk_bin(vm_op(op), x, y);
}

// Compile a tree into a register program; leaves are looked up by leaf(name or agg).
struct Compiler {
  alk_program p{};
  uint32_t nconst = 0, live = 0;
  std::vector<std::string> slots;  // column slots (names or "#agg<i>")
  Compiler() { std::memset(&p, 0, sizeof(p)); }
  uint16_t slot(const std::string& n) {
    auto it = std::find(slots.begin(), slots.end(), n);
    if (it != slots.end()) return (uint16_t)(it - slots.begin());
    slots.push_back(n);
    if (slots.size() > 16) unsupported("expression reads more than 16 columns");
    return (uint16_t)(slots.size() - 1);
  }
  uint16_t konst(int64_t v) {
    for (uint32_t i = 0; i < nconst; i++)
      if (p.consts[i] == v) return (uint16_t)i;
    if (nconst >= ALK_MAX_CONST) unsupported("expression has too many constants");
    p.consts[nconst] = v;
    return (uint16_t)nconst++;
  }
  // returns (kind, idx)
  std::pair<uint8_t, uint16_t> gen(const AstP& a) {
    switch (a->k) {
      case Ast::Col: return {ALK_K_COL, slot(a->col)};
      case Ast::Agg: return {ALK_K_COL, slot("#agg" + std::to_string(a->agg))};
      case Ast::Const: return {ALK_K_CONST, konst(a->v)};
      default: break;
    }
    auto x = gen(a->l);
    auto y = gen(a->r);
    if (x.first == ALK_K_REG) live &= ~(1u << x.second);
    if (y.first == ALK_K_REG) live &= ~(1u << y.second);
    uint32_t r = 0;
    while (r < ALK_MAX_REGS && ((live >> r) & 1)) r++;
    if (r >= ALK_MAX_REGS) unsupported("expression needs more than 8 registers");
    live |= 1u << r;
    if (p.n_instr >= ALK_MAX_INSTR) unsupported("expression too long");
    alk_instr& in = p.ins[p.n_instr++];
    in.op = a->op;
    in.dst = (uint8_t)r;
    in.ka = x.first;
    in.a = x.second;
    in.kb = y.first;
    in.b = y.second;
    return {ALK_K_REG, (uint16_t)r};
  }
  alk_program finish(const AstP& a) {
    auto res = gen(a);
    if (res.first != ALK_K_REG) {
      alk_instr& in = p.ins[p.n_instr++];
      in.op = ALK_OP_MOV;
      in.dst = 0;
      in.ka = in.kb = res.first;
      in.a = in.b = res.second;
      res = {ALK_K_REG, 0};
    }
    p.result = res.second;
    return p;
  }
};

struct AggSpec {
  uint8_t kind = ALK_AGG_SUM;  // SUM for SUM and AVG
  AstP input;                  // null for COUNT
};
struct OutSpec {
  std::string name;
  int grp_type = 3;  // 0 COUNT, 1 AVG, 2 SUM, 3 none, 4 MIN, 5 MAX (select.cu:838-860)
  int col_type = 0;  // 0 number, 1 field, 2 vector
  int64_t num = 0;
  std::string field;
  AstP vec;
  uint32_t prec = 0;
};

// Symbolic select() (select.cu:359-952): the same stack discipline, producing output
// column specifications and the aggregate list.
void compile_select(Statement& st, Var* a, bool grouped, std::vector<OutSpec>& outs, std::vector<AggSpec>& aggs,
                    bool& one_line) {
  std::vector<std::string> et, ev;
  std::vector<AstP> evec;
  std::vector<int64_t> en;
  std::vector<uint32_t> ep;
  size_t iv = 0, in = 0, ip = 0;  // op_value, op_nums, op_nums_precision positions
  one_line = false;
  auto is_col = [&](const std::string& s) { return a->has(s); };
  auto get_dec = [&](const std::string& s) -> uint32_t { return is_col(s) ? a->meta[s].dz : pop(ep); };
  auto get_vec = [&](const std::string& s) -> AstP { return is_col(s) ? mk_col(s) : pop(evec); };
  std::string grp_type = "NULL";
  for (auto& ss : st.op_type) {
    if (ss == "emit sel_name") {
      OutSpec o;
      o.name = st.op_value[iv++];
      const std::string& g = grp_type;
      o.grp_type = g == "COUNT" ? 0 : g == "AVG" ? 1 : g == "SUM" ? 2 : g == "MIN" ? 4 : g == "MAX" ? 5 : 3;
      int kinds = 0;
      if (!en.empty()) {
        o.col_type = 0;
        o.num = pop(en);
        o.prec = pop(ep);
        kinds++;
      }
      if (!ev.empty() && ev.back() != "") {
        o.col_type = 1;
        o.field = pop(ev);
        o.prec = a->meta[o.field].dz;
        kinds++;
      }
      if (!evec.empty()) {
        o.col_type = 2;
        o.vec = pop(evec);
        o.prec = pop(ep);
        pop(ev);
        kinds++;
      }
      if (kinds != 1) unsupported("select item " + o.name + " does not reduce to one value");
      outs.push_back(o);
      continue;
    }
    grp_type = "NULL";
    if (ss == "DISTINCT" || ss == "YEAR" || ss == "MONTH" || ss == "DAY" || ss == "CAST" || ss == "CASE")
      unsupported(ss + " in a select list");
    if (ss == "COUNT" || ss == "SUM" || ss == "AVG" || ss == "MIN" || ss == "MAX") {
      if (!grouped) one_line = true;
      grp_type = ss;
      pop(et);
      std::string s1v = pop(ev);
      AggSpec ag;
      if (ss == "COUNT") {
        ag.kind = ALK_AGG_COUNT;
      } else {
        ag.kind = ss == "MIN" ? ALK_AGG_MIN : (ss == "MAX" ? ALK_AGG_MAX : ALK_AGG_SUM);
        if (!is_col(s1v)) {
          ag.input = pop(evec);
          if (ss != "SUM") ep.push_back(pop(ep));
        } else {
          ag.input = mk_col(s1v);
          ep.push_back(a->meta[s1v].dz);
        }
        if (has_agg(ag.input)) unsupported("nested aggregate");
      }
      if (ss == "COUNT") ep.push_back(0);
      auto leaf = std::make_shared<Ast>();
      leaf->k = Ast::Agg;
      leaf->agg = (int)aggs.size();
      aggs.push_back(ag);
      evec.push_back(leaf);
      et.push_back("NAME");
      ev.push_back("");
      continue;
    }
    if (ss == "NAME" || ss == "NUMBER") {
      et.push_back(ss);
      if (ss == "NUMBER") {
        en.push_back(st.op_nums[in]);
        ep.push_back(st.op_nums_precision[ip++]);
        in++;
      } else {
        ev.push_back(st.op_value[iv++]);
      }
      continue;
    }
    if (ss == "MUL" || ss == "ADD" || ss == "DIV" || ss == "MINUS") {
      std::string s1 = pop(et), s2 = pop(et);
      if (s1 == "NUMBER" && s2 == "NUMBER") {
        int64_t n1 = pop(en), n2 = pop(en);
        uint32_t p1 = pop(ep), p2 = pop(ep);
        ep.push_back(precision_func(p1, p2, ss));
        if (p1) n1 = wmul(n1, pow10u(p1));
        if (p2) n2 = wmul(n2, pow10u(p2));
        evec.push_back(mk_const(arith(ss, n1, n2)));  // top operand first (select.cu:727-736)
        et.push_back("NAME");
        ev.push_back("");
      } else if (s1 == "NAME" && s2 == "NUMBER") {
        std::string v = pop(ev);
        int64_t n1 = pop(en);
        uint32_t p1 = pop(ep);
        uint32_t p2 = get_dec(v);
        AstP t = get_vec(v);
        ep.push_back(precision_func(p2, p1, ss));
        et.push_back("NAME");
        ev.push_back("");
        evec.push_back(ast_op_const(t, n1, ss, true, p2, p1));
      } else if (s1 == "NUMBER" && s2 == "NAME") {
        int64_t n1 = pop(en);
        std::string v = pop(ev);
        uint32_t p1 = pop(ep);
        uint32_t p2 = get_dec(v);
        AstP t = get_vec(v);
        ep.push_back(precision_func(p2, p1, ss));
        et.push_back("NAME");
        ev.push_back("");
        evec.push_back(ast_op_const(t, n1, ss, false, p2, p1));
      } else if (s1 == "NAME" && s2 == "NAME") {
        std::string v1 = pop(ev), v2 = pop(ev);
        AstP t1 = get_vec(v1);
        AstP t = get_vec(v2);
        uint32_t p1 = get_dec(v1), p2 = get_dec(v2);
        ep.push_back(precision_func(p1, p2, ss));
        et.push_back("NAME");
        ev.push_back("");
        evec.push_back(ast_op_vec(t, t1, ss, p2, p1));
      } else {
        unsupported("arithmetic on " + s1 + "/" + s2 + " in a select list");
      }
      continue;
    }
    unsupported("token " + ss + " in a select list");
  }
}

struct GroupOut {
  uint64_t g = 0;
  std::vector<DevBufP> keys, vals;
  DevBufP first;
};
}  // namespace

// One SELECT's state between its aggregation and its output columns; for the dense
// (batched) group-by also the scan and the accumulators.
struct SelectCtx {
  Statement* st = nullptr;
  Var* a = nullptr;
  int grp_cnt = 0;
  std::vector<std::string> group_cols;
  std::vector<OutSpec> outs;
  std::vector<AggSpec> aggs;
  size_t cycles = 1;
  GroupOut G;
  std::vector<int64_t*> okeys;
  const Rows* R = nullptr;
  std::unique_ptr<Var> out;
  // dense group-by
  ScanPlan plan;
  std::vector<alk_colseg> cs;
  alk_gb_query q{};
  size_t acc_words = 0;       // accumulators: slots x (aggregates + 1)
  std::vector<int64_t> hacc;  // the accumulators on the host
  std::vector<uint64_t> seg_rows;
  std::vector<int64_t> kmin, kspan;
};

// ------------------------------------------------------------------ FILTER
// emit_filter (operators.cu:2306-2408): lazy; a filter of a filter appends an AND.
void Engine::emit_filter(Statement& st) {
  Var* a = var(st.f);
  auto b = std::make_unique<Var>();
  b->kind = Var::Filtered;
  b->name = st.s;
  b->columnNames = a->columnNames;
  b->meta = a->meta;
  b->fil_type = st.op_type;
  b->fil_value = st.op_value;
  b->fil_nums = st.op_nums;
  b->fil_prec = st.op_nums_precision;
  if (a->kind == Var::Filtered) {
    b->source = a->source;
    b->fil_value.insert(b->fil_value.end(), a->fil_value.begin(), a->fil_value.end());
    b->fil_type.insert(b->fil_type.end(), a->fil_type.begin(), a->fil_type.end());
    b->fil_type.push_back("AND");
    b->fil_nums.insert(b->fil_nums.end(), a->fil_nums.begin(), a->fil_nums.end());
    b->fil_prec.insert(b->fil_prec.end(), a->fil_prec.begin(), a->fil_prec.end());
  } else if (a->kind == Var::Base) {
    b->source = st.f;
  } else {
    unsupported("FILTER over a materialized result");
  }
  vars_[st.s] = std::move(b);
}

// ------------------------------------------------------------------ SELECT
// emit_select (operators.cu:1801-2084) as one global pass: fused scan, expression
// evaluation, hash aggregation, then the reference's output order (key order for a
// single-segment source, MurmurHash64A order of the group keys for a multi-segment
// source, merge.cu:118-203) and count_avg / count_simple (merge.cu:271-496).
void Engine::emit_select(Statement& st) {
  {
    SelectCtx c;
    if (dense_select_prepare(st, c)) {
      dense_select_run({&c});
      dense_select_finish(c);
      return;
    }
  }
  if (hash_select(st)) return;
  Var* a = var(st.f);
  const int grp_cnt = st.grp_cnt;
  std::vector<std::string> group_cols(st.op_value.end() - grp_cnt, st.op_value.end());
  for (auto& g : group_cols)
    if (!a->has(g)) unsupported("GROUP BY column " + g + " is not a column of " + st.f);
  std::vector<OutSpec> outs;
  std::vector<AggSpec> aggs;
  bool one_line = false;
  compile_select(st, a, grp_cnt != 0, outs, aggs, one_line);
  std::set<std::string> field_set;
  for (auto& v : st.op_value)
    if (a->has(v)) field_set.insert(v);
  std::vector<std::string> fields(field_set.begin(), field_set.end());
  const size_t cycles = cycle_count(a);
  Rows R = materialize(a, fields, !grp_cnt && one_line);
  auto out = std::make_unique<Var>();
  out->kind = Var::Mat;
  out->name = st.s;
  // the reference leaves the select-list order reversed when its first segment is empty
  bool first_empty = !R.seg_counts.empty() && R.seg_counts[0] == 0;
  if (R.n == 0) {
    vars_[st.s] = std::move(out);  // no segment produced rows: empty result without columns
    return;
  }
  if (first_empty) std::reverse(outs.begin(), outs.end());
  // aggregate inputs (row level)
  std::vector<DevBufP> agg_in(aggs.size());
  for (size_t k = 0; k < aggs.size(); k++) {
    if (aggs[k].kind == ALK_AGG_COUNT) continue;
    const AstP& in = aggs[k].input;
    if (in->k == Ast::Col) {
      agg_in[k] = R.col.at(in->col);
      continue;
    }
    Compiler c;
    alk_program prog = c.finish(in);
    std::vector<const int64_t*> cols;
    for (auto& sname : c.slots) cols.push_back(R.col.at(sname)->as<int64_t>());
    agg_in[k] = mkbuf(R.n * 8, stream_);
    check(alk_eval(cols.data(), (uint32_t)cols.size(), R.n, &prog, agg_in[k]->as<int64_t>(), (alk_stream)stream_),
          "expression");
  }
  // group keys: GROUP BY columns, or the source segment for aggregate-only selects
  std::vector<const int64_t*> keys;
  DevBufP segkey;
  if (grp_cnt) {
    for (auto& g : group_cols) keys.push_back(R.col.at(g)->as<int64_t>());
  } else if (one_line) {
    segkey = mkbuf(R.n * 8, stream_);
    check(alk_widen_u32(R.seg_of_row->as<uint32_t>(), R.n, segkey->as<int64_t>(), (alk_stream)stream_), "widen");
    keys.push_back(segkey->as<int64_t>());
  }
  if (keys.empty()) {
    // projection: one output row per input row
    out->n = R.n;
    for (auto& o : outs) {
      ColMeta m;
      m.dz = o.prec;
      DevBufP col;
      if (o.col_type == 1) {
        col = R.col.at(o.field);
        m.string_map = a->meta[o.field].string_map;
        m.type = 0;
      } else if (o.col_type == 2) {
        if (has_agg(o.vec)) unsupported("aggregate in a projection");
        Compiler c;
        alk_program prog = c.finish(o.vec);
        std::vector<const int64_t*> cols;
        for (auto& sname : c.slots) cols.push_back(R.col.at(sname)->as<int64_t>());
        col = mkbuf(R.n * 8, stream_);
        check(alk_eval(cols.data(), (uint32_t)cols.size(), R.n, &prog, col->as<int64_t>(), (alk_stream)stream_),
              "projection");
      } else {
        std::vector<int64_t> h(R.n, (int64_t)(int)o.num);
        col = mkbuf(R.n * 8, stream_);
        ck(cudaMemcpyAsync(col->as<void>(), h.data(), R.n * 8, cudaMemcpyHostToDevice, stream_), "const");
      }
      out->columnNames.push_back(o.name);
      out->meta[o.name] = m;
      out->data[o.name] = col;
      out->grp_type[o.name] = o.grp_type;
    }
    vars_[st.s] = std::move(out);
    return;
  }
  // hash aggregation
  std::vector<const int64_t*> vals;
  std::vector<uint8_t> kinds;
  for (size_t k = 0; k < aggs.size(); k++) {
    kinds.push_back(aggs[k].kind);
    vals.push_back(aggs[k].kind == ALK_AGG_COUNT ? nullptr : agg_in[k]->as<int64_t>());
  }
  GroupOut G;
  std::vector<int64_t*> okeys, ovals;
  for (size_t j = 0; j < keys.size(); j++) {
    G.keys.push_back(mkbuf(R.n * 8, stream_));
    okeys.push_back(G.keys.back()->as<int64_t>());
  }
  for (size_t k = 0; k < vals.size(); k++) {
    G.vals.push_back(mkbuf(R.n * 8, stream_));
    ovals.push_back(G.vals.back()->as<int64_t>());
  }
  G.first = mkbuf(R.n * 4, stream_);
  // hash or sort: the expected group count decides (groups beyond kHashGroupsMax take the
  // reference's sort-based form, which skips the sort when the rows are in key order)
  const uint64_t groups = grp_cnt ? expected_groups(a, group_cols, R.n) : R.n;
  const bool sorted_gb = groupby_mode_ == 2 || (groupby_mode_ == 0 && groups > kHashGroupsMax);
  if (timing_) cudaEventRecord(ev0_, stream_);
  if (sorted_gb) {
    int in_order = 0;
    check(alk_groupby_sort(keys.data(), (uint32_t)keys.size(), vals.data(), kinds.data(), (uint32_t)vals.size(), R.n,
                           okeys.data(), ovals.data(), G.first->as<uint32_t>(), &G.g, &in_order,
                           (alk_stream)stream_),
          "sort group-by");
    stats_.sort_groupbys++;
  } else {
    check(alk_groupby_hash(keys.data(), (uint32_t)keys.size(), vals.data(), kinds.data(), (uint32_t)vals.size(), R.n,
                           okeys.data(), ovals.data(), G.first->as<uint32_t>(), &G.g, (alk_stream)stream_),
          "hash group-by");
  }
  if (timing_) {  // the group-by's own device time (both forms synchronize before returning)
    cudaEventRecord(ev1_, stream_);
    cudaEventSynchronize(ev1_);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    stats_.hot_kernel_ms += ms;
    stats_.hot_kernel_launches += 1;
    stats_.hot_kernel_bytes += R.n * 8 * (keys.size() + vals.size());
  }
  SelectCtx c;
  c.st = &st;
  c.a = a;
  c.grp_cnt = grp_cnt;
  c.group_cols = group_cols;
  c.outs = std::move(outs);
  c.cycles = cycles;
  c.G = std::move(G);
  c.okeys = okeys;
  c.R = &R;
  c.out = std::move(out);
  select_output(c);
}

// The grouped part of emit_select (select.cu:359-952 and the merge of merge.cu): output
// order of the groups (key order for one segment, MurmurHash64A order of the key tuple
// across segments), the output columns, count_simple / count_avg finalisation.
void Engine::select_output(SelectCtx& c) {
  Statement& st = *c.st;
  Var* a = c.a;
  const int grp_cnt = c.grp_cnt;
  const std::vector<std::string>& group_cols = c.group_cols;
  std::vector<OutSpec>& outs = c.outs;
  const size_t cycles = c.cycles;
  GroupOut& G = c.G;
  std::vector<int64_t*>& okeys = c.okeys;
  std::unique_ptr<Var>& out = c.out;
  const uint64_t ng = G.g;
  // output order
  auto perm = mkbuf(ng * 4, stream_);
  if (grp_cnt && cycles > 1) {
    auto h = mkbuf(ng * 8, stream_);
    std::vector<const int64_t*> kc(okeys.begin(), okeys.end());
    check(alk_hash_tuples(kc.data(), (uint32_t)kc.size(), ng, kHashSeed, h->as<uint64_t>(), (alk_stream)stream_),
          "group hash");
    check(alk_sort_perm_u64(h->as<uint64_t>(), ng, perm->as<uint32_t>(), (alk_stream)stream_), "hash order");
  } else {
    std::vector<const int64_t*> kc(okeys.begin(), okeys.end());
    std::vector<uint8_t> desc(kc.size(), 0);
    check(alk_sort_perm(kc.data(), desc.data(), (uint32_t)kc.size(), ng, perm->as<uint32_t>(), (alk_stream)stream_),
          "key order");
  }
  auto gathered = [&](const DevBufP& src) {
    auto d = mkbuf(ng * 8, stream_);
    check(alk_gather(src->as<int64_t>(), perm->as<uint32_t>(), ng, d->as<int64_t>(), (alk_stream)stream_), "gather");
    return d;
  };
  std::vector<DevBufP> sk, sv;
  for (auto& k : G.keys) sk.push_back(gathered(k));
  for (auto& v : G.vals) sv.push_back(gathered(v));
  DevBufP sfirst;
  {
    // first input row of each group, in output order
    auto f64 = mkbuf(ng * 8, stream_);
    check(alk_widen_u32(G.first->as<uint32_t>(), ng, f64->as<int64_t>(), (alk_stream)stream_), "widen");
    sfirst = gathered(f64);
  }
  std::vector<std::string> names;
  std::vector<DevBufP> cols;
  std::vector<ColMeta> metas;
  std::vector<int> gtypes;
  for (auto& o : outs) {
    ColMeta m;
    m.dz = o.prec;
    DevBufP col;
    if (o.col_type == 1) {
      auto it = std::find(group_cols.begin(), group_cols.end(), o.field);
      if (grp_cnt && it != group_cols.end()) {
        col = sk[it - group_cols.begin()];
      } else {
        if (grp_cnt && cycles > 1) unsupported("non-key column " + o.field + " in a multi-segment GROUP BY");
        if (!c.R) unsupported("non-key column " + o.field + " in a dense GROUP BY");
        const Rows& R = *c.R;
        // value at the group's first row (segreduce gathers at grp offsets after a stable sort)
        auto idx32 = mkbuf(ng * 4, stream_);
        check(alk_narrow_u32(sfirst->as<int64_t>(), ng, idx32->as<uint32_t>(), (alk_stream)stream_), "narrow");
        col = mkbuf(ng * 8, stream_);
        check(alk_gather(R.col.at(o.field)->as<int64_t>(), idx32->as<uint32_t>(), ng, col->as<int64_t>(),
                         (alk_stream)stream_),
              "gather");
      }
      m.string_map = a->meta[o.field].string_map;
    } else if (o.col_type == 2) {
      if (has_col(o.vec)) unsupported("row-level expression in a grouped select");
      if (o.vec->k == Ast::Agg) {
        col = sv[o.vec->agg];
      } else {
        Compiler c;
        alk_program prog = c.finish(o.vec);
        std::vector<const int64_t*> cc;
        for (auto& sname : c.slots) cc.push_back(sv[std::stoi(sname.substr(4))]->as<int64_t>());
        col = mkbuf(ng * 8, stream_);
        check(alk_eval(cc.data(), (uint32_t)cc.size(), ng, &prog, col->as<int64_t>(), (alk_stream)stream_),
              "aggregate expression");
      }
    } else {
      std::vector<int64_t> h(ng, (int64_t)(int)o.num);
      col = mkbuf(ng * 8, stream_);
      ck(cudaMemcpyAsync(col->as<void>(), h.data(), ng * 8, cudaMemcpyHostToDevice, stream_), "const");
    }
    names.push_back(o.name);
    cols.push_back(col);
    metas.push_back(m);
    gtypes.push_back(o.grp_type);
  }
  if (!grp_cnt) {
    // count_simple (merge.cu:271-311) over the per-segment rows, ordered by segment
    std::vector<std::vector<int64_t>> h(cols.size(), std::vector<int64_t>(ng));
    for (size_t c = 0; c < cols.size(); c++)
      ck(cudaMemcpyAsync(h[c].data(), cols[c]->as<void>(), ng * 8, cudaMemcpyDeviceToHost, stream_), "d2h");
    ck(cudaStreamSynchronize(stream_), "sync");
    stats_.d2h_bytes += ng * 8 * cols.size();
    int64_t count = 0;
    bool have = false;
    std::vector<int64_t> res(cols.size());
    for (size_t c = 0; c < cols.size(); c++) {
      res[c] = h[c][0];
      if (gtypes[c] == 0) {
        count = 0;
        for (auto x : h[c]) count = wadd(count, x);
        res[c] = count;
        have = true;
      }
    }
    for (size_t c = 0; c < cols.size(); c++) {
      if (gtypes[c] == 1) {
        if (!have) unsupported("AVG needs a COUNT column in the same select");
        int64_t s = 0;
        for (auto x : h[c]) s = wadd(s, x);
        res[c] = sdiv(s, count);
      } else if (gtypes[c] == 2) {
        int64_t s = 0;
        for (auto x : h[c]) s = wadd(s, x);
        res[c] = s;
      }
    }
    for (size_t c = 0; c < cols.size(); c++) {
      auto d = mkbuf(8, stream_);
      ck(cudaMemcpyAsync(d->as<void>(), &res[c], 8, cudaMemcpyHostToDevice, stream_), "h2d");
      cols[c] = d;
    }
    ck(cudaStreamSynchronize(stream_), "sync");
    out->n = 1;
  } else {
    out->n = ng;
    // AVG finalisation of count_avg (merge.cu:446-458): (sum*100)/count when the scale
    // is at most 2 (scale + 2), sum/count otherwise.
    int countc = -1;
    for (size_t c = 0; c < cols.size(); c++)
      if (gtypes[c] == 0) {
        countc = (int)c;
        break;
      }
    for (size_t c = 0; c < cols.size(); c++) {
      if (gtypes[c] != 1) continue;
      if (countc < 0) unsupported("AVG needs a COUNT column in the same select");
      auto l = mk_col("s");
      auto r = mk_col("c");
      AstP e = metas[c].dz <= 2 ? mk_bin(ALK_OP_DIV, mk_bin(ALK_OP_MUL, l, mk_const(100)), r)
                                : mk_bin(ALK_OP_DIV, l, r);
      Compiler cc;
      alk_program prog = cc.finish(e);
      std::vector<const int64_t*> in;
      for (auto& sname : cc.slots) in.push_back((sname == "s" ? cols[c] : cols[countc])->as<int64_t>());
      auto d = mkbuf(ng * 8, stream_);
      check(alk_eval(in.data(), (uint32_t)in.size(), ng, &prog, d->as<int64_t>(), (alk_stream)stream_), "avg");
      cols[c] = d;
      if (metas[c].dz <= 2) metas[c].dz += 2;
      gtypes[c] = 3;
    }
  }
  for (size_t c = 0; c < cols.size(); c++) {
    out->columnNames.push_back(names[c]);
    out->meta[names[c]] = metas[c];
    out->data[names[c]] = cols[c];
    out->grp_type[names[c]] = gtypes[c];
  }
  vars_[st.s] = std::move(out);
}

// ------------------------------------------------------------------ dense group-by
namespace {
// The device register machine's arithmetic (wrapping; x / 0 = 0; INT64_MIN / -1 wraps),
// for the few rows of a dense group-by result.
int64_t host_mul(int64_t a, int64_t b) { return (int64_t)((uint64_t)a * (uint64_t)b); }
int64_t host_div(int64_t a, int64_t b) {
  if (b == 0) return 0;
  if (b == -1) return (int64_t)(0 - (uint64_t)a);
  return a / b;
}
int64_t host_apply(uint8_t op, int64_t a, int64_t b) {
  switch (op) {
    case ALK_OP_ADD: return (int64_t)((uint64_t)a + (uint64_t)b);
    case ALK_OP_SUB: return (int64_t)((uint64_t)a - (uint64_t)b);
    case ALK_OP_MUL: return host_mul(a, b);
    case ALK_OP_DIV: return host_div(a, b);
    case ALK_OP_LT: return a < b;
    case ALK_OP_GT: return a > b;
    case ALK_OP_LE: return a <= b;
    case ALK_OP_GE: return a >= b;
    case ALK_OP_EQ: return a == b;
    case ALK_OP_NE: return a != b;
    case ALK_OP_AND: return (a != 0) && (b != 0);
    case ALK_OP_OR: return (a != 0) || (b != 0);
    case ALK_OP_INSET: throw EngineError(ALK_ERR_UNSUPPORTED, "a code-set test outside a filter");
    default: return a;
  }
}
void host_eval(const alk_program& p, const std::vector<const int64_t*>& cols, uint64_t n, int64_t* out) {
  int64_t regs[ALK_MAX_REGS];
  for (uint64_t i = 0; i < n; i++) {
    for (uint32_t pc = 0; pc < p.n_instr; pc++) {
      const alk_instr& in = p.ins[pc];
      const int64_t a = in.ka == ALK_K_REG ? regs[in.a] : (in.ka == ALK_K_COL ? cols[in.a][i] : p.consts[in.a]);
      const int64_t b = in.kb == ALK_K_REG ? regs[in.b] : (in.kb == ALK_K_COL ? cols[in.b][i] : p.consts[in.b]);
      regs[in.dst] = host_apply(in.op, a, b);
    }
    out[i] = regs[p.result];
  }
}
// An aggregate input as (am * A + ac) * (bm * B + bc) in wrapping int64 arithmetic: the
// ring identities hold modulo 2^64, so this form equals the expression tree's value
// whenever the tree uses only +, - and * (no division).
struct Sym {
  int kind = 0;  // 0 constant, 1 affine term, 2 product of two affine terms
  int64_t c = 0;
  std::string a, b;
  int64_t am = 0, ac = 0, bm = 0, bc = 0;
};
int64_t u_add(int64_t x, int64_t y) { return (int64_t)((uint64_t)x + (uint64_t)y); }
int64_t u_sub(int64_t x, int64_t y) { return (int64_t)((uint64_t)x - (uint64_t)y); }
int64_t u_mul(int64_t x, int64_t y) { return (int64_t)((uint64_t)x * (uint64_t)y); }
bool sym_of(const AstP& e, Sym& out) {
  if (!e) return false;
  if (e->k == Ast::Const) {
    out = Sym{};
    out.c = e->v;
    return true;
  }
  if (e->k == Ast::Col) {
    out = Sym{};
    out.kind = 1;
    out.a = e->col;
    out.am = 1;
    return true;
  }
  if (e->k != Ast::Bin) return false;
  Sym x, y;
  if (!sym_of(e->l, x) || !sym_of(e->r, y)) return false;
  out = Sym{};
  switch (e->op) {
    case ALK_OP_ADD:
    case ALK_OP_SUB: {
      const bool sub = e->op == ALK_OP_SUB;
      if (x.kind == 0 && y.kind == 0) {
        out.c = sub ? u_sub(x.c, y.c) : u_add(x.c, y.c);
        return true;
      }
      if (x.kind == 1 && y.kind == 0) {
        out = x;
        out.ac = sub ? u_sub(x.ac, y.c) : u_add(x.ac, y.c);
        return true;
      }
      if (x.kind == 0 && y.kind == 1) {
        out = y;
        out.am = sub ? u_sub(0, y.am) : y.am;
        out.ac = sub ? u_sub(x.c, y.ac) : u_add(x.c, y.ac);
        return true;
      }
      if (x.kind == 1 && y.kind == 1 && x.a == y.a) {
        out = x;
        out.am = sub ? u_sub(x.am, y.am) : u_add(x.am, y.am);
        out.ac = sub ? u_sub(x.ac, y.ac) : u_add(x.ac, y.ac);
        return true;
      }
      return false;
    }
    case ALK_OP_MUL: {
      if (x.kind == 0 && y.kind == 0) {
        out.c = u_mul(x.c, y.c);
        return true;
      }
      if (x.kind == 0) std::swap(x, y);  // constant on the right
      if (y.kind == 0 && x.kind == 1) {
        out = x;
        out.am = u_mul(x.am, y.c);
        out.ac = u_mul(x.ac, y.c);
        return true;
      }
      if (y.kind == 0 && x.kind == 2) {
        out = x;
        out.am = u_mul(x.am, y.c);
        out.ac = u_mul(x.ac, y.c);
        return true;
      }
      if (x.kind == 1 && y.kind == 1) {
        out.kind = 2;
        out.a = x.a;
        out.am = x.am;
        out.ac = x.ac;
        out.b = y.a;
        out.bm = y.am;
        out.bc = y.ac;
        return true;
      }
      return false;
    }
    default: return false;
  }
}
}  // namespace

// Expected group count of a GROUP BY over n rows: the learned estimator's distinct-key
// prediction when it is trained and enabled (single-key group-bys over a base table),
// else the exact bound the zone maps give (the product of the key ranges), at most n.
uint64_t Engine::expected_groups(Var* a, const std::vector<std::string>& group_cols, uint64_t n) {
  Var* src = a->kind == Var::Filtered ? var(a->source) : a;
  if (src->kind != Var::Base) return n;
  for (auto& g : group_cols)
    if (!src->has(g) || src->meta[g].type > 2) return n;
  if (card_use_ && card_mlp_ && group_cols.size() == 1) {
    const alk_stats saved = stats_;  // the estimate's scan plan is not a scan of the query
    uint64_t hits = 0, keys = 0;
    ScanPlan p = plan_scan(a);
    CardStage cst;
    cst.p = &p;
    cst.key_slot = (int32_t)p.slot(group_cols[0]);
    auto cs = colsegs(p);
    cst.cs = &cs;
    BaseCol& bc = basecol(src, group_cols[0]);
    read_headers(src, group_cols[0], bc);
    int64_t lo = INT64_MAX, hi = INT64_MIN;
    for (auto& sg : bc.segs) {
      lo = std::min(lo, std::min(sg.m.lower, sg.m.upper));
      hi = std::max(hi, std::max(sg.m.lower, sg.m.upper));
    }
    cst.key_range = {lo, hi};
    const bool ok = card_estimate(cst, &hits, &keys);
    const uint32_t estimates = stats_.card_estimates;
    stats_ = saved;
    stats_.card_estimates = estimates;
    if (ok) return std::min<uint64_t>(n, keys);
  }
  long double bound = 1;
  for (auto& g : group_cols) {
    BaseCol& bc = basecol(src, g);
    read_headers(src, g, bc);
    int64_t lo = INT64_MAX, hi = INT64_MIN;
    for (auto& sg : bc.segs) {
      lo = std::min(lo, std::min(sg.m.lower, sg.m.upper));
      hi = std::max(hi, std::max(sg.m.lower, sg.m.upper));
    }
    bound *= (long double)((uint64_t)hi - (uint64_t)lo) + 1.0L;
  }
  return bound < (long double)n ? (uint64_t)bound : n;
}

bool Engine::dense_select_prepare(Statement& st, SelectCtx& c) {
  if ((flags_ & ALK_SESSION_PLAIN) || !st.grp_cnt) return false;
  Var* a = vars_.count(st.f) ? var(st.f) : nullptr;
  if (!a || (a->kind != Var::Filtered && a->kind != Var::Base)) return false;
  if (a->kind == Var::Filtered && var(a->source)->kind != Var::Base) return false;
  c.st = &st;
  c.a = a;
  c.grp_cnt = st.grp_cnt;
  c.group_cols.assign(st.op_value.end() - st.grp_cnt, st.op_value.end());
  if (c.group_cols.size() > 2) return false;
  for (auto& g : c.group_cols)
    if (!a->has(g) || a->meta[g].type > 2) return false;
  bool one_line = false;
  compile_select(st, a, true, c.outs, c.aggs, one_line);
  for (auto& o : c.outs) {
    if (o.col_type == 1 && std::find(c.group_cols.begin(), c.group_cols.end(), o.field) == c.group_cols.end())
      return false;
    if (o.col_type == 2 && has_col(o.vec)) return false;
  }
  if (c.aggs.size() > 8) return false;
  std::vector<Sym> sym(c.aggs.size());
  for (size_t k = 0; k < c.aggs.size(); k++)
    if (c.aggs[k].kind != ALK_AGG_COUNT && !sym_of(c.aggs[k].input, sym[k])) return false;
  c.cycles = cycle_count(a);
  const uint32_t skipped = stats_.segments_skipped;
  c.plan = plan_scan(a);
  auto fail = [&]() {
    stats_.segments_skipped = skipped;  // the operator plan scans again
    return false;
  };
  if (c.plan.has_pred) {
    std::vector<CardConj> cj;
    if (!program_conjuncts(c.plan.pred, cj) || cj.size() > 4) return fail();
  }
  Var* src = c.plan.src;
  alk_gb_query& q = c.q;
  std::memset(&q, 0, sizeof(q));
  q.nkeys = (uint32_t)c.group_cols.size();
  uint64_t nslots = 1;
  c.kmin.assign(q.nkeys, 0);
  c.kspan.assign(q.nkeys, 0);
  for (uint32_t j = 0; j < q.nkeys; j++) {
    q.key_col[j] = (int32_t)c.plan.slot(c.group_cols[j]);
    BaseCol& bc = basecol(src, c.group_cols[j]);
    read_headers(src, c.group_cols[j], bc);
    int64_t lo = INT64_MAX, hi = INT64_MIN;
    for (uint32_t g = 0; g < src->segCount; g++) {
      if (!c.plan.mode[g]) continue;
      lo = std::min(lo, std::min(bc.segs[g].m.lower, bc.segs[g].m.upper));
      hi = std::max(hi, std::max(bc.segs[g].m.lower, bc.segs[g].m.upper));
    }
    if (hi < lo) lo = hi = 0;  // nothing scanned
    const uint64_t span = (uint64_t)hi - (uint64_t)lo + 1;
    if (span == 0 || span > 64) return fail();
    q.key_min[j] = lo;
    q.key_max[j] = hi;
    c.kmin[j] = lo;
    c.kspan[j] = (int64_t)span;
    nslots *= span;
  }
  q.nagg = (uint32_t)c.aggs.size();
  if (nslots * (q.nagg + 1) > 64) return fail();
  for (size_t k = 0; k < c.aggs.size(); k++) {
    alk_gb_agg& g = q.agg[k];
    g.kind = c.aggs[k].kind;
    g.a = q.key_col[0] >= 0 && q.nkeys ? q.key_col[0] : 0;
    g.b = -1;
    g.am = 1;
    if (g.kind == ALK_AGG_COUNT) continue;
    const Sym& y = sym[k];
    if (y.kind == 0) {  // a constant input
      g.am = 0;
      g.ac = y.c;
      continue;
    }
    g.a = (int32_t)c.plan.slot(y.a);
    g.am = y.am;
    g.ac = y.ac;
    if (y.kind == 2) {
      g.b = (int32_t)c.plan.slot(y.b);
      g.bm = y.bm;
      g.bc = y.bc;
    }
  }
  if (c.plan.slots.size() > 8) return fail();
  for (auto& n : c.plan.slots)
    if (src->meta[n].type > 2) return fail();
  c.cs = colsegs(c.plan);
  for (auto& d : c.cs)
    if (d.rows && ((uintptr_t)d.data & 15)) return fail();
  q.cols = c.cs.data();
  q.ncols = (uint32_t)c.plan.slots.size();
  q.nseg = src->segCount;
  q.seg_mode = c.plan.mode.data();
  q.pred = c.plan.has_pred ? &c.plan.pred : nullptr;
  c.acc_words = nslots * (q.nagg + 1);  // the accumulators live in the batch's arena
  c.seg_rows.assign(src->segCount, 0);
  q.h_seg_rows = c.seg_rows.data();
  return true;
}

// One launch for every prepared select. The launch shape (consumer warps, tiles in
// flight, blocks per SM) is autotuned per workload signature: the first batch of a
// signature runs under each candidate shape (every run is complete and exact; the last
// one's results stand) and the fastest shape is kept for later batches.
void Engine::dense_select_run(const std::vector<SelectCtx*>& cs) {
  // every select's accumulators in one device buffer: one allocation, one copy back
  size_t total = 0;
  std::vector<size_t> at(cs.size());
  for (size_t i = 0; i < cs.size(); i++) {
    at[i] = total;
    total += cs[i]->acc_words;
  }
  auto arena = mkbuf(std::max<size_t>(total, 1) * 8, stream_);
  for (size_t i = 0; i < cs.size(); i++) cs[i]->q.d_acc = arena->as<int64_t>() + at[i];
  std::vector<alk_gb_query> qs;
  std::string sig = std::to_string(cs.size());
  uint64_t rows = 0;
  for (auto* c : cs) {
    qs.push_back(c->q);
    sig += "|" + std::to_string(c->q.ncols) + "," + std::to_string(c->q.nagg) + "," + std::to_string(c->q.nkeys);
    for (uint32_t k = 0; k < c->q.ncols; k++) sig += ":" + std::to_string(c->cs[(size_t)k * c->q.nseg].bits);
    for (uint32_t g = 0; g < c->q.nseg; g++)
      if (c->q.seg_mode[g]) rows += c->cs[g].rows;
  }
  auto it = gb_tune_.find(sig);
  alk_gb_tuning best{};
  if (fixed_tuning_.consumer_warps) {
    best = fixed_tuning_;
  } else if (it != gb_tune_.end()) {
    best = it->second;
  } else if (rows >= (64ull << 20) && autotune_) {
    // candidates, timed with events around the launch on the engine stream
    float best_ms = 1e30f;
    for (uint32_t cw : {8u, 4u})
      for (uint32_t nst : {2u, 3u, 4u})
        for (uint32_t bps : {1u, 2u, 3u, 4u}) {
          alk_gb_tuning t{cw, nst, bps}, used{};
          cudaEventRecord(ev0_, stream_);
          int rc = alk_batch_groupby(qs.data(), (uint32_t)qs.size(), &t, &used, nullptr, (alk_stream)stream_);
          cudaEventRecord(ev1_, stream_);
          if (rc == ALK_ERR_UNSUPPORTED) continue;
          check(rc, "batched group-by");
          if (used.blocks_per_sm != bps) continue;  // capped by shared memory: a duplicate
          ck(cudaEventSynchronize(ev1_), "sync");
          float ms = 0;
          cudaEventElapsedTime(&ms, ev0_, ev1_);
          if (ms < best_ms) {
            best_ms = ms;
            best = used;
          }
        }
    gb_tune_[sig] = best;
  }
  alk_gb_tuning used{};
  alk_event_timer tm{timing_ ? 1 : 0, ev0_, ev1_, 0.0, 0};
  check(alk_batch_groupby(qs.data(), (uint32_t)qs.size(), best.consumer_warps ? &best : nullptr, &used, &tm,
                          (alk_stream)stream_),
        "batched group-by");
  last_tuning_ = used;
  // every select's accumulators back in one copy and one synchronisation
  std::vector<int64_t> all(total);
  if (total) ck(cudaMemcpyAsync(all.data(), arena->as<void>(), total * 8, cudaMemcpyDeviceToHost, stream_), "d2h");
  stats_.d2h_bytes += total * 8;
  ck(cudaStreamSynchronize(stream_), "sync");
  for (size_t i = 0; i < cs.size(); i++) {
    const size_t n = (i + 1 < cs.size() ? at[i + 1] : total) - at[i];
    cs[i]->hacc.assign(all.begin() + at[i], all.begin() + at[i] + n);
  }
  if (tm.launches) {
    // algorithmic bytes: every scanned row's stored values of the columns the queries read
    uint64_t bytes = 0;
    for (auto* c : cs)
      for (uint32_t k = 0; k < c->q.ncols; k++)
        for (uint32_t g = 0; g < c->q.nseg; g++)
          if (c->q.seg_mode[g])
            bytes += (uint64_t)c->cs[(size_t)k * c->q.nseg + g].rows * (c->cs[(size_t)k * c->q.nseg + g].bits / 8);
    stats_.hot_kernel_ms += tm.ms;
    stats_.hot_kernel_launches += tm.launches;
    stats_.hot_kernel_bytes += bytes;
  }
}

void Engine::dense_select_finish(SelectCtx& c) {
  Statement& st = *c.st;
  auto out = std::make_unique<Var>();
  out->kind = Var::Mat;
  out->name = st.s;
  uint64_t n = 0;
  for (auto r : c.seg_rows) n += r;
  if (n == 0) {  // no segment produced rows: empty result without columns
    vars_[st.s] = std::move(out);
    return;
  }
  // the reference leaves the select-list order reversed when its first segment is empty
  if (c.seg_rows[0] == 0) std::reverse(c.outs.begin(), c.outs.end());
  const alk_gb_query& q = c.q;
  uint64_t nslots = 1;
  for (uint32_t j = 0; j < q.nkeys; j++) nslots *= (uint64_t)c.kspan[j];
  const uint32_t nacc = q.nagg + 1;
  const std::vector<int64_t>& h = c.hacc;  // copied back by dense_select_run
  if (h.size() < nslots * nacc) throw EngineError(ALK_ERR_ARG, "dense group-by: accumulators missing");
  std::vector<std::vector<int64_t>> keys(q.nkeys), vals(q.nagg);
  for (uint64_t sl = 0; sl < nslots; sl++) {
    if (h[(size_t)q.nagg * nslots + sl] == 0) continue;  // no row in this slot
    uint64_t rest = sl;
    for (int j = (int)q.nkeys - 1; j >= 0; j--) {  // slot = sum (key - min) * stride, last key fastest
      keys[j].push_back(c.kmin[j] + (int64_t)(rest % (uint64_t)c.kspan[j]));
      rest /= (uint64_t)c.kspan[j];
    }
    for (uint32_t k = 0; k < q.nagg; k++) vals[k].push_back(h[(size_t)k * nslots + sl]);
  }
  const uint64_t ng = keys.empty() ? 0 : keys[0].size();
  // output order (as select_output): MurmurHash64A of the key tuple across segments,
  // stable; key order within one segment
  std::vector<uint32_t> perm(ng);
  std::iota(perm.begin(), perm.end(), 0);
  if (c.cycles > 1) {
    std::vector<uint64_t> hs(ng);
    std::vector<int64_t> tuple(q.nkeys);
    for (uint64_t g = 0; g < ng; g++) {
      for (uint32_t j = 0; j < q.nkeys; j++) tuple[j] = keys[j][g];
      hs[g] = murmur64a(tuple.data(), (int)(8 * q.nkeys), kHashSeed);
    }
    std::stable_sort(perm.begin(), perm.end(), [&](uint32_t x, uint32_t y) { return hs[x] < hs[y]; });
  } else {
    std::stable_sort(perm.begin(), perm.end(), [&](uint32_t x, uint32_t y) {
      for (uint32_t j = 0; j < q.nkeys; j++)
        if (keys[j][x] != keys[j][y]) return keys[j][x] < keys[j][y];
      return false;
    });
  }
  auto permuted = [&](const std::vector<int64_t>& v) {
    std::vector<int64_t> o(ng);
    for (uint64_t g = 0; g < ng; g++) o[g] = v[perm[g]];
    return o;
  };
  std::vector<std::vector<int64_t>> sk, sv;
  for (auto& k : keys) sk.push_back(permuted(k));
  for (auto& v : vals) sv.push_back(permuted(v));
  // output columns (select_output's rules, evaluated on the host for the few groups)
  std::vector<std::string> names;
  std::vector<std::vector<int64_t>> cols;
  std::vector<ColMeta> metas;
  std::vector<int> gtypes;
  for (auto& o : c.outs) {
    ColMeta m;
    m.dz = o.prec;
    std::vector<int64_t> col;
    if (o.col_type == 1) {
      auto it = std::find(c.group_cols.begin(), c.group_cols.end(), o.field);
      col = sk[it - c.group_cols.begin()];
      m.string_map = c.a->meta[o.field].string_map;
    } else if (o.col_type == 2 && o.vec->k == Ast::Agg) {
      col = sv[o.vec->agg];
    } else if (o.col_type == 2) {
      Compiler cc;
      alk_program prog = cc.finish(o.vec);
      std::vector<const int64_t*> in;
      for (auto& sname : cc.slots) in.push_back(sv[std::stoi(sname.substr(4))].data());
      col.resize(ng);
      host_eval(prog, in, ng, col.data());
    } else {
      col.assign(ng, (int64_t)(int)o.num);
    }
    names.push_back(o.name);
    cols.push_back(std::move(col));
    metas.push_back(m);
    gtypes.push_back(o.grp_type);
  }
  // AVG finalisation of count_avg (merge.cu:446-458)
  int countc = -1;
  for (size_t k = 0; k < cols.size(); k++)
    if (gtypes[k] == 0) {
      countc = (int)k;
      break;
    }
  for (size_t k = 0; k < cols.size(); k++) {
    if (gtypes[k] != 1) continue;
    if (countc < 0) unsupported("AVG needs a COUNT column in the same select");
    for (uint64_t g = 0; g < ng; g++)
      cols[k][g] = metas[k].dz <= 2 ? host_div(host_mul(cols[k][g], 100), cols[countc][g])
                                    : host_div(cols[k][g], cols[countc][g]);
    if (metas[k].dz <= 2) metas[k].dz += 2;
    gtypes[k] = 3;
  }
  out->n = ng;
  for (size_t k = 0; k < cols.size(); k++) {
    out->columnNames.push_back(names[k]);
    out->meta[names[k]] = metas[k];
    out->grp_type[names[k]] = gtypes[k];
    out->host[names[k]] = std::move(cols[k]);
  }
  vars_[st.s] = std::move(out);
  stats_.plan = std::max<uint32_t>(stats_.plan, 1);
}

// ------------------------------------------------------------------ JOIN
// emit_join (operators.cu:797-924): a chain of emit_multijoin steps, then aliases.
void Engine::emit_join(Statement& st) {
  if (star_join_applies(st)) {  // emit_join's star branch (operators.cu:828-832)
    star_join(st);
    return;
  }
  std::vector<std::string> op_m = st.op_value;
  if (st.join_tab_cnt > 1) {
    size_t oi = 0;
    for (unsigned i = 1; i <= st.join_tab_cnt; i++) {
      std::string tab_name = i == st.join_tab_cnt ? st.s : st.s + std::to_string(i);
      std::string j, j2;
      if (i == 1) {
        j2 = st.op_join[oi++];
        j = st.op_join[oi++];
      } else {
        j = oi < st.op_join.size() ? st.op_join[oi++] : st.f;
        j2 = st.s + std::to_string(i - 1);
      }
      multijoin(st, tab_name, j, j2, i);
      if (i > 1) vars_.erase(st.s + std::to_string(i - 1));
    }
  } else {
    multijoin(st, st.s, st.f, st.op_join.at(0), 1);
  }
  Var* r = var(st.s);
  for (unsigned k = 0; k < st.sel_count; k++) {
    const std::string& from = op_m[2 * k];
    const std::string& to = op_m[2 * k + 1];
    if (from == to) continue;
    auto it = std::find(r->columnNames.begin(), r->columnNames.end(), from);
    if (it == r->columnNames.end()) continue;
    *it = to;
    r->data[to] = r->data[from];
    r->data.erase(from);
    // the rename carries the type and the decimal flag but not decimal_zeroes
    // (operators.cu:877-906): the alias keeps its previous scale, 0 for a new name, and
    // that scale is what later arithmetic (get_decimals, cm.cu:4371) and STORE use
    uint32_t dz_to = r->meta.count(to) ? r->meta[to].dz : 0;
    r->meta[to] = r->meta[from];
    r->meta[to].dz = dz_to;
  }
}

// The AND-ed key pairs of a join (operators.cu:1288-1348) on its pairs (pl, pr): extra pair
// m keeps the pairs whose first extra columns compare equal (not equal when the m-th
// queued equality is '!='). The pairs are compacted in order; returns their count.
uint64_t Engine::filter_pairs(DevBufP& pl, DevBufP& pr, uint64_t pairs, const DevBufP& lcol, const DevBufP& rcol,
                              unsigned jac, const std::vector<char>& eq_type) {
  for (unsigned m = 0; m < jac && pairs; m++) {
    const int neq = m < eq_type.size() && eq_type[m] == 'N';
    auto flags = mkbuf(pairs * 8, stream_);
    check(alk_pair_match(pl->as<uint32_t>(), pr->as<uint32_t>(), pairs, lcol->as<int64_t>(), rcol->as<int64_t>(), neq,
                         flags->as<uint64_t>(), (alk_stream)stream_),
          "join AND pair");
    auto idx = mkbuf(pairs * 4, stream_);
    uint64_t kept = 0;
    check(alk_flags_compact(flags->as<uint64_t>(), pairs, idx->as<uint32_t>(), &kept, (alk_stream)stream_),
          "join AND compact");
    auto npl = mkbuf(std::max<uint64_t>(kept, 1) * 4, stream_), npr = mkbuf(std::max<uint64_t>(kept, 1) * 4, stream_);
    check(alk_gather_u32(pl->as<uint32_t>(), idx->as<uint32_t>(), kept, npl->as<uint32_t>(), (alk_stream)stream_),
          "join AND gather");
    check(alk_gather_u32(pr->as<uint32_t>(), idx->as<uint32_t>(), kept, npr->as<uint32_t>(), (alk_stream)stream_),
          "join AND gather");
    pl = npl;
    pr = npr;
    pairs = kept;
  }
  return pairs;
}

// Semi and anti joins (operators.cu:1357-1399, 1473-1530): the rows of one side that have
// (semi) or lack (anti) a partner after the AND-ed pairs, each once.
//  '1' left semi, '3' left anti: left rows in left order. A left segment whose filtered key
//     range misses the right side's key range adds nothing, even to an anti join (the
//     range test skips the segment before the join kinds are told apart,
//     operators.cu:1215-1220).
//  '2' right semi, '4' right anti: right rows in the order of the right side sorted by
//     its key (the reference sorts it for the merge join, stably), across all left segments.
void Engine::semi_anti_join(Var* c, Rows& L, Rows& R, const std::string& lkey, const std::string& rkey,
                            const std::string& f3, const std::string& f4, unsigned jac,
                            const std::vector<char>& eq_type, char kind) {
  const bool left_rows = kind == '1' || kind == '3';
  const uint64_t nrows = left_rows ? L.n : R.n;
  DevBufP pl, pr;
  uint64_t pairs = 0;
  if (L.n && R.n) {
    alk_join_table* t = nullptr;
    check(alk_join_build(R.col.at(rkey)->as<int64_t>(), R.n, &t, (alk_stream)stream_), "join build");
    struct TableGuard {
      alk_join_table* t;
      cudaStream_t s;
      ~TableGuard() { alk_join_free(t, (alk_stream)s); }
    } guard{t, stream_};
    uint64_t cap = std::max<uint64_t>(L.n, 1024);
    for (int attempt = 0; attempt < 2; attempt++) {
      pl = mkbuf(cap * 4, stream_);
      pr = mkbuf(cap * 4, stream_);
      int rc = alk_join_probe(t, L.col.at(lkey)->as<int64_t>(), L.n, pl->as<uint32_t>(), pr->as<uint32_t>(), cap,
                              &pairs, (alk_stream)stream_);
      if (rc == ALK_ERR_OVERFLOW && attempt == 0) {
        cap = pairs;
        continue;
      }
      check(rc, "join probe");
      break;
    }
    if (jac) pairs = filter_pairs(pl, pr, pairs, L.col.at(f3), R.col.at(f4), jac, eq_type);
  }
  const bool anti = kind == '3' || kind == '4';
  auto flags = mkbuf(std::max<uint64_t>(nrows, 1) * 8, stream_);
  if (nrows) check(alk_fill_i64(flags->as<int64_t>(), nrows, anti ? 1 : 0, (alk_stream)stream_), "join flags");
  if (pairs)
    check(alk_rows_mark((left_rows ? pl : pr)->as<uint32_t>(), pairs, flags->as<uint64_t>(), anti ? 0 : 1,
                        (alk_stream)stream_),
          "join mark");
  if (kind == '3' && nrows) {
    // left segments whose key range misses the right side's
    std::vector<uint64_t> start(L.seg_counts.size() + 1, 0);
    for (size_t g = 0; g < L.seg_counts.size(); g++) start[g + 1] = start[g] + L.seg_counts[g];
    int64_t rr[2] = {INT64_MAX, INT64_MIN};
    if (R.n) {
      const uint64_t rs[2] = {0, R.n};
      check(alk_seg_minmax(R.col.at(rkey)->as<int64_t>(), rs, 1, rr, (alk_stream)stream_), "join range");
    }
    std::vector<int64_t> lr(2 * L.seg_counts.size());
    check(alk_seg_minmax(L.col.at(lkey)->as<int64_t>(), start.data(), (uint32_t)L.seg_counts.size(), lr.data(),
                         (alk_stream)stream_),
          "join range");
    for (size_t g = 0; g < L.seg_counts.size(); g++) {
      if (!L.seg_counts[g]) continue;
      if (!R.n || lr[2 * g] > rr[1] || lr[2 * g + 1] < rr[0])
        check(alk_fill_i64(flags->as<int64_t>() + start[g], L.seg_counts[g], 0, (alk_stream)stream_), "join flags");
    }
  }
  // the kept rows, in the side's order (right: sorted by key, stably)
  DevBufP order;
  if (!left_rows && nrows) {
    order = mkbuf(nrows * 4, stream_);
    const int64_t* keys[1] = {R.col.at(rkey)->as<int64_t>()};
    const uint8_t asc[1] = {0};
    check(alk_sort_perm(keys, asc, 1, nrows, order->as<uint32_t>(), (alk_stream)stream_), "join order");
    auto sorted_flags = mkbuf(nrows * 8, stream_);
    check(alk_gather(flags->as<int64_t>(), order->as<uint32_t>(), nrows, sorted_flags->as<int64_t>(),
                     (alk_stream)stream_),
          "join order");
    flags = sorted_flags;
  }
  auto idx = mkbuf(std::max<uint64_t>(nrows, 1) * 4, stream_);
  uint64_t kept = 0;
  if (nrows)
    check(alk_flags_compact(flags->as<uint64_t>(), nrows, idx->as<uint32_t>(), &kept, (alk_stream)stream_),
          "join compact");
  if (order && kept) {
    auto rows = mkbuf(kept * 4, stream_);
    check(alk_gather_u32(order->as<uint32_t>(), idx->as<uint32_t>(), kept, rows->as<uint32_t>(), (alk_stream)stream_),
          "join order");
    idx = rows;
  }
  Rows& side = left_rows ? L : R;
  c->n = kept;
  for (auto& n : c->columnNames) {
    auto d = mkbuf(std::max<uint64_t>(kept, 1) * 8, stream_);
    if (kept)
      check(alk_gather(side.col.at(n)->as<int64_t>(), idx->as<uint32_t>(), kept, d->as<int64_t>(), (alk_stream)stream_),
            "join gather");
    c->data[n] = d;
  }
  ck(cudaStreamSynchronize(stream_), "join sync");
}

// emit_multijoin (operators.cu:940-1582): inner equi-join of a (filtered) left side
// with a right side; the right side is hashed (MurmurHash64A, linear probing) instead
// of sorted, so pairs come out as a multiset.
void Engine::multijoin(Statement& st, const std::string& s, const std::string& j1, const std::string& j2,
                       unsigned tab) {
  Var* left = var(j1);
  Var* right = var(j2);
  std::vector<std::string> op_sel, op_g;
  size_t k = 0;
  for (unsigned i = 0; i < st.sel_count; i++, k += 2) op_sel.push_back(st.op_value.at(k));
  op_g.assign(st.op_value.begin() + k, st.op_value.end());
  std::vector<std::string> op_sel_s = op_sel;
  size_t gi = 0;
  for (unsigned z = 0; z < st.join_tab_cnt - tab; z++) {
    unsigned jac = st.join_and_cnt.count(z) ? st.join_and_cnt.at(z) : 0;
    for (unsigned j = 0; j < jac * 2 + 2; j++) op_sel_s.push_back(op_g.at(gi++));
  }
  std::string f1 = op_g.at(gi), f2 = op_g.at(gi + 1);
  unsigned jac = st.join_and_cnt.count(st.join_tab_cnt - tab) ? st.join_and_cnt.at(st.join_tab_cnt - tab) : 0;
  const char kind = st.join_type.at(tab - 1);
  if (kind != 'I' && kind != '1' && kind != '2' && kind != '3' && kind != '4')
    unsupported("outer joins");  // the reference's outer joins are commented out (operators.cu:1242-1260)
  if ((jac || kind != 'I') && st.join_tab_cnt != 1) unsupported("multi-column / semi / anti joins in a join chain");
  // AND-ed key pairs (operators.cu:1288-1348): every extra pair tests the first extra pair's
  // columns (the queue is copied afresh each time), with the equality type of the step's
  // queued '=' / '!=' in order, the first being the primary key's
  std::string f3, f4;
  if (jac) {
    f3 = op_g.at(gi + 2);
    f4 = op_g.at(gi + 3);
    if (!left->has(f3) || !right->has(f4)) unsupported("AND-ed join column outside its side");
  }
  auto c = std::make_unique<Var>();
  c->kind = Var::Mat;
  c->name = s;
  for (auto& n : op_sel_s) {
    if (c->has(n)) continue;
    if (right->has(n)) c->meta[n] = right->meta[n];
    else if (left->has(n)) c->meta[n] = left->meta[n];
    else continue;
    c->columnNames.push_back(n);
  }
  std::string colname1, colname2;
  if (left->has(f1)) {
    colname1 = f1;
    if (!right->has(f2)) throw EngineError(ALK_ERR_ARG, "Couldn't find column " + f2);
    colname2 = f2;
  } else if (right->has(f1)) {
    colname2 = f1;
    if (!left->has(f2)) throw EngineError(ALK_ERR_ARG, "Couldn't find column " + f2);
    colname1 = f2;
  } else {
    throw EngineError(ALK_ERR_ARG, "Couldn't find column " + f1);
  }
  if (left->meta[colname1].type != right->meta[colname2].type) unsupported("join of different column types");
  // Char keys are dictionary codes. Codes of one dictionary compare as they are; the
  // reference compares codes of two different dictionaries too, which matches nothing in
  // particular. Here such keys compare by value: each row's key becomes the
  // MurmurHash64A / 2 of its value zero-padded to the wider of the two widths (the form
  // of the reference's .hash files, filter.cu:428-449 and cm.cu:1808-1812).
  const bool by_value = left->meta[colname1].type == 2 &&
                        left->meta[colname1].string_map != right->meta[colname2].string_map;
  if (by_value && kind != 'I') unsupported("semi / anti join on char columns of different dictionaries");
  // a left semi / anti join outputs left rows only, a right one right rows only (the
  // reference gathers the other side through pairs it has since reordered)
  const bool left_rows = kind == '1' || kind == '3', right_rows = kind == '2' || kind == '4';
  for (auto& n : c->columnNames) {
    if (left_rows && !left->has(n)) unsupported("right-side column in a left semi / anti join");
    if (right_rows && !right->has(n)) unsupported("left-side column in a right semi / anti join");
  }
  std::vector<std::string> rfields, lfields;
  for (auto& n : c->columnNames)
    if ((right_rows || !left->has(n)) && right->has(n)) rfields.push_back(n);
  rfields.push_back(colname2);
  if (jac) rfields.push_back(f4);
  for (auto& n : c->columnNames)
    if (!right_rows && left->has(n)) lfields.push_back(n);
  lfields.push_back(colname1);
  if (jac) lfields.push_back(f3);
  Rows R = materialize(right, rfields);
  Rows L = materialize(left, lfields);
  c->n = 0;
  if (kind != 'I') {
    semi_anti_join(c.get(), L, R, colname1, colname2, f3, f4, jac, st.join_eq_type, kind);
    vars_[s] = std::move(c);
    return;
  }
  DevBufP lkey = L.col.count(colname1) ? L.col.at(colname1) : nullptr, rkey = R.col.count(colname2) ? R.col.at(colname2) : nullptr;
  if (by_value && R.n && L.n) {
    const uint32_t w = std::max(left->meta[colname1].width, right->meta[colname2].width);
    auto keyed = [&](const DevBufP& codes, uint64_t n, const ColMeta& m) {
      DevBufP h = dict_hashes(m, w), k = mkbuf(n * 8, stream_);
      auto idx = mkbuf(n * 4, stream_);
      check(alk_narrow_u32(codes->as<int64_t>(), n, idx->as<uint32_t>(), (alk_stream)stream_), "codes");
      check(alk_gather(h->as<int64_t>(), idx->as<uint32_t>(), n, k->as<int64_t>(), (alk_stream)stream_), "key hash");
      return k;
    };
    lkey = keyed(L.col.at(colname1), L.n, left->meta[colname1]);
    rkey = keyed(R.col.at(colname2), R.n, right->meta[colname2]);
  }
  if (R.n && L.n) {
    alk_join_table* t = nullptr;
    check(alk_join_build(rkey->as<int64_t>(), R.n, &t, (alk_stream)stream_), "join build");
    struct TableGuard {
      alk_join_table* t;
      cudaStream_t s;
      ~TableGuard() { alk_join_free(t, (alk_stream)s); }
    } guard{t, stream_};
    uint64_t cap = std::max<uint64_t>(L.n, 1024), pairs = 0;
    DevBufP pl, pr;
    for (int attempt = 0; attempt < 2; attempt++) {
      pl = mkbuf(cap * 4, stream_);
      pr = mkbuf(cap * 4, stream_);
      int rc = alk_join_probe(t, lkey->as<int64_t>(), L.n, pl->as<uint32_t>(), pr->as<uint32_t>(), cap, &pairs,
                              (alk_stream)stream_);
      if (rc == ALK_ERR_OVERFLOW && attempt == 0) {
        cap = pairs;
        continue;
      }
      check(rc, "join probe");
      break;
    }
    if (jac) pairs = filter_pairs(pl, pr, pairs, L.col.at(f3), R.col.at(f4), jac, st.join_eq_type);
    c->n = pairs;
    for (auto& n : c->columnNames) {
      bool from_left = left->has(n);
      const DevBufP& src = from_left ? L.col.at(n) : R.col.at(n);
      auto d = mkbuf(std::max<uint64_t>(pairs, 1) * 8, stream_);
      check(alk_gather(src->as<int64_t>(), (from_left ? pl : pr)->as<uint32_t>(), pairs, d->as<int64_t>(),
                       (alk_stream)stream_),
            "join gather");
      c->data[n] = d;
    }
    ck(cudaStreamSynchronize(stream_), "join sync");
  } else {
    for (auto& n : c->columnNames) c->data[n] = mkbuf(8, stream_);
  }
  vars_[s] = std::move(c);
}

// ------------------------------------------------------------------ ORDER
// emit_order (operators.cu:1641-1798): stable sort, first key most significant, ties
// in input order.
void Engine::emit_order(Statement& st) {
  Var* a = var(st.f);
  std::vector<std::string> keys;
  std::vector<uint8_t> desc;
  size_t iv = 0;
  for (auto& t : st.op_type) {
    if (t == "NAME") {
      keys.push_back(st.op_value.at(iv++));
      desc.push_back(0);
    } else {
      keys.push_back(t);
      desc.push_back(st.op_value.at(iv++) == "DESC");
    }
    if (!a->has(keys.back())) throw EngineError(ALK_ERR_ARG, "Couldn't find name " + keys.back());
  }
  Rows R = materialize(a, a->columnNames);
  auto b = std::make_unique<Var>();
  b->kind = Var::Mat;
  b->name = st.s;
  b->columnNames = a->columnNames;
  b->meta = a->meta;
  b->grp_type = a->grp_type;
  b->n = R.n;
  if (R.n) {
    std::vector<const int64_t*> kc;
    std::vector<DevBufP> ranked;  // char keys: each row's dictionary code replaced by its rank
    for (auto& kname : keys) {
      const ColMeta& m = a->meta[kname];
      if (m.type != 2 && m.string_map.empty()) {
        kc.push_back(R.col.at(kname)->as<int64_t>());
        continue;
      }
      // the reference sorts the strings themselves, bytes compared unsigned over the full
      // width, stably (update_char_permutation cm.cu:4218, str_sort
      // strings_sort_device.cu:125): the same order as the entries' ranks in the sorted
      // dictionary, equal strings sharing a rank
      const DevBufP& rank = dict_ranks(m);
      auto key = mkbuf(R.n * 8, stream_);
      check(alk_code_lookup(R.col.at(kname)->as<int64_t>(), R.n, rank->as<int64_t>(), rank->bytes() / 8,
                            key->as<int64_t>(), (alk_stream)stream_),
            "order char key");
      ranked.push_back(key);
      kc.push_back(key->as<int64_t>());
    }
    auto perm = mkbuf(R.n * 4, stream_);
    check(alk_sort_perm(kc.data(), desc.data(), (uint32_t)kc.size(), R.n, perm->as<uint32_t>(), (alk_stream)stream_),
          "order");
    for (auto& n : a->columnNames) {
      auto d = mkbuf(R.n * 8, stream_);
      check(alk_gather(R.col.at(n)->as<int64_t>(), perm->as<uint32_t>(), R.n, d->as<int64_t>(), (alk_stream)stream_),
            "order gather");
      b->data[n] = d;
    }
  } else {
    for (auto& n : a->columnNames) b->data[n] = mkbuf(8, stream_);
  }
  vars_[st.s] = std::move(b);
}

// MurmurHash64A / 2 of a char column's dictionary entries, each zero-padded to `width`
// bytes, on the device (index: the code): keys that compare two dictionaries' values.
DevBufP Engine::dict_hashes(const ColMeta& m, uint32_t width) {
  const auto dot = m.string_map.find('.');
  Var* b = dot == std::string::npos ? nullptr : base_table(m.string_map.substr(0, dot));
  if (!b) throw EngineError(ALK_ERR_IO, "missing dictionary " + m.string_map);
  BaseCol& bc = basecol(b, m.string_map.substr(dot + 1));
  load_dict(b, m.string_map.substr(dot + 1), bc);
  const size_t n = bc.dict.size();
  std::vector<uint8_t> raw(std::max<size_t>(n, 1) * width, 0);
  for (size_t i = 0; i < n; i++) std::memcpy(&raw[i * width], bc.dict[i].data(), std::min<size_t>(width, bc.dict[i].size()));
  auto d_raw = mkbuf(raw.size(), stream_);
  ck(cudaMemcpyAsync(d_raw->as<void>(), raw.data(), raw.size(), cudaMemcpyHostToDevice, stream_), "dictionary h2d");
  stats_.h2d_bytes += raw.size();
  auto h = mkbuf(std::max<size_t>(n, 1) * 8, stream_);
  check(alk_hash_strings(d_raw->as<uint8_t>(), n, width, kHashSeed, h->as<uint64_t>(), (alk_stream)stream_),
        "dictionary hash");
  ck(cudaStreamSynchronize(stream_), "dictionary hash");
  return h;
}

// Dense ranks of a char column's dictionary entries in byte order (unsigned, full
// width), on the device, kept with the column.
const DevBufP& Engine::dict_ranks(const ColMeta& m) {
  const auto dot = m.string_map.find('.');
  Var* b = dot == std::string::npos ? nullptr : base_table(m.string_map.substr(0, dot));
  if (!b) throw EngineError(ALK_ERR_IO, "missing dictionary " + m.string_map);
  BaseCol& bc = basecol(b, m.string_map.substr(dot + 1));
  if (bc.ranks) return bc.ranks;
  load_dict(b, m.string_map.substr(dot + 1), bc);
  const size_t n = bc.dict.size();
  std::vector<uint32_t> order(n);
  std::iota(order.begin(), order.end(), 0u);
  auto less = [&](uint32_t x, uint32_t y) {
    return std::memcmp(bc.dict[x].data(), bc.dict[y].data(), bc.dict[x].size()) < 0;
  };
  std::stable_sort(order.begin(), order.end(), less);
  std::vector<int64_t> rank(std::max<size_t>(n, 1), 0);
  int64_t r = 0;
  for (size_t i = 0; i < n; i++) {
    if (i && less(order[i - 1], order[i])) r++;
    rank[order[i]] = r;
  }
  bc.ranks = mkbuf(rank.size() * 8, stream_);
  ck(cudaMemcpyAsync(bc.ranks->as<void>(), rank.data(), rank.size() * 8, cudaMemcpyHostToDevice, stream_),
     "ranks h2d");
  ck(cudaStreamSynchronize(stream_), "ranks h2d");
  stats_.h2d_bytes += rank.size() * 8;
  return bc.ranks;
}

// ------------------------------------------------------------------ STORE
// emit_store / CudaSet::Store text output (operators.cu:2410-2444, cm.cu:1479-1560).
void Engine::emit_store(Statement& st) {
  Var* a = var(st.s);
  size_t limit = st.op_nums.empty() ? 0 : (size_t)st.op_nums[0];
  bool on_host = a->kind == Var::Mat;
  for (auto& c : a->columnNames) on_host = on_host && a->host.count(c);
  std::vector<std::vector<int64_t>> h(a->columnNames.size());
  size_t mcount = 0;
  if (on_host) {  // a small result already on the host
    mcount = (limit != 0 && limit < a->n) ? limit : a->n;
    for (size_t c = 0; c < a->columnNames.size(); c++) {
      const auto& src = a->host.at(a->columnNames[c]);
      h[c].assign(src.begin(), src.begin() + mcount);
    }
  } else {
    Rows R = materialize(a, a->columnNames);
    mcount = (limit != 0 && limit < R.n) ? limit : R.n;
    for (size_t c = 0; c < a->columnNames.size(); c++) {
      h[c].resize(mcount);
      if (!mcount) continue;
      ck(cudaMemcpyAsync(h[c].data(), R.col.at(a->columnNames[c])->as<void>(), mcount * 8, cudaMemcpyDeviceToHost,
                         stream_),
         "store d2h");
      stats_.d2h_bytes += mcount * 8;
    }
    ck(cudaStreamSynchronize(stream_), "store sync");
  }
  std::string path = st.f;
  if (path.empty() || path[0] != '/') path = dir_ + "/" + path;
  std::vector<const std::vector<std::string>*> dicts(a->columnNames.size(), nullptr);
  std::vector<uint32_t> widths(a->columnNames.size(), 0);
  for (size_t c = 0; c < a->columnNames.size(); c++) {
    const ColMeta& m = a->meta[a->columnNames[c]];
    if (m.string_map.empty()) continue;
    auto dot = m.string_map.find('.');
    Var* b = base_table(m.string_map.substr(0, dot));
    if (!b) throw EngineError(ALK_ERR_IO, "missing dictionary " + m.string_map);
    std::string col = m.string_map.substr(dot + 1);
    BaseCol& bc = basecol(b, col);
    load_dict(b, col, bc);
    dicts[c] = &bc.dict;
    widths[c] = bc.meta.width;
  }
  // rows formatted in parallel chunks (integers through std::to_chars), written in order
  auto format_rows = [&](size_t r0, size_t r1, std::string& out) {
    char num[32];
    for (size_t i = r0; i < r1; i++) {
      for (size_t c = 0; c < a->columnNames.size(); c++) {
        const ColMeta& m = a->meta[a->columnNames[c]];
        const int64_t v = h[c][i];
        if (!dicts[c]) {
          const auto res = std::to_chars(num, num + sizeof(num), v);
          std::string_view d(num, (size_t)(res.ptr - num));
          if (m.dz) {
            std::string sd(d);
            while (sd.size() <= m.dz) sd = '0' + sd;
            sd.insert(sd.size() - m.dz, ".");
            out += sd;
          } else {
            out += d;
          }
        } else {
          const std::string& sv = (v >= 0 && (size_t)v < dicts[c]->size()) ? (*dicts[c])[v] : std::string();
          out.append(sv.data(), std::min(sv.size(), std::strlen(sv.c_str())));
        }
        out += st.sep;
      }
      if (i != mcount - 1) out += "\n";
    }
  };
  const size_t nthreads =
      std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), mcount / 65536));
  std::vector<std::string> parts(nthreads);
  if (nthreads == 1) {
    format_rows(0, mcount, parts[0]);
  } else {
    std::vector<std::thread> ths;
    for (size_t t = 0; t < nthreads; t++)
      ths.emplace_back(format_rows, mcount * t / nthreads, mcount * (t + 1) / nthreads, std::ref(parts[t]));
    for (auto& th : ths) th.join();
  }
  if (deferred_writes_) {
    PendingWrite w{path, std::string(), deferred_run_};
    for (auto& part : parts) w.data += part;
    deferred_writes_->push_back(std::move(w));
    return;
  }
  std::string all;
  if (parts.size() == 1) {
    all.swap(parts[0]);
  } else {
    for (auto& part : parts) all += part;
  }
  if (!write_file(path, all.data(), all.size())) throw EngineError(ALK_ERR_IO, "Could not open file " + path);
}

// STORE v INTO 'name' [APPEND] [LIMIT n] BINARY: the binary branch of CudaSet::Store
// (cm.cu:1040-1240) under emit_store_binary (operators.cu:2446-2515). Every column of v
// becomes one more segment file <name>.<column>.<segment>, encoded on the device in the
// reference's byte format (FOR; FOR-delta for sorted columns when the session has the
// delta switch), then the column headers (writeHeader, cm.cu:1251-1263) and the table's
// catalog entry (cm.cu:1686-1701, saved as save_col_data does). A result with columns
// and no rows writes the headers only (cm.cu:1481-1486); an empty select result has no
// columns and writes nothing. SORT SEGMENTS BY / PRESORTED BY and char columns are
// outside the supported surface.
void Engine::emit_store_binary(Statement& st) {
  Var* a = var(st.s);
  if (st.store_sort) unsupported("STORE BINARY with SORT SEGMENTS BY / PRESORTED BY");
  std::vector<std::string> icols, ccols;  // integer columns; a LOAD's char columns
  for (auto& c : a->columnNames) {
    if (a->meta[c].raw) ccols.push_back(c);
    else if (a->meta[c].type != 0 || !a->meta[c].string_map.empty()) unsupported("STORE BINARY of char columns");
    else icols.push_back(c);
  }
  if (!ccols.empty() && st.append) unsupported("STORE BINARY APPEND of char columns");
  if (st.f.empty() || st.f.find('/') != std::string::npos) unsupported("STORE BINARY outside the data directory");
  Rows R = materialize(a, icols);
  if (icols.empty()) R.n = a->n;
  const size_t limit = st.op_nums.empty() ? 0 : (size_t)st.op_nums[0];
  const uint64_t n = (limit != 0 && limit < R.n) ? limit : R.n;
  if (n > UINT32_MAX) unsupported("a segment of more than 2^32 - 1 rows");
  const std::string base = dir_ + "/" + st.f;
  uint64_t total = n;
  uint32_t seg = 0, max_recs = (uint32_t)n;
  if (st.append) {  // continue the table: its header gives the segment count (cm.cu:1050-1060)
    ColHeader h;
    std::string e;
    if (!a->columnNames.empty() && read_col_header(base + "." + a->columnNames[0] + ".header", h, e)) {
      seg = h.segs;
      total += h.total;
      max_recs = std::max(max_recs, h.max_recs);
    }
  }
  if (n == 0) {
    for (auto& c : a->columnNames) {
      const std::string prefix = base + "." + c;
      if (!write_col_header(prefix + ".header", ColHeader{total, seg, max_recs, cnt_counts_[prefix]}))
        throw EngineError(ALK_ERR_IO, "Could not write " + prefix + ".header");
    }
    return;
  }
  // A LOAD's char columns (compress_char, cm.cu:1765-1844): codes in first-appearance
  // order of the values' MurmurHash64A / 2 (one code sequence per column name for the
  // session, as the reference keys its char_hash), or a running count from 1 under NO
  // ENCODING; the dictionary file gets each new value, the .hash file every row's hash,
  // and the codes are written as the .idx segment.
  std::map<std::string, DevBufP> code_cols;
  for (auto& c : ccols) {
    const ColMeta& m = a->meta[c];
    const uint32_t w = m.width;
    const DevBufP& raw = a->data.at(c);
    auto dh = mkbuf(n * 8, stream_);
    check(alk_hash_strings(raw->as<uint8_t>(), n, w, 100, dh->as<uint64_t>(), (alk_stream)stream_), "string hash");
    std::vector<uint64_t> h(n);
    std::vector<uint8_t> chars((size_t)n * w);
    ck(cudaMemcpyAsync(h.data(), dh->as<void>(), n * 8, cudaMemcpyDeviceToHost, stream_), "d2h");
    ck(cudaMemcpyAsync(chars.data(), raw->as<void>(), (size_t)n * w, cudaMemcpyDeviceToHost, stream_), "d2h");
    ck(cudaStreamSynchronize(stream_), "d2h");
    stats_.d2h_bytes += n * 8 + (uint64_t)n * w;
    std::vector<int64_t> codes(n);
    std::vector<uint8_t> dict;
    auto& known = char_codes_[c];
    if (!m.no_encoding) {
      for (uint64_t i = 0; i < n; i++) {
        auto it = known.find(h[i]);
        if (it == known.end()) {
          const int64_t code = (int64_t)known.size();
          known.emplace(h[i], code);
          dict.insert(dict.end(), chars.begin() + (size_t)i * w, chars.begin() + (size_t)(i + 1) * w);
          codes[i] = code;
        } else {
          codes[i] = it->second;
        }
      }
    } else {
      int64_t cnt = known.count(0) ? known[0] : 0;
      for (uint64_t i = 0; i < n; i++) codes[i] = ++cnt;
      known[0] = cnt;
      dict = chars;
    }
    const std::string prefix = base + "." + c;
    if (!write_file(prefix, dict.data(), dict.size())) throw EngineError(ALK_ERR_IO, "Could not write " + prefix);
    std::vector<uint8_t> hf(4 + (size_t)n * 8);
    const uint32_t n32 = (uint32_t)n;
    std::memcpy(hf.data(), &n32, 4);
    std::memcpy(hf.data() + 4, h.data(), (size_t)n * 8);
    const std::string hp = prefix + "." + std::to_string(seg) + ".hash";
    if (!write_file(hp, hf.data(), hf.size())) throw EngineError(ALK_ERR_IO, "Could not write " + hp);
    auto dc = mkbuf(n * 8, stream_);
    ck(cudaMemcpyAsync(dc->as<void>(), codes.data(), n * 8, cudaMemcpyHostToDevice, stream_), "h2d");
    ck(cudaStreamSynchronize(stream_), "h2d");
    code_cols[c] = dc;
  }
  // every column's segment image (char columns: their codes) in one call of the device writer
  const size_t ncol = a->columnNames.size();
  const size_t cap = (kSegHeadBytes + (size_t)n * 8 + kSegTailBytes + 255) & ~size_t(255);
  auto imgs = mkbuf(cap * ncol, stream_);
  std::vector<const int64_t*> src(ncol);
  std::vector<uint32_t> counts(ncol, (uint32_t)n);
  std::vector<void*> dst(ncol);
  std::vector<size_t> caps(ncol, cap), lens(ncol, 0);
  for (size_t k = 0; k < ncol; k++) {
    const std::string& c = a->columnNames[k];
    src[k] = code_cols.count(c) ? code_cols[c]->as<int64_t>() : R.col.at(c)->as<int64_t>();
    dst[k] = imgs->as<uint8_t>() + k * cap;
  }
  check(alk_encode_segments_device(src.data(), counts.data(), (uint32_t)ncol, (flags_ & ALK_SESSION_DELTA) ? 2 : 0,
                                   dst.data(), caps.data(), lens.data(), (alk_stream)stream_),
        "segment writer");
  std::vector<uint8_t> host;
  for (size_t k = 0; k < ncol; k++) {
    const std::string& c = a->columnNames[k];
    const size_t len = lens[k];
    host.resize(len);
    ck(cudaMemcpyAsync(host.data(), dst[k], len, cudaMemcpyDeviceToHost, stream_), "segment d2h");
    ck(cudaStreamSynchronize(stream_), "segment d2h");
    stats_.d2h_bytes += len;
    const std::string prefix = base + "." + c;
    const std::string seg_file = prefix + "." + std::to_string(seg) + (code_cols.count(c) ? ".idx" : "");
    if (!write_file(seg_file, host.data(), len)) throw EngineError(ALK_ERR_IO, "Could not write " + seg_file);
    uint32_t cnt = 0;
    std::memcpy(&cnt, host.data(), 4);
    cnt_counts_[prefix] = std::max(cnt_counts_[prefix], cnt);
    if (!write_col_header(prefix + ".header", ColHeader{total, seg + 1, max_recs, cnt_counts_[prefix]}))
      throw EngineError(ALK_ERR_IO, "Could not write " + prefix + ".header");
  }
  for (auto& c : a->columnNames)
    dd_[st.f][c] = a->meta[c].raw ? ColData{2, a->meta[c].width} : ColData{0, a->meta[c].dz};
  if (!save_data_dict(dir_ + "/data.dictionary", dd_)) throw EngineError(ALK_ERR_IO, "Could not write data.dictionary");
  bases_.erase(st.f);  // the table is read afresh by the next statement that names it
  basecols_.erase(st.f);
}

// LOAD 'file' USING (sep) AS (...) (emit_load, operators.cu:2565-2589, and the text source
// CudaSet::LoadBigFile reads, cm.cu:1852-2080): the file is parsed on the device
// (alk_text_load) into a variable of int64 columns, which the statements after it use
// like any computed result (STORE ... BINARY writes it as segments). The reference reads
// the file when a statement first needs the variable; here the LOAD reads it.
void Engine::emit_load(Statement& st) {
  if (st.load_cols.empty()) unsupported("LOAD without columns");
  if (st.load_cols.size() > 32) unsupported("LOAD of more than 32 columns");
  std::vector<alk_text_col> cols(st.load_cols.size());
  for (size_t i = 0; i < st.load_cols.size(); i++) {
    const LoadCol& lc = st.load_cols[i];
    cols[i].field = (uint32_t)std::max(lc.field, 0);
    if (lc.type == "int") {
      cols[i].kind = ALK_TEXT_INT;
    } else if (lc.type == "decimal") {
      cols[i].kind = ALK_TEXT_DECIMAL;
      cols[i].scale = (uint32_t)std::max(lc.size, 0);
    } else if (lc.type == "float" || lc.type == "timestamp") {
      unsupported("LOAD of " + lc.type + " columns (" + lc.name + ")");
    } else {  // every other type name is a char column of the declared width (cm.cu:3006-3012)
      if (lc.size <= 0) unsupported("LOAD of a char column without a width (" + lc.name + ")");
      cols[i].kind = ALK_TEXT_CHAR;
      cols[i].width = (uint32_t)lc.size;
    }
  }
  const std::string path = !st.f.empty() && st.f[0] == '/' ? st.f : dir_ + "/" + st.f;
  // the file straight into the session's pinned staging buffer (a fast copy to the device)
  FILE* fp = std::fopen(path.c_str(), "rb");
  if (!fp) throw EngineError(ALK_ERR_IO, "Could not open file " + st.f);
  std::fseek(fp, 0, SEEK_END);
  const long flen = std::ftell(fp);
  std::fseek(fp, 0, SEEK_SET);
  const size_t tlen = flen > 0 ? (size_t)flen : 0;
  char* text = (char*)pinned(tlen + 1);
  const size_t got_bytes = tlen ? std::fread(text, 1, tlen, fp) : 0;
  std::fclose(fp);
  if (got_bytes != tlen) throw EngineError(ALK_ERR_IO, "Could not read file " + st.f);
  uint64_t rows = 0;  // the records: newline-terminated lines
  for (const char* p = text; (p = (const char*)std::memchr(p, '\n', (size_t)(text + tlen - p))) != nullptr; p++)
    rows++;
  auto out = std::make_unique<Var>();
  out->kind = Var::Mat;
  out->name = st.s;
  out->n = rows;
  std::vector<void*> dst;
  for (size_t i = 0; i < st.load_cols.size(); i++) {
    const LoadCol& lc = st.load_cols[i];
    const bool chr = cols[i].kind == ALK_TEXT_CHAR;
    auto b = mkbuf(std::max<uint64_t>(rows, 1) * (chr ? cols[i].width : 8), stream_);
    out->data[lc.name] = b;
    dst.push_back(b->as<void>());
    out->columnNames.push_back(lc.name);
    ColMeta m;
    m.type = chr ? 2 : 0;
    m.dz = lc.type == "decimal" ? (uint32_t)std::max(lc.size, 0) : 0;  // decimal_zeroes (cm.cu:3000-3005)
    m.width = chr ? cols[i].width : 0;
    m.raw = chr;
    m.no_encoding = chr && lc.no_encoding;
    out->meta[lc.name] = m;
  }
  uint64_t got = 0;
  uint32_t dates = 0;
  check(alk_text_load(text, tlen, st.sep.empty() ? '|' : st.sep[0], cols.data(), (uint32_t)cols.size(), dst.data(),
                      std::max<uint64_t>(rows, 1), &got, &dates, (alk_stream)stream_),
        "text load");
  stats_.h2d_bytes += tlen;
  vars_[st.s] = std::move(out);
}

// ------------------------------------------------------------------ script
void Engine::exec(Statement& st) {
  if (st.op_case) unsupported("CASE expressions");
  // a star join moved the filter queues of its fact and dimension variables into the
  // fact's (check_bitmaps_exist, cm.cu:4151-4206); what later statements would see of
  // them is not restated
  for (const std::string* n : {&st.f})
    if (!n->empty() && star_consumed_.count(*n) && st.kind != StmtKind::Store)
      unsupported("a statement reading " + *n + " after a star join used it");
  for (auto& j : st.op_join)
    if (star_consumed_.count(j)) unsupported("a statement reading " + j + " after a star join used it");
  switch (st.kind) {
    case StmtKind::Filter: emit_filter(st); break;
    case StmtKind::Select: emit_select(st); break;
    case StmtKind::Join: emit_join(st); break;
    case StmtKind::Order: emit_order(st); break;
    case StmtKind::Store: emit_store(st); break;
    case StmtKind::StoreBinary: emit_store_binary(st); break;
    case StmtKind::Display: break;
    case StmtKind::Load: emit_load(st); break;
    case StmtKind::CreateBitmapIndex: emit_create_bitmap_index(st); break;
    default: unsupported("statement kind (catalog commands)");
  }
}

void Engine::reset_script_state() {
  vars_.clear();
  star_sets_.clear();
  star_consumed_.clear();
  stats_ = alk_stats{};
}

// Variables of the catalog tables a script names (load_vars, operators.cu:2708-2747) and
// the last statement that uses every variable (the liveness of the reference's pass one).
void Engine::begin_script(const std::vector<Statement>& sts, std::map<std::string, size_t>& last) {
  std::set<std::string> names;
  for (auto& st : sts) {
    names.insert(st.s);
    names.insert(st.f);
    for (auto& j : st.op_join) names.insert(j);
  }
  for (auto& n : names) {
    Var* b = base_table(n);
    if (b) vars_[n] = std::make_unique<Var>(*b);
  }
  for (size_t i = 0; i < sts.size(); i++) {
    auto& st = sts[i];
    last[st.s] = std::max(last[st.s], i);
    if (!st.f.empty() && st.kind != StmtKind::Store) last[st.f] = i;
    for (auto& j : st.op_join) last[j] = i;
  }
}

void Engine::drop_dead(const std::map<std::string, size_t>& last, size_t i) {
  for (auto it = vars_.begin(); it != vars_.end();) {
    auto l = last.find(it->first);
    if (it->second->kind == Var::Mat && (l == last.end() || l->second <= i)) it = vars_.erase(it);
    else ++it;
  }
}

// Many scripts with one launch for their group-bys: each script runs up to its first
// SELECT that the dense group-by takes, every such SELECT then runs in one batched
// launch, and each script continues from there. Scripts without one run as usual.
// Writes the files on up to 16 threads; writes to one path stay in order on one thread.
void Engine::write_files(const std::vector<PendingWrite>& writes,
                         const std::function<void(size_t, const std::string&)>& failed) {
  std::map<std::string, std::vector<size_t>> by_path;
  for (size_t k = 0; k < writes.size(); k++) by_path[writes[k].path].push_back(k);
  std::vector<const std::vector<size_t>*> groups;
  for (auto& p : by_path) groups.push_back(&p.second);
  std::vector<char> ok(writes.size(), 1);
  std::atomic<size_t> next{0};
  auto worker = [&] {
    for (size_t g; (g = next.fetch_add(1)) < groups.size();)
      for (size_t k : *groups[g]) {
        if (!write_file(writes[k].path, writes[k].data.data(), writes[k].data.size())) ok[k] = 0;
      }
  };
  const size_t nth = std::min<size_t>(groups.size(), std::min<size_t>(16, std::max(1u, std::thread::hardware_concurrency())));
  if (nth <= 1) {
    worker();
  } else {
    std::vector<std::thread> ths;
    for (size_t t = 0; t < nth; t++) ths.emplace_back(worker);
    for (auto& th : ths) th.join();
  }
  for (size_t k = 0; k < writes.size(); k++)
    if (!ok[k]) failed(writes[k].run, writes[k].path);
}

int Engine::execute_batch(const std::vector<std::string>& scripts) {
  struct Run {
    std::vector<Statement> sts;
    std::map<std::string, size_t> last;
    std::map<std::string, std::unique_ptr<Var>> vars;
    std::string text;
    size_t i = 0;
    bool pending = false;
    SelectCtx c;
    int rc = ALK_OK;
    std::string err;
  };
  err_.clear();
  stats_ = alk_stats{};
  const uint64_t k0 = g_kernel_launches;
  std::vector<std::unique_ptr<Run>> runs;
  auto fail = [&](Run& r, int rc, const std::string& m) {
    r.rc = rc;
    r.err = m;
    r.pending = false;
    cudaStreamSynchronize(stream_);
  };
  auto wall = [] {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
  };
  const double w0 = wall();
  // phase 1: every script up to its dense group-by
  for (auto& text : scripts) {
    runs.push_back(std::make_unique<Run>());
    Run& r = *runs.back();
    r.text = text;
    std::string perr;
    if (!parse_script(text, r.sts, perr)) {
      fail(r, ALK_ERR_PARSE, "parse: " + perr);
      continue;
    }
    vars_.clear();
    cur_script_ = text;
    try {
      begin_script(r.sts, r.last);
      for (; r.i < r.sts.size(); r.i++) {
        if (r.sts[r.i].kind == StmtKind::Select && dense_select_prepare(r.sts[r.i], r.c)) {
          r.pending = true;
          break;
        }
        if (!(flags_ & ALK_SESSION_PLAIN) && try_fused(r.sts, r.i)) continue;
        exec(r.sts[r.i]);
        drop_dead(r.last, r.i);
      }
    } catch (const EngineError& e) {
      fail(r, e.code, e.what());
    } catch (const std::exception& e) {
      fail(r, ALK_ERR_ARG, e.what());
    }
    r.vars = std::move(vars_);
    vars_.clear();
  }
  const double w1 = wall();
  // phase 2: one launch
  std::vector<SelectCtx*> batch;
  for (auto& r : runs)
    if (r->pending) batch.push_back(&r->c);
  if (!batch.empty()) {
    try {
      dense_select_run(batch);
    } catch (const EngineError& e) {
      for (auto& r : runs)
        if (r->pending) fail(*r, e.code, e.what());
    }
  }
  const double w2 = wall();
  // phase 3: the rest of every script that waited; a script's last statement, when it
  // is a STORE, leaves its file to be written after the loop
  std::vector<PendingWrite> writes;
  for (size_t k = 0; k < runs.size(); k++) {
    Run& r = *runs[k];
    if (!r.pending) continue;
    vars_ = std::move(r.vars);
    cur_script_ = r.text;
    try {
      dense_select_finish(r.c);
      drop_dead(r.last, r.i);
      for (r.i++; r.i < r.sts.size(); r.i++) {
        if (!(flags_ & ALK_SESSION_PLAIN) && try_fused(r.sts, r.i)) continue;
        const bool defer = r.i + 1 == r.sts.size() && r.sts[r.i].kind == StmtKind::Store;
        deferred_writes_ = defer ? &writes : nullptr;
        deferred_run_ = k;
        exec(r.sts[r.i]);
        deferred_writes_ = nullptr;
        drop_dead(r.last, r.i);
      }
      ck(cudaStreamSynchronize(stream_), "script");
    } catch (const EngineError& e) {
      fail(r, e.code, e.what());
    } catch (const std::exception& e) {
      fail(r, ALK_ERR_ARG, e.what());
    }
    deferred_writes_ = nullptr;
    vars_.clear();
  }
  write_files(writes, [&](size_t run, const std::string& path) {
    fail(*runs[run], ALK_ERR_IO, "Could not open file " + path);
  });
  stats_.batch_host_ms[0] = w1 - w0;
  stats_.batch_host_ms[1] = w2 - w1;
  stats_.batch_host_ms[2] = wall() - w2;
  int rc = ALK_OK;
  for (size_t k = 0; k < runs.size(); k++)
    if (runs[k]->rc != ALK_OK && rc == ALK_OK) {
      rc = runs[k]->rc;
      err_ = "script " + std::to_string(k) + ": " + runs[k]->err;
    }
  if (!(flags_ & ALK_SESSION_RESIDENT)) {
    for (auto& t : basecols_)
      for (auto& c : t.second) {
        if (!c.second.device_only)
          for (auto& d : c.second.dev) d.reset();
        if (c.first.find('.') != std::string::npos) c.second.headers_read = false;  // index: reread
      }
  }
  cudaStreamSynchronize(stream_);
  stats_.kernels = g_kernel_launches - k0;
  return rc;
}

int Engine::execute(const std::string& script) {
  std::vector<Statement> sts;
  std::string perr;
  err_.clear();
  // a script seen before is not parsed again: each run works on a copy of its statements
  auto pc = parsed_.find(script);
  if (pc != parsed_.end()) {
    sts = pc->second;
  } else {
    if (!parse_script(script, sts, perr)) {
      err_ = "parse: " + perr;
      return ALK_ERR_PARSE;
    }
    if (parsed_.size() >= 256) parsed_.clear();
    parsed_.emplace(script, sts);
  }
  return execute_statements(std::move(sts), script);
}

// Runs parsed statements, as the reference's second pass does (bison.y:346-360): from the
// engine's own parser, or from the reference's grammar actions through the emit_*
// boundary. key names the script for the per-script caches (fused graphs, records).
int Engine::execute_statements(std::vector<Statement> sts, const std::string& key) {
  err_.clear();
  reset_script_state();
  cur_script_ = key;
  uint64_t k0 = g_kernel_launches;
  int rc = ALK_OK;
  try {
    // the reference's bitmap CREATE INDEX leaves its four names in the argument queues,
    // and the next statement of another kind reads them as its own (operators.cu:2188-2205
    // never calls clean_queues)
    for (size_t i = 0; i + 1 < sts.size(); i++)
      if (sts[i].kind == StmtKind::CreateBitmapIndex && sts[i + 1].kind != StmtKind::CreateBitmapIndex)
        unsupported("a statement after CREATE INDEX in the same script (the reference passes it the index's names)");
    std::map<std::string, size_t> last;
    begin_script(sts, last);
    for (size_t i = 0; i < sts.size(); i++) {
      if (!(flags_ & ALK_SESSION_PLAIN) && try_fused(sts, i)) continue;
      exec(sts[i]);
      drop_dead(last, i);
    }
    ck(cudaStreamSynchronize(stream_), "script");
  } catch (const EngineError& e) {
    err_ = e.what();
    rc = e.code;
    cudaStreamSynchronize(stream_);
  } catch (const std::exception& e) {
    err_ = e.what();
    rc = ALK_ERR_ARG;
    cudaStreamSynchronize(stream_);
  }
  vars_.clear();
  star_sets_.clear();
  if (!(flags_ & ALK_SESSION_RESIDENT)) {
    for (auto& t : basecols_)
      for (auto& c : t.second) {
        if (!c.second.device_only)
          for (auto& d : c.second.dev) d.reset();
        if (c.first.find('.') != std::string::npos) c.second.headers_read = false;  // index: reread
      }
  }
  cudaStreamSynchronize(stream_);
  stats_.kernels = g_kernel_launches - k0;
  return rc;
}

// ------------------------------------------------------------------ fused pipelines
namespace {
struct FusedFallback : std::runtime_error {
  using std::runtime_error::runtime_error;
};
[[noreturn]] void fallback(const std::string& why) { throw FusedFallback(why); }
// A stage overflowed the size its recorded counts gave it (the counts are now exact),
// or (big) more candidates tie at the LIMIT boundary than the first copy brought back.
struct RerunFused {
  bool big = false;
};

// Counters of the fused stages, copied into pinned host memory ahead of the result rows.
struct FusedStatus {
  alk_stage_status st[3];  // build stage 1, build stage 2, probe-aggregate
  alk_ht_status ht[2];
  int32_t late;  // the late payload fetch could not name a candidate's row
  int32_t pad;
};
constexpr uint64_t kSmallCand = 1024;     // candidate rows returned with the first copy
constexpr uint64_t kCandCap = 1 << 16;    // candidates at most (more ties: operator plan)

// RAII for a stream capture: a capture that does not reach its end (an exception) is
// ended and discarded, with the pinned uploads it made.
struct CaptureGuard {
  cudaStream_t s = nullptr;
  bool active = false;
  void begin(cudaStream_t st) {
    alk::capture_host_buffers().clear();
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed) == cudaSuccess) {
      s = st;
      active = true;
    }
  }
  // ends the capture and returns the graph (null on failure); the pinned uploads move to `bufs`
  cudaGraph_t end(std::vector<void*>& bufs) {
    cudaGraph_t g = nullptr;
    if (!active) return nullptr;
    active = false;
    if (cudaStreamEndCapture(s, &g) != cudaSuccess) g = nullptr;
    bufs.swap(alk::capture_host_buffers());
    alk::capture_host_buffers().clear();
    return g;
  }
  ~CaptureGuard() {
    if (!active) return;
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(s, &g);
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    for (void* p : alk::capture_host_buffers()) cudaFreeHost(p);
    alk::capture_host_buffers().clear();
  }
};
}  // namespace

// An instantiated fused query with the host state its replays need.
struct FusedGraph {
  cudaGraphExec_t exec = nullptr;
  std::vector<void*> host_bufs;  // pinned uploads the graph copies from
  FusedTail tail;
  ~FusedGraph() {
    if (exec) cudaGraphExecDestroy(exec);
    for (void* p : host_bufs) cudaFreeHost(p);
  }
};

namespace {

// One emit_multijoin step resolved like operators.cu:961-1033.
struct StepInfo {
  std::string left, right, lkey, rkey;
  std::vector<std::string> out;  // result columns (op_sel_s order, unique)
};

// Remap column operands of a compiled program from Compiler slot order to the stage's
// operand numbering (scan slot, or 32 + payload column).
void remap(alk_program& p, const std::vector<std::string>& names, const std::map<std::string, uint32_t>& where) {
  for (uint32_t i = 0; i < p.n_instr; i++) {
    alk_instr& in = p.ins[i];
    if (in.ka == ALK_K_COL) in.a = (uint16_t)where.at(names.at(in.a));
    if (in.kb == ALK_K_COL) in.b = (uint16_t)where.at(names.at(in.b));
  }
}

struct HtGuard {
  alk_ht* h = nullptr;
  cudaStream_t s = nullptr;
  void release() {
    alk_ht_free(h, (alk_stream)s);
    h = nullptr;
  }
  ~HtGuard() { release(); }
};
}  // namespace

// Recognises  J := SELECT .. FROM fact JOIN d1 ON .. [JOIN d2 ON ..];
//             F := SELECT .. FROM J GROUP BY ..;  R := ORDER F BY ..;  STORE R .. LIMIT n;
// where J, F and R feed nothing else, and runs it as build stages over the dimension
// side(s), one probe-aggregate pass over the fact table and a top-k selection. The
// result is the reference's: groups equal build rows (the last build key is a group key
// and unique), F's row order is its group-key order (single-segment source), and ORDER
// is stable. Any precondition that fails at run time (duplicate build keys, too many
// ties at the LIMIT boundary) falls back to the operator-at-a-time plan.
bool Engine::try_fused(std::vector<Statement>& sts, size_t& i) {
  if (i + 3 >= sts.size()) return false;
  Statement& J = sts[i];
  Statement& F = sts[i + 1];
  Statement& O = sts[i + 2];
  Statement& S = sts[i + 3];
  if (J.kind != StmtKind::Join || F.kind != StmtKind::Select || O.kind != StmtKind::Order ||
      S.kind != StmtKind::Store)
    return false;
  if (F.f != J.s || O.f != F.s || S.s != O.s || F.grp_cnt == 0) return false;
  if (S.op_nums.empty() || S.op_nums[0] <= 0 || S.op_nums[0] > 4096) return false;
  for (size_t k = 0; k < sts.size(); k++) {
    if (k >= i && k <= i + 3) continue;
    for (const std::string* n : {&J.s, &F.s, &O.s}) {
      if (sts[k].f == *n || sts[k].s == *n) return false;
      for (auto& j : sts[k].op_join)
        if (j == *n) return false;
    }
  }
  if (J.join_tab_cnt < 1 || J.join_tab_cnt > 2) return false;
  if (star_join_applies(J)) return false;  // the reference runs it as a star join
  for (char t : J.join_type)
    if (t != 'I') return false;
  for (auto& kv : J.join_and_cnt)
    if (kv.second) return false;
  // graphs only where every input stays resident between queries
  const std::string gkey = ((flags_ & ALK_SESSION_RESIDENT) && !(flags_ & ALK_SESSION_NOGRAPH))
                               ? cur_script_ + "\n#" + std::to_string(i)
                               : std::string();
  big_fetch_ = false;
  for (int attempt = 0;; attempt++) {
    // this run would capture the query into a graph (its second successful run)
    const bool capturing = !gkey.empty() && fused_seen_.count(gkey) && !fused_graphs_.count(gkey) &&
                           !fused_nograph_.count(gkey);
    try {
      run_fused(J, F, O, S, fused_nograph_.count(gkey) ? std::string() : gkey);
      break;
    } catch (const EngineError& e) {
      if (!capturing) throw;
      // the query could not be captured: it runs without a graph from now on
      cudaGetLastError();
      fused_nograph_.insert(gkey);
      if (attempt >= 2) throw;
    } catch (const FusedFallback& e) {
      big_fetch_ = false;
      return false;
    } catch (const RerunFused& r) {
      // a rerun uses the exact counts the overflowing stage reported, or fetches every
      // tied candidate
      stats_.card_reruns++;
      fused_graphs_.erase(gkey);
      fused_seen_.erase(gkey);
      if (r.big) big_fetch_ = true;
      if (attempt >= 2) {
        big_fetch_ = false;
        return false;
      }
    }
  }
  big_fetch_ = false;
  stats_.plan = std::max<uint32_t>(stats_.plan, 1);
  i += 3;
  return true;
}

// GROUP BY over a base table or a FILTER of one, with group keys and aggregate inputs
// among its columns: the filter and the hash aggregation run as one pass over the resident
// segments (alk_pipeline_groupby), reading every column at its stored width; the groups
// then take the output path of the materialized forms (select_output: key order for one
// segment, MurmurHash64A order of the key tuple across segments). The sort-based form
// keeps the selects whose rows are already in key order (its sort is then skipped), and
// the ones the session pins to it.
bool Engine::hash_select(Statement& st) {
  if ((flags_ & ALK_SESSION_PLAIN) || st.grp_cnt < 1 || st.grp_cnt > 4 || groupby_mode_ == 2) return false;
  Var* a = vars_.count(st.f) ? var(st.f) : nullptr;
  if (!a || (a->kind != Var::Filtered && a->kind != Var::Base)) return false;
  Var* src = a->kind == Var::Filtered ? var(a->source) : a;
  if (src->kind != Var::Base) return false;
  std::vector<std::string> group_cols(st.op_value.end() - st.grp_cnt, st.op_value.end());
  for (auto& g : group_cols)
    if (!a->has(g) || !src->has(g) || a->meta[g].type > 2) return false;
  std::vector<OutSpec> outs;
  std::vector<AggSpec> aggs;
  bool one_line = false;
  compile_select(st, a, true, outs, aggs, one_line);
  for (auto& o : outs) {
    if (o.col_type == 1 && std::find(group_cols.begin(), group_cols.end(), o.field) == group_cols.end()) return false;
    if (o.col_type == 2 && has_col(o.vec)) return false;
  }
  if (aggs.size() > 7) return false;
  const uint32_t skipped = stats_.segments_skipped;
  const uint64_t rows_before = stats_.rows_scanned;
  ScanPlan p = plan_scan(a);
  auto fail = [&]() {
    stats_.segments_skipped = skipped;  // the materialized plan scans again
    stats_.rows_scanned = rows_before;
    return false;
  };
  std::vector<int32_t> key_slots;
  for (auto& g : group_cols) key_slots.push_back((int32_t)p.slot(g));
  std::vector<alk_program> progs(aggs.size());
  std::vector<uint8_t> kinds(aggs.size());
  for (size_t k = 0; k < aggs.size(); k++) {
    kinds[k] = aggs[k].kind;
    std::memset(&progs[k], 0, sizeof(alk_program));
    if (aggs[k].kind == ALK_AGG_COUNT) continue;
    Compiler c;
    progs[k] = c.finish(aggs[k].input);
    std::map<std::string, uint32_t> where;
    for (auto& n : c.slots) {
      if (!src->has(n) || src->meta[n].type > 2) return fail();
      where[n] = p.slot(n);
    }
    remap(progs[k], c.slots, where);
  }
  for (auto& n : p.slots)
    if (src->meta[n].type > 2) return fail();
  auto cs = colsegs(p);
  uint64_t rows = 0;
  for (uint32_t g = 0; g < src->segCount; g++)
    if (p.mode[g]) rows += cs[g].rows;
  uint64_t groups = expected_groups(a, group_cols, std::max<uint64_t>(rows, 1));
  if (groupby_mode_ == 0 && groups > kHashGroupsMax && group_cols.size() == 1) {
    // rows in key order across the scanned segments: the sort-based form skips its sort
    BaseCol& kb = basecol(src, group_cols[0]);
    const uint32_t ks = (uint32_t)key_slots[0];
    std::vector<alk_colseg> kcs(cs.begin() + (size_t)ks * src->segCount, cs.begin() + (size_t)(ks + 1) * src->segCount);
    bool ordered = segs_ascending(kb, kcs, p.mode, true);
    int64_t prev_hi = INT64_MIN;
    for (uint32_t g = 0; ordered && g < src->segCount; g++) {
      if (!p.mode[g]) continue;
      // ascending: the header bounds are the segment's first and last values
      if (kb.segs[g].m.lower < prev_hi) ordered = false;
      prev_hi = kb.segs[g].m.upper;
    }
    if (ordered) return fail();
  }
  // key ranges over the scanned segments (zone maps): a small key space indexes the
  // accumulators directly
  std::vector<int64_t> kmin(group_cols.size(), INT64_MAX), kmax(group_cols.size(), INT64_MIN);
  for (size_t j = 0; j < group_cols.size(); j++) {
    BaseCol& bc = basecol(src, group_cols[j]);
    read_headers(src, group_cols[j], bc);
    for (uint32_t g = 0; g < src->segCount; g++) {
      if (!p.mode[g]) continue;
      kmin[j] = std::min(kmin[j], std::min(bc.segs[g].m.lower, bc.segs[g].m.upper));
      kmax[j] = std::max(kmax[j], std::max(bc.segs[g].m.lower, bc.segs[g].m.upper));
    }
  }
  const size_t cycles = cycle_count(a);
  GroupOut G;
  std::vector<int64_t*> okeys, ovals;
  std::vector<uint64_t> seg_rows(src->segCount, 0);
  uint64_t ng = 0;
  for (int attempt = 0;; attempt++) {
    const uint64_t out_cap = std::max<uint64_t>(groups, 1);
    G.keys.clear();
    G.vals.clear();
    okeys.clear();
    ovals.clear();
    for (size_t j = 0; j < group_cols.size(); j++) {
      G.keys.push_back(mkbuf(out_cap * 8, stream_));
      okeys.push_back(G.keys.back()->as<int64_t>());
    }
    for (size_t k = 0; k < aggs.size(); k++) {
      G.vals.push_back(mkbuf(out_cap * 8, stream_));
      ovals.push_back(G.vals.back()->as<int64_t>());
    }
    if (timing_) cudaEventRecord(ev0_, stream_);
    const int rc = alk_pipeline_groupby(cs.data(), (uint32_t)p.slots.size(), src->segCount, p.mode.data(),
                                        p.has_pred ? &p.pred : nullptr, key_slots.data(),
                                        (uint32_t)key_slots.size(), progs.data(), kinds.data(),
                                        (uint32_t)aggs.size(), groups, kmin.data(), kmax.data(), okeys.data(),
                                        ovals.data(), out_cap, &ng,
                                        seg_rows.data(), nullptr, (alk_stream)stream_);
    if (timing_) {
      cudaEventRecord(ev1_, stream_);
      cudaEventSynchronize(ev1_);
      float ms = 0;
      cudaEventElapsedTime(&ms, ev0_, ev1_);
      stats_.hot_kernel_ms += ms;
      stats_.hot_kernel_launches += 1;
      stats_.hot_kernel_bytes += scan_bytes(p, std::vector<uint32_t>());
    }
    if (rc == ALK_ERR_OVERFLOW && attempt < 3) {
      // more groups than the estimate: size for the count the run reported (or for every
      // row when the table itself filled up)
      groups = std::min<uint64_t>(std::max<uint64_t>(rows, 1), std::max(ng > out_cap ? ng : out_cap * 4, groups));
      continue;
    }
    // a key equal to the free-slot marker, or outside the zone maps' range (the header
    // bounds of a FOR-delta segment are its first and last values)
    if (rc == ALK_ERR_UNSUPPORTED) return fail();
    check(rc, "hash group-by");
    break;
  }
  stats_.hash_groupbys++;
  auto out = std::make_unique<Var>();
  out->kind = Var::Mat;
  out->name = st.s;
  uint64_t kept = 0;
  for (auto n : seg_rows) kept += n;
  if (kept == 0) {
    vars_[st.s] = std::move(out);  // no segment produced rows: empty result without columns
    return true;
  }
  // the reference leaves the select-list order reversed when its first segment is empty
  if (seg_rows[0] == 0) std::reverse(outs.begin(), outs.end());
  G.g = ng;
  G.first = mkbuf(std::max<uint64_t>(ng, 1) * 4, stream_);  // no column reads a group's first row
  ck(cudaMemsetAsync(G.first->as<void>(), 0, std::max<uint64_t>(ng, 1) * 4, stream_), "memset");
  SelectCtx c;
  c.st = &st;
  c.a = a;
  c.grp_cnt = st.grp_cnt;
  c.group_cols = group_cols;
  c.outs = std::move(outs);
  c.cycles = cycles;
  c.G = std::move(G);
  c.okeys = okeys;
  c.R = nullptr;
  c.out = std::move(out);
  select_output(c);
  return true;
}

bool Engine::segs_ascending(BaseCol& bc, const std::vector<alk_colseg>& segs, const std::vector<uint8_t>& mode,
                            bool may_sync) {
  const size_t nseg = segs.size();
  if (bc.dev.size() != nseg || mode.size() != nseg) return false;
  bc.order_buf.resize(nseg);
  bc.ascending.resize(nseg, 0);
  std::vector<uint32_t> todo;
  for (uint32_t g = 0; g < nseg; g++)
    if (mode[g] && (!bc.dev[g] || bc.order_buf[g].lock() != bc.dev[g])) todo.push_back(g);
  if (!todo.empty()) {
    if (!may_sync) return false;
    std::vector<alk_colseg> d;
    for (uint32_t g : todo) {
      if (!bc.dev[g] || segs[g].data != bc.dev[g]->as<void>()) return false;
      d.push_back(segs[g]);
    }
    std::vector<uint8_t> asc(todo.size());
    check(alk_seg_sorted(d.data(), (uint32_t)d.size(), asc.data(), (alk_stream)stream_), "segment order");
    for (size_t k = 0; k < todo.size(); k++) {
      bc.order_buf[todo[k]] = bc.dev[todo[k]];
      bc.ascending[todo[k]] = (int8_t)asc[k];
    }
  }
  for (uint32_t g = 0; g < nseg; g++)
    if (mode[g] && !bc.ascending[g]) return false;
  return true;
}

void Engine::run_fused(Statement& J, Statement& F, Statement& O, Statement& S, const std::string& gkey) {
  cudaStream_t s = stream_;
  // a captured graph of this very query: replay it and do the host part
  if (!gkey.empty() && !big_fetch_) {
    auto it = fused_graphs_.find(gkey);
    if (it != fused_graphs_.end()) {
      std::shared_ptr<FusedGraph> g = it->second;
      cudaEventRecord(evq0_, s);
      ck(cudaGraphLaunch(g->exec, s), "graph launch");
      cudaEventRecord(evq1_, s);
      ck(cudaStreamSynchronize(s), "sync");
      float qms = 0;
      if (cudaEventElapsedTime(&qms, evq0_, evq1_) == cudaSuccess) stats_.query_device_ms += qms;
      g_kernel_launches += g->tail.kernels;
      stats_.d2h_bytes += g->tail.d2h;
      stats_.rows_scanned += g->tail.rows;
      finish_fused(g->tail);
      stats_.plan = 2;
      return;
    }
  }
  const uint64_t rows_before = stats_.rows_scanned;
  // [min, max] of a base column over every segment, from the segment headers (zone maps)
  auto range_of = [&](Var* src, const std::string& col) {
    BaseCol& bc = basecol(src, col);
    read_headers(src, col, bc);
    int64_t lo = INT64_MAX, hi = INT64_MIN;
    for (auto& sg : bc.segs) {
      lo = std::min(lo, std::min(sg.m.lower, sg.m.upper));
      hi = std::max(hi, std::max(sg.m.lower, sg.m.upper));
    }
    return std::make_pair(lo, hi);
  };
  // ---- resolve the join chain (emit_join, operators.cu:832-859)
  std::vector<std::string> op_sel, op_alias;
  for (unsigned k = 0; k < J.sel_count; k++) {
    op_sel.push_back(J.op_value.at(2 * k));
    op_alias.push_back(J.op_value.at(2 * k + 1));
  }
  std::vector<std::string> op_g(J.op_value.begin() + 2 * J.sel_count, J.op_value.end());
  auto step_cols = [&](unsigned tab, Var* left, const std::vector<std::string>& right_cols, StepInfo& si) {
    std::vector<std::string> op_sel_s = op_sel;
    size_t gi = 0;
    for (unsigned z = 0; z < J.join_tab_cnt - tab; z++)
      for (unsigned j = 0; j < 2; j++) op_sel_s.push_back(op_g.at(gi++));
    std::string f1 = op_g.at(gi), f2 = op_g.at(gi + 1);
    auto rhas = [&](const std::string& c) {
      return std::find(right_cols.begin(), right_cols.end(), c) != right_cols.end();
    };
    for (auto& n : op_sel_s)
      if (std::find(si.out.begin(), si.out.end(), n) == si.out.end() && (rhas(n) || left->has(n))) si.out.push_back(n);
    if (left->has(f1) && rhas(f2)) {
      si.lkey = f1;
      si.rkey = f2;
    } else if (rhas(f1) && left->has(f2)) {
      si.rkey = f1;
      si.lkey = f2;
    } else {
      fallback("join columns");
    }
  };
  Var* fact = var(J.f);
  Var* d1 = nullptr;
  Var* d2 = nullptr;  // d2 joins d1 (innermost step) when there are two joins
  StepInfo st1, st2;
  if (J.join_tab_cnt == 2) {
    d2 = var(J.op_join.at(0));
    d1 = var(J.op_join.at(1));
    step_cols(1, d1, d2->columnNames, st1);
    step_cols(2, fact, st1.out, st2);
  } else {
    d1 = var(J.op_join.at(0));
    step_cols(1, fact, d1->columnNames, st2);
  }
  for (Var* v : {fact, d1, d2})
    if (v && v->kind == Var::Mat) fallback("materialized join input");
  // source table of every result column of J (left side wins, operators.cu:1416)
  auto origin = [&](const std::string& c) -> Var* {
    if (fact->has(c)) return fact;
    if (d1->has(c)) return d1;
    if (d2 && d2->has(c)) return d2;
    fallback("column " + c);
  };
  // ---- F over J: compile its select list against J's (aliased) columns
  Var jv;
  jv.kind = Var::Mat;
  std::map<std::string, std::string> src_of;  // J alias -> source column
  for (auto& n : st2.out) {
    auto it = std::find(op_sel.begin(), op_sel.end(), n);
    std::string alias = it == op_sel.end() ? n : op_alias[it - op_sel.begin()];
    jv.columnNames.push_back(alias);
    jv.meta[alias] = origin(n)->meta[n];
    if (alias != n) {
      // an aliased join column keeps the alias's scale, not its own (operators.cu:877-906):
      // the scale of a selected column of that name, else 0
      bool named = std::find(st2.out.begin(), st2.out.end(), alias) != st2.out.end();
      jv.meta[alias].dz = named ? origin(alias)->meta[alias].dz : 0;
    }
    src_of[alias] = n;
  }
  std::vector<std::string> group_cols(F.op_value.end() - F.grp_cnt, F.op_value.end());
  for (auto& g : group_cols)
    if (!jv.has(g) || origin(src_of[g]) == fact) fallback("group key outside the build side");
  const std::string& build_key = st2.rkey;  // unique key of the last build stage
  for (const StepInfo* sp : {&st1, &st2})  // the stages join on integer key values
    if ((sp->rkey.size() && origin(sp->rkey)->meta[sp->rkey].type == 2) ||
        (sp->lkey.size() && origin(sp->lkey)->meta[sp->lkey].type == 2))
      fallback("join on char columns");
  bool key_grouped = false;
  for (auto& g : group_cols)
    if (src_of[g] == build_key) key_grouped = true;
  if (!key_grouped) fallback("build key is not a group key");
  std::vector<OutSpec> outs;
  std::vector<AggSpec> aggs;
  bool one_line = false;
  try {
    compile_select(F, &jv, true, outs, aggs, one_line);
  } catch (const EngineError&) {
    fallback("select list");
  }
  if (aggs.empty() || aggs.size() > 7) fallback("aggregate count");
  // ---- payload columns carried by the last build stage: every build-side column F uses
  std::vector<std::string> payload;  // source column names
  auto need_payload = [&](const std::string& src) {
    if (origin(src) == fact) return;
    if (std::find(payload.begin(), payload.end(), src) == payload.end()) payload.push_back(src);
  };
  // Group and output columns that are the last table's build key read its key column;
  // the key is carried as payload only when an aggregate input reads it.
  for (auto& g : group_cols)
    if (src_of[g] != build_key) need_payload(src_of[g]);
  for (auto& o : outs) {
    if (o.col_type == 1) {
      if (origin(src_of.at(o.field)) == fact) fallback("fact column outside an aggregate");
      if (src_of.at(o.field) != build_key) need_payload(src_of.at(o.field));
    }
    if (o.col_type == 2 && has_col(o.vec)) fallback("row-level expression in a grouped select");
  }
  std::set<std::string> fact_cols;
  bool agg_reads_build = false;  // an aggregate input reads a build-side column
  for (auto& ag : aggs) {
    if (!ag.input) continue;
    std::vector<AstP> stack = {ag.input};
    while (!stack.empty()) {
      AstP a = stack.back();
      stack.pop_back();
      if (!a) continue;
      if (a->k == Ast::Col) {
        const std::string& src = src_of.at(a->col);
        if (origin(src) == fact) fact_cols.insert(src);
        else {
          need_payload(src);
          agg_reads_build = true;
        }
      }
      stack.push_back(a->l);
      stack.push_back(a->r);
    }
  }
  if (payload.size() > 8) fallback("payload width");
  // the first ORDER key is ranked on the device: a build-side column there needs its
  // values for every slot
  bool order_by_build_col = false;
  if (!O.op_type.empty()) {
    const std::string name = O.op_type[0] == "NAME" ? O.op_value.at(0) : O.op_type[0];
    for (auto& o : outs)
      if (o.name == name && o.col_type == 1) order_by_build_col = true;
  }
  // ---- build stages
  // Stage sizes come from the exact counts the previous run of the same stage recorded
  // (the counts the engine learns from its own runs): hash tables from the inserted key
  // count, survivor lists from the survivor count; without a record, the exact upper
  // bound (rows scanned). The stages run without host synchronisation. Their counters
  // are checked once the query's result is back, and a stage that overflowed makes the
  // whole query run again with the counts it reported.
  FusedTail tail;
  tail.small = big_fetch_ ? kCandCap : kSmallCand;
  tail.cand_cap = kCandCap;
  const size_t nback_max = outs.size() + group_cols.size();
  uint8_t* pin = (uint8_t*)pinned(sizeof(FusedStatus) + 8 + tail.small * 8 * nback_max);
  FusedStatus* fs = (FusedStatus*)pin;
  std::memset(fs, 0, sizeof(FusedStatus));
  // On a query's second successful run in a resident session, its device work (from here
  // to the copies of the result) is captured into a CUDA graph and replayed afterwards.
  CaptureGuard cap;
  // the device-side top-k (LIMIT <= 16) keeps the query free of host round trips
  const bool fast = S.op_nums[0] <= 16 && nback_max <= 32;
  const bool capture = fast && !gkey.empty() && !big_fetch_ && !card_record_ && fused_seen_.count(gkey);
  const uint64_t k_before = g_kernel_launches;
  if (capture) cap.begin(s);
  else cudaEventRecord(evq0_, s);
  auto hit_cap_for = [&](const std::string& sig) -> uint64_t {
    auto it = card_feedback_.find(sig + "#hits");
    return it == card_feedback_.end() ? 0 : it->second + it->second / 4 + 4096;
  };
  // A stage without recorded counts is sized by the learned estimator when it is on;
  // returns the fraction of the key range the table is expected to hold (the exact
  // fraction when recording), a feature of the stage that probes it.
  auto is_dense = [](std::pair<int64_t, int64_t> range) {
    return range.second >= range.first && (uint64_t)range.second - (uint64_t)range.first < ALK_DENSE_MAX_SPAN;
  };
  auto build_stage = [&](HtGuard& g, const std::string& sig, uint64_t upper, uint32_t npay,
                         std::pair<int64_t, int64_t> range, int mode, int idx, const CardStage& cst,
                         const std::function<int(alk_ht*, uint64_t, alk_stage_status*)>& run) -> double {
    auto it = card_feedback_.find(sig);
    uint64_t est = it == card_feedback_.end() ? upper : std::min(upper, it->second + it->second / 4 + 1024);
    uint64_t hcap = hit_cap_for(sig);
    uint64_t e_hits = 0, e_keys = 0;
    if (it == card_feedback_.end() && !card_feedback_.count(sig + "#hits") &&
        card_estimate(cst, &e_hits, &e_keys)) {
      est = std::min(upper, e_keys + e_keys / 4 + 1024);
      hcap = std::min(upper, e_hits + e_hits / 4 + 4096);
    }
    if (card_record_) card_record(cst);
    g.s = s;
    // a key range below 2^32 values (the zone maps) takes the dense, rank-addressed
    // table (a bitmap of span/8 bytes plus a u32 rank per bitmap word: 150 MB for the
    // 600M-wide o_orderkey range of a 150M-row orders table); wider ranges the hash table
    const bool dense = is_dense(range);
    if (dense)
      check(alk_ht_create_dense_mode(est, npay, range.first, range.second, mode, &g.h, (alk_stream)s),
            "dense table");
    else check(alk_ht_create_range(est, npay, range.first, range.second, &g.h, (alk_stream)s), "hash table");
    check(run(g.h, hcap, &fs->st[idx]), "build stage");
    check(alk_ht_info_async(g.h, &fs->ht[idx], (alk_stream)s), "hash table");
    tail.pending.push_back({sig, idx, idx, upper});
    stats_.reserved_bytes +=
        alk_ht_bytes(g.h) + (hcap ? hcap : upper) * 8 * (dense && mode == ALK_DENSE_FULL ? 2 + npay : 1);
    const double span = range.second >= range.first ? (double)range.second - (double)range.first + 1.0 : 0.0;
    if (span <= 0) return 0.0;
    if (card_record_) {
      uint64_t n = 0;
      check(alk_ht_info(g.h, &n, nullptr, (alk_stream)s), "hash table");
      return std::min(1.0, (double)n / span);
    }
    return std::min(1.0, (double)est / span);
  };
  auto rows_of = [&](const ScanPlan& p, const std::vector<alk_colseg>& cs) {
    uint64_t n = 0;
    for (uint32_t g = 0; g < p.src->segCount; g++)
      if (p.mode[g]) n += cs[g].rows;
    return n;
  };
  auto plan_sig = [&](const ScanPlan& p) {
    return p.src->table + "|" + std::string((const char*)&p.pred, sizeof(p.pred)) + "|" +
           std::string((const char*)p.mode.data(), p.mode.size());
  };
  HtGuard ht1, ht2;
  alk_ht* last = nullptr;
  std::string last_sig;  // signature of the stage that built `last`
  std::map<std::string, uint32_t> last_pay;  // payload column index in the last table
  double last_fill = 0;                      // fraction of its key range the last table holds
  std::pair<int64_t, int64_t> last_range;    // and that key range
  ScanPlan last_scan;                        // the scan that built it
  // Late payload: when F reads the last table's key and payload columns only as group or
  // output columns (no aggregate input, not the device-ranked ORDER key), and the build
  // table's key column is ascending in its segments, that table keeps ranks only; after
  // the top-k the candidate slots' keys and payload are fetched from the build table's
  // rows by binary search (alk_ht_late_rows). A key found in no row or in several makes
  // the query run again with the full table.
  bool late = false;
  std::map<std::string, uint32_t> late_pay;  // payload column -> late column 1 + index
  std::vector<alk_colseg> late_cs;           // [1 + npay][nseg]: key, payload columns
  std::vector<int64_t> late_lo, late_hi;     // key zone bounds per segment
  auto late_plan = [&](ScanPlan& p, const std::vector<alk_colseg>& cs, const std::string& sig,
                       std::pair<int64_t, int64_t> range) -> bool {
    if (!fast || agg_reads_build || order_by_build_col || late_off_.count(sig) || !is_dense(range)) return false;
    if (p.src->segCount == 0 || p.src->segCount > 65535) return false;
    if (cs.size() < (size_t)p.slots.size() * p.src->segCount) return false;
    for (auto& c : payload)
      if (!p.src->has(c)) return false;  // carried from the inner table
    // exact zone bounds: a FOR header holds the segment's minimum and maximum, a FOR-delta
    // header its first and last value, the same in an ascending segment (checked below)
    BaseCol& kb = basecol(p.src, build_key);
    read_headers(p.src, build_key, kb);
    const uint32_t nseg = p.src->segCount;
    // the candidates' rows are found by binary search: the key column must be ascending
    // in every scanned segment (checked once per resident segment, outside a capture)
    std::vector<alk_colseg> kcs(cs.begin() + (size_t)p.slot(build_key) * nseg,
                                cs.begin() + (size_t)(p.slot(build_key) + 1) * nseg);
    if (!segs_ascending(kb, kcs, p.mode, !capture)) return false;
    std::vector<std::string> names = {build_key};
    names.insert(names.end(), payload.begin(), payload.end());
    late_cs.clear();
    for (auto& c : names) {
      const uint32_t sl = p.slot(c);
      for (uint32_t g = 0; g < nseg; g++) late_cs.push_back(cs.at((size_t)sl * nseg + g));
    }
    late_lo.assign(nseg, 0);
    late_hi.assign(nseg, 0);
    for (uint32_t g = 0; g < nseg; g++) {
      late_lo[g] = kb.segs[g].m.lower;
      late_hi[g] = kb.segs[g].m.upper;
    }
    for (size_t k = 0; k < payload.size(); k++) late_pay[payload[k]] = 1 + (uint32_t)k;
    return true;
  };
  if (J.join_tab_cnt == 2) {
    // stage 1: d2 (innermost right) keyed on st1.rkey, carrying the d2 columns needed later
    ScanPlan p1 = plan_scan(d2);
    uint32_t k1 = p1.slot(st1.rkey);
    std::vector<std::string> pay1;
    for (auto& c : payload)
      if (origin(c) == d2) pay1.push_back(c);
    if (d2->has(build_key) && !d1->has(build_key)) pay1.push_back(build_key);
    std::vector<int32_t> src1;
    for (auto& c : pay1) src1.push_back((int32_t)p1.slot(c));
    auto cs1 = colsegs(p1);
    std::string sig1 = plan_sig(p1) + "|" + st1.rkey;
    CardStage c1;
    c1.p = &p1;
    c1.cs = &cs1;
    c1.key_slot = (int32_t)k1;
    c1.key_range = range_of(p1.src, st1.rkey);
    // a table that carries no payload is probed for membership only
    const int mode1 = pay1.empty() ? ALK_DENSE_BITS : ALK_DENSE_FULL;
    const double fill1 = build_stage(ht1, sig1, rows_of(p1, cs1), (uint32_t)pay1.size(), range_of(p1.src, st1.rkey),
                                     mode1, 0, c1,
                [&](alk_ht* h, uint64_t cap, alk_stage_status* st) {
                  return alk_pipeline_build_async(cs1.data(), (uint32_t)p1.slots.size(), p1.src->segCount,
                                                  p1.mode.data(), p1.has_pred ? &p1.pred : nullptr, nullptr, -1, h,
                                                  (int32_t)k1, src1.data(), cap, st, (alk_stream)s);
                });
    // stage 2: d1 probes stage 1 on st1.lkey and is keyed on the final build key
    ScanPlan p2 = plan_scan(d1);
    uint32_t probe2 = p2.slot(st1.lkey);
    auto slot_or_pay = [&](const std::string& c) -> int32_t {
      if (d1->has(c)) return (int32_t)p2.slot(c);
      auto it = std::find(pay1.begin(), pay1.end(), c);
      if (it == pay1.end()) fallback("payload routing");
      return 32 + (int32_t)(it - pay1.begin());
    };
    int32_t key2 = slot_or_pay(build_key);
    if (key2 >= 32) fallback("build key from the inner table");
    std::vector<int32_t> src2;
    for (auto& c : payload) {
      src2.push_back(slot_or_pay(c));
      last_pay[c] = (uint32_t)src2.size() - 1;
    }
    auto cs2 = colsegs(p2);
    std::string sig2 = plan_sig(p2) + "|" + build_key + "|" + sig1;
    CardStage c2;
    c2.p = &p2;
    c2.cs = &cs2;
    c2.kind = 1;
    c2.probe_slot = (int32_t)probe2;
    c2.probe = ht1.h;
    c2.probe_fill = fill1;
    c2.probe_range = range_of(p1.src, st1.rkey);
    c2.up = &p1;
    c2.key_slot = key2;
    c2.key_range = range_of(p2.src, build_key);
    late = late_plan(p2, cs2, sig2, c2.key_range);
    if (late) {
      src2.clear();
      last_pay.clear();
    }
    last_fill = build_stage(ht2, sig2, rows_of(p2, cs2), (uint32_t)src2.size(), range_of(p2.src, build_key),
                            late ? ALK_DENSE_RANKS : ALK_DENSE_FULL, 1, c2,
                [&](alk_ht* h, uint64_t cap, alk_stage_status* st) {
                  return alk_pipeline_build_async(cs2.data(), (uint32_t)p2.slots.size(), p2.src->segCount,
                                                  p2.mode.data(), p2.has_pred ? &p2.pred : nullptr, ht1.h,
                                                  (int32_t)probe2, h, key2, src2.data(), cap, st, (alk_stream)s);
                });
    last = ht2.h;
    last_sig = sig2;
    last_range = c2.key_range;
    last_scan = p2;
  } else {
    ScanPlan p1 = plan_scan(d1);
    uint32_t k1 = p1.slot(build_key);
    std::vector<int32_t> src1;
    for (auto& c : payload) {
      src1.push_back((int32_t)p1.slot(c));
      last_pay[c] = (uint32_t)src1.size() - 1;
    }
    auto cs1 = colsegs(p1);
    std::string sig1 = plan_sig(p1) + "|" + build_key;
    CardStage c1;
    c1.p = &p1;
    c1.cs = &cs1;
    c1.key_slot = (int32_t)k1;
    c1.key_range = range_of(p1.src, build_key);
    late = late_plan(p1, cs1, sig1, c1.key_range);
    if (late) {
      src1.clear();
      last_pay.clear();
    }
    last_fill = build_stage(ht1, sig1, rows_of(p1, cs1), (uint32_t)src1.size(), range_of(p1.src, build_key),
                            late ? ALK_DENSE_RANKS : ALK_DENSE_FULL, 0, c1,
                [&](alk_ht* h, uint64_t cap, alk_stage_status* st) {
                  return alk_pipeline_build_async(cs1.data(), (uint32_t)p1.slots.size(), p1.src->segCount,
                                                  p1.mode.data(), p1.has_pred ? &p1.pred : nullptr, nullptr, -1, h,
                                                  (int32_t)k1, src1.data(), cap, st, (alk_stream)s);
                });
    last = ht1.h;
    last_sig = sig1;
    last_range = c1.key_range;
    last_scan = p1;
  }
  const uint64_t nslots = alk_ht_slots(last);  // accumulators are indexed by table position
  // ---- probe-aggregate over the fact table
  ScanPlan pf = plan_scan(fact);
  uint32_t probe_f = pf.slot(st2.lkey);
  std::map<std::string, uint32_t> where;  // J alias -> operand index
  for (auto& alias : jv.columnNames) {
    const std::string& src = src_of[alias];
    if (fact_cols.count(src)) where[alias] = pf.slot(src);
    else if (last_pay.count(src)) where[alias] = 32 + last_pay[src];
  }
  std::vector<alk_program> progs(aggs.size());
  std::vector<uint8_t> kinds(aggs.size());
  for (size_t g = 0; g < aggs.size(); g++) {
    kinds[g] = aggs[g].kind;
    std::memset(&progs[g], 0, sizeof(alk_program));
    if (aggs[g].kind == ALK_AGG_COUNT) continue;
    Compiler c;
    progs[g] = c.finish(aggs[g].input);
    remap(progs[g], c.slots, where);
  }
  auto csf = colsegs(pf);
  const uint64_t stride = std::max<uint64_t>(nslots, 1);
  auto acc = mkbuf(stride * 8 * aggs.size(), s);
  auto cnt = mkbuf(stride * 8, s);
  for (size_t g = 0; g < aggs.size(); g++) {
    int64_t init = aggs[g].kind == ALK_AGG_MIN ? INT64_MAX : (aggs[g].kind == ALK_AGG_MAX ? INT64_MIN : 0);
    check(alk_fill_i64(acc->as<int64_t>() + g * stride, stride, init, (alk_stream)s), "init");
  }
  ck(cudaMemsetAsync(cnt->as<void>(), 0, stride * 8, s), "init");
  // events bracket the probe-aggregate stage when timing is on, and always in a graph
  alk_event_timer tm{(timing_ || capture) ? 1 : 0, ev0_, ev1_, 0.0, 0};
  // the probe-aggregate kernel accumulates into slot-indexed arrays sized for every slot
  const std::string sigf = plan_sig(pf) + "|" + st2.lkey + "|" + last_sig;
  if (nslots) {
    CardStage cf;
    cf.p = &pf;
    cf.cs = &csf;
    cf.kind = 2;
    cf.probe_slot = (int32_t)probe_f;
    cf.probe = last;
    cf.probe_fill = last_fill;
    cf.probe_range = last_range;
    cf.key_slot = (int32_t)probe_f;
    cf.key_range = last_range;
    cf.up = &last_scan;
    const uint64_t upper_f = rows_of(pf, csf);
    uint64_t hcap = hit_cap_for(sigf), e_hits = 0, e_keys = 0;
    if (!card_feedback_.count(sigf + "#hits") && card_estimate(cf, &e_hits, &e_keys))
      hcap = std::min(upper_f, e_hits + e_hits / 4 + 4096);
    if (card_record_) card_record(cf);
    stats_.reserved_bytes += (hcap ? hcap : upper_f) * 8;
    check(alk_pipeline_probe_agg_async(csf.data(), (uint32_t)pf.slots.size(), pf.src->segCount, pf.mode.data(),
                                       pf.has_pred ? &pf.pred : nullptr, last, (int32_t)probe_f, progs.data(),
                                       kinds.data(), (uint32_t)aggs.size(), acc->as<int64_t>(), stride,
                                       cnt->as<uint64_t>(), hcap, &fs->st[2], (alk_stream)s, &tm),
          "probe-aggregate");
    tail.pending.push_back({sigf, 2, -1, 0});
    tail.timed = tm.launches > 0;
  }
  // algorithmic bytes of the probe-aggregate stage: the columns every row needs
  // (predicate and probe key) over all rows scanned, plus one value of each aggregate
  // input column per survivor
  {
    std::set<uint32_t> streamed = {probe_f}, per_hit;
    auto cols_of = [](const alk_program& p, std::set<uint32_t>& out) {
      for (uint32_t i = 0; i < p.n_instr; i++) {
        if (p.ins[i].ka == ALK_K_COL && p.ins[i].a < 32) out.insert(p.ins[i].a);
        if (p.ins[i].kb == ALK_K_COL && p.ins[i].b < 32) out.insert(p.ins[i].b);
      }
    };
    if (pf.has_pred) cols_of(pf.pred, streamed);
    for (auto& p : progs) cols_of(p, per_hit);
    for (uint32_t c : streamed) per_hit.erase(c);
    for (uint32_t c : per_hit) {
      uint32_t w = 1;
      BaseCol& bc = basecol(pf.src, pf.slots[c]);
      for (uint32_t g = 0; g < pf.src->segCount; g++)
        if (pf.mode[g]) w = std::max<uint32_t>(w, bc.res_bits.size() > g ? bc.res_bits[g] / 8 : bc.segs[g].m.bits / 8);
      tail.hit_bytes += w;
    }
    tail.streamed_bytes = scan_bytes(pf, std::vector<uint32_t>(streamed.begin(), streamed.end()));
  }
  // ---- F's columns over slots
  std::vector<DevBufP> late_buf;  // slot-indexed key and payload columns, written late
  std::vector<int64_t*> late_ptr;
  if (late)
    for (size_t c = 0; c <= payload.size(); c++) {
      late_buf.push_back(mkbuf(stride * 8, s));
      late_ptr.push_back(late_buf.back()->as<int64_t>());
    }
  auto slot_col = [&](const std::string& alias) -> const int64_t* {
    const std::string& src = src_of.at(alias);
    if (late) return late_ptr.at(src == build_key ? 0 : late_pay.at(src));
    if (src == build_key && !last_pay.count(src)) return alk_ht_keys(last);
    return alk_ht_payload(last, last_pay.at(src));
  };
  std::vector<DevBufP> keep;
  std::vector<const int64_t*> fcol(outs.size());
  std::vector<ColMeta> fmeta(outs.size());
  std::vector<int> fgt(outs.size());
  int countc = -1;
  for (size_t c = 0; c < outs.size(); c++)
    if (outs[c].grp_type == 0 && countc < 0) countc = (int)c;
  for (size_t c = 0; c < outs.size(); c++) {
    const OutSpec& o = outs[c];
    fmeta[c].dz = o.prec;
    fgt[c] = o.grp_type;
    if (o.col_type == 1) {
      fcol[c] = slot_col(o.field);
      fmeta[c].string_map = jv.meta[o.field].string_map;
    } else if (o.col_type == 2 && o.vec->k == Ast::Agg) {
      fcol[c] = acc->as<int64_t>() + (size_t)o.vec->agg * stride;
    } else if (o.col_type == 2) {
      Compiler cc;
      alk_program prog = cc.finish(o.vec);
      std::vector<const int64_t*> in;
      for (auto& sname : cc.slots) in.push_back(acc->as<int64_t>() + std::stoi(sname.substr(4)) * stride);
      auto d = mkbuf(stride * 8, s);
      check(alk_eval(in.data(), (uint32_t)in.size(), nslots, &prog, d->as<int64_t>(), (alk_stream)s), "eval");
      keep.push_back(d);
      fcol[c] = d->as<int64_t>();
    } else {
      auto d = mkbuf(stride * 8, s);
      check(alk_fill_i64(d->as<int64_t>(), stride, (int64_t)(int)o.num, (alk_stream)s), "const");
      keep.push_back(d);
      fcol[c] = d->as<int64_t>();
    }
  }
  for (size_t c = 0; c < outs.size(); c++) {  // AVG finalisation (merge.cu:446-458)
    if (fgt[c] != 1) continue;
    if (countc < 0) fallback("AVG without COUNT");
    AstP e = fmeta[c].dz <= 2 ? mk_bin(ALK_OP_DIV, mk_bin(ALK_OP_MUL, mk_col("s"), mk_const(100)), mk_col("c"))
                              : mk_bin(ALK_OP_DIV, mk_col("s"), mk_col("c"));
    Compiler cc;
    alk_program prog = cc.finish(e);
    std::vector<const int64_t*> in;
    for (auto& sname : cc.slots) in.push_back(sname == "s" ? fcol[c] : fcol[countc]);
    auto d = mkbuf(stride * 8, s);
    check(alk_eval(in.data(), (uint32_t)in.size(), nslots, &prog, d->as<int64_t>(), (alk_stream)s), "avg");
    keep.push_back(d);
    fcol[c] = d->as<int64_t>();
    if (fmeta[c].dz <= 2) fmeta[c].dz += 2;
  }
  // ---- ORDER keys (operators.cu:1641-1798) and the top-k superset
  std::vector<int> okey;
  std::vector<bool> odesc;
  {
    size_t iv = 0;
    for (auto& t : O.op_type) {
      std::string name = t == "NAME" ? O.op_value.at(iv) : t;
      bool desc = t != "NAME" && O.op_value.at(iv) == "DESC";
      iv++;
      int idx = -1;
      for (size_t c = 0; c < outs.size(); c++)
        if (outs[c].name == name) idx = (int)c;
      if (idx < 0) throw EngineError(ALK_ERR_ARG, "Couldn't find name " + name);
      if (!fmeta[idx].string_map.empty()) fallback("ORDER BY on a char column");
      okey.push_back(idx);
      odesc.push_back(desc);
    }
  }
  if (okey.empty()) fallback("ORDER without keys");
  const int64_t* rank = fcol[okey[0]];
  DevBufP rank_buf;
  if (!odesc[0]) {  // ascending: rank by -1 - v (order reversing, no overflow)
    AstP e = mk_bin(ALK_OP_SUB, mk_const(-1), mk_col("v"));
    Compiler cc;
    alk_program prog = cc.finish(e);
    const int64_t* in[1] = {rank};
    rank_buf = mkbuf(stride * 8, s);
    check(alk_eval(in, 1, nslots, &prog, rank_buf->as<int64_t>(), (alk_stream)s), "rank");
    rank = rank_buf->as<int64_t>();
  }
  const uint32_t limit = (uint32_t)S.op_nums[0];
  // the candidate rows come back with F's columns followed by the group keys
  std::vector<const int64_t*> gcol;
  for (auto& g : group_cols) gcol.push_back(slot_col(g));
  std::vector<const int64_t*> back_cols(fcol);
  back_cols.insert(back_cols.end(), gcol.begin(), gcol.end());
  const size_t nback = back_cols.size();
  tail.nouts = outs.size();
  tail.ngroups = gcol.size();
  tail.okey = okey;
  tail.odesc = odesc;
  tail.fmeta = fmeta;
  tail.limit = limit;
  tail.first_key = O.op_type.at(0) == "NAME" ? O.op_value.at(0) : O.op_type.at(0);
  tail.path = S.f;
  tail.sep = S.sep;
  auto cand = mkbuf(kCandCap * 4, s);
  if (fast) {
    // threshold, candidates and their rows on the device; one copy back, the query's only
    // synchronisation
    auto dcount = mkbuf(8, s);
    auto tmp = mkbuf(tail.small * 8 * nback, s);
    check(alk_topk_select(rank, cnt->as<uint64_t>(), nslots, limit, cand->as<uint32_t>(), kCandCap,
                          dcount->as<uint64_t>(), (alk_stream)s),
          "top-k");
    if (late) {
      auto lst = mkbuf(4, s);
      ck(cudaMemsetAsync(lst->as<void>(), 0, 4, s), "late status");
      check(alk_ht_late_rows(last, cand->as<uint32_t>(), dcount->as<uint64_t>(), (uint32_t)kCandCap,
                             late_cs.data(), (uint32_t)payload.size(), last_scan.src->segCount,
                             last_scan.mode.data(), late_lo.data(), late_hi.data(), late_ptr.data(),
                             lst->as<int32_t>(), (alk_stream)s),
            "late rows");
      ck(cudaMemcpyAsync(&fs->late, lst->as<void>(), 4, cudaMemcpyDeviceToHost, s), "d2h");
      tail.late_sig = last_sig;
    }
    check(alk_gather_rows(back_cols.data(), (uint32_t)nback, cand->as<uint32_t>(), dcount->as<uint64_t>(),
                          tail.small, tmp->as<int64_t>(), (alk_stream)s),
          "gather");
    uint8_t* res = pin + sizeof(FusedStatus);
    ck(cudaMemcpyAsync(res, dcount->as<void>(), 8, cudaMemcpyDeviceToHost, s), "d2h");
    ck(cudaMemcpyAsync(res + 8, tmp->as<void>(), tail.small * 8 * nback, cudaMemcpyDeviceToHost, s), "d2h");
    tail.d2h = 8 + tail.small * 8 * nback;
    stats_.d2h_bytes += tail.d2h;
    // every device buffer of the query is released in stream order before the
    // synchronisation (a captured graph owns all of them)
    dcount.reset();
    tmp.reset();
    cand.reset();
    rank_buf.reset();
    keep.clear();
    late_buf.clear();
    acc.reset();
    cnt.reset();
    ht2.release();
    ht1.release();
    tail.kernels = g_kernel_launches - k_before;
    tail.rows = stats_.rows_scanned - rows_before;
    if (capture) {
      auto g = std::make_shared<FusedGraph>();
      g->tail = tail;
      cudaGraph_t graph = cap.end(g->host_bufs);
      const bool ok = graph && cudaGraphInstantiate(&g->exec, graph, 0) == cudaSuccess;
      if (graph) cudaGraphDestroy(graph);
      if (!ok) {
        cudaGetLastError();
        throw EngineError(ALK_ERR_CUDA, "capture of the fused query into a CUDA graph failed");
      }
      cudaEventRecord(evq0_, s);
      ck(cudaGraphLaunch(g->exec, s), "graph launch");
      fused_graphs_[gkey] = g;
    }
    cudaEventRecord(evq1_, s);
    ck(cudaStreamSynchronize(s), "sync");
    float qms = 0;
    if (cudaEventElapsedTime(&qms, evq0_, evq1_) == cudaSuccess) stats_.query_device_ms += qms;
    finish_fused(tail);
    if (!gkey.empty()) fused_seen_.insert(gkey);
    return;
  }
  // LIMIT above 16: the top-k threshold through the host, then every candidate's row
  uint64_t ncand = 0;
  int rc = alk_topk_candidates(rank, cnt->as<uint64_t>(), nslots, limit, cand->as<uint32_t>(), kCandCap, &ncand,
                               (alk_stream)s);
  tail.small = 0;
  finish_fused(tail);  // checks the stages (no rows in pinned memory)
  if (rc == ALK_ERR_OVERFLOW) fallback("too many ties at the LIMIT boundary");
  check(rc, "top-k");
  if (ncand == 0) throw EngineError(ALK_ERR_ARG, "Couldn't find name " + tail.first_key);
  std::vector<std::vector<int64_t>> hf(outs.size(), std::vector<int64_t>(ncand)),
      hg(gcol.size(), std::vector<int64_t>(ncand));
  {
    auto tmp = mkbuf(ncand * 8 * nback, s);
    for (size_t c = 0; c < nback; c++)
      check(alk_gather(back_cols[c], cand->as<uint32_t>(), ncand, tmp->as<int64_t>() + c * ncand, (alk_stream)s),
            "gather");
    for (size_t c = 0; c < nback; c++) {
      auto& dst = c < outs.size() ? hf[c] : hg[c - outs.size()];
      ck(cudaMemcpyAsync(dst.data(), tmp->as<int64_t>() + c * ncand, ncand * 8, cudaMemcpyDeviceToHost, s), "d2h");
    }
    ck(cudaStreamSynchronize(s), "sync");
    stats_.d2h_bytes += ncand * 8 * nback;
  }
  store_fused_rows(tail, hf, hg, ncand);
}

// After the query's one synchronisation: record what every stage counted, or, when a
// stage overflowed, keep the counts up to that stage and drop the later stages' records
// (they ran on incomplete input) and run the query again; then the probe-aggregate
// stage's device time, and (t.small > 0) the rows from pinned memory into the STORE.
void Engine::finish_fused(const FusedTail& t) {
  const FusedStatus* fs = (const FusedStatus*)pin_;
  bool rerun = false;
  for (auto& p : t.pending) {
    if (rerun) {
      card_feedback_.erase(p.sig);
      card_feedback_.erase(p.sig + "#hits");
      continue;
    }
    const alk_stage_status& st = fs->st[p.st];
    if (st.err != ALK_OK && st.err != ALK_ERR_OVERFLOW) throw EngineError(st.err, "fused stage: wait expired");
    card_feedback_[p.sig + "#hits"] = st.hits;
    if (st.err == ALK_ERR_OVERFLOW) {
      rerun = true;  // nothing of this stage was applied; its table count means nothing
      continue;
    }
    if (p.ht < 0) continue;
    const alk_ht_status& h = fs->ht[p.ht];
    if (h.flags[1]) {
      card_feedback_[p.sig] = p.upper;
      rerun = true;
    } else if (h.flags[0] || h.flags[3]) {
      fallback("duplicate build keys or an inconsistent key range");
    } else {
      card_feedback_[p.sig] = h.inserted;
    }
  }
  if (rerun) throw RerunFused();
  if (!t.late_sig.empty() && fs->late) {
    // a candidate key matched no row or several: this stage keeps its payload from now on
    late_off_.insert(t.late_sig);
    throw RerunFused();
  }
  if (timing_ && t.timed) {
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0_, ev1_);
    stats_.hot_kernel_ms += ms;
    stats_.hot_kernel_launches += 1;
    stats_.hot_kernel_bytes += t.streamed_bytes + fs->st[2].hits * t.hit_bytes;
  }
  if (!t.small) return;
  const uint8_t* res = (const uint8_t*)pin_ + sizeof(FusedStatus);
  uint64_t ncand = 0;
  std::memcpy(&ncand, res, 8);
  if (ncand > t.cand_cap) fallback("too many ties at the LIMIT boundary");
  // An empty join leaves the reference's SELECT a column-less set (emit_select,
  // operators.cu:1847-1856), in which ORDER BY cannot find its first key.
  if (ncand == 0) throw EngineError(ALK_ERR_ARG, "Couldn't find name " + t.first_key);
  if (ncand > t.small) throw RerunFused{true};
  const int64_t* rowsb = (const int64_t*)(res + 8);
  std::vector<std::vector<int64_t>> hf(t.nouts), hg(t.ngroups);
  for (size_t c = 0; c < t.nouts + t.ngroups; c++) {
    auto& dst = c < t.nouts ? hf[c] : hg[c - t.nouts];
    dst.assign(rowsb + c * t.small, rowsb + c * t.small + ncand);
  }
  store_fused_rows(t, hf, hg, ncand);
}

// ORDER of the candidates with the full key list (ties: F's group-key order), then STORE
// ... LIMIT (cm.cu:1479-1560).
void Engine::store_fused_rows(const FusedTail& t, std::vector<std::vector<int64_t>>& hf,
                              std::vector<std::vector<int64_t>>& hg, uint64_t ncand) {
  const auto& okey = t.okey;
  const auto& odesc = t.odesc;
  const auto& fmeta = t.fmeta;
  const size_t nouts = t.nouts;
  const uint32_t limit = t.limit;
  std::vector<uint32_t> ord(ncand);
  std::iota(ord.begin(), ord.end(), 0);
  std::sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) {
    for (size_t k = 0; k < okey.size(); k++) {
      int64_t a = hf[okey[k]][x], b = hf[okey[k]][y];
      if (a != b) return odesc[k] ? a > b : a < b;
    }
    for (auto& g : hg)  // F's own row order: group keys ascending
      if (g[x] != g[y]) return g[x] < g[y];
    return false;
  });
  size_t rows = std::min<size_t>(ncand, limit);
  // ---- STORE (cm.cu:1479-1560)
  std::string path = t.path;
  if (path.empty() || path[0] != '/') path = dir_ + "/" + path;
  std::vector<const std::vector<std::string>*> dicts(nouts, nullptr);
  for (size_t c = 0; c < nouts; c++) {
    const std::string& sm = fmeta[c].string_map;
    if (sm.empty()) continue;
    auto dot = sm.find('.');
    Var* b = base_table(sm.substr(0, dot));
    if (!b) throw EngineError(ALK_ERR_IO, "missing dictionary " + sm);
    BaseCol& bc = basecol(b, sm.substr(dot + 1));
    load_dict(b, sm.substr(dot + 1), bc);
    dicts[c] = &bc.dict;
  }
  std::string line, all;
  for (size_t r = 0; r < rows; r++) {
    line.clear();
    for (size_t c = 0; c < nouts; c++) {
      int64_t v = hf[c][ord[r]];
      if (!dicts[c]) {
        if (fmeta[c].dz) {
          std::string d = std::to_string(v);
          while (d.size() <= fmeta[c].dz) d = '0' + d;
          d.insert(d.size() - fmeta[c].dz, ".");
          line += d;
        } else {
          line += std::to_string(v);
        }
      } else {
        std::string d = (v >= 0 && (size_t)v < dicts[c]->size()) ? (*dicts[c])[v] : std::string();
        line += d.substr(0, std::strlen(d.c_str()));
      }
      line += t.sep;
    }
    if (r + 1 != rows) line += "\n";
    all += line;
  }
  if (!write_file(path, all.data(), all.size())) throw EngineError(ALK_ERR_IO, "Could not open file " + path);
}

}  // namespace alk
