// ORACLE — test infrastructure only (see oracle.h). CPU restatement of the
// reference's operators; every function cites the reference file:line it follows.
// The host-side front end (alenka_b200/host/script.cpp) and the catalog/header
// readers (alenka_b200/host/format.cpp) are shared with the product because they
// are the reference's own boundary formats; every codec, predicate, expression,
// aggregation, join and ordering step below is independent of the product.
#include "oracle.h"

#include <omp.h>

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <parallel/algorithm>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../alenka_b200/host/format.h"
#include "../alenka_b200/host/script.h"

namespace orc {

// LIKE as gpu_regex (filter.cu:67-129) matches one fixed-width dictionary entry: '%' any
// run of characters, '?' any character except '.', every other pattern character
// itself. An entry ends at its first NUL or at the width; at most `width` characters are
// examined in all, counting each retry one character further after a '%'. pat is
// NUL-terminated.
bool like_match(const char* entry, uint32_t width, const char* pat) {
  bool after_pct = false;
  uint32_t seen = 0;
  const char* from = entry;  // where the current attempt starts in the entry
  const char* pfrom = pat;   // and in the pattern
  for (;;) {
    const char* s = from;
    const char* p = pfrom;
    int how = 0;  // 0 entry exhausted (or the count reached), 1 a '%' restarts, 2 mismatch
    while (seen < width && *s) {
      if (*p == '%') {
        after_pct = true;
        from = s;
        pfrom = p + 1;
        while (*pfrom == '%') ++pfrom;
        if (!*pfrom) return true;
        how = 1;
        break;
      }
      if (*p == '?' ? *s == '.' : *s != *p) {
        how = 2;
        break;
      }
      ++s;
      ++p;
      ++seen;
    }
    if (how == 1) continue;
    if (how == 0) {
      while (*p == '%') ++p;
      return *p == 0;
    }
    if (!after_pct) return false;
    ++from;
    ++seen;
  }
}
using std::map;
using std::set;
using std::string;
using std::vector;
using i64 = int64_t;
using u32 = uint32_t;

// getFreeMem() (cm.cu:3184) drives segmentation choices in the reference; it is
// pinned to a B200's 180 GB so that segment counts are deterministic.
constexpr size_t kFreeMem = 180ull * 1000 * 1000 * 1000;

struct Error : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// MurmurHash64A, MurmurHash2_64.cu:201-242 (public-domain MurmurHash2, 64-bit A).
uint64_t murmur(const void* key, int len, u32 seed) {
  const uint64_t m = 0xc6a4a7935bd1e995ULL;
  uint64_t h = seed ^ ((uint64_t)(i64)len * m);
  const unsigned char* d = (const unsigned char*)key;
  int nblocks = len / 8;
  for (int b = 0; b < nblocks; b++) {
    uint64_t k = 0;
    for (int j = 7; j >= 0; j--) k = (k << 8) | d[8 * b + j];
    k *= m;
    k ^= k >> 47;
    k *= m;
    h ^= k;
    h *= m;
  }
  const unsigned char* t = d + 8 * nblocks;
  int rem = len & 7;
  if (rem) {
    for (int j = rem - 1; j >= 0; j--) h ^= (uint64_t)t[j] << (8 * j);
    h *= m;
  }
  h ^= h >> 47;
  h *= m;
  h ^= h >> 47;
  return h;
}

// pfor_decompress, compress.cu:180-267 (phase_copy off: always widened to int64).
struct Decoded {
  vector<i64> v;
  i64 orig_lower = 0, header_upper = 0, header_lower = 0;
};
bool decode_image(const uint8_t* img, size_t len, Decoded& out) {
  if (len < 56) return false;
  u32 cnt;
  std::memcpy(&cnt, img, 4);
  if ((size_t)cnt + 56 > len) return false;
  std::memcpy(&out.header_lower, img + 4, 8);
  std::memcpy(&out.header_upper, img + 12, 8);
  u32 comp_type;
  std::memcpy(&comp_type, img + 20, 4);
  const uint8_t* tail = img + cnt;  // fields are read relative to host + cnt
  u32 rec, bits, fit;
  i64 start;
  std::memcpy(&rec, tail + 28, 4);
  std::memcpy(&bits, tail + 32, 4);
  std::memcpy(&out.orig_lower, tail + 36, 8);
  std::memcpy(&fit, tail + 44, 4);
  std::memcpy(&start, tail + 48, 8);
  const uint8_t* p = img + 24;
  out.v.resize(rec);
  if (comp_type == 1) {
    // decompress_functor_int (compress.cu:123-144) then d[0] = start_val; inclusive_scan
    if (bits == 0 || bits > 64 || fit == 0) return false;
    if ((uint64_t)((rec + fit - 1) / fit) * 8 > cnt) return false;
    for (u32 i = 0; i < rec; i++) {
      uint64_t w;
      std::memcpy(&w, p + 8 * (size_t)(i / fit), 8);
      uint64_t tmp = w >> (64 - bits - (i % fit) * bits);
      tmp = tmp << (64 - bits);
      tmp = tmp >> (64 - bits);
      out.v[i] = (i64)(tmp + (uint64_t)out.orig_lower);
    }
    if (rec) out.v[0] = start;
    for (u32 i = 1; i < rec; i++) out.v[i] = (i64)((uint64_t)out.v[i - 1] + (uint64_t)out.v[i]);
    return true;
  }
  if (comp_type != 0) return false;
  // type_to_int64<T> (compress.cu:33-46): dest = (int64)src + lower
  size_t w = bits / 8;
  if (!(bits == 8 || bits == 16 || bits == 32 || bits == 64) || (size_t)rec * w > cnt) return false;
  for (u32 i = 0; i < rec; i++) {
    uint64_t x = 0;
    std::memcpy(&x, p + (size_t)i * w, w);
    i64 s = bits == 64 ? (i64)x : (i64)x;  // unsigned source widened
    out.v[i] = (i64)((uint64_t)s + (uint64_t)out.orig_lower);
  }
  return true;
}

i64 pow10u(u32 p) { return (i64)(unsigned int)std::pow(10.0, (double)p); }

// precision_func, zone_map.cu:668-712 (arguments are updated in place).
u32 precision_func(u32& p1, u32& p2, const string& op) {
  if (op != "DIV") {
    if (op != "MUL") {
      u32 res;
      if (p1 > p2) {
        res = p1;
        p2 = p1 - p2;
        p1 = 0;
      } else {
        res = p1;
        p1 = p2 - p1;
        p2 = 0;
      }
      return res;
    }
    u32 res = p1 + p2;
    p1 = 0;
    p2 = 0;
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

// reverse_op, cm.cu:3166-3180
i64 reverse_op(i64 op) {
  if (op == 2) return 1;
  if (op == 1) return 2;
  if (op == 6) return 5;
  if (op == 5) return 6;
  return op;
}

inline i64 idiv(i64 a, i64 b) { return b == 0 ? 0 : (b == -1 ? (i64)(0 - (uint64_t)a) : a / b); }
inline i64 wadd(i64 a, i64 b) { return (i64)((uint64_t)a + (uint64_t)b); }
inline i64 wsub(i64 a, i64 b) { return (i64)((uint64_t)a - (uint64_t)b); }
inline i64 wmul(i64 a, i64 b) { return (i64)((uint64_t)a * (uint64_t)b); }
inline i64 arith(const string& op, i64 a, i64 b) {
  if (op == "MUL") return wmul(a, b);
  if (op == "ADD") return wadd(a, b);
  if (op == "MINUS") return wsub(a, b);
  return idiv(a, b);
}
inline bool cmp_ll(i64 op, i64 x, i64 y) {  // x OP y with the reference's codes (fl.l:121-127)
  switch (op) {
    case 1: return x < y;
    case 2: return x > y;
    case 5: return x <= y;
    case 6: return x >= y;
    case 4: return x == y;
    default: return x != y;
  }
}

struct ColInfo {
  int type = 0;  // 0 int (decimal/date/dictionary code), 2 char
  bool decimal = false;
  u32 dz = 0;
  u32 char_size = 0;
  string string_map;  // dictionary file path
};

using Vec = vector<i64>;
using VecP = std::shared_ptr<Vec>;

struct Var {
  string name;
  bool not_compressed = true;
  string load_file_name;
  vector<string> columnNames;
  map<string, ColInfo> info;
  size_t segCount = 1, maxRecs = 0, hostRecCount = 0, mRecCount = 0;
  map<string, Vec> h;
  map<string, int> grp_type;
  bool filtered = false;
  string source_name;
  vector<string> fil_type, fil_value;
  vector<i64> fil_nums;
  vector<u32> fil_prec;
  bool has(const string& c) const {
    return std::find(columnNames.begin(), columnNames.end(), c) != columnNames.end();
  }
};

struct Seg {  // one segment of a variable after filtering: int64 columns
  map<string, Vec> c;
  size_t n = 0;
};

class Engine {
 public:
  Engine(string dir, int threads) : dir_(std::move(dir)) {
    if (threads > 0) omp_set_num_threads(threads);
    string e;
    alk::load_data_dict(dir_ + "/data.dictionary", dd_, e);
  }
  uint64_t rows_scanned = 0;

  void run(const string& script) {
    vector<alk::Statement> sts;
    string err;
    if (!alk::parse_script(script, sts, err)) throw Error("parse: " + err);
    // load_vars (operators.cu:2708-2747): every catalog table named in the script
    // becomes a variable holding the columns the script references.
    set<string> names;
    for (auto& st : sts) {
      for (auto& v : st.op_value) names.insert(v);
      names.insert(st.s);
      names.insert(st.f);
      for (auto& j : st.op_join) names.insert(j);
      for (auto& x : st.index_args) names.insert(x);
    }
    for (size_t i = 0; i + 1 < sts.size(); i++)  // emit_create_bitmap_index leaves its names queued
      if (sts[i].kind == alk::StmtKind::CreateBitmapIndex && sts[i + 1].kind != alk::StmtKind::CreateBitmapIndex)
        throw Error("a statement after CREATE INDEX in the same script reads the index's names as its own");
    for (auto& t : dd_) {
      if (!names.count(t.first)) continue;
      load_table(t.first, names);
    }
    for (auto& st : sts) exec(st);
  }

 private:
  string dir_;
  alk::DataDict dd_;
  map<string, std::unique_ptr<Var>> vars_;
  map<string, bool> min_max_eq_;           // compress.cu:196-199, keyed by column name
  map<string, vector<uint8_t>> files_;      // segment file cache

  // emit_load_binary / CudaSet::initialize (operators.cu:2518-2552, cm.cu:2849-2955)
  void load_table(const string& t, const set<string>& referenced) {
    auto v = std::make_unique<Var>();
    v->name = t;
    v->not_compressed = false;
    v->load_file_name = dir_ + "/" + t;
    string first;
    for (auto& c : dd_[t]) {
      if (!referenced.count(c.first)) continue;
      ColInfo ci;
      if (c.second.col_type == 0) {
        ci.type = 0;
        ci.decimal = c.second.col_length != 0 && c.second.col_length != UINT_MAX;
        ci.dz = ci.decimal ? c.second.col_length : 0;
      } else if (c.second.col_type == 2) {
        ci.type = 2;
        ci.char_size = c.second.col_length;
        ci.string_map = dir_ + "/" + t + "." + c.first;
      } else {
        throw Error("float columns are not supported");
      }
      v->columnNames.push_back(c.first);
      v->info[c.first] = ci;
      if (first.empty()) first = c.first;
    }
    if (first.empty()) return;
    alk::ColHeader hdr;
    string e;
    if (!alk::read_col_header(v->load_file_name + "." + first + ".header", hdr, e)) throw Error(e);
    v->segCount = hdr.segs;
    v->maxRecs = hdr.max_recs;
    v->hostRecCount = v->mRecCount = hdr.total;
    vars_[t] = std::move(v);
  }

  const vector<uint8_t>& file(const string& path) {
    auto it = files_.find(path);
    if (it != files_.end()) return it->second;
    vector<uint8_t> b;
    string e;
    if (!alk::read_file(path, b, e)) throw Error(e);
    return files_[path] = std::move(b);
  }
  string seg_path(Var* t, const string& col, unsigned seg) {
    string p = t->load_file_name + "." + col + "." + std::to_string(seg);
    if (t->info[col].type == 2) p += ".idx";
    return p;
  }
  // CopyColumnToGpu(colname, segment) for compressed data (cm.cu:699-798)
  Vec decode_col(Var* t, const string& col, unsigned seg) {
    const auto& img = file(seg_path(t, col, seg));
    Decoded d;
    if (!decode_image(img.data(), img.size(), d)) throw Error("bad segment " + seg_path(t, col, seg));
    min_max_eq_[col] = d.orig_lower == d.header_upper;
    return std::move(d.v);
  }

  Var* var(const string& n) {
    auto it = vars_.find(n);
    if (it == vars_.end()) throw Error("couldn't find variable " + n);
    return it->second.get();
  }

  // ---------------- zone maps: zone_map_check (zone_map.cu:720-1135) ----------------
  static char host_logical_and(char a, char b) {
    if (a == 'A' && b == 'A') return 'A';
    if (a == 'N' || b == 'N') return 'N';
    return 'R';
  }
  static char host_logical_or(char a, char b) {
    if (a == 'A' && b == 'A') return 'A';
    if (a == 'N' && b == 'N') return 'N';
    return 'R';
  }
  static char host_compare_nums(i64 s, i64 d, i64 op) {  // zone_map.cu:78-104
    char res = 'N';
    if (op == 2 && d > s) res = 'A';
    else if (op == 1 && d < s) res = 'A';
    else if (op == 6 && d >= s) res = 'A';
    else if (op == 5 && d <= s) res = 'A';
    else if (op == 4 && d == s) res = 'A';
    else if (d != s) res = 'A';
    return res;
  }
  static char host_compare_range(const i64* c, i64 d, i64 op) {  // zone_map.cu:130-174
    char res = 'R';
    if (op == 2) {
      if (c[1] <= d) res = 'N';
      else if (c[0] > d) res = 'A';
    } else if (op == 1) {
      if (c[0] >= d) res = 'N';
      else if (c[1] < d) res = 'A';
    } else if (op == 6) {
      if (c[1] < d) res = 'N';
      else if (c[0] >= d) res = 'A';
    } else if (op == 5) {
      if (c[0] > d) res = 'N';
      else if (c[1] <= d) res = 'A';
    } else if (op == 4 && c[0] == d && c[1] == d) {
      res = 'A';
    }
    return res;
  }
  static std::array<i64, 2> host_op_scalar(const i64* c, i64 d, const string& op, int reverse) {  // zone_map.cu:513-561
    std::array<i64, 2> t;
    if (reverse == 0 || op == "MUL" || op == "ADD") {
      t[0] = arith(op, c[0], d);
      t[1] = arith(op, c[1], d);
    } else {
      t[0] = arith(op, d, c[0]);
      t[1] = arith(op, d, c[1]);
    }
    return t;
  }
  static std::array<i64, 2> host_op_pair(const i64* c1, const i64* c2, const string& op, int reverse) {  // zone_map.cu:413-458
    std::array<i64, 2> t;
    if (reverse == 0 || op == "MUL" || op == "ADD") {
      t[0] = arith(op, c1[0], c2[0]);
      t[1] = arith(op, c1[1], c2[1]);
    } else {
      t[0] = arith(op, c2[0], c1[0]);
      t[1] = arith(op, c2[1], c1[1]);
    }
    return t;
  }

  char zone_map_check(Var* f, Var* a, unsigned segment, size_t& recs) {
    if (a->not_compressed) return 'R';
    // per-column [min, max] from the segment headers, and the segment row count
    map<string, std::array<i64, 2>> mm;
    for (auto& name : f->fil_value) {
      if (mm.count(name) || !a->has(name)) continue;
      if (a->info[name].type > 1) continue;
      const auto& img = file(seg_path(a, name, segment));
      std::array<i64, 2> r;
      std::memcpy(&r[0], img.data() + 4, 8);
      std::memcpy(&r[1], img.data() + 12, 8);
      u32 cnt, rc;
      std::memcpy(&cnt, img.data(), 4);
      std::memcpy(&rc, img.data() + 28 + cnt, 4);
      recs = rc;
      mm[name] = r;
    }
    vector<string> exe_type, exe_value;
    vector<std::array<i64, 2>> exe_vectors;
    vector<i64> exe_nums;
    vector<char> bools;
    vector<u32> exe_prec;
    size_t iv = 0, in = 0, ip = 0;  // op_value, op_nums, op_nums_precision positions
    auto pop = [](auto& s) { auto x = s.back(); s.pop_back(); return x; };
    auto get_decimals = [&](const string& s) -> u32 {
      if (a->has(s)) return a->info[s].dz;
      return pop(exe_prec);
    };
    auto get_host_vec = [&](const string& s) -> std::array<i64, 2>* {
      if (a->has(s)) return &mm[s];
      exe_vectors.push_back(exe_vectors.back());  // keep storage stable
      exe_vectors.pop_back();
      return nullptr;
    };
    for (auto& ss : f->fil_type) {
      if (ss == "NAME" || ss == "NUMBER" || ss == "FLOAT" || ss == "STRING") {
        exe_type.push_back(ss);
        if (ss == "NUMBER") {
          exe_nums.push_back(f->fil_nums[in]);
          exe_prec.push_back(f->fil_prec[ip++]);
          in++;
        } else if (ss == "NAME" || ss == "STRING") {
          if (ss == "NAME" && !a->has(f->fil_value[iv])) throw Error("Couldn't find column " + f->fil_value[iv]);
          exe_value.push_back(f->fil_value[iv++]);
        }
        continue;
      }
      if (ss == "MUL" || ss == "ADD" || ss == "DIV" || ss == "MINUS") {
        string s1 = pop(exe_type), s2 = pop(exe_type);
        if (s1 == "NUMBER" && s2 == "NUMBER") {
          i64 n1 = pop(exe_nums), n2 = pop(exe_nums);
          u32 p1 = pop(exe_prec), p2 = pop(exe_prec);
          u32 pres = precision_func(p1, p2, ss);
          exe_prec.push_back(pres);
          if (p1) n1 = wmul(n1, pow10u(p1));
          if (p2) n2 = wmul(n2, pow10u(p2));
          exe_type.push_back("NUMBER");
          exe_nums.push_back(arith(ss, n1, n2));
        } else if ((s1 == "NAME" && s2 == "NUMBER") || (s1 == "NUMBER" && s2 == "NAME")) {
          string name = pop(exe_value);
          i64 n1 = pop(exe_nums);
          u32 p2 = pop(exe_prec);
          u32 p1 = get_decimals(name);
          std::array<i64, 2> t;
          if (a->has(name)) t = mm[name];
          else t = pop(exe_vectors);
          u32 pres = precision_func(p1, p2, ss);
          exe_prec.push_back(pres);
          if (p1) {
            t[0] = wmul(t[0], pow10u(p1));
            t[1] = wmul(t[1], pow10u(p1));
            if (a->has(name)) mm[name] = t;  // the reference scales the cached range in place
          }
          if (p2) n1 = wmul(n1, pow10u(p2));
          exe_type.push_back("NAME");
          exe_value.push_back("");
          exe_vectors.push_back(host_op_scalar(t.data(), n1, ss, s1 == "NAME" ? 1 : 0));
        } else if (s1 == "NAME" && s2 == "NAME") {
          string v1 = pop(exe_value), v2 = pop(exe_value);
          u32 p1 = get_decimals(v1), p2 = get_decimals(v2);
          std::array<i64, 2> t = a->has(v1) ? mm[v1] : pop(exe_vectors);
          std::array<i64, 2> s3 = a->has(v2) ? mm[v2] : pop(exe_vectors);
          exe_type.push_back("NAME");
          exe_value.push_back("");
          u32 pres = precision_func(p1, p2, ss);
          exe_prec.push_back(pres);
          if (p1) {
            t[0] = wmul(t[0], pow10u(p1));
            t[1] = wmul(t[1], pow10u(p1));
            if (a->has(v1)) mm[v1] = t;
          }
          if (p2) {
            s3[0] = wmul(s3[0], pow10u(p2));
            s3[1] = wmul(s3[1], pow10u(p2));
            if (a->has(v2)) mm[v2] = s3;
          }
          exe_vectors.push_back(host_op_pair(t.data(), s3.data(), ss, 1));
        } else {
          return 'R';  // string arithmetic: not evaluable on ranges
        }
        continue;
      }
      if (ss == "CMP") {
        i64 cmp = f->fil_nums[in++];
        string s1 = pop(exe_type), s2 = pop(exe_type);
        if (s1 == "NUMBER" && s2 == "NUMBER") {
          i64 n1 = pop(exe_nums), n2 = pop(exe_nums);
          u32 p1 = pop(exe_prec), p2 = pop(exe_prec);
          u32 pres = std::max(p1, p2);
          exe_prec.push_back(pres);
          exe_type.push_back("NAME");
          exe_value.push_back("");
          if (p1) n1 = wmul(n1, pow10u(pres - p1));
          if (p2) n2 = wmul(n2, pow10u(pres - p2));
          bools.push_back(host_compare_nums(n1, n2, cmp));
        } else if ((s1 == "STRING" && s2 == "NAME") || (s1 == "NAME" && s2 == "STRING")) {
          pop(exe_value);
          pop(exe_value);
          bools.push_back('R');
          exe_type.push_back("NAME");
          exe_value.push_back("");
        } else if ((s1 == "NUMBER" && s2 == "NAME") || (s1 == "NAME" && s2 == "NUMBER")) {
          if (s1 == "NAME") cmp = reverse_op(cmp);
          i64 n1 = pop(exe_nums);
          string name = pop(exe_value);
          u32 p2 = pop(exe_prec);
          u32 p1 = get_decimals(name);
          std::array<i64, 2> t = a->has(name) ? mm[name] : pop(exe_vectors);
          u32 pres = std::max(p1, p2);
          exe_prec.push_back(pres);
          if (p1) {
            t[0] = wmul(t[0], pow10u(pres - p1));
            t[1] = wmul(t[1], pow10u(pres - p1));
            if (a->has(name)) mm[name] = t;
          }
          if (p2) n1 = wmul(n1, pow10u(pres - p2));
          exe_type.push_back("NAME");
          exe_value.push_back("");
          bools.push_back(host_compare_range(t.data(), n1, cmp));
        } else {
          return 'R';
        }
        continue;
      }
      if (ss == "AND" || ss == "OR") {
        char s3 = pop(bools), s2 = pop(bools);
        exe_type.push_back("NAME");
        bools.push_back(ss == "AND" ? host_logical_and(s2, s3) : host_logical_or(s2, s3));
        continue;
      }
      if (ss == "JOIN") throw Error("operation = is not valid");
      throw Error("operation " + ss + " is not valid");
    }
    (void)get_host_vec;
    if (bools.empty()) return 'R';
    return bools.back();
  }

  // ---------------- filter(): filter.cu:133-643 ----------------
  // Segment columns in `cols` (full-width int64), n rows.
  vector<uint8_t> filter_eval(Var* f, Var* a, unsigned segment, map<string, Vec>& cols, size_t n) {
    vector<string> exe_type, exe_value;
    vector<VecP> exe_vectors;
    vector<u32> exe_prec;
    vector<i64> exe_nums;
    vector<std::shared_ptr<vector<uint8_t>>> bools;
    size_t iv = 0, in = 0, ip = 0;  // op_value, op_nums, op_nums_precision positions
    auto pop = [](auto& s) { auto x = s.back(); s.pop_back(); return x; };
    auto get_decimals = [&](const string& s) -> u32 {
      if (a->has(s)) return a->info[s].dz;
      return pop(exe_prec);
    };
    auto get_vec = [&](const string& s) -> VecP {
      if (a->has(s)) return std::make_shared<Vec>(cols.at(s));
      return pop(exe_vectors);
    };
    for (auto& ss : f->fil_type) {
      if (ss == "NAME" || ss == "NUMBER" || ss == "FLOAT" || ss == "STRING" || ss == "FIELD") {
        if (ss == "NUMBER") {
          exe_nums.push_back(f->fil_nums[in]);
          exe_prec.push_back(f->fil_prec[ip++]);
          in++;
          exe_type.push_back(ss);
        } else if (ss == "NAME" || ss == "STRING") {
          exe_value.push_back(f->fil_value[iv++]);
          exe_type.push_back(ss);
        } else {
          throw Error("unsupported operand " + ss + " in a filter");
        }
        continue;
      }
      if (ss == "MUL" || ss == "ADD" || ss == "DIV" || ss == "MINUS") {
        string s1 = pop(exe_type), s2 = pop(exe_type);
        if (s1 == "NUMBER" && s2 == "NUMBER") {
          i64 n1 = pop(exe_nums), n2 = pop(exe_nums);
          u32 p1 = pop(exe_prec), p2 = pop(exe_prec);
          u32 pres = precision_func(p1, p2, ss);
          exe_prec.push_back(pres);
          if (p1) n1 = wmul(n1, pow10u(p1));
          if (p2) n2 = wmul(n2, pow10u(p2));
          i64 res = arith(ss, n1, n2);
          exe_type.push_back("NAME");
          exe_value.push_back("");
          exe_vectors.push_back(std::make_shared<Vec>(n, res));
        } else if (s1 == "NAME" && s2 == "NUMBER") {
          string s1v = pop(exe_value);
          i64 n1 = pop(exe_nums);
          u32 p1 = pop(exe_prec);
          u32 p2 = get_decimals(s1v);
          VecP t = get_vec(s1v);
          u32 pres = precision_func(p1, p2, ss);
          exe_prec.push_back(pres);
          exe_type.push_back("NAME");
          exe_value.push_back("");
          exe_vectors.push_back(op_const(*t, n1, ss, true, p1, p2));
        } else if (s1 == "NUMBER" && s2 == "NAME") {
          i64 n1 = pop(exe_nums);
          string s2v = pop(exe_value);
          u32 p1 = pop(exe_prec);
          u32 p2 = get_decimals(s2v);
          VecP t = get_vec(s2v);
          u32 pres = precision_func(p2, p1, ss);
          exe_prec.push_back(pres);
          exe_type.push_back("NAME");
          exe_value.push_back("");
          exe_vectors.push_back(op_const(*t, n1, ss, false, p2, p1));
        } else if (s1 == "NAME" && s2 == "NAME") {
          string s1v = pop(exe_value), s2v = pop(exe_value);
          VecP t1 = get_vec(s1v);
          VecP t = get_vec(s2v);
          u32 p1 = get_decimals(s1v), p2 = get_decimals(s2v);
          u32 pres = precision_func(p1, p2, ss);
          exe_prec.push_back(pres);
          exe_type.push_back("NAME");
          exe_value.push_back("");
          exe_vectors.push_back(op_vec(*t, *t1, ss, false, p2, p1));
        } else {
          throw Error("unsupported string arithmetic in a filter");
        }
        continue;
      }
      if (ss == "CMP") {
        i64 cmp = f->fil_nums[in++];
        string s1 = pop(exe_type), s2 = pop(exe_type);
        auto res = std::make_shared<vector<uint8_t>>(n, 0);
        if (s1 == "NUMBER" && s2 == "NUMBER") {
          i64 n1 = pop(exe_nums), n2 = pop(exe_nums);
          exe_type.push_back("NAME");
          exe_value.push_back("");
          u32 p1 = pop(exe_prec), p2 = pop(exe_prec);
          u32 pres = precision_func(p1, p2, "CMP");
          exe_prec.push_back(pres);
          if (p1) n1 = wmul(n1, pow10u(p1));
          if (p2) n2 = wmul(n2, pow10u(p2));
          bool r = cmp_ll(cmp, n2, n1);  // compare(s, d, op): d OP s (cm.cu:2132-2175)
          std::fill(res->begin(), res->end(), r ? 1 : 0);
          bools.push_back(res);
        } else if ((s1 == "STRING" && s2 == "NAME") || (s1 == "NAME" && s2 == "STRING")) {
          string v1 = pop(exe_value), v2 = pop(exe_value);
          if (s1 == "NAME" && s2 == "STRING") std::swap(v1, v2);  // v1 literal, v2 column
          if (v2.find('.') != string::npos) {
            // a bitmap join index (filter.cu:397-415): the literal padded (or cut) to the
            // dimension column's width, hashed and halved, looked up in the segment's
            // dictionary; cmp_functor_dict keeps the code for == and the others otherwise
            const auto dot = v2.find('.');
            const u32 len = dd_[v2.substr(0, dot)][v2.substr(dot + 1)].col_length;
            string lit = v1;
            while (lit.size() < len) lit.push_back('\0');
            const i64 key = (i64)(murmur(lit.data(), (int)len, alk::kHashSeed) / 2);
            index_compare(a, v2, segment, key, cmp, n, *res);
            exe_type.push_back("NAME");
            bools.push_back(res);
            continue;
          }
          const ColInfo& ci = a->info.at(v2);
          if (cmp == 7) {
            // LIKE: every dictionary entry is matched once and a row passes when its
            // code is among the matches (filter.cu:454-500)
            const auto& dict = file(a->load_file_name + "." + v2);
            const uint32_t w = ci.char_size;
            const size_t entries = w ? dict.size() / w : 0;
            std::vector<char> pat(std::max<size_t>(w, v1.size()) + 1, '\0');
            std::memcpy(pat.data(), v1.data(), v1.size());
            std::vector<char> hit(entries);
            for (size_t k = 0; k < entries; k++)
              hit[k] = like_match((const char*)dict.data() + k * w, w, pat.data());
            const Vec& codes = cols.at(v2);
            for (size_t i = 0; i < n; i++) {
              const i64 c = codes[i];
              (*res)[i] = (c >= 0 && (size_t)c < entries && hit[c]) ? 1 : 0;
            }
            exe_type.push_back("NAME");
            bools.push_back(res);
            continue;
          }
          string lit = v1;
          while (lit.size() < ci.char_size) lit.push_back('\0');
          uint64_t hv = murmur(lit.data(), (int)lit.size(), alk::kHashSeed) / 2;
          // per-row hashes from "<table>.<col>.<seg>.hash" (filter.cu:428-449)
          const auto& hb = file(a->load_file_name + "." + v2 + "." + std::to_string(segment) + ".hash");
          for (size_t i = 0; i < n; i++) {
            uint64_t x;
            std::memcpy(&x, hb.data() + 4 + 8 * i, 8);
            bool eq = x == hv;
            (*res)[i] = cmp == 4 ? eq : (cmp == 3 ? !eq : 0);
          }
          exe_type.push_back("NAME");
          bools.push_back(res);
        } else if ((s1 == "NUMBER" || s2 == "NUMBER") && (s1 == "NAME" || s2 == "NAME") &&
                   !exe_value.empty() && exe_value.back().find('.') != string::npos) {
          // a bitmap join index against a number (filter.cu:519-535, 560-577): the number
          // as it is, looked up in the segment's dictionary; the precision stack is left
          // as it was
          if (s1 == "NAME") cmp = reverse_op(cmp);
          i64 n1 = pop(exe_nums);
          string v = pop(exe_value);
          index_compare(a, v, segment, n1, cmp, n, *res);
          exe_type.push_back("NAME");
          bools.push_back(res);
        } else if (s1 == "NUMBER" && s2 == "NAME") {
          i64 n1 = pop(exe_nums);
          string s1v = pop(exe_value);
          VecP t = get_vec(s1v);
          u32 p2 = pop(exe_prec);
          u32 p1 = get_decimals(s1v);
          u32 pres = std::max(p1, p2);
          exe_prec.push_back(pres);
          exe_type.push_back("NAME");
          compare_const(*t, n1, cmp, pres - p1, pres - p2, *res);
          bools.push_back(res);
        } else if (s1 == "NAME" && s2 == "NUMBER") {
          cmp = reverse_op(cmp);
          i64 n1 = pop(exe_nums);
          string s2v = pop(exe_value);
          VecP t = get_vec(s2v);
          u32 p2 = pop(exe_prec);
          u32 p1 = get_decimals(s2v);
          u32 pres = std::max(p1, p2);
          exe_prec.push_back(pres);
          exe_type.push_back("NAME");
          compare_const(*t, n1, cmp, p1, p2, *res);
          bools.push_back(res);
        } else if (s1 == "NAME" && s2 == "NAME") {
          string s1v = pop(exe_value), s2v = pop(exe_value);
          exe_type.push_back("NAME");
          VecP t = get_vec(s1v);
          VecP t1 = get_vec(s2v);
          u32 p1 = get_decimals(s1v), p2 = get_decimals(s2v);
          exe_prec.push_back(std::max(p1, p2));
          // compare(t1, t, op, p2, p1) (cm.cu:2298-2437); the second operand is read past
          // its end when its scale is non-zero, so only an unscaled right side is defined.
          if (p1) throw Error("column comparison with a scaled right operand is undefined in the reference");
          i64 s2 = pow10u(p2);
          for (size_t i = 0; i < n; i++) (*res)[i] = cmp_ll(cmp, p2 ? wmul((*t1)[i], s2) : (*t1)[i], (*t)[i]);
          bools.push_back(res);
        } else {
          throw Error("unsupported comparison");
        }
        continue;
      }
      if (ss == "AND" || ss == "OR") {
        auto s3 = pop(bools), s2 = pop(bools);
        exe_type.push_back("NAME");
        for (size_t i = 0; i < n; i++) (*s2)[i] = ss == "AND" ? ((*s2)[i] && (*s3)[i]) : ((*s2)[i] || (*s3)[i]);
        bools.push_back(s2);
        continue;
      }
      throw Error("operation " + ss + " is not valid");
    }
    if (bools.empty()) throw Error("filter has no comparison");
    return *bools.back();
  }

  // CudaSet::compare(int_type* column1, int_type d, op, p1, p2) (cm.cu:2250-2295)
  static void compare_const(const Vec& c, i64 d, i64 op, u32 p1, u32 p2, vector<uint8_t>& out) {
    if (p2) d = wmul(d, (i64)std::pow(10.0, (double)p2));
    i64 s1 = pow10u(p1);
    size_t n = c.size();
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) out[i] = cmp_ll(op, p1 ? wmul(c[i], s1) : c[i], d);
  }

  // CudaSet::op(int_type* column1, int_type d, op, reverse, p1, p2) (cm.cu:2480-2556)
  static VecP op_const(const Vec& c, i64 d, const string& op, bool reverse, u32 p1, u32 p2) {
    auto out = std::make_shared<Vec>(c.size());
    i64 d1 = (i64)(unsigned int)d;
    if (p2) d = wmul(d, pow10u(p2));
    i64 s1 = pow10u(p1), s2 = pow10u(p2);
    size_t n = c.size();
    Vec& o = *out;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) {
      i64 x = c[i];
      if (!reverse) {
        if (op == "MUL") o[i] = wmul(x, d1);
        else if (!p1) o[i] = arith(op, x, wmul(d, s2));  // constant scaled twice when p2 != 0
        else o[i] = arith(op, wmul(x, s1), d);
      } else {
        o[i] = arith(op, d, p1 ? wmul(x, s1) : x);
      }
    }
    return out;
  }

  // CudaSet::op(int_type* column1, int_type* column2, op, reverse, p1, p2) (cm.cu:2559-2655)
  static VecP op_vec(const Vec& c1, const Vec& c2, const string& op, bool reverse, u32 p1, u32 p2) {
    auto out = std::make_shared<Vec>(c1.size());
    i64 s1 = pow10u(p1), s2 = pow10u(p2);
    size_t n = c1.size();
    Vec& o = *out;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) {
      i64 a = c1[i], b = c2[i];
      if (op == "MUL") {
        o[i] = wmul(a, b);
        continue;
      }
      if (p1) a = wmul(a, s1);
      if (p2) b = wmul(b, s2);
      o[i] = reverse ? arith(op, b, a) : arith(op, a, b);
    }
    return out;
  }

  // copyColumns (cm.cu:3305-3347) with filter_op (cm.cu:3609-3666) for one segment.
  Seg fetch(Var* a, const vector<string>& fields, unsigned segment) {
    Seg s;
    if (a->filtered) {
      Var* t = var(a->source_name);
      size_t recs = 0;
      char zm = zone_map_check(a, t, segment, recs);
      vector<u32> prm;
      bool all = false;
      if (zm == 'R') {
        map<string, Vec> pc;
        size_t n = 0;
        for (auto& fv : a->fil_value)
          if (t->has(fv) && !pc.count(fv)) {
            pc[fv] = decode_col(t, fv, segment);
            n = pc[fv].size();
          }
        rows_scanned += n;
        vector<uint8_t> mask = filter_eval(a, t, segment, pc, n);
        for (size_t i = 0; i < n; i++)
          if (mask[i]) prm.push_back((u32)i);
      } else if (zm == 'A') {
        all = true;
        rows_scanned += recs;
      }
      if (!all && prm.empty()) return s;
      for (auto& fl : fields) {
        if (s.c.count(fl) || !a->has(fl)) continue;
        Vec full = decode_col(t, fl, segment);
        if (all) {
          s.n = full.size();
          s.c[fl] = std::move(full);
        } else {
          Vec g(prm.size());
          for (size_t i = 0; i < prm.size(); i++) g[i] = full[prm[i]];
          s.n = g.size();
          s.c[fl] = std::move(g);
        }
      }
      if (fields.empty() || s.c.empty()) s.n = all ? recs : prm.size();
      return s;
    }
    if (!a->not_compressed) {
      size_t n = 0;
      for (auto& fl : fields) {
        if (s.c.count(fl) || !a->has(fl)) continue;
        s.c[fl] = decode_col(a, fl, segment);
        n = s.c[fl].size();
      }
      s.n = n;
      rows_scanned += n;
      return s;
    }
    // not_compressed host data (CopyColumnToGpu, cm.cu:702-731)
    size_t begin = segment * a->maxRecs;
    size_t cnt = segment < a->segCount - 1 ? a->maxRecs : a->hostRecCount - a->maxRecs * (a->segCount - 1);
    for (auto& fl : fields) {
      if (s.c.count(fl) || !a->has(fl)) continue;
      const Vec& src = a->h.at(fl);
      s.c[fl] = Vec(src.begin() + begin, src.begin() + begin + cnt);
    }
    s.n = cnt;
    return s;
  }

  size_t cycles(Var* a) {
    if (a->filtered) return var(a->source_name)->segCount;
    return a->segCount;
  }

  // ---------------- star join with bitmap join indexes ----------------
  // Index segment <fact>.<dimension>.<column>.<segment> as loadIndex reads it
  // (cm.cu:2775-2845): the dictionary and every row's code.
  struct IndexSeg {
    vector<i64> dict;
    vector<u32> codes;
  };
  map<string, IndexSeg> index_cache_;
  const IndexSeg& index_seg(Var* a, const string& name, unsigned segment) {
    const string path = a->load_file_name + "." + name + "." + std::to_string(segment);
    auto it = index_cache_.find(path);
    if (it != index_cache_.end()) return it->second;
    vector<uint8_t> b;
    string e;
    if (!alk::read_file(path, b, e)) throw Error(e);
    IndexSeg x;
    u32 sz, fit, bits, vals, real;
    std::memcpy(&sz, b.data(), 4);
    x.dict.resize(sz);
    std::memcpy(x.dict.data(), b.data() + 4, (size_t)sz * 8);
    const size_t h = 4 + (size_t)sz * 8;
    std::memcpy(&fit, b.data() + h, 4);
    std::memcpy(&bits, b.data() + h + 4, 4);
    std::memcpy(&vals, b.data() + h + 8, 4);
    std::memcpy(&real, b.data() + h + 12, 4);
    x.codes.resize(real);
    for (u32 i = 0; i < real; i++) {  // cmp_functor_dict (filter.cu:30-50)
      uint64_t w;
      std::memcpy(&w, b.data() + h + 16 + (size_t)(i / fit) * 8, 8);
      uint64_t t = w >> ((fit - (i % fit)) - 1) * bits;
      t = t << (64 - bits);
      t = t >> (64 - bits);
      x.codes[i] = (u32)t;
    }
    return index_cache_[path] = std::move(x);
  }
  // filter.cu:397-415 and cmp_functor_dict: key's position in the segment's dictionary;
  // == keeps that code, every other operator the other codes; a key the dictionary lacks
  // keeps nothing
  void index_compare(Var* a, const string& name, unsigned segment, i64 key, i64 cmp, size_t n,
                     vector<uint8_t>& out) {
    const IndexSeg& x = index_seg(a, name, segment);
    if (x.codes.size() != n) throw Error("index " + name + " holds another row count than its segment");
    auto it = std::find(x.dict.begin(), x.dict.end(), key);
    if (it == x.dict.end()) {
      std::fill(out.begin(), out.end(), 0);
      return;
    }
    const u32 idx = (u32)(it - x.dict.begin());
    for (size_t i = 0; i < n; i++) out[i] = cmp == 4 ? (x.codes[i] == idx) : (x.codes[i] != idx);
  }

  // std::lower_bound over v[0, m)
  static size_t lower_bound_pos(const Vec& v, size_t m, i64 key) {
    return (size_t)(std::lower_bound(v.begin(), v.begin() + m, key) - v.begin());
  }

  // emit_create_bitmap_index (operators.cu:2188-2268) with compress_int (cm.cu:4271-4336)
  void create_bitmap_index(alk::Statement& st) {
    const string& ltable = st.f;
    const string& rtable = st.index_args.at(0);
    const string& rcol = st.index_args.at(1);
    const string& lid = st.index_args.at(2);
    const string& rid = st.index_args.at(3);
    Var* left = var(ltable);
    Var* right = var(rtable);
    if (right->segCount != 1) throw Error("a bitmap index over a dimension of several segments");
    Vec keys = decode_col(right, rid, 0);
    const size_t m = keys.size();
    const bool chr = right->info.at(rcol).type == 2;
    Vec rv;
    if (!chr) {
      rv = decode_col(right, rcol, 0);
    } else {
      const auto& hb = file(right->load_file_name + "." + rcol + ".0.hash");
      u32 cnt;
      std::memcpy(&cnt, hb.data(), 4);
      rv.resize(cnt);
      std::memcpy(rv.data(), hb.data() + 4, (size_t)cnt * 8);
    }
    for (unsigned i = 0; i < left->segCount; i++) {
      Vec fk = decode_col(left, lid, i);
      const size_t n = fk.size();
      // res_h: the segment's values, then (char) the dimension's hashes past n
      vector<i64> res(chr ? std::max(n, rv.size()) : n, 0);
      if (chr)
        for (size_t k = n; k < rv.size(); k++) res[k] = rv[k];
      for (size_t k = 0; k < n; k++) {
        const size_t p = lower_bound_pos(keys, m, fk[k]);
        if (p >= m) throw Error("a foreign key past the dimension's last key");
        res[k] = rv[p];
      }
      // compress_int: dictionary of the distinct values in order, codes, packing
      std::set<i64> dict_s(res.begin(), res.end());
      map<i64, u32> d_ordered;
      u32 c = 0;
      for (i64 v : dict_s) d_ordered[v] = c++;
      vector<u32> dict_val;
      for (i64 v : res) dict_val.push_back(d_ordered[v]);
      const u32 bits = (u32)std::ceil(std::log2(double(d_ordered.size() + 1)));
      const u32 sz = (u32)d_ordered.size();
      string out;
      auto put = [&](const void* p, size_t k) { out.append((const char*)p, k); };
      put(&sz, 4);
      for (auto& kv : d_ordered) put(&kv.first, 8);
      const u32 fit_count = 64 / bits;
      put(&fit_count, 4);
      put(&bits, 4);
      u32 vals_count = (u32)dict_val.size() / fit_count;
      if (!vals_count || dict_val.size() % fit_count) vals_count++;
      put(&vals_count, 4);
      const u32 real_count = (u32)dict_val.size();
      put(&real_count, 4);
      uint64_t val = 0;
      u32 curr = 1;
      for (size_t k = 0; k < dict_val.size(); k++) {
        val = val | dict_val[k];
        if (curr < fit_count) val = val << bits;
        if (curr == fit_count || k == dict_val.size() - 1) {
          if (curr < fit_count) val = val << ((fit_count - curr) - 1) * bits;
          curr = 1;
          put(&val, 8);
          val = 0;
        } else {
          curr++;
        }
      }
      const string path = dir_ + "/" + ltable + "." + rtable + "." + rcol + "." + std::to_string(i);
      if (!alk::write_file(path, out.data(), out.size())) throw Error("cannot write " + path);
      index_cache_.erase(path);
    }
  }

  string table_of(Var* v) {
    Var* b = v->filtered ? var(v->source_name) : v;
    if (b->not_compressed) throw Error("a star join over a materialized result");
    return b->name;
  }
  static bool file_exists(const string& p) {
    FILE* f = std::fopen(p.c_str(), "rb");
    if (!f) return false;
    std::fclose(f);
    return true;
  }
  // check_star_join (operators.cu:408-437) with check_bitmap_file_exist (cm.cu:4131-4149)
  bool check_star_join(alk::Statement& st) {
    if (st.join_tab_cnt == 0) return false;
    Var* left = var(st.f);
    for (size_t k = 2 * (size_t)st.sel_count; k < st.op_value.size(); k += 2)
      if (!left->has(st.op_value[k])) return false;
    if (st.join_tab_cnt == 1) {
      Var* right = var(st.op_join.at(0));
      if (right->fil_value.empty()) return false;
      const string lt = table_of(left), rt = table_of(right);
      for (auto& c : right->fil_value)
        if (right->has(c) && !file_exists(dir_ + "/" + lt + "." + rt + "." + c + ".0")) return false;
    }
    return true;
  }
  // the stored value of row r of a FOR segment file as star_join reads it
  // (operators.cu:594-650): 8-bit values through a signed char, plus the header's lower
  i64 stored_value(Var* t, const string& col, unsigned seg, u32 r, size_t n) {
    const auto& img = file(seg_path(t, col, seg));
    u32 cnt, comp, bits;
    i64 lower;
    std::memcpy(&cnt, img.data(), 4);
    std::memcpy(&lower, img.data() + 4, 8);
    std::memcpy(&comp, img.data() + 20, 4);
    std::memcpy(&bits, img.data() + 24 + cnt + 8, 4);
    if (comp != 0) throw Error("a star join over the FOR-delta column " + col);
    if (r >= n) throw Error("a star join row past its segment");
    const uint8_t* p = img.data() + 24;
    i64 raw;
    if (bits == 8) raw = (i64)(int8_t)p[r];
    else if (bits == 16) { uint16_t x; std::memcpy(&x, p + 2 * (size_t)r, 2); raw = x; }
    else if (bits == 32) { u32 x; std::memcpy(&x, p + 4 * (size_t)r, 4); raw = x; }
    else std::memcpy(&raw, p + 8 * (size_t)r, 8);
    return (i64)((uint64_t)raw + (uint64_t)lower);
  }
  // star_join (operators.cu:440-794)
  void star_join(alk::Statement& st) {
    Var* left = var(st.f);
    Var* lbase = left->filtered ? var(left->source_name) : left;
    const string ltab = table_of(left);
    vector<string> sel;
    for (unsigned k = 0; k < st.sel_count; k++) {
      if (st.op_value[2 * k] != st.op_value[2 * k + 1]) throw Error("an alias in a star join");
      sel.push_back(st.op_value[2 * k]);
    }
    Var f = *left;  // the fact's filter with the dimensions' appended (check_bitmaps_exist)
    f.h.clear();
    struct Dim {
      string fk, key;
      Var* base;
      Var* r;
    };
    map<string, Dim> dims;  // key_map
    const size_t g0 = 2 * (size_t)st.sel_count;
    for (unsigned i = 0; i < st.join_tab_cnt; i++) {
      Dim d;
      d.fk = st.op_value.at(g0 + 2 * i);
      d.key = st.op_value.at(g0 + 2 * i + 1);
      const string jvar = st.op_join.at(st.join_tab_cnt - 1 - i);
      d.r = var(jvar);
      d.base = d.r->filtered ? var(d.r->source_name) : d.r;
      if (d.base->segCount != 1) throw Error("a star join with a dimension of several segments");
      const string rt = table_of(d.r);
      if (!d.r->fil_value.empty()) {
        for (auto& c : d.r->fil_value)
          if (d.r->has(c) && !file_exists(dir_ + "/" + ltab + "." + rt + "." + c + ".0"))
            throw Error("Required bitmap on table " + jvar + " doesn't exists");
        const bool add_and = !f.fil_type.empty();
        f.fil_nums.insert(f.fil_nums.end(), d.r->fil_nums.begin(), d.r->fil_nums.end());
        f.fil_prec.insert(f.fil_prec.end(), d.r->fil_prec.begin(), d.r->fil_prec.end());
        for (auto& c : d.r->fil_value) f.fil_value.push_back(d.r->has(c) ? rt + "." + c : c);
        f.fil_type.insert(f.fil_type.end(), d.r->fil_type.begin(), d.r->fil_type.end());
        if (add_and) f.fil_type.push_back("AND");
      }
      dims[jvar] = d;
    }
    if (f.fil_type.empty()) throw Error("a star join without a filter");
    auto c = std::make_unique<Var>();
    c->name = st.s;
    c->not_compressed = true;
    for (auto& name : sel) {
      if (c->has(name)) continue;
      c->columnNames.push_back(name);
      if (left->has(name)) c->info[name] = lbase->info.at(name);
      else {
        bool found = false;
        for (auto& kv : dims)
          if (kv.second.r->has(name)) {
            c->info[name] = kv.second.base->info.at(name);
            found = true;
            break;
          }
        if (!found) throw Error("the star join column " + name + " is in no joined table");
      }
      if (left->has(name) && c->info[name].type == 2) throw Error("a char fact column in a star join");
    }
    map<string, std::pair<Vec, Vec>> dim_cols;  // (key column, value column) per dimension column
    vector<u32> prm;                              // left->prm_d, kept from segment to segment
    size_t total = 0;
    bool seg0_rows = false;
    for (unsigned g = 0; g < lbase->segCount; g++) {
      map<string, Vec> cols;
      size_t n = 0;
      for (auto& fv : f.fil_value)
        if (lbase->has(fv) && !cols.count(fv)) {
          cols[fv] = decode_col(lbase, fv, g);
          n = cols[fv].size();
        }
      if (!n) n = decode_col(lbase, lbase->columnNames.at(0), g).size();
      rows_scanned += n;
      vector<uint8_t> mask = filter_eval(&f, lbase, g, cols, n);
      size_t cnt = 0;
      for (size_t i = 0; i < n; i++) cnt += mask[i] != 0;
      if (!cnt) continue;
      if (g == 0) seg0_rows = true;
      prm.resize(cnt, 0);
      size_t w = 0;
      for (size_t i = 0; i + 1 < n; i++)  // copy_if over [0, n - 1)
        if (mask[i]) prm[w++] = (u32)i;
      for (auto& name : sel) {
        Vec& out = c->h[name];
        if (out.size() > total) continue;  // a repeated column
        if (left->has(name)) {
          for (size_t k = 0; k < cnt; k++) out.push_back(stored_value(lbase, name, g, prm[k], n));
          continue;
        }
        for (auto& kv : dims) {
          Dim& d = kv.second;
          if (!d.r->has(name)) continue;
          auto& dc = dim_cols[kv.first + "." + name];
          if (dc.first.empty()) {
            dc.first = decode_col(d.base, d.key, 0);
            dc.second = decode_col(d.base, name, 0);
          }
          const auto& fimg = file(seg_path(lbase, d.fk, g));
          i64 lower;
          std::memcpy(&lower, fimg.data() + 4, 8);
          for (size_t k = 0; k < cnt; k++) {
            const i64 raw = (i64)((uint64_t)stored_value(lbase, d.fk, g, prm[k], n) - (uint64_t)lower);
            u32 t = (u32)raw;
            if (lower != 1) t += (u32)(lower - 1);
            const size_t p = lower_bound_pos(dc.first, dc.first.size(), (i64)t);
            if (p >= dc.first.size()) throw Error("a star join key past the dimension's last key");
            out.push_back(dc.second[p]);
          }
          break;
        }
      }
      total += cnt;
    }
    // a char dimension column gets its dictionary while the first segment is gathered
    // (operators.cu:672-677); without rows there it has none
    for (auto& name : c->columnNames)
      if (!left->has(name) && c->info[name].type == 2 && total && !seg0_rows)
        throw Error("a char dimension column whose first fact segment keeps no row");
    for (auto& name : c->columnNames) c->h[name].resize(total);
    c->mRecCount = c->hostRecCount = c->maxRecs = total;
    vars_[st.s] = std::move(c);
  }

  // ---------------- statements ----------------
  void exec(alk::Statement& st) {
    switch (st.kind) {
      case alk::StmtKind::Filter: emit_filter(st); break;
      case alk::StmtKind::Select: emit_select(st); break;
      case alk::StmtKind::Join: emit_join(st); break;
      case alk::StmtKind::Order: emit_order(st); break;
      case alk::StmtKind::Store: emit_store(st); break;
      case alk::StmtKind::Display: break;
      case alk::StmtKind::CreateBitmapIndex: create_bitmap_index(st); break;
      default: throw Error("statement kind not supported by the oracle");
    }
  }

  // emit_filter (operators.cu:2306-2408): lazy; a filter over a filtered variable
  // appends its program and an AND.
  void emit_filter(alk::Statement& st) {
    Var* a = var(st.f);
    auto b = std::make_unique<Var>();
    *b = *a;
    b->h.clear();
    b->name = st.s;
    b->fil_type = st.op_type;
    b->fil_value = st.op_value;
    b->fil_nums = st.op_nums;
    b->fil_prec = st.op_nums_precision;
    b->filtered = true;
    if (a->filtered) {
      b->source_name = a->source_name;
      b->fil_value.insert(b->fil_value.end(), a->fil_value.begin(), a->fil_value.end());
      b->fil_type.insert(b->fil_type.end(), a->fil_type.begin(), a->fil_type.end());
      b->fil_type.push_back("AND");
      b->fil_nums.insert(b->fil_nums.end(), a->fil_nums.begin(), a->fil_nums.end());
      b->fil_prec.insert(b->fil_prec.end(), a->fil_prec.begin(), a->fil_prec.end());
    } else {
      if (a->not_compressed) throw Error("FILTER over a materialized result is not supported by the oracle");
      b->source_name = st.f;
    }
    vars_[st.s] = std::move(b);
  }

  struct OutCol {
    string name;
    Vec v;
    u32 dz = 0;
    int grp_type = 3;
    string string_map;
  };

  // select() (select.cu:359-952) over one segment `a` with group starts `grp`.
  bool select_seg(alk::Statement& st, Var* av, Seg& a, const vector<u32>& grp, size_t grp_count,
                  vector<OutCol>& b, size_t& b_rows) {
    vector<string> exe_type, exe_value;
    vector<VecP> exe_vectors;
    vector<i64> exe_nums;
    vector<u32> exe_prec;
    struct Rec { string col_val, grp_type; int col_type; i64 num = 0; u32 prec = 0; string value; VecP vec; };
    vector<Rec> recs;
    bool one_line = false;
    size_t n = a.n;
    size_t res_size = (grp_count && n != 0) ? grp_count : 0;
    size_t iv = 0, in = 0, ip = 0;  // op_value, op_nums, op_nums_precision positions
    auto pop = [](auto& s) { auto x = s.back(); s.pop_back(); return x; };
    auto is_col = [&](const string& s) { return av->has(s); };
    auto get_decimals = [&](const string& s) -> u32 {
      if (is_col(s)) return av->info[s].dz;
      return pop(exe_prec);
    };
    auto get_vec = [&](const string& s) -> VecP {
      if (is_col(s)) return std::make_shared<Vec>(a.c.at(s));
      return pop(exe_vectors);
    };
    auto segreduce = [&](const Vec& x, int kind) {  // 0 sum, 1 min, 2 max over grp segments
      Vec out(res_size);
      for (size_t g = 0; g < grp_count; g++) {
        size_t lo = grp[g], hi = g + 1 < grp_count ? grp[g + 1] : n;
        i64 acc = kind == 0 ? 0 : x[lo];
        for (size_t i = lo; i < hi; i++) {
          if (kind == 0) acc = wadd(acc, x[i]);
          else if (kind == 1) acc = std::min(acc, x[i]);
          else acc = std::max(acc, x[i]);
        }
        out[g] = acc;
      }
      return out;
    };
    auto reduce = [&](const Vec& x, int kind) {
      i64 acc = kind == 0 ? 0 : (n ? x[0] : 0);
      for (size_t i = 0; i < n; i++) {
        if (kind == 0) acc = wadd(acc, x[i]);
        else if (kind == 1) acc = std::min(acc, x[i]);
        else acc = std::max(acc, x[i]);
      }
      return acc;
    };
    string grp_type = "NULL";
    for (auto& ss : st.op_type) {
      if (ss == "emit sel_name") {
        Rec r;
        r.col_val = st.op_value[iv++];
        r.grp_type = grp_type;
        bool any = false;
        if (!exe_nums.empty()) {
          r.col_type = 0;
          r.num = pop(exe_nums);
          r.prec = pop(exe_prec);
          recs.push_back(r);
          any = true;
        }
        if (!exe_value.empty() && exe_value.back() != "") {
          Rec q = r;
          q.col_type = 1;
          q.value = pop(exe_value);
          q.prec = av->info[q.value].dz;
          recs.push_back(q);
          any = true;
        }
        if (!exe_vectors.empty()) {
          Rec q = r;
          q.col_type = 2;
          q.vec = pop(exe_vectors);
          q.prec = pop(exe_prec);
          pop(exe_value);
          recs.push_back(q);
          any = true;
        }
        (void)any;
        continue;
      }
      grp_type = "NULL";
      bool is_agg = ss == "COUNT" || ss == "SUM" || ss == "AVG" || ss == "MIN" || ss == "MAX";
      if (ss == "DISTINCT" || ss == "YEAR" || ss == "MONTH" || ss == "DAY" || ss == "CAST")
        throw Error(ss + " is not supported by the oracle");
      if (is_agg) {
        if (!grp_count) one_line = true;
        if (ss == "COUNT") {
          grp_type = "COUNT";
          pop(exe_type);
          pop(exe_value);
          VecP v;
          if (grp_count > 1) {
            Vec ones(n, 1);
            v = std::make_shared<Vec>(segreduce(ones, 0));
          } else {
            v = std::make_shared<Vec>(1, (i64)n);
          }
          exe_vectors.push_back(v);
          exe_type.push_back("NAME");
          exe_prec.push_back(0);
          exe_value.push_back("");
        } else {
          int kind = ss == "MIN" ? 1 : (ss == "MAX" ? 2 : 0);
          grp_type = ss;
          pop(exe_type);
          string s1v = pop(exe_value);
          VecP v;
          if (!is_col(s1v)) {
            VecP s3 = pop(exe_vectors);
            if (grp_count > 1) v = std::make_shared<Vec>(segreduce(*s3, kind));
            else v = std::make_shared<Vec>(1, reduce(*s3, kind));
            if (ss != "SUM") exe_prec.push_back(pop(exe_prec));
          } else {
            const Vec& col = a.c.at(s1v);
            if (grp_count > 1) v = std::make_shared<Vec>(segreduce(col, kind));
            else if (ss == "SUM" && !one_line) v = std::make_shared<Vec>(n, reduce(col, kind));
            else v = std::make_shared<Vec>(1, reduce(col, kind));
            exe_prec.push_back(av->info[s1v].dz);
          }
          exe_vectors.push_back(v);
          exe_type.push_back("NAME");
          exe_value.push_back("");
        }
        continue;
      }
      if (ss == "NAME" || ss == "NUMBER") {
        exe_type.push_back(ss);
        if (ss == "NUMBER") {
          exe_nums.push_back(st.op_nums[in]);
          exe_prec.push_back(st.op_nums_precision[ip++]);
          in++;
        } else {
          exe_value.push_back(st.op_value[iv++]);
        }
        continue;
      }
      if (ss == "MUL" || ss == "ADD" || ss == "DIV" || ss == "MINUS") {
        string s1 = pop(exe_type), s2 = pop(exe_type);
        if (s1 == "NUMBER" && s2 == "NUMBER") {
          i64 n1 = pop(exe_nums), n2 = pop(exe_nums);
          u32 p1 = pop(exe_prec), p2 = pop(exe_prec);
          u32 pres = precision_func(p1, p2, ss);
          exe_prec.push_back(pres);
          if (p1) n1 = wmul(n1, pow10u(p1));
          if (p2) n2 = wmul(n2, pow10u(p2));
          i64 res = arith(ss, n1, n2);  // the top operand is the left one here (select.cu:727-736)
          exe_vectors.push_back(std::make_shared<Vec>(n, res));
          exe_type.push_back("NAME");
          exe_value.push_back("");
        } else if (s1 == "NAME" && s2 == "NUMBER") {
          string s1v = pop(exe_value);
          i64 n1 = pop(exe_nums);
          u32 p1 = pop(exe_prec);
          u32 p2 = get_decimals(s1v);
          VecP t = get_vec(s1v);
          u32 pres = precision_func(p2, p1, ss);
          exe_prec.push_back(pres);
          exe_type.push_back("NAME");
          exe_value.push_back("");
          exe_vectors.push_back(op_const(*t, n1, ss, true, p2, p1));
        } else if (s1 == "NUMBER" && s2 == "NAME") {
          i64 n1 = pop(exe_nums);
          string s1v = pop(exe_value);
          u32 p1 = pop(exe_prec);
          u32 p2 = get_decimals(s1v);
          VecP t = get_vec(s1v);
          u32 pres = precision_func(p2, p1, ss);
          exe_prec.push_back(pres);
          exe_type.push_back("NAME");
          exe_value.push_back("");
          exe_vectors.push_back(op_const(*t, n1, ss, false, p2, p1));
        } else if (s1 == "NAME" && s2 == "NAME") {
          string s1v = pop(exe_value), s2v = pop(exe_value);
          VecP t1 = get_vec(s1v);
          VecP t = get_vec(s2v);
          u32 p1 = get_decimals(s1v), p2 = get_decimals(s2v);
          u32 pres = precision_func(p1, p2, ss);
          exe_prec.push_back(pres);
          exe_type.push_back("NAME");
          exe_value.push_back("");
          exe_vectors.push_back(op_vec(*t, *t1, ss, false, p2, p1));
        } else {
          throw Error("unsupported arithmetic operands in a select list");
        }
        continue;
      }
      // other tokens (trailing GROUP BY names are NAME and handled above)
      throw Error("token " + ss + " is not supported by the oracle");
    }
    // Build output columns in stack order, then the select-list order is restored by
    // the caller (select.cu:836-952, operators.cu:1985-1986).
    b.clear();
    for (auto it = recs.rbegin(); it != recs.rend(); ++it) {
      OutCol oc;
      oc.name = it->col_val;
      const string& g = it->grp_type;
      oc.grp_type = g == "COUNT" ? 0 : g == "AVG" ? 1 : g == "SUM" ? 2 : g == "MIN" ? 4 : g == "MAX" ? 5 : 3;
      size_t rows = grp_count ? res_size : n;
      if (it->col_type == 0) {
        if (grp_count) oc.v.assign(res_size, (i64)(int)it->num);
        else oc.v.assign(n, (i64)(int)it->num);
        oc.dz = it->prec;
      } else if (it->col_type == 1) {
        const Vec& col = a.c.at(it->value);
        if (grp_count) {
          oc.v.resize(res_size);
          for (size_t gi = 0; gi < res_size; gi++) {
            if (grp[gi] >= col.size()) throw Error("group offset outside the segment");
            oc.v[gi] = col[grp[gi]];
          }
        } else {
          oc.v = col;
        }
        oc.dz = it->prec;
        if (av->info[it->value].type == 2 || !av->info[it->value].string_map.empty())
          oc.string_map = av->info[it->value].string_map;
      } else {
        const Vec& vv = *it->vec;
        size_t take = grp_count ? res_size : (one_line ? 1 : n);
        if (vv.size() < take) throw Error("expression result shorter than the output");
        oc.v.assign(vv.begin(), vv.begin() + take);
        oc.dz = it->prec;
      }
      (void)rows;
      b.push_back(std::move(oc));
    }
    if (!grp_count) b_rows = one_line ? 1 : n;
    else b_rows = res_size;
    return one_line;
  }

  // emit_select (operators.cu:1801-2084)
  void emit_select(alk::Statement& st) {
    Var* a = var(st.f);
    int grp_cnt = st.grp_cnt;
    vector<string> group_cols(st.op_value.end() - grp_cnt, st.op_value.end());
    // aliases of group columns (operators.cu:1871-1894)
    map<string, string> aliases;
    {
      size_t i = 0;
      auto& ov = st.op_value;
      while (i < ov.size()) {
        if (a->has(ov[i])) {
          string tt = ov[i];
          i++;
          if (i < ov.size() && !a->has(ov[i]) && !aliases.count(tt)) aliases[tt] = ov[i];
        }
        if (i < ov.size()) i++;
      }
    }
    set<string> field_set;
    for (auto& v : st.op_value)
      if (a->has(v)) field_set.insert(v);
    vector<string> fields(field_set.begin(), field_set.end());
    size_t cycle_count = cycles(a);
    if (!a->filtered && a->segCount <= 1) {  // setSegments (cm.cu:3565-3580)
      size_t tot = 0;
      for (auto& fl : fields) tot += a->info[fl].type != 2 ? 8 : a->info[fl].char_size;
      if (a->mRecCount * tot > kFreeMem / 3) throw Error("re-segmentation is not supported by the oracle");
    }
    auto c = std::make_unique<Var>();
    c->name = st.s;
    bool c_set = false, one_liner = false, first_reversed = true;
    vector<string> c_names;
    vector<uint64_t> h_merge;
    for (size_t i = 0; i < cycle_count; i++) {
      Seg sg = fetch(a, fields, (unsigned)i);
      if (!sg.n) continue;
      vector<u32> grp;
      size_t grp_count = 0;
      if (grp_cnt) {
        bool not_srt_and_eq = false;
        for (auto& g : group_cols)
          if (!min_max_eq_[g]) not_srt_and_eq = true;
        if (not_srt_and_eq) {
          // order_inplace: stable sort by the group columns, first column most significant
          vector<u32> perm(sg.n);
          std::iota(perm.begin(), perm.end(), 0);
          vector<const Vec*> keys;
          for (auto& g : group_cols) keys.push_back(&sg.c.at(g));
          __gnu_parallel::stable_sort(perm.begin(), perm.end(), [&](u32 x, u32 y) {
            for (auto* k : keys) {
              if ((*k)[x] < (*k)[y]) return true;
              if ((*k)[x] > (*k)[y]) return false;
            }
            return false;
          });
          for (auto& kv : sg.c) {
            Vec p(sg.n);
            for (size_t r = 0; r < sg.n; r++) p[r] = kv.second[perm[r]];
            kv.second.swap(p);
          }
          // CudaSet::GroupBy head flags (cm.cu:910-956)
          grp.push_back(0);
          for (size_t r = 0; r + 1 < sg.n; r++) {
            bool diff = false;
            for (auto* k : keys)
              if ((*k)[r] != (*k)[r + 1]) diff = true;
            if (diff) grp.push_back((u32)(r + 1));
          }
          grp_count = grp.size();
        } else {
          grp = {1};
          grp_count = 1;
        }
      }
      vector<OutCol> b;
      size_t b_rows = 0;
      one_liner = select_seg(st, a, sg, grp, grp_count, b, b_rows);
      if (i == 0) first_reversed = false;
      if (!first_reversed) std::reverse(b.begin(), b.end());
      if (!c_set && b_rows > 0) {  // create_c (merge.cu:57-90)
        for (auto& oc : b) {
          c->columnNames.push_back(oc.name);
          ColInfo ci;
          ci.dz = oc.dz;
          ci.string_map = oc.string_map;
          c->info[oc.name] = ci;
          c->grp_type[oc.name] = oc.grp_type;
          c->h[oc.name];
        }
        c_set = true;
      }
      if (grp_cnt && cycle_count > 1 && b_rows > 0) {
        add(c.get(), b, b_rows, group_cols, aliases, h_merge);
      } else {
        for (auto& oc : b) {
          Vec& dst = c->h[oc.name];
          dst.insert(dst.end(), oc.v.begin(), oc.v.begin() + std::min(b_rows, oc.v.size()));
        }
        c->mRecCount += b_rows;
      }
    }
    if (!c_set) {
      vars_[st.s] = std::move(c);
      return;
    }
    if (grp_cnt) count_avg(c.get(), h_merge);
    else if (one_liner) count_simple(c.get());
    c->segCount = 1;
    c->maxRecs = c->hostRecCount = c->mRecCount;
    c->not_compressed = true;
    vars_[st.s] = std::move(c);
  }

  // add (merge.cu:92-268): per-segment groups hashed on the group key tuple, sorted by
  // hash and merged into c in hash order.
  void add(Var* c, vector<OutCol>& b, size_t b_rows, const vector<string>& group_cols,
           map<string, string>& aliases, vector<uint64_t>& h_merge) {
    vector<string> opv;
    map<string, size_t> bidx;
    for (size_t k = 0; k < b.size(); k++) bidx[b[k].name] = k;
    for (auto& g : group_cols) {
      string al = aliases.count(g) ? aliases[g] : "";
      opv.push_back(bidx.count(al) ? al : g);
    }
    for (auto& o : opv)
      if (!bidx.count(o)) throw Error("group column " + o + " is not in the select list");
    size_t K = opv.size();
    vector<uint64_t> hashes(b_rows);
    for (size_t r = 0; r < b_rows; r++) {
      vector<i64> tup(K);
      for (size_t z = 0; z < K; z++) tup[z] = b[bidx[opv[z]]].v[r];
      hashes[r] = murmur(tup.data(), (int)(8 * K), alk::kHashSeed);
    }
    vector<u32> v(b_rows);
    std::iota(v.begin(), v.end(), 0);
    std::stable_sort(v.begin(), v.end(), [&](u32 x, u32 y) { return hashes[x] < hashes[y]; });
    vector<uint64_t> hh(b_rows);
    for (size_t r = 0; r < b_rows; r++) hh[r] = hashes[v[r]];
    // stable merge of (h_merge, c) with (hh, b): c's rows first on equal hashes
    size_t m = h_merge.size();
    vector<size_t> from_c, from_b;
    vector<uint64_t> merged;
    merged.reserve(m + b_rows);
    vector<std::pair<int, size_t>> order;
    size_t i = 0, j = 0;
    while (i < m || j < b_rows) {
      if (j >= b_rows || (i < m && !(hh[j] < h_merge[i]))) {
        order.push_back({0, i});
        merged.push_back(h_merge[i++]);
      } else {
        order.push_back({1, j});
        merged.push_back(hh[j++]);
      }
    }
    for (size_t k = 0; k < b.size(); k++) {
      const string& cn = c->columnNames[k];
      Vec& cv = c->h[cn];
      Vec out(order.size());
      for (size_t q = 0; q < order.size(); q++)
        out[q] = order[q].first == 0 ? cv[order[q].second] : b[k].v[v[order[q].second]];
      cv.swap(out);
    }
    h_merge.swap(merged);
    c->mRecCount = h_merge.size();
  }

  // count_avg (merge.cu:314-496)
  void count_avg(Var* c, vector<uint64_t>& h_merge) {
    string countstr;
    for (auto& n : c->columnNames)
      if (c->grp_type[n] == 0) {
        countstr = n;
        break;
      }
    if (c->mRecCount == 0) return;
    if (!h_merge.empty()) {
      vector<size_t> starts;
      for (size_t i = 0; i < h_merge.size(); i++)
        if (i == 0 ? h_merge[0] != 0 : h_merge[i] != h_merge[i - 1]) starts.push_back(i);
      size_t res_count = starts.size();
      auto run_end = [&](size_t g) { return g + 1 < starts.size() ? starts[g + 1] : h_merge.size(); };
      for (auto& n : c->columnNames) {
        Vec& col = c->h[n];
        int gt = c->grp_type[n];
        Vec out(res_count);
        if (gt <= 2) {
          // overflow probe in double (merge.cu:351-371)
          double max_overflow = 0;
          for (size_t g = 0; g < res_count; g++) {
            double s = 0;
            for (size_t i = starts[g]; i < run_end(g); i++) s += (double)col[i];
            if (s > 9223372036854775807.0 && s - 9223372036854775807.0 > max_overflow) max_overflow = s;
          }
          if (max_overflow) {
            unsigned pw = (unsigned)std::ceil(std::log10(max_overflow / 9223372036854775807.0));
            i64 dv = (i64)std::pow(10.0, (double)pw);
            for (auto& x : col) x = idiv(x, dv);
            c->info[n].dz -= pw;
          }
          for (size_t g = 0; g < res_count; g++) {
            i64 s = 0;
            for (size_t i = starts[g]; i < run_end(g); i++) s = wadd(s, col[i]);
            out[g] = s;
          }
        } else {
          for (size_t g = 0; g < res_count; g++) {
            i64 acc = col[starts[g]];
            for (size_t i = starts[g]; i < run_end(g); i++)
              acc = gt == 4 ? std::min(acc, col[i]) : std::max(acc, col[i]);
            out[g] = acc;
          }
        }
        col.swap(out);
      }
      c->mRecCount = res_count;
    }
    for (auto& n : c->columnNames) {
      if (c->grp_type[n] != 1) continue;
      if (countstr.empty()) throw Error("AVG needs a COUNT column in the same select");
      Vec& col = c->h[n];
      const Vec& cnt = c->h[countstr];
      if (c->info[n].dz <= 2) {
        for (size_t r = 0; r < c->mRecCount; r++) col[r] = idiv(wmul(col[r], 100), cnt[r]);
        c->info[n].dz += 2;
      } else {
        for (size_t r = 0; r < c->mRecCount; r++) col[r] = idiv(col[r], cnt[r]);
      }
      c->grp_type[n] = 3;
    }
  }

  // count_simple (merge.cu:271-311)
  void count_simple(Var* c) {
    i64 count = 0;
    bool have = false;
    for (auto& n : c->columnNames)
      if (c->grp_type[n] == 0) {
        Vec& col = c->h[n];
        count = std::accumulate(col.begin(), col.begin() + c->mRecCount, (i64)0, wadd);
        col[0] = count;
        have = true;
      }
    if (c->mRecCount != 0) {
      for (auto& n : c->columnNames) {
        Vec& col = c->h[n];
        int gt = c->grp_type[n];
        if (gt == 1) {
          if (!have) throw Error("AVG needs a COUNT column in the same select");
          i64 s = std::accumulate(col.begin(), col.begin() + c->mRecCount, (i64)0, wadd);
          col[0] = idiv(s, count);
        } else if (gt == 2) {
          col[0] = std::accumulate(col.begin(), col.begin() + c->mRecCount, (i64)0, wadd);
        }
      }
    }
    c->mRecCount = 1;
    for (auto& n : c->columnNames) c->h[n].resize(1);
  }

  // All rows of a variable, every segment (load_queue, cm.cu:3482-3525).
  Seg load_all(Var* a, const vector<string>& fields) {
    Seg out;
    size_t cyc = cycles(a);
    for (size_t i = 0; i < cyc; i++) {
      Seg s = fetch(a, fields, (unsigned)i);
      for (auto& fl : fields) {
        if (!a->has(fl)) continue;
        Vec& d = out.c[fl];
        auto it = s.c.find(fl);
        if (it != s.c.end()) d.insert(d.end(), it->second.begin(), it->second.end());
      }
      out.n += s.n;
    }
    return out;
  }

  // emit_join (operators.cu:797-924) and emit_multijoin (operators.cu:940-1582), inner joins.
  void emit_join(alk::Statement& st) {
    if (check_star_join(st)) {  // emit_join's star branch (operators.cu:828-832)
      star_join(st);
      return;
    }
    vector<string> op_m = st.op_value;
    if (st.join_tab_cnt > 1) {
      vector<string> oj = st.op_join;
      size_t oi = 0;
      for (unsigned i = 1; i <= st.join_tab_cnt; i++) {
        string tab_name = i == st.join_tab_cnt ? st.s : st.s + std::to_string(i);
        string j, j2;
        if (i == 1) {
          j2 = oj[oi++];
          j = oj[oi++];
        } else {
          j = oi < oj.size() ? oj[oi++] : st.f;
          j2 = st.s + std::to_string(i - 1);
        }
        multijoin(st, tab_name, j, j2, i);
      }
    } else {
      multijoin(st, st.s, st.f, st.op_join[0], 1);
    }
    // rename selected columns to their aliases (operators.cu:862-906)
    Var* r = var(st.s);
    for (unsigned k = 0; k < st.sel_count; k++) {
      const string& from = op_m[2 * k];
      const string& to = op_m[2 * k + 1];
      if (from == to) continue;
      auto it = std::find(r->columnNames.begin(), r->columnNames.end(), from);
      if (it == r->columnNames.end()) continue;
      *it = to;
      r->h[to] = std::move(r->h[from]);
      r->h.erase(from);
      // the rename carries type and the decimal flag but not decimal_zeroes
      // (operators.cu:877-906): an aliased decimal column of a join result keeps the
      // alias's previous scale, 0 for a new name, for printing and for arithmetic
      // (get_decimals, cm.cu:4371)
      u32 dz_to = r->info.count(to) ? r->info[to].dz : 0;
      r->info[to] = r->info[from];
      r->info[to].dz = dz_to;
    }
  }

  void multijoin(alk::Statement& st, const string& s, const string& j1, const string& j2, unsigned tab) {
    Var* left = var(j1);
    Var* right = var(j2);
    vector<string> op_sel, op_g;
    size_t k = 0;
    for (unsigned i = 0; i < st.sel_count; i++, k += 2) op_sel.push_back(st.op_value[k]);
    op_g.assign(st.op_value.begin() + k, st.op_value.end());
    vector<string> op_sel_s = op_sel;
    size_t gi = 0;
    for (unsigned z = 0; z < st.join_tab_cnt - tab; z++) {
      unsigned jac = st.join_and_cnt.count(z) ? st.join_and_cnt.at(z) : 0;
      for (unsigned j = 0; j < jac * 2 + 2; j++) op_sel_s.push_back(op_g[gi++]);
    }
    string f1 = op_g[gi], f2 = op_g[gi + 1];
    gi += 2;
    unsigned jac = st.join_and_cnt.count(st.join_tab_cnt - tab) ? st.join_and_cnt.at(st.join_tab_cnt - tab) : 0;
    char kind = st.join_type[tab - 1];
    if (kind != 'I' && kind != '1' && kind != '2' && kind != '3' && kind != '4')
      throw Error("outer joins are not supported by the oracle");
    if ((jac || kind != 'I') && st.join_tab_cnt != 1)
      throw Error("multi-column / semi / anti joins in a join chain are not supported by the oracle");
    // AND-ed pairs (operators.cu:1288-1348): each of the jac checks reads the first extra
    // pair (the queue is copied afresh) and the m-th queued equality type
    string f3, f4;
    if (jac) {
      f3 = op_g[gi];
      f4 = op_g[gi + 1];
    }
    const bool left_rows = kind == '1' || kind == '3', right_rows = kind == '2' || kind == '4';
    // result layout: CudaSet(right, left, op_sel_s) (cm.cu:3078-3160)
    auto c = std::make_unique<Var>();
    c->name = s;
    for (auto& n : op_sel_s) {
      if (std::find(c->columnNames.begin(), c->columnNames.end(), n) != c->columnNames.end()) continue;
      if (right->has(n)) c->info[n] = right->info[n];
      else if (left->has(n)) c->info[n] = left->info[n];
      else continue;
      c->columnNames.push_back(n);
      c->h[n];
    }
    string colname1, colname2;
    if (left->has(f1)) {
      colname1 = f1;
      if (!right->has(f2)) throw Error("Couldn't find column " + f2);
      colname2 = f2;
    } else if (right->has(f1)) {
      colname2 = f1;
      string tmp = f1;
      f1 = f2;
      if (!left->has(f2)) throw Error("Couldn't find column " + f2);
      colname1 = f2;
      f2 = tmp;
    } else {
      throw Error("Couldn't find column " + f1);
    }
    // right side: every output column it holds plus the key, all segments, then a stable
    // sort on the key (order_inplace, operators.cu:1117-1157)
    vector<string> rfields;
    for (auto& n : op_sel)
      if (right->has(n)) rfields.push_back(n);
    for (auto& n : op_sel_s)
      if (right->has(n) && std::find(rfields.begin(), rfields.end(), n) == rfields.end()) rfields.push_back(n);
    if (std::find(rfields.begin(), rfields.end(), f2) == rfields.end()) rfields.push_back(f2);
    if (jac && std::find(rfields.begin(), rfields.end(), f4) == rfields.end()) rfields.push_back(f4);
    for (auto& n : c->columnNames) {
      if (left_rows && !left->has(n)) throw Error("right-side column in a left semi / anti join");
      if (right_rows && !right->has(n)) throw Error("left-side column in a right semi / anti join");
    }
    Seg R = load_all(right, rfields);
    size_t cnt_r = R.n;
    const Vec& rk0 = R.c.at(colname2);
    vector<u32> rperm(cnt_r);
    std::iota(rperm.begin(), rperm.end(), 0);
    if (!std::is_sorted(rk0.begin(), rk0.end()))
      __gnu_parallel::stable_sort(rperm.begin(), rperm.end(), [&](u32 x, u32 y) { return rk0[x] < rk0[y]; });
    map<string, Vec> RS;
    for (auto& kv : R.c) {
      Vec p(cnt_r);
      for (size_t r = 0; r < cnt_r; r++) p[r] = kv.second[rperm[r]];
      RS[kv.first] = std::move(p);
    }
    const Vec& rk = RS.at(colname2);
    vector<string> lfields;
    for (auto& n : op_sel_s)
      if (left->has(n) && std::find(lfields.begin(), lfields.end(), n) == lfields.end()) lfields.push_back(n);
    if (std::find(lfields.begin(), lfields.end(), colname1) == lfields.end()) lfields.push_back(colname1);
    if (jac && std::find(lfields.begin(), lfields.end(), f3) == lfields.end()) lfields.push_back(f3);
    std::set<u32> ranj;  // right semi / anti: right rows matched over all left segments
    size_t cyc = cycles(left);
    for (size_t i = 0; i < cyc && cnt_r; i++) {
      Seg L = fetch(left, lfields, (unsigned)i);
      size_t cnt_l = L.n;
      if (!cnt_l) continue;
      const Vec& lk = L.c.at(colname1);
      vector<u32> vl(cnt_l);
      std::iota(vl.begin(), vl.end(), 0);
      __gnu_parallel::stable_sort(vl.begin(), vl.end(), [&](u32 x, u32 y) { return lk[x] < lk[y]; });
      if (lk[vl[0]] > rk[cnt_r - 1] || lk[vl[cnt_l - 1]] < rk[0]) continue;
      // merge-join pairs ordered by left sorted position, then right position
      vector<u32> pl, pr;
      size_t rj = 0;
      for (size_t li = 0; li < cnt_l; li++) {
        i64 key = lk[vl[li]];
        while (rj < cnt_r && rk[rj] < key) rj++;
        for (size_t q = rj; q < cnt_r && rk[q] == key; q++) {
          pl.push_back(vl[li]);
          pr.push_back((u32)q);
        }
      }
      for (unsigned m = 0; m < jac; m++) {  // stable: the pairs keep their order
        const bool neq = m < st.join_eq_type.size() && st.join_eq_type[m] == 'N';
        const Vec& a = L.c.at(f3);
        const Vec& b = RS.at(f4);
        vector<u32> ql, qr;
        for (size_t q = 0; q < pl.size(); q++)
          if ((a[pl[q]] == b[pr[q]]) != neq) {
            ql.push_back(pl[q]);
            qr.push_back(pr[q]);
          }
        pl.swap(ql);
        pr.swap(qr);
      }
      if (right_rows) {  // accumulated; output after every left segment (operators.cu:1376-1399)
        ranj.insert(pr.begin(), pr.end());
        continue;
      }
      if (left_rows) {  // left semi: matched left rows once; anti: the others; left order
        vector<char> hit(cnt_l, 0);
        for (u32 x : pl) hit[x] = 1;
        pl.clear();
        for (u32 r = 0; r < cnt_l; r++)
          if (hit[r] == (kind == '1')) pl.push_back(r);
      }
      for (auto& n : c->columnNames) {
        Vec& dst = c->h[n];
        if (left->has(n)) {
          const Vec& src = L.c.at(n);
          for (size_t q = 0; q < pl.size(); q++) dst.push_back(src[pl[q]]);
        } else {
          const Vec& src = RS.at(n);
          for (size_t q = 0; q < pr.size(); q++) dst.push_back(src[pr[q]]);
        }
      }
      c->mRecCount += pl.size();
    }
    if (right_rows) {  // right rows in the sorted right side's order
      vector<u32> rows;
      for (u32 r = 0; r < cnt_r; r++)
        if (ranj.count(r) == (size_t)(kind == '2')) rows.push_back(r);
      for (auto& n : c->columnNames) {
        Vec& dst = c->h[n];
        const Vec& src = RS.at(n);
        for (u32 r : rows) dst.push_back(src[r]);
      }
      c->mRecCount = rows.size();
    }
    c->hostRecCount = c->maxRecs = c->mRecCount;
    c->segCount = 1;
    c->not_compressed = true;
    vars_[s] = std::move(c);
  }

  // emit_order (operators.cu:1641-1798): stable sorts from the last key to the first.
  void emit_order(alk::Statement& st) {
    Var* a = var(st.f);
    vector<string> keys, dirs;
    size_t iv = 0;
    for (auto& t : st.op_type) {
      if (t == "NAME") {
        keys.push_back(st.op_value[iv++]);
        dirs.push_back("ASC");
      } else {
        keys.push_back(t);
        dirs.push_back(st.op_value[iv++]);
      }
      if (!a->has(keys.back())) throw Error("Couldn't find name " + keys.back());
    }
    Seg s = load_all(a, a->columnNames);
    vector<u32> perm(s.n);
    std::iota(perm.begin(), perm.end(), 0);
    for (size_t k = keys.size(); k-- > 0;) {
      bool desc = dirs[k] == "DESC";
      if (a->info[keys[k]].type == 2 || !a->info[keys[k]].string_map.empty()) {
        // the rows' strings read from the dictionary by code and sorted stably as unsigned
        // bytes over the column width (update_char_permutation cm.cu:4218, str_sort
        // strings_sort_device.cu:125)
        const string& sm = a->info[keys[k]].string_map;
        const auto& dict = file(sm);
        auto pos = sm.find_last_of('/');
        string base = pos == string::npos ? sm : sm.substr(pos + 1);
        auto dot = base.find('.');
        const u32 w = dd_[base.substr(0, dot)][base.substr(dot + 1)].col_length;
        const Vec& code = s.c.at(keys[k]);
        auto str = [&](u32 r) { return dict.data() + (size_t)code[r] * w; };
        __gnu_parallel::stable_sort(perm.begin(), perm.end(), [&](u32 x, u32 y) {
          const int c = std::memcmp(str(x), str(y), w);
          return desc ? c > 0 : c < 0;
        });
        continue;
      }
      const Vec& key = s.c.at(keys[k]);
      __gnu_parallel::stable_sort(perm.begin(), perm.end(), [&](u32 x, u32 y) {
        return desc ? key[x] > key[y] : key[x] < key[y];
      });
    }
    auto b = std::make_unique<Var>();
    b->name = st.s;
    b->columnNames = a->columnNames;
    b->info = a->info;
    for (auto& n : a->columnNames) {
      Vec& src = s.c[n];
      Vec p(s.n);
      for (size_t r = 0; r < s.n; r++) p[r] = src[perm[r]];
      b->h[n] = std::move(p);
    }
    b->mRecCount = b->hostRecCount = b->maxRecs = s.n;
    b->segCount = 1;
    b->not_compressed = true;
    vars_[st.s] = std::move(b);
  }

  // emit_store / CudaSet::Store text output (operators.cu:2410-2444, cm.cu:1479-1560)
  void emit_store(alk::Statement& st) {
    Var* a = var(st.s);
    size_t limit = st.op_nums.empty() ? 0 : (size_t)st.op_nums[0];
    Seg s;
    if (a->not_compressed && !a->filtered) {
      s.n = a->mRecCount;
      for (auto& n : a->columnNames) s.c[n] = a->h[n];
    } else {
      s = load_all(a, a->columnNames);
    }
    size_t mCount = (limit != 0 && limit < s.n) ? limit : s.n;
    string path = st.f;
    if (path.empty() || path[0] != '/') path = dir_ + "/" + path;
    FILE* fp = std::fopen(path.c_str(), "w");
    if (!fp) throw Error("Could not open file " + path);
    map<string, vector<char>> dicts;
    map<string, u32> lens;
    for (auto& n : a->columnNames) {
      const string& sm = a->info[n].string_map;
      if (sm.empty() || dicts.count(sm)) continue;
      string e;
      vector<uint8_t> raw;
      if (!alk::read_file(sm, raw, e)) throw Error(e);
      dicts[sm] = vector<char>(raw.begin(), raw.end());
      auto pos = sm.find_last_of('/');
      string base = pos == string::npos ? sm : sm.substr(pos + 1);
      auto dot = base.find('.');
      lens[sm] = dd_[base.substr(0, dot)][base.substr(dot + 1)].col_length;
    }
    for (size_t i = 0; i < mCount; i++) {
      for (auto& n : a->columnNames) {
        const ColInfo& ci = a->info[n];
        i64 v = s.c[n][i];
        if (ci.string_map.empty()) {
          if (ci.dz) {
            string str = std::to_string(v);
            while (str.size() <= ci.dz) str = '0' + str;
            str.insert(str.size() - ci.dz, ".");
            std::fputs(str.c_str(), fp);
          } else {
            std::fprintf(fp, "%lld", (long long)v);
          }
        } else {
          u32 len = lens[ci.string_map];
          const vector<char>& d = dicts[ci.string_map];
          size_t off = (size_t)v * len;
          string val = off + len <= d.size() ? string(&d[off], len) : string();
          std::fprintf(fp, "%.*s", (int)len, val.c_str());
        }
        std::fputs(st.sep.c_str(), fp);
      }
      if (i != mCount - 1) std::fputs("\n", fp);
    }
    std::fclose(fp);
  }
};

}  // namespace orc

static uint64_t g_rows_scanned = 0;

extern "C" {
int oracle_execute(const char* dir, const char* script, int threads, char* err, int err_len) {
  try {
    orc::Engine e(dir, threads);
    e.run(script);
    g_rows_scanned = e.rows_scanned;
  } catch (const std::exception& ex) {
    if (err && err_len > 0) std::snprintf(err, (size_t)err_len, "%s", ex.what());
    return 1;
  }
  return 0;
}
int oracle_like(const char* entry, uint32_t width, const char* pattern) {
  return orc::like_match(entry, width, pattern) ? 1 : 0;
}

int64_t oracle_decode_segment(const uint8_t* image, size_t len, int64_t* out, size_t out_cap) {
  orc::Decoded d;
  if (!orc::decode_image(image, len, d)) return -1;
  if (d.v.size() > out_cap) return -1;
  std::memcpy(out, d.v.data(), d.v.size() * 8);
  return (int64_t)d.v.size();
}
uint64_t oracle_murmur64a(const void* key, int len, uint32_t seed) { return orc::murmur(key, len, seed); }
uint64_t oracle_rows_scanned(void) { return g_rows_scanned; }
}
