// Seeded synthetic tables in the reference's segment format. They stand in for
// the TPC-H-shaped inputs of the benchmark workloads (no dbgen data or query text
// is used): a lineitem table for the single-table filter + group-by workload, and
// customer / orders / lineitem for the three-way filter -> join -> group-by
// pipeline. Column types follow the reference's load scripts: int, decimal(...,2)
// money, int yyyymmdd dates and dictionary-encoded char columns.
#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "format.h"

namespace alk {
namespace {

struct Rng {  // splitmix64
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
  }
  int64_t uniform(int64_t lo, int64_t hi) {  // inclusive
    uint64_t span = (uint64_t)(hi - lo) + 1;
    return lo + (int64_t)(next() % span);
  }
};

uint64_t mix(uint64_t seed, uint64_t stream) { return seed * 0x9e3779b97f4a7c15ULL + stream * 0xd1b54a32d192ed03ULL + 1; }

// days since 1970-01-01 <-> yyyymmdd (proleptic Gregorian civil calendar)
int64_t days_from_civil(int64_t y, int64_t m, int64_t d) {
  y -= m <= 2;
  int64_t era = (y >= 0 ? y : y - 399) / 400;
  int64_t yoe = y - era * 400;
  int64_t doy = (153 * (m + (m > 2 ? -3 : 9)) + 2) / 5 + d - 1;
  int64_t doe = yoe * 365 + yoe / 4 - yoe / 100 + doy;
  return era * 146097 + doe - 719468;
}
int64_t yyyymmdd(int64_t z) {
  z += 719468;
  int64_t era = (z >= 0 ? z : z - 146096) / 146097;
  int64_t doe = z - era * 146097;
  int64_t yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
  int64_t y = yoe + era * 400;
  int64_t doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
  int64_t mp = (5 * doy + 2) / 153;
  int64_t d = doy - (153 * mp + 2) / 5 + 1;
  int64_t m = mp + (mp < 10 ? 3 : -9);
  y += m <= 2;
  return y * 10000 + m * 100 + d;
}

bool flush(TableWriter& w, const std::vector<std::vector<int64_t>>& ints,
           const std::vector<std::vector<char>>& chars, size_t ncols, uint64_t begin, uint64_t end,
           const std::vector<uint32_t>& widths, std::string& err) {
  std::vector<const int64_t*> ip(ncols, nullptr);
  std::vector<const char*> cp(ncols, nullptr);
  for (size_t c = 0; c < ncols; c++) {
    if (widths[c]) cp[c] = chars[c].data() + begin * widths[c];
    else ip[c] = ints[c].data() + begin;
  }
  return w.write_segment(ip, cp, (uint32_t)(end - begin), err);
}

bool write_table(const std::string& dir, const std::string& name, const std::vector<ColumnSpec>& spec,
                 const std::vector<std::vector<int64_t>>& ints, const std::vector<std::vector<char>>& chars,
                 uint64_t rows, uint32_t seg_rows, DataDict& dd, std::string& err) {
  TableWriter w(dir, name, spec);
  std::vector<uint32_t> widths;
  for (auto& c : spec) widths.push_back(c.kind == 2 ? c.width : 0);
  if (seg_rows == 0) seg_rows = (uint32_t)rows;
  for (uint64_t b = 0; b < rows; b += seg_rows) {
    uint64_t e = std::min<uint64_t>(rows, b + seg_rows);
    if (!flush(w, ints, chars, spec.size(), b, e, widths, err)) return false;
  }
  return w.finish(dd, err);
}

void put_str(std::vector<char>& buf, uint64_t row, uint32_t width, const char* s) {
  size_t L = std::strlen(s);
  std::memcpy(&buf[row * width], s, std::min<size_t>(L, width));
}

const char* kSegments[5] = {"AUTOMOBILE", "BUILDING", "FURNITURE", "HOUSEHOLD", "MACHINERY"};

}  // namespace

// Single-table workload: lineitem with orderkey (1-7 rows per key), quantity U[1,50],
// extendedprice cents U[90000,10500000], discount U[0,10] hundredths, shipdate uniform
// yyyymmdd over 1992-01-02..1998-12-01, returnflag in {A,N,R}, linestatus in {F,O}.
bool gen_lineitem_flat(const std::string& dir, uint64_t rows, uint32_t seg_rows, uint64_t seed,
                       bool delta, std::string& err) {
  std::vector<ColumnSpec> spec = {
      {"l_orderkey", 0, 0, 0, delta}, {"l_quantity", 0, 0, 0, delta},
      {"l_extendedprice", 1, 2, 0, delta}, {"l_discount", 1, 2, 0, delta},
      {"l_shipdate", 0, 0, 0, delta}, {"l_returnflag", 2, 0, 1, false},
      {"l_linestatus", 2, 0, 1, false}};
  std::vector<std::vector<int64_t>> ints(spec.size());
  std::vector<std::vector<char>> chars(spec.size());
  for (int c = 0; c < 5; c++) ints[c].resize(rows);
  chars[5].assign(rows, 0);
  chars[6].assign(rows, 0);
  Rng rk(mix(seed, 1)), rq(mix(seed, 2)), rp(mix(seed, 3)), rd(mix(seed, 4)), rs(mix(seed, 5)),
      rf(mix(seed, 6)), rl(mix(seed, 7));
  int64_t d0 = days_from_civil(1992, 1, 2), d1 = days_from_civil(1998, 12, 1);
  int64_t key = 1, left = rk.uniform(1, 7);
  static const char* flags = "ANR";
  static const char* stat = "FO";
  for (uint64_t i = 0; i < rows; i++) {
    if (left == 0) {
      key++;
      left = rk.uniform(1, 7);
    }
    left--;
    ints[0][i] = key;
    ints[1][i] = rq.uniform(1, 50);
    ints[2][i] = rp.uniform(90000, 10500000);
    ints[3][i] = rd.uniform(0, 10);
    ints[4][i] = yyyymmdd(rs.uniform(d0, d1));
    chars[5][i] = flags[rf.uniform(0, 2)];
    chars[6][i] = stat[rl.uniform(0, 1)];
  }
  DataDict dd;
  std::string e2;
  load_data_dict(dir + "/data.dictionary", dd, e2);  // absent on first use
  if (!write_table(dir, "lineitem", spec, ints, chars, rows, seg_rows, dd, err)) return false;
  return save_data_dict(dir + "/data.dictionary", dd);
}

// Three-way workload: customer (custkey dense 1..C, mktsegment of 5 values), orders
// (orderkey = 4*i, custkey uniform FK, orderdate uniform over 7 years, shippriority 0),
// lineitem (orderkey FK in key order, shipdate = orderdate + U[1,121] days,
// extendedprice, discount). Rows per order: 1-7 uniform, or (zipf_s > 0) the skewed join
// of the compressed config: order i gets round(N F(i)) - round(N F(i - 1)) rows, F the
// Zipf(s) distribution over the orders (F(k) = H(k, s) / H(orders, s), H the generalised
// harmonic number), so the keys stay in order and the counts sum to N exactly.
bool gen_three_way(const std::string& dir, uint64_t customers, uint64_t orders, uint64_t lineitems,
                   uint32_t seg_rows, uint64_t seed, bool delta, double zipf_s, std::string& err) {
  DataDict dd;
  std::string e2;
  load_data_dict(dir + "/data.dictionary", dd, e2);
  {
    std::vector<ColumnSpec> spec = {{"c_custkey", 0, 0, 0, delta}, {"c_mktsegment", 2, 0, 10, false}};
    std::vector<std::vector<int64_t>> ints(2);
    std::vector<std::vector<char>> chars(2);
    ints[0].resize(customers);
    chars[1].assign(customers * 10, 0);
    Rng r(mix(seed, 11));
    for (uint64_t i = 0; i < customers; i++) {
      ints[0][i] = (int64_t)i + 1;
      put_str(chars[1], i, 10, kSegments[r.uniform(0, 4)]);
    }
    if (!write_table(dir, "customer", spec, ints, chars, customers, seg_rows, dd, err)) return false;
  }
  int64_t d0 = days_from_civil(1992, 1, 1), d1 = d0 + 7 * 365 - 1;
  std::vector<int64_t> odays(orders);
  {
    std::vector<ColumnSpec> spec = {{"o_orderkey", 0, 0, 0, delta}, {"o_custkey", 0, 0, 0, delta},
                                    {"o_orderdate", 0, 0, 0, delta}, {"o_shippriority", 0, 0, 0, delta}};
    std::vector<std::vector<int64_t>> ints(4);
    std::vector<std::vector<char>> chars(4);
    for (auto& v : ints) v.resize(orders);
    Rng rc(mix(seed, 21)), rd(mix(seed, 22));
    for (uint64_t i = 0; i < orders; i++) {
      ints[0][i] = 4 * ((int64_t)i + 1);
      ints[1][i] = rc.uniform(1, (int64_t)customers);
      odays[i] = rd.uniform(d0, d1);
      ints[2][i] = yyyymmdd(odays[i]);
      ints[3][i] = 0;
    }
    if (!write_table(dir, "orders", spec, ints, chars, orders, seg_rows, dd, err)) return false;
  }
  {
    std::vector<ColumnSpec> spec = {{"l_orderkey", 0, 0, 0, delta}, {"l_shipdate", 0, 0, 0, delta},
                                    {"l_extendedprice", 1, 2, 0, delta}, {"l_discount", 1, 2, 0, delta}};
    std::vector<std::vector<int64_t>> ints(4);
    std::vector<std::vector<char>> chars(4);
    for (auto& v : ints) v.resize(lineitems);
    Rng rk(mix(seed, 31)), rs(mix(seed, 32)), rp(mix(seed, 33)), rd(mix(seed, 34));
    uint64_t o = 0;
    int64_t left = 0;
    // Zipf: the cumulative row count after order o, from the running harmonic sum
    long double htotal = 0, hrun = 0;
    uint64_t emitted_to = 0;  // rows assigned to orders <= o
    auto zipf_next = [&]() -> int64_t {
      hrun += std::pow((long double)(o + 1), -(long double)zipf_s);
      const uint64_t upto = o + 1 >= orders ? lineitems
                                            : std::min<uint64_t>(lineitems, (uint64_t)std::llround((long double)lineitems * hrun / htotal));
      const int64_t n = (int64_t)(upto - emitted_to);
      emitted_to = upto;
      return n;
    };
    if (zipf_s > 0) {
      for (uint64_t k = 1; k <= orders; k++) htotal += std::pow((long double)k, -(long double)zipf_s);
      left = zipf_next();
      while (left == 0 && o + 1 < orders) {
        o++;
        left = zipf_next();
      }
    } else {
      left = rk.uniform(1, 7);
    }
    for (uint64_t i = 0; i < lineitems; i++) {
      while (left == 0) {
        if (zipf_s > 0) {
          o++;  // the counts sum to the row count: o stays below orders
          left = zipf_next();
        } else {
          o = (o + 1) % orders;  // wraps only when lineitems exceed 7 x orders
          left = rk.uniform(1, 7);
        }
      }
      left--;
      ints[0][i] = 4 * ((int64_t)o + 1);
      ints[1][i] = yyyymmdd(odays[o] + rs.uniform(1, 121));
      ints[2][i] = rp.uniform(90000, 10500000);
      ints[3][i] = rd.uniform(0, 10);
    }
    if (!write_table(dir, "lineitem", spec, ints, chars, lineitems, seg_rows, dd, err)) return false;
  }
  return save_data_dict(dir + "/data.dictionary", dd);
}

// Names workload for string predicates: table "names" with n_key (1..rows) and n_name,
// a char(12) column drawn from `distinct` generated strings over the letters A, B, X and
// the characters '.', '%', '_' (lengths 0 to 12, so some fill the width and carry no
// terminator): the cases that the LIKE matcher's wildcards and its '?'-against-'.' rule
// tell apart.
bool gen_names(const std::string& dir, uint64_t rows, uint32_t distinct, uint32_t seg_rows, uint64_t seed,
               std::string& err) {
  DataDict dd;
  std::string e2;
  load_data_dict(dir + "/data.dictionary", dd, e2);
  const char alphabet[] = "ABXAB.%_";
  Rng r(mix(seed, 41));
  std::vector<std::string> vocab(std::max<uint32_t>(distinct, 1));
  for (auto& w : vocab) {
    const int64_t len = r.uniform(0, 12);
    for (int64_t k = 0; k < len; k++) w.push_back(alphabet[r.uniform(0, 7)]);
  }
  std::vector<ColumnSpec> spec = {{"n_key", 0, 0, 0, false}, {"n_name", 2, 0, 12, false}};
  std::vector<std::vector<int64_t>> ints(2);
  std::vector<std::vector<char>> chars(2);
  ints[0].resize(rows);
  chars[1].assign(rows * 12, 0);
  for (uint64_t i = 0; i < rows; i++) {
    ints[0][i] = (int64_t)i + 1;
    const std::string& w = vocab[r.uniform(0, (int64_t)vocab.size() - 1)];
    std::memcpy(&chars[1][i * 12], w.data(), w.size());
  }
  if (!write_table(dir, "names", spec, ints, chars, rows, seg_rows, dd, err)) return false;
  return save_data_dict(dir + "/data.dictionary", dd);
}

}  // namespace alk

extern "C" {
// Generator entry points (tests and benchmarks). Return 0 on success; errors are
// written into err (err_len bytes).
int alk_gen_lineitem_flat(const char* dir, uint64_t rows, uint32_t seg_rows, uint64_t seed, int delta,
                          char* err, int err_len) {
  std::string e;
  bool ok = alk::gen_lineitem_flat(dir, rows, seg_rows, seed, delta != 0, e);
  if (!ok && err && err_len > 0) std::snprintf(err, (size_t)err_len, "%s", e.c_str());
  return ok ? 0 : 1;
}
int alk_gen_three_way(const char* dir, uint64_t customers, uint64_t orders, uint64_t lineitems,
                      uint32_t seg_rows, uint64_t seed, int delta, char* err, int err_len) {
  std::string e;
  bool ok = alk::gen_three_way(dir, customers, orders, lineitems, seg_rows, seed, delta != 0, 0.0, e);
  if (!ok && err && err_len > 0) std::snprintf(err, (size_t)err_len, "%s", e.c_str());
  return ok ? 0 : 1;
}
int alk_gen_three_way_zipf(const char* dir, uint64_t customers, uint64_t orders, uint64_t lineitems,
                           uint32_t seg_rows, uint64_t seed, int delta, double zipf_s, char* err, int err_len) {
  std::string e;
  if (!(zipf_s > 0) || orders == 0) {
    if (err && err_len > 0) std::snprintf(err, (size_t)err_len, "zipf exponent and orders must be positive");
    return 1;
  }
  bool ok = alk::gen_three_way(dir, customers, orders, lineitems, seg_rows, seed, delta != 0, zipf_s, e);
  if (!ok && err && err_len > 0) std::snprintf(err, (size_t)err_len, "%s", e.c_str());
  return ok ? 0 : 1;
}
int alk_gen_names(const char* dir, uint64_t rows, uint32_t distinct, uint32_t seg_rows, uint64_t seed, char* err,
                  int err_len) {
  std::string e;
  bool ok = alk::gen_names(dir, rows, distinct, seg_rows, seed, e);
  if (!ok && err && err_len > 0) std::snprintf(err, (size_t)err_len, "%s", e.c_str());
  return ok ? 0 : 1;
}
int64_t alk_date_add_days(int64_t yyyymmdd_value, int64_t days) {
  int64_t y = yyyymmdd_value / 10000, m = (yyyymmdd_value / 100) % 100, d = yyyymmdd_value % 100;
  return alk::yyyymmdd(alk::days_from_civil(y, m, d) + days);
}
}
