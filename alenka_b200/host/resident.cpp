// Tables generated in device memory (no files): the single-table lineitem shape at sizes
// whose files would not fit the host's disk or time budget. The session holds them as
// catalog tables whose every column segment is resident; their zone maps and
// frame-of-reference bases are exact per segment, as the file encoder would write them.
#include <algorithm>
#include <cmath>
#include <cstring>

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
// stored width for a value range: the smallest of 8/16/32/64 bits holding max - min
// (the file encoder's choice, pfor_compress compress.cu:271-360)
uint32_t width_for(int64_t lo, int64_t hi) {
  const uint64_t span = (uint64_t)hi - (uint64_t)lo;
  if (span < (1ull << 8)) return 8;
  if (span < (1ull << 16)) return 16;
  if (span < (1ull << 32)) return 32;
  return 64;
}
struct GenCol {
  const char* name;
  int type;        // 0 int / decimal, 2 char
  uint32_t len;    // decimals, or char width
  const char* dict[3];
};
const GenCol kCols[7] = {{"l_orderkey", 0, 0, {}},      {"l_quantity", 0, 0, {}},
                         {"l_extendedprice", 0, 2, {}}, {"l_discount", 0, 2, {}},
                         {"l_shipdate", 0, 0, {}},      {"l_returnflag", 2, 1, {"A", "N", "R"}},
                         {"l_linestatus", 2, 1, {"F", "O", nullptr}}};
}  // namespace

int Engine::gen_resident_flat(const std::string& t, const std::vector<uint32_t>& seg_rows, uint64_t seed,
                              uint64_t row_base) {
  try {
    const uint32_t nseg = (uint32_t)seg_rows.size();
    if (nseg == 0 || t.empty() || bases_.count(t) || dd_.count(t)) throw EngineError(ALK_ERR_ARG, "table exists: " + t);
    std::vector<int64_t> mm((size_t)nseg * 7 * 2);
    check(alk_gen_flat_minmax(seed, row_base, seg_rows.data(), nseg, mm.data(), (alk_stream)stream_), "generator");
    auto v = std::make_shared<Var>();
    v->kind = Var::Base;
    v->name = v->table = t;
    v->load_file_name = dir_ + "/" + t;
    v->segCount = nseg;
    for (auto r : seg_rows) {
      v->maxRecs = std::max(v->maxRecs, r);
      v->total += r;
    }
    std::vector<alk_colseg> cs((size_t)7 * nseg);
    for (int c = 0; c < 7; c++) {
      const GenCol& gc = kCols[c];
      ColData cd;
      cd.col_type = (uint32_t)gc.type;
      cd.col_length = gc.len;
      dd_[t][gc.name] = cd;
      ColMeta m;
      m.type = gc.type;
      if (gc.type == 0) m.dz = gc.len;
      else {
        m.width = gc.len;
        m.string_map = t + "." + gc.name;
      }
      v->columnNames.push_back(gc.name);
      v->meta[gc.name] = m;
      BaseCol& bc = basecols_[t][gc.name];
      bc.meta = m;
      bc.segs.resize(nseg);
      bc.host_img.assign(nseg, nullptr);
      bc.host_len.assign(nseg, 0);
      bc.dev.resize(nseg);
      bc.res_lower.assign(nseg, 0);
      bc.res_bits.assign(nseg, 64);
      bc.headers_read = true;
      bc.device_only = true;
      for (uint32_t g = 0; g < nseg; g++) {
        const int64_t lo = mm[((size_t)g * 7 + c) * 2], hi = mm[((size_t)g * 7 + c) * 2 + 1];
        SegMeta& s = bc.segs[g].m;
        s.bits = width_for(lo, hi);
        s.rec_count = seg_rows[g];
        s.cnt = (uint32_t)((uint64_t)seg_rows[g] * (s.bits / 8));
        s.lower = lo;
        s.upper = hi;
        s.comp_type = 0;
        s.orig_lower = lo;
        s.fit_count = 64 / s.bits;
        s.start_val = 0;
        bc.dev[g] = std::make_shared<DevBuf>(((size_t)s.cnt + 255) / 256 * 256 + 256, stream_);
        bc.res_lower[g] = lo;
        bc.res_bits[g] = s.bits;
        alk_colseg& d = cs[(size_t)c * nseg + g];
        d.data = bc.dev[g]->as<void>();
        d.lower = lo;
        d.rows = seg_rows[g];
        d.bits = s.bits;
      }
      if (gc.type == 2) {
        for (int k = 0; k < 3 && gc.dict[k]; k++) {
          std::string str(gc.dict[k]);
          str.resize(gc.len, '\0');
          bc.hash_to_code[murmur64a(str.data(), (int)gc.len, kHashSeed) / 2] = k;
          bc.dict.push_back(str);
        }
        bc.dict_loaded = true;
      }
    }
    check(alk_gen_flat_write(seed, row_base, seg_rows.data(), nseg, cs.data(), (alk_stream)stream_), "generator");
    bases_[t] = v;
  } catch (const EngineError& e) {
    err_ = e.what();
    return e.code;
  }
  return ALK_OK;
}

}  // namespace alk
