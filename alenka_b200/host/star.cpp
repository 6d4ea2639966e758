// Star join with bitmap join indexes: CREATE INDEX ... ON fact(dim.col) FROM fact, dim
// WHERE fact.fk = dim.key (emit_create_bitmap_index, operators.cu:2188-2268), and the
// join of a fact table with filtered dimensions through those indexes (check_star_join
// operators.cu:408-437, star_join operators.cu:440-794, check_bitmaps_exist
// cm.cu:4151-4206, loadIndex cm.cu:2775-2845).
//
// Device side: the index segments are built on the GPU (alk_bitmap_index_build) and kept
// resident as one code a row at 8, 16 or 32 bits (alk_bitmap_index_decode), with each
// segment's codes offset by the sizes of the dictionaries before it, so that all of an
// index's segments share one code space. A comparison with an index column compiles to a
// set-membership test (ALK_OP_INSET) over that space, built per comparison from each
// segment's dictionary, and the star join's filter is one fused scan of the fact table.
// The rows then get the reference's row-list quirk (alk_star_rows_fixup) and their
// columns are gathered from the stored segments (alk_star_gather).
#include <sys/stat.h>

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
void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw EngineError(e == cudaErrorMemoryAllocation ? ALK_ERR_NOMEM : ALK_ERR_CUDA,
                      std::string(what) + ": " + cudaGetErrorString(e));
}
[[noreturn]] void unsupported(const std::string& m) { throw EngineError(ALK_ERR_UNSUPPORTED, m); }
DevBufP mkbuf(size_t bytes, cudaStream_t s) { return std::make_shared<DevBuf>(bytes, s); }
bool file_exists(const std::string& p) {
  struct stat sb;
  return stat(p.c_str(), &sb) == 0;
}
template <class T>
void put(std::string& out, T v) {
  out.append((const char*)&v, sizeof(T));
}
}  // namespace

// The table whose files a variable reads: a catalog table, or the one a FILTER reads.
std::string Engine::star_table(Var* v) {
  if (v->kind == Var::Base) return v->table;
  if (v->kind == Var::Filtered) {
    Var* s = var(v->source);
    if (s->kind == Var::Base) return s->table;
  }
  unsupported("a star join or bitmap index over the materialized result " + v->name);
}

// emit_create_bitmap_index (operators.cu:2188-2268): for every segment i of ltable, the
// file <ltable>.<rtable>.<rcolumn>.<i> holds rcolumn of the dimension row that
// lower_bound finds for each row's lid in the dimension's rid column (the dimension's
// first segment), as compress_int writes it: u32 distinct count, the distinct values
// ascending (int64), u32 values per word, u32 bits, u32 words, u32 rows, the words. A
// char rcolumn contributes the dimension rows' .hash values; when the dimension has more
// rows than the fact segment, its remaining hashes follow the segment's values.
void Engine::emit_create_bitmap_index(Statement& st) {
  if (st.index_args.size() != 4) unsupported("CREATE INDEX without its four names");
  const std::string& ltable = st.f;
  const std::string& rtable = st.index_args[0];
  const std::string& rcol = st.index_args[1];
  const std::string& lid = st.index_args[2];
  const std::string& rid = st.index_args[3];
  Var* left = base_table(ltable);
  Var* right = base_table(rtable);
  if (!left) unsupported("Couldn't find " + ltable);
  if (!right) unsupported("Couldn't find " + rtable);
  if (!left->has(lid) || !right->has(rid) || !right->has(rcol))
    unsupported("CREATE INDEX names a column its table lacks");
  if (right->segCount != 1)
    unsupported("a bitmap index over a dimension of " + std::to_string(right->segCount) +
                " segments (the reference reads the dimension's first segment only)");
  const ColMeta rm = right->meta.at(rcol);
  if (rm.type != 0 && rm.type != 2) unsupported("a bitmap index on a float column");
  if (right->meta.at(rid).type != 0 || left->meta.at(lid).type != 0) unsupported("a bitmap index on char keys");
  Rows dim = materialize(right, {rid, rcol});
  const uint32_t m = (uint32_t)dim.n;
  DevBufP vals = dim.col.at(rcol);
  std::vector<uint64_t> hashes;
  if (rm.type == 2) {
    // the dimension rows' MurmurHash64A / 2 values from its first segment's .hash file
    std::vector<uint8_t> img;
    std::string e;
    const std::string p = dir_ + "/" + rtable + "." + rcol + ".0.hash";
    if (!read_file(p, img, e)) throw EngineError(ALK_ERR_IO, e);
    if (img.size() < 4) throw EngineError(ALK_ERR_IO, p + ": truncated");
    uint32_t cnt = 0;
    std::memcpy(&cnt, img.data(), 4);
    if (img.size() < 4 + (size_t)cnt * 8) throw EngineError(ALK_ERR_IO, p + ": truncated");
    hashes.resize(cnt);
    std::memcpy(hashes.data(), img.data() + 4, (size_t)cnt * 8);
    vals = mkbuf(std::max<size_t>(cnt, 1) * 8, stream_);
    ck(cudaMemcpyAsync(vals->as<void>(), hashes.data(), (size_t)cnt * 8, cudaMemcpyHostToDevice, stream_),
       "hash upload");
    stats_.h2d_bytes += (uint64_t)cnt * 8;
    if (cnt < m) unsupported("a dimension .hash file shorter than its segment");
  }
  Rows fk = materialize(left, {lid});
  const DevBufP& fkcol = fk.col.at(lid);
  uint64_t off = 0;
  std::vector<int64_t> dict;
  std::vector<uint64_t> words;
  for (uint32_t g = 0; g < left->segCount; g++) {
    const uint32_t n = (uint32_t)fk.seg_counts[g];
    if (n == 0) unsupported("a bitmap index over an empty segment");
    const uint32_t ntail = rm.type == 2 && hashes.size() > n ? (uint32_t)(hashes.size() - n) : 0;
    const int64_t* tail = ntail ? vals->as<int64_t>() + n : nullptr;
    dict.resize((size_t)n + ntail);
    words.resize((size_t)n + ntail);
    uint32_t dn = 0, wn = 0, bits = 0;
    const int rc = alk_bitmap_index_build(fkcol->as<int64_t>() + off, n, dim.col.at(rid)->as<int64_t>(), m,
                                          vals->as<int64_t>(), tail, ntail, dict.data(), &dn, words.data(), &wn,
                                          &bits, (alk_stream)stream_);
    if (rc == ALK_ERR_UNSUPPORTED)
      unsupported("a foreign key of " + ltable + "." + lid + " lies past the last key of " + rtable + "." + rid +
                  " (the reference reads past its key column there)");
    check(rc, "bitmap index build");
    stats_.kernels++;
    std::string img;
    put<uint32_t>(img, dn);
    img.append((const char*)dict.data(), (size_t)dn * 8);
    put<uint32_t>(img, 64 / bits);
    put<uint32_t>(img, bits);
    put<uint32_t>(img, wn);
    put<uint32_t>(img, n + ntail);
    img.append((const char*)words.data(), (size_t)wn * 8);
    const std::string path = dir_ + "/" + ltable + "." + rtable + "." + rcol + "." + std::to_string(g);
    if (!write_file(path, img.data(), img.size())) throw EngineError(ALK_ERR_IO, "cannot write " + path);
    off += n;
  }
  // a resident copy of an older index of this name is stale now
  auto t = basecols_.find(ltable);
  if (t != basecols_.end()) t->second.erase(rtable + "." + rcol);
}

// An index column of a fact table ("<dimension table>.<column>"): every segment's file
// <fact>.<dimension>.<column>.<segment>, its dictionary kept on the host and its codes
// resident at the narrowest of 8, 16 or 32 bits, offset by the dictionary sizes of the
// segments before it.
void Engine::load_star_index(Var* base, const std::string& col, BaseCol& bc) {
  if (bc.headers_read) return;
  bc.meta = ColMeta{};
  bc.segs.assign(base->segCount, SegInfo{});
  bc.host_img.assign(base->segCount, nullptr);
  bc.host_len.assign(base->segCount, 0);
  bc.dev.assign(base->segCount, nullptr);
  bc.res_lower.assign(base->segCount, 0);
  bc.res_bits.assign(base->segCount, 8);
  bc.idx_dict.assign(base->segCount, {});
  bc.idx_off.assign(base->segCount, 0);
  uint64_t space = 0;
  for (uint32_t g = 0; g < base->segCount; g++) {
    const std::string p = dir_ + "/" + base->table + "." + col + "." + std::to_string(g);
    std::vector<uint8_t> img;
    std::string e;
    if (!read_file(p, img, e)) throw EngineError(ALK_ERR_IO, e);
    auto bad = [&]() { throw EngineError(ALK_ERR_IO, p + ": malformed bitmap index segment"); };
    if (img.size() < 4) bad();
    uint32_t sz = 0;
    std::memcpy(&sz, img.data(), 4);
    const size_t head = 4 + (size_t)sz * 8;
    if (img.size() < head + 16) bad();
    uint32_t fit = 0, bits = 0, vals = 0, real = 0;
    std::memcpy(&fit, img.data() + head, 4);
    std::memcpy(&bits, img.data() + head + 4, 4);
    std::memcpy(&vals, img.data() + head + 8, 4);
    std::memcpy(&real, img.data() + head + 12, 4);
    if (bits == 0 || bits > 32 || fit != 64 / bits || (uint64_t)vals * fit < real ||
        img.size() < head + 16 + (size_t)vals * 8)
      bad();
    std::vector<int64_t>& d = bc.idx_dict[g];
    d.resize(sz);
    std::memcpy(d.data(), img.data() + 4, (size_t)sz * 8);
    const uint32_t out_bits = bits <= 8 ? 8 : (bits <= 16 ? 16 : 32);
    auto w = mkbuf(std::max<size_t>(vals, 1) * 8, stream_);
    ck(cudaMemcpyAsync(w->as<void>(), img.data() + head + 16, (size_t)vals * 8, cudaMemcpyHostToDevice, stream_),
       "index upload");
    ck(cudaStreamSynchronize(stream_), "index upload");  // img is pageable and goes out of scope
    stats_.h2d_bytes += (uint64_t)vals * 8;
    const size_t bytes = (size_t)real * (out_bits / 8);
    auto codes = mkbuf((bytes + 255) / 256 * 256 + 256, stream_);
    check(alk_bitmap_index_decode(w->as<uint64_t>(), real, bits, fit, codes->as<void>(), out_bits,
                                  (alk_stream)stream_),
          "bitmap index decode");
    stats_.kernels++;
    SegMeta& m = bc.segs[g].m;
    m.cnt = (uint32_t)bytes;
    m.rec_count = real;
    m.bits = out_bits;
    m.lower = m.orig_lower = (int64_t)space;
    m.upper = (int64_t)space + (sz ? sz - 1 : 0);
    bc.dev[g] = codes;
    bc.res_lower[g] = (int64_t)space;
    bc.res_bits[g] = out_bits;
    bc.idx_off[g] = space;
    space += sz;
  }
  bc.headers_read = true;
  ck(cudaStreamSynchronize(stream_), "index decode");
}

// The codes of an index column that a comparison with `key` keeps, as a set over the
// index's code space (filter.cu:397-415, 519-535, 560-577 with cmp_functor_dict): in a
// segment whose dictionary holds key, the code of key for ==, every other code for any
// other operator; in a segment whose dictionary lacks key, no code at all. The words are
// ALK_OP_INSET's layout: the space's size, then the bits.
std::vector<uint32_t> Engine::star_set(Var* base, const std::string& col, bool eq, int64_t key) {
  ensure_base_col(base, col, true);
  BaseCol& bc = basecol(base, col);
  uint64_t space = 0;
  for (auto& d : bc.idx_dict) space += d.size();
  if (space > 0xFFFFFFFFull) unsupported("bitmap index dictionaries above 2^32 codes");
  std::vector<uint32_t> w(1 + (space + 31) / 32, 0);
  w[0] = (uint32_t)space;
  for (size_t g = 0; g < bc.idx_dict.size(); g++) {
    const auto& d = bc.idx_dict[g];
    auto it = std::lower_bound(d.begin(), d.end(), key);
    if (it == d.end() || *it != key) continue;
    const uint64_t k = (uint64_t)(it - d.begin());
    for (uint64_t c = 0; c < d.size(); c++) {
      if ((c == k) != eq) continue;
      const uint64_t b = bc.idx_off[g] + c;
      w[1 + b / 32] |= 1u << (b % 32);
    }
  }
  return w;
}

// A code set on the device, kept until the script ends.
DevBufP Engine::star_upload(const std::vector<uint32_t>& w) {
  auto buf = mkbuf(w.size() * 4, stream_);
  ck(cudaMemcpyAsync(buf->as<void>(), w.data(), w.size() * 4, cudaMemcpyHostToDevice, stream_), "index set upload");
  ck(cudaStreamSynchronize(stream_), "index set upload");
  star_sets_.push_back(buf);
  return buf;
}

// The key a string literal compared with an index column stands for: MurmurHash64A of
// the literal NUL-padded (or cut) to the dimension column's width, halved (filter.cu:397-409).
int64_t Engine::star_string_key(const std::string& col, const std::string& lit) {
  const size_t dot = col.find('.');
  const std::string table = col.substr(0, dot), c = col.substr(dot + 1);
  auto t = dd_.find(table);
  if (t == dd_.end() || !t->second.count(c)) unsupported("bitmap index on an unknown column " + col);
  const uint32_t len = t->second.at(c).col_length;
  std::string s = lit;
  while (s.size() < len) s.push_back('\0');
  return (int64_t)(murmur64a(s.data(), (int)len, kHashSeed) / 2);
}

// check_star_join (operators.cu:408-437) with check_bitmap_file_exist (cm.cu:4131-4149):
// every ON pair starts with a column of the fact variable, and a single dimension has a
// filter whose every column of its own has an index file for the fact table.
bool Engine::star_join_applies(Statement& st) {
  if (st.join_tab_cnt == 0 || !vars_.count(st.f)) return false;
  Var* left = var(st.f);
  for (size_t k = 2 * (size_t)st.sel_count; k < st.op_value.size(); k += 2)
    if (!left->has(st.op_value[k])) return false;
  if (st.join_tab_cnt == 1) {
    if (st.op_join.empty() || !vars_.count(st.op_join[0])) return false;
    Var* right = var(st.op_join[0]);
    if (right->kind != Var::Filtered || right->fil_value.empty()) return false;
    if (left->kind == Var::Mat || var(right->source)->kind != Var::Base) return false;
    const std::string lt = star_table(left), rt = star_table(right);
    for (auto& c : right->fil_value)
      if (right->has(c) && !file_exists(dir_ + "/" + lt + "." + rt + "." + c + ".0")) return false;
  }
  return true;
}

// star_join (operators.cu:440-794). The dimensions' filters join the fact variable's
// filter with their columns renamed to the fact table's index columns, AND-ed in
// (check_bitmaps_exist, cm.cu:4151-4206); the fact rows passing it keep the reference's
// row lists; fact columns are read from the stored segments, dimension columns through
// the row lower_bound finds for (foreign key - 1) in the dimension's key column (the path
// the reference takes: its index files carry no sort flag).
void Engine::star_join(Statement& st) {
  Var* left = var(st.f);
  const std::string ltab = star_table(left);
  Var* lsrc = base_table(ltab);
  if (left->kind == Var::Filtered && left->scanned)
    unsupported("a star join over " + st.f + " after another statement read it (its row list is reused)");
  if (star_consumed_.count(st.f)) unsupported("a second star join over " + st.f);
  std::vector<std::pair<std::string, std::string>> sel;
  for (unsigned k = 0; k < st.sel_count; k++) {
    sel.push_back({st.op_value[2 * k], st.op_value[2 * k + 1]});
    if (sel.back().first != sel.back().second)
      unsupported("an alias in a star join (the reference names its columns by alias but fills them by name)");
  }
  Var f;
  f.kind = Var::Filtered;
  f.name = st.f;
  f.source = ltab;
  f.columnNames = lsrc->columnNames;
  f.meta = lsrc->meta;
  if (left->kind == Var::Filtered) {
    f.fil_type = left->fil_type;
    f.fil_value = left->fil_value;
    f.fil_nums = left->fil_nums;
    f.fil_prec = left->fil_prec;
  }
  struct Dim {
    std::string jvar, fk, key;
    Var* base = nullptr;
  };
  std::map<std::string, Dim> dims;  // key_map: by join variable name
  const size_t g0 = 2 * (size_t)st.sel_count;
  for (unsigned i = 0; i < st.join_tab_cnt; i++) {
    if (g0 + 2 * i + 1 >= st.op_value.size() || st.join_tab_cnt - 1 - i >= st.op_join.size())
      unsupported("a star join with fewer ON pairs than tables");
    Dim d;
    d.fk = st.op_value[g0 + 2 * i];
    d.key = st.op_value[g0 + 2 * i + 1];
    d.jvar = st.op_join[st.join_tab_cnt - 1 - i];
    Var* r = var(d.jvar);
    const std::string rtab = star_table(r);
    d.base = base_table(rtab);
    if (d.base->segCount != 1)
      unsupported("a star join with the dimension " + rtab + " of " + std::to_string(d.base->segCount) + " segments");
    if (star_consumed_.count(d.jvar)) unsupported("a second star join with " + d.jvar);
    if (r->kind == Var::Filtered && !r->fil_value.empty()) {
      for (auto& c : r->fil_value)
        if (r->has(c) && !file_exists(dir_ + "/" + ltab + "." + rtab + "." + c + ".0"))
          unsupported("Required bitmap on table " + d.jvar + " doesn't exists");
      const bool add_and = !f.fil_type.empty();
      f.fil_nums.insert(f.fil_nums.end(), r->fil_nums.begin(), r->fil_nums.end());
      f.fil_prec.insert(f.fil_prec.end(), r->fil_prec.begin(), r->fil_prec.end());
      for (auto& c : r->fil_value) f.fil_value.push_back(r->has(c) ? rtab + "." + c : c);
      f.fil_type.insert(f.fil_type.end(), r->fil_type.begin(), r->fil_type.end());
      if (add_and) f.fil_type.push_back("AND");
    }
    dims[d.jvar] = d;
  }
  if (f.fil_type.empty()) unsupported("a star join without a filter");

  // the filter: one scan of the fact table over its columns and index columns
  ScanPlan p;
  p.src = lsrc;
  p.pred = compile_filter(&f, lsrc, p.slots);
  p.has_pred = true;
  p.mode.assign(lsrc->segCount, 2);
  if (p.slots.size() > 16) unsupported("scan reads more than 16 columns");
  std::vector<alk_colseg> cs = colsegs(p);
  const uint32_t nseg = lsrc->segCount;
  std::vector<uint32_t> seg_rows(nseg);
  {
    BaseCol& bc = basecol(lsrc, lsrc->columnNames.at(0));
    read_headers(lsrc, lsrc->columnNames.at(0), bc);
    for (uint32_t g = 0; g < nseg; g++) seg_rows[g] = bc.segs[g].m.rec_count;
  }
  for (size_t s = 0; s < p.slots.size(); s++)
    for (uint32_t g = 0; g < nseg; g++)
      if (cs[s * nseg + g].rows != seg_rows[g])
        unsupported("the index " + p.slots[s] + " holds another row count than segment " + std::to_string(g));
  uint64_t cap = 0;
  for (uint32_t g = 0; g < nseg; g++) cap += seg_rows[g];
  auto rowid = mkbuf(std::max<uint64_t>(cap, 1) * 4, stream_);
  auto segof = mkbuf(std::max<uint64_t>(cap, 1) * 4, stream_);
  auto segc = mkbuf((size_t)nseg * 8, stream_);
  uint64_t count = 0;
  check(alk_scan_filter(cs.data(), (uint32_t)p.slots.size(), nseg, p.mode.data(), &p.pred, nullptr, 0, nullptr,
                        rowid->as<uint32_t>(), segof->as<uint32_t>(), segc->as<uint64_t>(), cap, &count,
                        (alk_stream)stream_),
        "star join scan");
  stats_.kernels++;
  std::vector<uint64_t> counts(nseg);
  ck(cudaMemcpyAsync(counts.data(), segc->as<void>(), (size_t)nseg * 8, cudaMemcpyDeviceToHost, stream_),
     "segment counts");
  ck(cudaStreamSynchronize(stream_), "star join scan");
  check(alk_star_rows_fixup(rowid->as<uint32_t>(), counts.data(), seg_rows.data(), nseg, (alk_stream)stream_),
        "star join rows");
  stats_.kernels++;

  auto stored = [&](const std::string& col) {
    ensure_base_col(lsrc, col, true);
    BaseCol& bc = basecol(lsrc, col);
    std::vector<alk_colseg> v(nseg);
    for (uint32_t g = 0; g < nseg; g++) {
      const SegMeta& m = bc.segs[g].m;
      if (m.comp_type != 0)
        unsupported("a star join reading the FOR-delta column " + col + " (the reference reads its packed bits raw)");
      v[g] = alk_colseg{bc.dev[g]->as<void>(), m.lower, m.rec_count, m.bits};
    }
    return v;
  };
  auto c = std::make_unique<Var>();
  c->kind = Var::Mat;
  c->name = st.s;
  c->n = count;
  for (auto& sc : sel) {
    const std::string& name = sc.first;
    if (std::find(c->columnNames.begin(), c->columnNames.end(), name) != c->columnNames.end()) continue;
    auto out = mkbuf(std::max<uint64_t>(count, 1) * 8, stream_);
    ColMeta meta;
    if (left->has(name)) {
      meta = lsrc->meta.at(name);
      if (meta.type == 2) unsupported("a char column of the fact table in a star join");
      std::vector<alk_colseg> v = stored(name);
      const int rc = alk_star_gather(v.data(), nseg, rowid->as<uint32_t>(), segof->as<uint32_t>(), count, nullptr,
                                     nullptr, out->as<int64_t>(), (alk_stream)stream_);
      if (rc == ALK_ERR_UNSUPPORTED)
        unsupported("a star join row reused from a longer segment (the reference reads past the segment)");
      check(rc, "star join gather");
    } else {
      const Dim* d = nullptr;
      for (auto& kv : dims)
        if (var(kv.first)->has(name)) {
          d = &kv.second;
          break;
        }
      if (!d) unsupported("the star join column " + name + " is in no joined table");
      meta = d->base->meta.at(name);
      if (meta.type == 2 && counts[0] == 0 && count)
        unsupported("a char dimension column in a star join whose first fact segment keeps no row");
      // the dimension's key and value columns at their resident widths (one segment)
      auto resident = [&](const std::string& col) {
        ensure_base_col(d->base, col, true);
        BaseCol& bc = basecol(d->base, col);
        return alk_colseg{bc.dev[0]->as<void>(), bc.res_lower[0], bc.segs[0].m.rec_count, bc.res_bits[0]};
      };
      const alk_colseg dk = resident(d->key), dv = resident(name);
      std::vector<alk_colseg> v = stored(d->fk);
      const int rc = alk_star_gather(v.data(), nseg, rowid->as<uint32_t>(), segof->as<uint32_t>(), count, &dk, &dv,
                                     out->as<int64_t>(), (alk_stream)stream_);
      if (rc == ALK_ERR_UNSUPPORTED)
        unsupported("a star join row past its segment or a foreign key past the last key of " + d->key);
      check(rc, "star join gather");
    }
    stats_.kernels++;
    c->columnNames.push_back(name);
    c->meta[name] = meta;
    c->data[name] = out;
  }
  star_consumed_.insert(st.f);
  for (auto& kv : dims) star_consumed_.insert(kv.first);
  vars_[st.s] = std::move(c);
}

}  // namespace alk
