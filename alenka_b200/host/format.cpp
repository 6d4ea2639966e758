// Alenka segment format: see format.h for the byte layout and reference citations.
#include "format.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include <fcntl.h>
#include <unistd.h>

namespace alk {

namespace {
template <typename T>
T rd(const uint8_t* p) {
  T v;
  std::memcpy(&v, p, sizeof(T));
  return v;
}
template <typename T>
void wr(std::vector<uint8_t>& out, T v) {
  const uint8_t* p = reinterpret_cast<const uint8_t*>(&v);
  out.insert(out.end(), p, p + sizeof(T));
}
}  // namespace

// Bits needed for a value range, computed as the reference does in double precision:
// (unsigned int)ceil(log2((double)((max - min) + 1))) (compress.cu:296, compress.cu:459).
uint32_t range_bits(int64_t lo, int64_t hi) {
  int64_t span = (int64_t)((uint64_t)hi - (uint64_t)lo + 1ULL);
  return (uint32_t)std::ceil(std::log2((double)span));
}

bool parse_segment(const uint8_t* buf, size_t len, SegMeta& m, const uint8_t** payload,
                   std::string& err) {
  if (len < kSegHeadBytes + kSegTailBytes) {
    err = "segment image too short";
    return false;
  }
  m.cnt = rd<uint32_t>(buf);
  m.lower = rd<int64_t>(buf + 4);
  m.upper = rd<int64_t>(buf + 12);
  m.comp_type = rd<uint32_t>(buf + 20);
  if ((size_t)m.cnt + kSegHeadBytes + kSegTailBytes > len) {
    err = "segment payload length exceeds file";
    return false;
  }
  const uint8_t* t = buf + kSegHeadBytes + m.cnt;
  // trailer: cnt, rec_count, bits, orig_lower, fit_count, start_val (compress.cu:184-189)
  m.rec_count = rd<uint32_t>(t + 4);
  m.bits = rd<uint32_t>(t + 8);
  m.orig_lower = rd<int64_t>(t + 12);
  m.fit_count = rd<uint32_t>(t + 20);
  m.start_val = rd<int64_t>(t + 24);
  if (m.comp_type == 0) {
    if (m.bits != 8 && m.bits != 16 && m.bits != 32 && m.bits != 64) {
      err = "FOR segment with invalid width";
      return false;
    }
    if ((uint64_t)m.rec_count * (m.bits / 8) > m.cnt) {
      err = "FOR segment payload shorter than rec_count";
      return false;
    }
  } else if (m.comp_type == 1) {
    if (m.bits == 0 || m.bits > 64 || m.fit_count == 0 || m.fit_count != 64 / m.bits) {
      err = "delta segment with invalid width";
      return false;
    }
    uint64_t words = (m.rec_count + m.fit_count - 1) / m.fit_count;
    if (words * 8 > m.cnt) {
      err = "delta segment payload shorter than rec_count";
      return false;
    }
  } else {
    err = "unsupported comp_type " + std::to_string(m.comp_type);
    return false;
  }
  *payload = buf + kSegHeadBytes;
  return true;
}

bool read_file(const std::string& path, std::vector<uint8_t>& out, std::string& err) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) {
    err = "cannot open " + path;
    return false;
  }
  std::fseek(f, 0, SEEK_END);
  long sz = std::ftell(f);
  std::fseek(f, 0, SEEK_SET);
  out.resize(sz > 0 ? (size_t)sz : 0);
  size_t got = sz > 0 ? std::fread(out.data(), 1, (size_t)sz, f) : 0;
  std::fclose(f);
  if (got != out.size()) {
    err = "short read on " + path;
    return false;
  }
  return true;
}

bool write_file(const std::string& path, const void* data, size_t len, bool append) {
  if (append) {
    FILE* f = std::fopen(path.c_str(), "ab");
    if (!f) return false;
    size_t put = len ? std::fwrite(data, 1, len, f) : 0;
    std::fclose(f);
    return put == len;
  }
  // the new contents over the old ones, then the file cut to their length: the same
  // result as truncating first, without freeing and reallocating the file's blocks
  // (an order of magnitude cheaper for the small results that queries store)
  const int fd = ::open(path.c_str(), O_WRONLY | O_CREAT, 0666);
  if (fd < 0) return false;
  const char* p = (const char*)data;
  size_t left = len;
  bool ok = true;
  while (left) {
    const ssize_t w = ::write(fd, p, left);
    if (w <= 0) {
      ok = false;
      break;
    }
    p += w;
    left -= (size_t)w;
  }
  if (ok && ::ftruncate(fd, (off_t)len) != 0) ok = false;
  if (::close(fd) != 0) ok = false;
  return ok;
}

void encode_for(const int64_t* v, uint32_t n, SegMeta& m, std::vector<uint8_t>& payload) {
  int64_t lo = n ? v[0] : 0, hi = lo;
  for (uint32_t i = 1; i < n; i++) {
    lo = std::min(lo, v[i]);
    hi = std::max(hi, v[i]);
  }
  uint32_t bits = range_bits(lo, hi);
  if (bits != 8 && bits != 16 && bits != 32 && bits != 64) {
    if (bits < 8) bits = 8;
    else if (bits < 16) bits = 16;
    else if (bits < 32) bits = 32;
    else bits = 64;
  }
  payload.resize((size_t)n * (bits / 8));
  for (uint32_t i = 0; i < n; i++) {
    uint64_t d = (uint64_t)v[i] - (uint64_t)lo;
    switch (bits) {
      case 8: payload[i] = (uint8_t)d; break;
      case 16: { uint16_t x = (uint16_t)d; std::memcpy(&payload[2 * (size_t)i], &x, 2); } break;
      case 32: { uint32_t x = (uint32_t)d; std::memcpy(&payload[4 * (size_t)i], &x, 4); } break;
      default: std::memcpy(&payload[8 * (size_t)i], &d, 8); break;
    }
  }
  m.cnt = (uint32_t)payload.size();
  m.lower = lo;
  m.upper = hi;
  m.comp_type = 0;
  m.rec_count = n;
  m.bits = bits;
  m.orig_lower = lo;
  m.fit_count = 64 / bits;
  m.start_val = 0;
}

void encode_delta(const int64_t* v, uint32_t n, SegMeta& m, std::vector<uint8_t>& payload) {
  std::vector<int64_t> d(n);
  for (uint32_t i = 0; i < n; i++) d[i] = i ? (int64_t)((uint64_t)v[i] - (uint64_t)v[i - 1]) : v[0];
  int64_t start = n ? d[0] : 0;
  if (n > 1) d[0] = d[1];
  int64_t lo = n ? d[0] : 0, hi = lo;
  for (uint32_t i = 1; i < n; i++) {
    lo = std::min(lo, d[i]);
    hi = std::max(hi, d[i]);
  }
  uint32_t bits = range_bits(lo, hi);
  if (bits == 0) bits = 1;
  uint32_t fit = 64 / bits;
  uint32_t words = (n + fit - 1) / fit;
  std::vector<uint64_t> w(words, 0);
  for (uint32_t i = 0; i < n; i++) {
    uint64_t val = (uint64_t)d[i] - (uint64_t)lo;
    uint32_t shift = 64 - bits - (i % fit) * bits;
    w[i / fit] += val << shift;  // the reference sums shifted values per word (reduce_by_key)
  }
  payload.resize((size_t)words * 8);
  if (words) std::memcpy(payload.data(), w.data(), payload.size());
  m.cnt = (uint32_t)payload.size();
  m.lower = n ? v[0] : 0;
  m.upper = n ? v[n - 1] : 0;
  m.comp_type = 1;
  m.rec_count = n;
  m.bits = bits;
  m.orig_lower = lo;
  m.fit_count = fit;
  m.start_val = start;
}

std::vector<uint8_t> segment_image(const SegMeta& m, const std::vector<uint8_t>& payload) {
  std::vector<uint8_t> out;
  out.reserve(kSegHeadBytes + payload.size() + kSegTailBytes);
  wr<uint32_t>(out, m.cnt);
  wr<int64_t>(out, m.lower);
  wr<int64_t>(out, m.upper);
  wr<uint32_t>(out, m.comp_type);
  out.insert(out.end(), payload.begin(), payload.end());
  wr<uint32_t>(out, m.cnt);
  wr<uint32_t>(out, m.rec_count);
  wr<uint32_t>(out, m.bits);
  wr<int64_t>(out, m.orig_lower);
  wr<uint32_t>(out, m.fit_count);
  wr<int64_t>(out, m.start_val);
  return out;
}

bool read_col_header(const std::string& path, ColHeader& h, std::string& err) {
  std::vector<uint8_t> b;
  if (!read_file(path, b, err)) return false;
  if (b.size() < 16) {
    err = "short column header " + path;
    return false;
  }
  h.total = rd<uint64_t>(b.data());
  h.segs = rd<uint32_t>(b.data() + 8);
  h.max_recs = rd<uint32_t>(b.data() + 12);
  h.max_cnt = b.size() >= 20 ? rd<uint32_t>(b.data() + 16) : 0;
  return true;
}

bool write_col_header(const std::string& path, const ColHeader& h) {
  std::vector<uint8_t> b;
  wr<uint64_t>(b, h.total);
  wr<uint32_t>(b, h.segs);
  wr<uint32_t>(b, h.max_recs);
  wr<uint32_t>(b, h.max_cnt);
  return write_file(path, b.data(), b.size());
}

uint64_t murmur64a(const void* key, int len, uint32_t seed) {
  const uint64_t m = 0xc6a4a7935bd1e995ULL;
  const int r = 47;
  uint64_t h = seed ^ ((uint64_t)(int64_t)len * m);
  const uint8_t* p = static_cast<const uint8_t*>(key);
  int blocks = len / 8;
  for (int i = 0; i < blocks; i++) {
    uint64_t k;
    std::memcpy(&k, p + 8 * i, 8);
    k *= m;
    k ^= k >> r;
    k *= m;
    h ^= k;
    h *= m;
  }
  const uint8_t* t = p + 8 * blocks;
  switch (len & 7) {
    case 7: h ^= (uint64_t)t[6] << 48; [[fallthrough]];
    case 6: h ^= (uint64_t)t[5] << 40; [[fallthrough]];
    case 5: h ^= (uint64_t)t[4] << 32; [[fallthrough]];
    case 4: h ^= (uint64_t)t[3] << 24; [[fallthrough]];
    case 3: h ^= (uint64_t)t[2] << 16; [[fallthrough]];
    case 2: h ^= (uint64_t)t[1] << 8; [[fallthrough]];
    case 1: h ^= (uint64_t)t[0]; h *= m;
  }
  h ^= h >> r;
  h *= m;
  h ^= h >> r;
  return h;
}

bool load_data_dict(const std::string& path, DataDict& dd, std::string& err) {
  std::vector<uint8_t> b;
  if (!read_file(path, b, err)) return false;
  size_t off = 0;
  auto need = [&](size_t k) { return off + k <= b.size(); };
  if (!need(8)) { err = "short data.dictionary"; return false; }
  uint64_t tabs = rd<uint64_t>(&b[off]); off += 8;
  for (uint64_t i = 0; i < tabs; i++) {
    if (!need(8)) { err = "truncated data.dictionary"; return false; }
    uint64_t l = rd<uint64_t>(&b[off]); off += 8;
    if (!need(l + 8)) { err = "truncated data.dictionary"; return false; }
    std::string t((const char*)&b[off], l); off += l;
    uint64_t ncol = rd<uint64_t>(&b[off]); off += 8;
    for (uint64_t j = 0; j < ncol; j++) {
      if (!need(8)) { err = "truncated data.dictionary"; return false; }
      uint64_t cl = rd<uint64_t>(&b[off]); off += 8;
      if (!need(cl + 8)) { err = "truncated data.dictionary"; return false; }
      std::string c((const char*)&b[off], cl); off += cl;
      ColData cd;
      cd.col_type = rd<uint32_t>(&b[off]); off += 4;
      cd.col_length = rd<uint32_t>(&b[off]); off += 4;
      dd[t][c] = cd;
    }
  }
  return true;
}

bool save_data_dict(const std::string& path, const DataDict& dd) {
  std::vector<uint8_t> b;
  wr<uint64_t>(b, dd.size());
  for (auto& t : dd) {
    wr<uint64_t>(b, t.first.size());
    b.insert(b.end(), t.first.begin(), t.first.end());
    wr<uint64_t>(b, t.second.size());
    for (auto& c : t.second) {
      wr<uint64_t>(b, c.first.size());
      b.insert(b.end(), c.first.begin(), c.first.end());
      wr<uint32_t>(b, c.second.col_type);
      wr<uint32_t>(b, c.second.col_length);
    }
  }
  return write_file(path, b.data(), b.size());
}

TableWriter::TableWriter(std::string dir, std::string table, std::vector<ColumnSpec> cols)
    : dir_(std::move(dir)), table_(std::move(table)), cols_(std::move(cols)) {
  max_cnt_.assign(cols_.size(), 0);
  dict_.resize(cols_.size());
}

bool TableWriter::write_segment(const std::vector<const int64_t*>& ints,
                                const std::vector<const char*>& chars, uint32_t rows,
                                std::string& err) {
  const std::string base = dir_ + "/" + table_ + ".";
  std::vector<int64_t> codes;
  for (size_t c = 0; c < cols_.size(); c++) {
    const ColumnSpec& cs = cols_[c];
    const int64_t* vals = nullptr;
    std::string seg_path = base + cs.name + "." + std::to_string(segs_);
    if (cs.kind == 2) {
      // dictionary codes in first-seen order keyed by MurmurHash64A/2 (cm.cu:1806-1819)
      const char* s = chars[c];
      codes.resize(rows);
      std::vector<int64_t> hashes(rows);
      std::string dict_append;
      for (uint32_t i = 0; i < rows; i++) {
        uint64_t h = murmur64a(s + (size_t)i * cs.width, (int)cs.width, kHashSeed) / 2;
        hashes[i] = (int64_t)h;
        auto it = dict_[c].find(h);
        if (it == dict_[c].end()) {
          int64_t code = (int64_t)dict_[c].size();
          dict_[c][h] = code;
          dict_append.append(s + (size_t)i * cs.width, cs.width);
          codes[i] = code;
        } else {
          codes[i] = it->second;
        }
      }
      if (!write_file(base + cs.name, dict_append.data(), dict_append.size(), segs_ != 0)) {
        err = "cannot write dictionary for " + cs.name;
        return false;
      }
      std::vector<uint8_t> hb;
      wr<uint32_t>(hb, rows);
      const uint8_t* hp = reinterpret_cast<const uint8_t*>(hashes.data());
      hb.insert(hb.end(), hp, hp + 8 * (size_t)rows);
      if (!write_file(seg_path + ".hash", hb.data(), hb.size())) {
        err = "cannot write hash file";
        return false;
      }
      vals = codes.data();
      seg_path += ".idx";
    } else {
      vals = ints[c];
    }
    SegMeta m;
    std::vector<uint8_t> payload;
    bool sorted = cs.delta && std::is_sorted(vals, vals + rows);
    if (sorted && rows > 0)
      encode_delta(vals, rows, m, payload);
    else
      encode_for(vals, rows, m, payload);
    std::vector<uint8_t> img = segment_image(m, payload);
    if (!write_file(seg_path, img.data(), img.size())) {
      err = "cannot write " + seg_path;
      return false;
    }
    max_cnt_[c] = std::max(max_cnt_[c], m.cnt);
  }
  segs_++;
  total_ += rows;
  max_recs_ = std::max(max_recs_, rows);
  return true;
}

bool TableWriter::finish(DataDict& dd, std::string& err) {
  for (size_t c = 0; c < cols_.size(); c++) {
    ColHeader h;
    h.total = total_;
    h.segs = segs_;
    h.max_recs = max_recs_;
    h.max_cnt = max_cnt_[c];
    if (!write_col_header(dir_ + "/" + table_ + "." + cols_[c].name + ".header", h)) {
      err = "cannot write header";
      return false;
    }
    ColData cd;
    cd.col_type = cols_[c].kind == 2 ? 2 : 0;
    cd.col_length = cols_[c].kind == 1 ? cols_[c].decimals : (cols_[c].kind == 2 ? cols_[c].width : 0);
    dd[table_][cols_[c].name] = cd;
  }
  return true;
}

}  // namespace alk
