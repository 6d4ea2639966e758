// Host engine: catalog and residency, zone maps, the predicate / select-list
// compilers (symbolic versions of the reference's stack machines) and operator
// execution. All device work goes through the operator-level C ABI.
#include "engine.h"

#include "../csrc/internal.h"

#include <algorithm>
#include <array>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>

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

// (unsigned int)pow(10, p) as the reference computes scale factors (cm.cu:159, 2488).
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
uint8_t vm_op(const std::string& op) {
  if (op == "MUL") return ALK_OP_MUL;
  if (op == "ADD") return ALK_OP_ADD;
  if (op == "MINUS") return ALK_OP_SUB;
  return ALK_OP_DIV;
}
uint8_t cmp_op(int64_t c) {
  switch (c) {
    case 1: return ALK_OP_LT;
    case 2: return ALK_OP_GT;
    case 5: return ALK_OP_LE;
    case 6: return ALK_OP_GE;
    case 4: return ALK_OP_EQ;
    case 3: return ALK_OP_NE;
    default: unsupported("comparison code " + std::to_string(c) + " (LIKE / <=>) is not supported");
  }
}
int64_t reverse_op(int64_t op) {  // cm.cu:3166-3180
  if (op == 2) return 1;
  if (op == 1) return 2;
  if (op == 6) return 5;
  if (op == 5) return 6;
  return op;
}
// precision_func (zone_map.cu:668-712), arguments updated in place.
uint32_t precision_func(uint32_t& p1, uint32_t& p2, const std::string& op) {
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

// ---------------- register-machine builder ----------------
struct Operand {
  uint8_t kind = ALK_K_CONST;
  uint16_t idx = 0;
};
struct ProgBuilder {
  alk_program p{};
  uint32_t live = 0;  // register in-use bitmask
  ProgBuilder() { std::memset(&p, 0, sizeof(p)); }
  Operand konst(int64_t v) {
    for (uint32_t i = 0; i < nconst; i++)
      if (p.consts[i] == v) return {ALK_K_CONST, (uint16_t)i};
    if (nconst >= ALK_MAX_CONST) unsupported("expression has too many constants");
    p.consts[nconst] = v;
    return {ALK_K_CONST, (uint16_t)nconst++};
  }
  Operand col(uint32_t slot) { return {ALK_K_COL, (uint16_t)slot}; }
  void release(Operand o) {
    if (o.kind == ALK_K_REG) live &= ~(1u << o.idx);
  }
  Operand emit(uint8_t op, Operand a, Operand b) {
    release(a);
    release(b);
    uint32_t r = 0;
    while (r < ALK_MAX_REGS && (live >> r) & 1) r++;
    if (r >= ALK_MAX_REGS) unsupported("expression needs more than 8 registers");
    live |= 1u << r;
    if (p.n_instr >= ALK_MAX_INSTR) unsupported("expression too long");
    alk_instr& in = p.ins[p.n_instr++];
    in.op = op;
    in.dst = (uint8_t)r;
    in.ka = a.kind;
    in.a = a.idx;
    in.kb = b.kind;
    in.b = b.idx;
    return {ALK_K_REG, (uint16_t)r};
  }
  alk_program finish(Operand res) {
    if (res.kind != ALK_K_REG) res = emit(ALK_OP_MOV, res, res);
    p.result = res.idx;
    return p;
  }
  uint32_t nconst = 0;
};

// CudaSet::op(int_type* column1, int_type d, op, reverse, p1, p2) (cm.cu:2480-2556) as
// register-machine instructions.
Operand op_const(ProgBuilder& b, Operand c, int64_t d, const std::string& op, bool reverse, uint32_t p1, uint32_t p2) {
  int64_t d1 = (int64_t)(unsigned int)d;
  if (p2) d = wmul(d, pow10u(p2));
  if (!reverse) {
    if (op == "MUL") return b.emit(ALK_OP_MUL, c, b.konst(d1));
    if (!p1) return b.emit(vm_op(op), c, b.konst(wmul(d, pow10u(p2))));  // scaled twice (cm.cu:2497)
    Operand cs = b.emit(ALK_OP_MUL, c, b.konst(pow10u(p1)));
    return b.emit(vm_op(op), cs, b.konst(d));
  }
  Operand x = p1 ? b.emit(ALK_OP_MUL, c, b.konst(pow10u(p1))) : c;
  return b.emit(vm_op(op), b.konst(d), x);
}
// CudaSet::op(int_type* column1, int_type* column2, op, reverse=0, p1, p2) (cm.cu:2559-2600)
Operand op_vec(ProgBuilder& b, Operand c1, Operand c2, const std::string& op, uint32_t p1, uint32_t p2) {
  if (op == "MUL") return b.emit(ALK_OP_MUL, c1, c2);
  Operand x = p1 ? b.emit(ALK_OP_MUL, c1, b.konst(pow10u(p1))) : c1;
  Operand y = p2 ? b.emit(ALK_OP_MUL, c2, b.konst(pow10u(p2))) : c2;
  return b.emit(vm_op(op), x, y);
}
}  // namespace

// ------------------------------------------------------------------ DevBuf
DevBuf::DevBuf(size_t bytes, cudaStream_t s) : n_(bytes), s_(s) {
  ck(cudaMallocAsync(&p_, std::max<size_t>(bytes, 16), s), "device allocation");
}
DevBuf::~DevBuf() { reset(); }
void DevBuf::reset() {
  if (p_) cudaFreeAsync(p_, s_);
  p_ = nullptr;
  n_ = 0;
}
DevBuf::DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_) { o.p_ = nullptr; }
DevBuf& DevBuf::operator=(DevBuf&& o) noexcept {
  reset();
  p_ = o.p_;
  n_ = o.n_;
  s_ = o.s_;
  o.p_ = nullptr;
  return *this;
}

bool Var::has(const std::string& c) const {
  return std::find(columnNames.begin(), columnNames.end(), c) != columnNames.end();
}

static DevBufP mkbuf(size_t bytes, cudaStream_t s) { return std::make_shared<DevBuf>(bytes, s); }

// ------------------------------------------------------------------ engine
Engine::Engine(std::string dir, uint32_t flags) : dir_(std::move(dir)), flags_(flags) {
  ck(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
  int dev = 0;
  cudaGetDevice(&dev);
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  cudaEventCreate(&ev0_);
  cudaEventCreate(&ev1_);
  cudaEventCreate(&evq0_);
  cudaEventCreate(&evq1_);
  std::string e;
  load_data_dict(dir_ + "/data.dictionary", dd_, e);
}

Engine::~Engine() {
  vars_.clear();
  star_sets_.clear();  // device buffers free on the stream, destroyed below
  for (auto& t : basecols_)
    for (auto& c : t.second) {
      for (auto* h : c.second.host_img)
        if (h) cudaFreeHost(h);
      c.second.dev.clear();
    }
  basecols_.clear();
  bases_.clear();
  if (card_mlp_) alk_mlp_free(card_mlp_, (alk_stream)stream_);
  cudaStreamSynchronize(stream_);
  if (ev0_) cudaEventDestroy(ev0_);
  if (ev1_) cudaEventDestroy(ev1_);
  if (evq0_) cudaEventDestroy(evq0_);
  if (evq1_) cudaEventDestroy(evq1_);
  if (pin_) cudaFreeHost(pin_);
  cudaStreamDestroy(stream_);
}

void* Engine::pinned(size_t bytes) {
  if (bytes > pin_n_) {
    cudaStreamSynchronize(stream_);  // the old buffer may still be a copy destination
    if (pin_) cudaFreeHost(pin_);
    pin_ = nullptr;
    pin_n_ = 0;
    const size_t n = std::max<size_t>(bytes, 1 << 20);
    ck(cudaMallocHost(&pin_, n), "pinned staging buffer");
    pin_n_ = n;
  }
  return pin_;
}

Var* Engine::var(const std::string& n) {
  auto it = vars_.find(n);
  if (it != vars_.end()) return it->second.get();
  throw EngineError(ALK_ERR_ARG, "couldn't find variable " + n);
}

// emit_load_binary / load_vars (operators.cu:2518-2552, 2708-2747): a catalog table
// becomes a variable holding every column of the catalog entry.
Var* Engine::base_table(const std::string& t) {
  auto it = bases_.find(t);
  if (it != bases_.end()) return it->second.get();
  auto dt = dd_.find(t);
  if (dt == dd_.end()) return nullptr;
  auto v = std::make_shared<Var>();
  v->kind = Var::Base;
  v->name = v->table = t;
  v->load_file_name = dir_ + "/" + t;
  std::string first;
  for (auto& c : dt->second) {
    ColMeta m;
    if (c.second.col_type == 0) {
      m.type = 0;
      m.dz = (c.second.col_length != 0 && c.second.col_length != UINT32_MAX) ? c.second.col_length : 0;
    } else if (c.second.col_type == 2) {
      m.type = 2;
      m.width = c.second.col_length;
      m.string_map = t + "." + c.first;
    } else {
      continue;  // float columns are outside the supported path
    }
    v->columnNames.push_back(c.first);
    v->meta[c.first] = m;
    if (first.empty()) first = c.first;
  }
  if (first.empty()) return nullptr;
  ColHeader h;
  std::string e;
  if (!read_col_header(v->load_file_name + "." + first + ".header", h, e)) throw EngineError(ALK_ERR_IO, e);
  v->segCount = h.segs;
  v->maxRecs = h.max_recs;
  v->total = h.total;
  bases_[t] = v;
  return v.get();
}

BaseCol& Engine::basecol(Var* base, const std::string& col) {
  BaseCol& bc = basecols_[base->table][col];
  if (col.find('.') == std::string::npos) bc.meta = base->meta.at(col);  // else a bitmap index column
  return bc;
}

void Engine::read_headers(Var* base, const std::string& col, BaseCol& bc) {
  if (bc.headers_read) return;
  if (col.find('.') != std::string::npos) {  // a bitmap join index column
    load_star_index(base, col, bc);
    return;
  }
  bc.segs.resize(base->segCount);
  bc.host_img.assign(base->segCount, nullptr);
  bc.host_len.assign(base->segCount, 0);
  bc.dev.resize(base->segCount);
  for (uint32_t g = 0; g < base->segCount; g++) {
    std::string p = base->load_file_name + "." + col + "." + std::to_string(g);
    if (bc.meta.type == 2) p += ".idx";
    std::vector<uint8_t> img;
    std::string e;
    if (!read_file(p, img, e)) throw EngineError(ALK_ERR_IO, e);
    const uint8_t* payload = nullptr;
    if (!parse_segment(img.data(), img.size(), bc.segs[g].m, &payload, e))
      throw EngineError(ALK_ERR_IO, p + ": " + e);
    bc.segs[g].file_off = kSegHeadBytes;
    uint8_t* h = nullptr;
    ck(cudaMallocHost((void**)&h, img.size()), "pinned host buffer");
    std::memcpy(h, img.data(), img.size());
    bc.host_img[g] = h;
    bc.host_len[g] = img.size();
  }
  bc.headers_read = true;
}

void Engine::ensure_base_col(Var* base, const std::string& col, bool device) {
  BaseCol& bc = basecol(base, col);
  read_headers(base, col, bc);
  if (!device) return;
  for (uint32_t g = 0; g < base->segCount; g++) {
    if (bc.dev[g]) continue;
    const SegMeta& m = bc.segs[g].m;
    size_t padded = ((size_t)m.cnt + 255) / 256 * 256 + 256;
    auto buf = mkbuf(padded, stream_);
    ck(cudaMemcpyAsync(buf->as<uint8_t>(), bc.host_img[g] + bc.segs[g].file_off, m.cnt, cudaMemcpyHostToDevice,
                       stream_),
       "segment upload");
    stats_.h2d_bytes += m.cnt;
    bc.res_lower.resize(base->segCount, 0);
    bc.res_bits.resize(base->segCount, 64);
    if (m.comp_type == 1) {
      // decoded once (bit unpack + prefix sum), then kept as FOR at the narrowest width
      // over the segment's exact range, padded like the FOR payloads (bulk tile copies
      // round their length up to 16 bytes); every scan kernel then reads it as FOR
      auto dec = mkbuf((size_t)m.rec_count * 8 + 256, stream_);
      check(alk_decode_segment(buf->as<void>(), 1, m.bits, m.fit_count, m.orig_lower, m.start_val, m.rec_count,
                               dec->as<int64_t>(), (alk_stream)stream_),
            "delta decode");
      const size_t cap = (size_t)m.rec_count * 8;
      auto narrow = mkbuf((cap + 255) / 256 * 256 + 256, stream_);
      int64_t lo = 0;
      uint32_t bits = 64;
      check(alk_for_reencode(dec->as<int64_t>(), m.rec_count, narrow->as<void>(), cap, &lo, &bits,
                             (alk_stream)stream_),
            "delta re-encode");
      bc.dev[g] = narrow;
      bc.res_lower[g] = lo;
      bc.res_bits[g] = bits;
    } else {
      bc.dev[g] = buf;
      bc.res_lower[g] = m.orig_lower;
      bc.res_bits[g] = m.bits;
    }
  }
}

void Engine::load_dict(Var* base, const std::string& col, BaseCol& bc) {
  if (bc.dict_loaded) return;
  std::vector<uint8_t> raw;
  std::string e;
  if (!read_file(base->load_file_name + "." + col, raw, e)) throw EngineError(ALK_ERR_IO, e);
  uint32_t w = bc.meta.width;
  for (size_t off = 0; off + w <= raw.size(); off += w) {
    std::string s((const char*)&raw[off], w);
    uint64_t h = murmur64a(s.data(), (int)w, kHashSeed) / 2;
    if (!bc.hash_to_code.count(h)) bc.hash_to_code[h] = (int64_t)bc.dict.size();
    bc.dict.push_back(s);
  }
  bc.dict_loaded = true;
}

// The codes of a char column whose dictionary entries match a LIKE pattern, on the
// device as [count, bits...]; kept per pattern with the column (the reference keeps its
// match list per column too, map_res in filter.cu:454-500).
DevBufP Engine::like_set(Var* base, const std::string& col, const std::string& pattern) {
  BaseCol& bc = basecol(base, col);
  auto it = bc.like_sets.find(pattern);
  if (it != bc.like_sets.end()) return it->second;
  if (pattern.size() >= 256) unsupported("a LIKE pattern of 256 bytes or more");
  load_dict(base, col, bc);
  const uint32_t w = bc.meta.width;
  const uint64_t count = bc.dict.size();
  std::string raw;
  raw.reserve(count * w);
  for (auto& s : bc.dict) raw += s;
  auto d_dict = mkbuf(std::max<size_t>(raw.size(), 1), stream_);
  if (!raw.empty())
    ck(cudaMemcpyAsync(d_dict->as<void>(), raw.data(), raw.size(), cudaMemcpyHostToDevice, stream_), "dictionary h2d");
  stats_.h2d_bytes += raw.size();
  auto set = mkbuf((1 + (count + 31) / 32) * 4, stream_);
  check(alk_like_dictionary(d_dict->as<char>(), w, count, pattern.data(), (uint32_t)pattern.size(),
                            set->as<uint32_t>(), (alk_stream)stream_),
        "LIKE");
  ck(cudaStreamSynchronize(stream_), "LIKE");  // the dictionary copy is released here
  bc.like_sets[pattern] = set;
  return set;
}

int Engine::preload(const std::string& table) {
  try {
    Var* b = base_table(table);
    if (!b) throw EngineError(ALK_ERR_ARG, "unknown table " + table);
    for (auto& c : b->columnNames) ensure_base_col(b, c, true);
    ck(cudaStreamSynchronize(stream_), "preload");
  } catch (const EngineError& e) {
    err_ = e.what();
    return e.code;
  }
  return ALK_OK;
}

size_t Engine::cycle_count(Var* v) {
  if (v->kind == Var::Filtered) return var(v->source)->segCount;
  if (v->kind == Var::Base) return v->segCount;
  return 1;
}

// ------------------------------------------------------------------ zone maps
// zone_map_check (zone_map.cu:720-1135) on the segment headers' [lower, upper].
std::vector<char> Engine::zone_maps(Var* f, Var* src) {
  std::vector<char> out(src->segCount, 'R');
  for (uint32_t g = 0; g < src->segCount; g++) {
    std::map<std::string, std::array<int64_t, 2>> mm;
    for (auto& n : f->fil_value) {
      if (mm.count(n) || !src->has(n) || src->meta[n].type > 1) continue;
      BaseCol& bc = basecol(src, n);
      read_headers(src, n, bc);
      mm[n] = {bc.segs[g].m.lower, bc.segs[g].m.upper};
    }
    std::vector<std::string> et, ev;
    std::vector<std::array<int64_t, 2>> evec;
    std::vector<int64_t> en;
    std::vector<uint32_t> ep;
    std::vector<char> bools;
    size_t iv = 0, in = 0, ip = 0;  // op_value, op_nums, op_nums_precision positions
    bool give_up = false;
    auto get_dec = [&](const std::string& s) -> uint32_t { return src->has(s) ? src->meta[s].dz : pop(ep); };
    for (auto& ss : f->fil_type) {
      if (ss == "NAME" || ss == "NUMBER" || ss == "FLOAT" || ss == "STRING") {
        et.push_back(ss);
        if (ss == "NUMBER") {
          en.push_back(f->fil_nums[in]);
          ep.push_back(f->fil_prec[ip++]);
          in++;
        } else if (ss == "NAME" || ss == "STRING") {
          if (ss == "NAME" && !src->has(f->fil_value[iv]))
            throw EngineError(ALK_ERR_ARG, "Couldn't find column " + f->fil_value[iv]);
          ev.push_back(f->fil_value[iv++]);
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
          et.push_back("NUMBER");
          en.push_back(arith(ss, n1, n2));
        } else if ((s1 == "NAME" && s2 == "NUMBER") || (s1 == "NUMBER" && s2 == "NAME")) {
          std::string nm = pop(ev);
          int64_t n1 = pop(en);
          uint32_t p2 = pop(ep);
          uint32_t p1 = get_dec(nm);
          std::array<int64_t, 2> t = src->has(nm) ? mm[nm] : pop(evec);
          ep.push_back(precision_func(p1, p2, ss));
          if (p1) {
            t[0] = wmul(t[0], pow10u(p1));
            t[1] = wmul(t[1], pow10u(p1));
            if (src->has(nm)) mm[nm] = t;
          }
          if (p2) n1 = wmul(n1, pow10u(p2));
          bool rev = s1 == "NAME";
          std::array<int64_t, 2> r;  // host_op (zone_map.cu:513-561)
          if (!rev || ss == "MUL" || ss == "ADD") {
            r = {arith(ss, t[0], n1), arith(ss, t[1], n1)};
          } else {
            r = {arith(ss, n1, t[0]), arith(ss, n1, t[1])};
          }
          et.push_back("NAME");
          ev.push_back("");
          evec.push_back(r);
        } else if (s1 == "NAME" && s2 == "NAME") {
          std::string v1 = pop(ev), v2 = pop(ev);
          uint32_t p1 = get_dec(v1), p2 = get_dec(v2);
          std::array<int64_t, 2> t = src->has(v1) ? mm[v1] : pop(evec);
          std::array<int64_t, 2> s3 = src->has(v2) ? mm[v2] : pop(evec);
          et.push_back("NAME");
          ev.push_back("");
          ep.push_back(precision_func(p1, p2, ss));
          if (p1) {
            t = {wmul(t[0], pow10u(p1)), wmul(t[1], pow10u(p1))};
            if (src->has(v1)) mm[v1] = t;
          }
          if (p2) {
            s3 = {wmul(s3[0], pow10u(p2)), wmul(s3[1], pow10u(p2))};
            if (src->has(v2)) mm[v2] = s3;
          }
          std::array<int64_t, 2> r;  // host_op(t, s3, op, reverse=1) (zone_map.cu:413-458)
          if (ss == "MUL" || ss == "ADD") r = {arith(ss, t[0], s3[0]), arith(ss, t[1], s3[1])};
          else r = {arith(ss, s3[0], t[0]), arith(ss, s3[1], t[1])};
          evec.push_back(r);
        } else {
          give_up = true;
          break;
        }
        continue;
      }
      if (ss == "CMP") {
        int64_t cmp = f->fil_nums[in++];
        std::string s1 = pop(et), s2 = pop(et);
        if (s1 == "NUMBER" && s2 == "NUMBER") {
          int64_t n1 = pop(en), n2 = pop(en);
          uint32_t p1 = pop(ep), p2 = pop(ep);
          uint32_t pres = std::max(p1, p2);
          ep.push_back(pres);
          et.push_back("NAME");
          ev.push_back("");
          if (p1) n1 = wmul(n1, pow10u(pres - p1));
          if (p2) n2 = wmul(n2, pow10u(pres - p2));
          // host_compare(int s, int d, op) (zone_map.cu:78-104): falls through to '!='
          char r = 'N';
          int64_t s = n1, d = n2;
          if (cmp == 2 && d > s) r = 'A';
          else if (cmp == 1 && d < s) r = 'A';
          else if (cmp == 6 && d >= s) r = 'A';
          else if (cmp == 5 && d <= s) r = 'A';
          else if (cmp == 4 && d == s) r = 'A';
          else if (d != s) r = 'A';
          bools.push_back(r);
        } else if ((s1 == "STRING" && s2 == "NAME") || (s1 == "NAME" && s2 == "STRING")) {
          pop(ev);
          pop(ev);
          bools.push_back('R');
          et.push_back("NAME");
          ev.push_back("");
        } else if ((s1 == "NUMBER" && s2 == "NAME") || (s1 == "NAME" && s2 == "NUMBER")) {
          if (s1 == "NAME") cmp = reverse_op(cmp);
          int64_t n1 = pop(en);
          std::string nm = pop(ev);
          uint32_t p2 = pop(ep);
          uint32_t p1 = get_dec(nm);
          std::array<int64_t, 2> t = src->has(nm) ? mm[nm] : pop(evec);
          uint32_t pres = std::max(p1, p2);
          ep.push_back(pres);
          if (p1) {
            t = {wmul(t[0], pow10u(pres - p1)), wmul(t[1], pow10u(pres - p1))};
            if (src->has(nm)) mm[nm] = t;
          }
          if (p2) n1 = wmul(n1, pow10u(pres - p2));
          et.push_back("NAME");
          ev.push_back("");
          // host_compare(int_type* column, d, op) (zone_map.cu:130-174)
          char r = 'R';
          int64_t d = n1;
          if (cmp == 2) {
            if (t[1] <= d) r = 'N';
            else if (t[0] > d) r = 'A';
          } else if (cmp == 1) {
            if (t[0] >= d) r = 'N';
            else if (t[1] < d) r = 'A';
          } else if (cmp == 6) {
            if (t[1] < d) r = 'N';
            else if (t[0] >= d) r = 'A';
          } else if (cmp == 5) {
            if (t[0] > d) r = 'N';
            else if (t[1] <= d) r = 'A';
          } else if (cmp == 4 && t[0] == d && t[1] == d) {
            r = 'A';
          }
          bools.push_back(r);
        } else {
          give_up = true;
          break;
        }
        continue;
      }
      if (ss == "AND" || ss == "OR") {
        char b3 = pop(bools), b2 = pop(bools);
        et.push_back("NAME");
        char r;
        if (ss == "AND") r = (b2 == 'A' && b3 == 'A') ? 'A' : ((b2 == 'N' || b3 == 'N') ? 'N' : 'R');
        else r = (b2 == 'A' && b3 == 'A') ? 'A' : ((b2 == 'N' && b3 == 'N') ? 'N' : 'R');
        bools.push_back(r);
        continue;
      }
      if (ss == "JOIN") throw EngineError(ALK_ERR_UNSUPPORTED, "operation = is not valid");
      throw EngineError(ALK_ERR_UNSUPPORTED, "operation " + ss + " is not valid");
    }
    out[g] = give_up || bools.empty() ? 'R' : bools.back();
  }
  return out;
}

// ------------------------------------------------------------------ predicate compiler
// Symbolic run of filter() (filter.cu:133-643) emitting register-machine code. slots
// receives the source columns the program reads, in slot order.
alk_program Engine::compile_filter(Var* f, Var* src, std::vector<std::string>& slots) {
  ProgBuilder b;
  std::vector<std::string> et, ev;
  std::vector<Operand> evec, bools;
  std::vector<int64_t> en;
  std::vector<uint32_t> ep;
  size_t iv = 0, in = 0, ip = 0;  // op_value, op_nums, op_nums_precision positions
  auto slot = [&](const std::string& c) {
    auto it = std::find(slots.begin(), slots.end(), c);
    if (it != slots.end()) return b.col((uint32_t)(it - slots.begin()));
    slots.push_back(c);
    return b.col((uint32_t)slots.size() - 1);
  };
  // Comparisons with a bitmap index column stay host-side code sets until something other
  // than AND / OR of sets over the same column consumes them: those fold into one set, so
  // a filter such as d == x OR d == y OR ... tests one set per row.
  constexpr uint8_t kPendingSet = 0xFF;
  std::vector<std::pair<std::string, std::vector<uint32_t>>> psets;
  auto pending = [&](const std::string& col, std::vector<uint32_t> w) {
    psets.push_back({col, std::move(w)});
    return Operand{kPendingSet, (uint16_t)(psets.size() - 1)};
  };
  // a pending set as an ALK_OP_INSET test of its index column
  auto materialize_set = [&](Operand o) -> Operand {
    if (o.kind != kPendingSet) return o;
    const DevBufP buf = star_upload(psets[o.idx].second);
    return b.emit(ALK_OP_INSET, slot(psets[o.idx].first), b.konst((int64_t)(uintptr_t)buf->as<void>()));
  };
  auto get_dec = [&](const std::string& s) -> uint32_t { return src->has(s) ? src->meta[s].dz : pop(ep); };
  auto get_vec = [&](const std::string& s) -> Operand { return src->has(s) ? slot(s) : pop(evec); };
  for (auto& ss : f->fil_type) {
    if (ss == "NAME" || ss == "NUMBER" || ss == "STRING") {
      if (ss == "NUMBER") {
        en.push_back(f->fil_nums[in]);
        ep.push_back(f->fil_prec[ip++]);
        in++;
      } else {
        ev.push_back(f->fil_value[iv++]);
      }
      et.push_back(ss);
      continue;
    }
    if (ss == "FLOAT" || ss == "FIELD") unsupported(ss + " operands in a filter are not supported");
    if (ss == "MUL" || ss == "ADD" || ss == "DIV" || ss == "MINUS") {
      std::string s1 = pop(et), s2 = pop(et);
      if (s1 == "NUMBER" && s2 == "NUMBER") {
        int64_t n1 = pop(en), n2 = pop(en);
        uint32_t p1 = pop(ep), p2 = pop(ep);
        ep.push_back(precision_func(p1, p2, ss));
        if (p1) n1 = wmul(n1, pow10u(p1));
        if (p2) n2 = wmul(n2, pow10u(p2));
        evec.push_back(b.emit(ALK_OP_MOV, b.konst(arith(ss, n1, n2)), b.konst(0)));
        et.push_back("NAME");
        ev.push_back("");
      } else if (s1 == "NAME" && s2 == "NUMBER") {
        std::string v = pop(ev);
        int64_t n1 = pop(en);
        uint32_t p1 = pop(ep);
        uint32_t p2 = get_dec(v);
        Operand t = get_vec(v);
        ep.push_back(precision_func(p1, p2, ss));
        et.push_back("NAME");
        ev.push_back("");
        evec.push_back(op_const(b, t, n1, ss, true, p1, p2));
      } else if (s1 == "NUMBER" && s2 == "NAME") {
        int64_t n1 = pop(en);
        std::string v = pop(ev);
        uint32_t p1 = pop(ep);
        uint32_t p2 = get_dec(v);
        Operand t = get_vec(v);
        ep.push_back(precision_func(p2, p1, ss));
        et.push_back("NAME");
        ev.push_back("");
        evec.push_back(op_const(b, t, n1, ss, false, p2, p1));
      } else if (s1 == "NAME" && s2 == "NAME") {
        std::string v1 = pop(ev), v2 = pop(ev);
        Operand t1 = get_vec(v1);
        Operand t = get_vec(v2);
        uint32_t p1 = get_dec(v1), p2 = get_dec(v2);
        ep.push_back(precision_func(p1, p2, ss));
        et.push_back("NAME");
        ev.push_back("");
        evec.push_back(op_vec(b, t, t1, ss, p2, p1));
      } else {
        unsupported("string arithmetic in a filter");
      }
      continue;
    }
    if (ss == "CMP") {
      int64_t cmp = f->fil_nums[in++];
      std::string s1 = pop(et), s2 = pop(et);
      if (s1 == "NUMBER" && s2 == "NUMBER") {
        int64_t n1 = pop(en), n2 = pop(en);
        et.push_back("NAME");
        ev.push_back("");
        uint32_t p1 = pop(ep), p2 = pop(ep);
        ep.push_back(precision_func(p1, p2, "CMP"));
        if (p1) n1 = wmul(n1, pow10u(p1));
        if (p2) n2 = wmul(n2, pow10u(p2));
        // CudaSet::compare(int s, int d, op) evaluates d OP s (cm.cu:2132-2175)
        bools.push_back(b.emit(cmp_op(cmp), b.konst(n2), b.konst(n1)));
      } else if ((s1 == "STRING" && s2 == "NAME") || (s1 == "NAME" && s2 == "STRING")) {
        std::string v1 = pop(ev), v2 = pop(ev);
        if (s1 == "NAME") std::swap(v1, v2);  // v1 literal, v2 column
        if (v2.find('.') != std::string::npos) {
          // a bitmap join index column: the literal's hash looked up in each segment's
          // dictionary, == keeps its code and any other operator the other codes
          // (filter.cu:397-415)
          bools.push_back(pending(v2, star_set(src, v2, cmp == 4, star_string_key(v2, v1))));
          et.push_back("NAME");
          continue;
        }
        if (cmp != 4 && cmp != 3 && cmp != 7) unsupported("string comparison other than == / != / LIKE");
        if (!src->has(v2) || src->meta[v2].type != 2) unsupported("string compared with a non-char column");
        if (cmp == 7) {
          // LIKE: the dictionary entries that match, as a set of codes (filter.cu:454-500)
          const DevBufP set = like_set(src, v2, v1);
          bools.push_back(b.emit(ALK_OP_INSET, slot(v2), b.konst((int64_t)(uintptr_t)set->as<void>())));
          et.push_back("NAME");
          continue;
        }
        // .hash rows equal MurmurHash64A(literal padded to the width)/2 exactly when the
        // row's dictionary code is the literal's code (cm.cu:1806-1819, filter.cu:428-449)
        BaseCol& bc = basecol(src, v2);
        load_dict(src, v2, bc);
        std::string lit = v1;
        while (lit.size() < bc.meta.width) lit.push_back('\0');
        uint64_t h = murmur64a(lit.data(), (int)lit.size(), kHashSeed) / 2;
        auto it = bc.hash_to_code.find(h);
        int64_t code = it == bc.hash_to_code.end() ? -1 : it->second;
        bools.push_back(b.emit(cmp == 4 ? ALK_OP_EQ : ALK_OP_NE, slot(v2), b.konst(code)));
        et.push_back("NAME");
      } else if (((s1 == "NUMBER" && s2 == "NAME") || (s1 == "NAME" && s2 == "NUMBER")) && !ev.empty() &&
                 ev.back().find('.') != std::string::npos) {
        // a bitmap join index column against a number: the number itself looked up in each
        // segment's dictionary (filter.cu:519-535, 560-577); the number's precision stays
        // on the precision stack, as the reference pops and pushes none there
        int64_t n1 = pop(en);
        std::string v = pop(ev);
        bools.push_back(pending(v, star_set(src, v, cmp == 4, n1)));
        et.push_back("NAME");
      } else if (s1 == "NUMBER" && s2 == "NAME") {
        int64_t n1 = pop(en);
        std::string v = pop(ev);
        Operand t = get_vec(v);
        uint32_t p2 = pop(ep);
        uint32_t p1 = get_dec(v);
        uint32_t pres = std::max(p1, p2);
        ep.push_back(pres);
        et.push_back("NAME");
        // compare(t, n1, op, pres-p1, pres-p2) (cm.cu:2250-2295)
        uint32_t cp1 = pres - p1, cp2 = pres - p2;
        int64_t d = cp2 ? wmul(n1, (int64_t)std::pow(10.0, (double)cp2)) : n1;
        Operand x = cp1 ? b.emit(ALK_OP_MUL, t, b.konst(pow10u(cp1))) : t;
        bools.push_back(b.emit(cmp_op(cmp), x, b.konst(d)));
      } else if (s1 == "NAME" && s2 == "NUMBER") {
        cmp = reverse_op(cmp);
        int64_t n1 = pop(en);
        std::string v = pop(ev);
        Operand t = get_vec(v);
        uint32_t p2 = pop(ep);
        uint32_t p1 = get_dec(v);
        ep.push_back(std::max(p1, p2));
        et.push_back("NAME");
        // compare(t, n1, op, p1, p2) with the raw precisions (filter.cu:590)
        int64_t d = p2 ? wmul(n1, (int64_t)std::pow(10.0, (double)p2)) : n1;
        Operand x = p1 ? b.emit(ALK_OP_MUL, t, b.konst(pow10u(p1))) : t;
        bools.push_back(b.emit(cmp_op(cmp), x, b.konst(d)));
      } else if (s1 == "NAME" && s2 == "NAME") {
        std::string v1 = pop(ev), v2 = pop(ev);
        et.push_back("NAME");
        Operand t = get_vec(v1);
        Operand t1 = get_vec(v2);
        uint32_t p1 = get_dec(v1), p2 = get_dec(v2);
        ep.push_back(std::max(p1, p2));
        if (p1) unsupported("column comparison with a scaled right operand (undefined in the reference)");
        Operand x = p2 ? b.emit(ALK_OP_MUL, t1, b.konst(pow10u(p2))) : t1;
        bools.push_back(b.emit(cmp_op(cmp), x, t));
      } else {
        unsupported("comparison operands " + s1 + "/" + s2);
      }
      continue;
    }
    if (ss == "AND" || ss == "OR") {
      Operand b3 = pop(bools), b2 = pop(bools);
      et.push_back("NAME");
      if (b2.kind == kPendingSet && b3.kind == kPendingSet && psets[b2.idx].first == psets[b3.idx].first) {
        std::vector<uint32_t> w = psets[b2.idx].second;
        const std::vector<uint32_t>& w3 = psets[b3.idx].second;
        for (size_t k = 1; k < w.size(); k++) w[k] = ss == "AND" ? (w[k] & w3[k]) : (w[k] | w3[k]);
        bools.push_back(pending(psets[b2.idx].first, std::move(w)));
        continue;
      }
      b2 = materialize_set(b2);
      b3 = materialize_set(b3);
      bools.push_back(b.emit(ss == "AND" ? ALK_OP_AND : ALK_OP_OR, b2, b3));
      continue;
    }
    unsupported("operation " + ss + " is not valid in a filter");
  }
  if (bools.empty()) unsupported("filter without a comparison");
  Operand res = materialize_set(bools.back());
  if (slots.size() > 16) unsupported("filter reads more than 16 columns");
  return b.finish(res);
}

// ------------------------------------------------------------------ materialization
Rows Engine::materialize(Var* v, const std::vector<std::string>& fields, bool want_seg) {
  Rows r;
  if (v->kind == Var::Mat) {
    r.n = v->n;
    for (auto& fl : fields) {
      if (!v->has(fl)) continue;
      if (v->meta.at(fl).raw) unsupported("the char column " + fl + " of a LOAD is read by STORE ... BINARY only");
      if (!v->data.count(fl) && v->host.count(fl)) {  // a host-held small result column
        const auto& h = v->host.at(fl);
        auto d = mkbuf(std::max<size_t>(h.size(), 1) * 8, stream_);
        if (!h.empty())
          ck(cudaMemcpyAsync(d->as<void>(), h.data(), h.size() * 8, cudaMemcpyHostToDevice, stream_), "h2d");
        stats_.h2d_bytes += h.size() * 8;
        v->data[fl] = d;
      }
      r.col[fl] = v->data.at(fl);
    }
    r.seg_counts = {v->n};
    if (want_seg) {
      r.seg_of_row = mkbuf(std::max<uint64_t>(v->n, 1) * 4, stream_);
      ck(cudaMemsetAsync(r.seg_of_row->as<void>(), 0, std::max<uint64_t>(v->n, 1) * 4, stream_), "memset");
    }
    return r;
  }
  Var* src = v->kind == Var::Filtered ? var(v->source) : v;
  if (src->kind != Var::Base) unsupported("FILTER over a materialized result");
  std::vector<std::string> slots;
  alk_program prog{};
  bool have_prog = false;
  std::vector<uint8_t> mode(src->segCount, 1);
  if (v->kind == Var::Filtered) {
    v->scanned = true;
    std::vector<char> zm = zone_maps(v, src);
    prog = compile_filter(v, src, slots);
    have_prog = true;
    for (uint32_t g = 0; g < src->segCount; g++) mode[g] = zm[g] == 'N' ? 0 : (zm[g] == 'A' ? 1 : 2);
  }
  std::vector<uint32_t> out_slots;
  std::vector<std::string> out_names;
  for (auto& fl : fields) {
    if (!src->has(fl) || std::find(out_names.begin(), out_names.end(), fl) != out_names.end()) continue;
    auto it = std::find(slots.begin(), slots.end(), fl);
    if (it == slots.end()) {
      slots.push_back(fl);
      it = slots.end() - 1;
    }
    out_slots.push_back((uint32_t)(it - slots.begin()));
    out_names.push_back(fl);
  }
  if (slots.empty()) slots.push_back(src->columnNames.at(0));  // row counts only
  if (slots.size() > 16) unsupported("scan reads more than 16 columns");
  uint64_t cap = 0;
  for (uint32_t g = 0; g < src->segCount; g++) {
    if (!mode[g]) {
      stats_.segments_skipped++;
      continue;
    }
  }
  std::vector<alk_colseg> cs(slots.size() * src->segCount);
  for (size_t c = 0; c < slots.size(); c++) {
    ensure_base_col(src, slots[c], true);
    BaseCol& bc = basecol(src, slots[c]);
    for (uint32_t g = 0; g < src->segCount; g++) {
      const SegMeta& m = bc.segs[g].m;
      alk_colseg& d = cs[c * src->segCount + g];
      d.data = bc.dev[g]->as<void>();
      d.rows = m.rec_count;
      d.lower = bc.res_lower[g];
      d.bits = bc.res_bits[g];
    }
  }
  for (uint32_t g = 0; g < src->segCount; g++)
    if (mode[g]) {
      cap += cs[g].rows;
      stats_.rows_scanned += cs[g].rows;
    }
  std::vector<int64_t*> outp;
  for (auto& n : out_names) {
    auto b = mkbuf(std::max<uint64_t>(cap, 1) * 8, stream_);
    r.col[n] = b;
    outp.push_back(b->as<int64_t>());
  }
  if (want_seg) r.seg_of_row = mkbuf(std::max<uint64_t>(cap, 1) * 4, stream_);
  auto segc = mkbuf(src->segCount * 8, stream_);
  uint64_t count = 0;
  int rc = alk_scan_filter(cs.data(), (uint32_t)slots.size(), src->segCount, mode.data(),
                           have_prog ? &prog : nullptr, out_slots.data(), (uint32_t)out_slots.size(), outp.data(),
                           nullptr, want_seg ? r.seg_of_row->as<uint32_t>() : nullptr, segc->as<uint64_t>(), cap,
                           &count, (alk_stream)stream_);
  check(rc, "segment scan");
  r.n = count;
  r.seg_counts.resize(src->segCount);
  ck(cudaMemcpyAsync(r.seg_counts.data(), segc->as<void>(), src->segCount * 8, cudaMemcpyDeviceToHost, stream_),
     "segment counts");
  ck(cudaStreamSynchronize(stream_), "scan sync");
  return r;
}

}  // namespace alk

namespace alk {

uint32_t ScanPlan::slot(const std::string& c) {
  auto it = std::find(slots.begin(), slots.end(), c);
  if (it != slots.end()) return (uint32_t)(it - slots.begin());
  slots.push_back(c);
  if (slots.size() > 16) throw EngineError(ALK_ERR_UNSUPPORTED, "scan reads more than 16 columns");
  return (uint32_t)slots.size() - 1;
}

ScanPlan Engine::plan_scan(Var* v) {
  ScanPlan p;
  p.src = v->kind == Var::Filtered ? var(v->source) : v;
  if (p.src->kind != Var::Base) throw EngineError(ALK_ERR_UNSUPPORTED, "scan of a materialized result");
  p.mode.assign(p.src->segCount, 1);
  if (v->kind == Var::Filtered) {
    v->scanned = true;
    std::vector<char> zm = zone_maps(v, p.src);
    p.pred = compile_filter(v, p.src, p.slots);
    p.has_pred = true;
    for (uint32_t g = 0; g < p.src->segCount; g++) {
      p.mode[g] = zm[g] == 'N' ? 0 : (zm[g] == 'A' ? 1 : 2);
      if (!p.mode[g]) stats_.segments_skipped++;
    }
  }
  return p;
}

std::vector<alk_colseg> Engine::colsegs(const ScanPlan& p) {
  Var* src = p.src;
  std::vector<alk_colseg> cs(p.slots.size() * src->segCount);
  for (size_t c = 0; c < p.slots.size(); c++) {
    ensure_base_col(src, p.slots[c], true);
    BaseCol& bc = basecol(src, p.slots[c]);
    for (uint32_t g = 0; g < src->segCount; g++) {
      const SegMeta& m = bc.segs[g].m;
      alk_colseg& d = cs[c * src->segCount + g];
      d.data = bc.dev[g]->as<void>();
      d.rows = m.rec_count;
      d.lower = bc.res_lower[g];
      d.bits = bc.res_bits[g];
    }
  }
  for (uint32_t g = 0; g < src->segCount; g++)
    if (p.mode[g] && !cs.empty()) stats_.rows_scanned += cs[g].rows;
  return cs;
}

uint64_t Engine::scan_bytes(const ScanPlan& p, const std::vector<uint32_t>& used) {
  uint64_t b = 0;
  for (uint32_t s : used) {
    BaseCol& bc = basecol(p.src, p.slots[s]);
    for (uint32_t g = 0; g < p.src->segCount; g++) {
      if (!p.mode[g]) continue;
      const SegMeta& m = bc.segs[g].m;
      b += (uint64_t)m.rec_count * (bc.res_bits.size() > g ? bc.res_bits[g] / 8 : m.bits / 8);
    }
  }
  return b;
}

}  // namespace alk
