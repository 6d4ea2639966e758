// The engine side of the learned cardinality estimator: per (stage, segment) features
// from the zone maps, 16-bin histograms of the predicate columns and the predicate
// constants; records of exact counts (alk_card_count) for training; and the estimates
// that size a fused stage's survivor list and hash table on a query's first run. The
// estimator only sizes buffers: a size that proves too small makes the query run again
// with the exact counts, so results never depend on it.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <random>

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
DevBufP mkbuf(size_t bytes, cudaStream_t s) { return std::make_shared<DevBuf>(bytes, s); }

constexpr int kF = ALK_CARD_FEATURES;
constexpr int kO = ALK_CARD_OUTPUTS;

// Fraction of a segment's values v with v OP x under a histogram of 16 equal bins over
// [lo, hi], values spread evenly inside a bin (the classical estimate).
double hist_fraction(const float* h, int64_t lo, int64_t hi, uint32_t op, double x) {
  const double w = (double)hi - (double)lo + 1.0;
  const double bw = w / 16.0;
  auto below = [&](double t) {  // fraction of values < t
    double f = 0;
    for (int b = 0; b < 16; b++) {
      const double b0 = (double)lo + b * bw, b1 = b0 + bw;
      if (t >= b1) f += h[b];
      else if (t > b0) f += h[b] * (t - b0) / bw;
    }
    return std::min(1.0, std::max(0.0, f));
  };
  // integer values: v < x for the smallest integer >= x, v <= x for floor(x)
  const double lt = below(std::ceil(x)), le = below(std::floor(x) + 1.0);
  const double eq = std::max(0.0, le - below(std::floor(x)));
  switch (op) {
    case ALK_OP_LT: return lt;
    case ALK_OP_LE: return le;
    case ALK_OP_GT: return 1.0 - le;
    case ALK_OP_GE: return 1.0 - lt;
    case ALK_OP_EQ: return std::floor(x) == x ? eq : 0.0;
    default: return std::floor(x) == x ? 1.0 - eq : 1.0;
  }
}
}  // namespace

const std::vector<std::array<float, 16>>& Engine::card_hist(const ScanPlan& p, const std::vector<alk_colseg>& cs,
                                                           uint32_t slot) {
  const std::string key = p.src->table + "." + p.slots[slot];
  auto it = card_hist_.find(key);
  const uint32_t nseg = p.src->segCount;
  if (it != card_hist_.end() && it->second.size() == nseg) return it->second;
  BaseCol& bc = basecol(p.src, p.slots[slot]);
  read_headers(p.src, p.slots[slot], bc);
  std::vector<std::array<float, 16>> out(nseg);
  auto d = mkbuf((size_t)nseg * 64, stream_);
  std::vector<uint32_t> h((size_t)nseg * 16, 0);
  for (uint32_t g = 0; g < nseg; g++) {
    const SegMeta& m = bc.segs[g].m;
    check(alk_card_hist16(&cs[(size_t)slot * nseg + g], std::min(m.lower, m.upper), std::max(m.lower, m.upper),
                          d->as<uint32_t>() + 16 * g, (alk_stream)stream_),
          "histogram");
  }
  ck(cudaMemcpyAsync(h.data(), d->as<void>(), (size_t)nseg * 64, cudaMemcpyDeviceToHost, stream_), "d2h");
  ck(cudaStreamSynchronize(stream_), "sync");
  for (uint32_t g = 0; g < nseg; g++) {
    double tot = 0;
    for (int b = 0; b < 16; b++) tot += h[16 * g + b];
    for (int b = 0; b < 16; b++) out[g][b] = tot > 0 ? (float)(h[16 * g + b] / tot) : 0.f;
  }
  return card_hist_[key] = std::move(out);
}

// One feature row per scanned segment (segments with mode != 0, in order):
//   0-2  stage kind (build, build probing another table, probe-aggregate)
//   3    log2(rows + 1) / 32        4  zone maps pass the whole segment
//   5    probes a table              6  fraction of the probed key range present
//   7    share of the segment's probe-key range inside the probed table's key range
//   8    the probed table's first constant placed within this segment's first conjunct
//        column range (relates two filters on columns of one domain, such as dates)
//   9    classical filter estimate (product over conjuncts)
//   10   classical probe estimate   11  classical distinct estimate   12 key counted
//   13-36 first conjunct: present, op one-hot (6), constant position within the
//         segment's [min, max], 16-bin histogram of the column over that range
//   37-52 second conjunct: the same with the histogram's bins summed in pairs (8)
//   53-60 first conjunct of the probed table's filter: present, op one-hot, constant
//         position within that column's [min, max] over all segments
//   61-62 the two conjuncts' classical estimates   63 ln(classical filter x probe) / 16
std::vector<float> Engine::card_features(const CardStage& st) {
  const ScanPlan& p = *st.p;
  const std::vector<alk_colseg>& cs = *st.cs;
  const uint32_t nseg = p.src->segCount;
  std::vector<CardConj> cj;
  const bool conj = !p.has_pred || program_conjuncts(p.pred, cj);
  std::vector<float> f;
  std::vector<const std::vector<std::array<float, 16>>*> hist(cj.size(), nullptr);
  for (size_t c = 0; c < cj.size() && c < 2; c++) hist[c] = &card_hist(p, cs, cj[c].slot);
  BaseCol* pk = st.probe_slot >= 0 ? &basecol(p.src, p.slots[st.probe_slot]) : nullptr;
  BaseCol* kk = st.key_slot >= 0 ? &basecol(p.src, p.slots[st.key_slot]) : nullptr;
  if (pk) read_headers(p.src, p.slots[st.probe_slot], *pk);
  if (kk) read_headers(p.src, p.slots[st.key_slot], *kk);
  // a comparison v * mul OP k as v OP' threshold
  auto normal = [](const CardConj& c, double mid, uint32_t* op) {
    *op = c.op;
    if (c.mul == 0) return mid;
    if (c.mul < 0)
      *op = c.op == ALK_OP_LT ? ALK_OP_GT : c.op == ALK_OP_GT ? ALK_OP_LT
          : c.op == ALK_OP_LE ? ALK_OP_GE : c.op == ALK_OP_GE ? ALK_OP_LE : c.op;
    return (double)c.k / (double)c.mul;
  };
  // the probed table's first conjunct, placed within its column's range over all segments
  float up[8] = {0};
  bool has_up = false;
  double up_thr = 0;
  if (st.up && st.up->has_pred) {
    std::vector<CardConj> ucj;
    if (program_conjuncts(st.up->pred, ucj) && !ucj.empty()) {
      const std::string& col = st.up->slots[ucj[0].slot];
      BaseCol& bc = basecol(st.up->src, col);
      read_headers(st.up->src, col, bc);
      double lo = 1e300, hi = -1e300;
      for (auto& sg : bc.segs) {
        lo = std::min(lo, (double)std::min(sg.m.lower, sg.m.upper));
        hi = std::max(hi, (double)std::max(sg.m.lower, sg.m.upper));
      }
      uint32_t op;
      const double thr = normal(ucj[0], 0.5 * (lo + hi), &op);
      has_up = true;
      up_thr = thr;
      up[0] = 1.f;
      if (op >= ALK_OP_LT && op <= ALK_OP_NE) up[1 + (op - ALK_OP_LT)] = 1.f;
      if (hi >= lo) up[7] = (float)std::min(1.5, std::max(-0.5, (thr - lo) / (hi - lo + 1.0)));
    }
  }
  for (uint32_t g = 0; g < nseg; g++) {
    if (!p.mode[g]) continue;
    float x[kF] = {0};
    const uint64_t rows = cs[g].rows;
    x[st.kind] = 1.f;
    x[3] = (float)(std::log2((double)rows + 1.0) / 32.0);
    x[4] = p.mode[g] == 1 ? 1.f : 0.f;
    double est_f = 1.0;
    if (conj && p.mode[g] != 1) {
      for (size_t c = 0; c < cj.size(); c++) {
        if (c >= 2) {
          est_f *= 0.5;  // beyond the two described conjuncts
          continue;
        }
        const SegMeta& m = basecol(p.src, p.slots[cj[c].slot]).segs[g].m;
        const int64_t lo = std::min(m.lower, m.upper), hi = std::max(m.lower, m.upper);
        uint32_t op;
        const double thr = normal(cj[c], 0.5 * ((double)lo + (double)hi), &op);
        const float* h = (*hist[c])[g].data();
        const double e = hist_fraction(h, lo, hi, op, thr);
        const int b = c == 0 ? 13 : 37;
        x[b] = 1.f;
        if (op >= ALK_OP_LT && op <= ALK_OP_NE) x[b + 1 + (op - ALK_OP_LT)] = 1.f;
        const double t = (thr - (double)lo) / ((double)hi - (double)lo + 1.0);
        x[b + 7] = (float)std::min(1.5, std::max(-0.5, t));
        if (c == 0 && has_up)
          x[8] = (float)std::min(1.5, std::max(-0.5, (up_thr - (double)lo) / ((double)hi - (double)lo + 1.0)));
        if (c == 0)
          for (int k = 0; k < 16; k++) x[b + 8 + k] = h[k];
        else
          for (int k = 0; k < 8; k++) x[b + 8 + k] = h[2 * k] + h[2 * k + 1];
        x[61 + c] = (float)e;
        est_f *= e;
      }
    } else if (!conj) {
      est_f = 0.5;  // a predicate of another form: no classical estimate
    }
    x[9] = (float)est_f;
    double est_j = 1.0;
    if (pk) {
      x[5] = 1.f;
      x[6] = (float)st.probe_fill;
      const SegMeta& m = pk->segs[g].m;
      const double lo = (double)std::min(m.lower, m.upper), hi = (double)std::max(m.lower, m.upper);
      const double ilo = std::max(lo, (double)st.probe_range.first), ihi = std::min(hi, (double)st.probe_range.second);
      const double ov = ihi >= ilo ? (ihi - ilo + 1.0) / (hi - lo + 1.0) : 0.0;
      x[7] = (float)ov;
      est_j = st.probe_fill * ov;
    }
    x[10] = (float)est_j;
    if (kk) {
      const SegMeta& m = kk->segs[g].m;
      const double span = std::fabs((double)m.upper - (double)m.lower) + 1.0;
      const double surv = (double)rows * est_f * est_j + 1.0;
      x[11] = (float)std::min(1.0, span / surv);
      x[12] = 1.f;
    } else {
      x[11] = 1.f;
    }
    for (int k = 0; k < 8; k++) x[53 + k] = up[k];
    x[63] = (float)(std::log(std::max(1e-9, est_f * est_j)) / 16.0);
    f.insert(f.end(), x, x + kF);
  }
  return f;
}

void Engine::card_record(const CardStage& st) {
  const ScanPlan& p = *st.p;
  const uint32_t nseg = p.src->segCount;
  std::vector<uint64_t> cnt((size_t)nseg * 3, 0);
  check(alk_card_count(st.cs->data(), (uint32_t)p.slots.size(), nseg, p.mode.data(), p.has_pred ? &p.pred : nullptr,
                       st.probe, st.probe_slot, st.key_slot, st.key_range.first, st.key_range.second, cnt.data(),
                       (alk_stream)stream_),
        "exact counts");
  std::vector<float> f = card_features(st);
  size_t r = 0;
  for (uint32_t g = 0; g < nseg; g++) {
    if (!p.mode[g]) continue;
    const float* x = f.data() + r * kF;
    r++;
    const double rows = (double)(*st.cs)[g].rows;
    if (rows == 0) continue;
    const double pass = (double)cnt[3 * g], join = (double)cnt[3 * g + 1];
    const uint64_t nd = cnt[3 * g + 2];
    float y[kO], m[kO];
    y[0] = (float)std::log(std::max(pass, 0.5) / rows);
    m[0] = 1.f;
    y[1] = (float)std::log(std::max(join, 0.5) / std::max(pass, 1.0));
    m[1] = st.probe && pass > 0 ? 1.f : 0.f;
    y[2] = nd == ~0ull ? 0.f : (float)std::log(std::max((double)nd, 0.5) / std::max(join, 1.0));
    m[2] = nd != ~0ull && join > 0 ? 1.f : 0.f;
    card_x_.insert(card_x_.end(), x, x + kF);
    card_y_.insert(card_y_.end(), y, y + kO);
    card_m_.insert(card_m_.end(), m, m + kO);
  }
}

bool Engine::card_estimate(const CardStage& st, uint64_t* hits, uint64_t* keys) {
  if (!card_use_ || !card_mlp_) return false;
  const ScanPlan& p = *st.p;
  std::vector<float> f = card_features(st);
  const size_t n = f.size() / kF;
  double h = 0, k = 0;
  if (n) {
    std::vector<float> y(n * kO);
    card_forward(f.data(), n, y.data());
    size_t r = 0;
    for (uint32_t g = 0; g < p.src->segCount; g++) {
      if (!p.mode[g]) continue;
      const float* yy = y.data() + kO * r++;
      const double rows = (double)(*st.cs)[g].rows;
      const double pass = rows * std::exp(std::min(0.f, yy[0]));
      const double join = st.probe ? pass * std::exp(std::min(0.f, yy[1])) : pass;
      // the scan drops non-members only where the probed table has a key bitmap (a key
      // range of at most 2^29 values); otherwise every filter survivor is a hit
      const bool bitmap = st.probe_range.second >= st.probe_range.first &&
                          (uint64_t)st.probe_range.second - (uint64_t)st.probe_range.first < (1ull << 29);
      h += st.probe && !bitmap ? pass : join;
      k += st.key_slot >= 0 ? join * std::exp(std::min(0.f, yy[2])) : join;
    }
  }
  *hits = (uint64_t)std::ceil(h);
  *keys = (uint64_t)std::ceil(k);
  stats_.card_estimates++;
  return true;
}

void Engine::card_forward(const float* h_x, uint64_t n, float* h_y) {
  if (!card_mlp_) throw EngineError(ALK_ERR_ARG, "the cardinality estimator is not trained");
  if (n == 0) return;
  auto dx = mkbuf(n * kF * 4, stream_);
  auto dy = mkbuf(n * kO * 4, stream_);
  ck(cudaMemcpyAsync(dx->as<void>(), h_x, n * kF * 4, cudaMemcpyHostToDevice, stream_), "h2d");
  check(alk_mlp_forward(card_mlp_, dx->as<float>(), n, dy->as<float>(), (alk_stream)stream_), "estimator");
  ck(cudaMemcpyAsync(h_y, dy->as<void>(), n * kO * 4, cudaMemcpyDeviceToHost, stream_), "d2h");
  ck(cudaStreamSynchronize(stream_), "sync");
}

int Engine::card_mode(bool record, bool use) {
  card_record_ = record;
  card_use_ = use;
  return ALK_OK;
}

uint64_t Engine::card_records(float* x, float* y, float* m, uint64_t cap) const {
  const uint64_t n = card_y_.size() / kO;
  const uint64_t c = std::min(cap, n);
  if (x) std::memcpy(x, card_x_.data(), c * kF * 4);
  if (y) std::memcpy(y, card_y_.data(), c * kO * 4);
  if (m) std::memcpy(m, card_m_.data(), c * kO * 4);
  return n;
}

int Engine::card_train(uint64_t first, uint64_t count, uint32_t epochs, uint32_t batch, float lr, uint64_t seed,
                       float* loss) {
  const uint64_t n = card_y_.size() / kO;
  if (first > n || count > n - first || count == 0) return ALK_ERR_ARG;
  try {
    if (!card_mlp_) check(alk_mlp_create(seed, &card_mlp_, (alk_stream)stream_), "estimator");
    std::vector<uint64_t> ord(count);
    std::iota(ord.begin(), ord.end(), first);
    std::mt19937_64 rng(seed);
    std::shuffle(ord.begin(), ord.end(), rng);
    std::vector<float> x(count * kF), y(count * kO), m(count * kO);
    for (uint64_t i = 0; i < count; i++) {
      std::memcpy(&x[i * kF], &card_x_[ord[i] * kF], kF * 4);
      std::memcpy(&y[i * kO], &card_y_[ord[i] * kO], kO * 4);
      std::memcpy(&m[i * kO], &card_m_[ord[i] * kO], kO * 4);
    }
    auto dx = mkbuf(x.size() * 4, stream_), dy = mkbuf(y.size() * 4, stream_), dm = mkbuf(m.size() * 4, stream_);
    ck(cudaMemcpyAsync(dx->as<void>(), x.data(), x.size() * 4, cudaMemcpyHostToDevice, stream_), "h2d");
    ck(cudaMemcpyAsync(dy->as<void>(), y.data(), y.size() * 4, cudaMemcpyHostToDevice, stream_), "h2d");
    ck(cudaMemcpyAsync(dm->as<void>(), m.data(), m.size() * 4, cudaMemcpyHostToDevice, stream_), "h2d");
    float l = 0;
    check(alk_mlp_train(card_mlp_, dx->as<float>(), dy->as<float>(), dm->as<float>(), count, epochs, batch, lr, &l,
                        (alk_stream)stream_),
          "training");
    if (loss) *loss = l;
  } catch (const EngineError& e) {
    err_ = e.what();
    return e.code;
  }
  return ALK_OK;
}

// The trained network as a file: "ALKMLP1\0", the parameter count (u32), then the FP32
// master parameters.
int Engine::card_save(const std::string& path) {
  if (!card_mlp_) {
    err_ = "the cardinality estimator is not trained";
    return ALK_ERR_ARG;
  }
  const uint32_t n = alk_mlp_param_count();
  std::vector<float> p(n);
  int rc = alk_mlp_params(card_mlp_, p.data(), nullptr, (alk_stream)stream_);
  if (rc) return rc;
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err_ = "cannot write " + path;
    return ALK_ERR_IO;
  }
  const char magic[8] = {'A', 'L', 'K', 'M', 'L', 'P', '1', 0};
  bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(&n, 4, 1, f) == 1 && std::fwrite(p.data(), 4, n, f) == n;
  ok = std::fclose(f) == 0 && ok;
  if (!ok) {
    err_ = "cannot write " + path;
    return ALK_ERR_IO;
  }
  return ALK_OK;
}

int Engine::card_load(const std::string& path) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) {
    err_ = "cannot read " + path;
    return ALK_ERR_IO;
  }
  char magic[8] = {0};
  uint32_t n = 0;
  std::vector<float> p;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "ALKMLP1", 8) == 0 &&
            std::fread(&n, 4, 1, f) == 1 && n == alk_mlp_param_count();
  if (ok) {
    p.resize(n);
    ok = std::fread(p.data(), 4, n, f) == n;
  }
  std::fclose(f);
  if (!ok) {
    err_ = path + ": not an estimator file of this network";
    return ALK_ERR_IO;
  }
  if (!card_mlp_) {
    int rc = alk_mlp_create(1, &card_mlp_, (alk_stream)stream_);
    if (rc) return rc;
  }
  return alk_mlp_set_params(card_mlp_, p.data(), (alk_stream)stream_);
}

void Engine::card_forget() {
  card_feedback_.clear();
  fused_graphs_.clear();
  fused_seen_.clear();
}

}  // namespace alk
