// Host restatement of the three moderngpu 2.x primitives the reference calls, for
// building the reference's operators on the CPU (moderngpu is not vendored with the
// reference, so its version is unpinned). Test infrastructure only.
//
//   inner_join(a, na, b, nb, less, ctx)   operators.cu:1239  sorted a, sorted b ->
//       every (i, j) with a[i] == b[j], ordered by i then j: lower_bound/upper_bound
//       of a[i] in b, then expansion of [lo, hi). This is the sort-merge form the
//       published moderngpu algorithm computes (sorted search + load-balancing search).
//   segreduce(in, n, seg, nseg, out, op, init, ctx)   select.cu:499-672
//       out[s] = fold of in[seg[s] .. seg[s+1]) (the last segment ends at n);
//       an empty segment yields init.
//   reduce(in, n, out, op, ctx)   select.cu:549-675
//       out[0] = fold of in[0 .. n).
#pragma once
#include <algorithm>
#include <cstddef>
#include <utility>
#include <vector>

namespace mgpu {

struct standard_context_t {
  standard_context_t() {}
  explicit standard_context_t(bool) {}
};

template <class T> struct plus_t { T operator()(T a, T b) const { return a + b; } };
template <class T> struct minimum_t { T operator()(T a, T b) const { return b < a ? b : a; } };
template <class T> struct maximum_t { T operator()(T a, T b) const { return a < b ? b : a; } };
template <class T> struct less_t { bool operator()(T a, T b) const { return a < b; } };

// A device allocation in moderngpu; host memory here (Thrust's host device system).
template <class T> class mem_t {
 public:
  mem_t() {}
  explicit mem_t(size_t n, standard_context_t&) : v_(n) {}
  mem_t(mem_t&& o) noexcept : v_(std::move(o.v_)) {}
  mem_t& operator=(mem_t&& o) noexcept { v_ = std::move(o.v_); return *this; }
  mem_t(const mem_t&) = delete;
  mem_t& operator=(const mem_t&) = delete;
  size_t size() const { return v_.size(); }
  T* data() { return v_.data(); }
  const T* data() const { return v_.data(); }
  std::vector<T>& vec() { return v_; }
 private:
  std::vector<T> v_;
};

template <class AIt, class BIt, class Comp>
mem_t<int2> inner_join(AIt a, int na, BIt b, int nb, Comp comp, standard_context_t&) {
  mem_t<int2> out;
  for (int i = 0; i < na; i++) {
    BIt lo = std::lower_bound(b, b + nb, a[i], comp);
    BIt hi = std::upper_bound(b, b + nb, a[i], comp);
    for (BIt j = lo; j != hi; ++j) out.vec().push_back(make_int2(i, (int)(j - b)));
  }
  return out;
}

template <class InIt, class SegIt, class OutIt, class Op, class T>
void segreduce(InIt in, int n, SegIt seg, int nseg, OutIt out, Op op, T init, standard_context_t&) {
  for (int s = 0; s < nseg; s++) {
    int lo = seg[s];
    int hi = s + 1 < nseg ? (int)seg[s + 1] : n;
    if (lo >= hi) { out[s] = init; continue; }
    T acc = in[lo];
    for (int k = lo + 1; k < hi; k++) acc = op(acc, in[k]);
    out[s] = acc;
  }
}

template <class InIt, class OutIt, class Op>
void reduce(InIt in, int n, OutIt out, Op op, standard_context_t&) {
  typedef typename std::decay<decltype(in[0])>::type T;
  T acc = n > 0 ? (T)in[0] : T();
  for (int k = 1; k < n; k++) acc = op(acc, in[k]);
  out[0] = acc;
}

}  // namespace mgpu
