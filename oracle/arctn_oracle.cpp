// ArcTN executor oracle -- TEST INFRASTRUCTURE ONLY.
//
// A literal CPU restatement of the reference ArcTN numerical contraction path,
// used as the checker for the B200 executor and as the timed CPU baseline
// ("port" kind).  Nothing in the product (arctn_b200/) may link, import or call
// this file; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// leg do.
//
// Each function cites the reference source it restates (paths relative to the
// ArcTN repository):
//   network validation          src/network.rs:171-229
//   path simulation / metrics   src/path.rs:32-42, 239-434
//   compiled plan               src/compiled.rs:254-366, 445-602
//   execution (+ strip)         src/compiled.rs:383-441, src/contract.rs:102-181
//   tensor kernels              src/tensor.rs:453-669
//   sliced execution            src/slice.rs:881-905, 960-1173
//   naive einsum                src/naive.rs:10-76
//   greedy path                 src/paths/greedy.rs:61-320
//   slice selection             src/slice.rs:28-97, 139-150, 209-288, 548-589
//
// The reference's GEMM backend (crate matrixmultiply 0.3.10, not vendored) is
// restated as a plain row-major triple loop accumulating over k in ascending
// order; the reference pins GEMM values by tolerance only, never bitwise.
//
// Parity pinning: the reference is Rust and cannot be built in this image (no
// cargo/rustc, crates not vendored).  This restatement is pinned by the
// reference's own known-answer tests, re-stated in tests/test_oracle_golden.py.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <queue>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>
#include <atomic>
#include <thread>
#include <tuple>

namespace oracle {

using Leg = uint32_t;
using usize = uint64_t;

struct Err : std::runtime_error {
  explicit Err(const std::string& s) : std::runtime_error(s) {}
};

// ---------------------------------------------------------------- scalars
// num-complex arithmetic uses the textbook product; std::complex may route
// through __muldc3, so a plain struct keeps the same formula.
template <class R>
struct Cx {
  R re, im;
};
template <class R> inline Cx<R> operator+(Cx<R> a, Cx<R> b) { return {a.re + b.re, a.im + b.im}; }
template <class R> inline Cx<R> operator*(Cx<R> a, Cx<R> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <class R> inline Cx<R>& operator+=(Cx<R>& a, Cx<R> b) { a.re += b.re; a.im += b.im; return a; }

template <class T> struct S;
template <> struct S<float> {
  static float zero() { return 0.f; }
  static float one() { return 1.f; }
  static double mag(float v) { return std::fabs((double)v); }
  static float scale(float v, double inv) { return (float)((double)v * inv); }
};
template <> struct S<double> {
  static double zero() { return 0.0; }
  static double one() { return 1.0; }
  static double mag(double v) { return std::fabs(v); }
  static double scale(double v, double inv) { return v * inv; }
};
template <> struct S<Cx<float>> {
  static Cx<float> zero() { return {0.f, 0.f}; }
  static Cx<float> one() { return {1.f, 0.f}; }
  static double mag(Cx<float> v) { return std::hypot((double)v.re, (double)v.im); }
  // T::from_real(1/f) then complex multiply, as src/compiled.rs:425-428.
  static Cx<float> scale(Cx<float> v, double inv) { return v * Cx<float>{(float)inv, 0.f}; }
};
template <> struct S<Cx<double>> {
  static Cx<double> zero() { return {0.0, 0.0}; }
  static Cx<double> one() { return {1.0, 0.0}; }
  static double mag(Cx<double> v) { return std::hypot(v.re, v.im); }
  static Cx<double> scale(Cx<double> v, double inv) { return v * Cx<double>{inv, 0.0}; }
};

// ---------------------------------------------------------------- network
struct Net {
  std::vector<std::vector<Leg>> inputs;
  std::vector<Leg> output;
  std::map<Leg, usize> size;  // ordered: deterministic iteration

  usize dim(Leg l) const {
    auto it = size.find(l);
    if (it == size.end()) throw Err("leg " + std::to_string(l) + " has no size_dict dimension");
    return it->second;
  }
  double log2_dim(Leg l) const { return std::log2((double)dim(l)); }
  size_t n() const { return inputs.size(); }
};

static usize checked_numel(const std::vector<usize>& shape) {
  // src/tensor.rs:11-22
  unsigned __int128 n = 1;
  for (size_t a = 0; a < shape.size(); ++a) {
    if (shape[a] == 0) throw Err("shape axis " + std::to_string(a) + " is 0");
    n *= shape[a];
    if (n > (unsigned __int128)UINT64_MAX) throw Err("shape element count overflows usize");
  }
  return (usize)n;
}

// src/network.rs:171-229
static void validate(const Net& net) {
  if (net.inputs.empty()) throw Err("TensorNetwork needs at least one input tensor");
  const usize max_gemm = (usize)INT64_MAX;
  for (auto& kv : net.size) {
    if (kv.second == 0) throw Err("leg " + std::to_string(kv.first) + " has dimension 0");
    if (kv.second > max_gemm) throw Err("leg dimension exceeds isize stride range");
  }
  std::set<Leg> held;
  for (size_t i = 0; i < net.inputs.size(); ++i) {
    std::map<Leg, int> counts;
    std::vector<usize> shape;
    for (Leg l : net.inputs[i]) {
      usize d = net.dim(l);
      counts[l]++;
      held.insert(l);
      shape.push_back(d);
    }
    for (auto& c : counts)
      if (c.second > 2) throw Err("leg appears more than twice in one input tensor");
    checked_numel(shape);
  }
  std::set<Leg> seen;
  std::vector<usize> oshape;
  for (Leg l : net.output) {
    if (!seen.insert(l).second) throw Err("output contains a repeated leg");
    if (!held.count(l)) throw Err("output leg not held by any input tensor");
    oshape.push_back(net.dim(l));
  }
  checked_numel(oshape);
  for (auto& kv : net.size)
    if (!held.count(kv.first)) throw Err("size_dict leg " + std::to_string(kv.first) + " is not used by any input tensor");
}

static std::vector<Leg> sorted_dedup(std::vector<Leg> v) {
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  return v;
}

// ---------------------------------------------------------------- path metrics
// src/path.rs:32-42
static double logaddexp2(double a, double b) {
  if (a == -INFINITY) return b;
  if (b == -INFINITY) return a;
  double hi = a > b ? a : b, lo = a > b ? b : a;
  return hi + std::log2(1.0 + std::exp2(lo - hi));
}

static std::vector<Leg> legs_union(const std::vector<Leg>& a, const std::vector<Leg>& b) {
  std::vector<Leg> out;
  size_t i = 0, j = 0;
  while (i < a.size() && j < b.size()) {
    if (a[i] < b[j]) out.push_back(a[i++]);
    else if (a[i] > b[j]) out.push_back(b[j++]);
    else { out.push_back(a[i]); ++i; ++j; }
  }
  while (i < a.size()) out.push_back(a[i++]);
  while (j < b.size()) out.push_back(b[j++]);
  return out;
}

using Path = std::vector<std::pair<usize, usize>>;

struct Stats {
  double log10_flops, log2_max_size, log2_max_contraction_size, log2_total_size, log2_read_write, log2_peak_size;
};

static double sum_log2(const Net& net, const std::vector<Leg>& legs) {
  double s = 0.0;
  for (Leg l : legs) s += net.log2_dim(l);
  return s;
}

// src/path.rs:239-434
static Stats simulate_path_full(const Net& net, const Path& path, std::vector<std::vector<Leg>>* step_legs_out) {
  validate(net);
  size_t n = net.n();
  size_t n_slots = n + path.size();
  std::vector<std::vector<Leg>> legs;
  std::vector<bool> live;
  std::map<Leg, usize> refcount;
  std::set<Leg> in_output(net.output.begin(), net.output.end());
  {
    auto od = net.output;
    std::sort(od.begin(), od.end());
    for (size_t i = 1; i < od.size(); ++i)
      if (od[i] == od[i - 1]) throw Err("output contains a repeated leg");
  }
  std::map<Leg, usize> appearances;
  for (auto& t : net.inputs)
    for (Leg l : t) appearances[l]++;
  for (Leg l : net.output) appearances[l]++;
  std::vector<double> contraction_slot_log2, read_write_slot_log2;
  for (auto& t : net.inputs) {
    auto d = t;
    std::sort(d.begin(), d.end());
    double leaf = 0.0;
    size_t i = 0;
    while (i < d.size()) {
      Leg l = d[i];
      size_t j = i + 1;
      while (j < d.size() && d[j] == l) ++j;
      if (j - i != appearances[l]) leaf += net.log2_dim(l);
      i = j;
    }
    d.erase(std::unique(d.begin(), d.end()), d.end());
    for (Leg l : d) refcount[l]++;
    legs.push_back(d);
    live.push_back(true);
    contraction_slot_log2.push_back(leaf);
    read_write_slot_log2.push_back(sum_log2(net, t));
  }
  for (auto& t : net.inputs) {
    std::map<Leg, int> c;
    for (Leg l : t) c[l]++;
    for (auto& kv : c)
      if (kv.second > 2) throw Err("leg appears more than twice in one tensor");
  }
  double log2_flops = -INFINITY;
  double log2_max_size = (n == 1) ? sum_log2(net, net.output) : 0.0;
  double log2_max_contraction_size = 0.0, log2_total_size = -INFINITY, log2_rw = -INFINITY;
  std::vector<double> slot_size;
  for (auto& t : net.inputs) slot_size.push_back(std::exp2(sum_log2(net, t)));
  double alive_sum = 0.0;
  for (double v : slot_size) alive_sum += v;
  double peak = alive_sum;
  std::vector<std::vector<Leg>> step_legs;
  for (size_t step = 0; step < path.size(); ++step) {
    usize a = path[step].first, b = path[step].second;
    if (a == b) throw Err("step " + std::to_string(step) + " contracts a tensor with itself");
    if (a >= legs.size() || !live[a] || b >= legs.size() || !live[b])
      throw Err("step " + std::to_string(step) + " references an invalid or consumed tensor");
    auto la = legs[a], lb = legs[b];
    live[a] = live[b] = false;
    auto uni = legs_union(la, lb);
    log2_flops = logaddexp2(log2_flops, sum_log2(net, uni));
    for (Leg l : la) refcount[l]--;
    for (Leg l : lb) refcount[l]--;
    std::vector<Leg> result;
    for (Leg l : uni)
      if (refcount[l] > 0 || in_output.count(l)) result.push_back(l);
    for (Leg l : result) refcount[l]++;
    double size_log2 = sum_log2(net, result);
    log2_max_size = std::max(log2_max_size, size_log2);
    double c2 = logaddexp2(logaddexp2(contraction_slot_log2[a], contraction_slot_log2[b]), size_log2);
    log2_max_contraction_size = std::max(log2_max_contraction_size, c2);
    double rw = logaddexp2(logaddexp2(read_write_slot_log2[a], read_write_slot_log2[b]), size_log2);
    log2_rw = logaddexp2(log2_rw, rw);
    contraction_slot_log2.push_back(size_log2);
    read_write_slot_log2.push_back(size_log2);
    log2_total_size = logaddexp2(log2_total_size, size_log2);
    double rsize = std::exp2(size_log2);
    peak = std::max(peak, alive_sum + rsize);
    alive_sum += rsize - slot_size[a] - slot_size[b];
    slot_size.push_back(rsize);
    step_legs.push_back(result);
    legs.push_back(result);
    live.push_back(true);
  }
  size_t alive = 0, which = 0;
  for (size_t i = 0; i < n_slots; ++i)
    if (live[i]) { ++alive; which = i; }
  if (alive != 1) throw Err("incomplete path: " + std::to_string(alive) + " tensors remain");
  auto fin = sorted_dedup(legs[which]);
  auto out = sorted_dedup(net.output);
  if (path.empty()) {
    for (Leg l : out)
      if (!std::binary_search(fin.begin(), fin.end(), l)) throw Err("final legs do not contain every output leg");
  } else if (fin != out) {
    throw Err("final legs do not match output");
  }
  if (step_legs_out) *step_legs_out = step_legs;
  const double LOG10_2 = 0.301029995663981195213738894724493027;
  return Stats{log2_flops * LOG10_2, log2_max_size, log2_max_contraction_size, log2_total_size, log2_rw, std::log2(peak)};
}

// ---------------------------------------------------------------- compiled plan
struct Prep {
  std::vector<usize> input_shape;
  std::vector<std::tuple<usize, usize, bool>> traces;
  std::vector<Leg> legs;
  std::vector<usize> shape;
};
struct Step {
  usize li, ri, out;
  std::vector<Leg> left_legs, right_legs, result_legs;
  std::vector<usize> left_shape, right_shape, result_shape;
  std::vector<usize> sum_a, sum_b, a_perm, b_perm;
  usize bt, m, k, n;
};
struct Fin {
  usize slot;
  std::vector<Leg> input_legs;
  std::vector<usize> input_shape, sum, perm, output_shape;
};
struct Plan {
  usize n_inputs;
  std::vector<Prep> preps;
  std::vector<Step> steps;
  Fin fin;
  double log10_flops, log2_peak_size;
};

static size_t pos_of(const std::vector<Leg>& v, Leg l) {
  for (size_t i = 0; i < v.size(); ++i)
    if (v[i] == l) return i;
  throw Err("internal: leg not found");
}

static usize dprod(const Net& net, const std::vector<Leg>& legs) {
  unsigned __int128 p = 1;
  for (Leg l : legs) {
    p *= net.dim(l);
    if (p > (unsigned __int128)UINT64_MAX) throw Err("GEMM dimension product overflows usize");
  }
  return (usize)p;
}

// src/contract.rs:49-100
static void checked_batch_gemm_geometry(usize bt, usize m, usize k, usize n) {
  const unsigned __int128 mx = (unsigned __int128)INT64_MAX;
  usize v[4] = {bt, m, k, n};
  for (usize x : v) {
    if (x == 0) throw Err("GEMM dimension is 0");
    if (x > (usize)INT64_MAX) throw Err("GEMM dimension exceeds isize stride range");
  }
  unsigned __int128 ab = (unsigned __int128)m * k, bb = (unsigned __int128)k * n, cb = (unsigned __int128)m * n;
  unsigned __int128 vals[6] = {ab, bb, cb, ab * bt, bb * bt, cb * bt};
  for (auto x : vals)
    if (x > mx) throw Err("GEMM element offset exceeds isize range");
}

// src/compiled.rs:445-478
static std::vector<std::tuple<usize, usize, bool>> plan_traces(std::vector<Leg>& legs, const std::map<Leg, usize>& refcount,
                                                               const std::set<Leg>& in_output) {
  std::vector<std::tuple<usize, usize, bool>> ops;
  for (;;) {
    bool found = false;
    size_t di = 0, dj = 0;
    for (size_t i = 0; i < legs.size() && !found; ++i)
      for (size_t j = i + 1; j < legs.size(); ++j)
        if (legs[i] == legs[j]) { di = i; dj = j; found = true; break; }
    if (!found) return ops;
    Leg l = legs[di];
    if (std::count(legs.begin(), legs.end(), l) > 2) throw Err("leg appears more than twice in one tensor");
    bool external = refcount.at(l) > 1 || in_output.count(l);
    if (external) {
      ops.emplace_back(di, dj, true);
      legs.erase(legs.begin() + dj);
    } else {
      ops.emplace_back(di, dj, false);
      legs.erase(legs.begin() + dj);
      legs.erase(legs.begin() + di);
    }
  }
}

// src/compiled.rs:481-602
static Step plan_pairwise(const Net& net, const std::vector<Leg>& la, const std::vector<Leg>& lb, usize li, usize ri, usize out,
                          const std::map<Leg, usize>& refcount, const std::set<Leg>& in_output) {
  auto keep = [&](Leg l) { return refcount.at(l) > 0 || in_output.count(l) > 0; };
  std::set<Leg> set_a(la.begin(), la.end()), set_b(lb.begin(), lb.end());
  std::vector<Leg> batch, con, free_a, sum_a_legs, free_b, sum_b_legs;
  for (Leg l : la) {
    if (set_b.count(l)) (keep(l) ? batch : con).push_back(l);
    else (keep(l) ? free_a : sum_a_legs).push_back(l);
  }
  for (Leg l : lb)
    if (!set_a.count(l)) (keep(l) ? free_b : sum_b_legs).push_back(l);
  Step st;
  std::vector<Leg> la_work = la, lb_work = lb;
  for (Leg l : sum_a_legs) {
    size_t ax = pos_of(la_work, l);
    st.sum_a.push_back(ax);
    la_work.erase(la_work.begin() + ax);
  }
  for (Leg l : sum_b_legs) {
    size_t ax = pos_of(lb_work, l);
    st.sum_b.push_back(ax);
    lb_work.erase(lb_work.begin() + ax);
  }
  for (auto* grp : {&batch, &free_a, &con})
    for (Leg l : *grp) st.a_perm.push_back(pos_of(la_work, l));
  for (auto* grp : {&batch, &con, &free_b})
    for (Leg l : *grp) st.b_perm.push_back(pos_of(lb_work, l));
  st.bt = dprod(net, batch);
  st.m = dprod(net, free_a);
  st.k = dprod(net, con);
  st.n = dprod(net, free_b);
  checked_batch_gemm_geometry(st.bt, st.m, st.k, st.n);
  for (auto* grp : {&batch, &free_a, &free_b})
    for (Leg l : *grp) st.result_legs.push_back(l);
  for (Leg l : st.result_legs) st.result_shape.push_back(net.dim(l));
  st.li = li;
  st.ri = ri;
  st.out = out;
  st.left_legs = la;
  st.right_legs = lb;
  for (Leg l : la) st.left_shape.push_back(net.dim(l));
  for (Leg l : lb) st.right_shape.push_back(net.dim(l));
  return st;
}

// src/compiled.rs:254-366
static Plan compile(const Net& net, const Path& path) {
  validate(net);
  Stats stats = simulate_path_full(net, path, nullptr);
  size_t n = net.n();
  std::set<Leg> in_output(net.output.begin(), net.output.end());
  std::map<Leg, usize> refcount;
  for (auto& t : net.inputs)
    for (Leg l : sorted_dedup(t)) refcount[l]++;
  std::vector<std::vector<Leg>> slots;
  std::vector<bool> live;
  Plan p;
  p.n_inputs = n;
  for (auto& legs0 : net.inputs) {
    auto legs = legs0;
    Prep pr;
    pr.traces = plan_traces(legs, refcount, in_output);
    for (Leg l : legs0) pr.input_shape.push_back(net.dim(l));
    for (Leg l : legs) pr.shape.push_back(net.dim(l));
    pr.legs = legs;
    p.preps.push_back(pr);
    slots.push_back(legs);
    live.push_back(true);
  }
  for (size_t step = 0; step < path.size(); ++step) {
    usize ia = path[step].first, ib = path[step].second;
    if (ia == ib) throw Err("step contracts a tensor with itself");
    if (ia >= slots.size() || !live[ia] || ib >= slots.size() || !live[ib]) throw Err("step references an invalid tensor");
    auto la = slots[ia], lb = slots[ib];
    live[ia] = live[ib] = false;
    for (Leg l : la) refcount[l]--;
    for (Leg l : lb) refcount[l]--;
    Step st = plan_pairwise(net, la, lb, ia, ib, slots.size(), refcount, in_output);
    for (Leg l : st.result_legs) refcount[l]++;
    slots.push_back(st.result_legs);
    live.push_back(true);
    p.steps.push_back(st);
  }
  size_t alive = 0, which = 0;
  for (size_t i = 0; i < slots.size(); ++i)
    if (live[i]) { ++alive; which = i; }
  if (alive != 1) throw Err("incomplete path");
  auto legs = slots[which];
  p.fin.slot = which;
  p.fin.input_legs = legs;
  for (Leg l : legs) p.fin.input_shape.push_back(net.dim(l));
  size_t i = 0;
  while (i < legs.size()) {
    if (!in_output.count(legs[i])) {
      p.fin.sum.push_back(i);
      legs.erase(legs.begin() + i);
    } else {
      ++i;
    }
  }
  if (sorted_dedup(legs) != sorted_dedup(net.output)) throw Err("final legs do not match output");
  for (Leg l : net.output) p.fin.perm.push_back(pos_of(legs, l));
  for (Leg l : net.output) p.fin.output_shape.push_back(net.dim(l));
  p.log10_flops = stats.log10_flops;
  p.log2_peak_size = stats.log2_peak_size;
  return p;
}

// ---------------------------------------------------------------- tensors
template <class T>
struct Tensor {
  std::vector<usize> shape;
  std::vector<T> data;
};

static std::vector<usize> strides_of(const std::vector<usize>& shape) {
  std::vector<usize> s(shape.size(), 1);
  for (size_t i = shape.size(); i-- > 1;) s[i - 1] = s[i] * shape[i];
  return s;
}

// src/tensor.rs:453-492
template <class T>
static Tensor<T> permute(const Tensor<T>& t, const std::vector<usize>& axes) {
  bool ident = true;
  for (size_t i = 0; i < axes.size(); ++i)
    if (axes[i] != i) ident = false;
  if (ident) return t;
  auto in_s = strides_of(t.shape);
  size_t nd = axes.size();
  std::vector<usize> oshape(nd), step(nd), idx(nd, 0);
  for (size_t d = 0; d < nd; ++d) { oshape[d] = t.shape[axes[d]]; step[d] = in_s[axes[d]]; }
  Tensor<T> out;
  out.shape = oshape;
  out.data.resize(t.data.size());
  usize off = 0;
  for (usize e = 0; e < t.data.size(); ++e) {
    out.data[e] = t.data[off];
    for (size_t d = nd; d-- > 0;) {
      idx[d]++;
      off += step[d];
      if (idx[d] < oshape[d]) break;
      off -= step[d] * oshape[d];
      idx[d] = 0;
    }
  }
  return out;
}

// Shared odometer for sum_axis / trace_pair (src/tensor.rs:503-547, 593-633).
template <class T>
static Tensor<T> reduce_strided(const Tensor<T>& t, const std::vector<size_t>& drop, usize d, usize red_step, usize base0) {
  auto st = strides_of(t.shape);
  std::vector<usize> oshape, osteps;
  for (size_t i = 0; i < t.shape.size(); ++i)
    if (std::find(drop.begin(), drop.end(), i) == drop.end()) { oshape.push_back(t.shape[i]); osteps.push_back(st[i]); }
  usize n_out = 1;
  for (usize x : oshape) n_out *= x;
  Tensor<T> out;
  out.shape = oshape;
  out.data.assign(n_out, S<T>::zero());
  std::vector<usize> idx(oshape.size(), 0);
  usize base = base0;
  for (usize o = 0; o < n_out; ++o) {
    T acc = S<T>::zero();
    usize off = base;
    for (usize r = 0; r < d; ++r) { acc += t.data[off]; off += red_step; }
    out.data[o] = acc;
    for (size_t dd = oshape.size(); dd-- > 0;) {
      idx[dd]++;
      base += osteps[dd];
      if (idx[dd] < oshape[dd]) break;
      base -= osteps[dd] * oshape[dd];
      idx[dd] = 0;
    }
  }
  return out;
}

template <class T>
static Tensor<T> sum_axis(const Tensor<T>& t, usize ax) {
  auto st = strides_of(t.shape);
  return reduce_strided(t, {(size_t)ax}, t.shape[ax], st[ax], 0);
}

template <class T>
static Tensor<T> trace_pair(const Tensor<T>& t, usize ai, usize aj) {
  auto st = strides_of(t.shape);
  return reduce_strided(t, {(size_t)ai, (size_t)aj}, t.shape[ai], st[ai] + st[aj], 0);
}

// src/tensor.rs:550-590
template <class T>
static Tensor<T> diag_pair(const Tensor<T>& t, usize ai, usize aj) {
  auto st = strides_of(t.shape);
  std::vector<usize> oshape;
  for (size_t k = 0; k < t.shape.size(); ++k)
    if (k != aj) oshape.push_back(t.shape[k]);
  size_t nd = oshape.size();
  std::vector<usize> step(nd);
  for (size_t o = 0; o < nd; ++o) {
    size_t in_ax = o < aj ? o : o + 1;
    step[o] = st[in_ax] + (o == ai ? st[aj] : 0);
  }
  usize n_out = 1;
  for (usize x : oshape) n_out *= x;
  Tensor<T> out;
  out.shape = oshape;
  out.data.resize(n_out);
  std::vector<usize> idx(nd, 0);
  usize off = 0;
  for (usize e = 0; e < n_out; ++e) {
    out.data[e] = t.data[off];
    for (size_t dd = nd; dd-- > 0;) {
      idx[dd]++;
      off += step[dd];
      if (idx[dd] < oshape[dd]) break;
      off -= step[dd] * oshape[dd];
      idx[dd] = 0;
    }
  }
  return out;
}

// src/tensor.rs:636-669
template <class T>
static Tensor<T> select_axis(const Tensor<T>& t, usize ax, usize i) {
  auto st = strides_of(t.shape);
  std::vector<usize> oshape, osteps;
  for (size_t d = 0; d < t.shape.size(); ++d)
    if (d != ax) { oshape.push_back(t.shape[d]); osteps.push_back(st[d]); }
  usize n_out = 1;
  for (usize x : oshape) n_out *= x;
  Tensor<T> out;
  out.shape = oshape;
  out.data.resize(n_out);
  std::vector<usize> idx(oshape.size(), 0);
  usize base = i * st[ax];
  for (usize e = 0; e < n_out; ++e) {
    out.data[e] = t.data[base];
    for (size_t dd = oshape.size(); dd-- > 0;) {
      idx[dd]++;
      base += osteps[dd];
      if (idx[dd] < oshape[dd]) break;
      base -= osteps[dd] * oshape[dd];
      idx[dd] = 0;
    }
  }
  return out;
}

// src/contract.rs:102-181 with the GEMM backend (matrixmultiply 0.3.10, not vendored) restated as a
// k-ascending loop: every output element starts at zero and adds its products for l = 0, 1, ..., k-1 in
// that order, each product formed as num-complex does ((ar*br - ai*bi), (ar*bi + ai*br)).  The loop is
// register-blocked (MR rows x NR columns of C held in registers across a KC-long slice of K, a packed
// KC x NR panel of B split into real and imaginary parts) so it runs near the host's vector rate; the
// blocking changes which values sit in registers, never the order of any output's additions, so the bits
// equal the plain triple loop's.  Built for AVX2 where the host has it.
template <class T> struct GemmParts { using R = T; static constexpr bool cx = false; };
template <class R_> struct GemmParts<Cx<R_>> { using R = R_; static constexpr bool cx = true; };

template <class T>
__attribute__((target_clones("avx2", "default"))) static void gemm_rows(const T* A, const T* B, T* C, usize m,
                                                                           usize k, usize n) {
  using R = typename GemmParts<T>::R;
  constexpr bool cx = GemmParts<T>::cx;
  constexpr usize MR = 4, NR = cx ? 8 : 16, KC = 256;
  alignas(64) R bre[KC * NR], bim[cx ? KC * NR : 1];
  for (usize j0 = 0; j0 < n; j0 += NR) {
    const usize nr = std::min<usize>(NR, n - j0);
    for (usize k0 = 0; k0 < k; k0 += KC) {
      const usize kc = std::min<usize>(KC, k - k0);
      for (usize l = 0; l < kc; ++l)
        for (usize c = 0; c < NR; ++c) {
          const T v = c < nr ? B[(k0 + l) * n + j0 + c] : S<T>::zero();
          if constexpr (cx) { bre[l * NR + c] = v.re; bim[l * NR + c] = v.im; }
          else bre[l * NR + c] = v;
        }
      for (usize i0 = 0; i0 < m; i0 += MR) {
        const usize mr = std::min<usize>(MR, m - i0);
        R ar_[MR][NR], ai_[MR][cx ? NR : 1];
        for (usize r = 0; r < MR; ++r)
          for (usize c = 0; c < NR; ++c) {
            const T v = (r < mr && c < nr) ? C[(i0 + r) * n + j0 + c] : S<T>::zero();
            if constexpr (cx) { ar_[r][c] = v.re; ai_[r][c] = v.im; }
            else ar_[r][c] = v;
          }
        for (usize l = 0; l < kc; ++l) {
          const R* br = bre + l * NR;
          const R* bi = bim + (cx ? l * NR : 0);
          for (usize r = 0; r < MR; ++r) {
            const T a = r < mr ? A[(i0 + r) * k + k0 + l] : S<T>::zero();
            if constexpr (cx) {
              const R xr = a.re, xi = a.im;
              for (usize c = 0; c < NR; ++c) {
                const R tr = xr * br[c] - xi * bi[c];
                const R ti = xr * bi[c] + xi * br[c];
                ar_[r][c] += tr;
                ai_[r][c] += ti;
              }
            } else {
              for (usize c = 0; c < NR; ++c) ar_[r][c] += a * br[c];
            }
          }
        }
        for (usize r = 0; r < mr; ++r)
          for (usize c = 0; c < nr; ++c) {
            if constexpr (cx) C[(i0 + r) * n + j0 + c] = T{ar_[r][c], ai_[r][c]};
            else C[(i0 + r) * n + j0 + c] = ar_[r][c];
          }
      }
    }
  }
}

template <class T>
static std::vector<T> batch_gemm(const std::vector<T>& a, const std::vector<T>& b, usize bt, usize m, usize k, usize n) {
  std::vector<T> c(bt * m * n, S<T>::zero());
  for (usize ib = 0; ib < bt; ++ib) gemm_rows(a.data() + ib * m * k, b.data() + ib * k * n, c.data() + ib * m * n, m, k, n);
  return c;
}

template <class T>
static Tensor<T> apply_prep(const Prep& pr, Tensor<T> t) {
  for (auto& op : pr.traces) {
    usize ai = std::get<0>(op), aj = std::get<1>(op);
    t = std::get<2>(op) ? diag_pair(t, ai, aj) : trace_pair(t, ai, aj);
  }
  return t;
}

template <class T>
static std::vector<T> step_gemm(const Step& st, const Tensor<T>& a0, const Tensor<T>& b0) {
  Tensor<T> a = a0, b = b0;
  for (usize ax : st.sum_a) a = sum_axis(a, ax);
  for (usize ax : st.sum_b) b = sum_axis(b, ax);
  a = permute(a, st.a_perm);
  b = permute(b, st.b_perm);
  return batch_gemm(a.data, b.data, st.bt, st.m, st.k, st.n);
}

template <class T>
static Tensor<T> apply_fin(const Fin& f, Tensor<T> t) {
  for (usize ax : f.sum) t = sum_axis(t, ax);
  return permute(t, f.perm);
}

static void check_shape(const std::vector<usize>& got, const std::vector<usize>& want, const char* label) {
  if (got != want) throw Err(std::string(label) + " shape does not match the compiled plan");
}

// src/compiled.rs:383-441
template <class T>
static Tensor<T> execute(const Plan& p, const std::vector<Tensor<T>>& tensors, bool strip, double* exponent_out) {
  if (tensors.size() != p.n_inputs) throw Err("tensor count does not match the compiled plan");
  for (size_t i = 0; i < tensors.size(); ++i) check_shape(tensors[i].shape, p.preps[i].input_shape, "input tensor");
  std::vector<Tensor<T>> slots;
  std::vector<bool> live;
  for (size_t i = 0; i < tensors.size(); ++i) { slots.push_back(apply_prep(p.preps[i], tensors[i])); live.push_back(true); }
  double exponent = 0.0;
  for (auto& st : p.steps) {
    if (!live[st.li] || !live[st.ri]) throw Err("plan references a consumed tensor");
    live[st.li] = live[st.ri] = false;
    std::vector<T> c = step_gemm(st, slots[st.li], slots[st.ri]);
    slots[st.li].data.clear(); slots[st.li].data.shrink_to_fit();
    slots[st.ri].data.clear(); slots[st.ri].data.shrink_to_fit();
    if (strip) {
      double fmax = 0.0;
      for (auto& v : c) { double mg = S<T>::mag(v); if (mg > fmax) fmax = mg; }
      if (fmax > 0.0 && std::isfinite(fmax)) {
        exponent += std::log10(fmax);
        double inv = 1.0 / fmax;
        for (auto& v : c) v = S<T>::scale(v, inv);
      }
    }
    Tensor<T> r;
    r.shape = st.result_shape;
    r.data = std::move(c);
    slots.push_back(std::move(r));
    live.push_back(true);
  }
  if (!live[p.fin.slot]) throw Err("final tensor missing");
  if (exponent_out) *exponent_out = exponent;
  return apply_fin(p.fin, slots[p.fin.slot]);
}

// ---------------------------------------------------------------- naive einsum
// src/naive.rs:10-76
template <class T>
static Tensor<T> naive_einsum(const Net& net, const std::vector<Tensor<T>>& ts) {
  validate(net);
  std::vector<Leg> all;
  for (auto& t : net.inputs) all.insert(all.end(), t.begin(), t.end());
  all.insert(all.end(), net.output.begin(), net.output.end());
  all = sorted_dedup(all);
  double space = 0.0;
  for (Leg l : all) space += net.log2_dim(l);
  if (space > 28.0) throw Err("joint index space too large for naive einsum");
  std::vector<usize> dims;
  std::map<Leg, size_t> pos;
  for (size_t i = 0; i < all.size(); ++i) { dims.push_back(net.dim(all[i])); pos[all[i]] = i; }
  std::vector<std::vector<std::pair<size_t, usize>>> maps;
  for (size_t i = 0; i < net.inputs.size(); ++i) {
    auto st = strides_of(ts[i].shape);
    std::vector<std::pair<size_t, usize>> mp;
    for (size_t a = 0; a < net.inputs[i].size(); ++a) mp.push_back({pos[net.inputs[i][a]], st[a]});
    maps.push_back(mp);
  }
  Tensor<T> out;
  for (Leg l : net.output) out.shape.push_back(net.dim(l));
  usize on = 1;
  for (usize x : out.shape) on *= x;
  out.data.assign(on, S<T>::zero());
  auto ost = strides_of(out.shape);
  std::vector<std::pair<size_t, usize>> omap;
  for (size_t a = 0; a < net.output.size(); ++a) omap.push_back({pos[net.output[a]], ost[a]});
  usize total = 1;
  for (usize d : dims) total *= d;
  std::vector<usize> idx(all.size(), 0);
  for (usize e = 0; e < total; ++e) {
    T term = S<T>::one();
    for (size_t t = 0; t < maps.size(); ++t) {
      usize off = 0;
      for (auto& ps : maps[t]) off += idx[ps.first] * ps.second;
      term = term * ts[t].data[off];
    }
    usize oo = 0;
    for (auto& ps : omap) oo += idx[ps.first] * ps.second;
    out.data[oo] += term;
    for (size_t d = idx.size(); d-- > 0;) {
      if (++idx[d] < dims[d]) break;
      idx[d] = 0;
    }
  }
  return out;
}

// ---------------------------------------------------------------- sliced execution
// src/slice.rs:881-888
static void decode_slice_index(usize s, const std::vector<usize>& dims, std::vector<usize>& idx) {
  for (size_t d = dims.size(); d-- > 0;) { idx[d] = s % dims[d]; s /= dims[d]; }
}

static const usize SLICE_MAX_CHUNKS = 256;         // src/slice.rs:921
static const usize SLICE_PARTIAL_BUDGET = 1u << 22;  // src/slice.rs:924

// src/slice.rs:893-905
static usize slice_parallel_chunks(usize n_slices, usize out_numel) {
  if (n_slices <= 1) return 1;
  usize budget = SLICE_PARTIAL_BUDGET / std::max<usize>(out_numel, 1);
  if (budget < 1) budget = 1;
  usize n0 = std::max<usize>(std::min(std::min(n_slices, SLICE_MAX_CHUNKS), budget), 1);
  if (n0 <= 1) return 1;
  usize chunk = (n_slices + n0 - 1) / n0;
  return (n_slices + chunk - 1) / chunk;
}

// src/slice.rs:139-150, 152-176
static bool slice_leg_allowed(const Net& net, Leg leg, bool allow_output) {
  auto it = net.size.find(leg);
  if (it == net.size.end() || it->second == 0) return false;
  if (!allow_output && std::find(net.output.begin(), net.output.end(), leg) != net.output.end()) return false;
  bool held = false;
  for (auto& t : net.inputs) {
    int c = (int)std::count(t.begin(), t.end(), leg);
    if (c > 1) return false;
    if (c > 0) held = true;
  }
  return held;
}

static void validate_slice_legs(const Net& net, const std::vector<Leg>& sliced) {
  std::set<Leg> seen;
  for (Leg l : sliced) {
    if (!seen.insert(l).second) throw Err("sliced leg " + std::to_string(l) + " is repeated");
    auto it = net.size.find(l);
    if (it == net.size.end()) throw Err("sliced leg " + std::to_string(l) + " is not in size_dict");
    if (it->second == 0) throw Err("sliced leg has dimension 0");
    bool held = false;
    for (auto& t : net.inputs) {
      int c = (int)std::count(t.begin(), t.end(), l);
      if (c > 1) throw Err("sliced leg " + std::to_string(l) + " is repeated within one input tensor");
      if (c) held = true;
    }
    if (!held) throw Err("sliced leg " + std::to_string(l) + " is not held by any input tensor");
  }
}

static void validate_shapes_net(const Net& net, const std::vector<std::vector<usize>>& shapes) {
  validate(net);
  if (shapes.size() != net.n()) throw Err("tensor count does not match the network");
  for (size_t i = 0; i < shapes.size(); ++i) {
    std::vector<usize> want;
    for (Leg l : net.inputs[i]) want.push_back(net.dim(l));
    if (want != shapes[i]) throw Err("tensor " + std::to_string(i) + " shape does not match its legs");
  }
}

template <class T>
static std::vector<std::vector<usize>> shapes_of(const std::vector<Tensor<T>>& ts) {
  std::vector<std::vector<usize>> s;
  for (auto& t : ts) s.push_back(t.shape);
  return s;
}

template <class T>
static Tensor<T> contract_network(const Net& net, const std::vector<Tensor<T>>& ts, const Path& path) {
  // src/contract.rs:328-417; bit-identical to compile+execute in the reference
  // (tests/correctness.rs:43-103), so it is restated through the compiled form.
  validate_shapes_net(net, shapes_of(ts));
  Plan p = compile(net, path);
  return execute(p, ts, false, nullptr);
}

template <class T>
static Tensor<T> contract_output_blocks(const Net& net, const std::vector<Tensor<T>>& ts, const Path& path,
                                        const std::vector<Leg>& sliced, int threads);

// src/slice.rs:960-1065
template <class T>
static Tensor<T> contract_network_sliced(const Net& net, const std::vector<Tensor<T>>& ts, const Path& path,
                                         const std::vector<Leg>& sliced, int threads) {
  validate_shapes_net(net, shapes_of(ts));
  validate_slice_legs(net, sliced);
  if (sliced.empty()) return contract_network(net, ts, path);
  for (Leg l : sliced)
    if (std::find(net.output.begin(), net.output.end(), l) != net.output.end())
      return contract_output_blocks(net, ts, path, sliced, threads);
  std::map<Leg, size_t> spos;
  for (size_t i = 0; i < sliced.size(); ++i) spos[sliced[i]] = i;
  Net sub = net;
  for (auto& t : sub.inputs) t.erase(std::remove_if(t.begin(), t.end(), [&](Leg l) { return spos.count(l) > 0; }), t.end());
  for (Leg l : sliced) sub.size.erase(l);
  std::vector<usize> dims;
  unsigned __int128 ns = 1;
  for (Leg l : sliced) {
    dims.push_back(net.dim(l));
    ns *= net.dim(l);
    if (ns > (unsigned __int128)UINT64_MAX) throw Err("slice count overflows usize");
  }
  usize n_slices = (usize)ns;
  Plan plan = compile(sub, path);  // same path reused for every slice
  auto run_one = [&](usize s) {
    std::vector<usize> idx(sliced.size());
    decode_slice_index(s, dims, idx);
    std::vector<Tensor<T>> sts;
    for (size_t i = 0; i < net.n(); ++i) {
      Tensor<T> t = ts[i];
      for (size_t ax = net.inputs[i].size(); ax-- > 0;) {
        auto it = spos.find(net.inputs[i][ax]);
        if (it != spos.end()) t = select_axis(t, ax, idx[it->second]);
      }
      sts.push_back(std::move(t));
    }
    return execute(plan, sts, false, nullptr);
  };
  usize out_numel = 1;
  {
    unsigned __int128 on = 1;
    bool ovf = false;
    for (Leg l : net.output) { on *= net.dim(l); if (on > (unsigned __int128)UINT64_MAX) ovf = true; }
    out_numel = ovf ? UINT64_MAX : (usize)on;
    if (out_numel < 1) out_numel = 1;
  }
  usize n_chunks = slice_parallel_chunks(n_slices, out_numel);
  if (n_chunks == 1) {
    Tensor<T> acc = run_one(0);
    for (usize s = 1; s < n_slices; ++s) {
      Tensor<T> part = run_one(s);
      for (size_t e = 0; e < acc.data.size(); ++e) acc.data[e] += part.data[e];
    }
    return acc;
  }
  usize chunk = (n_slices + n_chunks - 1) / n_chunks;
  std::vector<Tensor<T>> partials(n_chunks);
  std::vector<std::string> errors(n_chunks);
  // Chunks run on a pool of host threads (the reference uses Rayon); chunk
  // boundaries depend only on (n_slices, out_numel), so rounding does not
  // depend on the thread count.
  std::atomic<long long> next{0};
  auto worker = [&]() {
    for (;;) {
    long long c = next.fetch_add(1);
    if (c >= (long long)n_chunks) return;
    try {
      usize lo = c * chunk, hi = std::min<usize>((c + 1) * chunk, n_slices);
      Tensor<T> acc = run_one(lo);
      for (usize s = lo + 1; s < hi; ++s) {
        Tensor<T> part = run_one(s);
        for (size_t e = 0; e < acc.data.size(); ++e) acc.data[e] += part.data[e];
      }
      partials[c] = std::move(acc);
    } catch (std::exception& ex) {
      errors[c] = ex.what();
    }
    }
  };
  int nt = std::max(1, std::min<int>(threads, (int)n_chunks));
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; ++t) pool.emplace_back(worker);
  worker();
  for (auto& th : pool) th.join();
  for (auto& e : errors)
    if (!e.empty()) throw Err(e);
  Tensor<T> acc = std::move(partials[0]);
  for (usize c = 1; c < n_chunks; ++c)
    for (size_t e = 0; e < acc.data.size(); ++e) acc.data[e] += partials[c].data[e];
  return acc;
}

// src/bin/tnmpi.rs:290-376 (contract_slice_range): slices [begin, end) of the
// mixed-radix slice numbering (last leg fastest) added into a zeroed full
// output at their block offset.  Internal sliced legs only move nothing;
// output legs shift by their stride.  The range is split into contiguous
// per-thread sub-ranges, each summed in order and merged in order.
template <class T>
static Tensor<T> contract_slice_range(const Net& net, const std::vector<Tensor<T>>& ts, const Path& path,
                                      const std::vector<Leg>& sliced, usize begin, usize end, int threads) {
  validate_shapes_net(net, shapes_of(ts));
  validate_slice_legs(net, sliced);
  std::map<Leg, size_t> spos;
  for (size_t i = 0; i < sliced.size(); ++i) spos[sliced[i]] = i;
  Net sub = net;
  for (auto& t : sub.inputs) t.erase(std::remove_if(t.begin(), t.end(), [&](Leg l) { return spos.count(l) > 0; }), t.end());
  sub.output.erase(std::remove_if(sub.output.begin(), sub.output.end(), [&](Leg l) { return spos.count(l) > 0; }), sub.output.end());
  for (Leg l : sliced) sub.size.erase(l);
  std::vector<usize> dims;
  for (Leg l : sliced) dims.push_back(net.dim(l));
  usize n_slices = checked_numel(dims);
  if (begin >= end || end > n_slices) throw Err("slice range is outside the slice count");
  Plan plan = compile(sub, path);
  std::vector<usize> oshape;
  for (Leg l : net.output) oshape.push_back(net.dim(l));
  auto ost = strides_of(oshape);
  std::vector<usize> leg_stride(sliced.size(), 0);
  std::vector<std::pair<usize, usize>> kept;  // (dim, stride) of unsliced output axes
  for (size_t ax = 0; ax < net.output.size(); ++ax) {
    auto it = spos.find(net.output[ax]);
    if (it != spos.end()) leg_stride[it->second] = ost[ax];
    else kept.push_back({oshape[ax], ost[ax]});
  }
  usize on = checked_numel(oshape);
  auto run_range = [&](usize lo, usize hi, Tensor<T>& total) {
    total.shape = oshape;
    total.data.assign(on, S<T>::zero());
    std::vector<usize> idx(sliced.size());
    for (usize s = lo; s < hi; ++s) {
      decode_slice_index(s, dims, idx);
      std::vector<Tensor<T>> sts;
      for (size_t i = 0; i < net.n(); ++i) {
        Tensor<T> t = ts[i];
        for (size_t ax = net.inputs[i].size(); ax-- > 0;) {
          auto it = spos.find(net.inputs[i][ax]);
          if (it != spos.end()) t = select_axis(t, ax, idx[it->second]);
        }
        sts.push_back(std::move(t));
      }
      Tensor<T> part = execute(plan, sts, false, nullptr);
      usize base = 0;
      for (size_t q = 0; q < idx.size(); ++q) base += idx[q] * leg_stride[q];
      for (usize e = 0; e < part.data.size(); ++e) {
        usize rem = e, off = base;
        for (size_t q = kept.size(); q-- > 0;) { off += (rem % kept[q].first) * kept[q].second; rem /= kept[q].first; }
        total.data[off] += part.data[e];
      }
    }
  };
  int nt = std::max(1, std::min<int>(threads, (int)(end - begin)));
  std::vector<Tensor<T>> parts(nt);
  std::vector<std::string> errors(nt);
  usize span = end - begin;
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t) {
    usize lo = begin + span * t / nt, hi = begin + span * (t + 1) / nt;
    pool.emplace_back([&, t, lo, hi]() {
      try { run_range(lo, hi, parts[t]); } catch (std::exception& e) { errors[t] = e.what(); }
    });
  }
  for (auto& th : pool) th.join();
  for (auto& e : errors)
    if (!e.empty()) throw Err(e);
  Tensor<T> acc = std::move(parts[0]);
  for (int t = 1; t < nt; ++t)
    for (usize e = 0; e < acc.data.size(); ++e) acc.data[e] += parts[t].data[e];
  return acc;
}

// src/slice.rs:1070-1173
template <class T>
static Tensor<T> contract_output_blocks(const Net& net, const std::vector<Tensor<T>>& ts, const Path& path,
                                        const std::vector<Leg>& sliced, int threads) {
  std::vector<Leg> outer, internal;
  std::map<Leg, size_t> opos;
  for (Leg l : net.output)
    if (std::find(sliced.begin(), sliced.end(), l) != sliced.end()) { opos[l] = outer.size(); outer.push_back(l); }
  for (Leg l : sliced)
    if (!opos.count(l)) internal.push_back(l);
  std::vector<usize> shape;
  for (Leg l : net.output) shape.push_back(net.dim(l));
  usize numel = checked_numel(shape);
  if ((unsigned __int128)numel * sizeof(T) > (unsigned __int128)INT64_MAX) throw Err("full output tensor byte size exceeds allocatable capacity");
  Tensor<T> result;
  result.shape = shape;
  result.data.assign(numel, S<T>::zero());
  auto strides = strides_of(shape);
  std::vector<std::pair<usize, usize>> kept;
  std::vector<usize> ostr(outer.size());
  for (size_t ax = 0; ax < net.output.size(); ++ax) {
    auto it = opos.find(net.output[ax]);
    if (it != opos.end()) ostr[it->second] = strides[ax];
    else kept.push_back({shape[ax], strides[ax]});
  }
  Net sub = net;
  for (auto& t : sub.inputs) t.erase(std::remove_if(t.begin(), t.end(), [&](Leg l) { return opos.count(l) > 0; }), t.end());
  sub.output.erase(std::remove_if(sub.output.begin(), sub.output.end(), [&](Leg l) { return opos.count(l) > 0; }), sub.output.end());
  for (Leg l : outer) sub.size.erase(l);
  std::vector<usize> dims;
  for (Leg l : outer) dims.push_back(net.dim(l));
  usize n_blocks = checked_numel(dims);
  std::vector<usize> vals(outer.size());
  for (usize bn = 0; bn < n_blocks; ++bn) {
    decode_slice_index(bn, dims, vals);
    std::vector<Tensor<T>> bts;
    for (size_t i = 0; i < net.n(); ++i) {
      Tensor<T> t = ts[i];
      for (size_t ax = net.inputs[i].size(); ax-- > 0;) {
        auto it = opos.find(net.inputs[i][ax]);
        if (it != opos.end()) t = select_axis(t, ax, vals[it->second]);
      }
      bts.push_back(std::move(t));
    }
    Tensor<T> block = contract_network_sliced(sub, bts, path, internal, threads);
    usize base = 0;
    for (size_t q = 0; q < vals.size(); ++q) base += vals[q] * ostr[q];
    for (usize bo = 0; bo < block.data.size(); ++bo) {
      usize rem = bo, off = base;
      for (size_t q = kept.size(); q-- > 0;) { off += (rem % kept[q].first) * kept[q].second; rem /= kept[q].first; }
      result.data[off] = block.data[bo];
    }
  }
  return result;
}

// ---------------------------------------------------------------- greedy path
// src/paths/greedy.rs:31-320 (costmod = 1, temperature = 0, nbranch = 1)
struct Cand {
  double cost;
  usize a, b;
};
struct CandGreater {  // min-heap on (cost, a, b)
  bool operator()(const Cand& x, const Cand& y) const {
    if (x.cost != y.cost) return x.cost > y.cost;
    if (x.a != y.a) return x.a > y.a;
    return x.b > y.b;
  }
};

static Path greedy(const Net& net) {
  validate(net);
  std::set<Leg> in_output(net.output.begin(), net.output.end());
  std::map<Leg, usize> refcount;
  std::map<Leg, std::set<usize>> holders;
  std::vector<std::vector<Leg>> node_legs;
  std::vector<bool> live;
  std::vector<double> node_size;
  auto legs_size = [&](const std::vector<Leg>& legs) { return std::exp2(sum_log2(net, legs)); };
  for (size_t i = 0; i < net.n(); ++i) {
    auto d = sorted_dedup(net.inputs[i]);
    for (Leg l : d) { refcount[l]++; holders[l].insert(i); }
    node_size.push_back(legs_size(d));
    node_legs.push_back(d);
    live.push_back(true);
  }
  std::priority_queue<Cand, std::vector<Cand>, CandGreater> heap;
  auto result_legs = [&](usize a, usize b) {
    const auto &la = node_legs[a], &lb = node_legs[b];
    std::vector<Leg> out;
    for (Leg l : legs_union(la, lb)) {
      usize rc = refcount[l];
      if (std::binary_search(la.begin(), la.end(), l)) rc -= 1;
      if (std::binary_search(lb.begin(), lb.end(), l)) rc -= 1;
      if (rc > 0 || in_output.count(l)) out.push_back(l);
    }
    return out;
  };
  auto push_cand = [&](usize a, usize b) {
    double rsize = legs_size(result_legs(a, b));
    double cost = rsize - 1.0 * (node_size[a] + node_size[b]);
    heap.push(Cand{cost, a, b});
  };
  {
    std::set<std::pair<usize, usize>> seen;
    for (auto& kv : holders) {
      std::vector<usize> v(kv.second.begin(), kv.second.end());
      for (size_t i = 0; i < v.size(); ++i)
        for (size_t j = i + 1; j < v.size(); ++j)
          if (seen.insert({v[i], v[j]}).second) push_cand(v[i], v[j]);
    }
  }
  auto contract = [&](usize a, usize b) {
    auto result = result_legs(a, b);
    auto la = node_legs[a], lb = node_legs[b];
    live[a] = live[b] = false;
    for (Leg l : la) { refcount[l]--; holders[l].erase(a); }
    for (Leg l : lb) { refcount[l]--; holders[l].erase(b); }
    usize nid = node_legs.size();
    for (Leg l : result) { refcount[l]++; holders[l].insert(nid); }
    node_size.push_back(legs_size(result));
    node_legs.push_back(result);
    live.push_back(true);
    std::set<usize> nbrs;
    for (Leg l : result)
      for (usize h : holders[l])
        if (h != nid) nbrs.insert(h);
    for (usize nb : nbrs) {
      if (nb < nid) push_cand(nb, nid);
      else push_cand(nid, nb);
    }
    return nid;
  };
  Path path;
  while (!heap.empty()) {
    Cand c = heap.top();
    heap.pop();
    if (!(live[c.a] && live[c.b])) continue;
    contract(c.a, c.b);
    path.push_back({c.a, c.b});
  }
  std::vector<usize> rest;
  for (size_t i = 0; i < node_legs.size(); ++i)
    if (live[i]) rest.push_back(i);
  while (rest.size() > 1) {
    std::stable_sort(rest.begin(), rest.end(), [&](usize x, usize y) { return node_size[x] < node_size[y]; });
    usize a = rest[0], b = rest[1];
    if (a > b) std::swap(a, b);
    usize nid = contract(a, b);
    path.push_back({a, b});
    rest.erase(rest.begin(), rest.begin() + 2);
    rest.push_back(nid);
  }
  return path;
}

// ---------------------------------------------------------------- slice selection
// src/slice.rs:46-97 (Elements target, exact integer feasibility)
static bool legs_feasible(const Net& net, const std::vector<Leg>& legs, usize target) {
  usize rem = target;
  for (Leg l : legs) {
    usize d = net.dim(l);
    if (d > rem) return false;
    rem /= d;
  }
  return true;
}

// src/slice.rs:209-215, 254-288, 557-589.  allow_output: output legs may be sliced too
// (find_slices_until_for_target_with_output_slicing with no deadline, src/slice.rs:254-289).
static bool find_slices_to_size(const Net& net, const Path& path, usize target, std::vector<Leg>& out_legs,
                                bool allow_output = false) {
  if (target == 0) return false;
  std::vector<Leg> sliced;
  for (;;) {
    Net cur = net;
    for (Leg l : sliced) cur.size[l] = 1;
    std::vector<std::vector<Leg>> step_legs;
    try {
      simulate_path_full(cur, path, &step_legs);
    } catch (Err&) {
      return false;
    }
    bool feasible;
    if (cur.n() == 1) feasible = legs_feasible(cur, cur.output, target);
    else {
      feasible = true;
      for (auto& sl : step_legs)
        if (!legs_feasible(cur, sl, target)) { feasible = false; break; }
    }
    if (feasible) { out_legs = sliced; return true; }
    std::map<Leg, std::pair<usize, double>> score;
    // A unary contraction has no steps but still produces its output (src/slice.rs:565-566).
    if (allow_output && net.n() == 1) step_legs.push_back(cur.output);
    for (auto& sl : step_legs) {
      if (legs_feasible(cur, sl, target)) continue;
      for (Leg l : sl) {
        double d = cur.log2_dim(l);
        if (d <= 0.0 || !slice_leg_allowed(net, l, allow_output)) continue;
        auto it = score.find(l);
        if (it == score.end()) score[l] = {1, d};
        else it->second.first += 1;
      }
    }
    if (score.empty()) return false;
    bool have = false;
    Leg best = 0;
    std::pair<usize, double> bs{0, 0.0};
    for (auto& kv : score) {  // max by (count, log2 dim, smaller leg id)
      if (!have) { have = true; best = kv.first; bs = kv.second; continue; }
      auto s = kv.second;
      bool better;
      if (s.first != bs.first) better = s.first > bs.first;
      else if (s.second != bs.second) better = s.second > bs.second;
      else better = kv.first < best;
      if (better) { best = kv.first; bs = s; }
    }
    sliced.push_back(best);
    std::sort(sliced.begin(), sliced.end());
  }
}

}  // namespace oracle

// ==================================================================== C ABI
using namespace oracle;

static thread_local std::string g_err;
static thread_local std::string g_json;

static Net make_net(uint64_t n_inputs, const uint64_t* offs, const uint32_t* legs, uint64_t n_out, const uint32_t* out,
                    uint64_t n_sizes, const uint32_t* size_legs, const uint64_t* size_dims) {
  Net net;
  for (uint64_t i = 0; i < n_inputs; ++i) net.inputs.emplace_back(legs + offs[i], legs + offs[i + 1]);
  net.output.assign(out, out + n_out);
  for (uint64_t i = 0; i < n_sizes; ++i) net.size[size_legs[i]] = size_dims[i];
  return net;
}

static Path make_path(uint64_t n_steps, const uint64_t* pairs) {
  Path p;
  for (uint64_t s = 0; s < n_steps; ++s) p.push_back({pairs[2 * s], pairs[2 * s + 1]});
  return p;
}

template <class T>
static std::vector<Tensor<T>> make_tensors(const Net& net, const void* const* ptrs) {
  std::vector<Tensor<T>> ts;
  for (size_t i = 0; i < net.n(); ++i) {
    Tensor<T> t;
    usize n = 1;
    for (Leg l : net.inputs[i]) { t.shape.push_back(net.dim(l)); n *= net.dim(l); }
    const T* p = (const T*)ptrs[i];
    t.data.assign(p, p + n);
    ts.push_back(std::move(t));
  }
  return ts;
}

// dtype codes: 0 f32, 1 f64, 2 c64, 3 c128
#define DISPATCH(dt, ...)                                    \
  switch (dt) {                                              \
    case 0: { using T = float; __VA_ARGS__; break; }         \
    case 1: { using T = double; __VA_ARGS__; break; }        \
    case 2: { using T = Cx<float>; __VA_ARGS__; break; }     \
    case 3: { using T = Cx<double>; __VA_ARGS__; break; }    \
    default: throw Err("unsupported dtype code");            \
  }

#define GUARD(...)                                     \
  try { __VA_ARGS__; return 0; } catch (std::exception& e) { g_err = e.what(); return 1; }

static void json_vec(std::string& s, const std::vector<usize>& v) {
  s += "[";
  for (size_t i = 0; i < v.size(); ++i) { if (i) s += ","; s += std::to_string(v[i]); }
  s += "]";
}
static void json_legs(std::string& s, const std::vector<Leg>& v) {
  s += "[";
  for (size_t i = 0; i < v.size(); ++i) { if (i) s += ","; s += std::to_string(v[i]); }
  s += "]";
}
static std::string json_double(double x) {
  if (std::isinf(x)) return x > 0 ? "\"inf\"" : "\"-inf\"";
  char buf[64];
  snprintf(buf, sizeof buf, "%.17g", x);
  return buf;
}

extern "C" {

const char* oracle_last_error() { return g_err.c_str(); }

// Plan bookkeeping as JSON (slots, legs, shapes, sums, perms, GEMM dims).
int oracle_plan_json(uint64_t n_inputs, const uint64_t* offs, const uint32_t* legs, uint64_t n_out, const uint32_t* out,
                     uint64_t n_sizes, const uint32_t* size_legs, const uint64_t* size_dims, uint64_t n_steps,
                     const uint64_t* pairs, const char** json_out) {
  GUARD({
    Net net = make_net(n_inputs, offs, legs, n_out, out, n_sizes, size_legs, size_dims);
    Plan p = compile(net, make_path(n_steps, pairs));
    std::string& s = g_json;
    s = "{\"n_inputs\":" + std::to_string(p.n_inputs) + ",\"log10_flops\":" + json_double(p.log10_flops) +
        ",\"log2_peak_size\":" + json_double(p.log2_peak_size) + ",\"preps\":[";
    for (size_t i = 0; i < p.preps.size(); ++i) {
      auto& pr = p.preps[i];
      if (i) s += ",";
      s += "{\"input_shape\":"; json_vec(s, pr.input_shape);
      s += ",\"traces\":[";
      for (size_t t = 0; t < pr.traces.size(); ++t) {
        if (t) s += ",";
        s += "[" + std::to_string(std::get<0>(pr.traces[t])) + "," + std::to_string(std::get<1>(pr.traces[t])) + "," +
             (std::get<2>(pr.traces[t]) ? "1" : "0") + "]";
      }
      s += "],\"legs\":"; json_legs(s, pr.legs);
      s += ",\"shape\":"; json_vec(s, pr.shape);
      s += "}";
    }
    s += "],\"steps\":[";
    for (size_t i = 0; i < p.steps.size(); ++i) {
      auto& st = p.steps[i];
      if (i) s += ",";
      s += "{\"left_slot\":" + std::to_string(st.li) + ",\"right_slot\":" + std::to_string(st.ri) +
           ",\"result_slot\":" + std::to_string(st.out);
      s += ",\"left_legs\":"; json_legs(s, st.left_legs);
      s += ",\"right_legs\":"; json_legs(s, st.right_legs);
      s += ",\"result_legs\":"; json_legs(s, st.result_legs);
      s += ",\"left_shape\":"; json_vec(s, st.left_shape);
      s += ",\"right_shape\":"; json_vec(s, st.right_shape);
      s += ",\"result_shape\":"; json_vec(s, st.result_shape);
      s += ",\"sum_a\":"; json_vec(s, st.sum_a);
      s += ",\"sum_b\":"; json_vec(s, st.sum_b);
      s += ",\"a_perm\":"; json_vec(s, st.a_perm);
      s += ",\"b_perm\":"; json_vec(s, st.b_perm);
      s += ",\"gemm_dims\":"; json_vec(s, {st.bt, st.m, st.k, st.n});
      s += "}";
    }
    s += "],\"finalize\":{\"slot\":" + std::to_string(p.fin.slot) + ",\"input_legs\":";
    json_legs(s, p.fin.input_legs);
    s += ",\"input_shape\":"; json_vec(s, p.fin.input_shape);
    s += ",\"sum\":"; json_vec(s, p.fin.sum);
    s += ",\"perm\":"; json_vec(s, p.fin.perm);
    s += ",\"output_shape\":"; json_vec(s, p.fin.output_shape);
    s += "}}";
    *json_out = s.c_str();
  })
}

// Path metrics: writes 6 doubles (log10_flops, log2_max_size, log2_max_contraction_size,
// log2_total_size, log2_read_write, log2_peak_size).
int oracle_simulate_path(uint64_t n_inputs, const uint64_t* offs, const uint32_t* legs, uint64_t n_out, const uint32_t* out,
                         uint64_t n_sizes, const uint32_t* size_legs, const uint64_t* size_dims, uint64_t n_steps,
                         const uint64_t* pairs, double* stats6) {
  GUARD({
    Net net = make_net(n_inputs, offs, legs, n_out, out, n_sizes, size_legs, size_dims);
    Stats st = simulate_path_full(net, make_path(n_steps, pairs), nullptr);
    double v[6] = {st.log10_flops, st.log2_max_size, st.log2_max_contraction_size, st.log2_total_size, st.log2_read_write, st.log2_peak_size};
    std::memcpy(stats6, v, sizeof v);
  })
}

// Compiled execution (mode 0: execute, 1: execute_stripped); out has numel(output) elements.
int oracle_execute(uint64_t n_inputs, const uint64_t* offs, const uint32_t* legs, uint64_t n_out, const uint32_t* out,
                   uint64_t n_sizes, const uint32_t* size_legs, const uint64_t* size_dims, uint64_t n_steps,
                   const uint64_t* pairs, int dtype, const void* const* inputs, void* result, int strip, double* exponent) {
  GUARD({
    Net net = make_net(n_inputs, offs, legs, n_out, out, n_sizes, size_legs, size_dims);
    Plan p = compile(net, make_path(n_steps, pairs));
    DISPATCH(dtype, {
      auto ts = make_tensors<T>(net, inputs);
      double e = 0.0;
      auto r = execute(p, ts, strip != 0, &e);
      std::memcpy(result, r.data.data(), r.data.size() * sizeof(T));
      if (exponent) *exponent = e;
    });
  })
}

int oracle_contract_sliced(uint64_t n_inputs, const uint64_t* offs, const uint32_t* legs, uint64_t n_out, const uint32_t* out,
                           uint64_t n_sizes, const uint32_t* size_legs, const uint64_t* size_dims, uint64_t n_steps,
                           const uint64_t* pairs, uint64_t n_sliced, const uint32_t* sliced, int dtype,
                           const void* const* inputs, void* result, int threads) {
  GUARD({
    Net net = make_net(n_inputs, offs, legs, n_out, out, n_sizes, size_legs, size_dims);
    std::vector<Leg> sl(sliced, sliced + n_sliced);
    DISPATCH(dtype, {
      auto ts = make_tensors<T>(net, inputs);
      auto r = contract_network_sliced(net, ts, make_path(n_steps, pairs), sl, threads < 1 ? 1 : threads);
      std::memcpy(result, r.data.data(), r.data.size() * sizeof(T));
    });
  })
}

int oracle_naive_einsum(uint64_t n_inputs, const uint64_t* offs, const uint32_t* legs, uint64_t n_out, const uint32_t* out,
                        uint64_t n_sizes, const uint32_t* size_legs, const uint64_t* size_dims, int dtype,
                        const void* const* inputs, void* result) {
  GUARD({
    Net net = make_net(n_inputs, offs, legs, n_out, out, n_sizes, size_legs, size_dims);
    DISPATCH(dtype, {
      auto ts = make_tensors<T>(net, inputs);
      auto r = naive_einsum(net, ts);
      std::memcpy(result, r.data.data(), r.data.size() * sizeof(T));
    });
  })
}

// Greedy path; path_out must hold 2*(n_inputs-1) entries.  Writes the step count.
int oracle_greedy(uint64_t n_inputs, const uint64_t* offs, const uint32_t* legs, uint64_t n_out, const uint32_t* out,
                  uint64_t n_sizes, const uint32_t* size_legs, const uint64_t* size_dims, uint64_t* path_out,
                  uint64_t* n_steps_out) {
  GUARD({
    Net net = make_net(n_inputs, offs, legs, n_out, out, n_sizes, size_legs, size_dims);
    Path p = greedy(net);
    for (size_t s = 0; s < p.size(); ++s) { path_out[2 * s] = p[s].first; path_out[2 * s + 1] = p[s].second; }
    *n_steps_out = p.size();
  })
}

// find_slices_to_size; legs_out must hold n_sizes entries.  *found = 0 when None.
int oracle_find_slices_to_size(uint64_t n_inputs, const uint64_t* offs, const uint32_t* legs, uint64_t n_out,
                               const uint32_t* out, uint64_t n_sizes, const uint32_t* size_legs, const uint64_t* size_dims,
                               uint64_t n_steps, const uint64_t* pairs, uint64_t target, uint32_t* legs_out,
                               uint64_t* n_legs_out, int* found) {
  GUARD({
    Net net = make_net(n_inputs, offs, legs, n_out, out, n_sizes, size_legs, size_dims);
    std::vector<Leg> sl;
    bool ok = find_slices_to_size(net, make_path(n_steps, pairs), target, sl);
    *found = ok ? 1 : 0;
    *n_legs_out = sl.size();
    for (size_t i = 0; i < sl.size(); ++i) legs_out[i] = sl[i];
  })
}

// The same search with output legs allowed when allow_output_slicing != 0.
int oracle_find_slices_with_output(uint64_t n_inputs, const uint64_t* offs, const uint32_t* legs, uint64_t n_out,
                                   const uint32_t* out, uint64_t n_sizes, const uint32_t* size_legs,
                                   const uint64_t* size_dims, uint64_t n_steps, const uint64_t* pairs, uint64_t target,
                                   int allow_output_slicing, uint32_t* legs_out, uint64_t* n_legs_out, int* found) {
  GUARD({
    Net net = make_net(n_inputs, offs, legs, n_out, out, n_sizes, size_legs, size_dims);
    std::vector<Leg> sl;
    bool ok = find_slices_to_size(net, make_path(n_steps, pairs), target, sl, allow_output_slicing != 0);
    *found = ok ? 1 : 0;
    *n_legs_out = sl.size();
    for (size_t i = 0; i < sl.size(); ++i) legs_out[i] = sl[i];
  })
}

int oracle_contract_slice_range(uint64_t n_inputs, const uint64_t* offs, const uint32_t* legs, uint64_t n_out,
                                const uint32_t* out, uint64_t n_sizes, const uint32_t* size_legs,
                                const uint64_t* size_dims, uint64_t n_steps, const uint64_t* pairs, uint64_t n_sliced,
                                const uint32_t* sliced, uint64_t begin, uint64_t end, int dtype,
                                const void* const* inputs, void* result, int threads) {
  GUARD({
    Net net = make_net(n_inputs, offs, legs, n_out, out, n_sizes, size_legs, size_dims);
    std::vector<Leg> sl(sliced, sliced + n_sliced);
    DISPATCH(dtype, {
      auto ts = make_tensors<T>(net, inputs);
      auto r = contract_slice_range(net, ts, make_path(n_steps, pairs), sl, begin, end, threads < 1 ? 1 : threads);
      std::memcpy(result, r.data.data(), r.data.size() * sizeof(T));
    });
  })
}

uint64_t oracle_slice_parallel_chunks(uint64_t n_slices, uint64_t out_numel) { return slice_parallel_chunks(n_slices, out_numel); }

}  // extern "C"
