// Host planning model: validation, path metrics, compiled plan, greedy path and
// slice selection, restated from the reference Rust crate (file:line cited per
// function).  Integer bookkeeping (slots, legs, permutations, GEMM dims) must
// be bit-identical to the reference; the greedy path and slice choice depend
// on IEEE log2/exp2 sums, computed in the same order as the reference.
#include "host.hpp"

#include <algorithm>
#include <cmath>
#include <queue>
#include <set>

namespace ab2 {

double Network::log2_dim(Leg l) const { return std::log2((double)dim(l)); }

u64 checked_numel(const std::vector<u64>& shape) {
  unsigned __int128 n = 1;
  for (size_t a = 0; a < shape.size(); ++a) {
    if (shape[a] == 0) fail("shape axis " + std::to_string(a) + " has length 0; zero-length axes are not supported");
    n *= shape[a];
    if (n > (unsigned __int128)UINT64_MAX) fail("shape element count overflows usize");
  }
  return (u64)n;
}

void check_gemm_geometry(u64 bt, u64 m, u64 k, u64 n) {
  const u64 lim = (u64)INT64_MAX;
  const char* names[4] = {"batch", "m", "k", "n"};
  u64 v[4] = {bt, m, k, n};
  for (int i = 0; i < 4; ++i) {
    if (v[i] == 0) fail(std::string("GEMM dimension ") + names[i] + "=0");
    if (v[i] > lim) fail(std::string("GEMM dimension ") + names[i] + " exceeds the isize stride range");
  }
  unsigned __int128 blocks[3] = {(unsigned __int128)m * k, (unsigned __int128)k * n, (unsigned __int128)m * n};
  for (auto b : blocks)
    if (b > lim || b * bt > lim) fail("GEMM element offset exceeds the isize range");
}

void Network::validate() const {
  if (inputs.empty()) fail("TensorNetwork needs at least one input tensor");
  for (auto& kv : size) {
    if (kv.second == 0) fail("leg " + std::to_string(kv.first) + " has dimension 0");
    if (kv.second > (u64)INT64_MAX) fail("leg " + std::to_string(kv.first) + " dimension exceeds the GEMM stride range");
  }
  std::set<Leg> held;
  for (size_t i = 0; i < inputs.size(); ++i) {
    std::vector<u64> shape;
    std::map<Leg, int> count;
    for (Leg l : inputs[i]) {
      shape.push_back(dim(l));
      held.insert(l);
      if (++count[l] > 2) fail("leg " + std::to_string(l) + " appears more than twice in input " + std::to_string(i));
    }
    try {
      checked_numel(shape);
    } catch (Error& e) {
      fail("input tensor " + std::to_string(i) + " shape is invalid: " + e.what());
    }
  }
  std::set<Leg> seen;
  std::vector<u64> oshape;
  for (Leg l : output) {
    if (!seen.insert(l).second) fail("output contains a repeated leg");
    if (!held.count(l)) fail("output leg " + std::to_string(l) + " is not held by any input tensor");
    oshape.push_back(dim(l));
  }
  checked_numel(oshape);
  for (auto& kv : size)
    if (!held.count(kv.first)) fail("size_dict leg " + std::to_string(kv.first) + " is not used by any input tensor");
}

// ---------------------------------------------------------------- metrics
static double lae2(double a, double b) {  // src/path.rs:32-42
  if (a == -INFINITY) return b;
  if (b == -INFINITY) return a;
  double hi = std::max(a, b), lo = std::min(a, b);
  return hi + std::log2(1.0 + std::exp2(lo - hi));
}

static std::vector<Leg> merge_union(const std::vector<Leg>& a, const std::vector<Leg>& b) {
  std::vector<Leg> u;
  u.reserve(a.size() + b.size());
  std::set_union(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(u));
  return u;
}

static std::vector<Leg> uniq_sorted(std::vector<Leg> v) {
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  return v;
}

PathStats simulate_path(const Network& net, const SsaPath& path, std::vector<std::vector<Leg>>* step_legs) {
  net.validate();
  const size_t n = net.n_tensors();
  auto ld = [&](const std::vector<Leg>& legs) {
    double s = 0.0;
    for (Leg l : legs) s += net.log2_dim(l);
    return s;
  };
  std::set<Leg> outs(net.output.begin(), net.output.end());
  if (outs.size() != net.output.size()) fail("output contains a repeated leg");
  std::map<Leg, u64> appear, rc;
  for (auto& t : net.inputs)
    for (Leg l : t) ++appear[l];
  for (Leg l : net.output) ++appear[l];
  std::vector<std::vector<Leg>> slot;
  std::vector<char> alive;
  std::vector<double> leaf_log2, rw_log2, slot_size;
  for (auto& t : net.inputs) {
    std::vector<Leg> srt = t;
    std::sort(srt.begin(), srt.end());
    double leaf = 0.0;
    for (size_t i = 0; i < srt.size();) {
      size_t j = i;
      while (j < srt.size() && srt[j] == srt[i]) ++j;
      if (j - i != appear[srt[i]]) leaf += net.log2_dim(srt[i]);
      i = j;
    }
    auto d = uniq_sorted(t);
    for (Leg l : d) ++rc[l];
    slot.push_back(d);
    alive.push_back(1);
    leaf_log2.push_back(leaf);
    rw_log2.push_back(ld(t));
    slot_size.push_back(std::exp2(ld(t)));
  }
  double flops = -INFINITY, max_size = (n == 1) ? ld(net.output) : 0.0, max_con = 0.0, total = -INFINITY, rw = -INFINITY;
  double live = 0.0;
  for (double v : slot_size) live += v;
  double peak = live;
  if (step_legs) step_legs->clear();
  for (size_t s = 0; s < path.size(); ++s) {
    u64 a = path[s].first, b = path[s].second;
    if (a == b) fail("step " + std::to_string(s) + " contracts tensor " + std::to_string(a) + " with itself");
    if (a >= slot.size() || !alive[a]) fail("step " + std::to_string(s) + " references invalid or consumed tensor " + std::to_string(a));
    if (b >= slot.size() || !alive[b]) fail("step " + std::to_string(s) + " references invalid or consumed tensor " + std::to_string(b));
    alive[a] = alive[b] = 0;
    auto uni = merge_union(slot[a], slot[b]);
    flops = lae2(flops, ld(uni));
    for (Leg l : slot[a]) --rc[l];
    for (Leg l : slot[b]) --rc[l];
    std::vector<Leg> res;
    for (Leg l : uni)
      if (rc[l] > 0 || outs.count(l)) res.push_back(l);
    for (Leg l : res) ++rc[l];
    double sz = ld(res);
    max_size = std::max(max_size, sz);
    max_con = std::max(max_con, lae2(lae2(leaf_log2[a], leaf_log2[b]), sz));
    rw = lae2(rw, lae2(lae2(rw_log2[a], rw_log2[b]), sz));
    leaf_log2.push_back(sz);
    rw_log2.push_back(sz);
    total = lae2(total, sz);
    double r = std::exp2(sz);
    peak = std::max(peak, live + r);
    live += r - slot_size[a] - slot_size[b];
    slot_size.push_back(r);
    if (step_legs) step_legs->push_back(res);
    slot.push_back(std::move(res));
    alive.push_back(1);
  }
  size_t n_alive = 0, last = 0;
  for (size_t i = 0; i < alive.size(); ++i)
    if (alive[i]) { ++n_alive; last = i; }
  if (n_alive != 1) fail("incomplete path: " + std::to_string(n_alive) + " tensors remain");
  auto fin = slot[last];
  auto want = uniq_sorted(net.output);
  if (path.empty()) {
    for (Leg l : want)
      if (!std::binary_search(fin.begin(), fin.end(), l)) fail("final legs do not contain every output leg");
  } else if (fin != want) {
    fail("final legs do not match the output legs");
  }
  return PathStats{flops * 0.301029995663981195213738894724493027, max_size, max_con, total, rw, std::log2(peak)};
}

// ---------------------------------------------------------------- compile
bool Finalize::identity() const {
  if (!sum.empty()) return false;
  for (size_t i = 0; i < perm.size(); ++i)
    if (perm[i] != i) return false;
  return true;
}

static size_t index_of(const std::vector<Leg>& v, Leg l) {
  return (size_t)(std::find(v.begin(), v.end(), l) - v.begin());
}

Plan compile_plan(const Network& net, const SsaPath& path) {
  net.validate();
  {
    std::set<Leg> o(net.output.begin(), net.output.end());
    if (o.size() != net.output.size()) fail("output contains a repeated leg");
  }
  PathStats stats = simulate_path(net, path);
  std::set<Leg> outs(net.output.begin(), net.output.end());
  std::map<Leg, u64> holders;
  for (auto& t : net.inputs)
    for (Leg l : uniq_sorted(t)) ++holders[l];

  Plan plan;
  plan.n_inputs = net.n_tensors();
  std::vector<std::vector<Leg>> slot;
  std::vector<char> alive;
  for (auto& legs0 : net.inputs) {
    InputPrep p;
    std::vector<Leg> legs = legs0;
    p.traces = plan_traces(legs, [&](Leg l) { return holders[l] > 1 || outs.count(l) > 0; });
    for (Leg l : legs0) p.input_shape.push_back(net.dim(l));
    for (Leg l : legs) p.shape.push_back(net.dim(l));
    p.legs = legs;
    plan.preps.push_back(std::move(p));
    slot.push_back(legs);
    alive.push_back(1);
  }
  auto dimprod = [&](const std::vector<Leg>& legs) {
    unsigned __int128 p = 1;
    for (Leg l : legs) {
      p *= net.dim(l);
      if (p > (unsigned __int128)UINT64_MAX) fail("GEMM dimension product overflows usize");
    }
    return (u64)p;
  };
  for (size_t s = 0; s < path.size(); ++s) {
    u64 ia = path[s].first, ib = path[s].second;
    if (ia == ib) fail("step " + std::to_string(s) + " contracts a tensor with itself");
    if (ia >= slot.size() || !alive[ia] || ib >= slot.size() || !alive[ib])
      fail("step " + std::to_string(s) + " references an invalid tensor");
    const std::vector<Leg> la = slot[ia], lb = slot[ib];
    alive[ia] = alive[ib] = 0;
    for (Leg l : la) --holders[l];
    for (Leg l : lb) --holders[l];
    auto keep = [&](Leg l) { return holders[l] > 0 || outs.count(l) > 0; };
    auto in = [](const std::vector<Leg>& v, Leg l) { return std::find(v.begin(), v.end(), l) != v.end(); };
    // src/compiled.rs:490-520: classify legs.
    std::vector<Leg> batch, con, free_a, free_b, drop_a, drop_b;
    for (Leg l : la) {
      if (in(lb, l)) (keep(l) ? batch : con).push_back(l);
      else (keep(l) ? free_a : drop_a).push_back(l);
    }
    for (Leg l : lb)
      if (!in(la, l)) (keep(l) ? free_b : drop_b).push_back(l);
    PairStep st;
    st.left_slot = ia;
    st.right_slot = ib;
    st.result_slot = slot.size();
    st.left_legs = la;
    st.right_legs = lb;
    std::vector<Leg> wa = la, wb = lb;
    for (Leg l : drop_a) { size_t ax = index_of(wa, l); st.sum_a.push_back(ax); wa.erase(wa.begin() + ax); }
    for (Leg l : drop_b) { size_t ax = index_of(wb, l); st.sum_b.push_back(ax); wb.erase(wb.begin() + ax); }
    for (Leg l : batch) st.a_perm.push_back(index_of(wa, l));
    for (Leg l : free_a) st.a_perm.push_back(index_of(wa, l));
    for (Leg l : con) st.a_perm.push_back(index_of(wa, l));
    for (Leg l : batch) st.b_perm.push_back(index_of(wb, l));
    for (Leg l : con) st.b_perm.push_back(index_of(wb, l));
    for (Leg l : free_b) st.b_perm.push_back(index_of(wb, l));
    st.bt = dimprod(batch);
    st.m = dimprod(free_a);
    st.k = dimprod(con);
    st.n = dimprod(free_b);
    check_gemm_geometry(st.bt, st.m, st.k, st.n);
    st.n_batch = batch.size();
    st.n_free_a = free_a.size();
    st.n_con = con.size();
    st.n_free_b = free_b.size();
    st.result_legs = batch;
    st.result_legs.insert(st.result_legs.end(), free_a.begin(), free_a.end());
    st.result_legs.insert(st.result_legs.end(), free_b.begin(), free_b.end());
    for (Leg l : st.result_legs) st.result_shape.push_back(net.dim(l));
    for (Leg l : la) st.left_shape.push_back(net.dim(l));
    for (Leg l : lb) st.right_shape.push_back(net.dim(l));
    for (Leg l : st.result_legs) ++holders[l];
    slot.push_back(st.result_legs);
    alive.push_back(1);
    plan.steps.push_back(std::move(st));
  }
  size_t n_alive = 0, last = 0;
  for (size_t i = 0; i < alive.size(); ++i)
    if (alive[i]) { ++n_alive; last = i; }
  if (n_alive != 1) fail("incomplete path: " + std::to_string(n_alive) + " tensors remain");
  Finalize& f = plan.fin;
  f.slot = last;
  std::vector<Leg> legs = slot[last];
  f.input_legs = legs;
  for (Leg l : legs) f.input_shape.push_back(net.dim(l));
  for (size_t i = 0; i < legs.size();) {
    if (!outs.count(legs[i])) { f.sum.push_back(i); legs.erase(legs.begin() + i); }
    else ++i;
  }
  if (uniq_sorted(legs) != uniq_sorted(net.output)) fail("final legs do not match the output legs");
  for (Leg l : net.output) { f.perm.push_back(index_of(legs, l)); f.output_shape.push_back(net.dim(l)); }
  plan.log10_flops = stats.log10_flops;
  plan.log2_peak_size = stats.log2_peak_size;
  return plan;
}

// ---------------------------------------------------------------- greedy
namespace {
struct Candidate {
  double cost;
  u64 a, b;
  bool operator>(const Candidate& o) const {
    if (cost != o.cost) return cost > o.cost;
    if (a != o.a) return a > o.a;
    return b > o.b;
  }
};
}  // namespace

SsaPath greedy_path(const Network& net) {
  net.validate();
  std::set<Leg> outs(net.output.begin(), net.output.end());
  std::map<Leg, u64> rc;
  std::map<Leg, std::set<u64>> hold;
  std::vector<std::vector<Leg>> legs;
  std::vector<double> size;
  std::vector<char> alive;
  auto linear_size = [&](const std::vector<Leg>& v) {
    double s = 0.0;
    for (Leg l : v) s += net.log2_dim(l);
    return std::exp2(s);
  };
  for (u64 i = 0; i < net.n_tensors(); ++i) {
    auto d = uniq_sorted(net.inputs[i]);
    for (Leg l : d) { ++rc[l]; hold[l].insert(i); }
    size.push_back(linear_size(d));
    legs.push_back(std::move(d));
    alive.push_back(1);
  }
  // Result legs of contracting a and b (src/path.rs:74-94).
  auto result_of = [&](u64 a, u64 b) {
    std::vector<Leg> r;
    for (Leg l : merge_union(legs[a], legs[b])) {
      u64 c = rc[l];
      c -= std::binary_search(legs[a].begin(), legs[a].end(), l);
      c -= std::binary_search(legs[b].begin(), legs[b].end(), l);
      if (c > 0 || outs.count(l)) r.push_back(l);
    }
    return r;
  };
  std::priority_queue<Candidate, std::vector<Candidate>, std::greater<Candidate>> heap;
  auto push = [&](u64 a, u64 b) { heap.push({linear_size(result_of(a, b)) - 1.0 * (size[a] + size[b]), a, b}); };
  {
    std::set<std::pair<u64, u64>> seen;
    for (auto& kv : hold) {
      std::vector<u64> h(kv.second.begin(), kv.second.end());
      for (size_t i = 0; i < h.size(); ++i)
        for (size_t j = i + 1; j < h.size(); ++j)
          if (seen.insert({h[i], h[j]}).second) push(h[i], h[j]);
    }
  }
  auto join = [&](u64 a, u64 b) {
    auto r = result_of(a, b);
    alive[a] = alive[b] = 0;
    for (Leg l : legs[a]) { --rc[l]; hold[l].erase(a); }
    for (Leg l : legs[b]) { --rc[l]; hold[l].erase(b); }
    u64 id = legs.size();
    for (Leg l : r) { ++rc[l]; hold[l].insert(id); }
    size.push_back(linear_size(r));
    legs.push_back(r);
    alive.push_back(1);
    std::set<u64> nb;
    for (Leg l : r)
      for (u64 h : hold[l])
        if (h != id) nb.insert(h);
    for (u64 x : nb) push(std::min(x, id), std::max(x, id));
    return id;
  };
  SsaPath path;
  while (!heap.empty()) {
    Candidate c = heap.top();
    heap.pop();
    if (!alive[c.a] || !alive[c.b]) continue;
    join(c.a, c.b);
    path.push_back({c.a, c.b});
  }
  // Disconnected components: smallest-first outer products (src/paths/greedy.rs:291-302).
  std::vector<u64> rest;
  for (u64 i = 0; i < legs.size(); ++i)
    if (alive[i]) rest.push_back(i);
  while (rest.size() > 1) {
    std::stable_sort(rest.begin(), rest.end(), [&](u64 x, u64 y) { return size[x] < size[y]; });
    u64 a = std::min(rest[0], rest[1]), b = std::max(rest[0], rest[1]);
    u64 id = join(a, b);
    path.push_back({a, b});
    rest.erase(rest.begin(), rest.begin() + 2);
    rest.push_back(id);
  }
  return path;
}

// ---------------------------------------------------------------- slicing
u64 slice_parallel_chunks(u64 n_slices, u64 out_numel) {
  const u64 max_chunks = 256, budget = 1ull << 22;  // src/slice.rs:921,924
  if (n_slices <= 1) return 1;
  u64 budget_chunks = std::max<u64>(budget / std::max<u64>(out_numel, 1), 1);
  u64 n0 = std::max<u64>(std::min({n_slices, max_chunks, budget_chunks}), 1);
  if (n0 <= 1) return 1;
  u64 chunk = (n_slices + n0 - 1) / n0;
  return (n_slices + chunk - 1) / chunk;
}

static bool sliceable(const Network& net, Leg leg, bool allow_output) {  // src/slice.rs:136-150
  auto it = net.size.find(leg);
  if (it == net.size.end() || it->second == 0) return false;
  if (!allow_output && std::find(net.output.begin(), net.output.end(), leg) != net.output.end()) return false;
  bool held = false;
  for (auto& t : net.inputs) {
    auto c = std::count(t.begin(), t.end(), leg);
    if (c > 1) return false;
    held |= c > 0;
  }
  return held;
}

void validate_slice_legs(const Network& net, const std::vector<Leg>& sliced) {
  std::set<Leg> seen;
  for (Leg l : sliced) {
    if (!seen.insert(l).second) fail("sliced leg " + std::to_string(l) + " appears twice");
    auto it = net.size.find(l);
    if (it == net.size.end()) fail("sliced leg " + std::to_string(l) + " is not in size_dict");
    if (it->second == 0) fail("sliced leg " + std::to_string(l) + " has dimension 0");
    bool held = false;
    for (auto& t : net.inputs) {
      auto c = std::count(t.begin(), t.end(), l);
      if (c > 1) fail("sliced leg " + std::to_string(l) + " is repeated inside one input tensor; not supported");
      held |= c > 0;
    }
    if (!held) fail("sliced leg " + std::to_string(l) + " is not held by any input tensor");
  }
}

namespace {
// Exact "product of dims <= target" without overflow (src/slice.rs:62-75).
bool legs_fit(const Network& cur, const std::vector<Leg>& legs, u64 target) {
  u64 rem = target;
  for (Leg l : legs) {
    u64 d = cur.dim(l);
    if (d > rem) return false;
    rem /= d;
  }
  return true;
}
}  // namespace

bool path_fits_target_size(const Network& net, const SsaPath& path, u64 target) {
  if (target == 0) fail("target_size must be greater than 0");
  std::vector<std::vector<Leg>> sl;
  simulate_path(net, path, &sl);
  if (net.n_tensors() == 1) return legs_fit(net, net.output, target);
  for (auto& legs : sl)
    if (!legs_fit(net, legs, target)) return false;
  return true;
}

PathStats sliced_path_stats(const Network& net, const SsaPath& path, const std::vector<Leg>& sliced) {
  validate_slice_legs(net, sliced);
  Network cur = net;
  for (Leg l : sliced) cur.size[l] = 1;
  return simulate_path(cur, path);
}

bool slice_result_fits_target_size(const Network& net, const SsaPath& path, const std::vector<Leg>& sliced,
                                   u64 target) {
  validate_slice_legs(net, sliced);
  Network cur = net;
  for (Leg l : sliced) cur.size[l] = 1;
  return path_fits_target_size(cur, path, target);
}

bool find_slices_to_size(const Network& net, const SsaPath& path, u64 target, std::vector<Leg>& out,
                         bool allow_output) {
  if (target == 0) return false;
  auto fits = [&](const Network& cur, const std::vector<Leg>& legs) { return legs_fit(cur, legs, target); };
  std::vector<Leg> sliced;
  for (;;) {
    Network cur = net;
    for (Leg l : sliced) cur.size[l] = 1;
    std::vector<std::vector<Leg>> sl;
    try {
      simulate_path(cur, path, &sl);
    } catch (Error&) {
      return false;
    }
    bool ok = true;
    if (cur.n_tensors() == 1) ok = fits(cur, cur.output);
    else
      for (auto& legs : sl)
        if (!fits(cur, legs)) { ok = false; break; }
    if (ok) { out = sliced; return true; }
    // src/slice.rs:557-589: most over-target intermediates, then larger leg, then smaller id.
    std::map<Leg, std::pair<u64, double>> score;
    // With output slicing, a unary contraction (no steps) still has its output to fit (src/slice.rs:565-566).
    if (allow_output && net.n_tensors() == 1) sl.push_back(cur.output);
    for (auto& legs : sl) {
      if (fits(cur, legs)) continue;
      for (Leg l : legs) {
        double d = cur.log2_dim(l);
        if (d <= 0.0 || !sliceable(net, l, allow_output)) continue;
        auto ins = score.emplace(l, std::make_pair(u64(0), d));
        ins.first->second.first += 1;
      }
    }
    if (score.empty()) return false;
    auto best = score.begin();
    for (auto it = std::next(score.begin()); it != score.end(); ++it) {
      const auto &s = it->second, &b = best->second;
      if (s.first > b.first || (s.first == b.first && s.second > b.second)) best = it;
      // equal (count, dim): keep the smaller leg id, which map order visits first
    }
    sliced.push_back(best->first);
    std::sort(sliced.begin(), sliced.end());
  }
}

}  // namespace ab2
