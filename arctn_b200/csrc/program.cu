// Device program: build (host) and execution (launch sequence / CUDA graph).
//
// Execution model.  Every slice of a sliced contraction runs the same plan
// (src/slice.rs:997-1016), so slices are executed as an extra batch dimension
// of each pairwise step rather than one after another.  A slot that holds no
// sliced leg is slice-invariant: the steps producing it run once, in a first
// phase, and their results are shared by all slices.  The remaining
// (slice-variant) steps run per group of S consecutive slices; each group's
// per-slice results are folded into FP64 chunk partials in the reference's
// deterministic chunk order (src/slice.rs:1020-1064, 1070-1173).
#include "program.hpp"

#include <algorithm>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <numeric>
#include <tuple>
#include <type_traits>
#include <set>

#include "tc_gemm.cuh"

namespace ab2 {

#define CK(x)                                                                                   \
  do {                                                                                          \
    cudaError_t e_ = (x);                                                                       \
    if (e_ != cudaSuccess) throw Error(E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

size_t dtype_bytes(int dt) {
  switch (dt) {
    case DT_F32: return 4;
    case DT_F64: return 8;
    case DT_C64: return 8;
    case DT_C128: return 16;
  }
  throw Error(E_INVALID, "unsupported dtype code " + std::to_string(dt));
}
static size_t wide_bytes(int dt) { return dtype_complex(dt) ? 16 : 8; }

namespace {

constexpr u64 kAlign = 256;
constexpr u64 kSpreadLimit = 64ull << 20;  // regions up to this size give every buffer its own bytes
constexpr u64 kInf = ~0ull;
// Split-K for tensor-core GEMMs.  Accuracy needs none (the kernel keeps TMEM chains short and sums
// them in registers), so K is split only to fill the GPU: an unsliced GEMM with fewer than two tiles
// per SM and a long K gets enough CTAs to cover the SMs twice, each taking at least kMinSplitTiles
// 16-wide K tiles; the FP32 partials are summed in FP64 in split order.
constexpr int kNumSMs = 148;
constexpr int kMinSplitTiles = 8;
inline u64 align_up(u64 x) { return (x + kAlign - 1) / kAlign * kAlign; }

// Per-slice strided view of a slot.
struct View {
  Ref ref;
  std::vector<u64> shape;
  std::vector<ll> strides;
  SliceOff so{};
  bool variant = false;
};

u64 prod(const std::vector<u64>& v) {
  unsigned __int128 p = 1;
  for (u64 x : v) {
    p *= x;
    if (p > (unsigned __int128)INT64_MAX) throw Error(E_UNSUPPORTED, "tensor element count exceeds the device index range");
  }
  return (u64)p;
}

// Offsets of every multi-index over (dims, strides), last axis fastest.
std::vector<ll> offsets(const std::vector<u64>& dims, const std::vector<ll>& strides) {
  const u64 n = prod(dims);
  std::vector<ll> out(n);
  std::vector<u64> idx(dims.size(), 0);
  ll off = 0;
  for (u64 e = 0; e < n; ++e) {
    out[e] = off;
    for (size_t d = dims.size(); d-- > 0;) {
      ++idx[d];
      off += strides[d];
      if (idx[d] < dims[d]) break;
      off -= strides[d] * (ll)dims[d];
      idx[d] = 0;
    }
  }
  return out;
}

std::vector<ll> rm_strides(const std::vector<u64>& shape) {
  std::vector<ll> s(shape.size(), 1);
  for (size_t i = shape.size(); i-- > 1;) s[i - 1] = s[i] * (ll)shape[i];
  return s;
}

// Axis indices left after removing `seq` one at a time (sum_axis order).
void split_removed(size_t rank, const std::vector<u64>& seq, std::vector<size_t>& kept, std::vector<size_t>& removed) {
  kept.resize(rank);
  std::iota(kept.begin(), kept.end(), 0);
  removed.clear();
  for (u64 r : seq) {
    removed.push_back(kept[r]);
    kept.erase(kept.begin() + r);
  }
}

template <class F>
void pick(const View& v, const std::vector<size_t>& axes, std::vector<u64>& dims, std::vector<ll>& strides, F&&) {
  dims.clear();
  strides.clear();
  for (size_t a : axes) { dims.push_back(v.shape[a]); strides.push_back(v.strides[a]); }
}

}  // namespace

Program::Program(const Network& net, const SsaPath& path, const std::vector<Leg>& sliced, const ProgramOptions& opt)
    : opt_(opt) {
  dtype_bytes(opt_.dtype);
  if (opt_.precision != PREC_FP32 && opt_.precision != PREC_TF32X3 && opt_.precision != PREC_BF16X3 &&
      opt_.precision != PREC_BF16X6)
    throw Error(E_INVALID, "unsupported precision mode " + std::to_string(opt_.precision));
  const u64 k_unit = opt_.precision == PREC_BF16X3 || opt_.precision == PREC_BF16X6 ? 2 * tc::BK : tc::BK;
  if (opt_.tc_k_chunk % k_unit != 0 || opt_.tc_k_chunk > (1ull << 30))
    throw Error(E_INVALID, "tc_k_chunk must be a multiple of " + std::to_string(k_unit) + " (0 for the default)");
  build(net, path, sliced);
  if (opt_.gradient && !sliced_) {
    // Over the workspace budget: drop the largest step results from what the adjoint sweep keeps
    // (it recomputes them) until the workspace fits, keeping the smallest layout seen.
    const u64 budget = opt_.workspace_budget ? opt_.workspace_budget : kDefaultBudget;
    if (ws_total_ > budget) {
      std::vector<size_t> cand;
      for (size_t s = 0; s < plan_.steps.size(); ++s)
        if (plan_.steps[s].result_slot != plan_.fin.slot) cand.push_back(s);
      std::stable_sort(cand.begin(), cand.end(), [&](size_t a, size_t b) {
        const PairStep &x = plan_.steps[a], &y = plan_.steps[b];
        return x.bt * x.m * x.n > y.bt * y.m * y.n;
      });
      std::set<size_t> best;
      u64 best_ws = ws_total_;
      for (size_t s : cand) {
        drop_.insert(s);
        build(net, path, sliced);
        if (ws_total_ < best_ws) { best_ws = ws_total_; best = drop_; }
        if (ws_total_ <= budget) break;
      }
      if (drop_ != best) {
        drop_ = best;
        build(net, path, sliced);
      }
    }
  }
  // Upload the offset tables now when a GPU is present (so a first execute may sit inside the caller's
  // stream capture); on a host without one the program stays inspectable (describe) and uploads on
  // its first execute.
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess) {
    cudaGetLastError();
    n_dev = 0;
  }
  if (n_dev > 0) {
    if (opt_.device < 0 || opt_.device >= n_dev)
      throw Error(E_INVALID, "device " + std::to_string(opt_.device) + " is not visible");
    int prev = 0;
    CK(cudaGetDevice(&prev));
    CK(cudaSetDevice(opt_.device));
    try {
      ensure_tables();
    } catch (...) {
      cudaSetDevice(prev);
      throw;
    }
    cudaSetDevice(prev);
  }
}

void Program::ensure_tables() {
  if (dev_tab_) return;
  cudaError_t e = cudaMalloc(&dev_tab_, std::max<size_t>(host_tab_.size(), 256));
  if (e == cudaSuccess) e = cudaMemcpy(dev_tab_, host_tab_.data(), host_tab_.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    if (dev_tab_) cudaFree(dev_tab_);
    dev_tab_ = nullptr;
    throw Error(E_CUDA, std::string("uploading offset tables: ") + cudaGetErrorString(e));
  }
}

Program::~Program() {
  if (!dev_tab_ && !gexec_ && side_.empty()) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(opt_.device);
  if (gexec_) cudaGraphExecDestroy(gexec_);
  if (dev_tab_) cudaFree(dev_tab_);
  for (auto e : ev_)
    if (e) cudaEventDestroy(e);
  for (auto e : join_ev_)
    if (e) cudaEventDestroy(e);
  if (fork_ev_) cudaEventDestroy(fork_ev_);
  for (auto s : side_)
    if (s) cudaStreamDestroy(s);
  cudaSetDevice(prev);
}

void Program::build(const Network& net, const SsaPath& path, const std::vector<Leg>& sliced) {
  ops_.clear();
  strip_ops_.clear();
  host_tab_.clear();
  net.validate();
  validate_slice_legs(net, sliced);
  const int dt = opt_.dtype;
  const u64 eb = dtype_bytes(dt);
  std::set<Leg> sl(sliced.begin(), sliced.end());
  std::vector<Leg> outer, internal;
  for (Leg l : net.output)
    if (sl.count(l)) outer.push_back(l);
  for (Leg l : sliced)
    if (std::find(outer.begin(), outer.end(), l) == outer.end()) internal.push_back(l);
  {
    unsigned __int128 t = 1;
    for (Leg l : sliced) {
      t *= net.dim(l);
      if (t > (unsigned __int128)UINT64_MAX) fail("slice count overflows usize");
    }
  }
  std::vector<u64> full_out_shape;
  for (Leg l : net.output) full_out_shape.push_back(net.dim(l));
  const u64 full_out_numel = checked_numel(full_out_shape);
  if (!outer.empty() && (unsigned __int128)full_out_numel * eb > (unsigned __int128)INT64_MAX)
    fail("the full output tensor's byte size exceeds the allocatable capacity");

  // Per-slice network: every sliced leg removed (src/slice.rs:990-996, 1113-1120).
  Network sub = net;
  for (auto& t : sub.inputs) t.erase(std::remove_if(t.begin(), t.end(), [&](Leg l) { return sl.count(l) > 0; }), t.end());
  sub.output.erase(std::remove_if(sub.output.begin(), sub.output.end(), [&](Leg l) { return sl.count(l) > 0; }), sub.output.end());
  for (Leg l : sliced) sub.size.erase(l);
  plan_ = compile_plan(sub, path);

  sliced_ = !sliced.empty();
  n_int_ = 1;
  for (Leg l : internal) n_int_ *= net.dim(l);
  n_blocks_ = 1;
  for (Leg l : outer) n_blocks_ *= net.dim(l);
  n_total_ = n_int_ * n_blocks_;
  range_begin_ = 0;
  range_end_ = n_total_;
  if (opt_.slice_begin || opt_.slice_end) {
    if (opt_.slice_end <= opt_.slice_begin || opt_.slice_end > n_total_)
      fail("slice range [" + std::to_string(opt_.slice_begin) + ", " + std::to_string(opt_.slice_end) +
           ") is outside [0, " + std::to_string(n_total_) + ")");
    range_begin_ = opt_.slice_begin;
    range_end_ = opt_.slice_end;
  }
  std::vector<u64> sub_out_shape;
  for (Leg l : sub.output) sub_out_shape.push_back(net.dim(l));
  const u64 n_e = std::max<u64>(prod(sub_out_shape), 1);
  n_chunks_ = internal.empty() ? 1 : slice_parallel_chunks(n_int_, n_e);

  double macs = 0;
  for (auto& st : plan_.steps) macs += (double)st.bt * st.m * st.k * st.n;
  flops_ = (dtype_complex(dt) ? 8.0 : 2.0) * macs * (double)(range_end_ - range_begin_);

  // ---------------------------------------------------------------- buffers / ops
  std::vector<Buf> bufs;
  std::vector<Op> ops1, ops2, strip1;
  bool fwd = true;  // ops emitted while true belong to the forward sweep (and its stripped variant)
  const bool want_strip = !sliced_;
  auto new_buf = [&](bool region2, u64 bytes, u64 first) {
    bufs.push_back(Buf{bytes, first, first, region2, 0});
    return (u64)bufs.size() - 1;
  };
  // A region-1 buffer read by a phase-2 op must outlive phase 1.
  auto touch = [&](const Ref& r, bool phase2, u64 at) {
    if (r.kind != Ref::WS) return;
    Buf& b = bufs[r.index];
    if (!b.region2 && phase2) b.last = kInf;
    else if (b.last != kInf) b.last = std::max(b.last, at);
  };
  auto tab_ll = [&](const std::vector<ll>& v) {
    u64 off = align_up(host_tab_.size());
    host_tab_.resize(off + v.size() * sizeof(ll));
    std::memcpy(host_tab_.data() + off, v.data(), v.size() * sizeof(ll));
    return off;
  };
  auto tab_i32 = [&](const std::vector<int>& v) {
    u64 off = align_up(host_tab_.size());
    host_tab_.resize(off + v.size() * sizeof(int));
    std::memcpy(host_tab_.data() + off, v.data(), v.size() * sizeof(int));
    return off;
  };
  std::vector<Op> ops3;  // after every group: the sliced adjoint's input-gradient finish
  int cur_gemm = -1, n_gemms = 0;  // ops emitted while a GEMM is being emitted serve it (packs, gathers)
  auto emit = [&](bool phase2, const Op& op0, bool also_strip) {
    Op op = op0;
    op.bwd = !fwd;
    op.gemm = cur_gemm;
    if (phase2) ops2.push_back(op);
    else {
      ops1.push_back(op);
      if (also_strip) strip1.push_back(op);
    }
  };
  auto opidx = [&](bool phase2) { return (u64)(phase2 ? ops2.size() : ops1.size()); };

  // Slice decode of every sliced leg: value = (g / div) % dim.
  std::map<Leg, std::pair<ll, ll>> decode;  // leg -> (div, mod)
  {
    ll div = 1;
    for (size_t q = internal.size(); q-- > 0;) { decode[internal[q]] = {div, (ll)net.dim(internal[q])}; div *= (ll)net.dim(internal[q]); }
    div = (ll)n_int_;
    for (size_t q = outer.size(); q-- > 0;) { decode[outer[q]] = {div, (ll)net.dim(outer[q])}; div *= (ll)net.dim(outer[q]); }
  }

  // FP64 partials [n_blocks][n_chunks][n_e] live through the whole run.
  u64 part_buf = kInf;
  if (sliced_) {
    part_buf = new_buf(false, n_blocks_ * n_chunks_ * n_e * wide_bytes(dt), 0);
    bufs[part_buf].last = kInf;
    Op z{Op::MEMSET};
    z.c = Ref{Ref::WS, part_buf};
    z.bytes = bufs[part_buf].bytes;
    emit(false, z, false);
  }
  // Device error word: bounded waits record where they gave up.
  const u64 err_buf = new_buf(false, 16, 0);
  bufs[err_buf].last = kInf;
  {
    Op z{Op::MEMSET};
    z.c = Ref{Ref::WS, err_buf};
    z.bytes = 16;
    emit(false, z, true);
  }
  if (want_strip) {
    u64 b = new_buf(false, 16, 0);
    bufs[b].last = kInf;
    strip_exp_off_ = b;  // patched to a byte offset after layout
    Op z{Op::MEMSET};
    z.c = Ref{Ref::WS, b};
    z.bytes = 16;
    strip1.push_back(z);
  }

  // ---------------------------------------------------------------- input views
  std::set<Leg> outs(net.output.begin(), net.output.end());
  std::map<Leg, u64> holders;
  for (auto& t : net.inputs) {
    std::set<Leg> u(t.begin(), t.end());
    for (Leg l : u) ++holders[l];
  }
  const size_t n_slots = plan_.n_inputs + plan_.steps.size();
  std::vector<View> view(n_slots);
  std::vector<Op> prep_gather(net.n_tensors(), Op{Op::MEMSET});  // kind GATHER where an input has traces
  for (size_t i = 0; i < net.n_tensors(); ++i) {
    struct Ax { u64 dim; ll stride; Leg leg; };
    std::vector<Ax> ax, red;
    std::vector<u64> shape0;
    for (Leg l : net.inputs[i]) shape0.push_back(net.dim(l));
    auto st0 = rm_strides(shape0);
    for (size_t a = 0; a < shape0.size(); ++a) ax.push_back({shape0[a], st0[a], net.inputs[i][a]});
    std::vector<Leg> legs = net.inputs[i];
    auto traces = plan_traces(legs, [&](Leg l) { return holders[l] > 1 || outs.count(l) > 0; });
    for (size_t t = 0; t < traces.size(); t += 3) {
      size_t ai = traces[t], aj = traces[t + 1];
      if (traces[t + 2]) {  // diagonal keeps axis ai and walks both strides
        ax[ai].stride += ax[aj].stride;
        ax.erase(ax.begin() + aj);
      } else {              // trace sums the diagonal and drops both axes
        red.push_back({ax[ai].dim, ax[ai].stride + ax[aj].stride, ax[ai].leg});
        ax.erase(ax.begin() + aj);
        ax.erase(ax.begin() + ai);
      }
    }
    View v;
    v.ref = Ref{Ref::INPUT, i};
    std::vector<u64> pdims;
    std::vector<ll> pstr;
    for (auto& a : ax) { pdims.push_back(a.dim); pstr.push_back(a.stride); }
    if (!traces.empty()) {
      // Materialise the prepared full tensor once (slice-invariant work).
      std::vector<u64> rd;
      std::vector<ll> rs;
      for (auto& r : red) { rd.push_back(r.dim); rs.push_back(r.stride); }
      u64 numel = prod(pdims);
      u64 b = new_buf(false, numel * eb, opidx(false));
      bufs[b].last = kInf;
      Op g{Op::GATHER};
      g.a = v.ref;
      g.c = Ref{Ref::WS, b};
      g.tab[0] = tab_ll(offsets(pdims, pstr));
      g.tab[1] = tab_ll(rd.empty() ? std::vector<ll>{0} : offsets(rd, rs));
      g.n_out = (ll)numel;
      g.n_red = rd.empty() ? 1 : (ll)prod(rd);
      g.S = 1;
      emit(false, g, true);
      prep_gather[i] = g;  // the reverse sweep scatters through the same tables
      v.ref = Ref{Ref::WS, b};
      pstr = rm_strides(pdims);
    }
    std::vector<std::pair<ll, std::pair<ll, ll>>> terms;  // (stride, (div, mod))
    for (size_t a = 0; a < ax.size(); ++a) {
      if (sl.count(ax[a].leg)) {
        auto dm = decode.at(ax[a].leg);
        terms.push_back({pstr[a], dm});
      } else {
        v.shape.push_back(pdims[a]);
        v.strides.push_back(pstr[a]);
      }
    }
    // Merge terms that address one contiguous run of sliced legs.
    std::sort(terms.begin(), terms.end(), [](auto& x, auto& y) { return x.second.first < y.second.first; });
    std::vector<SliceTerm> merged;
    for (auto& t : terms) {
      SliceTerm nt{t.second.first, t.second.second, t.first};
      if (!merged.empty()) {
        SliceTerm& p = merged.back();
        if (p.div * p.mod == nt.div && p.stride * p.mod == nt.stride) { p.mod *= nt.mod; continue; }
      }
      merged.push_back(nt);
    }
    if (merged.size() > (size_t)kMaxSliceTerms)
      throw Error(E_UNSUPPORTED, "input " + std::to_string(i) + " holds sliced legs that need more than " +
                                     std::to_string(kMaxSliceTerms) + " slice-offset terms");
    v.so.local_stride = 0;
    v.so.n = (int)merged.size();
    for (size_t t = 0; t < merged.size(); ++t) v.so.t[t] = merged[t];
    v.variant = !merged.empty();
    if (v.shape != plan_.preps[i].shape) throw Error(E_INVALID, "internal: prepared input shape mismatch");
    view[i] = v;
  }

  // ---------------------------------------------------------------- pairwise steps
  auto reduce_view = [&](View v, const std::vector<u64>& seq, bool phase2, Op* strip_dummy) -> View {
    (void)strip_dummy;
    if (seq.empty()) return v;
    std::vector<size_t> kept, removed;
    split_removed(v.shape.size(), seq, kept, removed);
    std::vector<u64> kd, rd;
    std::vector<ll> ks, rs;
    pick(v, kept, kd, ks, 0);
    pick(v, removed, rd, rs, 0);
    u64 numel = prod(kd);
    u64 b = new_buf(phase2, numel * eb, opidx(phase2));
    Op g{Op::GATHER};
    g.a = v.ref;
    g.sa = v.so;
    g.c = Ref{Ref::WS, b};
    g.tab[0] = tab_ll(offsets(kd, ks));
    g.tab[1] = tab_ll(offsets(rd, rs));
    g.n_out = (ll)numel;
    g.n_red = (ll)prod(rd);
    touch(v.ref, phase2, opidx(phase2));
    emit(phase2, g, fwd);
    View r;
    r.ref = g.c;
    r.shape = kd;
    r.strides = rm_strides(kd);
    r.so.local_stride = v.variant ? (ll)numel : 0;
    r.so.n = 0;
    r.variant = v.variant;
    return r;
  };

  // A GEMM operand read through offset tables: batch, rows (M of A / N of B) and K.
  struct Operand {
    Ref ref;
    SliceOff so;
    bool variant;
    std::vector<ll> tB, tR, tK;
    // per-leg dims and strides of the three groups, for the leg-aware pack
    std::vector<u64> dB, dR, dK;
    std::vector<ll> sB, sR, sK;
  };
  auto legs_of = [](const std::vector<u64>& d, const std::vector<ll>& s_, size_t lo, size_t hi) {
    return std::make_pair(std::vector<u64>(d.begin() + lo, d.begin() + hi), std::vector<ll>(s_.begin() + lo, s_.begin() + hi));
  };
  // Operand from (dims, strides) leg lists of its batch, row and K groups.
  auto make_operand = [&](Ref ref, SliceOff so, bool var, std::pair<std::vector<u64>, std::vector<ll>> b,
                          std::pair<std::vector<u64>, std::vector<ll>> r, std::pair<std::vector<u64>, std::vector<ll>> k) {
    Operand o;
    o.ref = ref;
    o.so = so;
    o.variant = var;
    o.tB = offsets(b.first, b.second);
    o.tR = offsets(r.first, r.second);
    o.tK = offsets(k.first, k.second);
    o.dB = b.first; o.sB = b.second;
    o.dR = r.first; o.sR = r.second;
    o.dK = k.first; o.sK = k.second;
    return o;
  };
  auto swap_rk = [](Operand o) {  // the same operand read with its row and K groups exchanged
    std::swap(o.tR, o.tK);
    std::swap(o.dR, o.dK);
    std::swap(o.sR, o.sK);
    return o;
  };
  // Leg-aware pack plan: destination strides are [z][rpad][kpad] with each group row-major.
  auto pack_plan = [&](const Operand& X, ll rpad, ll kpad, Op& p) -> bool {
    std::vector<u64> dims;
    std::vector<ll> ss, ds;
    auto add_group = [&](const std::vector<u64>& d, const std::vector<ll>& s_, ll unit) {
      auto rm = rm_strides(d);
      for (size_t i = 0; i < d.size(); ++i) {
        if (d[i] <= 1) continue;
        dims.push_back(d[i]);
        ss.push_back(s_[i]);
        ds.push_back(rm[i] * unit);
      }
    };
    add_group(X.dB, X.sB, rpad * kpad);
    add_group(X.dR, X.sR, kpad);
    add_group(X.dK, X.sK, 1);
    const size_t L = dims.size();
    std::vector<char> in_tile(L, 0);
    u64 T = 1;
    // Innermost legs of one side (by stride) until that side's contiguous run reaches `want` elements.
    auto take = [&](const std::vector<ll>& key, u64 want) {
      std::vector<size_t> order(L);
      std::iota(order.begin(), order.end(), 0);
      std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return key[a] < key[b]; });
      u64 covered = 1;  // product of this side's innermost legs already in the tile
      for (size_t i : order) {
        if (covered >= want) break;
        if (in_tile[i]) { covered *= dims[i]; continue; }
        if (T * dims[i] > (u64)tc::kPackTile) break;
        in_tile[i] = 1;
        T *= dims[i];
        covered *= dims[i];
      }
    };
    take(ss, 32);  // a warp's read covers 32 contiguous source elements
    take(ds, 32);  // and its write 32 contiguous floats of each plane
    take(ss, tc::kPackTile);  // then grow along the source to a full tile: fewer, longer tiles
    if (T < 32) return false;
    std::vector<u64> td, od;
    std::vector<ll> tss, tds, oss, ods;
    for (size_t i = 0; i < L; ++i) {
      if (in_tile[i]) { td.push_back(dims[i]); tss.push_back(ss[i]); tds.push_back(ds[i]); }
      else { od.push_back(dims[i]); oss.push_back(ss[i]); ods.push_back(ds[i]); }
    }
    const std::vector<ll> so_ = offsets(td, tss), do_ = offsets(td, tds);
    for (ll v : so_) if (v < 0 || v > INT32_MAX) return false;
    for (ll v : do_) if (v < 0 || v > INT32_MAX) return false;
    // Tile elements numbered by destination offset (rank); the read list in source-offset order.
    std::vector<int> rd(T), wr(T), rank(T);
    std::iota(rd.begin(), rd.end(), 0);
    std::iota(wr.begin(), wr.end(), 0);
    std::stable_sort(rd.begin(), rd.end(), [&](int a, int b) { return so_[a] < so_[b]; });
    std::stable_sort(wr.begin(), wr.end(), [&](int a, int b) { return do_[a] < do_[b]; });
    for (u64 r = 0; r < T; ++r) rank[wr[r]] = (int)r;
    std::vector<int> rd_rank(T), rd_off(T), wr_off(T);
    for (u64 i = 0; i < T; ++i) {
      rd_rank[i] = rank[rd[i]];
      rd_off[i] = (int)so_[rd[i]];
      wr_off[i] = (int)do_[wr[i]];
    }
    p.tab[0] = tab_i32(rd_rank);
    p.tab[1] = tab_i32(rd_off);
    p.tab[2] = tab_i32(wr_off);
    p.tab[4] = tab_ll(offsets(od, oss));
    p.tab[5] = tab_ll(offsets(od, ods));
    p.tile_T = (ll)T;
    p.n_outer = (ll)prod(od);
    return true;
  };
  // Emits C[s,b,i,j] = sum_l A(s,b,i,l) * B(s,b,l,j) into `out`.  Dense complex64 GEMMs under tf32x3
  // go through the planar pack (permute + split, conjugating on the fly) and the tcgen05 kernel.
  auto emit_gemm = [&](bool ph2, const Operand& A, const Operand& B, u64 bt, u64 m, u64 k, u64 n, Ref out,
                       bool conj_a, bool conj_b) {
    cur_gemm = n_gemms++;
    struct Done { int& c; ~Done() { c = -1; } } done{cur_gemm};
    auto rows_contiguous = [](const std::vector<ll>& r, const std::vector<ll>& c) {
      const bool r1 = r.size() > 1 && r[1] - r[0] == 1, c1 = c.size() > 1 && c[1] - c[0] == 1;
      return r1 && !c1;  // the pack then reads the source along rows
    };
    Op g{Op::GEMM_SMALL};
    g.tab[0] = tab_ll(A.tB);
    g.tab[1] = tab_ll(A.tR);
    g.tab[2] = tab_ll(A.tK);
    g.tab[3] = tab_ll(B.tB);
    g.tab[4] = tab_ll(B.tK);
    g.tab[5] = tab_ll(B.tR);
    g.bt = (ll)bt;
    g.m = (ll)m;
    g.k = (ll)k;
    g.n = (ll)n;
    g.a = A.ref;
    g.b = B.ref;
    g.sa = A.so;
    g.sb = B.so;
    g.c = out;
    g.conj_a = conj_a && dtype_complex(dt);
    g.conj_b = conj_b && dtype_complex(dt);
    // A long K over an output too small to give every SM a tile would run serially on a few SMs in the
    // tile kernels; one warp per output spreads the K loop over all of them instead.
    // A one-slice GEMM (phase 1) whose tile grid would leave SMs idle spreads its outputs over warps
    // instead: the tile kernels only win once every SM has a tile.  Phase-2 GEMMs are multiplied by
    // the slice group, so they keep the tile kernels.
    const u64 outs = bt * m * n;
    const u64 tiles64 = ((m + 63) / 64) * ((n + 63) / 64) * bt, tiles32 = ((m + 31) / 32) * ((n + 31) / 32) * bt;
    const bool long_k_few_tiles = k >= 1024 && tiles32 < 2 * (u64)kNumSMs && outs <= (1u << 17);
    if (outs <= 64 && k >= 256) g.kind = Op::GEMM_DOT;
    else if (long_k_few_tiles) g.kind = Op::GEMM_WARP;
    else if (dt == DT_F32 && m >= 128 && n >= 128 &&
             (ph2 || ((m + 127) / 128) * ((n + 127) / 128) * bt >= (u64)kNumSMs))
      g.kind = Op::GEMM_TILE128;  // large real FP32 steps: the 128 x 128 tile (same bits as the 64 x 64 one)
    else if (m >= 64 && n >= 64 && (ph2 || tiles64 >= (u64)kNumSMs)) g.kind = Op::GEMM_TILE64;
    else if (m >= 24 && n >= 24 && (ph2 || tiles32 >= (u64)kNumSMs)) g.kind = Op::GEMM_TILE32;
    else if (k >= 32) g.kind = Op::GEMM_WARP;  // a serial k loop per thread would dominate
    // A tuning table entry for this shape replaces the heuristic choice (SIMT kind, or the tensor core with
    // a given tile order / K split); the entry must name a variant this dtype and precision can run.
    g.key = GemmKey{dt, opt_.precision, ph2 ? 2 : 1, A.variant ? 1 : 0, B.variant ? 1 : 0, bt, m, k, n};
    const bool tc_allowed = (opt_.precision == PREC_TF32X3 || opt_.precision == PREC_BF16X3 ||
                             opt_.precision == PREC_BF16X6) && (dt == DT_C64 || dt == DT_F32);
    int forced = GV_AUTO;
    if (auto it = opt_.tuning.find(g.key); it != opt_.tuning.end()) forced = it->second;
    const bool forced_tc = forced == GV_TC_MFAST || forced == GV_TC_NFAST || forced == GV_TC_SPLITK ||
                           forced == GV_TC_STREAM || forced == GV_TC_DEEP || forced == GV_TC_PAIR ||
                           forced == GV_TC_PAIR_STREAM;
    if (forced == GV_TC_STREAM && opt_.precision != PREC_TF32X3)
      throw Error(E_INVALID, "tuning entry asks for the streaming-epilogue tensor-core GEMM, which is split-TF32 only");
    if ((forced == GV_TC_PAIR || forced == GV_TC_PAIR_STREAM) && opt_.precision != PREC_TF32X3)
      throw Error(E_INVALID, "tuning entry asks for the CTA-pair tensor-core GEMM, which is split-TF32 only");
    if (forced == GV_TC_DEEP && opt_.precision != PREC_TF32X3)
      throw Error(E_INVALID, "tuning entry asks for the deep-ring tensor-core GEMM, which is split-TF32 only");
    if (forced_tc && !tc_allowed)
      throw Error(E_INVALID, "tuning entry asks for the tensor-core GEMM, which needs precision tf32x3, bf16x3 or "
                             "bf16x6 and a float32 or complex64 network");
    if (forced == GV_TILE128 && dt != DT_F32) throw Error(E_INVALID, "tuning entry asks for the 128 x 128 tile, "
                                                                     "which is float32 only");
    switch (forced) {
      case GV_SMALL: g.kind = Op::GEMM_SMALL; break;
      case GV_TILE64: g.kind = Op::GEMM_TILE64; break;
      case GV_TILE32: g.kind = Op::GEMM_TILE32; break;
      case GV_WARP: g.kind = Op::GEMM_WARP; break;
      case GV_TILE128: g.kind = Op::GEMM_TILE128; break;
      case GV_DOT: g.kind = Op::GEMM_DOT; break;
      default: break;
    }
    g.tuned = forced != GV_AUTO;
    // Tensor cores for dense c64 steps; also for a small output side with a long K, where the padded
    // tile wastes MMA work but the K split (below) still fills the GPU.
    if (g.kind == Op::GEMM_DOT && k >= 16384) {
      // Too few outputs for the SMs: split each dot over CTAs (at least 2048 of k per CTA).
      const u64 outs = bt * m * n;
      const u64 parts = std::min<u64>((2 * kNumSMs + outs - 1) / outs, k / 2048);
      if (parts >= 2) {
        g.splits = (int)parts;
        g.kt_chunk = (int)((k + parts - 1) / parts);
        const u64 pbuf = new_buf(ph2, parts * outs * wide_bytes(dt), opidx(ph2));
        bufs[pbuf].fixed = ph2 && !(A.variant || B.variant);
        g.d = Ref{Ref::WS, pbuf};
        touch(g.d, ph2, opidx(ph2));
      }
    }
    // A single 16-wide K tile (no K split possible) only pays once the slice group or the batch gives
    // every SM an output tile; its epilogue can then write the next GEMM's packed operand directly.
    const u64 tc_tiles = ((m + tc::BM - 1) / tc::BM) * ((n + tc::BN - 1) / tc::BN) * bt;
    const bool six = opt_.precision == PREC_BF16X6;
    const bool bf16 = opt_.precision == PREC_BF16X3 || six;
    const ll planes = six ? 6 : tc::PLANES;  // planes per packed operand
    // Real float32 steps use the same complex kernel on half the K (Op::real): two of its four real
    // products per complex MAC are useful, still several times the FP32 SIMT rate.  (Holding the
    // mid-size ones back for the SIMT kernels measured slower on the many-network batch.)
    const u64 kc = (k + 1) / 2;
    bool real_tc = (opt_.precision == PREC_TF32X3 || bf16) && dt == DT_F32 && kc >= 32 &&
                   ((m >= 96 && n >= 96) || (std::min(m, n) >= 16 && kc >= 256));
    if (forced != GV_AUTO) real_tc = false;  // set again below when the pinned variant is a tensor-core one
    const bool heuristic_tc = real_tc || ((opt_.precision == PREC_TF32X3 || bf16) && dt == DT_C64 &&
                              ((k >= 32 && ((m >= 96 && n >= 96) || (std::min(m, n) >= 16 && k >= 256))) ||
                               (k >= 16 && m >= 96 && n >= 96 && (ph2 || tc_tiles >= (u64)kNumSMs))));
    const bool use_tc = forced == GV_AUTO ? heuristic_tc : forced_tc;
    if (forced_tc && dt == DT_F32) real_tc = true;  // a pinned tensor-core variant of a float32 step folds K
    g.variant = forced != GV_AUTO ? forced : GV_AUTO;
    if (!use_tc && g.variant == GV_AUTO) {
      switch (g.kind) {
        case Op::GEMM_SMALL: g.variant = GV_SMALL; break;
        case Op::GEMM_TILE64: g.variant = GV_TILE64; break;
        case Op::GEMM_TILE32: g.variant = GV_TILE32; break;
        case Op::GEMM_WARP: g.variant = GV_WARP; break;
        case Op::GEMM_TILE128: g.variant = GV_TILE128; break;
        case Op::GEMM_DOT: g.variant = GV_DOT; break;
        default: break;
      }
    }
    if (use_tc) {
      const ll kt_el = bf16 ? 2 * tc::BK : tc::BK;  // K per 64-byte packed row
      const ll el = bf16 ? 2 : 4;                  // bytes per plane element
      const ll kpk = real_tc ? (ll)kc : (ll)k;     // K of the complex product
      const ll kpad = (kpk + kt_el - 1) / kt_el * kt_el;
      const ll rpa = ((ll)m + tc::BM - 1) / tc::BM * tc::BM;
      const ll rpb = ((ll)n + tc::BN - 1) / tc::BN * tc::BN;
      // A phase-2 operand that is the whole unsplit output of an earlier tensor-core GEMM, read by nothing
      // else, is packed by that GEMM's epilogue: the offsets of the packed layout separate into a row
      // table, a column table and a batch table over the producer's row-major [bt][m][n] result.  Only
      // layouts without padding (nothing to zero first) qualify whose tables repeat from one output tile
      // to the next and whose packed runs inside a tile average at least 32 floats (coalesced stores).
      auto fuse_into_producer = [&](const Operand& X, ll rows, ll rpad, bool conj, u64 pbuf) -> bool {
        if (real_tc || bf16 || !ph2 || !X.variant || opt_.gradient || conj || X.ref.kind != Ref::WS || X.so.n != 0)
          return false;
        if (rows != rpad || (ll)k != kpad) return false;
        size_t pi = ops2.size();
        for (size_t q = ops2.size(); q-- > 0;)
          if (ops2[q].c.kind == Ref::WS && ops2[q].c.index == X.ref.index) { pi = q; break; }
        if (pi == ops2.size()) return false;
        auto reads_x = [&](const Ref& r) { return r.kind == Ref::WS && r.index == X.ref.index; };
        for (size_t q = pi + 1; q < ops2.size(); ++q) {
          const Op& o = ops2[q];
          if (reads_x(o.a) || reads_x(o.b) || reads_x(o.c) || reads_x(o.d) || reads_x(o.pk)) return false;
        }
        Op& P = ops2[pi];
        if (P.kind != Op::GEMM_TC || P.splits > 1 || P.pk.kind != Ref::NONE || P.bwd) return false;
        const ll mp = P.m, np = P.n, btp = P.bt, mn = mp * np;
        if (X.so.local_stride != btp * mn) return false;
        struct L { ll d, s, t; };
        std::vector<L> grp[3];  // producer columns, rows, batch
        auto add = [&](const std::vector<u64>& d, const std::vector<ll>& s_, ll unit) {
          auto rm = rm_strides(d);
          for (size_t q = 0; q < d.size(); ++q) {
            if (d[q] <= 1) continue;
            const ll sv = s_[q];
            grp[sv >= mn ? 2 : sv >= np ? 1 : 0].push_back(L{(ll)d[q], sv, rm[q] * unit});
          }
        };
        add(X.dB, X.sB, rpad * kpad);
        add(X.dR, X.sR, kpad);
        add(X.dK, X.sK, 1);
        const ll unit[3] = {1, np, mn}, extent[3] = {np, mn, btp * mn};
        for (int g = 0; g < 3; ++g) {  // each group must tile its index range exactly
          std::sort(grp[g].begin(), grp[g].end(), [](const L& x, const L& y) { return x.s < y.s; });
          ll expect = unit[g];
          for (const L& l : grp[g]) {
            if (l.s != expect) return false;
            expect *= l.d;
          }
          if (expect != extent[g]) return false;
        }
        auto table = [&](int g, ll count) {
          std::vector<ll> t((size_t)count, 0);
          for (ll x = 0; x < count; ++x)
            for (const L& l : grp[g]) t[(size_t)x] += ((x * unit[g] / l.s) % l.d) * l.t;
          return t;
        };
        const std::vector<ll> ti = table(1, mp), tj = table(0, np);
        auto periodic = [](const std::vector<ll>& t, ll tile) {
          for (size_t x = 0; x < t.size(); ++x)
            if (t[x] != t[x / tile * tile] + t[x % tile]) return false;
          return true;
        };
        if (!periodic(ti, tc::BM) || !periodic(tj, tc::BN)) return false;
        // The tile's elements in packed order must split into chunks of 32 consecutive packed floats
        // that share one (row, column) pattern relative to their first element.
        const ll tr = std::min<ll>(mp, tc::BM), tcn = std::min<ll>(np, tc::BN);
        std::vector<std::pair<ll, std::pair<ll, ll>>> walk;
        for (ll r = 0; r < tr; ++r)
          for (ll c = 0; c < tcn; ++c) walk.push_back({ti[r] + tj[c], {r, c}});
        std::sort(walk.begin(), walk.end());
        // The epilogue stages 32 output rows at a time, so every chunk must stay inside one such group.
        if (walk.size() % 32 || walk.back().first > INT32_MAX) return false;
        std::vector<int> lane(32);
        std::vector<std::vector<int>> by_quad(tc::BM / tc::kStageRows);  // pairs (r0 << 16 | c0, offset)
        for (size_t q = 0; q < walk.size(); q += 32) {
          const ll r0 = walk[q].second.first, c0 = walk[q].second.second;
          for (size_t l = 0; l < 32; ++l) {
            const ll dr = walk[q + l].second.first - r0, dc = walk[q + l].second.second - c0;
            if (walk[q + l].first != walk[q].first + (ll)l || dr < 0 || dc < 0) return false;
            if (r0 % tc::kStageRows + dr >= tc::kStageRows) return false;
            const int pat = (int)(dr << 16 | dc);
            if (q == 0) lane[l] = pat;
            else if (lane[l] != pat) return false;
          }
          auto& v = by_quad[(size_t)(r0 / tc::kStageRows)];
          v.push_back((int)(r0 << 16 | c0));
          v.push_back((int)walk[q].first);
        }
        std::vector<int> chunks;
        for (size_t q = 0; q < by_quad.size(); ++q) {
          P.pk_qbeg[q] = (int)(chunks.size() / 2);
          chunks.insert(chunks.end(), by_quad[q].begin(), by_quad[q].end());
        }
        P.pk_qbeg[by_quad.size()] = (int)(chunks.size() / 2);
        P.pk = Ref{Ref::WS, pbuf};
        P.pk_tab[0] = tab_ll(ti);
        P.pk_tab[1] = tab_ll(tj);
        P.pk_tab[2] = tab_ll(table(2, btp));
        P.pk_tab[3] = tab_i32(chunks);
        P.pk_tab[4] = tab_i32(lane);
        P.pk_rows = 1;
        for (int l : lane) P.pk_rows = std::max(P.pk_rows, (l >> 16) + 1);
        P.pk_slice = (ll)bt * rpad * kpad;
        // 16-byte stores need every chunk start 4-float aligned: tile bases (row / column tables at tile
        // starts, batch table), chunk offsets inside a tile, and the slice stride (the plane stride is a
        // multiple of it and the pack buffer is 256-byte aligned).
        {
          bool vec = P.pk_slice % 4 == 0;
          for (ll r = 0; r < mp && vec; r += tc::BM) vec = ti[(size_t)r] % 4 == 0;
          for (ll c = 0; c < np && vec; c += tc::BN) vec = tj[(size_t)c] % 4 == 0;
          for (ll v : table(2, btp)) vec = vec && v % 4 == 0;
          for (size_t q = 1; q < chunks.size() && vec; q += 2) vec = chunks[q] % 4 == 0;
          P.pk_vec = vec;
        }
        bufs[pbuf].first = std::min<u64>(bufs[pbuf].first, (u64)pi);
        P.c = Ref{};  // the plain result is never written
        bufs[X.ref.index].bytes = 0;
        return true;
      };
      auto pack = [&](const Operand& X, ll rows, ll rpad, bool conj) {
        const u64 pbuf = new_buf(ph2, (u64)(planes * (ll)bt * rpad * kpad * el), opidx(ph2));
        bufs[pbuf].fixed = ph2 && !X.variant;
        if (fuse_into_producer(X, rows, rpad, conj, pbuf)) return pbuf;
        Op p{Op::PACK};
        p.bf16 = bf16;
        p.six = six;
        p.a = X.ref;
        p.sa = X.so;
        p.c = Ref{Ref::WS, pbuf};
        p.bt = (ll)bt;
        p.rows = rows;
        p.cols = kpk;
        p.rpad = rpad;
        p.kpad = kpad;
        p.a_var = X.variant;
        p.conj_a = conj && (dtype_complex(dt) || real_tc);
        p.real = real_tc;
        p.kfull = (ll)k;
        touch(X.ref, ph2, opidx(ph2));
        if (!real_tc && pack_plan(X, rpad, kpad, p)) {
          p.kind = Op::PACK_TILED;
          if (rows < rpad || (ll)k < kpad) {  // the tiled pack writes only real elements: zero the padding
            Op z{Op::MEMSET};
            z.c = p.c;
            z.bytes = 0;  // set per launch from the group size (see launch_op)
            z.rpad = rpad;
            z.kpad = kpad;
            z.bt = (ll)bt;
            z.a_var = X.variant;
            z.bf16 = bf16;
            z.six = six;
            emit(ph2, z, fwd);
          }
        } else {
          p.tab[0] = tab_ll(X.tB);
          p.tab[1] = tab_ll(X.tR);
          p.tab[2] = tab_ll(X.tK);
          p.b_var = rows_contiguous(X.tR, X.tK);
        }
        emit(ph2, p, fwd);
        return pbuf;
      };
      // A real step packs B conjugated: Re((A1 + i A2) . conj(B1 + i B2)) = A1 . B1 + A2 . B2.
      const u64 pa = pack(A, (ll)m, rpa, real_tc ? false : conj_a);
      const u64 pb = pack(B, (ll)n, rpb, real_tc ? true : conj_b);
      touch(Ref{Ref::WS, pa}, ph2, opidx(ph2));
      // K split across CTAs (see TcArgs): partials [split][z][m][n].  A caller's tc_k_chunk fixes the
      // chunk; otherwise only a one-slice GEMM with too few tiles to fill the GPU is split.
      const int kt_total = (int)(kpad / kt_el);
      int chunk = kt_total;
      if (opt_.tc_k_chunk) {
        chunk = (int)std::max<ll>(1, (ll)opt_.tc_k_chunk / kt_el);
      } else if ((forced == GV_AUTO && !ph2) || forced == GV_TC_SPLITK) {
        const ll ctas = (rpa / tc::BM) * (rpb / tc::BN) * (ll)bt;
        const ll want = std::min<ll>((2 * kNumSMs + ctas - 1) / ctas, kt_total / kMinSplitTiles);
        if (want >= 2) chunk = (int)((kt_total + want - 1) / want);
      }
      if (kt_total > chunk) {
        g.kt_chunk = chunk;
        g.splits = (kt_total + chunk - 1) / chunk;
        const u64 pbuf = new_buf(ph2, (u64)g.splits * bt * m * n * 8, opidx(ph2));
        bufs[pbuf].fixed = ph2 && !(A.variant || B.variant);
        g.d = Ref{Ref::WS, pbuf};
        touch(g.d, ph2, opidx(ph2));
      }
      g.kind = Op::GEMM_TC;
      g.bf16 = bf16;
      g.six = six;
      g.real = real_tc;
      const ll mt = (ll)(m + tc::BM - 1) / tc::BM, nt = (ll)(n + tc::BN - 1) / tc::BN;
      g.raster = forced == GV_TC_MFAST ? 1 : forced == GV_TC_NFAST ? 0 : -1;
      g.stream = forced == GV_TC_STREAM || forced == GV_TC_PAIR_STREAM;
      g.deep = forced == GV_TC_DEEP;
      g.pair = forced == GV_TC_PAIR || forced == GV_TC_PAIR_STREAM;
      // Forward-only split-TF32 programs accumulate 64 of K per TMEM chain before the FP32 register sum (48 MMAs
      // per accumulator): fewer drains and a longer MMA run-ahead past each epilogue, measured about 8% faster on
      // the sliced headline's large steps for an error of 2.9e-6 instead of 2.5e-6 against FP64.  Gradient
      // programs keep 32 of K: their long-K adjoint GEMMs carry the tightest error budget (grid8: 7.9e-6).
      g.chunk_mul = (!opt_.gradient && opt_.precision == PREC_TF32X3) ? 2 : 1;
      if (g.deep && g.splits > 1) g.kt_chunk *= tc::BK / tc::kDeepBK;  // the deep ring's K tiles are 8 wide
      if (g.variant == GV_AUTO) g.variant = g.splits > 1 ? GV_TC_SPLITK : (mt <= nt ? GV_TC_MFAST : GV_TC_NFAST);
      g.a = Ref{Ref::WS, pa};
      g.b = Ref{Ref::WS, pb};
      if (real_tc)  // the complex product lands in a scratch buffer; a gather keeps its real part
        g.c = Ref{Ref::WS, new_buf(ph2, bt * m * n * 8, opidx(ph2))};
      g.rpad = rpa;
      g.rpad_b = rpb;
      g.kpad = kpad;
      g.a_var = A.variant;
      g.b_var = B.variant;
      g.conj_a = g.conj_b = false;  // conjugation happened in the packs
      touch(g.a, ph2, opidx(ph2));
      touch(g.b, ph2, opidx(ph2));
    }
    touch(A.ref, ph2, opidx(ph2));
    touch(B.ref, ph2, opidx(ph2));
    emit(ph2, g, fwd);
    if (g.real) {
      const u64 numel = bt * m * n;
      Op rg{Op::GATHER};  // out[s][e] = the real half of the complex result's element e
      rg.a = g.c;
      rg.sa.local_stride = ph2 ? (ll)(2 * numel) : 0;
      rg.c = out;
      std::vector<ll> re((size_t)numel);
      for (u64 e = 0; e < numel; ++e) re[(size_t)e] = (ll)(2 * e);
      rg.tab[0] = tab_ll(re);
      rg.tab[1] = tab_ll(std::vector<ll>{0});
      rg.n_out = (ll)numel;
      rg.n_red = 1;
      touch(g.c, ph2, opidx(ph2));
      emit(ph2, rg, fwd);
    }
    return g;
  };
  struct StepRec {
    Operand a, b;          // the GEMM operands of the forward step (after dangling sums, in perm order)
    std::vector<u64> da, db;  // their shapes in [batch, free_a, con] / [batch, con, free_b] order
  };
  std::vector<StepRec> recs;
  // One pairwise step on the current views of its operand slots: dangling sums, then the GEMM with
  // the step's permutes folded into its operand tables.  Returns the operands and the result view.
  auto step_operands = [&](size_t s, View A, View B) {
    const PairStep& st = plan_.steps[s];
    const Ref lref = A.ref, rref = B.ref;
    const bool ph2 = A.variant || B.variant;
    A = reduce_view(A, st.sum_a, ph2, nullptr);
    B = reduce_view(B, st.sum_b, ph2, nullptr);
    std::vector<u64> da, db;
    std::vector<ll> sa, sb;
    for (u64 p : st.a_perm) { da.push_back(A.shape[p]); sa.push_back(A.strides[p]); }
    for (u64 p : st.b_perm) { db.push_back(B.shape[p]); sb.push_back(B.strides[p]); }
    const size_t nb = st.n_batch, nfa = st.n_free_a, nc = st.n_con;
    Operand oa = make_operand(A.ref, A.so, A.variant, legs_of(da, sa, 0, nb), legs_of(da, sa, nb, nb + nfa),
                              legs_of(da, sa, nb + nfa, da.size()));
    Operand ob = make_operand(B.ref, B.so, B.variant, legs_of(db, sb, 0, nb), legs_of(db, sb, nb + nc, db.size()),
                              legs_of(db, sb, nb, nb + nc));
    touch(lref, ph2, opidx(ph2));
    touch(rref, ph2, opidx(ph2));
    return StepRec{oa, ob, da, db};
  };
  // Rank of each axis of step s's result in the packed operand layout of the step that reads it
  // ([batch][rows][K], outermost first); empty when a dangling sum or the final result reads it.
  auto consumer_rank = [&](size_t s) {
    const PairStep& st = plan_.steps[s];
    std::vector<size_t> rank;
    for (size_t c = s + 1; c < plan_.steps.size(); ++c) {
      const PairStep& u = plan_.steps[c];
      const bool left = u.left_slot == st.result_slot;
      if (!left && u.right_slot != st.result_slot) continue;
      if (!(left ? u.sum_a : u.sum_b).empty()) break;
      std::vector<u64> order;
      const auto& pm = left ? u.a_perm : u.b_perm;
      const size_t nb = u.n_batch, nc = u.n_con;
      if (left) order = pm;
      else {  // b_perm is [batch, con, free_b]; the pack lays out [batch, free_b, con]
        order.assign(pm.begin(), pm.begin() + nb);
        order.insert(order.end(), pm.begin() + nb + nc, pm.end());
        order.insert(order.end(), pm.begin() + nb, pm.begin() + nb + nc);
      }
      rank.assign(st.result_shape.size(), 0);
      for (size_t q = 0; q < order.size(); ++q) rank[order[q]] = q;
      break;
    }
    return rank;
  };
  // Each intermediate's physical leg order is free: rows and columns of a step's result are laid out
  // in the order its consumer packs them, so the consumer's contiguous runs fall inside one output
  // tile of the producer (the fused epilogue pack needs that; a separate pack reads longer runs).
  // Gradient programs keep the plan's order, which the adjoint sweep's operand views assume.
  auto reorder_result = [&](size_t s, StepRec& rec) {
    const PairStep& st = plan_.steps[s];
    std::vector<size_t> phys(st.result_shape.size());
    std::iota(phys.begin(), phys.end(), 0);
    const std::vector<size_t> rank = opt_.gradient ? std::vector<size_t>{} : consumer_rank(s);
    if (rank.empty()) return phys;
    const size_t nb = st.n_batch, nfa = st.n_free_a;
    auto regroup = [&](Operand& o, size_t lo, size_t hi) {
      std::vector<size_t> q(hi - lo);
      std::iota(q.begin(), q.end(), 0);
      std::stable_sort(q.begin(), q.end(), [&](size_t x, size_t y) { return rank[lo + x] < rank[lo + y]; });
      std::vector<u64> d;
      std::vector<ll> sv;
      for (size_t y = 0; y < q.size(); ++y) {
        d.push_back(o.dR[q[y]]);
        sv.push_back(o.sR[q[y]]);
        phys[lo + y] = lo + q[y];
      }
      o.dR = d;
      o.sR = sv;
      o.tR = offsets(d, sv);
    };
    regroup(rec.a, nb, nb + nfa);
    regroup(rec.b, nb + nfa, st.result_shape.size());
    return phys;
  };
  auto fwd_step = [&](size_t s, const View& A, const View& B, View& C) {
    const PairStep& st = plan_.steps[s];
    const bool ph2 = A.variant || B.variant;
    StepRec rec = step_operands(s, A, B);
    const std::vector<size_t> phys = reorder_result(s, rec);
    const u64 cnumel = prod({st.bt, st.m, st.n});
    const u64 cb = new_buf(ph2, cnumel * eb, opidx(ph2));
    emit_gemm(ph2, rec.a, rec.b, st.bt, st.m, st.k, st.n, Ref{Ref::WS, cb}, false, false);
    C.ref = Ref{Ref::WS, cb};
    C.shape = st.result_shape;
    C.strides.assign(phys.size(), 0);
    {
      ll stride = 1;
      for (size_t q = phys.size(); q-- > 0;) {
        C.strides[phys[q]] = stride;
        stride *= (ll)st.result_shape[phys[q]];
      }
    }
    C.so.local_stride = ph2 ? (ll)cnumel : 0;
    C.so.n = 0;
    C.variant = ph2;
    return rec;
  };

  for (size_t s = 0; s < plan_.steps.size(); ++s) {
    const PairStep& st = plan_.steps[s];
    View C;
    recs.push_back(fwd_step(s, view[st.left_slot], view[st.right_slot], C));
    const u64 cnumel = prod({st.bt, st.m, st.n});
    if (!C.variant && want_strip) {
      Op z{Op::MEMSET};
      z.c = Ref{Ref::WS, (u64)strip_exp_off_};
      z.bytes = 8;  // the max word (first 8 bytes); the exponent sits in the second 8
      strip1.push_back(z);
      Op mx{Op::MAXABS};
      mx.c = C.ref;
      mx.n_out = (ll)cnumel;
      mx.a = Ref{Ref::WS, (u64)strip_exp_off_};
      strip1.push_back(mx);
      Op sc{Op::STRIP};
      sc.c = C.ref;
      sc.n_out = (ll)cnumel;
      sc.a = Ref{Ref::WS, (u64)strip_exp_off_};
      strip1.push_back(sc);
    }
    view[st.result_slot] = C;
  }

  // ---------------------------------------------------------------- finalize
  const Finalize& fin = plan_.fin;
  View Fv = view[fin.slot];
  std::vector<size_t> kept, removed;
  split_removed(Fv.shape.size(), fin.sum, kept, removed);
  std::vector<u64> od, rd;
  std::vector<ll> os, rs;
  for (u64 p : fin.perm) { od.push_back(Fv.shape[kept[p]]); os.push_back(Fv.strides[kept[p]]); }
  pick(Fv, removed, rd, rs, 0);
  Op fg{Op::GATHER};
  fg.a = Fv.ref;
  fg.sa = Fv.so;
  fg.tab[0] = tab_ll(offsets(od, os));
  fg.tab[1] = tab_ll(rd.empty() ? std::vector<ll>{0} : offsets(rd, rs));
  fg.n_out = (ll)n_e;
  fg.n_red = rd.empty() ? 1 : (ll)prod(rd);
  const bool fin_ph2 = sliced_;
  touch(Fv.ref, fin_ph2, opidx(fin_ph2));
  u64 fbuf = kInf;
  if (!sliced_) {
    fg.c = Ref{Ref::OUTPUT, 0};
    emit(false, fg, true);
  } else {
    fbuf = new_buf(true, n_e * eb, opidx(true));
    fg.c = Ref{Ref::WS, fbuf};
    emit(true, fg, false);
    Op ac{Op::ACCUM};
    ac.a = Ref{Ref::WS, fbuf};
    ac.c = Ref{Ref::WS, part_buf};
    ac.n_e = (ll)n_e;
    touch(ac.a, true, opidx(true));
    emit(true, ac, false);
  }

  // ---------------------------------------------------------------- adjoint (reverse) sweep
  // Reverse-mode through the step loop with PyTorch's complex convention (grad = dL/d conj(x)):
  // for C = A.B:  dA = dC . conj(B)^T,  dB = conj(A)^T . dC, mapped back through the step's permutes,
  // broadcast over the legs the step summed away, then through the input traces / diagonals.
  if (opt_.gradient) {
    // Sliced programs run the reverse sweep inside every slice group, right after that group's forward
    // (phase 2, batched over the group's slices); each input's per-slice gradients then accumulate in
    // a wide buffer that is narrowed into the caller's gradient after the last group.
    const bool bph = sliced_;
    fwd = false;
    bwd_begin_ = ops1.size();
    // Forward values the sweep reads stay alive through the last op that reads them (touch).  Step
    // results listed in drop_ are not read from the forward: the sweep recomputes each of them from its
    // step's operands the first time it needs it, and the recomputed value then lives until its
    // consumer's adjoint step, so every dropped step runs at most once more.
    std::vector<char> have(n_slots, 0);
    std::vector<View> cur(view);
    for (size_t i = 0; i < n_slots; ++i) have[i] = i < plan_.n_inputs || !drop_.count(i - plan_.n_inputs);
    std::function<View(size_t)> value = [&](size_t slot) -> View {
      if (!have[slot]) {
        const size_t p = slot - plan_.n_inputs;
        const PairStep& ps = plan_.steps[p];
        const View L = value(ps.left_slot), R = value(ps.right_slot);
        fwd_step(p, L, R, cur[slot]);
        have[slot] = 1;
      }
      return cur[slot];
    };
    auto dropped = [&](size_t slot) { return slot >= plan_.n_inputs && drop_.count(slot - plan_.n_inputs) > 0; };
    std::vector<View> dv(n_slots);
    // A contiguous per-slice gradient buffer (one copy per slice of the group when sliced).
    auto contiguous = [&](u64 buf, const std::vector<u64>& shape) {
      View v;
      v.ref = Ref{Ref::WS, buf};
      v.shape = shape;
      v.strides = rm_strides(shape);
      v.so.local_stride = bph ? (ll)prod(shape) : 0;
      v.so.n = 0;
      v.variant = bph;
      return v;
    };
    // Final slot: the incoming gradient broadcast over finalize's summed legs, permuted to slot order.
    // A sliced program reads each slice's block of grad_output through its output-leg digits.
    {
      const auto& shp = fin.input_shape;
      auto full_st = rm_strides(full_out_shape);
      std::vector<ll> st(shp.size(), 0);
      std::vector<size_t> k2, r2;
      split_removed(shp.size(), fin.sum, k2, r2);
      for (size_t j = 0; j < k2.size(); ++j) {
        const Leg leg = fin.input_legs[k2[j]];
        const size_t q = std::find(net.output.begin(), net.output.end(), leg) - net.output.begin();
        st[k2[j]] = full_st[q];
      }
      const u64 numel = prod(shp);
      const u64 b = new_buf(bph, numel * eb, opidx(bph));
      Op g{Op::GATHER};
      g.a = Ref{Ref::GRAD_OUT, 0};
      g.c = Ref{Ref::WS, b};
      g.tab[0] = tab_ll(offsets(shp, st));
      g.tab[1] = tab_ll({0});
      g.n_out = (ll)numel;
      g.n_red = 1;
      if (bph) {
        g.sa.local_stride = 0;
        g.sa.n = 0;
        for (size_t q = 0; q < net.output.size(); ++q) {
          if (!sl.count(net.output[q])) continue;
          if (g.sa.n >= kMaxSliceTerms) throw Error(E_UNSUPPORTED, "too many sliced output legs for the adjoint");
          const auto dm = decode.at(net.output[q]);
          g.sa.t[g.sa.n++] = SliceTerm{dm.first, dm.second, full_st[q]};
        }
      }
      emit(bph, g, false);
      dv[fin.slot] = contiguous(b, shp);
    }
    // A GEMM result laid out in `order` dims (rm strides) seen in a slot's own leg order, broadcast over the
    // legs the forward step summed away (`sum_seq`, stride 0).  An intermediate slot's gradient stays this
    // strided view of the GEMM result: its one consumer, the adjoint of the step that produced the slot,
    // reads it through its operand tables.  An input's gradient is materialised contiguously when a sliced
    // accumulation or a trace scatter reads it; otherwise the final copy reads the view.
    auto to_slot = [&](u64 src_buf, const std::vector<u64>& order_dims, const std::vector<u64>& perm,
                       const std::vector<u64>& sum_seq, const std::vector<u64>& slot_shape, bool materialise) {
      const auto src_st = rm_strides(order_dims);
      std::vector<size_t> k2, r2;
      split_removed(slot_shape.size(), sum_seq, k2, r2);
      std::vector<ll> st(slot_shape.size(), 0);
      for (size_t j = 0; j < k2.size(); ++j) {
        const size_t p = std::find(perm.begin(), perm.end(), (u64)j) - perm.begin();
        st[k2[j]] = src_st[p];
      }
      if (!materialise) {
        View v;
        v.ref = Ref{Ref::WS, src_buf};
        v.shape = slot_shape;
        v.strides = st;
        v.so.local_stride = bph ? (ll)prod(order_dims) : 0;
        v.so.n = 0;
        v.variant = bph;
        return v;
      }
      const u64 numel = prod(slot_shape);
      const u64 b = new_buf(bph, numel * eb, opidx(bph));
      Op g{Op::GATHER};
      g.a = Ref{Ref::WS, src_buf};
      g.c = Ref{Ref::WS, b};
      g.tab[0] = tab_ll(offsets(slot_shape, st));
      g.tab[1] = tab_ll({0});
      g.n_out = (ll)numel;
      g.n_red = 1;
      g.sa.local_stride = bph ? (ll)prod(order_dims) : 0;
      g.sa.n = 0;
      touch(g.a, bph, opidx(bph));
      emit(bph, g, false);
      return contiguous(b, slot_shape);
    };
    // Input slots whose gradient a sliced accumulation or a trace scatter reads element by element.
    auto keep_dense = [&](u64 slot) {
      return slot < net.n_tensors() && (bph || prep_gather[(size_t)slot].kind == Op::GATHER);
    };
    for (size_t s = plan_.steps.size(); s-- > 0;) {
      const PairStep& st = plan_.steps[s];
      StepRec rec = recs[s];
      if (dropped(st.left_slot) || dropped(st.right_slot)) {
        const View L = value(st.left_slot), R = value(st.right_slot);
        StepRec r2 = step_operands(s, L, R);
        if (dropped(st.left_slot)) rec.a = r2.a;
        if (dropped(st.right_slot)) rec.b = r2.b;
      }
      const View dC = dv[st.result_slot];
      const size_t nb = st.n_batch, nfa = st.n_free_a;
      const auto& rsh = st.result_shape;
      const auto& rst = dC.strides;
      const auto dcB = legs_of(rsh, rst, 0, nb), dcM = legs_of(rsh, rst, nb, nb + nfa),
                 dcN = legs_of(rsh, rst, nb + nfa, rsh.size());
      // dA' [batch, free_a, con] = dC [batch, free_a, free_b] . conj(B') [batch, con, free_b]^T
      {
        Operand a = make_operand(dC.ref, dC.so, dC.variant, dcB, dcM, dcN);
        Operand b = swap_rk(rec.b);
        const u64 tbuf = new_buf(bph, prod({st.bt, st.m, st.k}) * eb, opidx(bph));
        emit_gemm(bph, a, b, st.bt, st.m, st.n, st.k, Ref{Ref::WS, tbuf}, false, true);
        dv[st.left_slot] = to_slot(tbuf, rec.da, st.a_perm, st.sum_a, st.left_shape, keep_dense(st.left_slot));
      }
      // dB' [batch, con, free_b] = conj(A') [batch, free_a, con]^T . dC [batch, free_a, free_b]
      {
        Operand a = swap_rk(rec.a);
        Operand b = make_operand(dC.ref, dC.so, dC.variant, dcB, dcN, dcM);
        const u64 tbuf = new_buf(bph, prod({st.bt, st.k, st.n}) * eb, opidx(bph));
        emit_gemm(bph, a, b, st.bt, st.k, st.m, st.n, Ref{Ref::WS, tbuf}, true, false);
        dv[st.right_slot] = to_slot(tbuf, rec.db, st.b_perm, st.sum_b, st.right_shape, keep_dense(st.right_slot));
      }
    }
    // Inputs: copy to the caller's gradient buffers, or scatter through an input's traces / diagonals.
    // Sliced: accumulate every slice's gradient of the (prepared) input into a wide buffer first.
    for (size_t i = 0; i < net.n_tensors(); ++i) {
      const View& d = dv[i];
      std::vector<u64> shape0;
      for (Leg l : net.inputs[i]) shape0.push_back(net.dim(l));
      const u64 numel0 = prod(shape0);
      const bool traced = prep_gather[i].kind == Op::GATHER;
      Ref src = d.ref;  // gradient of the prepared input: per slice (sliced) or whole
      if (bph) {
        // Prepared full shape (sliced axes included): the input itself, or the materialised prep.
        const u64 prep_numel = traced ? (u64)prep_gather[i].n_out : numel0;
        const u64 acc = new_buf(false, prep_numel * wide_bytes(dt), 0);
        bufs[acc].last = kInf;
        Op z{Op::MEMSET};
        z.c = Ref{Ref::WS, acc};
        z.bytes = prep_numel * wide_bytes(dt);
        emit(false, z, false);
        Op ga{Op::GRAD_ACCUM};
        ga.a = d.ref;
        ga.c = Ref{Ref::WS, acc};
        ga.sa = view[i].so;  // the input's slice terms over its prepared layout
        ga.tab[0] = tab_ll(offsets(view[i].shape, view[i].strides));
        ga.n_e = (ll)prod(view[i].shape);
        touch(ga.a, true, opidx(true));
        emit(true, ga, false);
        Op nw{Op::NARROW};
        nw.a = Ref{Ref::WS, acc};
        nw.n_out = (ll)prep_numel;
        if (!traced) {
          nw.c = Ref{Ref::GRADS, i};
          nw.bwd = true;
          ops3.push_back(nw);
          continue;
        }
        const u64 pb = new_buf(false, prep_numel * eb, 0);
        bufs[pb].last = kInf;
        nw.c = Ref{Ref::WS, pb};
        nw.bwd = true;
        ops3.push_back(nw);
        src = Ref{Ref::WS, pb};
      }
      if (!traced) {
        Op g{Op::GATHER};
        g.a = src;
        g.c = Ref{Ref::GRADS, i};
        g.tab[0] = tab_ll(offsets(shape0, bph ? rm_strides(shape0) : d.strides));
        g.tab[1] = tab_ll({0});
        g.n_out = (ll)numel0;
        g.n_red = 1;
        touch(g.a, false, opidx(false));
        emit(false, g, false);
      } else {
        Op z{Op::MEMSET};
        z.c = Ref{Ref::GRADS, i};
        z.bytes = numel0 * eb;
        z.bwd = true;
        Op sc = prep_gather[i];
        sc.kind = Op::SCATTER;
        sc.a = src;
        sc.c = Ref{Ref::GRADS, i};
        sc.bwd = true;
        if (bph) {
          ops3.push_back(z);
          ops3.push_back(sc);
        } else {
          emit(false, z, false);
          touch(sc.a, false, opidx(false));
          emit(false, sc, false);
        }
      }
    }
  }

  // ---------------------------------------------------------------- group size and layout
  u64 region1 = 0, per_slice2 = 0;
  // Buffers with overlapping lifetimes never share bytes; others may.  Sharing bytes orders the ops that
  // touch them in the graph, so a region whose buffers fit in kSpreadLimit without any sharing gets its own
  // bytes per buffer: independent steps then stay independent.
  auto layout = [&](bool region2, u64 mult) {
    std::vector<size_t> ids;
    for (size_t b = 0; b < bufs.size(); ++b)
      if (bufs[b].region2 == region2) ids.push_back(b);
    u64 spread = 0;
    for (size_t id : ids) spread += align_up(bufs[id].fixed ? bufs[id].bytes : bufs[id].bytes * mult);
    const u64 budget_cap = opt_.workspace_budget ? opt_.workspace_budget : kDefaultBudget;
    if (spread <= kSpreadLimit && spread <= budget_cap) {
      u64 off = 0;
      for (size_t id : ids) {
        bufs[id].offset = off;
        off += align_up(bufs[id].fixed ? bufs[id].bytes : bufs[id].bytes * mult);
      }
      return off;
    }
    std::sort(ids.begin(), ids.end(), [&](size_t x, size_t y) { return bufs[x].bytes > bufs[y].bytes || (bufs[x].bytes == bufs[y].bytes && x < y); });
    std::vector<size_t> placed;
    u64 top = 0;
    for (size_t id : ids) {
      Buf& b = bufs[id];
      const u64 sz = align_up(b.fixed ? b.bytes : b.bytes * mult);
      std::vector<std::pair<u64, u64>> busy;
      for (size_t p : placed) {
        const Buf& o = bufs[p];
        if (o.first <= b.last && b.first <= o.last)
          busy.push_back({o.offset, o.offset + align_up(o.fixed ? o.bytes : o.bytes * mult)});
      }
      std::sort(busy.begin(), busy.end());
      u64 off = 0;
      for (auto& iv : busy) {
        if (off + sz <= iv.first) break;
        off = std::max(off, iv.second);
      }
      b.offset = off;
      top = std::max(top, off + sz);
      placed.push_back(id);
    }
    return top;
  };
  region1 = layout(false, 1);
  per_slice2 = layout(true, 1);
  const u64 budget = opt_.workspace_budget ? opt_.workspace_budget : kDefaultBudget;
  S_ = 1;
  if (sliced_) {
    u64 room = budget > region1 ? budget - region1 : 0;
    const u64 n_range = range_end_ - range_begin_;
    u64 s_fit = per_slice2 ? std::max<u64>(room / (per_slice2 + kAlign), 1) : n_range;
    S_ = std::min<u64>(n_range, s_fit);
    if (opt_.max_slices_per_group) S_ = std::min<u64>(S_, opt_.max_slices_per_group);
    S_ = std::max<u64>(S_, 1);
  }
  const u64 region2 = sliced_ ? layout(true, S_) : 0;
  ws_total_ = align_up(region1) + region2;
  n_groups_ = sliced_ ? (range_end_ - range_begin_ + S_ - 1) / S_ : 1;

  auto resolve = [&](Ref& r) {
    if (r.kind != Ref::WS) return;
    const Buf& b = bufs[r.index];
    r.index = b.region2 ? align_up(region1) + b.offset : b.offset;
  };
  auto finish = [&](Op& op) {
    resolve(op.a);
    resolve(op.b);
    resolve(op.c);
    resolve(op.d);
    resolve(op.pk);
  };
  if (want_strip) strip_exp_off_ = bufs[strip_exp_off_].offset;
  err_off_ = bufs[err_buf].offset;
  // Memory footprint of an op of the main sequence, from its buffers before they are resolved to offsets.
  foot_.clear();
  auto note_foot = [&](const Op& op) {
    std::vector<Foot> f;
    auto add = [&](const Ref& r) {
      if (r.kind == Ref::WS) {
        const Buf& b = bufs[r.index];
        const u64 lo = b.region2 ? align_up(region1) + b.offset : b.offset;
        f.push_back(Foot{0, lo, lo + align_up(b.fixed ? b.bytes : b.bytes * (b.region2 ? S_ : 1))});
      } else if (r.kind == Ref::OUTPUT) {
        f.push_back(Foot{1, 0, ~0ull});
      } else if (r.kind == Ref::GRADS) {
        f.push_back(Foot{2 + (int)r.index, 0, ~0ull});
      }  // inputs and grad_output are only read
    };
    add(op.a);
    add(op.b);
    add(op.c);
    add(op.d);
    add(op.pk);
    if (op.kind == Op::GEMM_TC) f.push_back(Foot{0, err_off_, err_off_ + 8});  // its bounded waits report here
    foot_.push_back(f);
  };

  // ---------------------------------------------------------------- final op sequence
  for (Op op : ops1) { note_foot(op); finish(op); ops_.push_back(op); }
  if (want_strip) {
    for (Op op : strip1) { finish(op); strip_ops_.push_back(op); }
  }
  if (sliced_) {
    const ll chunk = (ll)((n_int_ + n_chunks_ - 1) / n_chunks_);
    for (u64 gi = 0; gi < n_groups_; ++gi) {
      const ll g0 = (ll)(range_begin_ + gi * S_), g1 = std::min<ll>(g0 + (ll)S_, (ll)range_end_);
      std::vector<ll> segs;  // triples (part, lo, hi)
      for (ll cur = g0; cur < g1;) {
        const ll blk = cur / (ll)n_int_, i = cur % (ll)n_int_, c = i / chunk;
        const ll end_i = std::min<ll>((c + 1) * chunk, (ll)n_int_);
        const ll run_end = std::min<ll>(blk * (ll)n_int_ + end_i, g1);
        segs.push_back(blk * (ll)n_chunks_ + c);
        segs.push_back(cur - g0);
        segs.push_back(run_end - g0);
        cur = run_end;
      }
      const u64 seg_tab = tab_ll(segs);
      for (Op op : ops2) {
        note_foot(op);
        finish(op);
        op.S = g1 - g0;
        op.g0 = g0;
        if (op.kind == Op::ACCUM) {
          op.tab[0] = seg_tab;
          op.n_segs = (ll)segs.size() / 3;
        }
        ops_.push_back(op);
      }
    }
    // Output assembly: block bases and the scatter of kept output axes.
    auto full_st = rm_strides(full_out_shape);
    std::vector<u64> odims;
    std::vector<ll> ostr, kstr;
    std::vector<u64> kdims;
    for (size_t a = 0; a < net.output.size(); ++a) {
      if (sl.count(net.output[a])) { odims.push_back(full_out_shape[a]); ostr.push_back(full_st[a]); }
      else { kdims.push_back(full_out_shape[a]); kstr.push_back(full_st[a]); }
    }
    Op out{Op::OUTPUT};
    out.a = Ref{Ref::WS, part_buf};
    out.c = Ref{Ref::OUTPUT, 0};
    note_foot(out);
    finish(out);
    out.tab[0] = tab_ll(odims.empty() ? std::vector<ll>{0} : offsets(odims, ostr));
    out.tab[1] = tab_ll(kdims.empty() ? std::vector<ll>{0} : offsets(kdims, kstr));
    out.n_blocks = (ll)n_blocks_;
    out.n_chunks = (ll)n_chunks_;
    out.n_e = (ll)n_e;
    ops_.push_back(out);
    for (Op op : ops3) {
      note_foot(op);
      finish(op);
      ops_.push_back(op);
    }
  }
  (void)fbuf;
  plan_dag();
}

void Program::plan_dag() {
  const size_t n = ops_.size();
  deps_.assign(n, {});
  waits_.assign(n, {});
  lane_.assign(n, 0);
  need_ev_.assign(n, 0);
  // Last toucher of every byte range, per space: disjoint segments lo -> (hi, op).
  std::map<int, std::map<u64, std::pair<u64, int>>> segs;
  for (size_t i = 0; i < n; ++i) {
    std::set<int> d;
    for (const Foot& f : foot_[i]) {
      if (f.hi <= f.lo) continue;
      auto& m = segs[f.space];
      auto it = m.upper_bound(f.lo);
      if (it != m.begin()) --it;
      std::vector<std::pair<u64, std::pair<u64, int>>> keep;
      while (it != m.end() && it->first < f.hi) {
        const u64 a = it->first, b = it->second.first;
        const int k = it->second.second;
        if (b <= f.lo) { ++it; continue; }
        if (k != (int)i) d.insert(k);
        if (a < f.lo) keep.push_back({a, {f.lo, k}});
        if (b > f.hi) keep.push_back({f.hi, {b, k}});
        it = m.erase(it);
      }
      for (auto& kv : keep) m.insert(kv);
      m[f.lo] = {f.hi, (int)i};
    }
    deps_[i].assign(d.begin(), d.end());
  }
  if (opt_.gradient) {  // gradient programs run op by op in program order: one unit per op, one lane
    units_.clear();
    unit_of_.assign(n, 0);
    for (size_t i = 0; i < n; ++i) {
      unit_of_[i] = (int)i;
      units_.push_back({(int)i});
    }
    waits_.assign(n, {});
    lane_.assign(n, 0);
    need_ev_.assign(n, 0);
    return;
  }
  // Levels of the op DAG; ops of one level are mutually independent.
  std::vector<int> level(n, 0);
  for (size_t i = 0; i < n; ++i)
    for (int d : deps_[i]) level[i] = std::max(level[i], level[(size_t)d] + 1);
  // Units: independent one-slice thin GEMMs of one level are grouped (same dtype for the whole program).
  auto groupable = [&](const Op& op) {
    return op.kind == Op::GEMM_SMALL && op.S == 1 && op.sa.n == 0 && op.sb.n == 0 && op.k <= 1024 &&
           op.bt * op.m * op.n <= (1ll << 20);
  };
  units_.clear();
  unit_of_.assign(n, -1);
  std::map<int, int> open;  // level -> unit being filled
  for (size_t i = 0; i < n; ++i) {
    if (groupable(ops_[i])) {
      auto it = open.find(level[i]);
      if (it != open.end() && units_[(size_t)it->second].size() < (size_t)kMaxGroup) {
        units_[(size_t)it->second].push_back((int)i);
        unit_of_[i] = it->second;
        continue;
      }
      open[level[i]] = (int)units_.size();
    }
    unit_of_[i] = (int)units_.size();
    units_.push_back({(int)i});
  }
  // Launch order: by level, then by first member (a topological order of the unit DAG).
  std::vector<int> order(units_.size());
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    return level[(size_t)units_[(size_t)x][0]] < level[(size_t)units_[(size_t)y][0]];
  });
  std::vector<std::vector<int>> sorted;
  std::vector<int> renum(units_.size());
  for (size_t u = 0; u < order.size(); ++u) {
    renum[(size_t)order[u]] = (int)u;
    sorted.push_back(units_[(size_t)order[u]]);
  }
  units_ = sorted;
  for (size_t i = 0; i < n; ++i) unit_of_[i] = renum[(size_t)unit_of_[i]];
  const size_t nu = units_.size();
  std::vector<std::vector<int>> udeps(nu);
  for (size_t u = 0; u < nu; ++u) {
    std::set<int> d;
    for (int i : units_[u])
      for (int x : deps_[(size_t)i]) d.insert(unit_of_[(size_t)x]);
    d.erase((int)u);
    udeps[u].assign(d.begin(), d.end());
  }
  // Lanes: continue the lane whose last unit is the latest dependency, else take the lane idle longest.
  waits_.assign(nu, {});
  lane_.assign(nu, 0);
  need_ev_.assign(nu, 0);
  std::vector<int> last(kLanes, -1);
  for (size_t u = 0; u < nu; ++u) {
    int lane = -1, best = -1;
    for (int d : udeps[u])
      if (last[lane_[(size_t)d]] == d && d > best) { best = d; lane = lane_[(size_t)d]; }
    if (lane < 0) {
      lane = 0;
      for (int l = 1; l < kLanes; ++l)
        if (last[l] < last[lane]) lane = l;
    }
    lane_[u] = lane;
    last[lane] = (int)u;
    for (int d : udeps[u])
      if (lane_[(size_t)d] != lane) {
        waits_[u].push_back(d);
        need_ev_[(size_t)d] = 1;
      }
  }
}

u64 Program::launches() const {  // kernels per execute: a split GEMM adds its reduce kernel
  u64 n = 0;
  for (size_t i = 0; i < ops_.size(); ++i) {
    const Op& op = ops_[i];
    // a grouped unit launches once, counted at its first member
    if (!units_.empty() && units_[(size_t)unit_of_[i]].size() > 1 && units_[(size_t)unit_of_[i]][0] != (int)i) continue;
    n += (op.kind != Op::MEMSET) + ((op.kind == Op::GEMM_TC || op.kind == Op::GEMM_DOT) && op.splits > 1);
  }
  return n;
}

// ---------------------------------------------------------------- launching
namespace {

inline int grid_for(ll total, int per_block = 256, int cap = 148 * 16) {
  ll g = (total + per_block - 1) / per_block;
  return (int)std::max<ll>(1, std::min<ll>(g, cap));
}

template <class T>
void launch_typed(const Op& op, const void* A, const void* B, void* C, void* D, const char* tab, bool out_f64,
                  cudaStream_t st) {
  using W = typename Num<T>::wide;
  auto T_ = [&](int i) { return (const ll*)(tab + op.tab[i]); };
  switch (op.kind) {
    case Op::GATHER: {
      const ll total = op.S * op.n_out;
      if (out_f64 && op.c.kind == Ref::OUTPUT)
        k_gather_reduce<T, W><<<grid_for(total), 256, 0, st>>>((const T*)A, (W*)C, T_(0), T_(1), op.n_out, op.n_red, op.S, op.sa, op.g0);
      else
        k_gather_reduce<T, T><<<grid_for(total), 256, 0, st>>>((const T*)A, (T*)C, T_(0), T_(1), op.n_out, op.n_red, op.S, op.sa, op.g0);
      break;
    }
    case Op::GEMM_SMALL:
    case Op::GEMM_DOT:
    case Op::GEMM_WARP:
    case Op::GEMM_TILE64:
    case Op::GEMM_TILE32:
    case Op::GEMM_TILE128: {
      GemmArgs g;
      g.A = A; g.B = B; g.C = C;
      g.bt = op.bt; g.m = op.m; g.k = op.k; g.n = op.n; g.S = op.S; g.g0 = op.g0;
      g.aB = T_(0); g.aM = T_(1); g.aK = T_(2); g.bB = T_(3); g.bK = T_(4); g.bN = T_(5);
      g.sa = op.sa; g.sb = op.sb;
      g.conj_a = op.conj_a ? 1 : 0;
      g.conj_b = op.conj_b ? 1 : 0;
      if (op.kind == Op::GEMM_SMALL) {
        const ll total = op.S * op.bt * op.m * op.n;
        const size_t smem = op.k <= 1024 ? (size_t)(2 * op.k * sizeof(ll)) : 0;
        k_gemm_small<T><<<grid_for(total, 256, 148 * 32), 256, smem, st>>>(g);
      } else if (op.kind == Op::GEMM_DOT && op.splits > 1) {
        const ll total = op.S * op.bt * op.m * op.n;
        k_gemm_dot_part<T><<<(int)std::min<ll>(total * op.splits, 148 * 16), 256, 0, st>>>(g, op.kt_chunk, op.splits,
                                                                                        (W*)D);
        k_dot_reduce<T><<<grid_for(total), 256, 0, st>>>((const W*)D, (T*)C, total, op.splits);
      } else if (op.kind == Op::GEMM_DOT) {
        const ll total = op.S * op.bt * op.m * op.n;
        k_gemm_dot<T><<<(int)std::min<ll>(total, 148 * 16), 256, 0, st>>>(g);
      } else if (op.kind == Op::GEMM_WARP) {
        const ll total = op.S * op.bt * op.m * op.n;
        k_gemm_warp<T><<<(int)std::min<ll>((total + 7) / 8, 148 * 16), 256, 0, st>>>(g);
      } else if (op.kind == Op::GEMM_TILE128) {
        if constexpr (std::is_same<T, float>::value) {
          const ll tiles = ((op.n + 127) / 128) * ((op.m + 127) / 128) * op.S * op.bt;
          k_gemm_tile128<<<(int)std::min<ll>(tiles, 148 * 2), 256, 0, st>>>(g);
        } else {
          throw Error(E_UNSUPPORTED, "the 128 x 128 tile GEMM is float32 only");
        }
      } else if (op.kind == Op::GEMM_TILE64) {
        const ll tiles = ((op.n + 63) / 64) * ((op.m + 63) / 64) * op.S * op.bt;
        k_gemm_tile<T, 64, 64, 16><<<(int)std::min<ll>(tiles, 148 * 8), 256, 0, st>>>(g);
      } else {
        const ll tiles = ((op.n + 31) / 32) * ((op.m + 31) / 32) * op.S * op.bt;
        k_gemm_tile<T, 32, 32, 16><<<(int)std::min<ll>(tiles, 148 * 16), 256, 0, st>>>(g);
      }
      break;
    }
    case Op::ACCUM: {
      const ll total = op.n_segs * op.n_e;
      k_slice_accumulate<T><<<grid_for(total), 256, 0, st>>>((const T*)A, (W*)C, (const Segment*)(tab + op.tab[0]), op.n_segs, op.n_e);
      break;
    }
    case Op::OUTPUT: {
      const ll total = op.n_blocks * op.n_e;
      if (out_f64)
        k_slice_output<T, W><<<grid_for(total), 256, 0, st>>>((const W*)A, (W*)C, T_(0), T_(1), op.n_blocks, op.n_chunks, op.n_e);
      else
        k_slice_output<T, T><<<grid_for(total), 256, 0, st>>>((const W*)A, (T*)C, T_(0), T_(1), op.n_blocks, op.n_chunks, op.n_e);
      break;
    }
    case Op::MAXABS:
      k_maxabs<T><<<grid_for(op.n_out), 256, 0, st>>>((const T*)C, op.n_out, (unsigned long long*)A);
      break;
    case Op::GRAD_ACCUM:
      k_grad_accum<T><<<grid_for(op.n_e), 256, 0, st>>>((const T*)A, (W*)C, T_(0), op.n_e, op.S, op.sa, op.g0);
      break;
    case Op::NARROW:
      k_narrow<T><<<grid_for(op.n_out), 256, 0, st>>>((const W*)A, (T*)C, op.n_out);
      break;
    case Op::SCATTER:
      k_scatter<T><<<grid_for(op.n_out * op.n_red), 256, 0, st>>>((const T*)A, (T*)C, T_(0), T_(1), op.n_out, op.n_red);
      break;
    case Op::STRIP:
      k_strip_scale<T><<<grid_for(op.n_out), 256, 0, st>>>((T*)C, op.n_out, (const unsigned long long*)A,
                                                             (double*)((char*)A + 8), 1);
      break;
    case Op::MEMSET:
      break;
  }
}

}  // namespace

namespace {

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiled)p;
  });
  if (!fn) throw Error(E_CUDA, "cuTensorMapEncodeTiled is unavailable from the driver");
  return fn;
}

// [re|im][z][rows][kpad] fp32 planes, boxes of 16 x 128 with 64-byte swizzle.
// Split-TF32 planes are fp32 (boxes of 16 x 128), split-BF16 planes bf16 (boxes of 32 x 128): 64-byte rows either way.
// The deep-ring kernel reads 8 of K per box (32-byte rows, 32-byte swizzle) from the same planes.
CUtensorMap plane_map(void* base, ll kpad, ll rows, ll zplanes, bool bf16, bool deep = false, int box_rows = tc::BM) {
  CUtensorMap m;
  const ll el = bf16 ? 2 : 4;
  cuuint64_t dims[3] = {(cuuint64_t)kpad, (cuuint64_t)rows, (cuuint64_t)zplanes};
  cuuint64_t strides[2] = {(cuuint64_t)(kpad * el), (cuuint64_t)(kpad * rows * el)};
  cuuint32_t box[3] = {(cuuint32_t)(deep ? tc::kDeepBK : bf16 ? 2 * tc::BK : tc::BK), (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = encode_fn()(&m, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base,
                           dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           deep ? CU_TENSOR_MAP_SWIZZLE_32B : CU_TENSOR_MAP_SWIZZLE_64B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(E_CUDA, "cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
  return m;
}

// Calls f with a value of the plane element type of op's packs: float (split-TF32), __nv_bfloat16 (split-BF16)
// or tc::bf16p3 (three BF16 pieces).
template <class Fn>
void with_plane_type(const Op& op, Fn&& f) {
  if (op.six) f(tc::bf16p3{});
  else if (op.bf16) f(__nv_bfloat16{});
  else f(0.f);
}

void launch_tc(const Op& op, void* A, void* B, void* C, void* D, void* PK, const char* tab, int* err,
               cudaStream_t st) {
  if (op.kind == Op::PACK) {
    const ll Z = (op.a_var ? op.S : 1) * op.bt;
    const ll tiles = Z * (op.rpad / 32) * ((op.kpad + 31) / 32);
    const int grid = (int)std::min<ll>(tiles, 148 * 16);
    const ll* t0 = (const ll*)(tab + op.tab[0]);
    const ll* t1 = (const ll*)(tab + op.tab[1]);
    const ll* t2 = (const ll*)(tab + op.tab[2]);
    with_plane_type(op, [&](auto tag) {
      using PT = decltype(tag);
      if (op.real)
        tc::k_pack_planar_real<PT><<<grid, 256, 0, st>>>((const float*)A, (PT*)C, t0, t1, t2, op.bt, op.rows, op.cols,
                                                         op.kfull, op.rpad, op.kpad, Z, op.sa, op.g0,
                                                         op.b_var ? 1 : 0, op.conj_a ? 1 : 0);
      else
        tc::k_pack_planar<PT><<<grid, 256, 0, st>>>((const cf32*)A, (PT*)C, t0, t1, t2, op.bt, op.rows, op.cols,
                                                    op.rpad, op.kpad, Z, op.sa, op.g0, op.b_var ? 1 : 0,
                                                    op.conj_a ? 1 : 0);
    });
    return;
  }
  if (op.kind == Op::PACK_TILED) {
    const ll n_slices = op.a_var ? op.S : 1;
    const ll slice_stride = op.bt * op.rpad * op.kpad;
    const ll plane = n_slices * slice_stride;
    const int grid = (int)std::min<ll>(op.n_outer * n_slices, 148 * 6);
    with_plane_type(op, [&](auto tag) {
      using PT = decltype(tag);
      tc::k_pack_tiled<PT><<<grid, tc::kPackThreads, 0, st>>>(
          (const cf32*)A, (PT*)C, (const int*)(tab + op.tab[0]), (const int*)(tab + op.tab[1]),
          (const int*)(tab + op.tab[2]), (int)op.tile_T, (const ll*)(tab + op.tab[4]), (const ll*)(tab + op.tab[5]),
          op.n_outer, n_slices, slice_stride, plane, op.sa, op.g0, op.conj_a ? 1 : 0);
    });
    return;
  }
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr_set[dev]) {
    const std::pair<decltype(&tc::k_tc_cgemm_tf32x3), int> kerns[7] = {
        {tc::k_tc_cgemm_tf32x3, tc::Fmt<tc::FMT_TF32X3>::kSmemBytes},
        {tc::k_tc_cgemm_bf16x3, tc::Fmt<tc::FMT_BF16X3>::kSmemBytes},
        {tc::k_tc_cgemm_bf16x6, tc::Fmt<tc::FMT_BF16X6>::kSmemBytes},
        {tc::k_tc_cgemm_tf32x3_stream, tc::kStreamSmemBytes},
        {tc::k_tc_cgemm_tf32x3_deep, tc::kDeepSmemBytes},
        {tc::k_tc_cgemm_tf32x3_pair, tc::kPairSmemBytes},
        {tc::k_tc_cgemm_tf32x3_pair_stream, tc::kPairStreamSmemBytes}};
    for (auto [kern, smem] : kerns) {
      CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
      // The kernel's setmaxnreg split assumes exactly kLaunchRegs registers a thread at launch.
      cudaFuncAttributes fa{};
      CK(cudaFuncGetAttributes(&fa, kern));
      if (fa.numRegs != tc::kLaunchRegs)
        throw Error(E_UNSUPPORTED, "tensor-core GEMM built with " + std::to_string(fa.numRegs) +
                                       " registers a thread, not " + std::to_string(tc::kLaunchRegs));
    }
    attr_set[dev] = true;
  }
  const ll s_eff = (op.a_var || op.b_var) ? op.S : 1;
  const ll za = (op.a_var ? op.S : 1) * op.bt, zb = (op.b_var ? op.S : 1) * op.bt;
  const ll planes = op.six ? 6 : tc::PLANES;
  const CUtensorMap ma = plane_map(A, op.kpad, op.rpad, planes * za, op.bf16, op.deep);
  // A pair's CTAs each load 64 of the tile's 128 B rows.
  const CUtensorMap mb = plane_map(B, op.kpad, op.rpad_b, planes * zb, op.bf16, op.deep, op.pair ? tc::BN / 2 : tc::BM);
  tc::TcArgs args;
  args.C = (cf32*)C;
  args.m = op.m;
  args.n = op.n;
  args.k_tiles = (int)(op.kpad / (op.deep ? tc::kDeepBK : op.bf16 ? 2 * tc::BK : tc::BK));
  args.chunk_tiles = (op.deep ? 4 : op.six ? 1 : tc::kChunkTiles) * op.chunk_mul;
  args.za = (int)za;
  args.zb = (int)zb;
  args.bt = (int)op.bt;
  args.a_var = op.a_var;
  args.b_var = op.b_var;
  args.err = err;
  if (PK) {
    args.pk = (float*)PK;
    args.pk_i = (const ll*)(tab + op.pk_tab[0]);
    args.pk_j = (const ll*)(tab + op.pk_tab[1]);
    args.pk_b = (const ll*)(tab + op.pk_tab[2]);
    args.pk_chunk = (const int2*)(tab + op.pk_tab[3]);
    args.pk_lane = (const int*)(tab + op.pk_tab[4]);
    for (int q = 0; q < 5; ++q) args.pk_qbeg[q] = op.pk_qbeg[q];
    args.pk_slice = op.pk_slice;
    args.pk_plane = s_eff * op.pk_slice;
    args.pk_vec = op.pk_vec && ((uintptr_t)PK & 15) == 0 ? 1 : 0;
  }
  const ll zc = s_eff * op.bt;
  args.zc = (int)zc;
  if (op.splits > 1) {
    args.kt_chunk = op.kt_chunk;
    args.part = (cf32*)D;
  }
  // The smaller operand's tiles run fastest, so it stays in L2 while the larger one streams once.  A CTA
  // pair's m-tiles are 256 rows.
  const ll tile_rows = op.pair ? 2 * tc::BM : tc::BM;
  const ll mt = (op.m + tile_rows - 1) / tile_rows, nt = (op.n + tc::BN - 1) / tc::BN;
  args.m_tiles = (int)mt;
  args.m_fast = op.raster >= 0 ? op.raster : (mt <= nt ? 1 : 0);
  const ll items = mt * nt * zc * op.splits;
  if (items > 0x7FFFFFFFll) throw Error(E_UNSUPPORTED, "tensor-core GEMM work items exceed 2^31");
  args.tiles = (int)(mt * nt);
  args.n_items = (int)items;
  static int sms[64] = {};
  if (dev < 64 && !sms[dev]) CK(cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev));
  const int n_sm = dev < 64 ? sms[dev] : 148;
  const unsigned grid = (unsigned)std::min<ll>(items, n_sm);
  if (op.pair) {
    // Clusters of two CTAs, as many as fit at once (persistent: each pair loops over items).
    static int pairs_fit[64][2] = {};
    const auto kern = op.stream ? tc::k_tc_cgemm_tf32x3_pair_stream : tc::k_tc_cgemm_tf32x3_pair;
    const int kv = op.stream ? 1 : 0;
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(tc::kThreads);
    cfg.dynamicSmemBytes = op.stream ? tc::kPairStreamSmemBytes : tc::kPairSmemBytes;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (dev < 64 && !pairs_fit[dev][kv]) {
      cfg.gridDim = dim3(2 * (unsigned)(n_sm / 2));
      int fit = 0;
      CK(cudaOccupancyMaxActiveClusters(&fit, kern, &cfg));
      if (fit < 1) throw Error(E_UNSUPPORTED, "no CTA pair of the tensor-core GEMM fits on this device");
      pairs_fit[dev][kv] = fit;
    }
    const ll fit = dev < 64 ? pairs_fit[dev][kv] : n_sm / 2;
    cfg.gridDim = dim3((unsigned)(2 * std::min<ll>(items, fit)));
    CK(cudaLaunchKernelEx(&cfg, kern, ma, mb, args));
  } else if (op.deep)
    tc::k_tc_cgemm_tf32x3_deep<<<grid, tc::kThreads, tc::kDeepSmemBytes, st>>>(ma, mb, args);
  else if (op.stream)
    tc::k_tc_cgemm_tf32x3_stream<<<grid, tc::kThreads, tc::kStreamSmemBytes, st>>>(ma, mb, args);
  else if (op.six)
    tc::k_tc_cgemm_bf16x6<<<grid, tc::kThreads, tc::Fmt<tc::FMT_BF16X6>::kSmemBytes, st>>>(ma, mb, args);
  else if (op.bf16)
    tc::k_tc_cgemm_bf16x3<<<grid, tc::kThreads, tc::Fmt<tc::FMT_BF16X3>::kSmemBytes, st>>>(ma, mb, args);
  else
    tc::k_tc_cgemm_tf32x3<<<grid, tc::kThreads, tc::Fmt<tc::FMT_TF32X3>::kSmemBytes, st>>>(ma, mb, args);
  if (op.splits > 1) {
    const ll count = zc * op.m * op.n;
    tc::k_splitk_reduce<<<grid_for(count), 256, 0, st>>>((const cf32*)D, (cf32*)C, count, op.splits);
  }
}

}  // namespace

void Program::launch_op(const Op& op, const void* const* inputs, void* output, char* ws, cudaStream_t st) {
  auto ptr = [&](const Ref& r) -> void* {
    switch (r.kind) {
      case Ref::INPUT: return const_cast<void*>(inputs[r.index]);
      case Ref::WS: return ws + r.index;
      case Ref::OUTPUT: return output;
      case Ref::GRAD_OUT: return const_cast<void*>(grad_out_);
      case Ref::GRADS: return grads_ ? grads_[r.index] : nullptr;
      default: return nullptr;
    }
  };
  if (op.kind == Op::MEMSET) {
    // bytes == 0: the padded planes of a tiled pack, [4 planes][slices of this group][bt][rpad][kpad] fp32
    const u64 bytes = op.bytes ? op.bytes
                               : (u64)((op.six ? 6 : tc::PLANES) * (op.a_var ? op.S : 1) * op.bt * op.rpad * op.kpad * (op.bf16 ? 2 : 4));
    CK(cudaMemsetAsync(ptr(op.c), 0, bytes, st));
    return;
  }
  if (op.kind == Op::PACK || op.kind == Op::PACK_TILED || op.kind == Op::GEMM_TC) {
    launch_tc(op, ptr(op.a), ptr(op.b), ptr(op.c), ptr(op.d), ptr(op.pk), dev_tab_, (int*)(ws + err_off_), st);
    CK(cudaGetLastError());
    return;
  }
  const bool out_f64 = out_f64_flag_;
  switch (opt_.dtype) {
    case DT_F32: launch_typed<float>(op, ptr(op.a), ptr(op.b), ptr(op.c), ptr(op.d), dev_tab_, out_f64, st); break;
    case DT_F64: launch_typed<double>(op, ptr(op.a), ptr(op.b), ptr(op.c), ptr(op.d), dev_tab_, out_f64, st); break;
    case DT_C64: launch_typed<cf32>(op, ptr(op.a), ptr(op.b), ptr(op.c), ptr(op.d), dev_tab_, out_f64, st); break;
    case DT_C128: launch_typed<cf64>(op, ptr(op.a), ptr(op.b), ptr(op.c), ptr(op.d), dev_tab_, out_f64, st); break;
  }
  CK(cudaGetLastError());
}

bool Program::in_part(size_t i, int part) const {
  return part == 0 || (part == 2 ? ops_[i].bwd : !ops_[i].bwd);
}

bool Program::interp_supported(size_t i) const {
  switch (ops_[i].kind) {
    case Op::GEMM_TC: case Op::PACK: case Op::PACK_TILED: case Op::MAXABS: case Op::STRIP: return false;
    default: return true;
  }
}

// The interpreter form of op i: the same body, sizes and pointers launch_op / launch_typed use.
void Program::interp_descs(size_t i, const void* const* inputs, const void* grad_out, void* const* grads,
                           void* output, char* ws, std::vector<IOp>& out) const {
  const Op& op = ops_[i];
  auto ptr = [&](const Ref& r) -> void* {
    switch (r.kind) {
      case Ref::INPUT: return inputs ? const_cast<void*>(inputs[r.index]) : nullptr;
      case Ref::WS: return ws ? ws + r.index : nullptr;
      case Ref::OUTPUT: return output;
      case Ref::GRAD_OUT: return const_cast<void*>(grad_out);
      case Ref::GRADS: return grads ? grads[r.index] : nullptr;
      default: return nullptr;
    }
  };
  auto T_ = [&](int q) { return dev_tab_ ? (const ll*)(dev_tab_ + op.tab[q]) : nullptr; };
  // Tasks of a step: about 1024 elements (4 a thread) per task for the elementwise kinds, fewer outputs for
  // the GEMMs by their K work; at most 512, which with a resident grid of ~2 CTAs an SM spreads one large
  // step over the whole GPU.
  auto tasks = [](ll work, ll per) { return (int)std::max<ll>(1, std::min<ll>((work + per - 1) / per, 512)); };
  IOp d{};
  d.dtype = opt_.dtype;
  d.a = ptr(op.a);
  d.c = ptr(op.c);
  d.d = ptr(op.d);
  auto gemm = [&]() {
    GemmArgs& g = d.g;
    g.A = ptr(op.a); g.B = ptr(op.b); g.C = ptr(op.c);
    g.bt = op.bt; g.m = op.m; g.k = op.k; g.n = op.n; g.S = op.S; g.g0 = op.g0;
    g.aB = T_(0); g.aM = T_(1); g.aK = T_(2); g.bB = T_(3); g.bK = T_(4); g.bN = T_(5);
    g.sa = op.sa; g.sb = op.sb;
    g.conj_a = op.conj_a ? 1 : 0;
    g.conj_b = op.conj_b ? 1 : 0;
  };
  const ll outs = op.S * op.bt * op.m * op.n;
  switch (op.kind) {
    case Op::GATHER:
      d.kind = I_GATHER;
      d.out_wide = 0;  // batches write outputs in the program's dtype
      d.t0 = T_(0); d.t1 = T_(1);
      d.n0 = op.n_out; d.n1 = op.n_red; d.n2 = op.S; d.n3 = op.g0;
      d.g.sa = op.sa;
      d.nvb = tasks(op.S * op.n_out * op.n_red, 1024);
      break;
    case Op::SCATTER:
      d.kind = I_SCATTER;
      d.t0 = T_(0); d.t1 = T_(1);
      d.n0 = op.n_out; d.n1 = op.n_red;
      d.nvb = tasks(op.n_out * op.n_red, 1024);
      break;
    case Op::GRAD_ACCUM:
      d.kind = I_GRAD_ACCUM;
      d.t0 = T_(0);
      d.n0 = op.n_e; d.n2 = op.S; d.n3 = op.g0;
      d.g.sa = op.sa;
      d.nvb = tasks(op.n_e * op.S, 1024);
      break;
    case Op::NARROW:
      d.kind = I_NARROW;
      d.n0 = op.n_out;
      d.nvb = tasks(op.n_out, 1024);
      break;
    case Op::ACCUM:
      d.kind = I_ACCUM;
      d.t0 = dev_tab_ ? (const ll*)(dev_tab_ + op.tab[0]) : nullptr;  // Segment triples
      d.n0 = op.n_segs; d.n1 = op.n_e;
      d.nvb = tasks(op.n_segs * op.n_e, 1024);
      break;
    case Op::OUTPUT:
      d.kind = I_OUTPUT;
      d.out_wide = 0;
      d.t0 = T_(0); d.t1 = T_(1);
      d.n0 = op.n_blocks; d.n1 = op.n_chunks; d.n2 = op.n_e;
      d.nvb = tasks(op.n_blocks * op.n_e * op.n_chunks, 1024);
      break;
    case Op::MEMSET:
      d.kind = I_MEMSET;
      d.n0 = (ll)(op.bytes ? op.bytes
                           : (u64)((op.six ? 6 : tc::PLANES) * (op.a_var ? op.S : 1) * op.bt * op.rpad * op.kpad * (op.bf16 ? 2 : 4)));
      d.nvb = tasks(d.n0, 256 * 16);
      break;
    case Op::GEMM_SMALL: gemm(); d.kind = I_GEMM_SMALL; d.nvb = tasks(outs * op.k, 8192); break;
    case Op::GEMM_WARP: gemm(); d.kind = I_GEMM_WARP; d.nvb = tasks(outs * op.k, 16384); break;
    case Op::GEMM_TILE64:
      gemm();
      d.kind = I_TILE64;
      d.nvb = tasks(((op.n + 63) / 64) * ((op.m + 63) / 64) * op.S * op.bt, 1);
      break;
    case Op::GEMM_TILE128:
      gemm();
      d.kind = I_TILE128;
      d.nvb = tasks(((op.n + 127) / 128) * ((op.m + 127) / 128) * op.S * op.bt, 1);
      break;
    case Op::GEMM_TILE32:
      gemm();
      d.kind = I_TILE32;
      d.nvb = tasks(((op.n + 31) / 32) * ((op.m + 31) / 32) * op.S * op.bt, 1);
      break;
    case Op::GEMM_DOT:
      gemm();
      if (op.splits > 1) {
        d.kind = I_DOT_PART;
        d.parts = op.splits;
        d.chunk = op.kt_chunk;
        d.nvb = tasks(outs * op.splits, 1);
        out.push_back(d);
        IOp r{};
        r.kind = I_DOT_REDUCE;
        r.dtype = opt_.dtype;
        r.a = ptr(op.d);
        r.c = ptr(op.c);
        r.n0 = outs;
        r.parts = op.splits;
        r.nvb = tasks(outs * op.splits, 1024);
        out.push_back(r);
        return;
      }
      d.kind = I_GEMM_DOT;
      d.nvb = tasks(outs, 1);
      break;
    default:
      throw Error(E_UNSUPPORTED, "the batch interpreter does not run this op kind");
  }
  out.push_back(d);
}

void Program::launch_one(size_t i, const void* const* inputs, const void* grad_out, void* const* grads,
                         void* output, char* ws, cudaStream_t st) {
  out_f64_flag_ = false;
  grad_out_ = grad_out;
  grads_ = grads;
  try {
    launch_op(ops_[i], inputs, output, ws, st);
  } catch (...) {
    grad_out_ = nullptr;
    grads_ = nullptr;
    throw;
  }
  grad_out_ = nullptr;
  grads_ = nullptr;
}

// One launch for a unit of independent one-slice thin GEMMs (k_gemm_small_grouped).
void Program::launch_group(const std::vector<int>& members, const void* const* inputs, void* output, char* ws,
                           cudaStream_t st) {
  auto ptr = [&](const Ref& r) -> const void* {
    switch (r.kind) {
      case Ref::INPUT: return inputs[r.index];
      case Ref::WS: return ws + r.index;
      case Ref::OUTPUT: return output;
      default: return nullptr;
    }
  };
  SmallGroup g;
  g.n = (int)members.size();
  int blocks = 0;
  ll kmax = 0;
  for (int q = 0; q < g.n; ++q) {
    const Op& op = ops_[(size_t)members[(size_t)q]];
    auto T_ = [&](int i) { return (const ll*)(dev_tab_ + op.tab[i]); };
    SmallProb& p = g.p[q];
    p.A = ptr(op.a);
    p.B = ptr(op.b);
    p.C = const_cast<void*>(ptr(op.c));
    p.aB = T_(0); p.aM = T_(1); p.aK = T_(2); p.bB = T_(3); p.bK = T_(4); p.bN = T_(5);
    p.bt = op.bt; p.m = op.m; p.k = op.k; p.n = op.n;
    p.conj_a = op.conj_a ? 1 : 0;
    p.conj_b = op.conj_b ? 1 : 0;
    p.block0 = blocks;
    blocks += (int)std::min<ll>((op.bt * op.m * op.n + 255) / 256, 148 * 32);
    kmax = std::max(kmax, op.k);
  }
  const size_t smem = (size_t)(2 * kmax * sizeof(ll));
  switch (opt_.dtype) {
    case DT_F32: k_gemm_small_grouped<float><<<blocks, 256, smem, st>>>(g); break;
    case DT_F64: k_gemm_small_grouped<double><<<blocks, 256, smem, st>>>(g); break;
    case DT_C64: k_gemm_small_grouped<cf32><<<blocks, 256, smem, st>>>(g); break;
    case DT_C128: k_gemm_small_grouped<cf64><<<blocks, 256, smem, st>>>(g); break;
  }
  CK(cudaGetLastError());
}

void Program::enqueue(const std::vector<Op>& ops, const void* const* inputs, void* output, char* ws, cudaStream_t st) {
  for (const Op& op : ops) launch_op(op, inputs, output, ws, st);
}

// The main sequence over kLanes streams, for capture into one graph whose edges are the op dependencies.
// Lane 0 is st; the side lanes join the capture through fork_ev_ and are joined back into st at the end.
void Program::ensure_lanes() {
  if (!side_.empty()) return;  // once per program, with its device current and outside any capture
  side_.resize(kLanes - 1, nullptr);
  for (auto& s : side_) CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&fork_ev_, cudaEventDisableTiming));
  join_ev_.resize(kLanes - 1, nullptr);
  for (auto& e : join_ev_) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  ev_.assign(units_.size(), nullptr);
  for (size_t u = 0; u < units_.size(); ++u)
    if (need_ev_[u]) CK(cudaEventCreateWithFlags(&ev_[u], cudaEventDisableTiming));
}

void Program::enqueue_dag(const void* const* inputs, void* output, char* ws, cudaStream_t st) {
  auto lane_stream = [&](int l) { return l == 0 ? st : side_[(size_t)l - 1]; };
  std::vector<char> used(kLanes, 0);
  used[0] = 1;
  CK(cudaEventRecord(fork_ev_, st));
  for (size_t u = 0; u < units_.size(); ++u) {
    const int l = lane_[u];
    cudaStream_t s = lane_stream(l);
    if (!used[l]) {
      CK(cudaStreamWaitEvent(s, fork_ev_, 0));
      used[l] = 1;
    }
    for (int d : waits_[u]) CK(cudaStreamWaitEvent(s, ev_[(size_t)d], 0));
    if (units_[u].size() == 1) launch_op(ops_[(size_t)units_[u][0]], inputs, output, ws, s);
    else launch_group(units_[u], inputs, output, ws, s);
    if (need_ev_[u]) CK(cudaEventRecord(ev_[u], s));
  }
  for (int l = 1; l < kLanes; ++l)
    if (used[l]) {
      CK(cudaEventRecord(join_ev_[(size_t)l - 1], side_[(size_t)l - 1]));
      CK(cudaStreamWaitEvent(st, join_ev_[(size_t)l - 1], 0));
    }
}

namespace {
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};
}  // namespace

void Program::execute(const void* const* inputs, void* output, bool f64_out, void* ws, u64 ws_bytes, cudaStream_t st) {
  if (ws_bytes < ws_total_)
    throw Error(E_WORKSPACE, "workspace of " + std::to_string(ws_bytes) + " bytes is smaller than the required " + std::to_string(ws_total_));
  if (!output) throw Error(E_INVALID, "output pointer is null");
  for (u64 i = 0; i < plan_.n_inputs; ++i)
    if (!inputs[i]) throw Error(E_INVALID, "input " + std::to_string(i) + " pointer is null");
  if (ws_total_ && !ws) throw Error(E_INVALID, "workspace pointer is null");
  DeviceGuard guard(opt_.device);
  std::lock_guard<std::mutex> lk(mu_);
  ensure_tables();
  out_f64_flag_ = f64_out;
  if (opt_.gradient) {  // plain execute of a gradient program: the forward ops only
    for (const Op& op : ops_)
      if (!op.bwd) launch_op(op, inputs, output, (char*)ws, st);
    return;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (st) CK(cudaStreamIsCapturing(st, &cs));
  const bool graph = opt_.use_graph && st != nullptr && cs == cudaStreamCaptureStatusNone;
  if (!graph) {
    enqueue(ops_, inputs, output, (char*)ws, st);
    return;
  }
  std::vector<const void*> key(inputs, inputs + plan_.n_inputs);
  key.push_back(output);
  key.push_back(ws);
  key.push_back((const void*)(uintptr_t)f64_out);
  if (!gexec_ || key != gkey_) {
    cudaGraph_t graph_h = nullptr;
    ensure_lanes();
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue_dag(inputs, output, (char*)ws, st);
    } catch (...) {
      cudaStreamEndCapture(st, &graph_h);
      if (graph_h) cudaGraphDestroy(graph_h);
      throw;
    }
    CK(cudaStreamEndCapture(st, &graph_h));
    bool updated = false;
    if (gexec_) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(gexec_, graph_h, &info) == cudaSuccess) updated = true;
      else {
        cudaGetLastError();
        cudaGraphExecDestroy(gexec_);
        gexec_ = nullptr;
      }
    }
    if (!updated) {
      cudaError_t e = cudaGraphInstantiate(&gexec_, graph_h, 0);
      if (e != cudaSuccess) {
        cudaGraphDestroy(graph_h);
        gexec_ = nullptr;
        throw Error(E_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
      }
    }
    cudaGraphDestroy(graph_h);
    gkey_ = key;
  }
  CK(cudaGraphLaunch(gexec_, st));
}

namespace {
double op_work(const Op& op, int dt) {
  const double eb = (double)dtype_bytes(dt);
  switch (op.kind) {
    case Op::GEMM_SMALL:
    case Op::GEMM_DOT:
    case Op::GEMM_WARP:
    case Op::GEMM_TC:
    case Op::GEMM_TILE64:
    case Op::GEMM_TILE32:
    case Op::GEMM_TILE128:
      return (dtype_complex(dt) ? 8.0 : 2.0) * (double)op.S * op.bt * op.m * op.k * op.n;
    case Op::GATHER: return (double)op.S * op.n_out * (op.n_red + 1) * eb;
    case Op::ACCUM: return (double)op.n_segs * op.n_e * (2.0 * wide_bytes(dt)) + (double)op.S * op.n_e * eb;
    case Op::OUTPUT: return (double)op.n_blocks * op.n_chunks * op.n_e * wide_bytes(dt);
    case Op::PACK:
    case Op::PACK_TILED:  // complex64 read once, four fp32 (or bf16) planes written (padding included)
      return (double)(op.a_var ? op.S : 1) * op.bt *
             (8.0 * op.rows * op.cols + (op.six ? 12.0 : op.bf16 ? 8.0 : 16.0) * op.rpad * op.kpad);
    default: return (double)op.n_out * eb;
  }
}
}  // namespace

void Program::profile(const void* const* inputs, void* output, void* ws, u64 ws_bytes, cudaStream_t st, float* ms,
                      int* kind, double* work, const void* grad_out, void* const* grads) {
  if (ws_bytes < ws_total_) throw Error(E_WORKSPACE, "workspace is smaller than required");
  if (opt_.gradient) check_run(0, inputs, grad_out, grads, output);
  DeviceGuard guard(opt_.device);
  std::lock_guard<std::mutex> lk(mu_);
  ensure_tables();
  out_f64_flag_ = false;
  grad_out_ = grad_out;
  grads_ = grads;
  struct Unbind {
    Program* p;
    ~Unbind() { p->grad_out_ = nullptr; p->grads_ = nullptr; }
  } unbind{this};
  // One entry per launch unit (a grouped unit is one launch; its work is its members' sum), in unit order.
  const size_t nu = units_.size();
  std::vector<cudaEvent_t> ev;
  for (size_t u = 0; u <= nu; ++u) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    ev.push_back(e);
  }
  try {
    for (size_t u = 0; u < nu; ++u) {
      CK(cudaEventRecord(ev[u], st));
      if (units_[u].size() == 1) launch_op(ops_[(size_t)units_[u][0]], inputs, output, (char*)ws, st);
      else launch_group(units_[u], inputs, output, (char*)ws, st);
    }
    CK(cudaEventRecord(ev[nu], st));
    CK(cudaEventSynchronize(ev[nu]));
    size_t j = 0;
    for (size_t u = 0; u < nu; ++u) {
      const Op& first = ops_[(size_t)units_[u][0]];
      if (first.kind == Op::MEMSET) continue;
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, ev[u], ev[u + 1]));
      double w = 0.0;
      for (int i : units_[u]) w += op_work(ops_[(size_t)i], opt_.dtype);
      ms[j] = t;
      kind[j] = (int)first.kind;
      work[j] = w;
      ++j;
    }
  } catch (...) {
    for (auto e : ev) cudaEventDestroy(e);
    throw;
  }
  for (auto e : ev) cudaEventDestroy(e);
}

u64 Program::forward_launches() const {
  u64 n = 0;
  for (const Op& op : ops_) n += !op.bwd && op.kind != Op::MEMSET;
  return n;
}

u64 Program::backward_launches() const {
  u64 n = 0;
  for (const Op& op : ops_) n += op.bwd && op.kind != Op::MEMSET;
  return n;
}

void Program::execute_gradient(int part, const void* const* inputs, const void* grad_out, void* const* grads,
                               void* output, void* ws, u64 ws_bytes, cudaStream_t st) {
  if (!opt_.gradient) throw Error(E_INVALID, "the program was built without gradient support");
  if (ws_bytes < ws_total_)
    throw Error(E_WORKSPACE, "workspace of " + std::to_string(ws_bytes) + " bytes is smaller than the required " +
                                 std::to_string(ws_total_));
  for (u64 i = 0; i < plan_.n_inputs; ++i)
    if (!inputs[i]) throw Error(E_INVALID, "input " + std::to_string(i) + " pointer is null");
  if (part != 2 && !output) throw Error(E_INVALID, "output pointer is null");
  if (part != 1) {
    if (!grad_out) throw Error(E_INVALID, "grad_output pointer is null");
    for (u64 i = 0; i < plan_.n_inputs; ++i)
      if (!grads || !grads[i]) throw Error(E_INVALID, "gradient buffer " + std::to_string(i) + " is null");
  }
  if (ws_total_ && !ws) throw Error(E_INVALID, "workspace pointer is null");
  DeviceGuard guard(opt_.device);
  std::lock_guard<std::mutex> lk(mu_);
  ensure_tables();
  out_f64_flag_ = false;
  grad_out_ = grad_out;
  grads_ = grads;
  if (sliced_ && part != 0)
    throw Error(E_UNSUPPORTED, "a sliced gradient program runs forward and reverse together (part 0): each slice "
                               "group's reverse sweep reuses that group's workspace");
  try {
    for (const Op& op : ops_)
      if (part == 0 || (part == 1) == !op.bwd) launch_op(op, inputs, output, (char*)ws, st);
  } catch (...) {
    grad_out_ = nullptr;
    grads_ = nullptr;
    throw;
  }
  grad_out_ = nullptr;
  grads_ = nullptr;
}

const char* gemm_variant_name(int v) {
  static const char* names[GV_COUNT] = {"auto", "simt_small", "simt_tile64", "simt_tile32", "simt_warp",
                                        "simt_tile128", "simt_dot", "tc_mfast", "tc_nfast", "tc_splitk", "tc_stream",
                                        "tc_deep", "tc_pair", "tc_pair_stream"};
  return v >= 0 && v < GV_COUNT ? names[v] : "?";
}

void Program::set_tc_chain(int k_per_chain) {
  if (k_per_chain != 32 && k_per_chain != 64 && k_per_chain != 128)
    throw Error(E_INVALID, "K per TMEM chain must be 32, 64 or 128");
  std::lock_guard<std::mutex> lk(mu_);
  for (auto* list : {&ops_, &strip_ops_})
    for (Op& op : *list)
      if (op.kind == Op::GEMM_TC && !op.bf16) op.chunk_mul = k_per_chain / 32;
  gkey_.clear();  // the captured graph holds the old launch parameters
}

std::vector<Program::GemmChoice> Program::gemm_choices() const {
  std::vector<GemmChoice> out;
  for (size_t i = 0; i < ops_.size(); ++i) {
    const Op& op = ops_[i];
    switch (op.kind) {
      case Op::GEMM_SMALL: case Op::GEMM_TILE64: case Op::GEMM_TILE32: case Op::GEMM_DOT: case Op::GEMM_TC:
      case Op::GEMM_WARP: case Op::GEMM_TILE128:
        out.push_back(GemmChoice{op.key, op.variant, op.tuned, i});
        break;
      default: break;
    }
  }
  return out;
}

std::string Program::describe() const {
  static const char* names[] = {"gather",    "gemm_small", "gemm_tile64", "gemm_tile32", "slice_accumulate",
                                "slice_output", "memset",  "maxabs",      "strip",       "gemm_tc",
                                "gemm_dot",  "pack",       "scatter",     "pack_tiled", "gemm_warp",  "grad_accum",
                                "narrow",    "gemm_tile128"};
  std::string s = "{\"workspace_bytes\":" + std::to_string(ws_total_) + ",\"n_slices\":" + std::to_string(n_total_) +
                  ",\"slice_begin\":" + std::to_string(range_begin_) + ",\"slice_end\":" + std::to_string(range_end_) +
                  ",\"slices_per_group\":" + std::to_string(S_) + ",\"groups\":" + std::to_string(n_groups_) +
                  ",\"launches\":" + std::to_string(launches()) + ",\"gradient\":" + (opt_.gradient ? "true" : "false") +
                  ",\"backward_begin\":" + std::to_string(opt_.gradient ? bwd_begin_ : ops_.size()) +
                  ",\"recomputed_steps\":[";
  bool first = true;
  for (size_t d : drop_) {
    s += (first ? "" : ",") + std::to_string(d);
    first = false;
  }
  s += "],\"ops\":[";
  for (size_t i = 0; i < ops_.size(); ++i) {
    const Op& op = ops_[i];
    s += std::string(i ? "," : "") + "{\"kind\":\"" + names[(int)op.kind] + "\"" + (op.bwd ? ",\"bwd\":1" : "");
    auto f = [&](const char* k, long long v) { s += std::string(",\"") + k + "\":" + std::to_string(v); };
    if (op.gemm >= 0) f("gemm", op.gemm);  // the GEMM (numbered in emit order) this op runs or serves
    // operands: reference kind (1 input, 2 workspace, 3 output, 4 grad_output, 5 grads) and index / offset
    f("a_kind", (long long)op.a.kind); f("a", (long long)op.a.index);
    if (op.b.kind != Ref::NONE) { f("b_kind", (long long)op.b.kind); f("b", (long long)op.b.index); }
    f("c_kind", (long long)op.c.kind); f("c", (long long)op.c.index);
    switch (op.kind) {
      case Op::GEMM_SMALL: case Op::GEMM_TILE64: case Op::GEMM_TILE32: case Op::GEMM_DOT: case Op::GEMM_TC:
      case Op::GEMM_WARP: case Op::GEMM_TILE128:
        f("S", op.S); f("bt", op.bt); f("m", op.m); f("k", op.k); f("n", op.n);
        f("splits", op.splits); f("conj_a", op.conj_a); f("conj_b", op.conj_b);
        if (op.pk.kind != Ref::NONE) {
          f("pack_into", (long long)op.pk.index);
          f("pack_vec", op.pk_vec ? 1 : 0);
          f("pack_chunk_rows", op.pk_rows);
        }
        if (op.kind == Op::GEMM_TC) {
          f("bf16", op.bf16); f("bf16x6", op.six); f("real", op.real);
          f("tmem_chunk_k", (op.bf16 && !op.six ? 64 : 32) * op.chunk_mul);  // K per TMEM chain, then FP32 sums
        }
        s += std::string(",\"variant\":\"") + gemm_variant_name(op.variant) + "\"";
        f("tuned", op.tuned ? 1 : 0);
        f("phase", op.key.phase); f("a_var", op.key.a_var); f("b_var", op.key.b_var);
        break;
      case Op::PACK: case Op::PACK_TILED:
        f("S", op.a_var ? op.S : 1); f("bt", op.bt); f("rows", op.rows); f("cols", op.cols); f("rpad", op.rpad);
        f("kpad", op.kpad); f("tile", op.tile_T); f("n_outer", op.n_outer); f("bf16", op.bf16); f("bf16x6", op.six);
        f("real", op.real);
        break;
      case Op::GATHER: case Op::SCATTER: case Op::MAXABS: case Op::STRIP:
        f("S", op.S); f("n_out", op.n_out); f("n_red", op.n_red);
        break;
      case Op::MEMSET: f("bytes", (long long)op.bytes); break;
      default: f("n_e", op.n_e); break;
    }
    // graph DAG: lane, the ops it must follow, and its footprint [space, lo, hi) (hi = -1: unbounded)
    if (i < unit_of_.size()) {
      f("unit", unit_of_[i]);
      f("lane", lane_[(size_t)unit_of_[i]]);
      s += ",\"deps\":[";
      for (size_t q = 0; q < deps_[i].size(); ++q) s += (q ? "," : "") + std::to_string(deps_[i][q]);
      s += "],\"foot\":[";
      for (size_t q = 0; q < foot_[i].size(); ++q) {
        const Foot& ft = foot_[i][q];
        s += std::string(q ? "," : "") + "[" + std::to_string(ft.space) + "," + std::to_string(ft.lo) + "," +
             (ft.hi == ~0ull ? std::string("-1") : std::to_string(ft.hi)) + "]";
      }
      s += "]";
    }
    s += "}";
  }
  return s + "]}";
}

void Program::check_run(int part, const void* const* inputs, const void* grad_out, void* const* grads,
                        const void* output) const {
  if (part < -1 || part > 2) throw Error(E_INVALID, "gradient part must be 0, 1 or 2");
  if (part >= 0 && !opt_.gradient) throw Error(E_INVALID, "the program was built without gradient support");
  if (sliced_ && (part == 1 || part == 2))
    throw Error(E_UNSUPPORTED, "a sliced gradient program runs forward and reverse together (part 0)");
  if (!inputs) throw Error(E_INVALID, "inputs pointer is null");
  for (u64 i = 0; i < plan_.n_inputs; ++i)
    if (!inputs[i]) throw Error(E_INVALID, "input " + std::to_string(i) + " pointer is null");
  if (part != 2 && !output) throw Error(E_INVALID, "output pointer is null");
  if (part == 0 || part == 2) {
    if (!grad_out) throw Error(E_INVALID, "grad_output pointer is null");
    for (u64 i = 0; i < plan_.n_inputs; ++i)
      if (!grads || !grads[i]) throw Error(E_INVALID, "gradient buffer " + std::to_string(i) + " is null");
  }
}

void Program::enqueue_part(int part, const void* const* inputs, const void* grad_out, void* const* grads,
                           void* output, void* ws, cudaStream_t st) {
  out_f64_flag_ = false;
  grad_out_ = grad_out;
  grads_ = grads;
  try {
    for (const Op& op : ops_) {
      const bool run = part == 0 || (part == 2 ? op.bwd : !op.bwd);
      if (run) launch_op(op, inputs, output, (char*)ws, st);
    }
  } catch (...) {
    grad_out_ = nullptr;
    grads_ = nullptr;
    throw;
  }
  grad_out_ = nullptr;
  grads_ = nullptr;
}

int Program::device_status(void* ws, cudaStream_t st) {
  DeviceGuard guard(opt_.device);
  int code = 0;
  CK(cudaMemcpyAsync(&code, (char*)ws + err_off_, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return code;
}

void Program::execute_stripped(const void* const* inputs, void* output, void* ws, u64 ws_bytes, cudaStream_t st,
                               double* exponent) {
  if (sliced_) throw Error(E_UNSUPPORTED, "execute_stripped applies to unsliced programs only");
  if (ws_bytes < ws_total_) throw Error(E_WORKSPACE, "workspace is smaller than required");
  DeviceGuard guard(opt_.device);
  std::lock_guard<std::mutex> lk(mu_);
  ensure_tables();
  out_f64_flag_ = false;
  enqueue(strip_ops_, inputs, output, (char*)ws, st);
  double e = 0.0;
  CK(cudaMemcpyAsync(&e, (char*)ws + strip_exp_off_ + 8, sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  *exponent = e;
}

}  // namespace ab2
