// batch.cpp - many independent polynomial operations sharing launches.
//
// Products are recorded into a BatchRec and flushed together: one descriptor
// upload and one launch set per transform size, whatever the mix of primes
// (direct products for short operands, native transforms, 3-prime CRT lifts
// with batched Garner reconstruction, crt_convolution.hpp:132-205).  The Newton
// loops of inv, log and exp (inverse.hpp:163-188, exponential.hpp:85-207)
// advance in lockstep over all jobs: one doubling step is two flushes for the
// inverse extensions (inv jobs, the inverse inside log, and exp's running
// inverse together) plus three for exp, however many jobs there are.
#include <algorithm>
#include <bit>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>

#include "engine.h"

namespace fpx {

namespace {
constexpr size_t kNaiveB = 40;                                        // base.hpp:89
const uint32_t kCrtPrimesB[3] = {167772161u, 469762049u, 754974721u};  // crt_convolution.hpp:14-18
// Batched transforms use rows of 2^12 points: at most 2^24 points.
constexpr int kBatchMaxLog = 24;
// Terms the fused Newton kernels (one CTA, or a cluster of three for CRT
// moduli) compute: longer inverses and exponentials start the lockstep loop there.
size_t fused_terms() { return size_t(1) << newton_inv_max_log(); }

Tw2 shoup_pair_b(uint32_t w, uint32_t p) { return Tw2{w, (uint32_t)(((uint64_t)w << 32) / p)}; }
size_t round64(size_t w) { return (w + 63) & ~size_t(63); }
}  // namespace

// c[0, k) -> c[0, wanted) for the inverse of a (extend_inverse, inverse.hpp:18-65).
struct ExtJob {
  uint32_t p;
  const uint32_t* a;
  size_t la;
  uint32_t* c;
  size_t k, wanted;
  uint32_t* cs;  // spectrum of c[0, k) at N = 2^ceil(log2 2k) (native primes), N words
  uint32_t* h;   // wanted - k words
};

class BatchRec {
 public:
  explicit BatchRec(Engine& e) : e_(e) {}

  // One cyclic product of size 2^logN on a native prime (Engine::cyc_product semantics).
  void cyc(uint32_t p, int logN, const Engine::CycOp& op) {
    XJob j;
    j.pt = &plan(p);
    j.logN = logN;
    j.x = op.x;
    j.y = op.y;
    j.ymode = op.ymode;
    j.yspec = op.yspec;
    j.yspec_out = op.yspec_out;
    j.epi = op.epi;
    const uint32_t N = 1u << logN;
    if (logN <= small_kernel_max_log()) {
      // 1/N, times 2^32 after a Montgomery pointwise product, times the caller's factor
      uint64_t s = op.ymode != 0 ? j.pt->inv_pow2_r[logN] : j.pt->inv_pow2[logN];
      if (j.epi.scale.w) s = s * j.epi.scale.w % p;
      j.epi.scale = shoup_pair_b((uint32_t)s, p);
      need_.push_back(0);
    } else {
      j.bt = &big(p, logN);
      if (j.epi.scale.w) j.epi.scale = shoup_pair_b(j.epi.scale.w % p, p);
      need_.push_back(op.ymode == 1 ? 2 * (size_t)N : N);
    }
    cref_.push_back(-1);
    plan_.xjobs.push_back(j);
  }

  // Coefficients [off, off+cnt) of a*b into out (times post_mont[i], negated),
  // any prime.  cyc_log > 0: the caller guarantees that a cyclic product of
  // 2^cyc_log points leaves the window free of wraparound (the Newton middle
  // products, crt_middle_product, crt_convolution.hpp:211-227).
  void product(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t off, size_t cnt,
               uint32_t* out, int cyc_log, const uint32_t* post_mont, bool negate) {
    if (cnt == 0) return;
    la = std::min(la, off + cnt);
    lb = std::min(lb, off + cnt);
    if (la == 0 || lb == 0 || la + lb - 1 <= off) {
      zero_.emplace_back(out, cnt);
      return;
    }
    const size_t full = la + lb - 1;
    if (off + cnt > full) {  // past the full product: zeros
      zero_.emplace_back(out + (full - off), off + cnt - full);
      cnt = full - off;
    }
    if (std::min(la, lb) <= kNaiveB) {  // convolution.hpp:33-95
      const bool swap = la > lb;
      DirectJob d{p, swap ? b : a, swap ? lb : la, swap ? a : b, swap ? la : lb, off, cnt, out};
      d.post_mont = post_mont;
      d.negate = negate ? 1 : 0;
      plan_.direct.push_back(d);
      return;
    }
    const int logN = cyc_log > 0 ? cyc_log : std::bit_width(full - 1);
    Epi epi;
    epi.lo = (uint32_t)off;
    epi.hi = (uint32_t)(off + cnt);
    if (e_.native(p, logN)) {
      Engine::CycOp op;
      op.x = InOp{a, (uint32_t)la, 0};
      if (a == b && la == lb) {
        op.ymode = 3;
      } else {
        op.ymode = 1;
        op.y = InOp{b, (uint32_t)lb, 0};
      }
      epi.out = out;
      epi.mul_mont = post_mont;
      epi.negate = negate ? 1 : 0;
      op.epi = epi;
      cyc(p, logN, op);
      return;
    }
    // 3-prime CRT: each auxiliary product lands in a scratch buffer assigned at
    // flush, then one Garner job reconstructs the window in the target field.
    const size_t primes = crt_prime_count(p, std::min(la, lb));
    GarnerJob g{p, (int)primes, nullptr, nullptr, nullptr, out, cnt};
    g.post_mont = post_mont;
    g.negate = negate ? 1 : 0;
    const int gi = (int)plan_.garner.size();
    for (size_t k = 0; k < primes; ++k) {
      Engine::CycOp op;
      op.x = InOp{a, (uint32_t)la, 1};
      if (a == b && la == lb) {
        op.ymode = 3;
      } else {
        op.ymode = 1;
        op.y = InOp{b, (uint32_t)lb, 1};
      }
      op.epi = epi;
      cyc(kCrtPrimesB[k], logN, op);
      cref_.back() = (int)cbuf_.size();
      cbuf_.push_back(CBuf{gi, (int)k, cnt});
    }
    plan_.garner.push_back(g);
  }

  bool empty() const { return plan_.xjobs.empty() && plan_.direct.empty() && plan_.garner.empty() && zero_.empty(); }

  void flush() {
    if (empty()) return;
    for (auto& [ptr, n] : zero_) e_.check(cudaMemsetAsync(ptr, 0, n * 4, e_.stream()), "memset");
    size_t words = 0;
    for (size_t w : need_) words += round64(w);
    for (const CBuf& c : cbuf_) words += round64(c.words);
    // (inside a graph capture the graph owns its blocks: one of its own)
    Buf arena;
    uint32_t* q = nullptr;
    if (words && e_.pool().capturing()) {
      arena = Buf(&e_.pool(), words);
      q = arena.get();
    } else if (words) {
      q = e_.flush_arena(words);
    }
    for (size_t i = 0; i < plan_.xjobs.size(); ++i) {
      XJob& j = plan_.xjobs[i];
      if (!need_[i]) continue;
      const size_t N = size_t(1) << j.logN;
      j.t1 = q;
      j.t2 = need_[i] > N ? q + N : nullptr;
      q += round64(need_[i]);
    }
    std::vector<uint32_t*> cptr(cbuf_.size());
    for (size_t c = 0; c < cbuf_.size(); ++c) {
      cptr[c] = q;
      q += round64(cbuf_[c].words);
      GarnerJob& g = plan_.garner[cbuf_[c].garner];
      (cbuf_[c].k == 0 ? g.c1 : cbuf_[c].k == 1 ? g.c2 : g.c3) = cptr[c];
    }
    for (size_t i = 0; i < plan_.xjobs.size(); ++i)
      if (cref_[i] >= 0) plan_.xjobs[i].epi.out = cptr[cref_[i]];
    for (GarnerJob& g : plan_.garner) {
      if (!g.c2) g.c2 = g.c1;
      if (!g.c3) g.c3 = g.c1;
    }
    const auto ts = std::chrono::steady_clock::now();
    Engine::Stage st = e_.stage(batch_descriptor_bytes(plan_));
    const auto tl = std::chrono::steady_clock::now();
    e_.prof_begin();
    e_.check(launch_batch(plan_, st.host, st.dev, e_.stream(), st.ev), "batch");
    e_.prof_end("batch");
    e_.host_phase("stage_wait", std::chrono::duration<double, std::milli>(tl - ts).count());
    e_.host_phase("launch_batch", std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tl).count());
    e_.count_batch(plan_);
    plan_ = BatchPlan();
    need_.clear();
    cref_.clear();
    cbuf_.clear();
    zero_.clear();
  }

 private:
  // plan lookups cached per recorder (a flush records thousands of products
  // over a handful of primes and sizes)
  const PrimeTables& plan(uint32_t p) {
    if (p != last_p_) {
      last_pt_ = &e_.prime_plan(p).t;
      last_p_ = p;
    }
    return *last_pt_;
  }
  const BigTables& big(uint32_t p, int logN) {
    const uint64_t key = ((uint64_t)p << 8) | (uint32_t)logN;
    if (key != last_big_) {
      last_bt_ = &e_.big_plan(p, logN).t;
      last_big_ = key;
    }
    return *last_bt_;
  }
  uint32_t last_p_ = 0;
  const PrimeTables* last_pt_ = nullptr;
  uint64_t last_big_ = 0;
  const BigTables* last_bt_ = nullptr;
  struct CBuf {
    int garner, k;
    size_t words;
  };
  Engine& e_;
  BatchPlan plan_;
  std::vector<size_t> need_;  // scratch words per xjob
  std::vector<int> cref_;     // xjob -> CRT buffer index, or -1
  std::vector<CBuf> cbuf_;
  std::vector<std::pair<uint32_t*, size_t>> zero_;
};

// ------------------------------------------------------------ staging ring

uint32_t* Engine::flush_arena(size_t words) {
  if (words > flush_arena_words_) {
    flush_arena_.reset();  // back to the pool in stream order, after the flushes that used it
    flush_arena_words_ = 0;
    flush_arena_ = Buf(&pool_, words);
    flush_arena_words_ = words;
  }
  return flush_arena_.get();
}

bool Engine::stage_fits(size_t bytes, size_t& off) const {
  const size_t cap = arena_.cap;
  if (live_.empty()) {
    off = 0;
    return bytes <= cap;
  }
  // free space: [head_, cap) and [0, tail) when head_ >= tail, else [head_, tail);
  // an allocation never ends exactly at tail, so head_ == tail means empty
  const size_t tail = live_.front().off;
  if (head_ >= tail) {
    if (cap - head_ >= bytes) {
      off = head_;
      return true;
    }
    off = 0;
    return bytes < tail;
  }
  off = head_;
  return bytes < tail - head_;
}

void Engine::stage_grow(size_t bytes) {
  const auto t0 = std::chrono::steady_clock::now();
  size_t cap = std::max(kMinArena, 2 * arena_.cap);
  while (cap < 2 * bytes) cap *= 2;
  StageArena a;
  check(cudaMallocHost(reinterpret_cast<void**>(&a.host), cap), "cudaMallocHost");
  try {
    a.dev = Buf(&pool_, cap / 4);
  } catch (...) {
    cudaFreeHost(a.host);
    throw;
  }
  a.cap = cap;
  if (arena_.host) old_arenas_.push_back(std::move(arena_));
  arena_ = std::move(a);
  for (const StageRegion& r : live_) pending_.push_back(r.ev);
  live_.clear();
  head_ = 0;
  count_host_alloc(t0);
}

Engine::Stage Engine::stage(size_t bytes) {
  bytes = (bytes + 255) & ~size_t(255);
  auto done = [&](cudaEvent_t e) {
    const cudaError_t q = cudaEventQuery(e);
    if (q == cudaErrorNotReady) return false;
    check(q, "staging query");
    return true;
  };
  while (!pending_.empty() && done(pending_.front())) {
    stage_free_ev_.push_back(pending_.front());
    pending_.pop_front();
  }
  while (!live_.empty() && done(live_.front().ev)) {
    stage_free_ev_.push_back(live_.front().ev);
    live_.pop_front();
  }
  if (live_.empty()) head_ = 0;
  size_t off = 0;
  while (!stage_fits(bytes, off)) {
    if (live_.empty() || arena_.cap < kMaxArena) {
      stage_grow(bytes);
      continue;
    }
    // the arena is at its largest: wait for the oldest region's copy
    check(cudaEventSynchronize(live_.front().ev), "staging wait");
    stage_free_ev_.push_back(live_.front().ev);
    live_.pop_front();
    if (live_.empty()) head_ = 0;
  }
  cudaEvent_t ev;
  if (!stage_free_ev_.empty()) {
    ev = stage_free_ev_.back();
    stage_free_ev_.pop_back();
  } else {
    check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
    stage_all_ev_.push_back(ev);
  }
  live_.push_back(StageRegion{off, ev});
  head_ = off + bytes;
  return Stage{arena_.host + off, static_cast<char*>(static_cast<void*>(arena_.dev.get())) + off, ev};
}

void Engine::free_stages() {
  for (Pin& q : pins_) {
    if (q.host) cudaFreeHost(q.host);
    if (q.ev) cudaEventDestroy(q.ev);
    q = Pin();
  }
  // the engine's streams are drained: every staging copy has completed
  live_.clear();
  pending_.clear();
  old_arenas_.push_back(std::move(arena_));
  arena_ = StageArena();
  for (StageArena& a : old_arenas_) {
    if (a.host) cudaFreeHost(a.host);
    a.host = nullptr;
    a.dev.reset();
  }
  old_arenas_.clear();
  for (cudaEvent_t e : stage_all_ev_) cudaEventDestroy(e);
  stage_all_ev_.clear();
  stage_free_ev_.clear();
  head_ = 0;
}

void Engine::count_batch(const BatchPlan& b) {
  std::vector<int> sizes;
  for (const XJob& j : b.xjobs) sizes.push_back(j.logN);
  std::sort(sizes.begin(), sizes.end());
  sizes.erase(std::unique(sizes.begin(), sizes.end()), sizes.end());
  uint64_t n = (b.direct.empty() ? 0 : 1) + (b.garner.empty() ? 0 : 1);
  for (int s : sizes) n += s <= small_kernel_max_log() ? 1 : 3;
  if (n) launches_ += n - 1;  // the flush's prof_end counted one
}

void Engine::gather_first(const std::vector<const uint32_t*>& ptrs, uint32_t* host_out) {
  Stage st = stage(ptrs.size() * 12 + 512);
  prof_begin();
  check(launch_gather_first(ptrs, st.host, st.dev, host_out, stream_), "gather");
  prof_end("gather");  // counts the launch
  sync();
}

void Engine::convert_repr(const std::vector<ReprSeg>& segs) {
  if (segs.empty()) return;
  Stage st = stage(repr_batch_bytes(segs.size()));
  prof_begin();
  check(launch_repr_batch(segs, st.host, st.dev, stream_, st.ev), "repr");
  prof_end("repr");
  launches_ += (segs.size() + 65534) / 65535;
}

void Engine::window_product(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t off,
                            size_t cnt, uint32_t* out, int cyc_log, const uint32_t* post_mont, bool negate) {
  BatchRec rec(*this);
  rec.product(p, a, la, b, lb, off, cnt, out, cyc_log, post_mont, negate);
  rec.flush();
}

// ------------------------------------------------- lockstep inverse extension

// Five transforms at N = 2k for a native prime (as Engine::extend_inverse):
// phase 1 = forward a, forward c (kept), inverse window [k, wanted) negated.
void Engine::ext_phase1(BatchRec& rec, const ExtJob& j) {
  const size_t hlen = j.wanted - j.k;
  const int logN = std::bit_width(2 * j.k - 1);
  const size_t aw = std::min(j.la, j.wanted);
  if (native(j.p, logN)) {
    CycOp op;
    op.x = InOp{j.a, (uint32_t)aw, 0};
    op.ymode = 1;
    op.y = InOp{j.c, (uint32_t)j.k, 0};
    op.yspec_out = j.cs;
    op.epi.out = j.h;
    op.epi.lo = (uint32_t)j.k;
    op.epi.hi = (uint32_t)(j.k + hlen);
    op.epi.negate = 1;
    rec.cyc(j.p, logN, op);
  } else {  // crt_middle_product (inverse.hpp:35-38)
    rec.product(j.p, j.a, aw, j.c, j.k, j.k, hlen, j.h, logN, nullptr, true);
  }
}

// phase 2 = forward h, times c's spectrum, inverse window [0, wanted - k) -> c + k.
void Engine::ext_phase2(BatchRec& rec, const ExtJob& j) {
  const size_t hlen = j.wanted - j.k;
  const int logN = std::bit_width(2 * j.k - 1);
  if (native(j.p, logN)) {
    CycOp op;
    op.x = InOp{j.h, (uint32_t)hlen, 0};
    op.ymode = 2;
    op.yspec = j.cs;
    op.epi.out = j.c + j.k;
    op.epi.lo = 0;
    op.epi.hi = (uint32_t)hlen;
    rec.cyc(j.p, logN, op);
  } else {  // conv_limbs (inverse.hpp:39-40)
    rec.product(j.p, j.h, hlen, j.c, j.k, 0, hlen, j.c + j.k, logN, nullptr, false);
  }
}

// ------------------------------------------------------------------ batch

namespace {
// kInvF / kExpF: inverse / exp on a transform prime up to 2^13 terms, one CTA
// per job in one launch (k_newton_b); kInv / kExp: the lockstep doubling loop.
// kDerived: sqrt / pow / divmod, as phases of batched operations where they can.
enum Route : uint8_t { kNone, kConv, kInv, kLog, kExp, kSingle, kInvF, kExpF, kDerived };
}

void Engine::batch(fpx_job* jobs, size_t count, const uint32_t* first_words, const fpx_job* host, bool host_mont) {
  std::vector<uint8_t> route(count, kNone);
  std::vector<const uint32_t*> firsts(count, nullptr);
  std::vector<size_t> conv_len(count, 0);
  std::vector<uint8_t> cont(count, 0);  // inv / exp continued from a fused 2^13-term start
  bool need_first = false;
  const size_t max_series = size_t(1) << kBatchMaxLog;
  for (size_t i = 0; i < count; ++i) {
    fpx_job& j = jobs[i];
    j.status = FPX_OK;
    j.out_len = 0;
    j.out2_len = 0;
    if (j.p < 2 || j.p >= (1u << 31) || !is_prime(j.p) || (j.la && !j.a)) {
      j.status = FPX_EINVAL;
      continue;
    }
    switch (j.op) {
      case FPX_OP_CONV: {
        if (j.lb && !j.b) { j.status = FPX_EINVAL; break; }
        if (j.la == 0 || j.lb == 0 || j.n == 0) break;  // convolution.hpp:17-31
        const size_t la = std::min(j.la, j.n), lb = std::min(j.lb, j.n);
        if (la > SIZE_MAX - (lb - 1)) { j.status = FPX_ELENGTH; break; }
        const size_t outn = std::min(la + lb - 1, j.n);
        if (!j.out) { j.status = FPX_EINVAL; break; }
        j.out_len = outn;
        conv_len[i] = outn;
        const bool fits = std::min(la, lb) <= kNaiveB || std::bit_width(la + lb - 2) <= kBatchMaxLog;
        route[i] = fits ? kConv : kSingle;
        break;
      }
      case FPX_OP_INV:
      case FPX_OP_LOG:
      case FPX_OP_EXP: {
        if (j.n == 0) break;
        if (!j.out) { j.status = FPX_EINVAL; break; }
        j.out_len = j.n;
        // log's final product has 2n - 3 terms: at most 2^24 points for n <= 2^23
        const size_t lim = j.op == FPX_OP_LOG ? max_series / 2 : max_series;
        if (j.p == 2 || j.n > lim) {
          route[i] = kSingle;
          break;
        }
        route[i] = j.op == FPX_OP_INV ? kInv : (j.op == FPX_OP_LOG ? kLog : kExp);
        if (j.la) firsts[i] = j.a;
        need_first = true;
        break;
      }
      case FPX_OP_SQRT:
      case FPX_OP_POW:
        if (j.n == 0) break;
        if (!j.out) { j.status = FPX_EINVAL; break; }
        j.out_len = j.n;
        route[i] = kDerived;
        break;
      case FPX_OP_DIVMOD:  // out / out2 may be null: quotient / remainder not wanted
        if (j.lb && !j.b) { j.status = FPX_EINVAL; break; }
        route[i] = kDerived;
        break;
      default:
        j.status = FPX_EINVAL;
    }
  }

  // ---- domain checks of inv / log / exp: one gather of every constant term
  if (need_first) {
    std::vector<uint32_t> a0(count, 0);
    if (first_words) {
      for (size_t i = 0; i < count; ++i)
        if (firsts[i]) a0[i] = first_words[i];
    } else {
      gather_first(firsts, a0.data());
    }
    for (size_t i = 0; i < count; ++i) {
      fpx_job& j = jobs[i];
      const uint32_t p = j.p;
      bool bad = false;
      if (route[i] == kInv) bad = j.la == 0 || a0[i] == 0;                         // inverse.hpp:165-166
      else if (route[i] == kLog) bad = j.la == 0 || a0[i] != 1 % p || j.n > p;     // exponential.hpp:86-90
      else if (route[i] == kExp) bad = (j.la != 0 && a0[i] != 0) || j.n - 1 >= p;  // exponential.hpp:108-111
      if (bad) {
        j.status = FPX_EDOMAIN;
        j.out_len = 0;
        route[i] = kNone;
        continue;
      }
      // one CTA (transform primes) or one cluster of three (CRT, odd p for exp)
      const bool small = j.n <= (size_t(1) << newton_inv_max_log()) &&
                         (native(p, newton_inv_max_log()) ||
                          (crt_newton_on() && (route[i] != kExp || (p & 1u))));
      if (small && route[i] == kInv) route[i] = kInvF;
      if (small && route[i] == kExp && std::min(j.la, j.n) > 1 && j.n > 1) route[i] = kExpF;
      // longer inverses and exponentials on the same moduli: their first 2^13
      // terms come from the same fused kernels, the lockstep loop continues
      const bool fusable = native(p, newton_inv_max_log()) || (crt_newton_on() && (route[i] != kExp || (p & 1u)));
      if (fusable && !small && (route[i] == kInv || (route[i] == kExp && std::min(j.la, j.n) > 1))) cont[i] = 1;
    }
  }

  // ---- convolutions: one flush per output-size class, largest first, so the
  // GPU works through the big products while the host records the small ones
  // (recording all of them before the first launch left the GPU idle for the
  // whole recording time)
  {
    std::vector<size_t> order;
    for (size_t i = 0; i < count; ++i)
      if (route[i] == kConv) order.push_back(i);
    auto cls = [&](size_t i) { return std::bit_width(conv_len[i]); };
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return cls(x) > cls(y); });
    using HClock = std::chrono::steady_clock;
    // One flush per output-size class, largest first.  Merging classes into
    // fewer, larger flushes measured slower (config-4 mix: 6.02 ms per batch
    // with one flush per class, 6.16 with at least 512 products per flush, 6.97
    // with one flush): the GPU starts later and the small-transform launches gain
    // little from being larger.
    for (size_t k = 0; k < order.size();) {
      BatchRec rec(*this);
      const int c = cls(order[k]);
      auto t0 = HClock::now();
      for (; k < order.size() && cls(order[k]) == c; ++k) {
        const fpx_job& j = jobs[order[k]];
        rec.product(j.p, j.a, std::min(j.la, j.n), j.b, std::min(j.lb, j.n), 0, conv_len[order[k]], j.out, 0,
                    nullptr, false);
      }
      auto t1 = HClock::now();
      rec.flush();
      host_phase("conv_record", std::chrono::duration<double, std::milli>(t1 - t0).count());
      host_phase("conv_flush", std::chrono::duration<double, std::milli>(HClock::now() - t1).count());
    }
  }

  // ---- series: scratch, preparation, seeds
  struct InvT {  // inverse of a[0, la) to n terms into out
    uint32_t p;
    const uint32_t* a;
    size_t la, n;
    uint32_t* out;
    uint32_t *cs, *h;
    size_t start = 32;  // terms present when the lockstep loop takes the job over
  };
  struct ExpT {
    size_t i;
    size_t lap, csize;
    uint32_t *ap, *c, *bs, *cs, *h, *t1, *t2;
    const uint32_t* tab;
    size_t start;  // terms of b present when the lockstep loop takes the job over
  };
  struct LogT {
    size_t i, ld;
    uint32_t *ap, *ia;
    const uint32_t* tab;
  };
  std::vector<InvT> invs;
  std::vector<ExpT> exps;
  std::vector<LogT> logs;
  size_t words = 0;
  std::map<uint32_t, size_t> tab_need;  // prime -> largest 1/i needed
  for (size_t i = 0; i < count; ++i) {
    const fpx_job& j = jobs[i];
    const size_t n = j.n, cnt = std::min(j.la, n);
    if (route[i] == kInv) words += round64(2 * n) + round64(n);
    if (route[i] == kExpF) {
      words += round64(n) + round64(n / 2 + 64);
      size_t& t = tab_need[j.p];
      t = std::max(t, n - 1);
    }
    if (route[i] == kLog && cnt > 1) {
      words += 3 * round64(n) + round64(2 * n);
      size_t& t = tab_need[j.p];
      t = std::max(t, n - 1);
    }
    if (route[i] == kExp) {
      words += 5 * round64(n) + 2 * round64(2 * n);
      if (cnt > 1 && n > 1) {
        size_t& t = tab_need[j.p];
        t = std::max(t, n - 1);
      }
    }
  }
  bool any_series = false;
  for (size_t i = 0; i < count; ++i)
    any_series |= route[i] == kInv || route[i] == kLog || route[i] == kExp || route[i] == kInvF || route[i] == kExpF;
  if (any_series) {
    for (auto& [p, need] : tab_need) inv_table(p, need);  // grow once per prime, before any pointer is kept
    Buf arena(&pool_, words ? words : 1);
    uint32_t* q = arena.get();
    auto take = [&](size_t w) {
      uint32_t* r = q;
      q += round64(w);
      return r;
    };
    std::vector<ExpPrep> preps;
    std::vector<SeedJob> seeds1, seeds2;
    std::vector<NewtonJob> fused;
    PrimeTables aux3[3];  // the CRT primes' plans, for the cluster jobs
    bool aux_set = false;
    auto crt_aux = [&]() -> const PrimeTables* {
      if (!aux_set) {
        const uint32_t ps[3] = {167772161u, 469762049u, 754974721u};
        for (int t = 0; t < 3; ++t) aux3[t] = prime_plan(ps[t]).t;
        aux_set = true;
      }
      return aux3;
    };
    for (size_t i = 0; i < count; ++i) {
      fpx_job& j = jobs[i];
      const size_t n = j.n, cnt = std::min(j.la, n);
      const bool nat = native(j.p, newton_inv_max_log());
      if (route[i] == kInvF) {
        if (nat) fused.push_back(NewtonJob{0, &prime_plan(j.p).t, j.a, cnt, nullptr, j.out, nullptr, n});
        else fused.push_back(NewtonJob{0, nullptr, j.a, cnt, nullptr, j.out, nullptr, n, crt_aux(), j.p});
      } else if (route[i] == kExpF) {
        uint32_t* ap = take(n);
        preps.push_back(ExpPrep{j.p, j.a, cnt, ap, j.out, n});  // a' (and out = 1, 0, ...)
        if (nat)
          fused.push_back(NewtonJob{1, &prime_plan(j.p).t, ap, cnt - 1, inv_table(j.p, n - 1), j.out,
                                    take(n / 2 + 64), n});
        else
          fused.push_back(NewtonJob{1, nullptr, ap, cnt - 1, inv_table(j.p, n - 1), j.out, take(n / 2 + 64), n,
                                    crt_aux(), j.p});
      } else if (route[i] == kInv) {
        InvT t{j.p, j.a, cnt, n, j.out, take(2 * n), take(n)};
        if (cont[i]) {  // c[0, 2^13) by the fused kernel, the lockstep loop from there
          t.start = fused_terms();
          if (nat) fused.push_back(NewtonJob{0, &prime_plan(j.p).t, j.a, cnt, nullptr, j.out, nullptr, fused_terms()});
          else fused.push_back(NewtonJob{0, nullptr, j.a, cnt, nullptr, j.out, nullptr, fused_terms(), crt_aux(), j.p});
        } else {
          seeds1.push_back(SeedJob{0, j.p, j.a, cnt, j.out, (int)std::min<size_t>(n, 32), 0});
        }
        invs.push_back(t);
      } else if (route[i] == kLog) {
        if (cnt <= 1 || n == 1) {  // log = 0
          ExpPrep e{j.p, j.a, 0, nullptr, j.out, n};
          e.out0 = 0;
          preps.push_back(e);
          continue;
        }
        LogT l{i, cnt - 1, take(n), take(n), inv_table(j.p, n - 1)};
        ExpPrep e{j.p, j.a, cnt, l.ap, j.out, n};
        e.out0 = 0;
        preps.push_back(e);
        // inverse of a to n - 1 terms (exponential.hpp:92-95)
        const size_t ila = std::min(cnt, n - 1);
        InvT t{j.p, j.a, ila, n - 1, l.ia, take(2 * n), take(n)};
        invs.push_back(t);
        seeds1.push_back(SeedJob{0, j.p, j.a, ila, l.ia, (int)std::min<size_t>(n - 1, 32), 0});
        logs.push_back(l);
      } else if (route[i] == kExp) {
        ExpT e{};
        e.i = i;
        e.lap = cnt ? cnt - 1 : 0;
        e.csize = 16;
        e.ap = take(n);
        e.c = take(n);
        e.bs = take(2 * n);
        e.cs = take(2 * n);
        e.h = take(n);
        e.t1 = take(n);
        e.t2 = take(n);
        e.start = 32;
        preps.push_back(ExpPrep{j.p, j.a, cnt, e.ap, j.out, n});
        if (e.lap && n > 1 && cont[i]) {
          // b[0, 2^13) and c = 1/b to 2^12 terms by the fused kernel
          e.tab = inv_table(j.p, n - 1);
          e.start = fused_terms();
          e.csize = fused_terms() / 2;
          if (nat) fused.push_back(NewtonJob{1, &prime_plan(j.p).t, e.ap, e.lap, e.tab, j.out, e.c, fused_terms()});
          else fused.push_back(NewtonJob{1, nullptr, e.ap, e.lap, e.tab, j.out, e.c, fused_terms(), crt_aux(), j.p});
        } else if (e.lap && n > 1) {
          e.tab = inv_table(j.p, n - 1);
          seeds1.push_back(SeedJob{1, j.p, e.ap, e.lap, j.out, (int)std::min<size_t>(n, 32), 0});
          if (n > 32) seeds2.push_back(SeedJob{0, j.p, j.out, 32, e.c, 16, 0});
        } else {
          e.lap = 0;
        }
        exps.push_back(e);
      }
    }
    if (!preps.empty()) {
      Stage st = stage(batch_aux_bytes(preps.size()));
      prof_begin();
      check(launch_exp_prep_batch(preps, st.host, st.dev, stream_, st.ev), "prep");
      prof_end("prep");
    }
    // the one-CTA Newton jobs depend on nothing the lockstep loop computes:
    // they run on the side stream, joined back before the arena is released
    // (their descriptors get a device buffer of their own: the staging ring's
    // device slots are reused in stream_ order, which the side stream does not follow)
    const bool side = !fused.empty() && !prof_on_;
    Buf fdesc;
    // joins the side stream back into stream_ before fdesc and the arena go back
    // to the pool, also when an error unwinds this block
    struct SideJoin {
      Engine& e;
      bool active = false;
      void join() {
        if (!active) return;
        active = false;
        e.check(cudaEventRecord(e.side_join_, e.side_), "cudaEventRecord");
        e.check(cudaStreamWaitEvent(e.stream_, e.side_join_, 0), "cudaStreamWaitEvent");
      }
      ~SideJoin() {
        if (active) {
          cudaEventRecord(e.side_join_, e.side_);
          cudaStreamWaitEvent(e.stream_, e.side_join_, 0);
        }
      }
    } side_join{*this};
    if (!fused.empty()) {
      // Longest first: the CTAs (one per SM, for their shared memory) start in
      // launch order, so the short jobs fill in behind the long ones instead of
      // a wave ending on a few long ones (config-4 batch 6.03 -> 5.74 ms; on
      // the main stream instead of the side stream it measured the same).
      // Outputs are per job: the order is free.
      std::stable_sort(fused.begin(), fused.end(), [](const NewtonJob& x, const NewtonJob& y) {
        return x.K * (x.kind == 1 ? 3 : 1) > y.K * (y.kind == 1 ? 3 : 1);  // exp: about three inverses' work
      });
      // one launch for the one-CTA jobs, one for the cluster jobs
      bool any_nat = false, any_crt = false;
      for (const NewtonJob& x : fused) (x.aux ? any_crt : any_nat) = true;
      const int newton_kernels = (int)any_nat + (int)any_crt;
      Stage st = stage(batch_newton_bytes(fused.size()));
      fdesc = Buf(&pool_, batch_newton_bytes(fused.size()) / 4 + 1);
      if (side) {
        check(cudaEventRecord(side_fork_, stream_), "cudaEventRecord");
        check(cudaStreamWaitEvent(side_, side_fork_, 0), "cudaStreamWaitEvent");
        side_join.active = true;
        check(launch_newton_batch(fused, st.host, fdesc.get(), side_, st.ev), "newton");
        launches_ += newton_kernels;
      } else {
        prof_begin();
        check(launch_newton_batch(fused, st.host, fdesc.get(), stream_, st.ev), "newton");
        prof_end("newton");
        launches_ += newton_kernels - 1;  // prof_end counted one
      }
    }
    if (!seeds1.empty()) {
      Stage st = stage(batch_aux_bytes(seeds1.size()));
      prof_begin();
      check(launch_seeds_batch(seeds1, st.host, st.dev, stream_, st.ev), "seed");
      prof_end("seed");
    }
    if (!seeds2.empty()) {
      Stage st = stage(batch_aux_bytes(seeds2.size()));
      prof_begin();
      check(launch_seeds_batch(seeds2, st.host, st.dev, stream_, st.ev), "seed");
      prof_end("seed");
    }

    // ---- lockstep doubling
    // jobs continued from the fused kernels need their first 2^13 terms
    bool any_cont = false;
    for (const InvT& t : invs) any_cont |= t.start > 32;
    for (const ExpT& e : exps) any_cont |= e.start > 32;
    if (any_cont) side_join.join();
    size_t m_end = 0;  // the loop runs until the longest job is complete
    for (const InvT& t : invs) m_end = std::max(m_end, t.n);
    for (const ExpT& e : exps)
      if (e.lap) m_end = std::max(m_end, jobs[e.i].n);
    for (size_t m = 32; m < m_end; m <<= 1) {
      std::vector<ExtJob> ext;
      for (const InvT& t : invs)
        if (m < t.n && m >= t.start) ext.push_back(ExtJob{t.p, t.a, t.la, t.out, m, std::min(2 * m, t.n), t.cs, t.h});
      std::vector<ExpT*> act;
      for (ExpT& e : exps) {
        const fpx_job& j = jobs[e.i];
        if (!e.lap || m >= j.n || m < e.start) continue;
        act.push_back(&e);
        const size_t hlen = std::min(2 * m, j.n) - m;
        if (e.csize < hlen) {  // exponential.hpp:158-163: extend the inverse of b
          ext.push_back(ExtJob{j.p, j.out, m, e.c, e.csize, hlen, e.cs, e.h});
          e.csize = hlen;
        }
      }
      if (ext.empty() && act.empty()) continue;
      if (!ext.empty()) {
        BatchRec r1(*this);
        for (const ExtJob& x : ext) ext_phase1(r1, x);
        r1.flush();
        BatchRec r2(*this);
        for (const ExtJob& x : ext) ext_phase2(r2, x);
        r2.flush();
      }
      if (act.empty()) continue;
      // exp step (exponential.hpp:165-205), eight transforms at N = 2m per job
      const int logN = std::bit_width(2 * m - 1);
      BatchRec r3(*this);
      for (ExpT* e : act) {  // (a' b)[m-1, m-1+hlen); b's spectrum kept
        const fpx_job& j = jobs[e->i];
        const size_t m2 = std::min(2 * m, j.n), hlen = m2 - m, lx = std::min(e->lap, m2 - 1);
        if (native(j.p, logN)) {
          CycOp op;
          op.x = InOp{e->ap, (uint32_t)lx, 0};
          op.ymode = 1;
          op.y = InOp{j.out, (uint32_t)m, 0};
          op.yspec_out = e->bs;
          op.epi.out = e->t1;
          op.epi.lo = (uint32_t)(m - 1);
          op.epi.hi = (uint32_t)(m - 1 + hlen);
          r3.cyc(j.p, logN, op);
        } else {
          r3.product(j.p, e->ap, lx, j.out, m, m - 1, hlen, e->t1, logN, nullptr, false);
        }
      }
      r3.flush();
      BatchRec r4(*this);
      for (ExpT* e : act) {  // (residual * c) mod x^hlen, integrated: times 1/(m+i)
        const fpx_job& j = jobs[e->i];
        const size_t hlen = std::min(2 * m, j.n) - m;
        if (native(j.p, logN)) {
          CycOp op;
          op.x = InOp{e->t1, (uint32_t)hlen, 0};
          op.ymode = 1;
          op.y = InOp{e->c, (uint32_t)e->csize, 0};
          op.epi.out = e->t2;
          op.epi.lo = 0;
          op.epi.hi = (uint32_t)hlen;
          op.epi.mul_mont = e->tab + m;
          r4.cyc(j.p, logN, op);
        } else {
          r4.product(j.p, e->t1, hlen, e->c, e->csize, 0, hlen, e->t2, logN, e->tab + m, false);
        }
      }
      r4.flush();
      BatchRec r5(*this);
      for (ExpT* e : act) {  // b[m, m+hlen) = (correction * b) mod x^hlen
        const fpx_job& j = jobs[e->i];
        const size_t hlen = std::min(2 * m, j.n) - m;
        if (native(j.p, logN)) {
          CycOp op;
          op.x = InOp{e->t2, (uint32_t)hlen, 0};
          op.ymode = 2;
          op.yspec = e->bs;
          op.epi.out = j.out + m;
          op.epi.lo = 0;
          op.epi.hi = (uint32_t)hlen;
          r5.cyc(j.p, logN, op);
        } else {
          r5.product(j.p, e->t2, hlen, j.out, m, 0, hlen, j.out + m, logN, nullptr, false);
        }
      }
      r5.flush();
    }

    side_join.join();

    // ---- log: integral(a' * inv(a)) (exponential.hpp:92-97)
    if (!logs.empty()) {
      BatchRec rl(*this);
      for (const LogT& l : logs) {
        const fpx_job& j = jobs[l.i];
        const size_t lp = std::min(l.ld + j.n - 2, j.n - 1);
        rl.product(j.p, l.ap, l.ld, l.ia, j.n - 1, 0, lp, j.out + 1, 0, l.tab + 1, false);
      }
      rl.flush();
    }
  }

  // ---- sqrt / pow / divmod through batched phases
  std::vector<size_t> derived;
  for (size_t i = 0; i < count; ++i)
    if (route[i] == kDerived) derived.push_back(i);
  if (!derived.empty()) batch_derived(jobs, derived, host, host_mont);

  // ---- jobs that share no launches run one after another
  for (size_t i = 0; i < count; ++i)
    if (route[i] == kSingle) batch_single(jobs[i]);
}

void Engine::batch_single(fpx_job& j) {
  try {
    switch (j.op) {
      case FPX_OP_CONV: j.out_len = conv(j.p, j.a, j.la, j.b, j.lb, j.n, j.out); break;
      case FPX_OP_INV: inv(j.p, j.a, std::min(j.la, j.n), j.n, j.out); break;
      case FPX_OP_LOG: log(j.p, j.a, std::min(j.la, j.n), j.n, j.out); break;
      case FPX_OP_EXP: exp(j.p, j.a, std::min(j.la, j.n), j.n, j.out); break;
      case FPX_OP_SQRT: sqrt(j.p, j.a, std::min(j.la, j.n), j.n, j.out); break;
      case FPX_OP_POW: pow(j.p, j.a, j.la, j.k, j.n, j.out); break;
      case FPX_OP_DIVMOD: {
        size_t lq = 0, lr = 0;
        divmod(j.p, j.a, j.la, j.b, j.lb, j.out, &lq, j.out2, &lr, j.out != nullptr, j.out2 != nullptr);
        j.out_len = lq;
        j.out2_len = lr;
        break;
      }
      default: j.status = FPX_EINVAL;
    }
  } catch (const Error& e) {
    if (e.code == FPX_ECUDA) throw;  // the stream is unusable: fail the whole batch
    j.status = e.code;
    j.out_len = 0;
    j.out2_len = 0;
  }
}


// ------------------------------------------------------- sqrt / pow / divmod

namespace {
// sqrt jobs above this many result terms keep the single path (one Newton
// loop, about half the work of the log and exp below).
constexpr size_t kDerivedSqrtMax = size_t(1) << 16;
// Longer pow / divmod jobs keep the single path too: a batch holds few of them
// (phases gain little), and their phase buffers, sized by the sum over the
// batch, asked the pool for new multi-GB classes (a served mix spent twice as
// long in cudaMalloc, single calls up to 110 ms, stalling every worker).
constexpr size_t kDerivedMax = size_t(1) << 17;

// FPX_BATCH_PHASED=0: every sqrt / pow / divmod job of a batch through the
// single path, one after another.
bool phased_on() {
  static const bool on = [] {
    const char* e = std::getenv("FPX_BATCH_PHASED");
    return !(e && e[0] == '0');
  }();
  return on;
}

// Operand reads for the host decisions (valuation, constant terms, degrees):
// the caller's host copy when batch_host has one, else the device.
struct OperandReader {
  Engine& e;
  bool mont;
  uint32_t p = 0, rinv = 1;  // 2^-32 mod p, for Montgomery host words
  size_t first(const uint32_t* dev, const uint32_t* host, size_t n) {
    if (!host) return e.find_nonzero(dev, n, false);
    for (size_t i = 0; i < n; ++i)
      if (host[i]) return i;
    return n;
  }
  size_t last(const uint32_t* dev, const uint32_t* host, size_t n) {
    if (!host) return e.find_nonzero(dev, n, true);
    for (size_t i = n; i-- > 0;)
      if (host[i]) return i;
    return n;
  }
  uint32_t word(const uint32_t* dev, const uint32_t* host, size_t at, uint32_t mod) {
    if (!host) return e.read_word(dev + at);
    if (!mont) return host[at];
    if (mod != p) {
      p = mod;
      rinv = invm((uint32_t)((uint64_t(1) << 32) % mod), mod);
    }
    return (uint32_t)((uint64_t)host[at] * rinv % mod);
  }
};

// One sqrt / pow / divmod job run as phases.
struct DerivedJob {
  size_t i;
  int op;
  // sqrt / pow: dst[0, inner) = post * exp(mid * log(u * pre)), u = ulen words
  const uint32_t* u = nullptr;
  size_t ulen = 0, inner = 0;
  uint32_t pre = 0, mid = 0, post = 0;
  uint32_t* dst = nullptr;
  uint32_t *nrm = nullptr, *l = nullptr;
  // divmod (division.hpp:12-80): q = reverse(reverse(a) / reverse(b)), r = a - b q
  size_t an = 0, bn = 0, dn = 0, nrb = 0, rn = 0, lp = 0;
  uint32_t *ra = nullptr, *rb = nullptr, *ib = nullptr, *rq = nullptr, *qd = nullptr, *prod = nullptr;
  bool failed = false;
};
}  // namespace

void Engine::batch_derived(fpx_job* jobs, const std::vector<size_t>& idx, const fpx_job* host, bool host_mont) {
  OperandReader rd{*this, host_mont};
  std::vector<DerivedJob> dj;
  std::vector<size_t> single;
  // ---- host decisions: the cases the single path settles without products,
  // or with binary powering, stay there; the rest become phases
  for (size_t i : idx) {
    fpx_job& j = jobs[i];
    const uint32_t p = j.p;
    const fpx_job* h = host ? host + i : nullptr;
    DerivedJob d;
    d.i = i;
    d.op = j.op;
    bool ok = false;
    const bool phased = phased_on() && p != 2;
    if (phased && j.op == FPX_OP_POW) {  // power.hpp:17-87, as Engine::pow
      const size_t n = j.n, la = j.la;
      const uint64_t k = j.k;
      const size_t v = k > 1 ? rd.first(j.a, h ? h->a : nullptr, la) : la;
      if (v < la && !(v != 0 && k > (n - 1) / v)) {
        const size_t sh = (size_t)(v * k), inner = n - sh;
        size_t ulen = std::min(la - v, inner);
        ulen = rd.last(j.a + v, h ? h->a + v : nullptr, ulen) + 1;
        if (ulen > 1 && k > 64 && inner <= p && inner <= kDerivedMax) {
          const uint32_t c0 = rd.word(j.a, h ? h->a : nullptr, v, p);
          d.u = j.a + v;
          d.ulen = ulen;
          d.inner = inner;
          d.pre = invm(c0, p);
          d.mid = (uint32_t)(k % p);
          d.post = powm(c0, k, p);
          d.dst = j.out + sh;
          ok = true;
        }
      }
    } else if (phased && j.op == FPX_OP_SQRT) {  // square_root.hpp, as exp(log(u / u0) / 2) * sqrt(u0)
      const size_t n = j.n, la = std::min(j.la, j.n);
      const size_t v = rd.first(j.a, h ? h->a : nullptr, la);
      uint32_t root0 = 0;
      if (v < la && !(v & 1)) {
        const uint32_t u0 = rd.word(j.a, h ? h->a : nullptr, v, p);
        const size_t half = v / 2;
        if (half < n && n - half <= std::min<size_t>(p, kDerivedSqrtMax) && sqrt_mod(u0, p, &root0)) {
          d.u = j.a + v;
          d.ulen = la - v;
          d.inner = n - half;
          d.pre = invm(u0, p);
          d.mid = (p + 1) / 2;
          d.post = root0;
          d.dst = j.out + half;
          ok = true;
        }
      }
    } else if (phased && j.op == FPX_OP_DIVMOD) {
      const size_t al = rd.last(j.a, h ? h->a : nullptr, j.la), bl = rd.last(j.b, h ? h->b : nullptr, j.lb);
      d.an = al < j.la ? al + 1 : 0;
      d.bn = bl < j.lb ? bl + 1 : 0;
      if (d.bn > 1 && d.an >= d.bn && d.an <= kDerivedMax) {
        d.dn = d.an - d.bn + 1;
        d.nrb = std::min(d.bn, d.dn);
        d.rn = d.bn - 1;
        d.lp = std::min(d.bn + d.dn - 1, d.rn);
        ok = true;
      }
    }
    if (ok) dj.push_back(d);
    else single.push_back(i);
  }
  // a failure other than a CUDA error (the pool limit, say) fails the phased
  // jobs only, as it fails one job on the single path
  try {
    // ---- scratch of every phased job: one pool block
    auto r64 = [](size_t w) { return (w + 63) & ~size_t(63); };
    size_t words = 0;
    for (const DerivedJob& d : dj) {
      const fpx_job& j = jobs[d.i];
      if (d.op == FPX_OP_DIVMOD)
        words += 3 * r64(d.dn) + r64(d.nrb) + (j.out ? 0 : r64(d.dn)) + (j.out2 ? r64(d.lp) : 0);
      else
        words += r64(d.ulen) + r64(d.inner);
    }
    Buf arena;
    if (words) arena = Buf(&pool_, words);
    uint32_t* q = arena.get();
    auto take = [&](size_t w) {
      uint32_t* r = q;
      q += r64(w);
      return r;
    };
    for (DerivedJob& d : dj) {
      fpx_job& j = jobs[d.i];
      if (d.op == FPX_OP_DIVMOD) {
        d.ra = take(d.dn);
        d.rb = take(d.nrb);
        d.ib = take(d.dn);
        d.rq = take(d.dn);
        d.qd = j.out ? j.out : take(d.dn);
        if (j.out2) d.prod = take(d.lp);
      } else {
        d.nrm = take(d.ulen);
        d.l = take(d.inner);
      }
    }
    auto launch = [&](const char* what, auto&& fn) {
      prof_begin();
      check(fn(), what);
      prof_end(what);
    };
    // One phase: the internal jobs as one batch (their constant terms are known:
    // 1 for log and inverse inputs, 0 for exp's), failures passed to their owners.
    std::vector<fpx_job> in;
    std::vector<size_t> owner;
    std::vector<uint32_t> firsts;
    auto add = [&](size_t d, int op, uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t n,
                   uint32_t* out, uint32_t first) {
      fpx_job x{};
      x.op = op;
      x.p = p;
      x.a = a;
      x.la = la;
      x.b = b;
      x.lb = lb;
      x.n = n;
      x.out = out;
      in.push_back(x);
      owner.push_back(d);
      firsts.push_back(first);
    };
    auto run = [&]() {
      if (!in.empty()) {
        batch(in.data(), in.size(), firsts.data());
        for (size_t t = 0; t < in.size(); ++t) {
          DerivedJob& d = dj[owner[t]];
          if (in[t].status != FPX_OK && !d.failed) {
            d.failed = true;
            jobs[d.i].status = in[t].status;
          }
        }
      }
      in.clear();
      owner.clear();
      firsts.clear();
    };

    // A: normalised operands (u / u0, u / c0) and reversed divmod operands
    for (DerivedJob& d : dj) {
      fpx_job& j = jobs[d.i];
      if (d.op == FPX_OP_DIVMOD) {
        launch("reverse", [&] { return launch_reverse(j.a + (d.an - d.dn), d.ra, d.dn, stream_); });
        launch("reverse", [&] { return launch_reverse(j.b + (d.bn - d.nrb), d.rb, d.nrb, stream_); });
      } else {
        check(cudaMemsetAsync(j.out, 0, j.n * 4, stream_), "memset");
        launch("normalise", [&] { return launch_scale(j.p, d.u, d.nrm, d.ulen, d.pre, stream_); });
      }
    }
    // B: log of the normalised operands; inverse of the reversed divisors
    for (size_t t = 0; t < dj.size(); ++t) {
      DerivedJob& d = dj[t];
      const uint32_t p = jobs[d.i].p;
      if (d.op == FPX_OP_DIVMOD) add(t, FPX_OP_INV, p, d.rb, d.nrb, nullptr, 0, d.dn, d.ib, 1);
      else add(t, FPX_OP_LOG, p, d.nrm, d.ulen, nullptr, 0, d.inner, d.l, 1);
    }
    run();
    // C: the log times k (pow) or 1/2 (sqrt)
    for (DerivedJob& d : dj)
      if (d.op != FPX_OP_DIVMOD && !d.failed)
        launch("scale", [&] { return launch_scale(jobs[d.i].p, d.l, d.l, d.inner, d.mid, stream_); });
    // D: exp of it into the result window; the reversed quotient
    for (size_t t = 0; t < dj.size(); ++t) {
      DerivedJob& d = dj[t];
      if (d.failed) continue;
      const uint32_t p = jobs[d.i].p;
      if (d.op == FPX_OP_DIVMOD) add(t, FPX_OP_CONV, p, d.ra, d.dn, d.ib, d.dn, d.dn, d.rq, 0);
      else add(t, FPX_OP_EXP, p, d.l, d.inner, nullptr, 0, d.inner, d.dst, 0);
    }
    run();
    // E: times c0^k (pow) or the constant term's root (sqrt); the quotient
    for (DerivedJob& d : dj) {
      if (d.failed) continue;
      const fpx_job& j = jobs[d.i];
      if (d.op == FPX_OP_DIVMOD)
        launch("reverse", [&] { return launch_reverse(d.rq, d.qd, d.dn, stream_); });
      else
        launch("scale", [&] { return launch_scale(j.p, d.dst, d.dst, d.inner, d.post, stream_); });
    }
    // F: b q over the remainder's window, G: r = a - b q and its length
    for (size_t t = 0; t < dj.size(); ++t) {
      DerivedJob& d = dj[t];
      const fpx_job& j = jobs[d.i];
      if (d.op == FPX_OP_DIVMOD && !d.failed && j.out2) add(t, FPX_OP_CONV, j.p, j.b, d.bn, d.qd, d.dn, d.lp, d.prod, 0);
    }
    run();
    std::vector<Segment> segs;
    std::vector<size_t> seg_of;
    for (size_t t = 0; t < dj.size(); ++t) {
      DerivedJob& d = dj[t];
      const fpx_job& j = jobs[d.i];
      if (d.op != FPX_OP_DIVMOD || d.failed || !j.out2) continue;
      launch("remainder", [&] { return launch_sub(j.p, j.a, d.prod, d.lp, j.out2, d.rn, stream_); });
      segs.push_back(Segment{j.out2, d.rn});
      seg_of.push_back(t);
    }
    std::vector<size_t> rlen(dj.size(), 0);
    if (!segs.empty()) {
      Stage st = stage(last_nonzero_batch_bytes(segs.size()));
      launch("remainder length", [&] { return launch_last_nonzero_batch(segs, st.host, st.dev, stream_); });
      sync();
      const auto* res = reinterpret_cast<const unsigned long long*>(static_cast<const char*>(st.host) +
                                                                    last_nonzero_results_offset(segs.size()));
      for (size_t s2 = 0; s2 < segs.size(); ++s2) rlen[seg_of[s2]] = res[s2] < segs[s2].n ? (size_t)res[s2] + 1 : 0;
    }
    for (size_t t = 0; t < dj.size(); ++t) {
      const DerivedJob& d = dj[t];
      fpx_job& j = jobs[d.i];
      if (d.failed) {
        j.out_len = 0;
        j.out2_len = 0;
      } else if (d.op == FPX_OP_DIVMOD) {
        j.out_len = j.out ? d.dn : 0;
        j.out2_len = j.out2 ? rlen[t] : 0;
      }
    }
  } catch (const Error& e) {
    if (e.code == FPX_ECUDA) throw;
    for (const DerivedJob& d : dj) {
      fpx_job& j = jobs[d.i];
      j.status = e.code;
      j.out_len = 0;
      j.out2_len = 0;
    }
  }
  // the rest: one after another
  for (size_t i : single) batch_single(jobs[i]);
}

// ------------------------------------------------------- host-buffer batches

// Packs the inputs into device copies through the pinned slots, runs the
// batch on them (host decisions read from the caller's buffers), and brings
// the outputs back the same way.
void Engine::batch_host(fpx_job* jobs, size_t count, int repr) {
  // Words each job reads and writes (host side); the device copy of a job
  // points into one input and one output region.
  std::vector<size_t> wa(count), wb(count), wo(count), wo2(count);
  size_t in_words = 0, out_words = 0;
  for (size_t i = 0; i < count; ++i) {
    const fpx_job& j = jobs[i];
    size_t a = 0, b = 0, o = 0, o2 = 0;
    switch (j.op) {
      case FPX_OP_CONV:
        a = j.la < j.n ? j.la : j.n;
        b = j.lb < j.n ? j.lb : j.n;
        if (a && b) o = a > SIZE_MAX - b ? j.n : (a + b - 1 < j.n ? a + b - 1 : j.n);
        break;
      case FPX_OP_INV:
      case FPX_OP_LOG:
      case FPX_OP_EXP:
      case FPX_OP_SQRT:
        a = j.la < j.n ? j.la : j.n;
        o = j.n;
        break;
      case FPX_OP_POW:
        a = j.la;
        o = j.n;
        break;
      case FPX_OP_DIVMOD:
        a = j.la;
        b = j.lb;
        o = j.out ? j.la : 0;
        o2 = j.out2 ? j.lb : 0;
        break;
      default:
        break;
    }
    if (a && !j.a) a = 0;  // the batch reports the null pointer
    if (b && !j.b) b = 0;
    if (o && !j.out) o = 0;
    wa[i] = a;
    wb[i] = b;
    wo[i] = o;
    wo2[i] = o2;
    in_words += a + b;
    out_words += o + o2;
  }
  const size_t total = in_words + out_words;
  Buf dbuf(&pool_, total ? total : 1);
  uint32_t* din = dbuf.get();
  uint32_t* dout = din + in_words;
  std::vector<fpx_job> dj(jobs, jobs + count);
  // Two chunks of about equal input words when the batch moves at least
  // 64 MiB: the host packs chunk c + 1 while the GPU runs chunk c, and unpacks
  // chunk c - 1 (copied back on the copy stream) meanwhile.  Four chunks
  // measured slower on the config-4 mix (147-158 k against 186-202 k polys/s):
  // every chunk runs its own launch set per size and Newton doubling step, so
  // the GPU's share grows with the chunk count and the host waits on it.
  constexpr size_t kChunkBytes = size_t(32) << 20;
  constexpr size_t kMaxChunks = 2;
  std::vector<size_t> bounds{0};
  const size_t want = in_words * 4 >= 2 * kChunkBytes ? std::min(kMaxChunks, in_words * 4 / kChunkBytes) : 1;
  if (count >= 2 && want > 1) {
    size_t acc = 0;
    for (size_t i = 0; i + 1 < count && bounds.size() < want; ++i) {
      acc += wa[i] + wb[i];
      if (acc * want >= in_words * bounds.size()) bounds.push_back(i + 1);  // one boundary per job at most
    }
  }
  bounds.push_back(count);
  const int nchunks = (int)bounds.size() - 1;
  std::vector<std::vector<ReprSeg>> segs(nchunks);
  std::vector<std::vector<HostSpan>> ins(nchunks);
  std::vector<size_t> in_off(nchunks + 1, in_words), out_off(nchunks + 1, out_words);
  size_t qi = 0, qo = 0;
  int ck = -1;
  for (size_t i = 0; i < count; ++i) {
    while (ck + 1 < nchunks && i == bounds[ck + 1]) {
      ++ck;
      in_off[ck] = qi;
      out_off[ck] = qo;
    }
    const fpx_job& j = jobs[i];
    fpx_job& d = dj[i];
    if (wa[i]) ins[ck].push_back(HostSpan{j.a, nullptr, wa[i]});
    d.a = j.a ? din + qi : nullptr;
    if (wa[i]) segs[ck].push_back(ReprSeg{j.p, din + qi, wa[i], 0});
    qi += wa[i];
    if (wb[i]) ins[ck].push_back(HostSpan{j.b, nullptr, wb[i]});
    d.b = j.b ? din + qi : nullptr;
    if (wb[i]) segs[ck].push_back(ReprSeg{j.p, din + qi, wb[i], 0});
    qi += wb[i];
    d.la = j.a ? wa[i] : j.la;  // a null pointer keeps its length: the batch reports it
    d.lb = j.b ? wb[i] : j.lb;
    d.out = j.out ? dout + qo : nullptr;
    qo += wo[i];
    d.out2 = j.out2 ? dout + qo : nullptr;
    qo += wo2[i];
  }
  // Constant terms for the domain checks of inv / log / exp, read from the
  // caller's buffers (canonical limbs only; Montgomery limbs are converted on
  // the device first, so those batches read them there).
  std::vector<uint32_t> first;
  if (repr != FPX_REPR_MONTGOMERY) {
    first.assign(count, 0);
    for (size_t i = 0; i < count; ++i)
      if (wa[i] && (jobs[i].op == FPX_OP_INV || jobs[i].op == FPX_OP_LOG || jobs[i].op == FPX_OP_EXP))
        first[i] = jobs[i].a[0];
  }
  if (!copy_stream_) check(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  while (chunk_ev_.size() < (size_t)nchunks) {
    cudaEvent_t e;
    check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
    chunk_ev_.push_back(e);
  }
  using HClock = std::chrono::steady_clock;
  auto ms_since = [](HClock::time_point t) { return std::chrono::duration<double, std::milli>(HClock::now() - t).count(); };

  // Copies into page-locked result buffers queued but not waited for: waited
  // for before the call returns, also when an error unwinds it (they read the
  // device buffer, which goes back to the pool after this guard).
  struct QueuedCopies {
    cudaStream_t s;
    bool queued = false;
    ~QueuedCopies() {
      if (queued) cudaStreamSynchronize(s);
    }
  } copies{copy_stream_};
  // Results of chunk c: statuses and lengths to the caller's records, then
  // every output region in device order (result words to the caller's buffer,
  // the rest skipped), copied on the copy stream once the chunk's work is done.
  auto drain = [&](int c) {
    std::vector<HostSpan> outs;
    for (size_t i = bounds[c]; i < bounds[c + 1]; ++i) {
      fpx_job& j = jobs[i];
      const fpx_job& d = dj[i];
      j.status = d.status;
      j.out_len = d.out_len;
      j.out2_len = d.out2_len;
      const bool ok = d.status == FPX_OK;
      const size_t n1 = ok && j.out ? std::min(d.out_len, wo[i]) : 0;
      const size_t n2 = ok && j.out2 ? std::min(d.out2_len, wo2[i]) : 0;
      if (n1) outs.push_back(HostSpan{nullptr, j.out, n1});
      if (wo[i] > n1) outs.push_back(HostSpan{nullptr, nullptr, wo[i] - n1});
      if (n2) outs.push_back(HostSpan{nullptr, j.out2, n2});
      if (wo2[i] > n2) outs.push_back(HostSpan{nullptr, nullptr, wo2[i] - n2});
    }
    check(cudaStreamWaitEvent(copy_stream_, chunk_ev_[c], 0), "cudaStreamWaitEvent");
    const auto t0 = HClock::now();
    if (!copy_out(dout + out_off[c], outs, copy_stream_, false)) copies.queued = true;
    host_phase("copy_out", ms_since(t0));
  };

  for (int c = 0; c < nchunks; ++c) {
    auto t0 = HClock::now();
    copy_in(ins[c], din + in_off[c]);
    host_phase("copy_in", ms_since(t0));
    t0 = HClock::now();
    if (repr == FPX_REPR_MONTGOMERY) convert_repr(segs[c]);
    batch(dj.data() + bounds[c], bounds[c + 1] - bounds[c], first.empty() ? nullptr : first.data() + bounds[c],
          jobs + bounds[c], repr == FPX_REPR_MONTGOMERY);
    if (repr == FPX_REPR_MONTGOMERY) {
      std::vector<ReprSeg> outs;
      for (size_t i = bounds[c]; i < bounds[c + 1]; ++i) {
        const fpx_job& d = dj[i];
        if (d.status != FPX_OK) continue;
        if (d.out && d.out_len) outs.push_back(ReprSeg{d.p, d.out, d.out_len, 1});
        if (d.out2 && d.out2_len) outs.push_back(ReprSeg{d.p, d.out2, d.out2_len, 1});
      }
      convert_repr(outs);
    }
    check(cudaEventRecord(chunk_ev_[c], stream_), "cudaEventRecord");
    host_phase("batch", ms_since(t0));
    if (c > 0) drain(c - 1);
  }
  drain(nchunks - 1);
  if (copies.queued) {
    copies.queued = false;
    check(cudaStreamSynchronize(copy_stream_), "D2H wait");
  }
}

// --------------------------------------------------------- pinned staging

namespace {
constexpr size_t kPinWords = size_t(8) << 20;  // 32 MiB per slot

// Host copies between the caller's buffers and the pinned staging slots, split
// across a small process-wide pool of threads: one thread moves about 10 GB/s
// of host memory, the PCIe link 50 GB/s each way, so a single-threaded packing
// loop would set the pace of every host-buffer batch.
struct CopyPiece {
  void* dst;
  const void* src;
  size_t bytes;
};

class CopyPool {
 public:
  static CopyPool& instance() {
    static CopyPool pool;
    return pool;
  }
  // Copies every piece; returns when all bytes are in place.  Small totals stay
  // on the calling thread.
  void run(const std::vector<CopyPiece>& pieces) {
    size_t total = 0;
    for (const CopyPiece& c : pieces) total += c.bytes;
    if (total < kParallelBytes || threads_.empty()) {
      part(pieces, 0, total);
      return;
    }
    std::lock_guard<std::mutex> call(call_mu_);  // one parallel copy at a time
    const int n = (int)threads_.size() + 1;
    {
      std::lock_guard<std::mutex> g(mu_);
      pieces_ = &pieces;
      total_ = total;
      parts_ = n;
      remaining_ = n - 1;
      ++gen_;
    }
    cv_.notify_all();
    part(pieces, 0, total / n);  // the caller's share: part 0
    std::unique_lock<std::mutex> g(mu_);
    done_.wait(g, [&] { return remaining_ == 0; });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> g(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : threads_) t.join();
  }

 private:
  static constexpr size_t kParallelBytes = size_t(2) << 20;
  // Threads per copy (the caller and the pool's): FPX_COPY_THREADS, else half
  // the hardware threads, at most 8.
  CopyPool() {
    const unsigned hw = std::thread::hardware_concurrency();
    int extra = (int)std::min(7u, hw > 2 ? hw / 2 - 1 : 0u);
    if (const char* e = std::getenv("FPX_COPY_THREADS")) {
      const int n = std::atoi(e);
      if (n >= 1) extra = std::min(n, 64) - 1;
    }
    for (int i = 1; i <= extra; ++i) threads_.emplace_back([this, i] { loop(i); });
  }
  // Bytes [lo, hi) of the concatenated pieces.
  static void part(const std::vector<CopyPiece>& pieces, size_t lo, size_t hi) {
    size_t at = 0;
    for (const CopyPiece& c : pieces) {
      const size_t a = std::max(lo, at), b = std::min(hi, at + c.bytes);
      if (a < b) std::memcpy(static_cast<char*>(c.dst) + (a - at), static_cast<const char*>(c.src) + (a - at), b - a);
      at += c.bytes;
      if (at >= hi) break;
    }
  }
  void loop(int id) {
    uint64_t seen = 0;
    for (;;) {
      const std::vector<CopyPiece>* pieces;
      size_t lo, hi;
      {
        std::unique_lock<std::mutex> g(mu_);
        cv_.wait(g, [&] { return stop_ || gen_ != seen; });
        if (stop_) return;
        seen = gen_;
        pieces = pieces_;
        lo = total_ * id / parts_;
        hi = total_ * (id + 1) / parts_;
      }
      part(*pieces, lo, hi);
      {
        std::lock_guard<std::mutex> g(mu_);
        --remaining_;
      }
      done_.notify_one();
    }
  }
  std::vector<std::thread> threads_;
  std::mutex call_mu_, mu_;
  std::condition_variable cv_, done_;
  const std::vector<CopyPiece>* pieces_ = nullptr;
  size_t total_ = 0;
  int parts_ = 1, remaining_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};
}

uint32_t* Engine::pin_slot(int k) {
  Pin& q = pins_[k];
  if (!q.host) {
    const auto t0 = std::chrono::steady_clock::now();
    check(cudaMallocHost(&q.host, kPinWords * 4), "cudaMallocHost");
    count_host_alloc(t0);
    check(cudaEventCreateWithFlags(&q.ev, cudaEventDisableTiming), "cudaEventCreate");
  } else {
    check(cudaEventSynchronize(q.ev), "staging wait");
  }
  return q.host;
}

namespace {
// Pageable host memory of at least this size goes through the pinned slots.
constexpr size_t kStagedBytes = size_t(1) << 20;
bool pinned(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost || a.type == cudaMemoryTypeManaged;
}
}  // namespace

void Engine::to_device(uint32_t* d_dst, const uint32_t* h_src, size_t words) {
  if (!words) return;
  if (words * 4 < kStagedBytes || pinned(h_src)) {
    check(cudaMemcpyAsync(d_dst, h_src, words * 4, cudaMemcpyHostToDevice, stream_), "H2D");
    return;
  }
  copy_in({HostSpan{h_src, nullptr, words}}, d_dst);
}

void Engine::to_host(uint32_t* h_dst, const uint32_t* d_src, size_t words) {
  if (words && (words * 4 < kStagedBytes || pinned(h_dst))) {
    check(cudaMemcpyAsync(h_dst, d_src, words * 4, cudaMemcpyDeviceToHost, stream_), "D2H");
  } else if (words) {
    copy_out(d_src, {HostSpan{nullptr, h_dst, words}});
  }
  sync();
}

void Engine::copy_in(const std::vector<HostSpan>& spans, uint32_t* dst) {
  size_t si = 0, so = 0;
  int k = 0;
  std::vector<CopyPiece> pieces;
  while (si < spans.size()) {
    uint32_t* h = pin_slot(k);
    size_t filled = 0;
    pieces.clear();
    while (si < spans.size() && filled < kPinWords) {
      const size_t take = std::min(spans[si].words - so, kPinWords - filled);
      pieces.push_back(CopyPiece{h + filled, spans[si].src + so, take * 4});
      filled += take;
      so += take;
      if (so == spans[si].words) {
        ++si;
        so = 0;
      }
    }
    const auto tp = std::chrono::steady_clock::now();
    CopyPool::instance().run(pieces);
    host_phase("pack", std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tp).count());
    check(cudaMemcpyAsync(dst, h, filled * 4, cudaMemcpyHostToDevice, stream_), "H2D");
    check(cudaEventRecord(pins_[k].ev, stream_), "event");
    dst += filled;
    k ^= 1;
  }
}

bool Engine::copy_out(const uint32_t* src, const std::vector<HostSpan>& spans, cudaStream_t s, bool wait) {
  if (!s) s = stream_;
  size_t total = 0;
  for (const HostSpan& s : spans) total += s.words;
  // Destinations that form a few long runs of page-locked memory (a batch's
  // results in one fpx_host_alloc buffer, laid out in device order): one
  // device-to-host copy per run, straight into place.
  {
    struct Run {
      size_t off, words;
      uint32_t* dst;
    };
    std::vector<Run> runs;
    size_t off = 0;
    for (const HostSpan& sp : spans) {
      if (sp.dst && !runs.empty() && runs.back().off + runs.back().words == off &&
          runs.back().dst + runs.back().words == sp.dst)
        runs.back().words += sp.words;
      else if (sp.dst)
        runs.push_back(Run{off, sp.words, sp.dst});
      off += sp.words;
    }
    constexpr size_t kMaxDirectRuns = 64;
    bool direct = !runs.empty() && runs.size() <= kMaxDirectRuns && total * 4 >= kStagedBytes;
    for (size_t r = 0; direct && r < runs.size(); ++r) direct = pinned(runs[r].dst);
    if (direct) {
      const auto tp = std::chrono::steady_clock::now();
      for (const Run& r : runs)
        check(cudaMemcpyAsync(r.dst, src + r.off, r.words * 4, cudaMemcpyDeviceToHost, s), "D2H");
      if (wait) check(cudaStreamSynchronize(s), "D2H wait");
      host_phase("direct_out", std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tp).count());
      return wait;
    }
  }
  const size_t chunks = (total + kPinWords - 1) / kPinWords;
  size_t si = 0, so = 0;
  std::vector<CopyPiece> pieces;
  auto issue = [&](size_t c) {  // D2H of chunk c into slot c % 2
    const int k = (int)(c & 1);
    uint32_t* h = pin_slot(k);
    const size_t off = c * kPinWords, w = std::min(kPinWords, total - off);
    check(cudaMemcpyAsync(h, src + off, w * 4, cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaEventRecord(pins_[k].ev, s), "event");
  };
  if (chunks > 0) issue(0);
  if (chunks > 1) issue(1);
  for (size_t c = 0; c < chunks; ++c) {
    const int k = (int)(c & 1);
    check(cudaEventSynchronize(pins_[k].ev), "D2H wait");
    const uint32_t* h = pins_[k].host;
    const size_t w = std::min(kPinWords, total - c * kPinWords);
    size_t used = 0;
    pieces.clear();
    while (used < w) {
      const size_t take = std::min(spans[si].words - so, w - used);
      if (spans[si].dst) pieces.push_back(CopyPiece{spans[si].dst + so, h + used, take * 4});
      used += take;
      so += take;
      if (so == spans[si].words) {
        ++si;
        so = 0;
      }
    }
    const auto tp = std::chrono::steady_clock::now();
    CopyPool::instance().run(pieces);
    host_phase("unpack", std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tp).count());
    if (c + 2 < chunks) issue(c + 2);
  }
  // every chunk's copy was waited for before its words were unpacked
  return true;
}

}  // namespace fpx
