// engine.cpp - host orchestration of the NTT path on one B200.
//
// Every routine here restates one of the reference's algorithms (cited by
// file:line) as a sequence of fused GPU passes on the context's stream.  The
// results are the reference's exactly: every operation is exact modular
// arithmetic, and where the reference picks between equivalent algorithms
// (direct vs NTT vs CRT products, special-cased short inputs) the GPU may pick
// differently without changing a single output residue.
#include "engine.h"

#include <algorithm>
#include <chrono>
#include <bit>
#include <cstdlib>
#include <cstring>

#include "fpx_b200.h"

namespace fpx {

// ------------------------------------------------------------------ numbers

uint32_t powm(uint32_t a, uint64_t e, uint32_t p) {
  uint64_t r = 1 % p, b = a % p;
  for (; e; e >>= 1) {
    if (e & 1) r = r * b % p;
    b = b * b % p;
  }
  return (uint32_t)r;
}

uint32_t invm(uint32_t a, uint32_t p) { return p == 2 ? (a & 1u) : powm(a, (uint64_t)p - 2, p); }

int v2_of(uint32_t p) {
  uint32_t t = p - 1;
  int k = 0;
  while (t && !(t & 1)) { t >>= 1; ++k; }
  return k;
}

// modint.hpp:28-52: the smallest primitive root.
uint32_t primitive_root(uint32_t p) {
  if (p == 2) return 1;
  uint32_t f[16];
  int nf = 0;
  uint32_t rem = p - 1;
  for (uint32_t d = 2; (uint64_t)d * d <= rem; ++d) {
    if (rem % d) continue;
    f[nf++] = d;
    while (rem % d == 0) rem /= d;
  }
  if (rem > 1) f[nf++] = rem;
  for (uint32_t g = 2; g < p; ++g) {
    bool ok = true;
    for (int i = 0; i < nf && ok; ++i) ok = powm(g, (p - 1) / f[i], p) != 1;
    if (ok) return g;
  }
  return 0;
}

namespace {
bool is_prime_mr(uint32_t n);
}  // namespace

// Batches check the modulus of every job, a handful of distinct primes over
// thousands of jobs: the last few answers are kept per thread.
bool is_prime(uint32_t n) {
  thread_local uint32_t seen[8] = {};
  thread_local bool ans[8] = {};
  thread_local int next = 0;
  for (int i = 0; i < 8; ++i)
    if (seen[i] == n && n) return ans[i];
  const bool r = is_prime_mr(n);
  seen[next] = n;
  ans[next] = r;
  next = (next + 1) & 7;
  return r;
}

namespace {
bool is_prime_mr(uint32_t n) {
  if (n < 2) return false;
  for (uint32_t q : {2u, 3u, 5u, 7u, 11u, 13u})
    if (n % q == 0) return n == q;
  uint32_t d = n - 1;
  int s = 0;
  while (!(d & 1)) { d >>= 1; ++s; }
  for (uint32_t a : {2u, 3u, 5u, 7u}) {  // deterministic below 3.2e9
    uint64_t x = powm(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool comp = true;
    for (int r = 1; r < s; ++r) {
      x = x * x % n;
      if (x == n - 1) { comp = false; break; }
    }
    if (comp) return false;
  }
  return true;
}
}  // namespace

// modint.hpp:139-166, the reference's root choice (Tonelli-Shanks, z from 2).
bool sqrt_mod(uint32_t x, uint32_t p, uint32_t* out) {
  if (p == 2) { *out = x & 1u; return true; }
  if (x == 0) { *out = 0; return true; }
  if (powm(x, (p - 1) / 2, p) != 1) return false;
  if (p % 4 == 3) { *out = powm(x, ((uint64_t)p + 1) / 4, p); return true; }
  uint64_t q = p - 1;
  int s = 0;
  while (q % 2 == 0) { q /= 2; ++s; }
  uint32_t z = 2;
  while (powm(z, (p - 1) / 2, p) != p - 1) z = (uint32_t)((z + 1ull) % p);
  uint32_t c = powm(z, q, p), r = powm(x, (q + 1) / 2, p), t = powm(x, q, p);
  int m = s;
  while (t != 1) {
    int i = 0;
    for (uint64_t t2 = t; t2 != 1; t2 = t2 * t2 % p) ++i;
    const uint32_t b = powm(c, (uint64_t)1 << (m - i - 1), p);
    r = (uint32_t)((uint64_t)r * b % p);
    c = (uint32_t)((uint64_t)b * b % p);
    t = (uint32_t)((uint64_t)t * c % p);
    m = i;
  }
  *out = r;
  return true;
}

// crt_convolution.hpp:78-83.
size_t crt_prime_count(uint32_t p, size_t terms) {
  const uint64_t square = (uint64_t)(p - 1) * (p - 1);
  const uint64_t P1 = 167772161u, P2 = 469762049u;
  if (square <= (P1 - 1) / terms) return 1;
  if (square <= (P1 * P2 - 1) / terms) return 2;
  return 3;
}

static const uint32_t kCrtPrimes[3] = {167772161u, 469762049u, 754974721u};
static constexpr size_t kCrtBlock = size_t(1) << 23;   // crt_convolution.hpp:19
static constexpr size_t kNaive = 40;                   // base.hpp:89

// Kernel launches go through kcheck: error check, launch counter and (when
// profiling is on) CUDA events on the launching stream around the launch.
#define kcheck(call, what)   \
  do {                       \
    prof_begin();            \
    check((call), what);     \
    prof_end(what);          \
  } while (0)

static Tw2 shoup_pair(uint32_t w, uint32_t p) { return Tw2{w, (uint32_t)(((uint64_t)w << 32) / p)}; }

// --------------------------------------------------------------------- pool

namespace {
// The stream-ordered pool of a device, created on first use and kept for the
// process: reserved memory is never handed back on synchronisation (release
// threshold: all of it), and an allocation never waits for another stream's
// work to reuse memory freed there (it takes completed frees or grows).
cudaMemPool_t stream_pool(int device) {
  static std::mutex mu;
  static cudaMemPool_t pools[64];
  static bool tried[64];
  if (device < 0 || device >= 64) return nullptr;
  std::lock_guard<std::mutex> g(mu);
  if (!tried[device]) {
    tried[device] = true;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t mp = nullptr;
    if (cudaMemPoolCreate(&mp, &props) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      int no = 0;
      if (cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &keep) == cudaSuccess &&
          cudaMemPoolSetAttribute(mp, cudaMemPoolReuseAllowInternalDependencies, &no) == cudaSuccess)
        pools[device] = mp;
      else
        cudaMemPoolDestroy(mp);
    }
    cudaGetLastError();
  }
  return pools[device];
}

uint64_t pool_reserved(cudaMemPool_t mp) {
  uint64_t v = 0;
  if (cudaMemPoolGetAttribute(mp, cudaMemPoolAttrReservedMemCurrent, &v) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return (uint64_t)v;
}
}  // namespace

Pool::~Pool() { release(); }

uint32_t* Pool::get(size_t words, size_t* cls_out) {
  size_t bytes = words * sizeof(uint32_t);
  size_t cls = 1024;
  while (cls < bytes) cls <<= 1;
  if (cls >= kStreamBytes) {
    // large: from the device's stream-ordered pool, rounded to 2 MiB
    cudaMemPool_t mp = nullptr;
    const size_t size = (bytes + (size_t(2) << 20) - 1) & ~((size_t(2) << 20) - 1);
    {
      std::lock_guard<std::mutex> g(mu_);
      if (!capturing_ && stream_) mp = stream_pool(device_);
      if (mp) {
        if (limit_ && in_use_bytes + size > limit_)
          throw Error{FPX_ENOMEM, "device pool limit reached (" + std::to_string(limit_) + " bytes)"};
        in_use_bytes += size;
      }
    }
    if (mp) {
      const auto t0 = std::chrono::steady_clock::now();
      const uint64_t r0 = pool_reserved(mp);
      void* p = nullptr;
      cudaError_t e = cudaMallocFromPoolAsync(&p, size, mp, *stream_);
      if (e != cudaSuccess) {
        cudaGetLastError();
        release();  // the free lists' cache, and the pool's unused reservation
        e = cudaMallocFromPoolAsync(&p, size, mp, *stream_);
      }
      if (e != cudaSuccess) {
        cudaGetLastError();
        std::lock_guard<std::mutex> g(mu_);
        in_use_bytes -= size;
        throw Error{FPX_ENOMEM, "device allocation of " + std::to_string(size) + " bytes failed"};
      }
      const bool grew = pool_reserved(mp) > r0;
      const uint64_t ns = static_cast<uint64_t>(
          std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count());
      std::lock_guard<std::mutex> g(mu_);
      async_.insert(p);
      if (grew) {
        ++system_allocations;
        alloc_ns += ns;
        alloc_ns_max = std::max(alloc_ns_max, ns);
      } else {
        ++cache_hits;
      }
      *cls_out = size;
      return static_cast<uint32_t*>(p);
    }
  }
  {
    std::lock_guard<std::mutex> g(mu_);
    if (capturing_) {
      auto ct = cap_free_.find(cls);
      if (ct != cap_free_.end() && !ct->second.empty()) {
        uint32_t* p = ct->second.back();
        ct->second.pop_back();
        *cls_out = cls;
        return p;
      }
    }
    auto it = free_.find(cls);
    if (it != free_.end() && !it->second.empty()) {
      void* p = it->second.back();
      it->second.pop_back();
      cached_bytes -= cls;
      --cached_blocks;
      ++cache_hits;
      in_use_bytes += cls;
      *cls_out = cls;
      if (capturing_) cap_owned_[static_cast<uint32_t*>(p)] = cls;
      return static_cast<uint32_t*>(p);
    }
    // A large class with nothing cached takes the smallest cached block of up
    // to four times its size: a batch's arena is sized by the sum of its jobs'
    // scratch, so batches of new shapes keep asking for classes not seen yet,
    // and a cudaMalloc of several GB holds the caller (and the driver's
    // allocation lock) for up to ~100 ms.
    if (cls >= kFitBytes) {
      for (auto ft = free_.upper_bound(cls); ft != free_.end() && ft->first <= 4 * cls; ++ft) {
        if (ft->second.empty() || (limit_ && in_use_bytes + ft->first > limit_)) continue;
        void* p = ft->second.back();
        ft->second.pop_back();
        cached_bytes -= ft->first;
        --cached_blocks;
        ++cache_hits;
        in_use_bytes += ft->first;
        *cls_out = ft->first;
        if (capturing_) cap_owned_[static_cast<uint32_t*>(p)] = ft->first;
        return static_cast<uint32_t*>(p);
      }
    }
    // The limit is checked and the block's bytes reserved under the lock, so
    // concurrent callers of one pool cannot together pass the limit.
    if (limit_ && in_use_bytes + cls > limit_)
      throw Error{FPX_ENOMEM, "device pool limit reached (" + std::to_string(limit_) + " bytes)"};
    in_use_bytes += cls;
  }
  auto unreserve = [&] {
    std::lock_guard<std::mutex> g(mu_);
    in_use_bytes -= cls;
  };
  bool trim;
  {
    std::lock_guard<std::mutex> g(mu_);
    trim = limit_ && in_use_bytes + cached_bytes > limit_;
  }
  if (trim) release();
  void* p = nullptr;
  const auto t0 = std::chrono::steady_clock::now();
  cudaError_t e = cudaMalloc(&p, cls);
  if (e != cudaSuccess) {
    cudaGetLastError();
    release();
    e = cudaMalloc(&p, cls);
    if (e != cudaSuccess) {
      cudaGetLastError();
      unreserve();
      throw Error{FPX_ENOMEM, "cudaMalloc of " + std::to_string(cls) + " bytes failed"};
    }
  }
  const uint64_t ns = static_cast<uint64_t>(
      std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count());
  std::lock_guard<std::mutex> g(mu_);
  ++system_allocations;
  alloc_ns += ns;
  alloc_ns_max = std::max(alloc_ns_max, ns);
  *cls_out = cls;
  if (capturing_) cap_owned_[static_cast<uint32_t*>(p)] = cls;
  return static_cast<uint32_t*>(p);
}

void Pool::put(uint32_t* p, size_t cls) {
  std::lock_guard<std::mutex> g(mu_);
  if (async_.erase(p)) {
    // back to the stream-ordered pool after the stream's work on it
    if (stream_) {
      if (cudaFreeAsync(p, *stream_) != cudaSuccess) cudaGetLastError();
    } else if (cudaFree(p) != cudaSuccess) {
      cudaGetLastError();
    }
    in_use_bytes -= cls;
    return;
  }
  if (capturing_ && cap_owned_.count(p)) {
    cap_free_[cls].push_back(p);  // reused only inside the graph being captured
    return;
  }
  free_[cls].push_back(p);
  cached_bytes += cls;
  ++cached_blocks;
  in_use_bytes -= cls;
}

void Pool::begin_capture() {
  std::lock_guard<std::mutex> g(mu_);
  capturing_ = true;
  cap_owned_.clear();
  cap_free_.clear();
}

std::vector<std::pair<uint32_t*, size_t>> Pool::end_capture() {
  std::lock_guard<std::mutex> g(mu_);
  capturing_ = false;
  std::vector<std::pair<uint32_t*, size_t>> r(cap_owned_.begin(), cap_owned_.end());
  cap_owned_.clear();
  cap_free_.clear();
  return r;
}

void Pool::give_back(const std::vector<std::pair<uint32_t*, size_t>>& blocks) {
  std::lock_guard<std::mutex> g(mu_);
  for (const auto& [p, cls] : blocks) {
    free_[cls].push_back(p);
    cached_bytes += cls;
    ++cached_blocks;
    in_use_bytes -= cls;
  }
}

Pool::Snapshot Pool::snapshot() {
  std::lock_guard<std::mutex> g(mu_);
  return {cached_bytes, in_use_bytes, system_allocations, flushes, alloc_ns, alloc_ns_max};
}

void Pool::release() {
  std::lock_guard<std::mutex> g(mu_);
  if (cached_blocks) ++flushes;
  for (auto& [cls, v] : free_)
    for (void* p : v) cudaFree(p);
  free_.clear();
  cached_bytes = 0;
  cached_blocks = 0;
  // the device pool's unused reservation (every engine's: only memory no
  // allocation holds is returned)
  if (device_ >= 0)
    if (cudaMemPool_t mp = stream_pool(device_))
      if (cudaMemPoolTrimTo(mp, 0) != cudaSuccess) cudaGetLastError();
}

// ------------------------------------------------------------------- engine

Engine::Engine(int device, size_t pool_limit) : device_(device), pool_(pool_limit), crt_block_(kCrtBlock) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    throw Error{FPX_EUNSUPPORTED, "no CUDA device"};
  }
  if (device < 0 || device >= n) throw Error{FPX_EINVAL, "device index out of range"};
  check(cudaSetDevice(device), "cudaSetDevice");
  check(cudaStreamCreateWithFlags(&own_stream_, cudaStreamNonBlocking), "cudaStreamCreate");
  stream_ = own_stream_;
  pool_.bind(device, &stream_);
  check(kernels_init(), "kernel attributes");
  check(cudaMalloc(&scratch_ull_, 16), "cudaMalloc");
  check(cudaMallocHost(&host_ull_, 16), "cudaMallocHost");
  check(cudaMallocHost(&host_one_, 4), "cudaMallocHost");
  *host_one_ = 1;
  check(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking), "cudaStreamCreate");
  check(cudaEventCreateWithFlags(&side_fork_, cudaEventDisableTiming), "cudaEventCreate");
  check(cudaEventCreateWithFlags(&side_join_, cudaEventDisableTiming), "cudaEventCreate");
  const char* g = std::getenv("FPX_GRAPHS");
  graphs_on_ = !(g && g[0] == '0');
}

Engine::~Engine() {
  cudaSetDevice(device_);
  if (stream_) cudaStreamSynchronize(stream_);
  drop_graphs();
  if (host_one_) cudaFreeHost(host_one_);
  if (side_) {
    cudaStreamSynchronize(side_);
    cudaStreamDestroy(side_);
  }
  if (side_fork_) cudaEventDestroy(side_fork_);
  if (side_join_) cudaEventDestroy(side_join_);
  if (copy_stream_) {
    cudaStreamSynchronize(copy_stream_);
    cudaStreamDestroy(copy_stream_);
  }
  for (cudaEvent_t e : chunk_ev_)
    if (e) cudaEventDestroy(e);
  primes_.clear();
  bigs_.clear();
  inv_tabs_.clear();
  drop_flush_arena();
  free_stages();
  for (auto& r : prof_recs_) { cudaEventDestroy(r.b); cudaEventDestroy(r.e); }
  for (auto ev : ev_free_) cudaEventDestroy(ev);
  if (scratch_ull_) cudaFree(scratch_ull_);
  if (host_ull_) cudaFreeHost(host_ull_);
  pool_.release();
  pool_.unbind();  // blocks the members still hold are freed synchronously
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

void Engine::check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error{FPX_ECUDA, std::string(what) + ": " + cudaGetErrorString(e)};
  }
}

void Engine::sync() { check(cudaStreamSynchronize(stream_), "cudaStreamSynchronize"); }

void Engine::prof_begin() {
  if (!prof_on_) return;
  if (ev_free_.size() < 2) {
    for (int i = 0; i < 64; ++i) {
      cudaEvent_t ev;
      check(cudaEventCreate(&ev), "cudaEventCreate");
      ev_free_.push_back(ev);
    }
  }
  cudaEvent_t ev = ev_free_.back();
  ev_free_.pop_back();
  check(cudaEventRecord(ev, stream_), "cudaEventRecord");
  prof_open_ = ev;
}

void Engine::prof_end(const char* what) {
  ++launches_;
  if (!prof_on_) return;
  cudaEvent_t ev = ev_free_.back();
  ev_free_.pop_back();
  check(cudaEventRecord(ev, stream_), "cudaEventRecord");
  prof_recs_.push_back(ProfRec{what, prof_open_, ev});
}

void Engine::profile(bool on) {
  sync();
  for (auto& r : prof_recs_) {
    ev_free_.push_back(r.b);
    ev_free_.push_back(r.e);
  }
  prof_recs_.clear();
  host_prof_.clear();
  prof_on_ = on;
}

std::string Engine::profile_report() {
  sync();
  std::map<std::string, std::pair<long, double>> agg = host_prof_;
  for (auto& r : prof_recs_) {
    float ms = 0;
    check(cudaEventElapsedTime(&ms, r.b, r.e), "cudaEventElapsedTime");
    auto& a = agg[r.name];
    a.first += 1;
    a.second += ms;
  }
  std::string out = "{";
  bool first = true;
  for (auto& [name, v] : agg) {
    out += (first ? "\"" : ", \"") + name + "\": [" + std::to_string(v.first) + ", " + std::to_string(v.second) + "]";
    first = false;
  }
  return out + "}";
}

void Engine::set_stream(cudaStream_t s) {
  // Pool blocks are recycled in stream order; drain the old stream first.
  sync();
  stream_ = s ? s : own_stream_;
}

// ---------------------------------------------------------------- graphs

namespace {
constexpr size_t kMaxGraphs = 16;
constexpr size_t kMaxGraphBytes = size_t(4) << 30;
constexpr size_t kMaxSeen = 256;
}  // namespace

void Engine::free_graph(GraphEntry& g) {
  if (g.exec) cudaGraphExecDestroy(g.exec);
  if (g.graph) cudaGraphDestroy(g.graph);
  pool_.give_back(g.blocks);
  g = GraphEntry{};
}

void Engine::drop_graphs() {
  graph_seen_.clear();
  if (graphs_.empty()) return;
  cudaStreamSynchronize(stream_);  // no replay in flight
  for (auto& [k, g] : graphs_) free_graph(g);
  graphs_.clear();
}

// Every product of a Newton operation of n terms transforms at most 2n points;
// on a prime with roots of that order no step needs the host (CRT products go
// through the descriptor staging ring, which waits on events).
bool Engine::graph_native(uint32_t p, size_t n) const { return n >= 2 && native(p, std::bit_width(2 * n - 1)); }

void Engine::run_graph(const GraphKey& key, const std::function<void()>& fn) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream_, &cs) != cudaSuccess) {
    cudaGetLastError();
    cs = cudaStreamCaptureStatusNone;
  }
  if (!graphs_on_ || prof_on_ || cs != cudaStreamCaptureStatusNone) {
    fn();  // (a caller capturing this stream records the launches itself)
    return;
  }
  auto it = graphs_.find(key);
  if (it == graphs_.end()) {
    if (!graph_seen_.count(key)) {
      // first call: run it directly (this also builds every plan and table the
      // operation needs, so the capture below makes no host round trip)
      if (graph_seen_.size() >= kMaxSeen) graph_seen_.clear();
      graph_seen_.insert(key);
      fn();
      return;
    }
    const uint64_t l0 = launches_;
    pool_.begin_capture();
    const cudaError_t be = cudaStreamBeginCapture(stream_, cudaStreamCaptureModeRelaxed);
    if (be != cudaSuccess) {
      cudaGetLastError();
      pool_.give_back(pool_.end_capture());
      throw Error{FPX_ECUDA, std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(be)};
    }
    GraphEntry e;
    try {
      fn();
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(stream_, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      pool_.give_back(pool_.end_capture());
      launches_ = l0;
      graph_seen_.erase(key);
      throw;
    }
    const cudaError_t ce = cudaStreamEndCapture(stream_, &e.graph);
    e.blocks = pool_.end_capture();
    if (ce != cudaSuccess) {
      cudaGetLastError();
      free_graph(e);
      throw Error{FPX_ECUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ce)};
    }
    const cudaError_t ie = cudaGraphInstantiate(&e.exec, e.graph, 0);
    if (ie != cudaSuccess) {
      cudaGetLastError();
      free_graph(e);
      throw Error{FPX_ECUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie)};
    }
    for (const auto& b : e.blocks) e.bytes += b.second;
    e.kernels = launches_ - l0;
    launches_ = l0;  // nothing ran during the capture
    // keep at most kMaxGraphs graphs and kMaxGraphBytes of graph scratch
    size_t total = e.bytes;
    for (const auto& [k, g] : graphs_) total += g.bytes;
    while (!graphs_.empty() && (graphs_.size() >= kMaxGraphs || total > kMaxGraphBytes)) {
      auto old = graphs_.begin();
      for (auto j = graphs_.begin(); j != graphs_.end(); ++j)
        if (j->second.last_use < old->second.last_use) old = j;
      cudaStreamSynchronize(stream_);
      total -= old->second.bytes;
      free_graph(old->second);
      graphs_.erase(old);
    }
    it = graphs_.emplace(key, std::move(e)).first;
  }
  it->second.last_use = ++graph_clock_;
  check(cudaGraphLaunch(it->second.exec, stream_), "cudaGraphLaunch");
  launches_ += it->second.kernels;
}

uint32_t Engine::read_word(const uint32_t* d) {
  check(cudaMemcpyAsync(host_ull_, d, 4, cudaMemcpyDeviceToHost, stream_), "read");
  sync();
  uint32_t v;
  std::memcpy(&v, host_ull_, 4);
  return v;
}

size_t Engine::find_nonzero(const uint32_t* a, size_t n, bool last) {
  if (n == 0) return 0;
  const unsigned long long init = last ? 0ull : ~0ull;
  check(cudaMemcpyAsync(scratch_ull_, &init, 8, cudaMemcpyHostToDevice, stream_), "scan init");
  kcheck(launch_find_nonzero(a, n, last ? 1 : 0, scratch_ull_, stream_), "scan");
  check(cudaMemcpyAsync(host_ull_, scratch_ull_, 8, cudaMemcpyDeviceToHost, stream_), "scan read");
  sync();
  const unsigned long long r = *host_ull_;
  if (last) {
    // 0 is ambiguous: distinguish "a[0] != 0" from "all zero".
    if (r == 0) return read_word(a) ? 0 : n;
    return (size_t)r;
  }
  return r == ~0ull ? n : (size_t)r;
}

bool Engine::native(uint32_t p, int logN) const {
  return (p & 1u) && p < (1u << 30) && logN >= 1 && logN <= 25 && logN <= v2_of(p);
}

// ---------------------------------------------------------------------- plans

namespace {
struct HostTables {
  std::vector<Tw2> fwd, inv;
};
}  // namespace

// Plans are uploaded on the engine's stream and waited for: the engine's stream
// does not synchronise with the legacy default stream, and a plan outlives
// stream changes (set_stream), so the tables must be complete before any use.
static uint32_t* upload(Engine& eng, Buf& dst, const std::vector<Tw2>& v) {
  dst = Buf(&eng.pool(), v.size() * 2);
  eng.check(cudaMemcpyAsync(dst.get(), v.data(), v.size() * sizeof(Tw2), cudaMemcpyHostToDevice, eng.stream()),
            "plan upload");
  eng.sync();
  return dst.get();
}

// Per-prime tables (the reference's per-stage tables, ntt.hpp:385-506, merged
// into one table indexed by block length): tw[h + k] = w_{2h}^k.
const PrimePlan& Engine::prime_plan(uint32_t p) {
  std::lock_guard<std::mutex> g(plan_mu_);
  return prime_plan_locked(p);
}

const PrimePlan& Engine::prime_plan_locked(uint32_t p) {
  auto it = primes_.find(p);
  if (it != primes_.end()) return *it->second;
  auto plan = std::make_unique<PrimePlan>();
  const int maxlog = v2_of(p);
  const int small = std::min(maxlog, 13);
  const uint32_t gen = primitive_root(p);
  std::vector<Tw2> fwd(size_t(1) << small), inv(size_t(1) << small);
  fwd[0] = inv[0] = shoup_pair(1, p);
  for (int lg = 1; lg <= small; ++lg) {
    const uint32_t len = 1u << lg, h = len / 2;
    const uint32_t w = powm(gen, (p - 1) / len, p), wi = invm(w, p);
    uint64_t c = 1, ci = 1;
    for (uint32_t k = 0; k < h; ++k) {
      fwd[h + k] = shoup_pair((uint32_t)c, p);
      inv[h + k] = shoup_pair((uint32_t)ci, p);
      c = c * w % p;
      ci = ci * wi % p;
    }
  }
  plan->t.p = p;
  plan->t.max_log = maxlog;
  plan->t.small_log = small;
  plan->t.fwd = reinterpret_cast<const Tw2*>(upload(*this, plan->fwd, fwd));
  plan->t.inv = reinterpret_cast<const Tw2*>(upload(*this, plan->inv, inv));
  plan->t.q1 = (uint32_t)((((uint64_t)1) << 32) / p);
  const uint64_t r32 = (((uint64_t)1) << 32) % p;
  for (int k = 0; k <= 13; ++k) {
    plan->t.inv_pow2[k] = invm((uint32_t)((((uint64_t)1) << k) % p), p);
    plan->t.inv_pow2_r[k] = (uint32_t)(plan->t.inv_pow2[k] * r32 % p);
  }
  auto& ref = *plan;
  primes_[p] = std::move(plan);
  return ref;
}

// Per-(prime, N) Bailey twiddles of the two-pass decomposition.
const BigPlan& Engine::big_plan(uint32_t p, int logN) {
  std::lock_guard<std::mutex> g(plan_mu_);
  auto key = std::make_pair(p, logN);
  auto it = bigs_.find(key);
  if (it != bigs_.end()) return *it->second;
  auto plan = std::make_unique<BigPlan>();
  const uint32_t gen = primitive_root(p);
  const uint64_t N = uint64_t(1) << logN;
  const uint32_t wN = powm(gen, (p - 1) / N, p);
  const uint32_t invN = invm((uint32_t)(N % p), p);
  const uint32_t R = (uint32_t)((((uint64_t)1) << 32) % p);
  // w_N^e = lo[e & 255] * mid[(e >> 8) & 255] * hi[e >> 16]; 1/N (and 2^32/N)
  // ride on the inverse lo table
  const size_t nhi = std::max<size_t>(1, N >> 16);
  std::vector<Tw2> lo_f(256), lo_i(256), lo_ir(256), mid_f(256), mid_i(256), hi_f(nhi), hi_i(nhi);
  auto fill = [&](std::vector<Tw2>& f, std::vector<Tw2>& fi, uint32_t step, size_t cnt) {
    const uint32_t stepi = invm(step, p);
    uint64_t c = 1, ci = 1;
    for (size_t y = 0; y < cnt; ++y) {
      f[y] = shoup_pair((uint32_t)c, p);
      fi[y] = shoup_pair((uint32_t)ci, p);
      c = c * step % p;
      ci = ci * stepi % p;
    }
  };
  fill(lo_f, lo_i, wN, 256);
  fill(mid_f, mid_i, powm(wN, 256, p), 256);
  fill(hi_f, hi_i, powm(wN, 65536, p), nhi);
  for (size_t y = 0; y < 256; ++y) {
    const uint32_t v = (uint32_t)((uint64_t)lo_i[y].w * invN % p);
    lo_i[y] = shoup_pair(v, p);
    lo_ir[y] = shoup_pair((uint32_t)((uint64_t)v * R % p), p);
  }
  plan->t.logN = logN;
  plan->t.logC = logN >= 25 ? 13 : 12;  // 2^24 = 2^12 x 2^12 keeps the fast 4096-point row pass
  plan->t.logR = logN - plan->t.logC;
  plan->t.lo_fwd = reinterpret_cast<const Tw2*>(upload(*this, plan->lo_fwd, lo_f));
  plan->t.mid_fwd = reinterpret_cast<const Tw2*>(upload(*this, plan->mid_fwd, mid_f));
  plan->t.hi_fwd = reinterpret_cast<const Tw2*>(upload(*this, plan->hi_fwd, hi_f));
  plan->t.lo_inv = reinterpret_cast<const Tw2*>(upload(*this, plan->lo_inv, lo_i));
  plan->t.lo_inv_r = reinterpret_cast<const Tw2*>(upload(*this, plan->lo_inv_r, lo_ir));
  plan->t.mid_inv = reinterpret_cast<const Tw2*>(upload(*this, plan->mid_inv, mid_i));
  plan->t.hi_inv = reinterpret_cast<const Tw2*>(upload(*this, plan->hi_inv, hi_i));
  // Column factors (BigTables::cf_fwd): for R >= 2^9 points per column
  // (transforms of 2^21 points and up), where they measured faster; smaller
  // transforms were as fast or slightly slower with them.  FPX_COL_FACTOR=0
  // keeps the three small-table products per point everywhere.  The column
  // kernels take the factored path for R >= 2^9 only.
  const char* cfe = std::getenv("FPX_COL_FACTOR");
  if (plan->t.logR >= 9 && !(cfe && cfe[0] == '0')) {
    const int G = col_last_group_log(plan->t.logR);
    const size_t C = size_t(1) << plan->t.logC, P = size_t(1) << G;
    std::vector<Tw2> cf(C * P), ci(C * P);
    const uint32_t step = powm(wN, uint64_t(1) << (plan->t.logR - G), p);
    const uint32_t stepi = invm(step, p);
    std::vector<uint32_t> pw(P), pwi(P);
    uint64_t u = 1, ui = 1;  // U_j, U_j^-1
    for (size_t j = 0; j < C; ++j) {
      pw[0] = pwi[0] = 1;
      for (size_t k = 1; k < P; ++k) {
        pw[k] = (uint32_t)(pw[k - 1] * u % p);
        pwi[k] = (uint32_t)(pwi[k - 1] * ui % p);
      }
      for (size_t i = 0; i < P; ++i) {
        size_t k = 0;  // bitrev_G(i)
        for (int b = 0; b < G; ++b) k |= ((i >> b) & 1) << (G - 1 - b);
        const size_t idx = 2 * ((j >> 1) * P + i) + (j & 1);
        cf[idx] = shoup_pair(pw[k], p);
        ci[idx] = shoup_pair(pwi[k], p);
      }
      u = u * step % p;
      ui = ui * stepi % p;
    }
    plan->t.cf_fwd = reinterpret_cast<const Tw2*>(upload(*this, plan->cf_fwd, cf));
    plan->t.cf_inv = reinterpret_cast<const Tw2*>(upload(*this, plan->cf_inv, ci));
  }
  plan->t.shapes = tuned_shapes_locked(p, plan->t);
  auto& ref = *plan;
  bigs_[key] = std::move(plan);
  return ref;
}

// Montgomery-form table of 1/i, i <= n (the reference's inv_series,
// calculus.hpp:53-94), cached per prime and grown on demand.
const uint32_t* Engine::inv_table(uint32_t p, size_t n) {
  std::lock_guard<std::mutex> g(plan_mu_);
  auto it = inv_tabs_.find(p);
  if (it != inv_tabs_.end() && it->second.first >= n) return it->second.second.get();
  size_t want = std::max<size_t>(n, 1024);
  if (it != inv_tabs_.end()) want = std::max(want, it->second.first * 2);
  want = std::min<size_t>(want, (size_t)p - 1);
  Buf b(&pool_, want + 1);
  kcheck(launch_inv_table(p, b.get(), want, stream_), "inv table");
  auto& slot = inv_tabs_[p];
  slot.first = want;
  slot.second = std::move(b);
  return slot.second.get();
}

// --------------------------------------------------------------- products

void Engine::cyc_product(uint32_t p, int logN, const CycOp& op) {
  const PrimeTables& pt = prime_plan(p).t;
  const uint32_t N = 1u << logN;
  Epi epi = op.epi;
  if (logN <= small_kernel_max_log()) {
    SmallJob j;
    j.forward = 1;
    j.x = op.x;
    j.ymode = op.ymode;
    j.y = op.y;
    j.yspec = op.yspec;
    j.yspec_out = op.yspec_out;
    j.inverse = 1;
    // 1/N, times 2^32 after a Montgomery pointwise product, times the caller's factor.
    uint64_t s = op.ymode != 0 ? pt.inv_pow2_r[logN] : pt.inv_pow2[logN];
    if (epi.scale.w) s = s * epi.scale.w % p;
    epi.scale = shoup_pair((uint32_t)s, p);
    j.epi = epi;
    if (logN == 12) kcheck(launch_cyc4096(pt, j, stream_), "cyc4096");
    else kcheck(launch_cyc_small(pt, logN, j, stream_), "small");
    return;
  }
  const BigTables& bt = big_plan(p, logN).t;
  if (epi.scale.w) epi.scale = shoup_pair(epi.scale.w % p, p);
  Buf t1(&pool_, N), t2;
  InOp ins[2] = {op.x, op.y};
  uint32_t* outs[2] = {t1.get(), nullptr};
  int nops = 1;
  if (op.ymode == 1) {
    t2 = Buf(&pool_, N);
    outs[1] = t2.get();
    nops = 2;
  }
  kcheck(launch_colfwd(pt, bt, nops, ins, outs, stream_), "colfwd");
  const uint32_t* y = op.ymode == 1 ? t2.get() : op.yspec;
  kcheck(launch_rows(pt, bt, t1.get(), y, op.ymode, op.yspec_out, 1, 1, stream_), "rows");
  kcheck(launch_colinv(pt, bt, t1.get(), op.ymode != 0, epi, stream_), "colinv");
}

void Engine::product(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t outn,
                     uint32_t* out, const uint32_t* post_mont, bool accumulate) {
  if (outn == 0) return;
  la = std::min(la, outn);  // coefficients at or beyond outn never reach the output
  lb = std::min(lb, outn);
  if (la == 0 || lb == 0) {
    if (!accumulate) check(cudaMemsetAsync(out, 0, outn * 4, stream_), "memset");
    return;
  }
  const size_t full = la + lb - 1;
  if (outn > full) {
    if (!accumulate) check(cudaMemsetAsync(out + full, 0, (outn - full) * 4, stream_), "memset");
    outn = full;
  }
  if (std::min(la, lb) <= kNaive) {
    // convolution.hpp:33-95: direct product for a short operand.
    const bool swap = la > lb;
    kcheck(launch_direct_product(p, swap ? b : a, swap ? lb : la, swap ? a : b, swap ? la : lb, 0, outn, out,
                                accumulate ? 1 : 0, stream_),
          "direct");
    if (post_mont) kcheck(launch_mul_mont_tab(p, out, post_mont, out, outn, stream_), "post scale");
    return;
  }
  const int logN = std::bit_width(full - 1);
  if (native(p, logN)) {
    CycOp op;
    op.x = InOp{a, (uint32_t)la, 0};
    if (a == b && la == lb) op.ymode = 3;
    else { op.ymode = 1; op.y = InOp{b, (uint32_t)lb, 0}; }
    op.epi.out = out;
    op.epi.lo = 0;
    op.epi.hi = (uint32_t)outn;
    op.epi.mul_mont = post_mont;
    op.epi.accumulate = accumulate ? 1 : 0;
    cyc_product(p, logN, op);
    return;
  }
  if (!accumulate && logN <= 20 && std::max(la, lb) <= crt_block_) {
    // one block pair of at most 2^20 points: the auxiliary primes' transforms
    // share one launch set and the Garner epilogue applies post_mont (larger
    // products measured 4 % faster on separate per-prime launches)
    window_product(p, a, la, b, lb, 0, outn, out, 0, post_mont, false);
    return;
  }
  crt_product(p, a, la, b, lb, outn, out, accumulate);
  if (post_mont) kcheck(launch_mul_mont_tab(p, out, post_mont, out, outn, stream_), "post scale");
}

// crt_convolution<M> (crt_convolution.hpp:187-205) with crt_product_window
// (:132-182): block pairs of at most 2^23 terms, each an exact integer product
// modulo 1, 2 or 3 auxiliary primes (lifted on load) and a Garner epilogue
// accumulating into the target field.
// Blocked CRT product with every block transformed once (crt_convolution.hpp
// multiplies the 2^23-term blocks pairwise).  Per auxiliary prime: the spectra
// of all blocks of a and b at N = 2^24, then for every output block s the sum
// of SA_i * SB_j over i + j = s in the spectral domain, one inverse transform,
// and the window added into that prime's residues at s * 2^23; one Garner pass
// at the end.  nA + nB forward and nA + nB - 1 inverse transforms per prime
// instead of 3 nA nB.  The whole coefficient is reconstructed at once, so this
// needs (p-1)^2 min(la, lb) below the auxiliary primes' product (false: not
// taken; crt_product's per-pair path reconstructs each pair separately).
void Engine::set_crt_block(size_t terms) {
  if (terms == 0) terms = kCrtBlock;
  if ((terms & (terms - 1)) || terms < (size_t(1) << 13) || terms > kCrtBlock)
    throw Error{FPX_EINVAL, "CRT block size must be a power of two in [2^13, 2^23]"};
  crt_block_ = terms;
}

bool Engine::crt_blocked(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t outn,
                         uint32_t* out, bool accumulate) {
  const size_t B = crt_block_;
  const size_t nA = (la + B - 1) / B, nB = (lb + B - 1) / B;
  if (nA * nB < 2 || std::min(la, lb) <= kNaive) return false;
  if (const char* e = std::getenv("FPX_CRT_BLOCKED"); e && e[0] == '0') return false;  // the per-pair path
  const unsigned __int128 P123 = (unsigned __int128)kCrtPrimes[0] * kCrtPrimes[1] * kCrtPrimes[2];
  if ((unsigned __int128)(p - 1) * (p - 1) * std::min(la, lb) >= P123) return false;
  const int logN = std::bit_width(2 * B - 1);
  for (uint32_t q : kCrtPrimes)
    if (!native(q, logN)) return false;
  const size_t N = size_t(1) << logN;
  const bool square = a == b && la == lb;
  // all scratch up front: without the memory (pool limit) the per-pair path,
  // which needs far less, takes over before anything is written
  std::vector<Buf> sa(nA), sb(square ? 0 : nB);
  Buf acc, win, res[3];
  try {
    for (auto& x : sa) x = Buf(&pool_, N);
    for (auto& x : sb) x = Buf(&pool_, N);
    acc = Buf(&pool_, N);
    win = Buf(&pool_, N);
    for (auto& r : res) r = Buf(&pool_, outn);
  } catch (const Error& e) {
    if (e.code != FPX_ENOMEM) throw;
    return false;
  }
  for (int k = 0; k < 3; ++k) {
    const uint32_t q = kCrtPrimes[k];
    const PrimeTables& pt = prime_plan(q).t;
    const BigTables& bt = big_plan(q, logN).t;
    check(cudaMemsetAsync(res[k].get(), 0, outn * 4, stream_), "memset");
    auto forward = [&](const uint32_t* src, size_t cnt, uint32_t* dst) {
      InOp in{src, (uint32_t)cnt, 1};  // target residues, reduced mod q on load
      uint32_t* outs[1] = {dst};
      kcheck(launch_colfwd(pt, bt, 1, &in, outs, stream_), "colfwd");
      kcheck(launch_rows(pt, bt, dst, nullptr, 0, nullptr, 1, 0, stream_), "rows");
    };
    for (size_t i = 0; i < nA; ++i) forward(a + i * B, std::min(B, la - i * B), sa[i].get());
    for (size_t j = 0; j < sb.size(); ++j) forward(b + j * B, std::min(B, lb - j * B), sb[j].get());
    for (size_t s = 0; s + 1 < nA + nB && s * B < outn; ++s) {
      std::vector<const uint32_t*> xs, ys;
      for (size_t i = 0; i < nA; ++i)
        if (s >= i && s - i < nB) {
          xs.push_back(sa[i].get());
          ys.push_back(square ? sa[s - i].get() : sb[s - i].get());
        }
      kcheck(launch_spec_mac(q, xs.data(), ys.data(), (int)xs.size(), acc.get(), N, 0, stream_), "spectral mac");
      kcheck(launch_rows(pt, bt, acc.get(), nullptr, 0, nullptr, 0, 1, stream_), "rows");
      // the window goes out through the plain epilogue (an accumulating one
      // reads every output back and measured 3.6x slower), then is added in
      const size_t w = std::min(2 * B - 1, outn - s * B);
      Epi e;  // 2^32 / N undoes the Montgomery factor of the products and the transform size
      e.out = win.get();
      e.lo = 0;
      e.hi = (uint32_t)w;
      kcheck(launch_colinv(pt, bt, acc.get(), 1, e, stream_), "colinv");
      kcheck(launch_add_into(q, res[k].get() + s * B, win.get(), w, stream_), "window add");
    }
  }
  kcheck(launch_garner(p, 3, res[0].get(), res[1].get(), res[2].get(), out, outn, accumulate ? 1 : 0, stream_),
         "garner");
  return true;
}

void Engine::crt_product(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t outn,
                         uint32_t* out, bool accumulate) {
  la = std::min(la, outn);
  lb = std::min(lb, outn);
  if (crt_blocked(p, a, la, b, lb, outn, out, accumulate)) return;
  if (!accumulate) check(cudaMemsetAsync(out, 0, outn * 4, stream_), "memset");
  for (size_t ai = 0; ai < la;) {
    const size_t na = std::min(crt_block_, la - ai);
    for (size_t bi = 0; bi < lb && bi < outn - ai;) {
      const size_t nb = std::min(crt_block_, lb - bi);
      const size_t cnt = std::min(na + nb - 1, outn - ai - bi);
      const uint32_t* pa = a + ai;
      const uint32_t* pb = b + bi;
      uint32_t* po = out + ai + bi;
      if (std::min(na, nb) <= kNaive) {
        const bool swap = na > nb;
        kcheck(launch_direct_product(p, swap ? pb : pa, swap ? nb : na, swap ? pa : pb, swap ? na : nb, 0, cnt, po, 1,
                                    stream_),
              "direct");
      } else {
        const size_t primes = crt_prime_count(p, std::min(na, nb));
        const int logN = std::bit_width(na + nb - 2);
        Buf c[3];
        for (size_t k = 0; k < primes; ++k) {
          c[k] = Buf(&pool_, cnt);
          CycOp op;
          op.x = InOp{pa, (uint32_t)na, 1};
          if (pa == pb && na == nb) op.ymode = 3;
          else { op.ymode = 1; op.y = InOp{pb, (uint32_t)nb, 1}; }
          op.epi.out = c[k].get();
          op.epi.lo = 0;
          op.epi.hi = (uint32_t)cnt;
          cyc_product(kCrtPrimes[k], logN, op);
        }
        kcheck(launch_garner(p, (int)primes, c[0].get(), c[1].get(), c[2].get(), po, cnt, 1, stream_), "garner");
      }
      bi += nb;
    }
    ai += na;
  }
}

void Engine::mul_window(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t off,
                        size_t cnt, uint32_t* out) {
  if (cnt == 0) return;
  const size_t lim = off + cnt;
  la = std::min(la, lim);
  lb = std::min(lb, lim);
  if (la == 0 || lb == 0 || la + lb - 1 <= off) {
    check(cudaMemsetAsync(out, 0, cnt * 4, stream_), "memset");
    return;
  }
  const size_t have = std::min(la + lb - 1, lim);
  Buf tmp(&pool_, have);
  product(p, a, la, b, lb, have, tmp.get());
  check(cudaMemcpyAsync(out, tmp.get() + off, (have - off) * 4, cudaMemcpyDeviceToDevice, stream_), "copy");
  if (have < lim) check(cudaMemsetAsync(out + (have - off), 0, (lim - have) * 4, stream_), "memset");
}

size_t Engine::conv(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t n,
                    uint32_t* out) {
  // conv_limbs (convolution.hpp:17-31): clamp, empty cases, output length.
  if (la == 0 || lb == 0 || n == 0) return 0;
  la = std::min(la, n);
  lb = std::min(lb, n);
  if (la > SIZE_MAX - (lb - 1)) throw Error{FPX_ELENGTH, "poly::conv: result length overflows size_t"};
  const size_t outn = std::min(la + lb - 1, n);
  product(p, a, la, b, lb, outn, out);
  return outn;
}

// ------------------------------------------------------------------ series

// extend_inverse (inverse.hpp:18-65): c[0,k) -> c[0,wanted), wanted <= 2k.
// Native: five transforms at N = 2k (two forward, a middle-product inverse
// window negated on the fly, one forward of the error, one inverse window).
void Engine::extend_inverse(uint32_t p, const uint32_t* a, size_t la, uint32_t* c, size_t k, size_t wanted) {
  const size_t hlen = wanted - k;
  if (hlen == 0) return;
  const int logN = std::bit_width(2 * k - 1);
  const size_t aw = std::min(la, wanted);
  if (native(p, logN)) {
    const uint32_t N = 1u << logN;
    Buf cs(&pool_, N), h(&pool_, hlen);
    CycOp op1;
    op1.x = InOp{a, (uint32_t)aw, 0};
    op1.ymode = 1;
    op1.y = InOp{c, (uint32_t)k, 0};
    op1.yspec_out = cs.get();
    op1.epi.out = h.get();
    op1.epi.lo = (uint32_t)k;
    op1.epi.hi = (uint32_t)(k + hlen);
    op1.epi.negate = 1;
    cyc_product(p, logN, op1);
    CycOp op2;
    op2.x = InOp{h.get(), (uint32_t)hlen, 0};
    op2.ymode = 2;
    op2.yspec = cs.get();
    op2.epi.out = c + k;
    op2.epi.lo = 0;
    op2.epi.hi = (uint32_t)hlen;
    cyc_product(p, logN, op2);
    return;
  }
  // crt_middle_product + conv_limbs (inverse.hpp:35-42).
  Buf e(&pool_, hlen);
  if (logN <= 24) {
    // the middle product is free of wraparound at N = 2k: CRT transforms of
    // 2k points instead of the full product's 4k, negation in the Garner epilogue
    window_product(p, a, aw, c, k, k, hlen, e.get(), logN, nullptr, true);
    window_product(p, e.get(), hlen, c, k, 0, hlen, c + k, logN, nullptr, false);
    return;
  }
  mul_window(p, a, aw, c, k, k, hlen, e.get());
  kcheck(launch_scale(p, e.get(), e.get(), hlen, p - 1, stream_), "negate");
  product(p, e.get(), hlen, c, k, hlen, c + k);
}

// How many terms of 1/b the fused exp / sqrt kernels leave after K terms of b:
// their schedule extends c to each step's length m2 - m by doublings.
static size_t fused_newton_csize(size_t K) {
  size_t csize = 1;
  for (size_t mm = 1; mm < K;) {
    const size_t h = std::min(2 * mm, K) - mm;
    while (csize < h) csize = std::min(2 * csize, h);
    mm += h;
  }
  return csize;
}

// The fused CRT Newton kernels for the small sizes (k_newton_*_crt);
// FPX_CRT_NEWTON=0 keeps the 32-term seeds and per-step CRT products.
bool crt_newton_on() {
  static const bool on = [] {
    const char* e = std::getenv("FPX_CRT_NEWTON");
    return !(e && e[0] == '0');
  }();
  return on;
}

void Engine::inv_into(uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out) {
  la = std::min(la, n);
  const size_t seed = std::min<size_t>(n, 32);
  size_t m = seed;
  if (native(p, newton_inv_max_log())) {
    // 1 / a[0] and every doubling step up to 2^13 terms in one CTA
    const size_t K = std::min(n, size_t(1) << newton_inv_max_log());
    kcheck(launch_newton_inv(prime_plan(p).t, a, la, out, 0, K, stream_), "newton inverse");
    m = K;
  } else if (crt_newton_on()) {
    // the same steps with three-prime CRT products, in one CTA
    const size_t K = std::min(n, size_t(1) << newton_inv_max_log());
    const PrimeTables aux[3] = {prime_plan(kCrtPrimes[0]).t, prime_plan(kCrtPrimes[1]).t,
                                prime_plan(kCrtPrimes[2]).t};
    kcheck(launch_newton_inv_crt(aux, p, a, la, out, K, stream_), "newton inverse (CRT)");
    m = K;
  } else {
    kcheck(launch_seed(0, p, a, la, out, (int)seed, 0, stream_), "inverse seed");
  }
  for (; m < n; m <<= 1) extend_inverse(p, a, la, out, m, std::min(2 * m, n));
}

// inv (inverse.hpp:163-188).
void Engine::inv(uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out) {
  if (n == 0) return;
  if (la == 0 || read_word(a) == 0) throw Error{FPX_EDOMAIN, "poly::inv: constant term is zero"};
  if (graph_native(p, n)) run_graph(GraphKey{FPX_OP_INV, p, n, la, a, out}, [&] { inv_into(p, a, la, n, out); });
  else inv_into(p, a, la, n, out);
}

// log (exponential.hpp:85-98): integral(a' * inv(a, n-1)) mod x^n.
void Engine::log_into(uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out) {
  check(cudaMemsetAsync(out, 0, n * 4, stream_), "memset");
  if (n == 1) return;
  const size_t cnt = std::min(la, n);
  if (cnt <= 1) return;
  const size_t ld = cnt - 1;
  if (p == 2) {  // n <= p = 2: log(1 + a1 x) = a1 x mod x^2
    check(cudaMemcpyAsync(out + 1, a + 1, 4, cudaMemcpyDeviceToDevice, stream_), "copy");
    return;
  }
  Buf d(&pool_, ld), ia(&pool_, n - 1);
  kcheck(launch_derivative(p, a, d.get(), cnt, stream_), "derivative");
  inv_into(p, a, la, n - 1, ia.get());
  const size_t lp = std::min(ld + n - 2, n - 1);
  const uint32_t* tab = inv_table(p, lp);
  product(p, d.get(), ld, ia.get(), n - 1, lp, out + 1, tab + 1);
}

void Engine::log(uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out) {
  if (n == 0) return;
  if (la == 0 || read_word(a) != 1 % p) throw Error{FPX_EDOMAIN, "poly::log: constant term must be 1"};
  if (n > p) throw Error{FPX_EDOMAIN, "poly::log: required denominators must be invertible (n <= mod)"};
  if (graph_native(p, n)) run_graph(GraphKey{FPX_OP_LOG, p, n, la, a, out}, [&] { log_into(p, a, la, n, out); });
  else log_into(p, a, la, n, out);
}

// exp (exponential.hpp:107-207): Newton on the high differential residual,
// eight transforms at N = 2m per doubling plus the running inverse of b.
void Engine::exp_into(uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out) {
  check(cudaMemsetAsync(out, 0, n * 4, stream_), "memset");
  check(cudaMemcpyAsync(out, host_one_, 4, cudaMemcpyHostToDevice, stream_), "one");
  const size_t cnt = std::min(la, n);
  if (cnt <= 1 || n == 1) return;
  const size_t lap = cnt - 1;
  if (p == 2) {  // n - 1 < p: exp(a1 x) = 1 + a1 x mod x^2
    check(cudaMemcpyAsync(out + 1, a + 1, 4, cudaMemcpyDeviceToDevice, stream_), "copy");
    return;
  }
  Buf ap(&pool_, lap);
  kcheck(launch_derivative(p, a, ap.get(), cnt, stream_), "derivative");
  Buf c(&pool_, n / 2 + 64);
  const uint32_t* tab = inv_table(p, n - 1);
  size_t m, csize;
  if (native(p, newton_inv_max_log())) {
    // every doubling step up to 2^13 terms (and 1/b alongside) in one CTA
    const size_t K = std::min(n, size_t(1) << newton_inv_max_log());
    kcheck(launch_newton_exp(prime_plan(p).t, ap.get(), lap, tab, out, c.get(), K, stream_), "newton exp");
    m = K;
    csize = fused_newton_csize(K);
  } else if (crt_newton_on()) {
    // the same steps with three-prime CRT products, on a three-CTA cluster
    const size_t K = std::min(n, size_t(1) << newton_inv_max_log());
    const PrimeTables aux[3] = {prime_plan(kCrtPrimes[0]).t, prime_plan(kCrtPrimes[1]).t,
                                prime_plan(kCrtPrimes[2]).t};
    kcheck(launch_newton_exp_crt(aux, p, ap.get(), lap, tab, out, c.get(), K, stream_), "newton exp (CRT)");
    m = K;
    csize = fused_newton_csize(K);
  } else {
    const size_t seed = std::min<size_t>(n, 32);
    kcheck(launch_seed(1, p, ap.get(), lap, out, (int)seed, 0, stream_), "exp seed");
    if (n == seed) return;
    csize = seed / 2;
    kcheck(launch_seed(0, p, out, seed, c.get(), (int)csize, 0, stream_), "inverse seed");
    m = seed;
  }
  for (; m < n; m *= 2) {
    const size_t m2 = std::min(2 * m, n), hlen = m2 - m;
    if (csize < hlen) {
      extend_inverse(p, out, m, c.get(), csize, hlen);
      csize = hlen;
    }
    const int logN = std::bit_width(2 * m - 1);
    const size_t lx = std::min(lap, m2 - 1);
    if (native(p, logN)) {
      const uint32_t N = 1u << logN;
      Buf bs(&pool_, N), t1(&pool_, hlen), t2(&pool_, hlen);
      CycOp op1;  // (a' b)[m-1, m-1+hlen)
      op1.x = InOp{ap.get(), (uint32_t)lx, 0};
      op1.ymode = 1;
      op1.y = InOp{out, (uint32_t)m, 0};
      op1.yspec_out = bs.get();
      op1.epi.out = t1.get();
      op1.epi.lo = (uint32_t)(m - 1);
      op1.epi.hi = (uint32_t)(m - 1 + hlen);
      cyc_product(p, logN, op1);
      CycOp op2;  // (residual * c) mod x^hlen, integrated: times 1/(m+i)
      op2.x = InOp{t1.get(), (uint32_t)hlen, 0};
      op2.ymode = 1;
      op2.y = InOp{c.get(), (uint32_t)csize, 0};
      op2.epi.out = t2.get();
      op2.epi.lo = 0;
      op2.epi.hi = (uint32_t)hlen;
      op2.epi.mul_mont = tab + m;
      cyc_product(p, logN, op2);
      CycOp op3;  // (correction * b) mod x^hlen
      op3.x = InOp{t2.get(), (uint32_t)hlen, 0};
      op3.ymode = 2;
      op3.yspec = bs.get();
      op3.epi.out = out + m;
      op3.epi.lo = 0;
      op3.epi.hi = (uint32_t)hlen;
      cyc_product(p, logN, op3);
    } else {
      Buf t1(&pool_, hlen), t2(&pool_, hlen);
      if (logN <= 24) window_product(p, ap.get(), lx, out, m, m - 1, hlen, t1.get(), logN, nullptr, false);
      else mul_window(p, ap.get(), lx, out, m, m - 1, hlen, t1.get());
      product(p, t1.get(), hlen, c.get(), csize, hlen, t2.get(), tab + m);
      product(p, t2.get(), hlen, out, m, hlen, out + m);
    }
  }
}

void Engine::exp(uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out) {
  if (n == 0) return;
  if (la != 0 && read_word(a) != 0) throw Error{FPX_EDOMAIN, "poly::exp: constant term must be 0"};
  if (n - 1 >= p) throw Error{FPX_EDOMAIN, "poly::inv_series: length must be < mod"};
  if (graph_native(p, n)) run_graph(GraphKey{FPX_OP_EXP, p, n, la, a, out}, [&] { exp_into(p, a, la, n, out); });
  else exp_into(p, a, la, n, out);
}

// sqrt (square_root.hpp:12-112).
void Engine::sqrt(uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out) {
  if (n == 0) return;
  check(cudaMemsetAsync(out, 0, n * 4, stream_), "memset");
  if (p == 2) {
    const size_t cnt = std::min(la, n);
    const unsigned long long zero = 0;
    check(cudaMemcpyAsync(scratch_ull_, &zero, 8, cudaMemcpyHostToDevice, stream_), "flag");
    kcheck(launch_sqrt_char2(a, cnt, out, scratch_ull_, stream_), "char2 sqrt");
    check(cudaMemcpyAsync(host_ull_, scratch_ull_, 8, cudaMemcpyDeviceToHost, stream_), "flag read");
    sync();
    if (*host_ull_) throw Error{FPX_EDOMAIN, "poly::sqrt: nonzero odd coefficient in characteristic 2"};
    return;
  }
  const size_t v = find_nonzero(a, la, false);
  if (v == la) return;
  if (v & 1) throw Error{FPX_EDOMAIN, "poly::sqrt: odd valuation, no square root"};
  uint32_t root0;
  if (!sqrt_mod(read_word(a + v), p, &root0)) throw Error{FPX_EDOMAIN, "poly::sqrt: non-residue constant term"};
  const size_t half = v / 2;
  if (half >= n) return;
  const size_t inner = n - half, ulen = la - v;
  const uint32_t* u = a + v;
  uint32_t* b = out + half;
  Buf c(&pool_, inner / 2 + 64);
  size_t m, csize;
  if (native(p, newton_inv_max_log())) {
    // every doubling step up to 2^13 terms (and 1/b alongside) in one CTA
    const size_t K = std::min(inner, size_t(1) << newton_inv_max_log());
    kcheck(launch_newton_sqrt(prime_plan(p).t, u, ulen, root0, invm(root0, p), b, c.get(), K, stream_),
           "newton sqrt");
    m = K;
    csize = fused_newton_csize(K);
  } else if (crt_newton_on()) {
    const size_t K = std::min(inner, size_t(1) << newton_inv_max_log());
    const PrimeTables aux[3] = {prime_plan(kCrtPrimes[0]).t, prime_plan(kCrtPrimes[1]).t,
                                prime_plan(kCrtPrimes[2]).t};
    kcheck(launch_newton_sqrt_crt(aux, p, u, ulen, root0, invm(root0, p), b, c.get(), K, stream_),
           "newton sqrt (CRT)");
    m = K;
    csize = fused_newton_csize(K);
  } else {
    const size_t seed = std::min<size_t>(inner, 32);
    kcheck(launch_seed(2, p, u, std::min(ulen, seed), b, (int)seed, root0, stream_), "sqrt seed");
    if (inner <= seed) return;
    csize = seed / 2;
    kcheck(launch_seed(0, p, b, seed, c.get(), (int)csize, 0, stream_), "inverse seed");
    m = seed;
  }
  const uint32_t half_inv = (p + 1) / 2;
  for (; m < inner; m *= 2) {
    const size_t m2 = std::min(2 * m, inner), hlen = m2 - m;
    if (csize < hlen) {
      extend_inverse(p, b, m, c.get(), csize, hlen);
      csize = hlen;
    }
    const int logN = std::bit_width(2 * m - 1);
    const size_t sub_len = ulen > m ? ulen - m : 0;
    if (native(p, logN)) {
      Buf t1(&pool_, hlen);
      CycOp op1;  // u[m+i] - (b^2)[m+i]
      op1.x = InOp{b, (uint32_t)m, 0};
      op1.ymode = 3;
      op1.epi.out = t1.get();
      op1.epi.lo = (uint32_t)m;
      op1.epi.hi = (uint32_t)(m + hlen);
      op1.epi.sub_from = u + m;
      op1.epi.sub_len = (uint32_t)std::min(sub_len, hlen);
      cyc_product(p, logN, op1);
      CycOp op2;  // (residual * c) / 2 mod x^hlen
      op2.x = InOp{t1.get(), (uint32_t)hlen, 0};
      op2.ymode = 1;
      op2.y = InOp{c.get(), (uint32_t)csize, 0};
      op2.epi.out = b + m;
      op2.epi.lo = 0;
      op2.epi.hi = (uint32_t)hlen;
      op2.epi.scale = Tw2{half_inv, 0};
      cyc_product(p, logN, op2);
    } else {
      Buf t1(&pool_, hlen), t2(&pool_, hlen);
      mul_window(p, b, m, b, m, m, hlen, t1.get());
      // residual = u[m..] - square
      Buf ut(&pool_, hlen);
      check(cudaMemsetAsync(ut.get(), 0, hlen * 4, stream_), "memset");
      if (sub_len) check(cudaMemcpyAsync(ut.get(), u + m, std::min(sub_len, hlen) * 4, cudaMemcpyDeviceToDevice,
                                         stream_), "copy");
      kcheck(launch_sub(p, ut.get(), t1.get(), hlen, t1.get(), hlen, stream_), "residual");
      product(p, t1.get(), hlen, c.get(), csize, hlen, t2.get());
      kcheck(launch_scale(p, t2.get(), b + m, hlen, half_inv, stream_), "half");
    }
  }
}

// pow (power.hpp:17-87): a^k mod x^n for a 64-bit exponent.
void Engine::pow(uint32_t p, const uint32_t* a, size_t la, uint64_t k, size_t n, uint32_t* out) {
  static const uint32_t one = 1;
  if (n == 0) return;
  check(cudaMemsetAsync(out, 0, n * 4, stream_), "memset");
  if (k == 0) {
    check(cudaMemcpyAsync(out, &one, 4, cudaMemcpyHostToDevice, stream_), "one");
    return;
  }
  if (k == 1) {
    if (la) check(cudaMemcpyAsync(out, a, std::min(la, n) * 4, cudaMemcpyDeviceToDevice, stream_), "copy");
    return;
  }
  const size_t v = find_nonzero(a, la, false);
  if (v == la) return;
  if (v != 0 && k > (n - 1) / v) return;
  const size_t sh = (size_t)(v * k), inner = n - sh;
  size_t ulen = std::min(la - v, inner);
  const uint32_t* u = a + v;
  ulen = find_nonzero(u, ulen, true) + 1;  // trim (basic.hpp:15-17); u[0] != 0
  if (ulen == 1) {
    const uint32_t r = powm(read_word(u), k, p);
    check(cudaMemcpyAsync(out + sh, &r, 4, cudaMemcpyHostToDevice, stream_), "value");
    sync();
    return;
  }
  if (k <= 64 || inner > p) {
    // binary powering (power.hpp:61-74), exact.
    Buf r(&pool_, inner), base(&pool_, inner), tmp(&pool_, inner);
    check(cudaMemcpyAsync(r.get(), &one, 4, cudaMemcpyHostToDevice, stream_), "one");
    check(cudaMemcpyAsync(base.get(), u, ulen * 4, cudaMemcpyDeviceToDevice, stream_), "copy");
    size_t lr = 1, lb = ulen;
    for (uint64_t e = k; e; e >>= 1) {
      if (e & 1) {
        const size_t lt = std::min(lr + lb - 1, inner);
        product(p, r.get(), lr, base.get(), lb, lt, tmp.get());
        std::swap(r, tmp);
        lr = lt;
      }
      if (e > 1) {
        const size_t lt = std::min(2 * lb - 1, inner);
        product(p, base.get(), lb, base.get(), lb, lt, tmp.get());
        std::swap(base, tmp);
        lb = lt;
      }
    }
    check(cudaMemcpyAsync(out + sh, r.get(), std::min(lr, inner) * 4, cudaMemcpyDeviceToDevice, stream_), "copy");
    sync();
    return;
  }
  // c^k * exp((k mod p) * log(u / c)) (power.hpp:76-86); the binomial shortcut
  // for a linear u (:44-59) computes the same series.
  const uint32_t c0 = read_word(u);
  Buf nrm(&pool_, ulen), l(&pool_, inner);
  kcheck(launch_scale(p, u, nrm.get(), ulen, invm(c0, p), stream_), "normalise");
  log_into(p, nrm.get(), ulen, inner, l.get());
  kcheck(launch_scale(p, l.get(), l.get(), inner, (uint32_t)(k % p), stream_), "scale");
  exp_into(p, l.get(), inner, inner, out + sh);
  kcheck(launch_scale(p, out + sh, out + sh, inner, powm(c0, k, p), stream_), "scale");
  sync();
}

// divide<Remainder> (division.hpp:12-80).  The reference's long division for
// short divisors/quotients (:29-55) yields the same q and r as the reversed
// series route used here for every size.
void Engine::divmod(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, uint32_t* q, size_t* lq,
                    uint32_t* r, size_t* lr, bool want_q, bool want_r) {
  *lq = 0;
  *lr = 0;
  size_t an_len = 0;
  if (la) {
    const size_t al = find_nonzero(a, la, true);
    an_len = al < la ? al + 1 : 0;
  }
  size_t bn_len = 0;
  if (lb) {
    const size_t bl = find_nonzero(b, lb, true);
    bn_len = bl < lb ? bl + 1 : 0;
  }
  if (bn_len == 0) throw Error{FPX_EDOMAIN, "poly::divmod: division by zero polynomial"};
  if (an_len < bn_len) {
    if (want_r && an_len) check(cudaMemcpyAsync(r, a, an_len * 4, cudaMemcpyDeviceToDevice, stream_), "copy");
    *lr = want_r ? an_len : 0;
    return;
  }
  if (bn_len == 1) {
    if (want_q) kcheck(launch_scale(p, a, q, an_len, invm(read_word(b), p), stream_), "scale");
    *lq = want_q ? an_len : 0;
    return;
  }
  const size_t dn = an_len - bn_len + 1;
  Buf ra(&pool_, dn), rb(&pool_, dn), ib(&pool_, dn), rq(&pool_, dn);
  const size_t nrb = std::min(bn_len, dn);
  kcheck(launch_reverse(a + (an_len - dn), ra.get(), dn, stream_), "reverse");
  kcheck(launch_reverse(b + (bn_len - nrb), rb.get(), nrb, stream_), "reverse");
  inv_into(p, rb.get(), nrb, dn, ib.get());
  product(p, ra.get(), dn, ib.get(), dn, dn, rq.get());
  uint32_t* qd = q;
  Buf qtmp;
  if (!want_q) {
    qtmp = Buf(&pool_, dn);
    qd = qtmp.get();
  }
  kcheck(launch_reverse(rq.get(), qd, dn, stream_), "reverse");
  *lq = want_q ? dn : 0;
  if (!want_r) return;
  const size_t rn = bn_len - 1;
  Buf prod(&pool_, rn);
  const size_t lp = std::min(bn_len + dn - 1, rn);
  product(p, b, bn_len, qd, dn, lp, prod.get());
  kcheck(launch_sub(p, a, prod.get(), lp, r, rn, stream_), "remainder");
  const size_t last = find_nonzero(r, rn, true);
  *lr = last < rn ? last + 1 : 0;
}

// NttPlan<M>::forward / inverse (ntt.hpp:140-192): in place, canonical output,
// the reference's bit-reversed spectrum order.
void Engine::ntt(uint32_t p, uint32_t* data, uint32_t n, bool inverse) {
  if (n < 2 || (n & (n - 1)) || std::countr_zero(n) > v2_of(p))
    throw Error{FPX_ESIZE, n < 2 || (n & (n - 1)) ? "NTT size must be a power of two"
                                                  : "NTT size exceeds 2^v2(mod-1) for this modulus"};
  const int logN = std::countr_zero(n);
  if (!native(p, logN)) throw Error{FPX_EINVAL, "GPU transforms need an odd prime below 2^30"};
  const PrimeTables& pt = prime_plan(p).t;
  if (logN <= small_kernel_max_log()) {
    SmallJob j;
    j.forward = inverse ? 0 : 1;
    j.x = InOp{data, n, 0};
    j.ymode = 0;
    j.inverse = inverse ? 1 : 0;
    j.spec_x = data;
    j.epi.out = data;
    j.epi.lo = 0;
    j.epi.hi = n;
    j.epi.scale = shoup_pair(invm(n % p, p), p);
    kcheck(launch_small(pt, logN, j, stream_), "small");
    return;
  }
  const BigTables& bt = big_plan(p, logN).t;
  if (!inverse) {
    InOp in{data, n, 0};
    uint32_t* outs[1] = {data};
    kcheck(launch_colfwd(pt, bt, 1, &in, outs, stream_), "colfwd");
    kcheck(launch_rows(pt, bt, data, nullptr, 0, nullptr, 1, 0, stream_), "rows");
  } else {
    kcheck(launch_rows(pt, bt, data, nullptr, 0, nullptr, 0, 1, stream_), "rows");
    Epi e;
    e.out = data;
    e.lo = 0;
    e.hi = n;
    kcheck(launch_colinv(pt, bt, data, 0, e, stream_), "colinv");
  }
}

}  // namespace fpx
