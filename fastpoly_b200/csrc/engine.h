// engine.h - host orchestration of the fastpoly hot path on one GPU.
//
// The Engine owns a device, a stream, a caching device-memory pool and the plan
// cache; every polynomial operation is a sequence of kernel launches on that
// stream composed here, following the reference's algorithms
// (include/fastpoly/detail/poly/*.hpp) with its transforms replaced by the
// fused GPU passes of kernels.cu.
#pragma once
#include <atomic>
#include <chrono>
#include <cstdint>
#include <functional>
#include <deque>
#include <map>
#include <set>
#include <tuple>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "fpx_b200.h"
#include "kernels.h"

namespace fpx {

struct Error {
  int code;
  std::string msg;
};

// Caching device allocator (the reference's ScratchPool, memory.hpp:117-187,
// as a device pool): power-of-two classes, blocks recycled in stream order.
class Pool {
 public:
  explicit Pool(size_t limit) : limit_(limit) {}
  ~Pool();
  uint32_t* get(size_t words, size_t* cls_out);
  void put(uint32_t* p, size_t cls);
  void release();
  // Cached, in-use and lifetime counters read together under the pool's lock.
  struct Snapshot {
    size_t cached_bytes, in_use_bytes, system_allocations, flushes;
    uint64_t alloc_ns, alloc_ns_max;
  };
  Snapshot snapshot();
  // Graph capture: between begin_capture and end_capture every block handed
  // out is owned by the graph being captured; released ones are recycled only
  // within the capture (stream order inside the graph), and end_capture hands
  // all of them to the caller, who keeps them for the graph's lifetime and
  // returns them with give_back.
  void begin_capture();
  std::vector<std::pair<uint32_t*, size_t>> end_capture();
  void give_back(const std::vector<std::pair<uint32_t*, size_t>>& blocks);
  size_t cached_bytes = 0, cached_blocks = 0, in_use_bytes = 0, system_allocations = 0, cache_hits = 0;
  size_t flushes = 0;  // release() calls that returned cached blocks to the device
  uint64_t alloc_ns = 0, alloc_ns_max = 0;  // host time in cudaMalloc: total and longest call
  size_t limit_ = 0;
  // Classes from this size up may be served by a cached block of a larger class.
  static constexpr size_t kFitBytes = size_t(64) << 20;
  // Blocks of this size and more (outside graph capture) come from a
  // stream-ordered memory pool that every engine on the device shares
  // (cudaMallocFromPoolAsync / cudaFreeAsync on the engine's stream, memory
  // kept reserved between uses): freed memory serves any later size, where
  // per-class free lists kept asking for new multi-GB classes, and a
  // cudaMalloc of several GB held every worker of a server for up to 240 ms.
  static constexpr size_t kStreamBytes = size_t(64) << 20;
  // The engine's device and its current stream (async blocks are allocated
  // and freed in its order); unbind() before the stream goes: later frees of
  // such blocks then synchronise.
  void bind(int device, const cudaStream_t* stream) {
    device_ = device;
    stream_ = stream;
  }
  void unbind() { stream_ = nullptr; }
  bool capturing() {
    std::lock_guard<std::mutex> g(mu_);
    return capturing_;
  }

 private:
  std::map<size_t, std::vector<void*>> free_;
  std::mutex mu_;
  int device_ = -1;
  const cudaStream_t* stream_ = nullptr;
  std::set<void*> async_;  // blocks from the stream-ordered pool
  bool capturing_ = false;
  std::map<uint32_t*, size_t> cap_owned_;
  std::map<size_t, std::vector<uint32_t*>> cap_free_;
};

class Engine;
class BatchRec;
struct ExtJob;

// RAII scratch buffer from the pool.
class Buf {
 public:
  Buf() = default;
  Buf(Pool* pool, size_t words) : pool_(pool) { ptr_ = pool->get(words ? words : 1, &cls_); }
  Buf(const Buf&) = delete;
  Buf& operator=(const Buf&) = delete;
  Buf(Buf&& o) noexcept { *this = std::move(o); }
  Buf& operator=(Buf&& o) noexcept {
    reset();
    pool_ = o.pool_; ptr_ = o.ptr_; cls_ = o.cls_;
    o.ptr_ = nullptr;
    return *this;
  }
  ~Buf() { reset(); }
  void reset() {
    if (ptr_) pool_->put(ptr_, cls_);
    ptr_ = nullptr;
  }
  uint32_t* get() const { return ptr_; }
  operator uint32_t*() const { return ptr_; }

 private:
  Pool* pool_ = nullptr;
  uint32_t* ptr_ = nullptr;
  size_t cls_ = 0;
};

struct PrimePlan {
  PrimeTables t;
  Buf fwd, inv;
};
struct BigPlan {
  BigTables t;
  Buf lo_fwd, mid_fwd, hi_fwd, lo_inv, lo_inv_r, mid_inv, hi_inv, cf_fwd, cf_inv;
};

// The cluster CRT Newton kernels for small series modulo primes without
// 2^13-th roots of unity (FPX_CRT_NEWTON=0 turns them off).
bool crt_newton_on();

// Host-side number theory.
uint32_t powm(uint32_t a, uint64_t e, uint32_t p);
uint32_t invm(uint32_t a, uint32_t p);
int v2_of(uint32_t p);  // v2(p - 1)
uint32_t primitive_root(uint32_t p);
bool is_prime(uint32_t p);
bool sqrt_mod(uint32_t x, uint32_t p, uint32_t* out);  // the reference's Tonelli-Shanks root choice
size_t crt_prime_count(uint32_t p, size_t terms);

class Engine {
 public:
  explicit Engine(int device, size_t pool_limit);
  ~Engine();

  int device() const { return device_; }
  cudaStream_t stream() const { return stream_; }
  void set_stream(cudaStream_t s);
  Pool& pool() { return pool_; }

  // Device-pointer operations (canonical residues).  Throw Error.
  size_t conv(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t n, uint32_t* out);
  void inv(uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out);
  void log(uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out);
  void exp(uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out);
  void sqrt(uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out);
  void pow(uint32_t p, const uint32_t* a, size_t la, uint64_t k, size_t n, uint32_t* out);
  void divmod(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, uint32_t* q, size_t* lq,
              uint32_t* r, size_t* lr, bool want_q, bool want_r);
  void ntt(uint32_t p, uint32_t* data, uint32_t n, bool inverse);

  // Many independent operations (device pointers) with shared launches:
  // products of all jobs in one launch set per transform size, the Newton loops
  // of inv / log / exp in lockstep.  Sets each job's status and lengths.
  // first_words (optional): a[0] of every job (0 when la == 0), canonical,
  // from a host copy of the inputs; the domain checks then need no device read
  // (which waits for all work queued before the batch).
  // host (optional): the same jobs with the caller's host pointers (batch_host),
  // read for the host decisions of sqrt / pow / divmod instead of the device;
  // host_mont: those host words are Montgomery limbs.
  void batch(fpx_job* jobs, size_t count, const uint32_t* first_words = nullptr, const fpx_job* host = nullptr,
             bool host_mont = false);
  // The same with host buffers (blocking): inputs packed through pinned
  // staging slots on several host threads, in two chunks pipelined with the
  // kernels when large, outputs brought back the same way; repr as the C ABI's
  // (canonical or Montgomery limbs).
  void batch_host(fpx_job* jobs, size_t count, int repr);
  // In-place representation changes of many arrays in one launch.
  void convert_repr(const std::vector<ReprSeg>& segs);

  void check(cudaError_t e, const char* what);
  void sync();

  // Host <-> device copies of the host-buffer entry points.  Pinned (or small)
  // host buffers go straight to cudaMemcpyAsync on the stream; pageable ones
  // through the engine's pinned slots, packed by several host threads while
  // the previous slot's DMA runs.  to_host returns with the words in place.
  void to_device(uint32_t* d_dst, const uint32_t* h_src, size_t words);
  void to_host(uint32_t* h_dst, const uint32_t* d_src, size_t words);

  // Column-pass tile shapes of N = 2^logN transforms on this device (kind 0:
  // forward pass of one operand, 1: of two or three, 2: inverse pass), chosen
  // by timing the compiled candidates once per process, device and size
  // (tune.cpp).  Every shape computes the same values.
  ColShape col_shape(int logN, int kind);
  int col_shape_candidates(int logN, int kind, ColShape* out, int max);
  void set_col_shape(int logN, int kind, const ColShape& sh);  // throws Error(FPX_EINVAL) if not compiled

  // CUDA graphs of single Newton operations (inv / log / exp on transform
  // primes): the second call with the same (operation, prime, sizes, device
  // pointers) captures the operation's launches into a graph, later calls
  // replay it.  FPX_GRAPHS=0 turns this off.  drop_graphs frees them all.
  void drop_graphs();

  // Terms per block of the block-pair CRT product (the reference's
  // crt_convolution<M, Block> parameter, crt_convolution.hpp:188; default
  // 2^23).  A power of two in [2^13, 2^23]; smaller blocks run the same block
  // loops on small inputs.  Every block size gives the same exact product.
  void set_crt_block(size_t terms);
  size_t crt_block() const { return crt_block_; }

  // Per-kernel timing (CUDA events on the launching stream) and launch count.
  void profile(bool on);
  std::string profile_report();  // {"kernel": [launches, total_ms], ...}
  uint64_t launches() const { return launches_; }

 private:
  friend class BatchRec;
  // ---- plans
  const PrimePlan& prime_plan(uint32_t p);
  const PrimePlan& prime_plan_locked(uint32_t p);  // plan_mu_ held
  const BigPlan& big_plan(uint32_t p, int logN);
  // The shapes big plans of N = bt's size point to; tunes them on first use
  // (plan_mu_ held, tables of bt uploaded).
  const ColShapes* tuned_shapes_locked(uint32_t p, const BigTables& bt);
  const uint32_t* inv_table(uint32_t p, size_t n);  // Montgomery form 1/i, i <= n

  bool native(uint32_t p, int logN) const;  // GPU NTT usable for (p, 2^logN)

  // ---- graphs
  struct GraphKey {
    int op;
    uint32_t p;
    size_t n, la;
    const void* a;
    void* out;
    bool operator<(const GraphKey& o) const {
      return std::tie(op, p, n, la, a, out) < std::tie(o.op, o.p, o.n, o.la, o.a, o.out);
    }
  };
  struct GraphEntry {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<std::pair<uint32_t*, size_t>> blocks;  // scratch owned by the graph
    size_t bytes = 0;
    uint64_t kernels = 0;  // launches the graph stands for
    uint64_t last_use = 0;
  };
  bool graph_native(uint32_t p, size_t n) const;
  // Runs fn, through a captured graph when `key` has been seen before.
  void run_graph(const GraphKey& key, const std::function<void()>& fn);
  void free_graph(GraphEntry& g);
  bool graphs_on_ = true;
  uint64_t graph_clock_ = 0;
  std::map<GraphKey, GraphEntry> graphs_;
  std::set<GraphKey> graph_seen_;
  uint32_t* host_one_ = nullptr;  // pinned constant 1 (capturable host->device copy)
  // Side stream for independent batch work (the one-CTA Newton jobs run there
  // beside the lockstep loop); joined back into stream_ by events.
  cudaStream_t side_ = nullptr;
  cudaEvent_t side_fork_ = nullptr, side_join_ = nullptr;

  // ---- transform compositions
  struct CycOp {
    InOp x;
    int ymode = 0;              // 0 none, 1 raw y, 2 y spectrum, 3 square x
    InOp y;
    const uint32_t* yspec = nullptr;
    uint32_t* yspec_out = nullptr;
    Epi epi;                    // window of the inverse; epi.scale = extra factor (0: none)
  };
  // Cyclic product at size 2^logN on a native prime, inverse window through epi.
  void cyc_product(uint32_t p, int logN, const CycOp& op);
  // Exact product (direct / native / CRT), truncated to outn; optional
  // post-multiplication by a Montgomery table (out[i] *= tab[i]).
  void product(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t outn, uint32_t* out,
               const uint32_t* post_mont = nullptr, bool accumulate = false);
  void crt_product(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t outn,
                   uint32_t* out, bool accumulate);
  bool crt_blocked(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t outn,
                   uint32_t* out, bool accumulate);
  // Exact coefficients [off, off+cnt) of a*b.
  // The same window through the batch recorder (batch.cpp): one launch set,
  // 3-prime CRT with batched Garner for non-native primes; cyc_log > 0 is a
  // cyclic size that leaves the window free of wraparound (<= 2^24 points).
  void window_product(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t off,
                      size_t cnt, uint32_t* out, int cyc_log, const uint32_t* post_mont, bool negate);
  void mul_window(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t off, size_t cnt,
                  uint32_t* out);
  // c[0,k) -> c[0,wanted) for the inverse of a (inverse.hpp:18-65).
  void extend_inverse(uint32_t p, const uint32_t* a, size_t la, uint32_t* c, size_t k, size_t wanted);
  void inv_into(uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out);
  void exp_into(uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out);
  void log_into(uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out);

  // ---- batches (batch.cpp)
  // Descriptor staging: one pinned host arena and its device mirror, carved
  // in ring order.  A region is reused once the event recorded after its
  // host->device copy has completed (device offsets are rewritten only by
  // later copies on the engine's stream, after the kernels that read them).
  // When the next region does not fit, the arena doubles (up to kMaxArena)
  // rather than waiting, so recording a batch never waits for the GPU to
  // catch up; outgrown arenas are kept until the engine goes, since copies
  // from them may be in flight and freeing pinned memory synchronises the device.
  struct Stage {
    void* host;
    void* dev;
    cudaEvent_t ev;  // the caller records it after the region's copy
  };
  struct StageArena {
    char* host = nullptr;
    Buf dev;
    size_t cap = 0;
  };
  struct StageRegion {
    size_t off;
    cudaEvent_t ev;
  };
  static constexpr size_t kMinArena = size_t(1) << 20, kMaxArena = size_t(256) << 20;
  StageArena arena_;
  std::vector<StageArena> old_arenas_;
  std::deque<StageRegion> live_;     // regions of arena_ in allocation order
  std::deque<cudaEvent_t> pending_;  // events of regions of outgrown arenas
  std::vector<cudaEvent_t> stage_free_ev_, stage_all_ev_;
  size_t head_ = 0;
  bool stage_fits(size_t bytes, size_t& off) const;
  void stage_grow(size_t bytes);
  // Two pinned staging slots of batch_host: host copies into one slot overlap
  // the DMA of the other.
  struct Pin {
    uint32_t* host = nullptr;
    cudaEvent_t ev = nullptr;  // recorded after the slot's last copy
  };
  Pin pins_[2];
  uint32_t* pin_slot(int k);  // waits for the slot's last copy
  struct HostSpan {
    const uint32_t* src;  // copy_in: host source
    uint32_t* dst;        // copy_out: host destination (null: skip)
    size_t words;
  };
  // Host spans, concatenated, -> dst (device), through the pinned slots.
  void copy_in(const std::vector<HostSpan>& spans, uint32_t* dst);
  // Device region [src, src + sum(words)) -> host spans (null ones skipped),
  // the copies on stream s (nullptr: the engine's stream); returns with every
  // word in place, except that with wait == false copies straight into
  // page-locked destinations are only queued (returns false then: the caller
  // synchronises s before reading them).
  bool copy_out(const uint32_t* src, const std::vector<HostSpan>& spans, cudaStream_t s = nullptr,
                bool wait = true);
  // Stream of batch_host's copies back, so that a chunk's results come back
  // while the next chunk's kernels run, and the events that order them.
  cudaStream_t copy_stream_ = nullptr;
  std::vector<cudaEvent_t> chunk_ev_;
  // A staging region of at least `bytes` whose previous copy has completed.
  Stage stage(size_t bytes);
  void free_stages();
  void count_batch(const BatchPlan& b);
  // Scratch of one batch flush, kept between flushes (grown when a flush
  // needs more): flushes run one after another on the engine's stream, so
  // each may reuse the last one's memory, with no pool operation in the stream
  // between their launches.
  uint32_t* flush_arena(size_t words);
  Buf flush_arena_;
  size_t flush_arena_words_ = 0;
  // One job of a batch through the single-operation path (errors to its status).
  void batch_single(fpx_job& j);
  // sqrt / pow / divmod jobs of a batch (indices idx) as phases of batched
  // log / exp / inverse / product calls; the rest of them one after another.
  void batch_derived(fpx_job* jobs, const std::vector<size_t>& idx, const fpx_job* host, bool host_mont);
  // host_out[i] = *ptrs[i] (0 for null), one launch, then synchronises.
  void gather_first(const std::vector<const uint32_t*>& ptrs, uint32_t* host_out);
  void ext_phase1(BatchRec& rec, const ExtJob& j);
  void ext_phase2(BatchRec& rec, const ExtJob& j);


  void prof_begin();
  void prof_end(const char* what);
  struct ProfRec {
    std::string name;
    cudaEvent_t b, e;
  };
  bool prof_on_ = false;
  // Wall time of named host phases while profiling (reported beside the
  // kernels as "host:<name>").
  std::map<std::string, std::pair<long, double>> host_prof_;
 public:
  void host_phase(const char* name, double ms) {
    if (!prof_on_) return;
    auto& a = host_prof_[std::string("host:") + name];
    a.first += 1;
    a.second += ms;
  }
  bool profiling() const { return prof_on_; }
  void drop_flush_arena() {
    flush_arena_.reset();
    flush_arena_words_ = 0;
  }
  // small device->host reads (synchronous)
  uint32_t read_word(const uint32_t* d);
  size_t find_nonzero(const uint32_t* a, size_t n, bool last);  // n if none
  // Pinned host allocations of the staging buffers (count, host time: total
  // and longest); written by the thread that drives the engine.
  std::atomic<uint64_t> host_allocs{0}, host_alloc_ns{0}, host_alloc_ns_max{0};
  void count_host_alloc(std::chrono::steady_clock::time_point t0) {
    const uint64_t ns = static_cast<uint64_t>(
        std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count());
    host_allocs.fetch_add(1, std::memory_order_relaxed);
    host_alloc_ns.fetch_add(ns, std::memory_order_relaxed);
    if (ns > host_alloc_ns_max.load(std::memory_order_relaxed)) host_alloc_ns_max.store(ns, std::memory_order_relaxed);
  }
 private:
  cudaEvent_t prof_open_ = nullptr;
  std::vector<ProfRec> prof_recs_;
  std::vector<cudaEvent_t> ev_free_;
  uint64_t launches_ = 0;

  int device_;
  cudaStream_t stream_ = nullptr, own_stream_ = nullptr;
  Pool pool_;
  std::mutex plan_mu_;
  std::map<uint32_t, std::unique_ptr<PrimePlan>> primes_;
  std::map<std::pair<uint32_t, int>, std::unique_ptr<BigPlan>> bigs_;
  std::map<uint32_t, std::pair<size_t, Buf>> inv_tabs_;
  size_t crt_block_;
  unsigned long long* scratch_ull_ = nullptr;  // device word for scans
  unsigned long long* host_ull_ = nullptr;     // pinned
};

}  // namespace fpx
