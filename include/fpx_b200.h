/*
 * fpx_b200.h - C ABI of the B200-native fastpoly hot path.
 *
 * Plain C types only.  Every function returns an fpx status (0 = success).
 * Values are 32-bit residues modulo a prime 2 <= p < 2^31, either canonical
 * (FPX_REPR_CANONICAL: x in [0, p)) or the reference's Montgomery limbs
 * (FPX_REPR_MONTGOMERY: x * 2^32 mod p, include/fastpoly/modint.hpp:57-98;
 * for p = 2 the limb is the bit itself), so a fpx::Poly<fpx::Mont<p>> can hand
 * over its storage unchanged.
 *
 * Two flavours of each operation:
 *   - host buffers (blocking): inputs are copied to the GPU, the result copied
 *     back; the call returns when the output is in place;
 *   - "_device" (asynchronous): all pointers are device pointers, canonical
 *     residues, work is queued on the context's stream (fpx_ctx_set_stream).
 *
 * Error conditions follow the reference exactly: FPX_EDOMAIN where it throws
 * fpx::poly::domain_error, FPX_ESIZE for fpx::ntt_size_error, FPX_ELENGTH for
 * std::length_error.  Nothing is written to outputs on error.
 */
#ifndef FPX_B200_H
#define FPX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum fpx_status {
  FPX_OK = 0,
  FPX_EDOMAIN = 1,      /* fpx::poly::domain_error (base.hpp:26-30) */
  FPX_ESIZE = 2,        /* fpx::ntt_size_error (ntt.hpp:59-70) */
  FPX_ELENGTH = 3,      /* std::length_error (convolution.hpp:20-21) */
  FPX_ENOMEM = 4,       /* device memory pool exhausted */
  FPX_ETIMEDOUT = 5,    /* a bounded device wait gave up */
  FPX_ECUDA = 6,        /* CUDA runtime error (see fpx_last_error_message) */
  FPX_EINVAL = 7,       /* bad argument (null pointer, modulus not prime < 2^31, ...) */
  FPX_EUNSUPPORTED = 8, /* no usable CUDA device */
  FPX_EPENDING = 9      /* fpx_serve_poll: the request has not completed yet */
};

enum fpx_repr { FPX_REPR_CANONICAL = 0, FPX_REPR_MONTGOMERY = 1 };

typedef struct fpx_ctx fpx_ctx;

typedef struct fpx_pool_stats_t {
  size_t cached_bytes;       /* idle bytes held for reuse */
  size_t cached_blocks;
  size_t in_use_bytes;       /* bytes handed out and not yet returned */
  size_t system_allocations; /* cudaMalloc calls made so far */
  size_t cache_hits;         /* requests served from the idle cache */
  size_t limit_bytes;        /* 0 = unlimited */
} fpx_pool_stats_t;

/* ---- context (replaces the reference's per-thread scratch pool and plan cache:
 *      memory.hpp:117-187, ntt.hpp:250-276) ------------------------------------ */
int fpx_ctx_create(int device, size_t pool_limit_bytes, fpx_ctx** out);
int fpx_ctx_destroy(fpx_ctx* ctx);
/* cudaStream_t passed as void*; NULL selects the context's own stream. */
int fpx_ctx_set_stream(fpx_ctx* ctx, void* stream);
void* fpx_ctx_stream(fpx_ctx* ctx);
int fpx_ctx_synchronize(fpx_ctx* ctx);
const char* fpx_last_error_message(fpx_ctx* ctx);
/* scratch_memory_stats() / release_scratch_memory() (memory.hpp:21-26, 252-258) */
int fpx_pool_stats(fpx_ctx* ctx, fpx_pool_stats_t* out);
int fpx_release_pool(fpx_ctx* ctx);
/* Page-locked host memory (no counterpart in the reference): copies between
 * it and the device need no staging, and fpx_batch_run writes a batch's
 * results straight into it where they lie in it in long contiguous runs.
 * fpx_host_free takes only pointers fpx_host_alloc returned. */
int fpx_host_alloc(size_t bytes, void** out);
int fpx_host_free(void* p);
/* Terms per block of products that go through the block-pair three-prime CRT
 * path (the reference's crt_convolution<M, Block> template parameter,
 * crt_convolution.hpp:188, default 2^23 = 0 here): a power of two in
 * [2^13, 2^23], else FPX_EINVAL.  Every block size gives the same exact
 * product; small blocks run the multi-block loops on small inputs (tests). */
int fpx_ctx_set_crt_block(fpx_ctx* ctx, size_t block_terms);

/* ---- instrumentation (the reference's bench harness timing, bench/bench.cpp:161-203,
 *      moved onto the device) ---------------------------------------------------
 * fpx_profile(ctx, 1) starts recording a CUDA event pair on the launching stream
 * around every kernel launch (and clears earlier records); fpx_profile_report
 * writes {"kernel": [launches, total_ms], ...} as a NUL-terminated JSON object.
 * fpx_launch_count counts every kernel launched by the context. */
int fpx_profile(fpx_ctx* ctx, int enable);
int fpx_profile_report(fpx_ctx* ctx, char* buf, size_t cap, size_t* needed);
uint64_t fpx_launch_count(fpx_ctx* ctx);
/* The GPU's measured 32-bit integer multiply rate (thread-level mul.hi.u32 and
 * mad.lo.u32 instructions per second, all SMs busy, CUDA-event timed): the
 * compute denominator of the transform roofline.  No context needed. */
int fpx_measure_imad_rate(int device, double* per_second);
/* The GPU's measured rate of the transforms' lazy DIF butterfly (one add with
 * conditional subtract, one Shoup product: mul.hi plus two mul.lo), all SMs
 * busy, butterflies per second: the compute ceiling of a transform pass. */
int fpx_measure_butterfly_rate(int device, double* per_second);

/* ---- column-pass tile shapes (no counterpart in the reference, whose NTT plan
 *      has one fixed schedule per size) ------------------------------------------
 * A transform of N = 2^log_n > 2^13 points runs two column passes over tiles of
 * 2^lw1 columns; with split != 0 the columns past the last full wave of wide
 * tiles go in narrow tiles of 2^lw2 columns.  The shape is chosen per process,
 * device and size by timing every compiled candidate on first use (environment:
 * FPX_AUTOTUNE=0 keeps the defaults, FPX_AUTOTUNE_CACHE=<file> persists the
 * choices).  kind: 0 forward pass of one operand, 1 of two or three, 2 inverse.
 * Every shape computes the same values; _set (for tests and experiments) takes
 * effect for every context of the process on that device. */
typedef struct fpx_col_shape {
  int lw1, lw2, split;
} fpx_col_shape;
int fpx_col_shape_candidates(fpx_ctx* ctx, int log_n, int kind, fpx_col_shape* out, int max, int* count);
int fpx_col_shape_get(fpx_ctx* ctx, int log_n, int kind, fpx_col_shape* out);
int fpx_col_shape_set(fpx_ctx* ctx, int log_n, int kind, const fpx_col_shape* shape);

/* ---- transforms (NttPlan<M>::forward / inverse, ntt.hpp:140-192) -------------
 * In place, n a power of two with 2 <= n <= 2^v2(p-1), p < 2^30 odd.  forward
 * leaves the spectrum in the reference's bit-reversed order; inverse takes that
 * order back and scales by 1/n.  Outputs canonical. */
int fpx_ntt_max_log(uint32_t p);
int fpx_ntt_forward(fpx_ctx* ctx, uint32_t p, uint32_t* data, uint32_t n, int repr);
int fpx_ntt_inverse(fpx_ctx* ctx, uint32_t p, uint32_t* data, uint32_t n, int repr);
int fpx_ntt_forward_device(fpx_ctx* ctx, uint32_t p, uint32_t* d_data, uint32_t n);
int fpx_ntt_inverse_device(fpx_ctx* ctx, uint32_t p, uint32_t* d_data, uint32_t n);

/* ---- polynomial operations (fpx::poly, include/fastpoly/detail/poly) ----------- */
/* conv(a, b, n): the product truncated to min(la+lb-1, n) terms, *out_len set;
 * n = SIZE_MAX for the full product (convolution.hpp:17-147).  out needs
 * min(la+lb-1, n) words. */
int fpx_conv(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t n,
             uint32_t* out, size_t* out_len, int repr);
int fpx_conv_device(fpx_ctx* ctx, uint32_t p, const uint32_t* d_a, size_t la, const uint32_t* d_b, size_t lb,
                    size_t n, uint32_t* d_out, size_t* out_len);

/* Series operations mod x^n; out needs n words (inverse.hpp:163, exponential.hpp:85,
 * :107, square_root.hpp:12, power.hpp:17). */
int fpx_inv(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out, int repr);
int fpx_log(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out, int repr);
int fpx_exp(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out, int repr);
int fpx_sqrt(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out, int repr);
int fpx_pow(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, uint64_t k, size_t n, uint32_t* out, int repr);
int fpx_inv_device(fpx_ctx* ctx, uint32_t p, const uint32_t* d_a, size_t la, size_t n, uint32_t* d_out);
int fpx_log_device(fpx_ctx* ctx, uint32_t p, const uint32_t* d_a, size_t la, size_t n, uint32_t* d_out);
int fpx_exp_device(fpx_ctx* ctx, uint32_t p, const uint32_t* d_a, size_t la, size_t n, uint32_t* d_out);
int fpx_sqrt_device(fpx_ctx* ctx, uint32_t p, const uint32_t* d_a, size_t la, size_t n, uint32_t* d_out);
int fpx_pow_device(fpx_ctx* ctx, uint32_t p, const uint32_t* d_a, size_t la, uint64_t k, size_t n,
                   uint32_t* d_out);

/* divmod(a, b) (division.hpp:86-104): q needs la words, r needs lb words; the
 * returned lengths are trimmed like the reference's results. */
int fpx_divmod(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, uint32_t* q,
               size_t* q_len, uint32_t* r, size_t* r_len, int repr);
int fpx_div(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, uint32_t* q,
            size_t* q_len, int repr);
int fpx_mod(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, uint32_t* r,
            size_t* r_len, int repr);

/* ---- batches (no counterpart in the reference, whose callers loop over the
 *      single-operation functions above on one or more host threads) -----------
 * One fpx_job per operation; the jobs are independent and may mix moduli and
 * sizes.  Results, lengths and error conditions are those of the single-job
 * functions, job by job.  The batch shares launches between jobs: all products
 * of a stage run as one launch set per transform size (mixed primes and CRT
 * lifts included), and the Newton loops of inv, log and exp advance in
 * lockstep.  sqrt, pow and divmod jobs of up to 2^17 terms (sqrt: 2^16) run as
 * phases of such batched calls (pow: log, then exp; sqrt: exp of half the log
 * times the root of the constant term; divmod: inverse of the reversed
 * divisor, then two products), with the remainders' lengths read back once
 * per batch.  Longer ones, pow with exponents up to 64 (binary powering),
 * characteristic 2, and transforms past 2^24 points run one after another
 * inside the same call (FPX_BATCH_PHASED=0: every sqrt / pow / divmod job). */
enum fpx_op {
  FPX_OP_CONV = 0,   /* out = conv(a, b, n)                     (convolution.hpp:145) */
  FPX_OP_INV = 1,    /* out = inv(a, n)                         (inverse.hpp:163) */
  FPX_OP_LOG = 2,    /* out = log(a, n)                         (exponential.hpp:85) */
  FPX_OP_EXP = 3,    /* out = exp(a, n)                         (exponential.hpp:107) */
  FPX_OP_SQRT = 4,   /* out = sqrt(a, n)                        (square_root.hpp:12) */
  FPX_OP_POW = 5,    /* out = pow(a, k, n)                      (power.hpp:17) */
  FPX_OP_DIVMOD = 6  /* out = quotient, out2 = remainder        (division.hpp:86) */
};

typedef struct fpx_job {
  int op;              /* enum fpx_op */
  uint32_t p;          /* modulus: a prime 2 <= p < 2^31 */
  const uint32_t* a;   /* first operand, la words */
  size_t la;
  const uint32_t* b;   /* conv: second factor; divmod: divisor (lb words) */
  size_t lb;
  uint64_t k;          /* pow: exponent */
  size_t n;            /* conv: truncation (SIZE_MAX = full product); inv/log/exp/sqrt/pow: length */
  uint32_t* out;       /* conv: min(la+lb-1, n) words; series: n words; divmod: quotient, la words */
  uint32_t* out2;      /* divmod: remainder, lb words (NULL: not wanted) */
  size_t out_len;      /* set: result length (conv, divmod quotient; n for series) */
  size_t out2_len;     /* set: divmod remainder length */
  int status;          /* set: this job's fpx status; nothing is written for a failed job */
} fpx_job;

/* Device pointers, canonical residues, queued on the context's stream.  Returns
 * when every job's status and lengths are set (the domain checks of inv, log and
 * exp read one word per job: one small device->host copy for the whole batch);
 * the results are complete when the stream reaches the point of the call
 * (fpx_batch_wait or fpx_ctx_synchronize).  Returns FPX_OK when every job
 * succeeded, else the first failing job's status (or a CUDA / memory error for
 * the whole batch). */
int fpx_batch_submit(fpx_ctx* ctx, fpx_job* jobs, size_t count);
int fpx_batch_wait(fpx_ctx* ctx);
/* Host buffers (blocking): inputs are packed through pinned staging slots by
 * several host threads while the DMA runs; a batch moving at least 64 MiB runs
 * as two chunks, the second packed while the first computes and the first
 * unpacked while the second computes.  Returns when every result is in the
 * caller's buffers.  repr as for the single-job functions. */
int fpx_batch_run(fpx_ctx* ctx, fpx_job* jobs, size_t count, int repr);

/* ---- serving (no counterpart in the reference) --------------------------------
 * A request loop on one GPU.  Requests are fpx_job records with HOST buffers;
 * the job record and its buffers must stay valid until fpx_serve_poll reports
 * completion.  Requests go to one of two size lanes: at most 2^17 terms (the
 * longest operand, or the series length) to the small lane, the rest to the
 * large lane; each lane has its own queue and worker threads (each with its own
 * stream and device pool), so a short request is never batched with, and held
 * behind, a long one.  A free worker forms a micro-batch from its lane's queue
 * in arrival order (continuous batching: what arrives while others run joins
 * the next micro-batch; the large lane's workers also take small requests when
 * their own queue is empty).  Admission is device-wide: a micro-batch is formed
 * only while the planned device bytes of everything on the GPU (operands,
 * results and transform scratch, fpx_serve_plan_bytes) stay within the budget,
 * charged when it is formed and refunded when it completes; a request larger
 * than the whole budget runs alone, and when the large lane's oldest request
 * does not fit, no lane admits new work until it does.  Every request's result
 * is the one the single-job function gives it, whatever it was batched with. */
typedef struct fpx_serve_config {
  size_t hbm_budget_bytes; /* planned device bytes of all requests on the GPU at once;
                              0 = a quarter of the device memory free at start, at most 32 GiB */
  size_t max_batch_jobs;   /* 0 = 4096 */
  int workers;             /* worker threads (at least 2): half for the large lane, the rest for the small
                              lane; 0 = 6 */
  int repr;                /* FPX_REPR_CANONICAL or FPX_REPR_MONTGOMERY for every request */
} fpx_serve_config;

typedef struct fpx_serve_stats {
  uint64_t submitted, completed, batches;
  uint64_t max_batch_jobs_seen;     /* largest micro-batch formed */
  uint64_t max_batch_bytes_seen;    /* largest planned device bytes admitted in one micro-batch (at most the
                                       budget over the lane's workers, unless one request alone is larger) */
  uint64_t oversize_requests;       /* requests that alone exceeded the budget (ran alone) */
  uint64_t max_in_flight_bytes;     /* largest planned device bytes of all micro-batches on the GPU at once */
  uint64_t device_pool_bytes;       /* device bytes the workers' scratch pools hold now (cached + in use) */
  uint64_t device_allocations;      /* cudaMalloc calls made by the workers' pools so far */
  uint64_t pool_flushes;            /* times a worker's pool returned its cache to the device (a failed cudaMalloc) */
  uint64_t device_alloc_ns;         /* host time the workers spent in those cudaMalloc calls */
  uint64_t device_alloc_ns_max;     /* the longest of them */
  uint64_t host_allocs;             /* pinned host allocations of the workers' staging buffers */
  uint64_t host_alloc_ns;           /* host time spent in them (frees of the buffers they replace included) */
  uint64_t host_alloc_ns_max;       /* the longest of them */
} fpx_serve_stats;

typedef struct fpx_server fpx_server;

int fpx_serve_start(int device, const fpx_serve_config* cfg, fpx_server** out);
/* Queues one request; *ticket identifies it for fpx_serve_poll. */
int fpx_serve_submit(fpx_server* srv, fpx_job* job, uint64_t* ticket);
/* wait = 0: returns FPX_EPENDING until the request is complete; wait != 0:
 * blocks until it is.  When complete, returns the job's status (also in
 * job->status) and, if latency_ns is not NULL, the time from submission to
 * completion (results in the host buffers).  A ticket is released once its
 * completion has been reported. */
int fpx_serve_poll(fpx_server* srv, uint64_t ticket, int wait, uint64_t* latency_ns);
int fpx_serve_stats_get(fpx_server* srv, fpx_serve_stats* out);
/* Finishes every queued request, then stops the workers and frees the server. */
int fpx_serve_stop(fpx_server* srv);
/* Planned device bytes of one request (the admission measure), 0 for an invalid job. */
size_t fpx_serve_plan_bytes(const fpx_job* job);

/* ---- allocation-free convolution (no counterpart in the reference) ------------
 * For callers that cannot allocate device memory when they need a product: code
 * whose device memory is owned by a host framework's allocator (often reserved
 * in full at start-up), or latency-critical loops that cannot take cudaMalloc's
 * implicit device synchronisation.  Same result and same output length as
 * fpx_conv_device, but no context is needed and nothing is allocated: the
 * transform buffers and twiddle tables live in one static device array sized
 * for transforms of up to 2^20 points (about 8.3 MiB, held by every GPU that
 * loads the library until the process exits).  Device pointers, canonical
 * residues, work queued on `stream` (a cudaStream_t, NULL = legacy default).
 * Limits: p an odd NTT prime below 2^30 (FPX_EINVAL otherwise); the padded
 * product length next_pow2(min(la,n) + min(lb,n) - 1) at most 2^20 and
 * 2^v2(p-1), unless the shorter operand has <= 40 terms (FPX_ESIZE otherwise).
 * The first call on a device looks the array up (cudaGetSymbolAddress) and
 * should come before any stream capture.  The device is the current one: the
 * stream must belong to it, and the looked-up address is kept for the life of
 * the process, so no cudaDeviceReset may come between calls.  A CUDA error
 * already pending when the call starts is left pending and the call returns
 * FPX_ECUDA without launching anything.  All calls share the array and keep
 * its last contents; calls that overlap on the GPU race and must be serialised
 * by the caller. */
int fpx_conv_noalloc(uint32_t p, const uint32_t* d_a, size_t la, const uint32_t* d_b, size_t lb, size_t n,
                     uint32_t* d_out, size_t* out_len, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FPX_B200_H */
