// kernels.h - host-side launchers for the sm_100a transform kernels.
// Only plain types cross this header; the engine (engine.cpp) composes them.
#pragma once
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

namespace fpx {

struct Tw2 { uint32_t w, q; };  // twiddle value + Shoup quotient (device: uint2)

// Per-prime, size-independent tables: tw[h + k] = w_{2h}^{+-k} for 2h <= 2^13.
struct PrimeTables {
  uint32_t p = 0;
  int max_log = 0;            // v2(p-1)
  int small_log = 0;          // tables cover block lengths up to 2^small_log
  const Tw2* fwd = nullptr;   // device
  const Tw2* inv = nullptr;   // device
  uint32_t q1 = 0;            // floor(2^32 / p)
  // host-side constants: inverse scale of a one-CTA product of 2^k points,
  // 1/2^k and (after a Montgomery pointwise product) 2^32/2^k mod p, k <= 13
  uint32_t inv_pow2[14] = {};
  uint32_t inv_pow2_r[14] = {};
};

// Tile shape of one column pass: wide tiles of 2^lw1 columns; with split != 0
// the columns past the last full wave of wide tiles (`slots` resident CTAs on
// the device) go in narrow tiles of 2^lw2 columns.  lw1 == 0: the default
// width, no split.  Every shape computes the same values.
struct ColShape {
  int lw1 = 0, lw2 = 0, split = 0, slots = 0;
};
struct ColShapes {
  ColShape fwd1, fwd2, inv;  // forward pass of one operand, of two or three; inverse pass
};

// Per-(prime, N) tables for the two-pass (four-step) decomposition.
// The Bailey twiddle w_N^e (e < N) is lo[e & 255] * mid[(e >> 8) & 255] *
// hi[e >> 16]: three small tables instead of one of N entries.
struct BigTables {
  int logN = 0, logR = 0, logC = 0;
  const ColShapes* shapes = nullptr;  // chosen column-pass tile shapes; nullptr: defaults
  const Tw2* lo_fwd = nullptr;     // w_N^y, y < 256
  const Tw2* mid_fwd = nullptr;    // w_N^(256 y), y < 256
  const Tw2* hi_fwd = nullptr;     // w_N^(65536 y), y < max(1, N / 65536)
  const Tw2* lo_inv = nullptr;     // w_N^-y / N
  const Tw2* lo_inv_r = nullptr;   // w_N^-y * 2^32 / N  (after a Montgomery pointwise)
  const Tw2* mid_inv = nullptr;    // w_N^-(256 y)
  const Tw2* hi_inv = nullptr;     // w_N^-(65536 y)
  // Column factors of the Bailey twiddle at the column passes' last (forward)
  // or first (inverse) butterfly group of 2^G rows, G = col_last_group_log(logR):
  // the twiddle of column j, row 2^G b + i is w_N^(j bitrev(b)) * U_j^bitrev_G(i)
  // with U_j = w_N^(j 2^(logR - G)).  Entry 2((j/2) 2^G + i) + (j & 1) holds
  // U_j^bitrev_G(i) (cf_inv: U_j^-bitrev_G(i), no 1/N) with its Shoup quotient,
  // so a column pair reads both of its factors in one 16-byte load.
  // nullptr: three small-table products per point instead.
  const Tw2* cf_fwd = nullptr;
  const Tw2* cf_inv = nullptr;
};

// log2 of the row count of the column passes' last forward group, which the
// column factors (BigTables::cf_fwd / cf_inv) are built for.
inline int col_last_group_log(int logR) { return logR / ((logR + 3) / 4); }

// A forward-transform input: values at ptr[0, count), zero beyond.
struct InOp {
  const uint32_t* ptr = nullptr;
  uint32_t count = 0;
  int reduce = 0;  // inputs may be >= 2p (any 32-bit value): reduce mod p on load
};

// Output epilogue of an inverse transform: natural-order outputs [lo, hi) go to
// out[i - lo] as: y = canonical(x); y = y * scale; y = y * mul[i-lo] (Montgomery
// table); y = -y; y = sub_from[i-lo] - y; y = out[i-lo] + y (accumulate).
struct Epi {
  uint32_t* out = nullptr;
  uint32_t lo = 0, hi = 0;
  Tw2 scale{0, 0};
  const uint32_t* mul_mont = nullptr;
  int negate = 0;
  const uint32_t* sub_from = nullptr;
  uint32_t sub_len = 0;
  int accumulate = 0;
};

// -------- single-CTA transforms, N = 2^logN <= 2^13 ----------------------------
// x: forward input.  y: second operand (mode 0 none, 1 raw input, 2 spectrum,
// 3 square x).  If spec_out != null the forward spectrum of y (mode 1) is stored
// there.  If inverse, the product (or x's spectrum) is inverse-transformed with
// scale epi.scale and written through the epilogue; otherwise x's spectrum
// (times y when mode != 0, Montgomery) is written to spec_x (lazy, [0, 2p)).
struct SmallJob {
  int forward = 1;   // 0: x already holds a spectrum (N words), inverse only
  InOp x;
  InOp y;
  int ymode = 0;
  const uint32_t* yspec = nullptr;
  uint32_t* yspec_out = nullptr;
  uint32_t* spec_x = nullptr;
  int inverse = 1;
  Epi epi;
};
cudaError_t launch_small(const PrimeTables& pt, int logN, const SmallJob& job, cudaStream_t s);

// -------- two-pass transforms, N = R*C > 2^13 ----------------------------------
// Compiled column-pass shapes for R = 2^logR, the default first; `inverse`
// selects the kernel whose occupancy gives `slots`.  Returns how many were
// written to out (at most max).
int col_shape_candidates(int logR, bool inverse, ColShape* out, int max);

// Pass A forward: column DIF over up to 3 operands, each to its own N-word buffer.
cudaError_t launch_colfwd(const PrimeTables& pt, const BigTables& bt, int nops, const InOp* in,
                          uint32_t* const* out, cudaStream_t s);
// Pass B: per row: DIF x (and y if ymode==1), pointwise (ymode 1/2/3), DIT if inverse.
// ymode: 0 none, 1 raw (after pass A), 2 spectrum, 3 square.  y_spec_out: store y's row spectrum.
cudaError_t launch_rows(const PrimeTables& pt, const BigTables& bt, uint32_t* x, const uint32_t* y, int ymode,
                        uint32_t* y_spec_out, int forward, int inverse, cudaStream_t s);
// Pass A inverse: Bailey twiddle (scaled), column DIT, epilogue on the window.
cudaError_t launch_colinv(const PrimeTables& pt, const BigTables& bt, const uint32_t* in, int mont_scaled,
                          const Epi& epi, cudaStream_t s);

// -------- elementwise ------------------------------------------------------------
// out[i] = mont(a[i], b[i]) for lazy spectra (result in (0, 2p)).
cudaError_t launch_pointwise(uint32_t p, uint32_t* a, const uint32_t* b, size_t n, cudaStream_t s);
// dst[i] = dst[i] + src[i] mod p, canonical inputs, i < n.
cudaError_t launch_add_into(uint32_t p, uint32_t* dst, const uint32_t* src, size_t n, cudaStream_t s);
// acc[i] (+)= sum_t x[t][i] * y[t][i] * 2^-32 mod p (canonical) over npairs
// spectra of n words (n a multiple of 4, inputs lazy below 4p).
cudaError_t launch_spec_mac(uint32_t p, const uint32_t* const* x, const uint32_t* const* y, int npairs, uint32_t* acc,
                            size_t n, int accumulate, cudaStream_t s);
// Garner reconstruction of `primes` auxiliary residues into the target field:
// out[i] (+)= CRT(c1[i], c2[i], c3[i]) mod target.  Inputs canonical.
cudaError_t launch_garner(uint32_t target, int primes, const uint32_t* c1, const uint32_t* c2,
                          const uint32_t* c3, uint32_t* out, size_t n, int accumulate, cudaStream_t s);
// Montgomery limbs <-> canonical residues (repr conversion), in place allowed.
cudaError_t launch_from_mont(uint32_t p, const uint32_t* in, uint32_t* out, size_t n, cudaStream_t s);
cudaError_t launch_to_mont(uint32_t p, const uint32_t* in, uint32_t* out, size_t n, cudaStream_t s);
// out[i] = a[i] * c (canonical, Shoup constant).
cudaError_t launch_scale(uint32_t p, const uint32_t* a, uint32_t* out, size_t n, uint32_t c, cudaStream_t s);
// 1/i for i in [1, n] into tab (Montgomery form: (1/i) * 2^32 mod p), tab[0] = 0.
cudaError_t launch_inv_table(uint32_t p, uint32_t* tab, size_t n, cudaStream_t s);
// r[i] = a[i+1] * (i+1) for i < cnt-1 (derivative of the first cnt coefficients).
cudaError_t launch_derivative(uint32_t p, const uint32_t* a, uint32_t* r, size_t cnt, cudaStream_t s);
// Direct (schoolbook) product window for short operands:
// out[i] = sum_j a[j] b[i+off-j], i < cnt (canonical).  Used for min(la,lb) <= 40.
cudaError_t launch_direct_product(uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb,
                                  size_t off, size_t cnt, uint32_t* out, int accumulate, cudaStream_t s);

int small_kernel_max_log();
cudaError_t kernels_init();

// One cyclic product of exactly 4096 points (as launch_small with forward =
// inverse = 1; epi.scale holds the full inverse scale) in the row pass's layout.
cudaError_t launch_cyc4096(const PrimeTables& pt, const SmallJob& job, cudaStream_t s);
// One cyclic product of 2^logN <= 2^13 points in one CTA (same contract).
cudaError_t launch_cyc_small(const PrimeTables& pt, int logN, const SmallJob& job, cudaStream_t s);
cudaError_t kernels_cyc_init();

}  // namespace fpx

namespace fpx {
// Seeds of the Newton loops (kind 0 inverse, 1 exp (a = a'), 2 sqrt (a = u, r0 = root)); n <= 64.
cudaError_t launch_seed(int kind, uint32_t p, const uint32_t* a, size_t la, uint32_t* out, int n, uint32_t r0,
                        cudaStream_t s);
// Series inverse c[k0, K) of a from c[0, k0) (k0 a power of two, or 0: from
// c[0] = 1 / a[0], a[0] != 0), all doubling steps in one CTA: needs
// K <= 2^small_log of pt and K <= 2^newton_inv_max_log().
int newton_inv_max_log();
// exp(a) b[0, K) from a' (ap, lap terms) and the Montgomery table 1/i (i < K),
// every doubling step in one CTA; also leaves 1/b in c[0, cs) with cs from
// m = 1, cs = 1: while m < K { h = min(2m, K) - m; while cs < h: cs = min(2cs, h); m += h }.
// Needs K <= 2^small_log of pt and K <= 2^newton_inv_max_log().
// sqrt(u) b[0, K) with b[0] = root (1/root = root_inv), every doubling step in
// one CTA; leaves 1/b in c[0, cs) with cs as for launch_newton_exp.
cudaError_t launch_newton_sqrt(const PrimeTables& pt, const uint32_t* u, size_t ulen, uint32_t root, uint32_t root_inv,
                               uint32_t* b, uint32_t* c, size_t K, cudaStream_t s);
// Many Newton inverses (kind 0: out = 1/a to K terms, a with la terms) and
// exponentials (kind 1: out = exp with a = a' of la terms, tab = 1/i Montgomery,
// c scratch of K/2 words) up to K <= 2^13 terms, one CTA per job, one launch.
struct NewtonJob {
  int kind;
  const PrimeTables* pt;
  const uint32_t* a;
  size_t la;
  const uint32_t* tab;
  uint32_t* out;
  uint32_t* c;
  size_t K;
  // a prime P without 2^13-th roots of unity: the three CRT primes' plans
  // (167772161, 469762049, 754974721 in that order; pt unused), one cluster
  // of three CTAs per job
  const PrimeTables* aux = nullptr;
  uint32_t P = 0;
};
size_t batch_newton_bytes(size_t jobs);
cudaError_t launch_newton_batch(const std::vector<NewtonJob>& jobs, void* host_staging, void* dev_desc,
                                cudaStream_t s, cudaEvent_t staged = nullptr);
cudaError_t launch_newton_exp(const PrimeTables& pt, const uint32_t* ap, size_t lap, const uint32_t* tab, uint32_t* b,
                              uint32_t* c, size_t K, cudaStream_t s);
cudaError_t launch_newton_inv(const PrimeTables& pt, const uint32_t* a, size_t la, uint32_t* c, size_t k0, size_t K,
                              cudaStream_t s);
// c[0, K) = 1 / a mod x^K mod the prime P (a canonical, a[0] != 0), every
// product a three-prime CRT product, in one CTA: aux = the plans of 167772161,
// 469762049 and 754974721 in that order; K <= 2^newton_inv_max_log().
cudaError_t launch_newton_inv_crt(const PrimeTables* aux, uint32_t P, const uint32_t* a, size_t la, uint32_t* c,
                                  size_t K, cudaStream_t s);
// The exponential and square-root counterparts of launch_newton_exp / _sqrt for
// such a modulus (P odd): b[0, K) and c = 1/b on the same schedule.
cudaError_t launch_newton_exp_crt(const PrimeTables* aux, uint32_t P, const uint32_t* ap, size_t lap,
                                  const uint32_t* tab, uint32_t* b, uint32_t* c, size_t K, cudaStream_t s);
cudaError_t launch_newton_sqrt_crt(const PrimeTables* aux, uint32_t P, const uint32_t* u, size_t ulen, uint32_t root,
                                   uint32_t root_inv, uint32_t* b, uint32_t* c, size_t K, cudaStream_t s);
// *res = min (mode 0) / max (mode 1) index with a[i] != 0; caller initialises *res.
cudaError_t launch_find_nonzero(const uint32_t* a, size_t n, int mode, unsigned long long* res, cudaStream_t s);
cudaError_t launch_reverse(const uint32_t* a, uint32_t* r, size_t n, cudaStream_t s);
cudaError_t launch_sub(uint32_t p, const uint32_t* a, const uint32_t* b, size_t lb, uint32_t* r, size_t n,
                       cudaStream_t s);
cudaError_t launch_sqrt_char2(const uint32_t* a, size_t cnt, uint32_t* out, unsigned long long* odd_flag,
                              cudaStream_t s);
cudaError_t launch_mul_mont_tab(uint32_t p, const uint32_t* a, const uint32_t* tab, uint32_t* out, size_t n,
                                cudaStream_t s);
}  // namespace fpx

#include <vector>
namespace fpx {
// ---- batched execution --------------------------------------------------------
// One cyclic product of size 2^logN on a native prime (logN <= 13: one CTA per
// job; 14 <= logN <= 23: the two-pass kernels with t1/t2 as N-word scratch).
// ymode as in SmallJob; the inverse always runs; epi.scale must already hold
// the full inverse scale for one-CTA jobs (1/N, times 2^32 after a product).
struct XJob {
  const PrimeTables* pt = nullptr;
  const BigTables* bt = nullptr;
  int logN = 0;
  InOp x, y;
  int ymode = 0;
  const uint32_t* yspec = nullptr;
  uint32_t* yspec_out = nullptr;
  uint32_t *t1 = nullptr, *t2 = nullptr;
  Epi epi;
};
// out[i] = (+)= [-] (sum_j a[j] b[i+off-j]) [* post_mont[i]], i < cnt
struct DirectJob {
  uint32_t p;
  const uint32_t* a;  // the short operand (<= 40 terms)
  size_t la;
  const uint32_t* b;
  size_t lb, off, cnt;
  uint32_t* out;
  int accumulate = 0;
  const uint32_t* post_mont = nullptr;
  int negate = 0;
};
struct GarnerJob {
  uint32_t target;
  int primes;
  const uint32_t *c1, *c2, *c3;
  uint32_t* out;
  size_t n;
  int accumulate = 0;
  const uint32_t* post_mont = nullptr;  // Montgomery table, odd target only
  int negate = 0;
};
struct BatchPlan {
  std::vector<XJob> xjobs;
  std::vector<DirectJob> direct;
  std::vector<GarnerJob> garner;  // run after every xjob
};
size_t batch_descriptor_bytes(const BatchPlan& b);
// Serialises the descriptors into host_staging (pinned, batch_descriptor_bytes),
// copies them to dev_desc and launches: direct jobs, then one launch set per
// transform size, then the Garner reconstructions.
cudaError_t launch_batch(const BatchPlan& b, void* host_staging, void* dev_desc, cudaStream_t s,
                         cudaEvent_t staged = nullptr);
// Newton seeds (kind as launch_seed) and exp preparations for many jobs at once.
struct SeedJob {
  int kind;
  uint32_t p;
  const uint32_t* a;
  size_t la;
  uint32_t* out;
  int n;
  uint32_t r0;
};
struct ExpPrep {
  uint32_t p;          // odd
  const uint32_t* a;
  size_t cnt;          // min(la, n)
  uint32_t* ap;        // cnt - 1 words: a'
  uint32_t* out;       // n words: out0, 0, 0, ...
  size_t n;
  uint32_t out0 = 1;   // 1 for exp, 0 for log
};
size_t batch_aux_bytes(size_t jobs);
cudaError_t launch_seeds_batch(const std::vector<SeedJob>& jobs, void* host_staging, void* dev_desc, cudaStream_t s,
                               cudaEvent_t staged = nullptr);
cudaError_t launch_exp_prep_batch(const std::vector<ExpPrep>& jobs, void* host_staging, void* dev_desc,
                                  cudaStream_t s, cudaEvent_t staged = nullptr);
cudaError_t kernels_batch_init();
}  // namespace fpx
namespace fpx {
// In-place representation change of many arrays: Montgomery limbs -> canonical
// (to_mont = 0) or back (to_mont = 1); p = 2 keeps the bit.
struct ReprSeg {
  uint32_t p;
  uint32_t* ptr;
  size_t n;
  int to_mont;
};
size_t repr_batch_bytes(size_t segs);
cudaError_t launch_repr_batch(const std::vector<ReprSeg>& segs, void* host_staging, void* dev_desc, cudaStream_t s,
                              cudaEvent_t staged = nullptr);
// host_out[i] = *ptrs[i]; dev_buf needs ptrs.size() * 12 + 256 bytes.
cudaError_t launch_gather_first(const std::vector<const uint32_t*>& ptrs, void* host_staging, void* dev_buf,
                                uint32_t* host_out, cudaStream_t s);
// For each segment (ptr, n): the index of its last nonzero word, n if none,
// one block per segment scanning back from the end.  The results land in the
// pinned staging region itself (host_staging + last_nonzero_results_offset);
// they are in place once the stream has passed the call.
struct Segment {
  const uint32_t* ptr;
  size_t n;
};
size_t last_nonzero_batch_bytes(size_t segs);
size_t last_nonzero_results_offset(size_t segs);
cudaError_t launch_last_nonzero_batch(const std::vector<Segment>& segs, void* host_staging, void* dev_buf,
                                      cudaStream_t s);
}  // namespace fpx
