/*
 * fpx_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity oracle).
 *
 * A plain-C, single-threaded CPU restatement of the fastpoly (xcx0902/fastpoly)
 * algorithms on the number-theoretic-transform path.  It is the checker that
 * the GPU library is compared against; it is never linked into, loaded by, or
 * called from the product library.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may use it.
 *
 * Every value here is a canonical residue in [0, p).  The reference stores
 * Montgomery limbs (x * 2^32 mod p, include/fastpoly/modint.hpp:57-180); that
 * representation only matters at the boundary (checksums, raw NTT limbs), and
 * fpo_to_mont() converts.  All operations below are exact, so the results are
 * the unique values the reference's algorithms produce; each function names the
 * reference lines whose algorithm and special cases it restates.
 *
 * Parity of this file is pinned by tests/test_oracle_golden.py against the
 * reference's published bench checksums (the bench CSV files) and against the
 * reference compiled from its own headers (oracle/_ref, see oracle/Makefile).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint32_t u32;
typedef uint64_t u64;

enum { FPO_OK = 0, FPO_EDOMAIN = 1, FPO_ESIZE = 2, FPO_ELENGTH = 3, FPO_ENOMEM = 4 };

#define NAIVE_THRESHOLD 40 /* include/fastpoly/detail/poly/base.hpp:89 */

/* ---------------------------------------------------------------- field ---- */

static inline u32 addm(u32 a, u32 b, u32 p) { u64 s = (u64)a + b; return (u32)(s >= p ? s - p : s); }
static inline u32 subm(u32 a, u32 b, u32 p) { return a >= b ? a - b : (u32)((u64)a + p - b); }
static inline u32 mulm(u32 a, u32 b, u32 p) { return (u32)((u64)a * b % p); }
static inline u32 negm(u32 a, u32 p) { return a == 0 ? 0 : p - a; }

static u32 powm(u32 a, u64 e, u32 p) {
  u64 r = 1 % p, b = a % p;
  for (; e; e >>= 1) {
    if (e & 1) r = r * b % p;
    b = b * b % p;
  }
  return (u32)r;
}
/* modint.hpp:133-136: inverse via Fermat; 0 maps to 0. */
static u32 invm(u32 a, u32 p) { return p == 2 ? a : powm(a, (u64)p - 2, p); }

/* modint.hpp:28-52: smallest primitive root by trial over the factors of p-1. */
u32 fpo_primitive_root(u32 p) {
  if (p == 2) return 1;
  u32 f[16]; int nf = 0; u32 rem = p - 1;
  for (u32 d = 2; (u64)d * d <= rem; ++d) {
    if (rem % d) continue;
    f[nf++] = d;
    while (rem % d == 0) rem /= d;
  }
  if (rem > 1) f[nf++] = rem;
  for (u32 g = 2; g < p; ++g) {
    int ok = 1;
    for (int i = 0; i < nf && ok; ++i) if (powm(g, (p - 1) / f[i], p) == 1) ok = 0;
    if (ok) return g;
  }
  return 0;
}

/* ntt.hpp:48-56: largest k with 2^k | p-1. */
int fpo_ntt_max_log(u32 p) { u32 t = p - 1; int k = 0; while (t && !(t & 1)) { t >>= 1; ++k; } return k; }

/* modint.hpp:139-166: Tonelli-Shanks with the reference's choice of root
 * (p%4==3 fast path, otherwise z searched upward from 2).  Returns 0 for a
 * non-residue. */
int fpo_sqrt_mod(u32 x, u32 p, u32* out) {
  if (p == 2) { *out = x; return 1; }
  if (x == 0) { *out = 0; return 1; }
  if (powm(x, (p - 1) / 2, p) != 1) return 0;
  if (p % 4 == 3) { *out = powm(x, ((u64)p + 1) / 4, p); return 1; }
  u64 q = p - 1; int s = 0;
  while (q % 2 == 0) { q /= 2; ++s; }
  u32 z = 2;
  while (powm(z, (p - 1) / 2, p) != p - 1) z = addm(z, 1, p);
  u32 c = powm(z, q, p), r = powm(x, (q + 1) / 2, p), t = powm(x, q, p);
  int m = s;
  while (t != 1) {
    int i = 0;
    for (u32 t2 = t; t2 != 1; t2 = mulm(t2, t2, p)) ++i;
    u32 b = powm(c, (u64)1 << (m - i - 1), p);
    r = mulm(r, b, p);
    c = mulm(b, b, p);
    t = mulm(t, c, p);
    m = i;
  }
  *out = r;
  return 1;
}

u32 fpo_to_mont(u32 p, u32 v) { return p == 2 ? (v & 1u) : (u32)(((u64)v << 32) % p); }
u32 fpo_from_mont(u32 p, u32 limb) {
  if (p == 2) return limb & 1u;
  return mulm(limb % p, invm((u32)(((u64)1 << 32) % p), p), p);
}

/* bench/bench.cpp:152-159: FNV-1a-64 over raw Montgomery limbs, xor size. */
u64 fpo_checksum_mont(u32 p, const u32* vals, size_t n) {
  u64 h = 14695981039346656037ull;
  for (size_t i = 0; i < n; ++i) { h ^= fpo_to_mont(p, vals[i]); h *= 1099511628211ull; }
  return h ^ (u64)n;
}

/* std::mt19937_64 (the reference bench's generator, bench/bench.cpp:216-220). */
void fpo_mt19937_64(u64 seed, u64* out, size_t count) {
  enum { NN = 312, MM = 156 };
  u64 mt[NN];
  mt[0] = seed;
  for (int i = 1; i < NN; ++i) mt[i] = 6364136223846793005ull * (mt[i - 1] ^ (mt[i - 1] >> 62)) + (u64)i;
  int idx = NN;
  for (size_t k = 0; k < count; ++k) {
    if (idx >= NN) {
      for (int i = 0; i < NN; ++i) {
        u64 x = (mt[i] & 0xFFFFFFFF80000000ull) | (mt[(i + 1) % NN] & 0x7FFFFFFFull);
        u64 xa = x >> 1;
        if (x & 1) xa ^= 0xB5026F5AA96619E9ull;
        mt[i] = mt[(i + MM) % NN] ^ xa;
      }
      idx = 0;
    }
    u64 y = mt[idx++];
    y ^= (y >> 29) & 0x5555555555555555ull;
    y ^= (y << 17) & 0x71D67FFFEDA60000ull;
    y ^= (y << 37) & 0xFFF7EEE000000000ull;
    y ^= y >> 43;
    out[k] = y;
  }
}

/* ---------------------------------------------------------------- NTT ------ */
/*
 * ntt.hpp:5-27, :284-308, :859-946: the forward transform is a radix-4
 * decimation-in-frequency sequence with no bit reversal and the inverse the
 * matching decimation-in-time sequence, 1/n folded into its last stage.  A
 * radix-4 DIF stage is exactly two radix-2 Gentleman-Sande levels with the
 * same twiddles, so the restatement below (radix-2 levels, twiddle w_len^k,
 * w_len = g^((p-1)/len)) reproduces the reference's output permutation: the
 * spectrum in bit-reversed order.
 */
typedef struct {
  u32 p, n;
  u32 *w, *wq;   /* w_n^k, k < n/2, and Shoup quotients floor(w*2^32/p) */
  u32 *iw, *iwq; /* w_n^-k */
  u32 inv_n, inv_nq;
} plan_t;

#define PLAN_CACHE 24
static plan_t g_plans[PLAN_CACHE];
static int g_plan_next;

static inline u32 shoup_q(u32 w, u32 p) { return (u32)(((u64)w << 32) / p); }
static inline u32 shoup_mul(u32 a, u32 w, u32 wq, u32 p) {
  u32 q = (u32)(((u64)a * wq) >> 32);
  u64 r = (u64)a * w - (u64)q * p;
  return (u32)(r >= p ? r - p : r);
}

static const plan_t* get_plan(u32 p, u32 n) {
  for (int i = 0; i < PLAN_CACHE; ++i)
    if (g_plans[i].p == p && g_plans[i].n == n && g_plans[i].w) return &g_plans[i];
  plan_t* pl = &g_plans[g_plan_next];
  g_plan_next = (g_plan_next + 1) % PLAN_CACHE;
  free(pl->w); free(pl->wq); free(pl->iw); free(pl->iwq);
  memset(pl, 0, sizeof *pl);
  u32 h = n / 2 ? n / 2 : 1;
  pl->w = malloc(h * 4); pl->wq = malloc(h * 4); pl->iw = malloc(h * 4); pl->iwq = malloc(h * 4);
  if (!pl->w || !pl->wq || !pl->iw || !pl->iwq) return NULL;
  u32 g = fpo_primitive_root(p);
  u32 wn = powm(g, (p - 1) / n, p), iwn = invm(wn, p);
  u32 c = 1, ic = 1;
  for (u32 k = 0; k < h; ++k) {
    pl->w[k] = c; pl->wq[k] = shoup_q(c, p);
    pl->iw[k] = ic; pl->iwq[k] = shoup_q(ic, p);
    c = mulm(c, wn, p); ic = mulm(ic, iwn, p);
  }
  pl->inv_n = invm(n % p, p); pl->inv_nq = shoup_q(pl->inv_n, p);
  pl->p = p; pl->n = n;
  return pl;
}

/* NttPlan::forward (ntt.hpp:142): DIF, canonical output, bit-reversed order. */
int fpo_ntt_forward(u32 p, u32* x, u32 n) {
  if (n < 2 || (n & (n - 1)) || n > ((u32)1 << fpo_ntt_max_log(p)) || fpo_ntt_max_log(p) > 31)
    return FPO_ESIZE;
  const plan_t* pl = get_plan(p, n);
  if (!pl) return FPO_ENOMEM;
  for (u32 len = n; len >= 2; len >>= 1) {
    u32 half = len / 2, stride = n / len;
    for (u32 b = 0; b < n; b += len)
      for (u32 k = 0; k < half; ++k) {
        u32 u = x[b + k], v = x[b + k + half];
        x[b + k] = addm(u, v, p);
        x[b + k + half] = shoup_mul(subm(u, v, p), pl->w[k * stride], pl->wq[k * stride], p);
      }
  }
  return FPO_OK;
}

/* NttPlan::inverse (ntt.hpp:179): DIT from bit-reversed order, scaled by 1/n. */
int fpo_ntt_inverse(u32 p, u32* x, u32 n) {
  if (n < 2 || (n & (n - 1)) || n > ((u32)1 << fpo_ntt_max_log(p)) || fpo_ntt_max_log(p) > 31)
    return FPO_ESIZE;
  const plan_t* pl = get_plan(p, n);
  if (!pl) return FPO_ENOMEM;
  for (u32 len = 2; len <= n; len <<= 1) {
    u32 half = len / 2, stride = n / len;
    for (u32 b = 0; b < n; b += len)
      for (u32 k = 0; k < half; ++k) {
        u32 u = x[b + k];
        u32 v = shoup_mul(x[b + k + half], pl->iw[k * stride], pl->iwq[k * stride], p);
        x[b + k] = addm(u, v, p);
        x[b + k + half] = subm(u, v, p);
      }
  }
  for (u32 i = 0; i < n; ++i) x[i] = shoup_mul(x[i], pl->inv_n, pl->inv_nq, p);
  return FPO_OK;
}

/* ------------------------------------------------------- products -------- */

static u32 next_pow2_u(u64 need) { u32 r = 1; while (r < need) r <<= 1; return r; }

/* Direct product, out[i] = sum a[j]*b[i-j] for i < cnt (convolution.hpp:33-95). */
static void direct_product(u32 p, const u32* a, size_t la, const u32* b, size_t lb, u32* out, size_t cnt) {
  memset(out, 0, cnt * 4);
  for (size_t i = 0; i < la && i < cnt; ++i) {
    if (!a[i]) continue;
    for (size_t j = 0; j < lb && i + j < cnt; ++j) out[i + j] = addm(out[i + j], mulm(a[i], b[j], p), p);
  }
}

/* Native NTT product (convolution.hpp:116-138): requires next_pow2(la+lb-1) <= 2^v2(p-1). */
static int ntt_product(u32 p, const u32* a, size_t la, const u32* b, size_t lb, u32* out, size_t cnt) {
  u32 N = next_pow2_u(la + lb - 1);
  if (N < 2) N = 2;
  u32* fa = calloc(N, 4);
  u32* fb = calloc(N, 4);
  if (!fa || !fb) { free(fa); free(fb); return FPO_ENOMEM; }
  memcpy(fa, a, la * 4); memcpy(fb, b, lb * 4);
  fpo_ntt_forward(p, fa, N);
  fpo_ntt_forward(p, fb, N);
  for (u32 i = 0; i < N; ++i) fa[i] = mulm(fa[i], fb[i], p);
  fpo_ntt_inverse(p, fa, N);
  memcpy(out, fa, cnt * 4);
  free(fa); free(fb);
  return FPO_OK;
}

/* crt_convolution.hpp:14-19: auxiliary primes, all below 2^30, with 2^24-point roots. */
static const u32 CRT_P[3] = {167772161u, 469762049u, 754974721u};

/* crt_convolution.hpp:78-83: strict bound min(la,lb)*(p-1)^2 < product of primes used. */
size_t fpo_crt_prime_count(u32 p, size_t terms) {
  const u64 square = (u64)(p - 1) * (p - 1);
  if (square <= (CRT_P[0] - 1ull) / terms) return 1;
  if (square <= ((u64)CRT_P[0] * CRT_P[1] - 1) / terms) return 2;
  return 3;
}

/* Exact integer product of a,b reduced mod auxiliary prime P, window [0,cnt)
 * (auxiliary_product, crt_convolution.hpp:37-73; inputs lifted per :25-32). */
static int aux_product(u32 P, const u32* a, size_t la, const u32* b, size_t lb, u32* out, size_t cnt) {
  u32* aa = malloc(la * 4);
  u32* bb = malloc(lb * 4);
  if (!aa || !bb) { free(aa); free(bb); return FPO_ENOMEM; }
  for (size_t i = 0; i < la; ++i) aa[i] = a[i] % P;
  for (size_t i = 0; i < lb; ++i) bb[i] = b[i] % P;
  int rc = FPO_OK;
  if ((la < lb ? la : lb) <= NAIVE_THRESHOLD) direct_product(P, aa, la, bb, lb, out, cnt);
  else rc = ntt_product(P, aa, la, bb, lb, out, cnt);
  free(aa); free(bb);
  return rc;
}

/* crt_product_window (crt_convolution.hpp:132-182) + Garner restore (:89-127):
 * dst[i] += (a*b)[i] mod p for i < cnt. */
static int crt_window_accumulate(u32 p, const u32* a, size_t la, const u32* b, size_t lb, u32* dst, size_t cnt) {
  const size_t primes = fpo_crt_prime_count(p, la < lb ? la : lb);
  u32* c[3] = {0, 0, 0};
  int rc = FPO_OK;
  for (size_t k = 0; k < primes; ++k) {
    c[k] = malloc(cnt * 4 + 4);
    if (!c[k]) { rc = FPO_ENOMEM; goto done; }
    rc = aux_product(CRT_P[k], a, la, b, lb, c[k], cnt);
    if (rc) goto done;
  }
  {
    const u64 P1 = CRT_P[0], P2 = CRT_P[1], P3 = CRT_P[2];
    const u32 inv12 = invm((u32)(P1 % P2), (u32)P2);
    const u32 inv123 = invm((u32)((P1 * P2) % P3), (u32)P3);
    const u64 p12_t = (P1 * P2) % p;
    for (size_t i = 0; i < cnt; ++i) {
      u64 x1 = c[0][i], value;
      if (primes == 1) value = x1 % p;
      else {
        u64 x2 = mulm((u32)((c[1][i] + P2 - x1 % P2) % P2), inv12, (u32)P2);
        u64 x12 = x1 + P1 * x2;
        if (primes == 2) value = x12 % p;
        else {
          u64 x3 = mulm((u32)((c[2][i] + P3 - x12 % P3) % P3), inv123, (u32)P3);
          value = (x12 % p + p12_t * x3 % p) % p;
        }
      }
      dst[i] = addm(dst[i], (u32)value, p);
    }
  }
done:
  for (int k = 0; k < 3; ++k) free(c[k]);
  return rc;
}

/* crt_convolution<M,BlockSize> (crt_convolution.hpp:187-205): block-pair loop. */
int fpo_crt_convolution(u32 p, const u32* a, size_t la, const u32* b, size_t lb, size_t outn, size_t block, u32* out) {
  memset(out, 0, outn * 4);
  if (la > outn) la = outn;
  if (lb > outn) lb = outn;
  for (size_t ai = 0; ai < la;) {
    size_t na = block < la - ai ? block : la - ai;
    for (size_t bi = 0; bi < lb && bi < outn - ai;) {
      size_t nb = block < lb - bi ? block : lb - bi;
      size_t cnt = na + nb - 1;
      if (cnt > outn - ai - bi) cnt = outn - ai - bi;
      int rc = crt_window_accumulate(p, a + ai, na, b + bi, nb, out + ai + bi, cnt);
      if (rc) return rc;
      bi += nb;
    }
    ai += na;
  }
  return FPO_OK;
}

/*
 * conv_limbs (convolution.hpp:17-141) and conv (:145-147).
 * Output length = min(min(la,lim)+min(lb,lim)-1, lim); empty operand or lim==0 -> empty.
 * Dispatch: direct product when the shorter operand has <= 40 terms; the native
 * NTT when the padded size fits 2^v2(p-1); the 3-prime CRT otherwise.  (The
 * reference's tail-repair branch, :105-115, computes the same exact product.)
 */
int fpo_conv(u32 p, const u32* a, size_t la, const u32* b, size_t lb, size_t lim, u32* out, size_t* out_len) {
  *out_len = 0;
  if (la == 0 || lb == 0 || lim == 0) return FPO_OK;
  if (la > lim) la = lim;
  if (lb > lim) lb = lim;
  if (la > SIZE_MAX - (lb - 1)) return FPO_ELENGTH;
  const size_t full = la + lb - 1, outn = full < lim ? full : lim;
  *out_len = outn;
  const size_t mn = la < lb ? la : lb;
  if (mn <= NAIVE_THRESHOLD) { direct_product(p, a, la, b, lb, out, outn); return FPO_OK; }
  const int vmax = fpo_ntt_max_log(p);
  if (p != 2 && vmax < 31 && (u64)next_pow2_u(full) <= ((u64)1 << vmax) && full <= ((u64)1 << 31))
    return ntt_product(p, a, la, b, lb, out, outn);
  return fpo_crt_convolution(p, a, la, b, lb, outn, (size_t)1 << 23, out);
}

/* Exact coefficients [off, off+cnt) of a*b (the Newton middle products,
 * crt_middle_product crt_convolution.hpp:210-227 and the high-half windows of
 * inverse.hpp:44-63). */
static int mul_window(u32 p, const u32* a, size_t la, const u32* b, size_t lb, size_t off, size_t cnt, u32* out) {
  memset(out, 0, cnt * 4);
  if (!la || !lb || !cnt) return FPO_OK;
  size_t lim = off + cnt;
  u32* tmp = malloc(lim * 4);
  if (!tmp) return FPO_ENOMEM;
  size_t got = 0;
  int rc = fpo_conv(p, a, la < lim ? la : lim, b, lb < lim ? lb : lim, lim, tmp, &got);
  if (!rc)
    for (size_t i = 0; i < cnt; ++i) out[i] = off + i < got ? tmp[off + i] : 0;
  free(tmp);
  return rc;
}

/* ------------------------------------------------------------ series ------ */

/* inverse_seed (inverse.hpp:68-77): c[i] = -(sum_{j=1..i} a[j] c[i-j]) c[0]. */
static void inverse_seed(u32 p, const u32* a, size_t la, u32* c, size_t n) {
  c[0] = invm(a[0], p);
  for (size_t i = 1; i < n; ++i) {
    u32 s = 0;
    for (size_t j = 1; j <= i && j < la; ++j) s = addm(s, mulm(a[j], c[i - j], p), p);
    c[i] = mulm(negm(s, p), c[0], p);
  }
}

/* extend_inverse (inverse.hpp:18-65): c[0,k) -> c[0,wanted), wanted <= 2k,
 * using the high half of a*c (the middle product) and one truncated product. */
static int extend_inverse(u32 p, const u32* a, size_t la, u32* c, size_t k, size_t wanted) {
  const size_t hlen = wanted - k;
  if (hlen <= 8) {
    for (size_t i = k; i < wanted; ++i) {
      u32 s = 0;
      for (size_t j = 1; j <= i && j < la; ++j) s = addm(s, mulm(a[j], c[i - j], p), p);
      c[i] = mulm(negm(s, p), c[0], p);
    }
    return FPO_OK;
  }
  u32* e = malloc(hlen * 4);
  u32* corr = malloc(hlen * 4);
  if (!e || !corr) { free(e); free(corr); return FPO_ENOMEM; }
  int rc = mul_window(p, a, la < wanted ? la : wanted, c, k, k, hlen, e);
  for (size_t i = 0; i < hlen; ++i) e[i] = negm(e[i], p);
  if (!rc) rc = mul_window(p, e, hlen, c, k, 0, hlen, corr);
  if (!rc) memcpy(c + k, corr, hlen * 4);
  free(e); free(corr);
  return rc;
}

/* inv (inverse.hpp:163-188). out has n entries. */
int fpo_inv(u32 p, const u32* a, size_t la, size_t n, u32* out) {
  if (n == 0) return FPO_OK;
  if (la == 0 || a[0] == 0) return FPO_EDOMAIN;
  size_t cnt = la < n ? la : n;
  while (cnt > 1 && a[cnt - 1] == 0) --cnt;
  memset(out, 0, n * 4);
  if (cnt == 1) { out[0] = invm(a[0], p); return FPO_OK; }
  const size_t seed = n < 32 ? n : 32;
  inverse_seed(p, a, cnt, out, seed);
  for (size_t m = seed; m < n; m <<= 1) {
    size_t w = 2 * m < n ? 2 * m : n;
    int rc = extend_inverse(p, a, cnt, out, m, w);
    if (rc) return rc;
  }
  return FPO_OK;
}

/* inv_series (calculus.hpp:53-94): 1/i for i <= n, requires n < p. tab has n+1 entries. */
int fpo_inv_series(u32 p, size_t n, u32* tab) {
  if (n >= p) return FPO_EDOMAIN;
  tab[0] = 0;
  if (n == 0) return FPO_OK;
  tab[1] = 1;
  for (size_t i = 2; i <= n; ++i) tab[i] = negm(mulm(p / (u32)i, tab[p % (u32)i], p), p);
  return FPO_OK;
}

/* derivative_prefix (calculus.hpp:17-39): r[i-1] = a[i]*i, i < min(la,cnt). */
static size_t derivative_prefix(u32 p, const u32* a, size_t la, size_t cnt, u32* r) {
  if (cnt > la) cnt = la;
  if (cnt <= 1) return 0;
  for (size_t i = 1; i < cnt; ++i) r[i - 1] = mulm(a[i], (u32)(i % p), p);
  return cnt - 1;
}

/* log (exponential.hpp:85-98): integral(a' * inv(a, n-1)) mod x^n, a0 == 1, n <= p. */
int fpo_log(u32 p, const u32* a, size_t la, size_t n, u32* out) {
  if (n == 0) return FPO_OK;
  if (la == 0 || a[0] != 1 % p) return FPO_EDOMAIN;
  if (n > p) return FPO_EDOMAIN;
  memset(out, 0, n * 4);
  if (n == 1) return FPO_OK;
  u32* d = malloc(n * 4);
  u32* ia = malloc(n * 4);
  u32* pr = malloc(n * 4);
  u32* tab = malloc((n + 1) * 4);
  int rc = FPO_ENOMEM;
  if (d && ia && pr && tab) {
    size_t ld = derivative_prefix(p, a, la, n, d), lp = 0;
    rc = fpo_inv(p, a, la, n - 1, ia);
    if (!rc) rc = fpo_conv(p, d, ld, ia, n - 1, n - 1, pr, &lp);
    if (!rc) rc = fpo_inv_series(p, lp, tab);
    if (!rc) for (size_t i = 0; i < lp; ++i) out[i + 1] = mulm(pr[i], tab[i + 1], p);
  }
  free(d); free(ia); free(pr); free(tab);
  return rc;
}

/* exp (exponential.hpp:107-207): Newton on the high differential residual. */
int fpo_exp(u32 p, const u32* a, size_t la, size_t n, u32* out) {
  if (n == 0) return FPO_OK;
  if (la != 0 && a[0] != 0) return FPO_EDOMAIN;
  if (n - 1 >= p) return FPO_EDOMAIN;
  memset(out, 0, n * 4);
  u32* ap = malloc(n * 4 + 4);
  if (!ap) return FPO_ENOMEM;
  size_t lap = derivative_prefix(p, a, la, n, ap);
  while (lap && ap[lap - 1] == 0) --lap; /* trim (basic.hpp:15-17) */
  out[0] = 1 % p;
  if (lap == 0) { free(ap); return FPO_OK; }
  const size_t seed = lap <= NAIVE_THRESHOLD ? n : (n < 32 ? n : 32);
  u32* den = malloc(n * 4 + 4);
  u32* c = calloc(n, 4);
  u32* t1 = malloc(n * 4 + 4);
  u32* t2 = malloc(n * 4 + 4);
  int rc = FPO_ENOMEM;
  if (!den || !c || !t1 || !t2) goto done;
  rc = fpo_inv_series(p, n - 1, den);
  if (rc) goto done;
  for (size_t i = 1; i < seed; ++i) {
    u32 s = 0;
    for (size_t j = 1; j <= i && j <= lap; ++j) s = addm(s, mulm(ap[j - 1], out[i - j], p), p);
    out[i] = mulm(s, den[i], p);
  }
  if (seed == n) { rc = FPO_OK; goto done; }
  size_t csize = seed / 2;
  inverse_seed(p, out, seed, c, csize);
  for (size_t m = seed; m < n; m *= 2) {
    size_t m2 = 2 * m < n ? 2 * m : n, hlen = m2 - m;
    if (hlen <= 8) {
      for (size_t i = m; i < m2; ++i) {
        u32 s = 0;
        for (size_t j = 1; j <= i && j <= lap; ++j) s = addm(s, mulm(ap[j - 1], out[i - j], p), p);
        out[i] = mulm(s, den[i], p);
      }
      continue;
    }
    if (csize < hlen) {
      rc = extend_inverse(p, out, m, c, csize, hlen);
      if (rc) goto done;
      csize = hlen;
    }
    /* residual = (a' b)[m-1, m-1+hlen); correction = (residual * c) / (m+i); b[m..] = (correction * b) */
    rc = mul_window(p, ap, lap < m2 - 1 ? lap : m2 - 1, out, m, m - 1, hlen, t1);
    if (!rc) rc = mul_window(p, t1, hlen, c, csize, 0, hlen, t2);
    if (rc) goto done;
    for (size_t i = 0; i < hlen; ++i) t2[i] = mulm(t2[i], den[m + i], p);
    rc = mul_window(p, t2, hlen, out, m, 0, hlen, t1);
    if (rc) goto done;
    memcpy(out + m, t1, hlen * 4);
  }
  rc = FPO_OK;
done:
  free(ap); free(den); free(c); free(t1); free(t2);
  return rc;
}

/* sqrt (square_root.hpp:12-112). */
int fpo_sqrt(u32 p, const u32* a, size_t la, size_t n, u32* out) {
  if (n == 0) return FPO_OK;
  memset(out, 0, n * 4);
  if (p == 2) {
    for (size_t i = 0; i < la && i < n; ++i) {
      if (i & 1) { if (a[i]) return FPO_EDOMAIN; }
      else out[i / 2] = a[i];
    }
    return FPO_OK;
  }
  size_t v = 0;
  while (v < la && a[v] == 0) ++v;
  if (v == la) return FPO_OK;
  if (v & 1) return FPO_EDOMAIN;
  u32 root0;
  if (!fpo_sqrt_mod(a[v], p, &root0)) return FPO_EDOMAIN;
  const size_t half = v / 2;
  if (half >= n) return FPO_OK;
  const size_t inner = n - half, ulen = la - v;
  const u32* u = a + v;
  const size_t ucnt = ulen < inner ? ulen : inner;
  int all_zero = 1;
  for (size_t i = 1; i < ucnt; ++i) if (u[i]) { all_zero = 0; break; }
  if (all_zero) { out[half] = root0; return FPO_OK; }
  u32* b = out + half;
  const size_t seed = inner < 32 ? inner : 32;
  const u32 half_inv = (p + 1) / 2;
  const u32 twice_root_inv = mulm(invm(root0, p), half_inv, p);
  b[0] = root0;
  for (size_t i = 1; i < seed; ++i) {
    u32 r = i < ulen ? u[i] : 0;
    for (size_t j = 1; j < i; ++j) r = subm(r, mulm(b[j], b[i - j], p), p);
    b[i] = mulm(r, twice_root_inv, p);
  }
  if (inner <= seed) return FPO_OK;
  u32* c = calloc(inner, 4);
  u32* t1 = malloc(inner * 4 + 4);
  u32* t2 = malloc(inner * 4 + 4);
  int rc = FPO_ENOMEM;
  if (!c || !t1 || !t2) goto done;
  size_t csize = seed / 2;
  inverse_seed(p, b, seed, c, csize);
  for (size_t m = seed; m < inner; m *= 2) {
    size_t m2 = 2 * m < inner ? 2 * m : inner, hlen = m2 - m;
    if (hlen <= 8) {
      for (size_t i = m; i < m2; ++i) {
        u32 r = i < ulen ? u[i] : 0;
        for (size_t j = 1; j < i; ++j) r = subm(r, mulm(b[j], b[i - j], p), p);
        b[i] = mulm(r, twice_root_inv, p);
      }
      continue;
    }
    if (csize < hlen) {
      rc = extend_inverse(p, b, m, c, csize, hlen);
      if (rc) goto done;
      csize = hlen;
    }
    /* residual = u[m..m2) - (b*b)[m..m2); b[m..] = (residual * c mod x^hlen) / 2 */
    rc = mul_window(p, b, m, b, m, m, hlen, t1);
    if (rc) goto done;
    for (size_t i = 0; i < hlen; ++i) t1[i] = subm(m + i < ulen ? u[m + i] : 0, t1[i], p);
    rc = mul_window(p, t1, hlen, c, csize, 0, hlen, t2);
    if (rc) goto done;
    for (size_t i = 0; i < hlen; ++i) b[m + i] = mulm(t2[i], half_inv, p);
  }
  rc = FPO_OK;
done:
  free(c); free(t1); free(t2);
  return rc;
}

/* pow (power.hpp:17-87): a^k mod x^n for 64-bit k. */
int fpo_pow(u32 p, const u32* a, size_t la, u64 k, size_t n, u32* out) {
  if (n == 0) return FPO_OK;
  memset(out, 0, n * 4);
  if (k == 0) { out[0] = 1 % p; return FPO_OK; }
  if (k == 1) { memcpy(out, a, (la < n ? la : n) * 4); return FPO_OK; }
  size_t v = 0;
  while (v < la && a[v] == 0) ++v;
  if (v == la) return FPO_OK;
  if (v != 0 && k > (n - 1) / v) return FPO_OK;
  const size_t sh = (size_t)(v * k), inner = n - sh;
  size_t ulen = la - v < inner ? la - v : inner;
  const u32* u = a + v;
  while (ulen && u[ulen - 1] == 0) --ulen;
  if (ulen == 1) { out[sh] = powm(u[0], k, p); return FPO_OK; }
  int rc = FPO_OK;
  if (k > 64 && ulen == 2 && inner <= p) {
    /* binomial series (power.hpp:44-59) */
    const u32 e = (u32)(k % p);
    const size_t cnt = inner < (size_t)e + 1 ? inner : (size_t)e + 1;
    u32* div = malloc(cnt * 4 + 4);
    if (!div) return FPO_ENOMEM;
    rc = fpo_inv_series(p, cnt - 1, div);
    if (!rc) {
      out[sh] = powm(u[0], k, p);
      const u32 ratio = mulm(u[1], invm(u[0], p), p);
      u32 factor = mulm(ratio, e % p, p);
      for (size_t j = 1; j < cnt; ++j) {
        out[sh + j] = mulm(mulm(out[sh + j - 1], factor, p), div[j], p);
        factor = subm(factor, ratio, p);
      }
    }
    free(div);
    return rc;
  }
  if (k <= 64 || inner > p) {
    /* binary powering (power.hpp:61-74) */
    u32* r = calloc(inner, 4);
    u32* base = calloc(inner, 4);
    u32* tmp = calloc(inner, 4);
    if (!r || !base || !tmp) { free(r); free(base); free(tmp); return FPO_ENOMEM; }
    size_t lr = 1, lb = ulen, lt = 0;
    r[0] = 1 % p;
    memcpy(base, u, ulen * 4);
    for (u64 e = k; e; e >>= 1) {
      if (e & 1) {
        rc = fpo_conv(p, r, lr, base, lb, inner, tmp, &lt);
        if (rc) break;
        memcpy(r, tmp, lt * 4); lr = lt;
      }
      if (e > 1) {
        rc = fpo_conv(p, base, lb, base, lb, inner, tmp, &lt);
        if (rc) break;
        memcpy(base, tmp, lt * 4); lb = lt;
      }
    }
    if (!rc) memcpy(out + sh, r, (lr < inner ? lr : inner) * 4);
    free(r); free(base); free(tmp);
    return rc;
  }
  /* c^k * exp(k * log(u / c)) (power.hpp:76-86) */
  const u32 c = u[0], ci = invm(c, p);
  u32* nrm = malloc(ulen * 4);
  u32* l = malloc(inner * 4);
  if (!nrm || !l) { free(nrm); free(l); return FPO_ENOMEM; }
  for (size_t i = 0; i < ulen; ++i) nrm[i] = mulm(u[i], ci, p);
  rc = fpo_log(p, nrm, ulen, inner, l);
  if (!rc) {
    const u32 km = (u32)(k % p);
    for (size_t i = 0; i < inner; ++i) l[i] = mulm(l[i], km, p);
    rc = fpo_exp(p, l, inner, inner, out + sh);
    const u32 ck = powm(c, k, p);
    if (!rc) for (size_t i = 0; i < inner; ++i) out[sh + i] = mulm(out[sh + i], ck, p);
  }
  free(nrm); free(l);
  return rc;
}

/* divide<Remainder> (division.hpp:12-80), divmod (:86-88).  q and r need
 * capacity la; lengths are returned trimmed like the reference's results. */
int fpo_divmod(u32 p, const u32* a, size_t la, const u32* b, size_t lb, u32* q, size_t* lq, u32* r, size_t* lr) {
  size_t an = la, bn = lb;
  *lq = 0; *lr = 0;
  while (an && a[an - 1] == 0) --an;
  while (bn && b[bn - 1] == 0) --bn;
  if (bn == 0) return FPO_EDOMAIN;
  if (an < bn) { memcpy(r, a, an * 4); *lr = an; return FPO_OK; }
  if (bn == 1) {
    const u32 bi = invm(b[0], p);
    for (size_t i = 0; i < an; ++i) q[i] = mulm(a[i], bi, p);
    *lq = an;
    return FPO_OK;
  }
  const size_t dn = an - bn + 1;
  int rc = FPO_OK;
  if (bn <= 16 || dn <= 32) {
    /* long division (:29-55) */
    u32* w = malloc(an * 4);
    if (!w) return FPO_ENOMEM;
    memcpy(w, a, an * 4);
    const u32 li = invm(b[bn - 1], p);
    for (size_t i = dn; i-- > 0;) {
      const u32 f = mulm(w[i + bn - 1], li, p);
      q[i] = f;
      if (!f) continue;
      for (size_t j = 0; j < bn - 1; ++j) w[i + j] = subm(w[i + j], mulm(f, b[j], p), p);
    }
    size_t rn = bn - 1;
    while (rn && w[rn - 1] == 0) --rn;
    memcpy(r, w, rn * 4);
    *lq = dn; *lr = rn;
    free(w);
    return FPO_OK;
  }
  /* q = rev(rev(a) * inv(rev(b), dn)) (:57-65); r = low(a - b q) (:69-79) */
  u32* ra = malloc(dn * 4);
  u32* rb = malloc(dn * 4);
  u32* ib = malloc(dn * 4);
  u32* rq = malloc(dn * 4);
  u32* prod = malloc(bn * 4);
  if (!ra || !rb || !ib || !rq || !prod) { rc = FPO_ENOMEM; goto done; }
  for (size_t i = 0; i < dn; ++i) ra[i] = a[an - 1 - i];
  const size_t nrb = bn < dn ? bn : dn;
  for (size_t i = 0; i < nrb; ++i) rb[i] = b[bn - 1 - i];
  rc = fpo_inv(p, rb, nrb, dn, ib);
  size_t lrq = 0;
  if (!rc) rc = fpo_conv(p, ra, dn, ib, dn, dn, rq, &lrq);
  if (rc) goto done;
  for (size_t i = lrq; i < dn; ++i) rq[i] = 0;
  for (size_t i = 0; i < dn; ++i) q[i] = rq[dn - 1 - i];
  *lq = dn;
  {
    const size_t rn = bn - 1;
    size_t lp = 0;
    rc = fpo_conv(p, b, bn, q, dn, rn, prod, &lp);
    if (rc) goto done;
    for (size_t i = 0; i < rn; ++i) r[i] = subm(a[i], i < lp ? prod[i] : 0, p);
    size_t t = rn;
    while (t && r[t - 1] == 0) --t;
    *lr = t;
  }
done:
  free(ra); free(rb); free(ib); free(rq); free(prod);
  return rc;
}
