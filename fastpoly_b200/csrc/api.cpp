// api.cpp - the extern "C" boundary (include/fpx_b200.h).
//
// Host-buffer entry points copy inputs to pool memory, run the device
// operation on the context's stream and copy the result back before
// returning.  Errors never escape as exceptions: each entry point returns an
// fpx status and records a message for fpx_last_error_message().
#include <cstring>
#include <memory>
#include <mutex>
#include <string>

#include "engine.h"
#include "fpx_b200.h"

struct fpx_ctx {
  std::unique_ptr<fpx::Engine> eng;
  std::string err;
  std::mutex mu;
};

namespace {

using fpx::Buf;
using fpx::Error;

template <class F>
int guarded(fpx_ctx* ctx, F&& f) {
  if (!ctx) return FPX_EINVAL;
  std::lock_guard<std::mutex> g(ctx->mu);
  try {
    ctx->eng->check(cudaSetDevice(ctx->eng->device()), "cudaSetDevice");
    f(*ctx->eng);
    ctx->err.clear();
    return FPX_OK;
  } catch (const Error& e) {
    ctx->err = e.msg;
    return e.code;
  } catch (const std::exception& e) {
    ctx->err = e.what();
    return FPX_EINVAL;
  }
}

void check_modulus(uint32_t p) {
  if (p < 2 || p >= (1u << 31) || !fpx::is_prime(p)) throw Error{FPX_EINVAL, "modulus must be a prime 2 <= p < 2^31"};
}

void check_ptr(const void* ptr, size_t n, const char* what) {
  if (n && !ptr) throw Error{FPX_EINVAL, std::string("null pointer: ") + what};
}

// Host input -> pool buffer, canonical.
Buf upload(fpx::Engine& e, uint32_t p, const uint32_t* h, size_t n, int repr) {
  Buf d(&e.pool(), n);
  if (n) {
    e.to_device(d.get(), h, n);
    if (repr == FPX_REPR_MONTGOMERY) e.check(fpx::launch_from_mont(p, d.get(), d.get(), n, e.stream()), "repr");
  }
  return d;
}

void download(fpx::Engine& e, uint32_t p, uint32_t* h, uint32_t* d, size_t n, int repr) {
  if (n && repr == FPX_REPR_MONTGOMERY) e.check(fpx::launch_to_mont(p, d, d, n, e.stream()), "repr");
  e.to_host(h, d, n);
}

void check_repr(int repr) {
  if (repr != FPX_REPR_CANONICAL && repr != FPX_REPR_MONTGOMERY) throw Error{FPX_EINVAL, "unknown repr"};
}

using SeriesFn = void (fpx::Engine::*)(uint32_t, const uint32_t*, size_t, size_t, uint32_t*);

int series_host(fpx_ctx* ctx, SeriesFn fn, uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out,
                int repr) {
  return guarded(ctx, [&](fpx::Engine& e) {
    check_modulus(p);
    check_repr(repr);
    check_ptr(a, la, "a");
    check_ptr(out, n, "out");
    if (n == 0) return;
    const size_t lx = la < n ? la : n;  // coefficients at or beyond n never matter
    Buf da = upload(e, p, a, lx, repr);
    Buf dout(&e.pool(), n);
    (e.*fn)(p, da.get(), lx, n, dout.get());
    download(e, p, out, dout.get(), n, repr);
  });
}

int series_dev(fpx_ctx* ctx, SeriesFn fn, uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out) {
  return guarded(ctx, [&](fpx::Engine& e) {
    check_modulus(p);
    check_ptr(a, la, "a");
    check_ptr(out, n, "out");
    (e.*fn)(p, a, la < n ? la : n, n, out);
  });
}

}  // namespace

extern "C" {

int fpx_ctx_create(int device, size_t pool_limit_bytes, fpx_ctx** out) {
  if (!out) return FPX_EINVAL;
  *out = nullptr;
  auto ctx = std::make_unique<fpx_ctx>();
  try {
    ctx->eng = std::make_unique<fpx::Engine>(device, pool_limit_bytes);
  } catch (const Error& e) {
    return e.code;
  } catch (...) {
    return FPX_ECUDA;
  }
  *out = ctx.release();
  return FPX_OK;
}

int fpx_ctx_destroy(fpx_ctx* ctx) {
  if (!ctx) return FPX_EINVAL;
  delete ctx;
  return FPX_OK;
}

int fpx_ctx_set_stream(fpx_ctx* ctx, void* stream) {
  return guarded(ctx, [&](fpx::Engine& e) { e.set_stream(static_cast<cudaStream_t>(stream)); });
}

void* fpx_ctx_stream(fpx_ctx* ctx) { return ctx ? static_cast<void*>(ctx->eng->stream()) : nullptr; }

int fpx_ctx_synchronize(fpx_ctx* ctx) {
  return guarded(ctx, [&](fpx::Engine& e) { e.sync(); });
}

const char* fpx_last_error_message(fpx_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int fpx_pool_stats(fpx_ctx* ctx, fpx_pool_stats_t* out) {
  if (!ctx || !out) return FPX_EINVAL;
  auto& p = ctx->eng->pool();
  out->cached_bytes = p.cached_bytes;
  out->cached_blocks = p.cached_blocks;
  out->in_use_bytes = p.in_use_bytes;
  out->system_allocations = p.system_allocations;
  out->cache_hits = p.cache_hits;
  out->limit_bytes = p.limit_;
  return FPX_OK;
}

int fpx_host_alloc(size_t bytes, void** out) {
  if (!out) return FPX_EINVAL;
  *out = nullptr;
  if (bytes == 0) return FPX_EINVAL;
  if (cudaHostAlloc(out, bytes, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    return FPX_ENOMEM;
  }
  return FPX_OK;
}

int fpx_host_free(void* p) {
  if (!p) return FPX_EINVAL;
  if (cudaFreeHost(p) != cudaSuccess) {
    cudaGetLastError();
    return FPX_EINVAL;
  }
  return FPX_OK;
}

int fpx_release_pool(fpx_ctx* ctx) {
  return guarded(ctx, [&](fpx::Engine& e) {
    e.sync();
    e.drop_graphs();
    e.drop_flush_arena();
    e.pool().release();
  });
}

int fpx_ctx_set_crt_block(fpx_ctx* ctx, size_t block_terms) {
  return guarded(ctx, [&](fpx::Engine& e) { e.set_crt_block(block_terms); });
}

int fpx_col_shape_candidates(fpx_ctx* ctx, int log_n, int kind, fpx_col_shape* out, int max, int* count) {
  if (!out || !count || max < 0) return FPX_EINVAL;
  return guarded(ctx, [&](fpx::Engine& e) {
    fpx::ColShape c[8];
    const int n = e.col_shape_candidates(log_n, kind, c, 8);
    *count = n;
    for (int i = 0; i < n && i < max; ++i) out[i] = fpx_col_shape{c[i].lw1, c[i].lw2, c[i].split};
  });
}

int fpx_col_shape_get(fpx_ctx* ctx, int log_n, int kind, fpx_col_shape* out) {
  if (!out) return FPX_EINVAL;
  return guarded(ctx, [&](fpx::Engine& e) {
    fpx::ColShape s = e.col_shape(log_n, kind);
    if (s.lw1 == 0) {  // the default shape, spelled out
      fpx::ColShape c[8];
      if (e.col_shape_candidates(log_n, kind, c, 8) > 0) s = c[0];
    }
    *out = fpx_col_shape{s.lw1, s.lw2, s.split};
  });
}

int fpx_col_shape_set(fpx_ctx* ctx, int log_n, int kind, const fpx_col_shape* shape) {
  if (!shape) return FPX_EINVAL;
  return guarded(ctx, [&](fpx::Engine& e) {
    fpx::ColShape s;
    s.lw1 = shape->lw1;
    s.lw2 = shape->lw2;
    s.split = shape->split;
    e.set_col_shape(log_n, kind, s);
  });
}

int fpx_profile(fpx_ctx* ctx, int enable) {
  return guarded(ctx, [&](fpx::Engine& e) { e.profile(enable != 0); });
}

int fpx_profile_report(fpx_ctx* ctx, char* buf, size_t cap, size_t* needed) {
  return guarded(ctx, [&](fpx::Engine& e) {
    const std::string r = e.profile_report();
    if (needed) *needed = r.size() + 1;
    if (buf && cap) {
      const size_t n = r.size() < cap - 1 ? r.size() : cap - 1;
      std::memcpy(buf, r.data(), n);
      buf[n] = 0;
    }
  });
}

uint64_t fpx_launch_count(fpx_ctx* ctx) { return ctx ? ctx->eng->launches() : 0; }

int fpx_ntt_max_log(uint32_t p) { return (p >= 2 && p < (1u << 31)) ? fpx::v2_of(p) : -1; }

int fpx_ntt_forward(fpx_ctx* ctx, uint32_t p, uint32_t* data, uint32_t n, int repr) {
  return guarded(ctx, [&](fpx::Engine& e) {
    check_modulus(p);
    check_repr(repr);
    check_ptr(data, n, "data");
    Buf d = upload(e, p, data, n, repr);
    e.ntt(p, d.get(), n, false);
    download(e, p, data, d.get(), n, repr);
  });
}

int fpx_ntt_inverse(fpx_ctx* ctx, uint32_t p, uint32_t* data, uint32_t n, int repr) {
  return guarded(ctx, [&](fpx::Engine& e) {
    check_modulus(p);
    check_repr(repr);
    check_ptr(data, n, "data");
    Buf d = upload(e, p, data, n, repr);
    e.ntt(p, d.get(), n, true);
    download(e, p, data, d.get(), n, repr);
  });
}

int fpx_ntt_forward_device(fpx_ctx* ctx, uint32_t p, uint32_t* d_data, uint32_t n) {
  return guarded(ctx, [&](fpx::Engine& e) {
    check_modulus(p);
    check_ptr(d_data, n, "data");
    e.ntt(p, d_data, n, false);
  });
}

int fpx_ntt_inverse_device(fpx_ctx* ctx, uint32_t p, uint32_t* d_data, uint32_t n) {
  return guarded(ctx, [&](fpx::Engine& e) {
    check_modulus(p);
    check_ptr(d_data, n, "data");
    e.ntt(p, d_data, n, true);
  });
}

int fpx_conv(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, size_t n,
             uint32_t* out, size_t* out_len, int repr) {
  return guarded(ctx, [&](fpx::Engine& e) {
    check_modulus(p);
    check_repr(repr);
    check_ptr(a, la, "a");
    check_ptr(b, lb, "b");
    if (!out_len) throw Error{FPX_EINVAL, "null out_len"};
    *out_len = 0;
    if (la == 0 || lb == 0 || n == 0) return;
    const size_t xa = la < n ? la : n, xb = lb < n ? lb : n;
    if (xa > SIZE_MAX - (xb - 1)) throw Error{FPX_ELENGTH, "poly::conv: result length overflows size_t"};
    const size_t outn = (xa + xb - 1) < n ? xa + xb - 1 : n;
    check_ptr(out, outn, "out");
    Buf da = upload(e, p, a, xa, repr);
    Buf db;
    const uint32_t* pb = da.get();
    if (!(a == b && xa == xb)) {
      db = upload(e, p, b, xb, repr);
      pb = db.get();
    }
    Buf dout(&e.pool(), outn);
    const size_t got = e.conv(p, da.get(), xa, pb, xb, n, dout.get());
    download(e, p, out, dout.get(), got, repr);
    *out_len = got;
  });
}

int fpx_conv_device(fpx_ctx* ctx, uint32_t p, const uint32_t* d_a, size_t la, const uint32_t* d_b, size_t lb,
                    size_t n, uint32_t* d_out, size_t* out_len) {
  return guarded(ctx, [&](fpx::Engine& e) {
    check_modulus(p);
    check_ptr(d_a, la, "a");
    check_ptr(d_b, lb, "b");
    if (!out_len) throw Error{FPX_EINVAL, "null out_len"};
    *out_len = 0;
    *out_len = e.conv(p, d_a, la, d_b, lb, n, d_out);
  });
}

int fpx_inv(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out, int repr) {
  return series_host(ctx, &fpx::Engine::inv, p, a, la, n, out, repr);
}
int fpx_log(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out, int repr) {
  return series_host(ctx, &fpx::Engine::log, p, a, la, n, out, repr);
}
int fpx_exp(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out, int repr) {
  return series_host(ctx, &fpx::Engine::exp, p, a, la, n, out, repr);
}
int fpx_sqrt(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, size_t n, uint32_t* out, int repr) {
  return guarded(ctx, [&](fpx::Engine& e) {
    check_modulus(p);
    check_repr(repr);
    check_ptr(a, la, "a");
    check_ptr(out, n, "out");
    if (n == 0) return;
    // sqrt reads coefficients up to the valuation plus n, so keep the whole input
    Buf da = upload(e, p, a, la, repr);
    Buf dout(&e.pool(), n);
    e.sqrt(p, da.get(), la, n, dout.get());
    download(e, p, out, dout.get(), n, repr);
  });
}
int fpx_pow(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, uint64_t k, size_t n, uint32_t* out, int repr) {
  return guarded(ctx, [&](fpx::Engine& e) {
    check_modulus(p);
    check_repr(repr);
    check_ptr(a, la, "a");
    check_ptr(out, n, "out");
    if (n == 0) return;
    Buf da = upload(e, p, a, la, repr);
    Buf dout(&e.pool(), n);
    e.pow(p, da.get(), la, k, n, dout.get());
    download(e, p, out, dout.get(), n, repr);
  });
}

int fpx_inv_device(fpx_ctx* ctx, uint32_t p, const uint32_t* d_a, size_t la, size_t n, uint32_t* d_out) {
  return series_dev(ctx, &fpx::Engine::inv, p, d_a, la, n, d_out);
}
int fpx_log_device(fpx_ctx* ctx, uint32_t p, const uint32_t* d_a, size_t la, size_t n, uint32_t* d_out) {
  return series_dev(ctx, &fpx::Engine::log, p, d_a, la, n, d_out);
}
int fpx_exp_device(fpx_ctx* ctx, uint32_t p, const uint32_t* d_a, size_t la, size_t n, uint32_t* d_out) {
  return series_dev(ctx, &fpx::Engine::exp, p, d_a, la, n, d_out);
}
int fpx_sqrt_device(fpx_ctx* ctx, uint32_t p, const uint32_t* d_a, size_t la, size_t n, uint32_t* d_out) {
  return guarded(ctx, [&](fpx::Engine& e) {
    check_modulus(p);
    check_ptr(d_a, la, "a");
    check_ptr(d_out, n, "out");
    e.sqrt(p, d_a, la, n, d_out);
  });
}
int fpx_pow_device(fpx_ctx* ctx, uint32_t p, const uint32_t* d_a, size_t la, uint64_t k, size_t n,
                   uint32_t* d_out) {
  return guarded(ctx, [&](fpx::Engine& e) {
    check_modulus(p);
    check_ptr(d_a, la, "a");
    check_ptr(d_out, n, "out");
    e.pow(p, d_a, la, k, n, d_out);
  });
}

static int divmod_host(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb,
                       uint32_t* q, size_t* q_len, uint32_t* r, size_t* r_len, int repr, bool want_q, bool want_r) {
  return guarded(ctx, [&](fpx::Engine& e) {
    check_modulus(p);
    check_repr(repr);
    check_ptr(a, la, "a");
    check_ptr(b, lb, "b");
    if (want_q && !q_len) throw Error{FPX_EINVAL, "null q_len"};
    if (want_r && !r_len) throw Error{FPX_EINVAL, "null r_len"};
    if (want_q) *q_len = 0;
    if (want_r) *r_len = 0;
    Buf da = upload(e, p, a, la, repr), db = upload(e, p, b, lb, repr);
    Buf dq(&e.pool(), la ? la : 1), dr(&e.pool(), lb ? lb : 1);
    size_t lq = 0, lr = 0;
    e.divmod(p, da.get(), la, db.get(), lb, dq.get(), &lq, dr.get(), &lr, want_q, want_r);
    if (want_q) {
      check_ptr(q, lq, "q");
      if (repr == FPX_REPR_MONTGOMERY && lq) e.check(fpx::launch_to_mont(p, dq.get(), dq.get(), lq, e.stream()), "repr");
      e.to_host(q, dq.get(), lq);
    }
    if (want_r) {
      check_ptr(r, lr, "r");
      if (repr == FPX_REPR_MONTGOMERY && lr) e.check(fpx::launch_to_mont(p, dr.get(), dr.get(), lr, e.stream()), "repr");
      e.to_host(r, dr.get(), lr);
    }
    e.sync();
    if (want_q) *q_len = lq;
    if (want_r) *r_len = lr;
  });
}

int fpx_divmod(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, uint32_t* q,
               size_t* q_len, uint32_t* r, size_t* r_len, int repr) {
  return divmod_host(ctx, p, a, la, b, lb, q, q_len, r, r_len, repr, true, true);
}
int fpx_div(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, uint32_t* q,
            size_t* q_len, int repr) {
  return divmod_host(ctx, p, a, la, b, lb, q, q_len, nullptr, nullptr, repr, true, false);
}
int fpx_mod(fpx_ctx* ctx, uint32_t p, const uint32_t* a, size_t la, const uint32_t* b, size_t lb, uint32_t* r,
            size_t* r_len, int repr) {
  return divmod_host(ctx, p, a, la, b, lb, nullptr, nullptr, r, r_len, repr, false, true);
}

// ---- batches

int fpx_batch_submit(fpx_ctx* ctx, fpx_job* jobs, size_t count) {
  if (count && !jobs) return FPX_EINVAL;
  const int rc = guarded(ctx, [&](fpx::Engine& e) { e.batch(jobs, count); });
  if (rc != FPX_OK) return rc;
  for (size_t i = 0; i < count; ++i)
    if (jobs[i].status != FPX_OK) {
      ctx->err = "job " + std::to_string(i) + " failed with status " + std::to_string(jobs[i].status);
      return jobs[i].status;
    }
  return FPX_OK;
}

int fpx_batch_wait(fpx_ctx* ctx) { return fpx_ctx_synchronize(ctx); }

int fpx_batch_run(fpx_ctx* ctx, fpx_job* jobs, size_t count, int repr) {
  if (count && !jobs) return FPX_EINVAL;
  const int rc = guarded(ctx, [&](fpx::Engine& e) {
    check_repr(repr);
    e.batch_host(jobs, count, repr);
  });
  if (rc != FPX_OK) return rc;
  for (size_t i = 0; i < count; ++i)
    if (jobs[i].status != FPX_OK) {
      ctx->err = "job " + std::to_string(i) + " failed with status " + std::to_string(jobs[i].status);
      return jobs[i].status;
    }
  return FPX_OK;
}

}  // extern "C"
