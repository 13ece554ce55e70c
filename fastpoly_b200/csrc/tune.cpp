// tune.cpp - tile shapes of the column passes, chosen by measurement.
//
// A two-pass transform of N = R x C points runs its column passes as a grid of
// tiles of 2^LW columns, and 148 SMs never divide the power-of-two tile count:
// with the default width the last wave of a 2^23-point transform's inverse
// column pass holds 68 tiles on 148 SMs, and those SMs run one CTA each while
// the other 80 idle.  Narrower tiles, or a grid whose wide tiles fill whole
// waves and whose remaining columns go in narrow tiles, shorten that tail, at
// the price of shorter row segments per tile.  Which wins depends on R and on
// the pass, so every compiled shape is timed once per process, device and size
// (CUDA events on the engine's stream, best of three rounds of four launches)
// and the fastest kept when it beats the default by more than 3 %.
//
// FPX_AUTOTUNE=0 keeps the default shapes.  FPX_AUTOTUNE_CACHE=<file> keeps the
// choices across processes: one line per (device name, SM count, log2 N).
// The shape never changes the results, only the time.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>

#include "engine.h"
#include "fpx_b200.h"
#include "kernels.h"

namespace fpx {
namespace {

constexpr int kMaxCand = 8;
// Shapes do not depend on the prime; a size's store entry is made through a plan
// of this one, which has roots of unity of every order up to 2^26.
constexpr uint32_t kPlanPrime = 469762049u;

struct ShapeStore {
  std::mutex mu;
  std::map<std::pair<int, int>, std::unique_ptr<ColShapes>> by_size;  // (device, logN)
  bool file_loaded = false;
  std::map<std::string, std::string> file;  // key -> "lw1,lw2,split lw1,lw2,split lw1,lw2,split"
};
ShapeStore& store() {
  static ShapeStore s;
  return s;
}

bool tunable(const BigTables& bt) { return bt.logC == 12 && bt.logR >= 2 && bt.logR <= 12; }

bool autotune_on() {
  const char* e = std::getenv("FPX_AUTOTUNE");
  return !(e && e[0] == '0');
}

std::string device_key(int dev, int logN) {
  cudaDeviceProp prop{};
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
    cudaGetLastError();
    return std::string();
  }
  char buf[512];
  std::snprintf(buf, sizeof buf, "%s|sm%d|logN%d", prop.name, prop.multiProcessorCount, logN);
  std::string s = buf;
  for (char& c : s)
    if (c == ' ' || c == '\t') c = '_';
  return s;
}

void load_file(ShapeStore& st) {
  if (st.file_loaded) return;
  st.file_loaded = true;
  const char* path = std::getenv("FPX_AUTOTUNE_CACHE");
  if (!path || !*path) return;
  FILE* f = std::fopen(path, "r");
  if (!f) return;
  char buf[1024];
  while (std::fgets(buf, sizeof buf, f)) {
    std::string line = buf;
    while (!line.empty() && (line.back() == '\n' || line.back() == '\r')) line.pop_back();
    const size_t t = line.find('\t');
    if (t != std::string::npos) st.file[line.substr(0, t)] = line.substr(t + 1);
  }
  std::fclose(f);
}

void save_line(const std::string& key, const std::string& val) {
  const char* path = std::getenv("FPX_AUTOTUNE_CACHE");
  if (!path || !*path || key.empty()) return;
  FILE* f = std::fopen(path, "a");
  if (!f) return;
  std::fprintf(f, "%s\t%s\n", key.c_str(), val.c_str());
  std::fclose(f);
}

std::string shape_text(const ColShape& s) {
  return std::to_string(s.lw1) + "," + std::to_string(s.lw2) + "," + std::to_string(s.split);
}

// The candidate of `cands` with the same widths and split as `want` (slots from
// this device), or the default.
ColShape match(const ColShape* cands, int n, int lw1, int lw2, int split) {
  for (int i = 0; i < n; ++i)
    if (cands[i].lw1 == lw1 && cands[i].lw2 == lw2 && cands[i].split == split) return cands[i];
  return cands[0];
}

}  // namespace

const ColShapes* Engine::tuned_shapes_locked(uint32_t p, const BigTables& bt) {
  ShapeStore& st = store();
  std::lock_guard<std::mutex> g(st.mu);
  const auto key = std::make_pair(device_, bt.logN);
  auto it = st.by_size.find(key);
  if (it != st.by_size.end()) return it->second.get();
  auto shapes = std::make_unique<ColShapes>();  // defaults
  if (tunable(bt) && autotune_on()) {
    ColShape cf[kMaxCand], ci[kMaxCand];
    const int nf = fpx::col_shape_candidates(bt.logR, false, cf, kMaxCand);
    const int ni = fpx::col_shape_candidates(bt.logR, true, ci, kMaxCand);
    load_file(st);
    const std::string fkey = device_key(device_, bt.logN);
    auto fit = st.file.find(fkey);
    int v[9];
    if (nf > 0 && ni > 0 && fit != st.file.end() &&
        std::sscanf(fit->second.c_str(), "%d,%d,%d %d,%d,%d %d,%d,%d", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5],
                    &v[6], &v[7], &v[8]) == 9) {
      shapes->fwd1 = match(cf, nf, v[0], v[1], v[2]);
      shapes->fwd2 = match(cf, nf, v[3], v[4], v[5]);
      shapes->inv = match(ci, ni, v[6], v[7], v[8]);
    } else if (nf > 1 || ni > 1) {
      try {
        const PrimeTables& pt = prime_plan_locked(p).t;
        const size_t N = size_t(1) << bt.logN;
        Buf in0(&pool_, N / 2), in1(&pool_, N / 2), t1(&pool_, N), t2(&pool_, N), out(&pool_, N);
        for (const Buf* b : {&in0, &in1})
          check(cudaMemsetAsync(b->get(), 0, N / 2 * 4, stream_), "tune memset");
        for (const Buf* b : {&t1, &t2, &out}) check(cudaMemsetAsync(b->get(), 0, N * 4, stream_), "tune memset");
        cudaEvent_t e0, e1;
        check(cudaEventCreate(&e0), "tune event");
        check(cudaEventCreate(&e1), "tune event");
        ColShapes trial;
        BigTables b2 = bt;
        b2.shapes = &trial;
        // best of three rounds of four launches; +inf if the shape does not launch
        auto time_of = [&](auto&& launch) -> float {
          float best = 1e30f;
          for (int w = 0; w < 2; ++w)
            if (launch() != cudaSuccess) {
              cudaGetLastError();
              return 1e30f;
            }
          for (int r = 0; r < 3; ++r) {
            check(cudaEventRecord(e0, stream_), "tune event");
            for (int k = 0; k < 4; ++k) check(launch(), "tune launch");
            check(cudaEventRecord(e1, stream_), "tune event");
            check(cudaEventSynchronize(e1), "tune sync");
            float ms = 0;
            check(cudaEventElapsedTime(&ms, e0, e1), "tune time");
            if (ms < best) best = ms;
          }
          return best;
        };
        auto pick = [&](const ColShape* c, int n, ColShape& slot, auto&& launch) {
          float t0 = 0, tb = 1e30f;
          int bi = 0;
          for (int i = 0; i < n; ++i) {
            slot = c[i];
            const float t = time_of(launch);
            if (i == 0) t0 = t;
            if (t < tb) tb = t, bi = i;
          }
          slot = tb < 0.97f * t0 ? c[bi] : c[0];
          return slot;
        };
        const InOp ins[2] = {InOp{in0.get(), (uint32_t)(N / 2), 0}, InOp{in1.get(), (uint32_t)(N / 2), 0}};
        uint32_t* outs[2] = {t1.get(), t2.get()};
        Epi epi;
        epi.out = out.get();
        epi.lo = 0;
        epi.hi = (uint32_t)N;
        shapes->fwd2 = pick(cf, nf, trial.fwd2, [&] { return launch_colfwd(pt, b2, 2, ins, outs, stream_); });
        shapes->fwd1 = pick(cf, nf, trial.fwd1, [&] { return launch_colfwd(pt, b2, 1, ins, outs, stream_); });
        shapes->inv = pick(ci, ni, trial.inv, [&] { return launch_colinv(pt, b2, t1.get(), 1, epi, stream_); });
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        save_line(fkey, shape_text(shapes->fwd1) + " " + shape_text(shapes->fwd2) + " " + shape_text(shapes->inv));
      } catch (const Error&) {
        // no memory for the trial buffers (pool limit) or a failed launch:
        // keep the defaults for this process
        cudaGetLastError();
        *shapes = ColShapes{};
      }
    }
  }
  const ColShapes* r = shapes.get();
  st.by_size[key] = std::move(shapes);
  return r;
}

namespace {
ColShape& kind_slot(ColShapes& s, int kind) { return kind == 0 ? s.fwd1 : (kind == 1 ? s.fwd2 : s.inv); }
const ColShape& kind_slot(const ColShapes& s, int kind) { return kind == 0 ? s.fwd1 : (kind == 1 ? s.fwd2 : s.inv); }
void check_size(int logN, int kind) {
  if (logN < 14 || logN > 25 || kind < 0 || kind > 2) throw Error{FPX_EINVAL, "no column pass for this size / kind"};
}
}  // namespace

ColShape Engine::col_shape(int logN, int kind) {
  check_size(logN, kind);
  const BigTables& bt = big_plan(kPlanPrime, logN).t;  // tunes on first use
  return bt.shapes ? kind_slot(*bt.shapes, kind) : ColShape{};
}

int Engine::col_shape_candidates(int logN, int kind, ColShape* out, int max) {
  check_size(logN, kind);
  const int logC = logN >= 25 ? 13 : 12;
  return fpx::col_shape_candidates(logN - logC, kind == 2, out, max);
}

void Engine::set_col_shape(int logN, int kind, const ColShape& sh) {
  ColShape c[kMaxCand];
  const int n = col_shape_candidates(logN, kind, c, kMaxCand);
  bool found = false;
  ColShape chosen;
  for (int i = 0; i < n; ++i)
    if ((c[i].lw1 == sh.lw1 && c[i].lw2 == sh.lw2 && c[i].split == sh.split) ||
        (i == 0 && sh.lw1 == 0)) {
      chosen = c[i];
      found = true;
      break;
    }
  if (!found) throw Error{FPX_EINVAL, "column shape not compiled for this size"};
  big_plan(kPlanPrime, logN);  // the store entry exists from here on
  ShapeStore& st = store();
  std::lock_guard<std::mutex> g(st.mu);
  auto it = st.by_size.find(std::make_pair(device_, logN));
  if (it == st.by_size.end()) throw Error{FPX_EINVAL, "no column pass for this size"};
  kind_slot(*it->second, kind) = chosen;
}

}  // namespace fpx
