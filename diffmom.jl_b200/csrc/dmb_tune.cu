// dmb_tune.cu -- online autotuner of launch shapes.
//
// A tuned launch site asks for a candidate with tune_choose and brackets the
// launch with tune_begin / tune_end (CUDA events on the context stream).  Per
// (device, family, shape bucket) each candidate is run on the first real
// calls until it has TUNE_SAMPLES timings -- no extra work, no host
// synchronisation: finished event pairs are read when they have completed --
// and from then on the fastest (minimum time) is used for the rest of the
// process.  The candidates of a family differ only in how the work is cut
// into CTAs or pipelined (tile width, pipeline depth), never in the order of
// the arithmetic of an output element, so every candidate writes the same
// bits; DMB_OPT_TUNE_* options pin one candidate (tests compare them).
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <sstream>
#include <tuple>
#include <vector>

#include "dmb_internal.h"

namespace {

constexpr int TUNE_SAMPLES = 2;

struct TuneEntry {
  int ncand = 0;
  std::vector<float> best_ms;   // per candidate, min over samples
  std::vector<int> samples;     // per candidate
  int chosen = -1;
  struct Pending {
    int cand;
    cudaEvent_t e0, e1;
  };
  std::vector<Pending> pending;
};

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int64_t, int64_t>, TuneEntry> g_tune;
std::map<int, std::vector<cudaEvent_t>> g_tune_events;  // recycled, per device

cudaEvent_t take_event(int device) {
  auto &pool = g_tune_events[device];
  if (!pool.empty()) {
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  DMB_CUDA(cudaEventCreate(&e));
  return e;
}

// fold finished measurements into the entry (caller holds the mutex)
void poll(int device, TuneEntry &en) {
  for (size_t i = 0; i < en.pending.size();) {
    auto &p = en.pending[i];
    if (cudaEventQuery(p.e1) != cudaSuccess) {
      i++;
      continue;
    }
    float ms = 0;
    if (cudaEventElapsedTime(&ms, p.e0, p.e1) == cudaSuccess) {
      float &b = en.best_ms[p.cand];
      b = en.samples[p.cand] == 0 ? ms : std::min(b, ms);
      en.samples[p.cand]++;
    }
    g_tune_events[device].push_back(p.e0);
    g_tune_events[device].push_back(p.e1);
    en.pending.erase(en.pending.begin() + i);
  }
  if (en.chosen >= 0) return;
  for (int k = 0; k < en.ncand; k++)
    if (en.samples[k] < TUNE_SAMPLES) return;
  int best = 0;
  for (int k = 1; k < en.ncand; k++)
    if (en.best_ms[k] < en.best_ms[best]) best = k;
  en.chosen = best;
}

TuneEntry &entry(int device, int family, int64_t b1, int64_t b2, int ncand) {
  TuneEntry &en = g_tune[std::make_tuple(device, family, b1, b2)];
  if (en.ncand == 0) {
    en.ncand = ncand;
    en.best_ms.assign(ncand, 0.f);
    en.samples.assign(ncand, 0);
  }
  return en;
}

const char *family_name(int f) {
  switch (f) {
    case dmb::TUNE_TC_GEMM_BN: return "k_tc_gemm shape (256 / 128 complex columns per tile / persistent 256)";
    case dmb::TUNE_TC_SYRK_STAGES:
      return "k_tc_syrk schedule (4 stages, 1 CTA/SM / 2 stages, 2 CTAs/SM / persistent, lower tiles only)";
    case dmb::TUNE_OZ_TILE: return "k_oz_gemm tile (one SM, 64 x 256 complex / CTA pair, 128 x 256 complex)";
    default: return "?";
  }
}

}  // namespace

namespace dmb {

int64_t tune_bucket(int64_t v) {
  int64_t b = 0;
  while (((int64_t)1 << (b + 1)) <= v) b++;
  return b;
}

int tune_choose(dmb_ctx *c, int family, int64_t b1, int64_t b2, int ncand) {
  const int pin = c->tune_pin[family];
  if (pin > 0) return std::min(pin, ncand) - 1;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  TuneEntry &en = entry(c->device, family, b1, b2, ncand);
  poll(c->device, en);
  if (en.chosen >= 0) return en.chosen;
  // the candidate with the fewest samples (finished or in flight)
  std::vector<int> n(en.samples);
  for (auto &p : en.pending) n[p.cand]++;
  int k = 0;
  for (int i = 1; i < ncand; i++)
    if (n[i] < n[k]) k = i;
  return k;
}

// bracket one launch of candidate `cand` (only while the bucket is measured)
bool tune_begin(dmb_ctx *c, int family, int64_t b1, int64_t b2, int cand, TuneMark &mk) {
  mk.active = false;
  if (c->tune_pin[family] > 0) return false;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(std::make_tuple(c->device, family, b1, b2));
  if (it == g_tune.end() || it->second.chosen >= 0) return false;
  mk.e0 = take_event(c->device);
  mk.e1 = take_event(c->device);
  DMB_CUDA(cudaEventRecord(mk.e0, c->stream));
  mk.active = true;
  mk.family = family;
  mk.b1 = b1;
  mk.b2 = b2;
  mk.cand = cand;
  return true;
}

void tune_end(dmb_ctx *c, TuneMark &mk) {
  if (!mk.active) return;
  DMB_CUDA(cudaEventRecord(mk.e1, c->stream));
  std::lock_guard<std::mutex> lk(g_tune_mu);
  TuneEntry &en = g_tune[std::make_tuple(c->device, mk.family, mk.b1, mk.b2)];
  en.pending.push_back({mk.cand, mk.e0, mk.e1});
  mk.active = false;
}

std::string tune_report() {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  std::ostringstream os;
  for (auto &kv : g_tune) {
    poll(std::get<0>(kv.first), kv.second);
    const TuneEntry &en = kv.second;
    os << "device " << std::get<0>(kv.first) << " | " << family_name(std::get<1>(kv.first)) << " | bucket ("
       << std::get<2>(kv.first) << ", " << std::get<3>(kv.first) << ") | ms";
    for (int k = 0; k < en.ncand; k++) os << " " << (en.samples[k] ? en.best_ms[k] : NAN);
    os << " | chosen " << en.chosen << "\n";
  }
  return os.str();
}

}  // namespace dmb
