// Error state and host-side FFT factorisation shared by all qe_b200 kernels.
#include <atomic>
#include <cstdarg>
#include <cstring>

#include "qeb_common.cuh"
#include "../../include/qe_b200.h"

namespace qeb {

static thread_local char g_last_error[512] = "";

void set_error(const char* fmt, ...) {
  va_list args;
  va_start(args, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, args);
  va_end(args);
}

int cuda_status(cudaError_t err, const char* where) {
  if (err == cudaSuccess) return QEB_OK;
  set_error("%s: %s", where, cudaGetErrorString(err));
  return QEB_ECUDA;
}

static std::atomic<int64_t> g_launches{0};

void count_launches(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

bool make_fft_desc(int n, FftDesc* d) {
  if (n < 1 || n > 1024) return false;
  d->n = n;
  d->nstages = 0;
  int rest = n;
  // Radix 4 first (cheapest butterfly per point), then 2, 3, 5.
  const int order[4] = {4, 2, 3, 5};
  for (int i = 0; i < 4; ++i) {
    const int r = order[i];
    while (rest % r == 0) {
      if (d->nstages >= kMaxStages) return false;
      d->radix[d->nstages++] = r;
      rest /= r;
    }
  }
  if (n == 1) {
    d->nstages = 0;
  }
  return rest == 1;
}

}  // namespace qeb

extern "C" const char* qeb_last_error(void) { return qeb::g_last_error; }

extern "C" int qeb_version(void) { return QEB_ABI_VERSION; }

extern "C" int64_t qeb_launch_count(void) { return qeb::g_launches.load(); }

// QE randy stream (a 97-entry shuffle table over the LCG
// seed <- (1366 seed + 150889) mod 714025), drawn in band-outer,
// plane-wave-inner order as (amplitude, phase) pairs; host code.
// Same recurrence as qepy_pw/_native_fft.pyx qe_random_pairs (:1411-1444).
extern "C" int qeb_qe_random_pairs(int64_t plane_waves, int64_t bands, int64_t* table,
                                   int64_t* current, int64_t* seed, double* first,
                                   double* second) {
  if (plane_waves < 0 || bands < 0 || table == nullptr || current == nullptr ||
      seed == nullptr || (plane_waves * bands > 0 && (first == nullptr || second == nullptr))) {
    qeb::set_error("qe_random_pairs: invalid arguments");
    return QEB_EINVAL;
  }
  int64_t cur = *current, s = *seed;
  for (int64_t b = 0; b < bands; ++b) {
    for (int64_t g = 0; g < plane_waves; ++g) {
      const int64_t out = g + b * plane_waves;
      int64_t i = (97 * cur) / 714025;
      cur = table[i];
      first[out] = (double)cur / 714025.0;
      s = (1366 * s + 150889) % 714025;
      table[i] = s;
      i = (97 * cur) / 714025;
      cur = table[i];
      second[out] = (double)cur / 714025.0;
      s = (1366 * s + 150889) % 714025;
      table[i] = s;
    }
  }
  *current = cur;
  *seed = s;
  return QEB_OK;
}

// The same stream as integers: first/second receive the raw table values
// (the draws times 714025), so the division happens where the draws are
// used (on the device, in qeb_random_trials).  Every quantity fits 32 bits
// (97 x 714024 and 1366 x 714024 + 150889 are below 2^32), so the two
// dependency chains (the shuffle index and the LCG) run on 32-bit integer
// arithmetic, and the output is half the bytes of the double pairs.
extern "C" int qeb_qe_random_draws(int64_t plane_waves, int64_t bands, int64_t* table,
                                   int64_t* current, int64_t* seed, int32_t* first,
                                   int32_t* second) {
  if (plane_waves < 0 || bands < 0 || table == nullptr || current == nullptr ||
      seed == nullptr || (plane_waves * bands > 0 && (first == nullptr || second == nullptr))) {
    qeb::set_error("qe_random_draws: invalid arguments");
    return QEB_EINVAL;
  }
  if (*current < 0 || *current >= 714025 || *seed < 0 || *seed >= 714025) {
    qeb::set_error("qe_random_draws: stream state out of range");
    return QEB_EINVAL;
  }
  uint32_t shuffle[97];
  for (int i = 0; i < 97; ++i) {
    if (table[i] < 0 || table[i] >= 714025) {
      qeb::set_error("qe_random_draws: shuffle table out of range");
      return QEB_EINVAL;
    }
    shuffle[i] = (uint32_t)table[i];
  }
  uint32_t cur = (uint32_t)*current, s = (uint32_t)*seed;
  const int64_t total = plane_waves * bands;
  for (int64_t out = 0; out < total; ++out) {
    uint32_t i = (97u * cur) / 714025u;
    cur = shuffle[i];
    s = (1366u * s + 150889u) % 714025u;
    shuffle[i] = s;
    first[out] = (int32_t)cur;
    i = (97u * cur) / 714025u;
    cur = shuffle[i];
    s = (1366u * s + 150889u) % 714025u;
    shuffle[i] = s;
    second[out] = (int32_t)cur;
  }
  for (int i = 0; i < 97; ++i) table[i] = shuffle[i];
  *current = cur;
  *seed = s;
  return QEB_OK;
}
