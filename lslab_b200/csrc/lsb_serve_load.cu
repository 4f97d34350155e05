// Open-loop load generator for the serving loop (lsb_serve_run_load): host
// code only, on the public C-ABI.  The calling thread issues requests at
// their scheduled times; a second thread takes results in FIFO order and
// records each request's latency from its scheduled arrival, so queueing
// delay on the host (a full queue) counts against latency as it would for a
// real client.
#include <pthread.h>
#include <sched.h>

#include <atomic>
#include <chrono>
#include <thread>
#include <vector>

#include "lsb.h"

namespace {
using Clock = std::chrono::steady_clock;

// longest wait for one request before the run is abandoned
constexpr uint64_t kWaitLimitNs = 30ull * 1000 * 1000 * 1000;

// The two busy threads each get a core of their own (the last two CPUs the
// process may use), so a scheduler migration does not stall a request.
inline void pin_to(int nth_from_last) {
  cpu_set_t set;
  if (sched_getaffinity(0, sizeof(set), &set) != 0) return;
  int seen = 0;
  for (int c = CPU_SETSIZE - 1; c >= 0; --c) {
    if (!CPU_ISSET(c, &set)) continue;
    if (seen++ == nth_from_last) {
      cpu_set_t one;
      CPU_ZERO(&one);
      CPU_SET(c, &one);
      pthread_setaffinity_np(pthread_self(), sizeof(one), &one);
      return;
    }
  }
}

inline uint64_t ns_since(Clock::time_point t0) {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now() - t0).count();
}
}  // namespace

extern "C" int lsb_serve_run_load(lsb_server* s, const lsb_serve_load* ld, uint64_t* latency_ns,
                                  uint64_t* wall_ns) {
  if (!s || !ld || !latency_ns || !ld->arrival_ns || !ld->pool_index || !ld->pool_off ||
      !ld->pool_n || !ld->keys || ld->pool_size == 0)
    return LSB_ERR_ARG;
  const uint64_t nreq = ld->nreq;
  for (uint64_t i = 0; i < nreq; ++i)
    if (ld->pool_index[i] >= ld->pool_size) return LSB_ERR_ARG;
  // first op of each issued request in `results`
  std::vector<uint64_t> res_off;
  if (ld->results) {
    res_off.resize(nreq);
    uint64_t o = 0;
    for (uint64_t i = 0; i < nreq; ++i) {
      res_off[i] = o;
      o += ld->pool_n[ld->pool_index[i]];
    }
  }
  std::vector<uint64_t> tickets(nreq, ~0ull);
  std::atomic<uint64_t> issued{0};
  std::atomic<int> error{LSB_OK};
  const Clock::time_point t0 = Clock::now();

  cpu_set_t saved;
  const bool have_saved = pthread_getaffinity_np(pthread_self(), sizeof(saved), &saved) == 0;
  std::thread taker([&] {
    pin_to(1);
    for (uint64_t i = 0; i < nreq; ++i) {
      while (issued.load(std::memory_order_acquire) <= i) {
        if (error.load() != LSB_OK) return;
        std::this_thread::yield();
      }
      const uint64_t t = tickets[i];
      int done = 0;
      const uint64_t wait_from = ns_since(t0);
      for (;;) {
        lsb_serve_poll(s, t, &done);
        if (done) break;
        if (error.load() != LSB_OK) return;
        if (ns_since(t0) - wait_from > kWaitLimitNs) {  // the loop is gone
          error.store(LSB_ERR_TIMEOUT);
          return;
        }
      }
      const uint64_t now = ns_since(t0);
      latency_ns[i] = now > ld->arrival_ns[i] ? now - ld->arrival_ns[i] : 0;
      int st = 0;
      const int rc = lsb_serve_take(s, t, ld->results ? ld->results + res_off[i] : nullptr, &st);
      if (rc != LSB_OK) {
        error.store(rc);
        return;
      }
    }
  });

  pin_to(0);
  for (uint64_t i = 0; i < nreq && error.load() == LSB_OK; ++i) {
    while (ns_since(t0) < ld->arrival_ns[i]) {
    }
    const uint32_t p = ld->pool_index[i];
    const uint64_t off = ld->pool_off[p];
    uint64_t ticket = 0;
    const uint64_t tried_from = ns_since(t0);
    for (;;) {
      const int rc = lsb_serve_submit(s, ld->types ? ld->types + off : nullptr, ld->keys + off,
                                      ld->vals ? ld->vals + off : nullptr, ld->pool_n[p], &ticket);
      if (rc == LSB_OK) break;
      if (rc != LSB_ERR_STATE) {
        error.store(rc);
        break;
      }
      // queue full: the taker frees slots, unless it gave up or the loop
      // stopped completing requests
      if (error.load() != LSB_OK) break;
      if (ns_since(t0) - tried_from > kWaitLimitNs) {
        error.store(LSB_ERR_TIMEOUT);
        break;
      }
      std::this_thread::yield();
    }
    if (error.load() != LSB_OK) break;
    tickets[i] = ticket;
    issued.store(i + 1, std::memory_order_release);
  }
  taker.join();
  if (wall_ns) *wall_ns = ns_since(t0);
  if (have_saved) pthread_setaffinity_np(pthread_self(), sizeof(saved), &saved);
  return error.load();
}
