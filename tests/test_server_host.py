"""CPU tests of the request server's host logic: the first-fit range allocator
behind its particle-slot and curve-staging arenas, compiled on its own and
checked against a slot-by-slot model (no GPU needed)."""
import shutil
import subprocess
from pathlib import Path

import pytest

CSRC = Path(__file__).resolve().parent.parent / "dpa_b200" / "csrc"

DRIVER = r"""
#include <cstdio>
#include <random>
#include <vector>
#include "range_allocator.hpp"

// The model: one flag per entry. allocate must return the lowest offset
// starting n free entries, or fail when no such run exists; release must make
// the range whole again (adjacent free ranges merge).
static bool fits_at(const std::vector<char>& used, uint64_t at, uint64_t n) {
  for (uint64_t i = at; i < at + n; ++i) if (used[i]) return false;
  return true;
}
static long lowest_fit(const std::vector<char>& used, uint64_t n) {
  for (uint64_t at = 0; at + n <= used.size(); ++at) if (fits_at(used, at, n)) return long(at);
  return -1;
}

int main() {
  for (unsigned seed = 0; seed < 40; ++seed) {
    std::mt19937_64 rng(seed);
    const uint64_t capacity = 1 + rng() % 400;
    dpa::range_allocator a(capacity);
    std::vector<char> used(capacity, 0);
    std::vector<std::pair<uint64_t, uint64_t>> live;
    for (int op = 0; op < 3000; ++op) {
      if (live.empty() || rng() % 5 < 3) {
        const uint64_t n = rng() % (capacity / 3 + 2);
        uint64_t at = 0;
        const bool ok = a.allocate(n, &at);
        const long want = n == 0 ? 0 : lowest_fit(used, n);
        if (ok != (want >= 0) || (ok && long(at) != want)) {
          std::printf("seed %u op %d: allocate(%llu) gave %d at %llu, model %ld\n", seed, op,
                      (unsigned long long)n, int(ok), (unsigned long long)at, want);
          return 1;
        }
        if (ok && n) {
          for (uint64_t i = at; i < at + n; ++i) used[i] = 1;
          live.push_back({at, n});
        }
      } else {
        const size_t k = rng() % live.size();
        a.release(live[k].first, live[k].second);
        for (uint64_t i = live[k].first; i < live[k].first + live[k].second; ++i) used[i] = 0;
        live.erase(live.begin() + long(k));
      }
      // Free ranges are maximal and match the model exactly.
      uint64_t expect = 0;
      long prev_end = -1;
      for (const auto& r : a.free_ranges()) {
        if (long(r.first) == prev_end || r.second == 0) {
          std::printf("seed %u op %d: free ranges not merged at %llu\n", seed, op,
                      (unsigned long long)r.first);
          return 1;
        }
        for (uint64_t i = r.first; i < r.first + r.second; ++i) {
          if (i >= capacity || used[i]) {
            std::printf("seed %u op %d: entry %llu free in the allocator, used in the model\n",
                        seed, op, (unsigned long long)i);
            return 1;
          }
        }
        expect += r.second;
        prev_end = long(r.first + r.second);
      }
      uint64_t model_free = 0;
      for (char u : used) model_free += !u;
      if (expect != model_free) {
        std::printf("seed %u op %d: %llu free in the allocator, %llu in the model\n", seed, op,
                    (unsigned long long)expect, (unsigned long long)model_free);
        return 1;
      }
    }
    for (const auto& r : live) a.release(r.first, r.second);
    uint64_t at = 1;
    if (!a.allocate(capacity, &at) || at != 0) {
      std::printf("seed %u: the emptied arena does not hold its capacity\n", seed);
      return 1;
    }
  }
  std::puts("ok");
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_range_allocator_is_first_fit_and_merges_free_ranges(tmp_path):
    src = tmp_path / "driver.cpp"
    exe = tmp_path / "driver"
    src.write_text(DRIVER)
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", str(CSRC), str(src), "-o", str(exe)],
                   check=True)
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0 and run.stdout.strip() == "ok", run.stdout + run.stderr


ADMISSION_DRIVER = r"""
#include <cstdio>
#include <deque>
#include <vector>
#include "admission.hpp"
#include "range_allocator.hpp"

struct req { int id; uint64_t seeds; double queued; };

// Runs one admission scan at time `now` over `q` with `free_slots` free (of
// `capacity`, allocated first fit) and returns the admitted ids in order.
static std::vector<int> scan(std::deque<req>& q, const dpa::admission_config& c, uint64_t used,
                             double now, int counters = 1000, uint64_t small = 0) {
  dpa::range_allocator slots(c.slot_capacity);
  uint64_t at = 0;
  if (used) slots.allocate(used, &at);
  std::vector<int> got;
  dpa::admit_waiting(
      q, c, used, small, [](const req& r) { return r.seeds; },
      [&](const req& r) { return now - r.queued; },
      [&](const req& r) { uint64_t o; return slots.allocate(r.seeds, &o); },
      [&](req& r) { got.push_back(r.id); --counters; }, [&] { return counters > 0; });
  return got;
}

static int fail(const char* what) { std::printf("%s\n", what); return 1; }

int main() {
  dpa::admission_config c;
  c.slot_capacity = 1000;
  c.small_seeds = 10;
  c.reserved_slots = 100;
  c.max_bypass_seconds = 1.0;
  {  // A small request passes a large one that has no room yet.
    std::deque<req> q = {{1, 600, 0.0}, {2, 5, 0.1}, {3, 8, 0.2}};
    const auto got = scan(q, c, 500, 0.5);
    if (got != std::vector<int>({2, 3}) || q.size() != 1 || q.front().id != 1)
      return fail("small requests did not pass the blocked large one");
  }
  {  // Large requests stop at capacity - reserved; small ones use the reserve.
    std::deque<req> q = {{1, 400, 0.0}, {2, 400, 0.0}, {3, 100, 0.0}, {4, 10, 0.0}, {5, 10, 0.0}};
    const auto got = scan(q, c, 0, 0.5);
    // Large requests fill up to 900 of the 1000 slots; the small ones then
    // take reserved slots.
    if (got != std::vector<int>({1, 2, 3, 4, 5})) return fail("fill up to the reserve");
    std::deque<req> q2 = {{6, 50, 0.0}, {7, 10, 0.0}};
    const auto got2 = scan(q2, c, 880, 0.5);
    if (got2 != std::vector<int>({7})) return fail("a large request took reserved slots");
  }
  {  // Once the oldest has waited max_bypass_seconds, no large request passes
     // it; small ones still do, while all small requests stay in the reserve...
    std::deque<req> q = {{1, 600, 0.0}, {2, 5, 0.1}, {3, 50, 0.2}, {4, 8, 0.3}};
    const auto got = scan(q, c, 500, 1.5, 1000, 0);  // the head has no room
    if (got != std::vector<int>({2, 4}) || q.size() != 2 || q.front().id != 1 ||
        q.back().id != 3)
      return fail("an overdue head: large requests passed it or small ones did not");
    std::deque<req> q2 = {{1, 600, 0.0}, {2, 5, 0.1}, {3, 8, 0.2}};
    const auto got2 = scan(q2, c, 500, 1.5, 1000, 90);  // 90 of 100 reserved slots held
    if (got2 != std::vector<int>({2}) || q2.size() != 2)
      return fail("small requests passed an overdue head beyond the reserve");
    c.reserved_slots = 0;  // no reserve: nothing passes an overdue head
    std::deque<req> q3 = {{1, 600, 0.0}, {2, 5, 0.1}};
    const auto got3 = scan(q3, c, 500, 1.5);
    c.reserved_slots = 100;
    if (!got3.empty() || q3.size() != 2) return fail("a request passed the overdue head");
  }
  {  // ...and it may then take reserved slots.
    std::deque<req> q = {{1, 950, 0.0}, {2, 5, 0.1}};
    const auto got = scan(q, c, 0, 1.5);
    if (got != std::vector<int>({1, 2})) return fail("the overdue head could not use the reserve");
  }
  {  // Admission stops when no request counter is free.
    std::deque<req> q = {{1, 5, 0.0}, {2, 5, 0.0}, {3, 5, 0.0}};
    const auto got = scan(q, c, 0, 0.0, 2);
    if (got != std::vector<int>({1, 2}) || q.size() != 1) return fail("counter limit ignored");
  }
  {  // A head that is not overdue may be passed, and a later one blocks nothing.
    std::deque<req> q = {{1, 600, 0.9}, {2, 700, 0.0}, {3, 5, 0.95}};
    const auto got = scan(q, c, 500, 1.2);
    if (got != std::vector<int>({3})) return fail("only the oldest may stop the scan");
  }
  std::puts("ok");
  return 0;
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="no C++ compiler")
def test_admission_passes_small_requests_within_the_reserve_and_bypass_limits(tmp_path):
    src = tmp_path / "admission.cpp"
    exe = tmp_path / "admission"
    src.write_text(ADMISSION_DRIVER)
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-I", str(CSRC), str(src), "-o", str(exe)],
                   check=True)
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0 and run.stdout.strip() == "ok", run.stdout + run.stderr
