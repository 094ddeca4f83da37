// admission.hpp -- which waiting requests the request server admits next.
// Host code only; the CPU tests compile it on its own.
//
// Requests wait in submission order. A scan over the queue admits every
// request whose seeds (and, for a recording request, curve staging) fit the
// arenas now, so that a small request does not wait behind a large one that
// has no room yet. Two rules bound what the scan may do:
//  - a share of the particle slots (reserved_slots) is kept for small
//    requests (at most small_seeds seeds): a large request is admitted only
//    while the slots in use stay below capacity - reserved_slots, so a burst
//    of large requests cannot take every slot from the small ones;
//  - once the oldest waiting request has waited max_bypass_seconds and still
//    has no room, no large request behind it is admitted, and small ones only
//    while all small requests together stay within the reserved share. It
//    may take reserved slots itself. The slots large requests hold can only
//    shrink until it is admitted, so it cannot be passed over indefinitely,
//    while small requests keep passing (a rule that stopped them too held
//    every request behind one large one for up to a second).
#pragma once

#include <cstdint>
#include <deque>

namespace dpa {

struct admission_config {
  uint64_t slot_capacity = 0;
  uint64_t small_seeds = 0;      // requests of at most this many seeds are small
  uint64_t reserved_slots = 0;   // slots large requests may not take
  double max_bypass_seconds = 0.0;
};

// Scans `queue` (oldest first) and admits what fits under the rules above.
// seeds(r) is a request's slot count; try_admit(r) allocates its arenas and
// returns false when they have no room; admitted(r) takes the request (it is
// then erased from the queue). used_slots is the number of slots in use and
// small_slots the part of it small requests hold; both are updated (the
// caller subtracts a request's seeds from both, or from used_slots alone for a
// large one, when it releases it). Stops early when capacity_left() is false
// (no request counter free).
template <class T, class Seeds, class Waited, class TryAdmit, class Admitted, class CapacityLeft>
void admit_waiting(std::deque<T>& queue, const admission_config& c, uint64_t& used_slots,
                   uint64_t& small_slots, Seeds seeds, Waited waited, TryAdmit try_admit,
                   Admitted admitted, CapacityLeft capacity_left) {
  const uint64_t large_limit =
      c.slot_capacity > c.reserved_slots ? c.slot_capacity - c.reserved_slots : 0;
  bool head = true;   // the element under the scan is the oldest still waiting
  bool held = false;  // an overdue oldest request is waiting for room
  for (auto it = queue.begin(); it != queue.end() && capacity_left();) {
    const uint64_t n = seeds(*it);
    const bool large = n > c.small_seeds;
    // The oldest request, once it has waited long enough, may use the
    // reserved share too (a request larger than capacity - reserved_slots
    // could not be admitted otherwise).
    const bool overdue = head && waited(*it) >= c.max_bypass_seconds;
    bool ok = held ? !large && small_slots + n <= c.reserved_slots
                   : !(large && !overdue && used_slots + n > large_limit);
    if (ok) ok = try_admit(*it);
    if (ok) {
      used_slots += n;
      if (!large) small_slots += n;
      admitted(*it);
      it = queue.erase(it);
      continue;  // the next element may be the new head
    }
    if (overdue) held = true;
    head = false;
    ++it;
  }
}

}  // namespace dpa
