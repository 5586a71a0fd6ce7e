// Channel order of a single rank: first-fit-decreasing by cost (main.cpp:94-115,
// balance.cpp:11-24, 91-140) degenerates to cost descending, index ascending.  Regular and
// modified channels share it.  Used by the host builder and by the device channel
// construction, so that both permute channels identically.
#ifndef CCD_CHANNEL_ORDER_H
#define CCD_CHANNEL_ORDER_H

#include <algorithm>
#include <cstdint>
#include <utility>
#include <vector>

#include "ccdgpu.h"

// order[i] = unpermuted index of the channel placed at position i.
inline std::vector<uint64_t> ffd_channel_order(const std::vector<ccdgpu_channel_dims> &d0) {
  const uint64_t nch = d0.size();
  std::vector<std::pair<double, uint64_t>> load(nch);
  for (uint64_t c = 0; c < nch; c++) {
    double pp = d0[c].pp, hh = d0[c].hh, ph = d0[c].ph, hp = d0[c].hp;
    double cost = 0;
    cost += hh * hh; cost += hh * hp; cost += hh * pp; cost += hp * ph;
    cost += hp * pp; cost += pp * pp; cost += hp * ph; cost += hp * hp;
    load[c] = {cost, c};
  }
  std::sort(load.begin(), load.end(), [](const std::pair<double, uint64_t> &a,
                                         const std::pair<double, uint64_t> &b) {
    if (a.first != b.first) return a.first > b.first;
    return a.second < b.second;
  });
  std::vector<uint64_t> order(nch);
  for (uint64_t i = 0; i < nch; i++) order[i] = load[i].second;
  return order;
}

#endif
