#include "plan.hpp"

#include <algorithm>

namespace qsv {

std::vector<Stage> plan_stages(const std::vector<Lowered>& gates, int n, int m,
                               int low, int max_gates, int max_red, size_t max_bytes,
                               size_t elem_bytes) {
  std::vector<Stage> stages;
  if (m > n) m = n;
  if (low > m) low = m;
  const uint64_t all = (n >= 64) ? ~0ull : ((1ull << n) - 1ull);
  const uint64_t lowmask = (low >= 64) ? ~0ull : ((1ull << low) - 1ull);

  std::vector<int> remaining;
  remaining.reserve(gates.size());
  for (int i = 0; i < (int)gates.size(); ++i)
    if (gates[i].shape != SH_NONE) remaining.push_back(i);

  std::vector<int> rest;
  while (!remaining.empty()) {
    uint64_t S = lowmask;
    uint64_t blocked = 0;
    Stage st;
    int nred = 0;
    size_t bytes = 0;
    rest.clear();
    for (size_t r = 0; r < remaining.size(); ++r) {
      const int gi = remaining[r];
      const uint64_t b = gate_bits(gates[gi]);
      const bool red = gates[gi].shape == SH_RED;
      const size_t gb = plan_bytes_of(gates[gi], elem_bytes);
      const bool full = (max_gates > 0 && (int)st.gates.size() >= max_gates) ||
                        (red && max_red > 0 && nred >= max_red) ||
                        (max_bytes > 0 && !st.gates.empty() && bytes + gb > max_bytes);
      if (full || (b & blocked)) {
        blocked |= b;
        rest.push_back(gi);
        continue;
      }
      if ((b & ~S) == 0) {
        st.gates.push_back(gi);
        nred += red;
        bytes += gb;
        continue;
      }
      if (__builtin_popcountll(S | b) <= m) {
        S |= b;
        st.gates.push_back(gi);
        nred += red;
        bytes += gb;
        continue;
      }
      blocked |= b;
      rest.push_back(gi);
    }
    // Fill the tile to exactly m bits (lowest unused bits first) so every
    // stage of a plan moves tiles of the same size.
    for (int b = 0; b < n && __builtin_popcountll(S) < m; ++b)
      if (!((S >> b) & 1ull)) S |= 1ull << b;
    S &= all;
    st.m = 0;
    for (int b = 0; b < n; ++b)
      if ((S >> b) & 1ull) st.bits[st.m++] = b;
    stages.push_back(std::move(st));
    remaining.swap(rest);
  }
  return stages;
}

namespace {

// One pass on bit set C: the ops of `remaining` (in order) with bits inside
// C and no bit shared with an earlier op left behind go to `taken`, the
// others to `left`.
void take_pass(const std::vector<uint32_t>& op_bits, const std::vector<int>& remaining,
               uint32_t C, std::vector<int>* taken, std::vector<int>* left) {
  uint32_t blocked = 0;
  for (int oi : remaining) {
    const uint32_t b = op_bits[oi];
    if (!(b & blocked) && (b & ~C) == 0) {
      if (taken) taken->push_back(oi);
      continue;
    }
    blocked |= b;
    left->push_back(oi);
  }
}

// The greedy pass: ops in order while their bits fit in r; returns its bit
// set (before padding) and splits the ops.
uint32_t greedy_pass(const std::vector<uint32_t>& op_bits, const std::vector<int>& remaining,
                     int r, std::vector<int>* taken, std::vector<int>* left) {
  uint32_t S = 0, blocked = 0;
  for (int oi : remaining) {
    const uint32_t b = op_bits[oi];
    if (b & blocked) {
      blocked |= b;
      left->push_back(oi);
      continue;
    }
    if ((b & ~S) == 0 || __builtin_popcount(S | b) <= r) {
      S |= b;
      if (taken) taken->push_back(oi);
      continue;
    }
    blocked |= b;
    left->push_back(oi);
  }
  return S;
}

// Passes the greedy planner needs for `remaining`.
int greedy_count(const std::vector<uint32_t>& op_bits, std::vector<int> remaining, int r) {
  int n = 0;
  std::vector<int> left;
  while (!remaining.empty()) {
    left.clear();
    greedy_pass(op_bits, remaining, r, nullptr, &left);
    remaining.swap(left);
    ++n;
  }
  return n;
}

}  // namespace

std::vector<Pass> plan_passes(const std::vector<uint32_t>& op_bits, int m, int r, bool search) {
  std::vector<Pass> passes;
  std::vector<int> remaining(op_bits.size()), rest, trial;
  for (size_t i = 0; i < op_bits.size(); ++i) remaining[i] = (int)i;
  while (!remaining.empty()) {
    Pass p;
    rest.clear();
    uint32_t S = greedy_pass(op_bits, remaining, r, &p.ops, &rest);
    for (int j = 0; j < m && __builtin_popcount(S) < r; ++j)
      if (!((S >> j) & 1u)) S |= 1u << j;
    if (search && r < m && m <= 16 && rest.size() > 0) {
      // r-bit sets holding the first remaining op's bits, each scored by the
      // passes of the whole remainder finished greedily; the greedy set wins ties
      const uint32_t first = op_bits[remaining[0]];
      int best = 1 + greedy_count(op_bits, rest, r);
      uint32_t bestS = S;
      const int need = r - __builtin_popcount(first);
      std::vector<int> free_bits;
      for (int j = 0; j < m; ++j)
        if (!((first >> j) & 1u)) free_bits.push_back(j);
      auto consider = [&](uint32_t C) {
        if (C == S) return;
        trial.clear();
        take_pass(op_bits, remaining, C, nullptr, &trial);
        const int c = 1 + greedy_count(op_bits, trial, r);
        if (c < best) { best = c; bestS = C; }
      };
      if (need == 0) {
        consider(first);
      } else if (need == 1) {
        for (int a : free_bits) consider(first | (1u << a));
      } else if (need == 2) {
        for (size_t i = 0; i < free_bits.size(); ++i)
          for (size_t k = i + 1; k < free_bits.size(); ++k)
            consider(first | (1u << free_bits[i]) | (1u << free_bits[k]));
      }
      if (bestS != S) {  // redo the pass on the chosen bits
        S = bestS;
        p.ops.clear();
        rest.clear();
        take_pass(op_bits, remaining, S, &p.ops, &rest);
      }
    }
    p.r = 0;
    for (int j = 0; j < m; ++j)
      if ((S >> j) & 1u) p.pos[p.r++] = j;
    passes.push_back(std::move(p));
    remaining.swap(rest);
  }
  return passes;
}

}  // namespace qsv
