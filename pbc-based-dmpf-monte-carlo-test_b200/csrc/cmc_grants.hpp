// cmc_grants.hpp -- the serving loop's grant policy, as a pure function.
//
// Given the jobs of one size class with trials left to issue, it decides how
// many trials each gets in the next step (or publication chunk):
//   * the step's size in AES-block equivalents is work_blocks, at least 2.5x
//     the latency of the slowest trial (so that trial's tail is covered) and
//     grown to an eighth of the outstanding work, at most 20x work_blocks;
//   * fifo_share of it goes to jobs in arrival order (no job starves, the tail
//     stays that of plain per-job launches), the rest shortest remaining work
//     first (small jobs finish at once);
//   * one grant per job, never across a batch boundary, at most max_trials in
//     all;
//   * the result is ordered heaviest trials first, so a launch ends on short
//     trials instead of on the longest walks.
// The caller advances each job's RNG counter by its share.
#pragma once
#include <cstdint>
#include <vector>

namespace cmc {

struct GrantCandidate {
    uint32_t id;            // the caller's job id (ties in arrival order break by id)
    uint64_t next, budget;  // trials issued so far, trials in all
    uint32_t bt;            // batches of 2^bt trials
    double cost;            // AES-block equivalents per trial
    double latency_blocks;  // one trial's latency, in blocks of GPU throughput
    uint64_t admitted_at;   // arrival order
};

struct GrantShare {
    uint32_t id;
    uint64_t trials;
};

std::vector<GrantShare> grant_shares(const std::vector<GrantCandidate>& jobs, uint64_t work_blocks,
                                     double fifo_share, uint64_t max_trials);

}  // namespace cmc
