// cmc_grants.cpp -- the serving loop's grant policy (see cmc_grants.hpp).
#include "cmc_grants.hpp"

#include <algorithm>

namespace cmc {

std::vector<GrantShare> grant_shares(const std::vector<GrantCandidate>& jobs, uint64_t work_blocks,
                                     double fifo_share, uint64_t max_trials) {
    const size_t n = jobs.size();
    auto remaining = [&](size_t i) { return double(jobs[i].budget - jobs[i].next) * jobs[i].cost; };
    double floor_blocks = 0, backlog = 0;
    for (size_t i = 0; i < n; ++i) {
        floor_blocks = std::max(floor_blocks, 2.5 * jobs[i].latency_blocks);
        backlog += remaining(i);
    }
    const double adaptive = std::min(backlog / 8.0, 20.0 * double(work_blocks));
    work_blocks = std::max<uint64_t>({work_blocks, uint64_t(floor_blocks), uint64_t(adaptive)});

    std::vector<uint64_t> share(n, 0);
    double left = double(work_blocks);
    uint64_t trials_left = max_trials;
    auto room = [&](size_t i) {  // trials job i can still take in this step
        const GrantCandidate& j = jobs[i];
        const uint64_t per = 1ULL << j.bt;
        const uint64_t next = j.next + share[i];
        if (next >= j.budget) return uint64_t(0);
        uint64_t r = std::min<uint64_t>(j.budget - next, per - (next & (per - 1)));
        if (share[i] > 0 && (next & (per - 1)) == 0) r = 0;  // one batch per grant
        return std::min<uint64_t>(r, 0xffffffffULL - share[i]);
    };
    auto give = [&](size_t i, double blocks) {
        uint64_t t = uint64_t(std::max(1.0, blocks / jobs[i].cost));
        t = std::min<uint64_t>({t, room(i), trials_left});
        share[i] += t;
        trials_left -= t;
        left -= double(t) * jobs[i].cost;
    };
    std::vector<size_t> fifo(n), order(n);
    for (size_t i = 0; i < n; ++i) fifo[i] = order[i] = i;
    std::sort(fifo.begin(), fifo.end(), [&](size_t a, size_t b) {
        return jobs[a].admitted_at != jobs[b].admitted_at ? jobs[a].admitted_at < jobs[b].admitted_at
                                                          : jobs[a].id < jobs[b].id;
    });
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return remaining(a) < remaining(b); });
    const double keep = double(work_blocks) * (1.0 - fifo_share);
    for (size_t i : fifo) {
        if (left <= keep || trials_left == 0) break;
        give(i, left - keep);
    }
    for (size_t i : order) {
        if (left <= 0 || trials_left == 0) break;
        give(i, left);
    }
    std::vector<size_t> heavy;
    for (size_t i = 0; i < n; ++i)
        if (share[i] > 0) heavy.push_back(i);
    std::stable_sort(heavy.begin(), heavy.end(), [&](size_t a, size_t b) { return jobs[a].cost > jobs[b].cost; });
    std::vector<GrantShare> out;
    for (size_t i : heavy) out.push_back(GrantShare{jobs[i].id, share[i]});
    return out;
}

}  // namespace cmc
