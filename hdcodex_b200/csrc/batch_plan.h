// batch_plan.h - how hdcx_render_batch deals the jobs of one device to lanes
// and sizes each lane's path arena. Host-only and free of CUDA, so that the
// rules are unit-tested on the CPU (tests/cpp/batch_plan_tests.cpp).
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

namespace hdcx {

// Lanes of one device: `members[l]` are indices into the `paths` given to
// planLanes, in the order the lane runs them; `capacity[l]` is the lane's
// wave size in paths.
struct LanePlan {
    std::vector<std::vector<uint32_t>> members;
    std::vector<uint64_t> capacity;
};

// Deals jobs of `paths[j]` spectral paths to `lanes` lanes: largest job first
// (ties keep the input order) onto the lane with the fewest paths so far
// (ties go to the lowest lane). A lane's wave holds its largest job's paths,
// at most `maxWave`, at most an equal share of `budget` paths of path state
// but never below `minShare`, and at least 3.
inline LanePlan planLanes(const std::vector<uint64_t>& paths, uint32_t lanes, uint64_t budget, uint64_t maxWave,
                          uint64_t minShare)
{
    LanePlan plan;
    if (paths.empty() || lanes == 0) return plan;
    lanes = std::min<uint32_t>(lanes, static_cast<uint32_t>(paths.size()));
    std::vector<uint32_t> order(paths.size());
    for (uint32_t j = 0; j < order.size(); ++j) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return paths[a] > paths[b]; });
    plan.members.assign(lanes, {});
    std::vector<uint64_t> total(lanes, 0);
    for (uint32_t j : order) {
        const uint32_t l = static_cast<uint32_t>(std::min_element(total.begin(), total.end()) - total.begin());
        plan.members[l].push_back(j);
        total[l] += paths[j];
    }
    const uint64_t share = std::max<uint64_t>(budget / lanes, minShare);
    for (uint32_t l = 0; l < lanes; ++l) {
        const uint64_t largest = paths[plan.members[l].front()];
        plan.capacity.push_back(std::max<uint64_t>(3, std::min({largest, maxWave, share})));
    }
    return plan;
}

}  // namespace hdcx
