// Unit tests of hdcx::planLanes (hdcodex_b200/csrc/batch_plan.h): how
// hdcx_render_batch deals jobs to lanes and sizes their path arenas. Prints
// one line per failed check and exits non-zero if any failed.
#include "batch_plan.h"

#include <cmath>
#include <cstdio>
#include <numeric>
#include <set>

namespace {

int failures = 0;

void expect(bool ok, const char* what, int line)
{
    if (!ok) {
        std::printf("FAILED line %d: %s\n", line, what);
        ++failures;
    }
}
#define EXPECT(c) expect((c), #c, __LINE__)

constexpr uint64_t kMaxWave = 48ull << 20;
constexpr uint64_t kMinShare = 1ull << 20;

uint64_t laneTotal(const hdcx::LanePlan& p, const std::vector<uint64_t>& paths, size_t l)
{
    uint64_t t = 0;
    for (uint32_t j : p.members[l]) t += paths[j];
    return t;
}

void everyJobExactlyOnce()
{
    const std::vector<uint64_t> paths = {5, 900, 17, 3000000, 42, 42, 1, 77777, 123456789, 8};
    const hdcx::LanePlan p = hdcx::planLanes(paths, 4, 0, kMaxWave, kMinShare);
    EXPECT(p.members.size() == 4 && p.capacity.size() == 4);
    std::multiset<uint32_t> seen;
    for (const auto& lane : p.members) seen.insert(lane.begin(), lane.end());
    EXPECT(seen.size() == paths.size());
    for (uint32_t j = 0; j < paths.size(); ++j) EXPECT(seen.count(j) == 1);
}

void largestFirstOntoTheLightestLane()
{
    // Longest-processing-time dealing: 8, 7, 6, 5 open the four lanes, then
    // 4 goes onto the lane of 5, 3 onto 6, 2 onto 7, 1 onto 8.
    const std::vector<uint64_t> paths = {1, 2, 3, 4, 5, 6, 7, 8};
    const hdcx::LanePlan p = hdcx::planLanes(paths, 4, 1ull << 40, kMaxWave, kMinShare);
    EXPECT(p.members[0].size() == 2 && p.members[0][0] == 7 && p.members[0][1] == 0);
    EXPECT(p.members[1].size() == 2 && p.members[1][0] == 6 && p.members[1][1] == 1);
    EXPECT(p.members[2].size() == 2 && p.members[2][0] == 5 && p.members[2][1] == 2);
    EXPECT(p.members[3].size() == 2 && p.members[3][0] == 4 && p.members[3][1] == 3);
    for (size_t l = 0; l < 4; ++l) EXPECT(laneTotal(p, paths, l) == 9);
    // A lane runs its largest job first, and its wave holds that job.
    for (size_t l = 0; l < 4; ++l) EXPECT(p.capacity[l] == paths[p.members[l][0]]);
}

void tiesKeepInputOrder()
{
    const std::vector<uint64_t> paths = {10, 10, 10};
    const hdcx::LanePlan p = hdcx::planLanes(paths, 2, 1ull << 40, kMaxWave, kMinShare);
    EXPECT(p.members[0].size() == 2 && p.members[0][0] == 0 && p.members[0][1] == 2);
    EXPECT(p.members[1].size() == 1 && p.members[1][0] == 1);
}

void fewerJobsThanLanes()
{
    const std::vector<uint64_t> paths = {100, 200};
    const hdcx::LanePlan p = hdcx::planLanes(paths, 4, 1ull << 40, kMaxWave, kMinShare);
    EXPECT(p.members.size() == 2);
    EXPECT(p.members[0][0] == 1 && p.members[1][0] == 0);
}

void capacityBounds()
{
    // The largest job is capped by the maximum wave...
    const std::vector<uint64_t> big = {400000000, 10, 10, 10};
    hdcx::LanePlan p = hdcx::planLanes(big, 4, 1ull << 40, kMaxWave, kMinShare);
    EXPECT(p.capacity[0] == kMaxWave);
    EXPECT(p.capacity[1] == 10);
    // ... and by an equal share of the budget, never below the minimum share ...
    p = hdcx::planLanes(big, 4, 40000000, kMaxWave, kMinShare);
    EXPECT(p.capacity[0] == 10000000);
    p = hdcx::planLanes(big, 4, 1000, kMaxWave, kMinShare);
    EXPECT(p.capacity[0] == kMinShare);
    EXPECT(p.capacity[1] == 10);
    // ... and a wave holds at least three paths (one sample's three lanes).
    const std::vector<uint64_t> tiny = {1};
    p = hdcx::planLanes(tiny, 4, 1ull << 40, kMaxWave, kMinShare);
    EXPECT(p.capacity.size() == 1 && p.capacity[0] == 3);
}

void emptyInputs()
{
    EXPECT(hdcx::planLanes({}, 4, 0, kMaxWave, kMinShare).members.empty());
    EXPECT(hdcx::planLanes({5, 6}, 0, 0, kMaxWave, kMinShare).members.empty());
}

void balanceOnASeededMix()
{
    // 64 jobs of a log-uniform size mix: the fullest lane exceeds the mean by
    // less than the largest job (the greedy bound of longest-first dealing).
    std::vector<uint64_t> paths;
    uint64_t state = 12345;
    for (int i = 0; i < 64; ++i) {
        state = state * 6364136223846793005ull + 1442695040888963407ull;
        const double u = static_cast<double>(state >> 11) / 9007199254740992.0;
        paths.push_back(static_cast<uint64_t>(786432.0 * std::pow(400.0, u)));
    }
    const hdcx::LanePlan p = hdcx::planLanes(paths, 4, 1ull << 40, kMaxWave, kMinShare);
    const uint64_t sum = std::accumulate(paths.begin(), paths.end(), uint64_t{0});
    const uint64_t largest = *std::max_element(paths.begin(), paths.end());
    uint64_t fullest = 0;
    for (size_t l = 0; l < 4; ++l) fullest = std::max(fullest, laneTotal(p, paths, l));
    EXPECT(fullest * 4 <= sum + 4 * largest);
}

}  // namespace

int main()
{
    everyJobExactlyOnce();
    largestFirstOntoTheLightestLane();
    tiesKeepInputOrder();
    fewerJobsThanLanes();
    capacityBounds();
    emptyInputs();
    balanceOnASeededMix();
    if (failures == 0) std::printf("all batch plan checks passed\n");
    return failures == 0 ? 0 : 1;
}
