// Frozen-bath collision operator state (the reference's local_workspace, _col_chain.cuh:36-96,
// plus the dev_col_* caches of swarm_runtime.cu:120-184) and its host controller.
#pragma once

#include <curand_kernel.h>

#include <cmath>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "gd_internal.cuh"

namespace gd {

// col_rate_bin (inc/swarm/_col_types.cuh:376-384)
struct RateBin {
    double mass, weighted_rate, weighted_change, weighted_second;
    int owner_count, invalid_count;
};

// col_audit_accum (inc/swarm/_col_types.cuh:386-403)
struct AuditBin {
    double mass, predicted_f, predicted_e, predicted_var_f, predicted_var_e, predicted_g, predicted_var_g,
        maximum_weight, maximum_g_jump, touched, event_weight, growth, end_mass;
    int owner_count, invalid_count;
};

// col_bath_state / col_bath_result (inc/swarm/_col_types.cuh:405-425)
struct BathState {
    double limit_scale = 1.0;
    int activity_streak = 0, quiet_streak = 0, floor_streak = 0;
};
struct BathResult {
    double max_f = 0, max_e = 0, max_touched = 0, max_events = 0, max_g = 0, max_g_upper = 0, d_bath = 0;
    bool activity_overshoot = false, distribution_overshoot = false, persistent_overshoot = false;
};

// Controller diagnostics of one output interval (col_bath_record / col_controller_summary,
// inc/swarm/_col_types.cuh:87-120): one record per finished group bath and the running extrema,
// kept by _record_col_bath (_col_bound.cuh:219-238) and written as save_col_controller writes them
// (:242-299).  continuation_launches counts chain launches per wave; this build's chain is
// persistent, so that is one per wave where the reference relaunches capped chains.
constexpr int kEventCategories = 7;  // EVENT_CATEGORIES (inc/swarm/_col_types.cuh:32)

struct BathRecord {
    int group_index = -1, operator_index = 0, bath_index = 0, merged_bins = 0, continuation_launches = 0;
    double duration = 0.0, limit_before = 1.0, limit_after = 1.0;
    BathResult result;
};
struct ControllerSummary {
    int operator_count = 0, bath_count = 0, wave_count = 0, continuation_launches = 0;
    int activity_overshoots = 0, distribution_overshoots = 0, persistent_overshoots = 0;
    double minimum_duration = HUGE_VAL, maximum_duration = 0.0, minimum_limit_scale = 1.0;
    double maximum_f = 0.0, maximum_e = 0.0, maximum_touched = 0.0, maximum_events = 0.0, maximum_g = 0.0,
           maximum_g_upper = 0.0, maximum_d_bath = 0.0;
    std::vector<BathRecord> baths;
    void record(const BathRecord &r);
    std::string json() const;
};

// Power-of-two group scheduler on a 2^52-tick lattice (local_schedule, _col_sched.cuh:17-183).
struct Schedule {
    double horizon = 0;
    std::vector<std::pair<int, int>> links;
    std::vector<int> level;
    std::vector<std::uint64_t> step, next;
    std::uint64_t end = 0;
    Status init(double h, const std::vector<double> &requested, const std::vector<unsigned int> &edges);
    std::uint64_t time() const;
    double seconds(std::uint64_t tick) const { return horizon * (double(tick) / double(end)); }
    std::vector<int> due(std::uint64_t tick) const;
    Status adapt(std::uint64_t tick, const std::vector<int> &groups, const std::vector<double> &requested,
                 const std::vector<bool> &passed);
    void advance(const std::vector<int> &groups) {
        for (int c : groups) next[c] += step[c];
    }
};

// Host controller pieces (inc/swarm/_col_bound.cuh:209-403), usable without a GPU.
struct ChangeBound {
    double duration;
    int reason;
};
Status change_limit(double A, double B, double epsilon, double horizon, ChangeBound &out);
int build_binmap(const Model &m, const std::vector<int> &raw_count, std::vector<int> &raw_to_merged);
Status choose_bath(const Model &m, const RateBin *bins, int count, double remaining, double limit_scale,
                   double &out, int *binding);
Status finish_bath(const Model &m, const AuditBin *bins, int count, BathState &state, BathResult &out);

struct Collider {
    int n = 0;
    // per-owner SoA state
    DevBuf<double> size_old, numr_old, time, hazard, jump1, jump2, jumpmax, rate, change_rate, second_rate;
    DevBuf<int> events, error;
    DevBuf<unsigned char> complete;
    // Reuse of bath-start rates: stamp[j] = publish wave at which particle j's reservoir value last
    // changed; rated[i] = publish wave at which owner i's rates were last evaluated (-1: never on
    // this geometry).  Rates depend only on the reservoir of the owner and its neighbours, the
    // neighbour list, measure, positions and lambda0, so an owner whose inputs are unchanged keeps
    // bit-identical stored rates.
    DevBuf<int> stamp, rated;
    int publish = 0;
    double rated_lambda0 = 0.0;
    DevBuf<double> env;               // 8 doubles per owner (query_environment)
    DevBuf<double> cached;            // 4 doubles per owner (cached_rate_moments)
    DevBuf<int> ids, queue, group_sorted, spatial;
    // per-group / per-bin device scratch, one contiguous block so one copy returns it
    DevBuf<unsigned char> small;      // see small_layout() in gd_collide.cu
    // pinned host mirror of `small`
    unsigned char *host_small = nullptr;
    // host controller state
    std::vector<int> group_start;     // [groups + 1] offsets into group_sorted
    std::vector<unsigned int> edges;  // dependency rows, LOCAL_WORDS per group
    std::vector<BathState> state;
    ControllerSummary summary;        // reset with `state` at output boundaries
    // COL_DIAGNOSTICS event bookkeeping of the last operator (when `diagnostics` is on): events
    // and summed log mass change per outcome category (event_work, _col_types.cuh:32-33)
    bool diagnostics = false;
    DevBuf<unsigned long long> event_count;
    DevBuf<double> event_log_mass;
    bool local_geometry_valid = false;
    gd_operator_stats stats{};
    long long launches = 0;           // kernels launched by the operator (reported by the ABI)
    ~Collider();
};

Status collider_alloc(Collider &c, const Model &m, int n);
void collider_reset_state(Collider &c);

// per-pair terms of the bath-start rate for the listed owners (diagnostics and parity checks)
Status pair_rates(const Model &m, const int *ids, int count, const gd_particle *part, const int32_t *codes,
                  const double *measure, const unsigned char *active, double total_dust_mass, int n, double *out,
                  cudaStream_t s);

// evolve_local_collisions (inc/swarm/_col_chain.cuh:108-539)
Status collision_operator(Collider &c, const Model &m, int n, gd_particle *part, curandState *rng,
                          const int32_t *codes, const double *measure, const unsigned char *active,
                          int32_t *spatial, double duration, double total_dust_mass, cudaStream_t s);

}  // namespace gd
