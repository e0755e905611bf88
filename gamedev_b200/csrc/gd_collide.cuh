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
    long long records_dropped = 0;  // baths beyond the device record buffer between two reads
    std::vector<BathRecord> baths;
    void record(const BathRecord &r);
    std::string json() const;
};

// Host controller pieces (inc/swarm/_col_bound.cuh:209-403), usable without a GPU; the arithmetic
// is gd_ctl_core.cuh's, shared with the device controller.
int build_binmap(const Model &m, const std::vector<int> &raw_count, std::vector<int> &raw_to_merged);
Status choose_bath(const Model &m, const RateBin *bins, int count, double remaining, double limit_scale,
                   double &out, int *binding);
Status finish_bath(const Model &m, const AuditBin *bins, int count, BathState &state, BathResult &out);
Status ctl_status(int code);  // a CtlCode as a status with the reference's message

// The wave the operator's kernels serve, read from device memory: the device controller writes it,
// so a wave's launches depend on nothing the host knows and the operator runs as one CUDA graph.
struct WaveInfo {
    int count;       // owners of this wave
    int full;        // 1: the wave holds every particle (kernels walk them in index order)
    int go;          // 1 while the operator runs
    int need_rates;  // 1: this wave publishes its reservoir and evaluates its rates (tick > 0, or tick 0)
    int publish;     // publish wave of the reservoir stamps (persists across operators)
    int pad[3];
};

// Results of an operator the host reads back: error, counters, the baths recorded.
struct CtlResult {
    int error;             // a CtlCode, or 100 + the chain's error flag
    int error_detail;
    int waves;
    int rec_count, rec_dropped;
    int operator_index;
    long long owner_updates;
    double min_duration, max_duration;
    int log_count, log_dropped;  // operator-log records written since the last read
};

// One group's line of the COL_DIAGNOSTICS per-operator log (local_group_stats and the schedule
// counters of _col_chain.cuh:25-31, 266-289, 488-517).
struct OperatorLogGroup {
    int owners, level, initial_level, binding;
    double dt, min_request, max_request, final_request, initial_request;
    double max_age, max_ratio, max_growth, max_activity;
    unsigned long long coarsened, refined, constrained, updates;
    int overshoots, persistent;
};
constexpr int kLogGroups = 256;  // groups one record holds (the controller's maximum)
// One operator's record of that log (_col_chain.cuh:488-535).  chain_launches counts the persistent
// chain's launches (one per wave) and chain_blocks the owners each launch started with; the
// reference relaunches capped chains and counts every relaunch.  The seconds are device time
// (%globaltimer) between the controller's marks.
struct OperatorLog {
    unsigned long long operator_id, finest_ticks, owner_updates, chain_blocks;
    int waves, chain_launches, G, pad;
    double clock_sim, duration, chain_seconds, audit_seconds, wall_seconds;
    double rate_seconds;  // the waves' reservoir publish, bath rates and bins (COL_PERF_VAL's rate phase)
    unsigned long long event_count[kEventCategories];
    double event_log_mass[kEventCategories];
    OperatorLogGroup g[kLogGroups];
};

struct CtlDev;  // the device controller's state (gd_devctl.cu)

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
    // bit-identical stored rates.  The publish counter lives in the device controller's WaveInfo.
    DevBuf<int> stamp, rated;
    double rated_lambda0 = 0.0;
    DevBuf<double> env;               // 8 doubles per owner (query_environment)
    DevBuf<double> height;            // R h_g(R) per particle (N_Z = 1 physical kernel), per geometry epoch
    DevBuf<double> cached;            // 4 doubles per owner (cached_rate_moments)
    // Stored pairs (n*K < 2^31 only, else left empty): four planes of n*K doubles, each pair's rate,
    // rate*mean, rate*second and maximum at owner*K + slot; the list of changed pairs of owners
    // whose own entry is unchanged (owner*K + slot), and those owners.
    DevBuf<double> leaf;
    DevBuf<unsigned int> pairs;
    DevBuf<int> folds;
    DevBuf<int> whole;                // the owners a wave evaluates whole (their own entry changed)
    DevBuf<int> ids, queue, group_sorted, spatial;
    // per-group / per-bin device scratch, one contiguous block (small_layout() in gd_collide.cu)
    DevBuf<unsigned char> small;
    size_t events_offset = 0;         // the events counter inside `small`
    // device controller: scheduler, bath states, wave table, accumulated results (gd_devctl.cu)
    DevBuf<unsigned char> ctl;        // one CtlDev
    DevBuf<double> conf_log;          // log(2 c / COL_BATH_ALPHA) for c = 0..raw bins, host-evaluated
    DevBuf<BathRecord> records;       // the baths of the operators since the last read
    int record_capacity = 0;
    unsigned char *host_ctl = nullptr;  // pinned: the CtlResult and the events counter read back
    bool results_pending = false;     // operators ran whose results were not read yet
    cudaStream_t capture_stream = nullptr;  // an eager operator is captured here, then launched
    cudaStream_t body_stream = nullptr;     // the wave body is captured here into the conditional node
    bool setup_done = false;          // kernel attributes raised, grids sized
    int sms = 0, chain_grid = 0;
    const void *chain_kernel = nullptr;  // the k_chain instantiation for the model's K
    size_t rate_smem = 0, chain_smem = 0;
    long long pending_launches = 0;   // launches outside the wave loop of the operators not read yet
    int body_launches = 0;            // kernels of one wave body
    ControllerSummary summary;        // reset with the bath states at output boundaries
    // COL_DIAGNOSTICS event bookkeeping of the last operator (when `diagnostics` is on): events
    // and summed log mass change per outcome category (event_work, _col_types.cuh:32-33)
    bool diagnostics = false;
    DevBuf<unsigned long long> event_count;
    DevBuf<double> event_log_mass;
    // the per-operator JSONL log of COL_DIAGNOSTICS: device records until read, then text
    DevBuf<OperatorLog> oplog;
    int oplog_capacity = 0;
    std::string operator_log;
    // device seconds per phase over the logged operators (the reference's COL_PERF_VAL split,
    // _col_chain.cuh:215-241): bath rates, events (skip scan + chains), audit, whole operators
    double phase_seconds[4] = {0.0, 0.0, 0.0, 0.0};
    bool local_geometry_valid = false;
    gd_operator_stats stats{};
    long long launches = 0;           // kernels launched by the operator (reported by the ABI)
    ~Collider();
};

constexpr int kRecordCapacity = 65536;  // bath records kept on the device between two reads
Status collider_alloc(Collider &c, const Model &m, int n, int record_capacity = kRecordCapacity);
// Bath states and the summary afresh (an output boundary); reads pending results first.
Status collider_reset_state(Collider &c, cudaStream_t s);
// Reads the results of the operators run since the last read (error, statistics, bath records)
// and clears the device accumulators: synchronises s.
Status collider_check(Collider &c, cudaStream_t s);
// The same for many colliders with three synchronisations in all; the first error, and in
// *first_failed the index of its collider (-1: none).
Status collider_check_many(Collider *const *cs, int count, cudaStream_t s, int *first_failed);

// One operator enqueued on q, which must be capturing (a graph the caller builds, e.g. many
// swarms' operators on forked streams): the results are read by collider_check(_many) after the
// graph ran.
Status collision_operator_enqueue(Collider &c, const Model &m, int n, gd_particle *part, curandState *rng,
                                  const int32_t *codes, const double *measure, const unsigned char *active,
                                  double duration, double total_dust_mass, cudaStream_t q);

// col_bath_rate for every owner, alone (gd_bath_rates): out4 [n][4] the cached rate moments
Status bath_rates(Collider &c, const Model &m, int n, const gd_particle *part, const int32_t *codes,
                  const double *measure, const unsigned char *active, double total_dust_mass, double *out4,
                  int *launches, cudaStream_t s);

// one frozen bath of `bath` seconds for every owner, eagerly (gd_bath_chain): bath-start rates,
// skip scan and chain; the particles and RNG streams advance in place, `events` counts the events
Status bath_chain(Collider &c, const Model &m, int n, gd_particle *part, curandState *rng, const int32_t *codes,
                  const double *measure, const unsigned char *active, double total_dust_mass, double bath,
                  unsigned long long *events, int *launches, cudaStream_t s);

// per-pair terms of the bath-start rate for the listed owners (diagnostics and parity checks)
Status pair_rates(const Model &m, const int *ids, int count, const gd_particle *part, const int32_t *codes,
                  const double *measure, const unsigned char *active, double total_dust_mass, int n, double *out,
                  cudaStream_t s);

// evolve_local_collisions (inc/swarm/_col_chain.cuh:108-539) as one CUDA graph: the bath-start
// pass, then a conditional WHILE node running one wave per iteration, every controller decision on
// the device.  Eager when s is not capturing (the graph runs, the results are read, an error is
// returned); inside the caller's capture it becomes part of that graph and collider_check reads the
// results later.  The horizon is `duration`, or duration_scale * *duration_dev when given.
Status collision_operator(Collider &c, const Model &m, int n, gd_particle *part, curandState *rng,
                          const int32_t *codes, const double *measure, const unsigned char *active,
                          int32_t *spatial, double duration, double total_dust_mass, cudaStream_t s,
                          const double *duration_dev = nullptr, double duration_scale = 1.0,
                          const double *clock_sim_dev = nullptr);
// The per-operator log (COL_DIAGNOSTICS) needs its device records: allocated when diagnostics turn on.
Status collider_enable_log(Collider &c);

}  // namespace gd
