// Arithmetic of the frozen-bath controller, written once for the host and the device:
//   * the power-of-two group scheduler (local_schedule, inc/swarm/_col_sched.cuh:17-183);
//   * the change-based bath bound (change_limit / _choose_col_bath, inc/swarm/_col_bound.cuh:209-310);
//   * the bath audit (_finish_col_bath, inc/swarm/_col_bound.cuh:313-403).
// The host compiles it for the gd_ctl_* entry points, which are pinned bit for bit against the
// reference's host code; the device controller (gd_devctl.cu, built without FMA contraction)
// compiles the same source, so the collision operator's baths and schedule equal the host
// controller's.  The one transcendental, the audit's confidence logarithm, comes from a table the
// host fills with its own log, so both sides read the same bits.
#pragma once

#include <cmath>

#include "gd_collide.cuh"

namespace gd {

constexpr int kCtlGroups = 256;                                  // controller groups at most
constexpr int kCtlLinks = kCtlGroups * (kCtlGroups - 1) / 2;     // linked group pairs at most

// Outcomes of the controller arithmetic; ctl_status (gd_collide.cu) gives each its gd_status and
// message.
enum CtlCode {
    kCtlOk = 0,
    kCtlBadHorizon,          // invalid local collision horizon
    kCtlBadTimestep,         // invalid local collision timestep
    kCtlTimeResolution,      // local collision timestep exceeds time resolution
    kCtlBadAdaptStep,        // invalid adaptive collision timestep
    kCtlAdaptResolution,     // adaptive collision time resolution exceeded
    kCtlBadRateMoments,      // invalid change-based rate moments
    kCtlBadChangeInputs,     // invalid change-based refresh inputs
    kCtlChangeUnderflow,     // change-based timestep underflow
    kCtlBadAudit,            // the bath controller returned an invalid audit state
    kCtlNoMass,              // the bath controller found no active represented mass
    kCtlWaveLimit,           // the scheduler advanced through too many empty waves in a row
};

__host__ __device__ inline bool ctl_finite(double x) { return x - x == 0.0; }
// std::max / std::min on doubles (the first argument wins ties and NaN-free order)
__host__ __device__ inline double ctl_max(double a, double b) { return (a < b) ? b : a; }
__host__ __device__ inline double ctl_min(double a, double b) { return (b < a) ? b : a; }
__host__ __device__ inline int ctl_imax(int a, int b) { return (a < b) ? b : a; }
__host__ __device__ inline int ctl_imin(int a, int b) { return (b < a) ? b : a; }

// Power-of-two group scheduler on a 2^52-tick lattice (local_schedule, _col_sched.cuh:17-183).
struct SchedCore {
    double horizon;
    int n, nlinks;
    unsigned long long end;
    int level[kCtlGroups];
    unsigned long long step[kCtlGroups], next[kCtlGroups];
    unsigned short link_c[kCtlLinks], link_d[kCtlLinks];  // pairs c < d linked by an edge either way
};

__host__ __device__ inline bool ctl_edge(const unsigned *edges, int words, int c, int d) {
    return (edges[c * words + d / 32] & (1u << (d % 32))) != 0;
}

// local_schedule::local_schedule (_col_sched.cuh:24-71)
__host__ __device__ inline int sched_init(SchedCore &s, double h, const double *requested, int n,
                                          const unsigned *edges) {
    s.horizon = h;
    s.n = n;
    s.nlinks = 0;
    s.end = 0;
    for (int c = 0; c < n; ++c) {
        s.level[c] = 0;
        s.step[c] = 0;
        s.next[c] = 0;
    }
    if (!(h > 0) || !ctl_finite(h)) return kCtlBadHorizon;
    const int words = (n + 31) / 32;
    for (int c = 0; c < n; ++c) {
        if (!(requested[c] > 0) || !ctl_finite(requested[c])) return kCtlBadTimestep;
        double dt = h;
        while (dt > requested[c]) {
            if (++s.level[c] > 52) return kCtlTimeResolution;
            dt *= 0.5;
        }
    }
    for (int c = 0; c < n; ++c)
        for (int d = c + 1; d < n; ++d)
            if (ctl_edge(edges, words, c, d) || ctl_edge(edges, words, d, c)) {
                s.link_c[s.nlinks] = static_cast<unsigned short>(c);
                s.link_d[s.nlinks] = static_cast<unsigned short>(d);
                ++s.nlinks;
            }
    // Linked groups stay within 4 levels: raise the coarser one until no pair is further apart.
    // Levels only grow, so the sweep order does not change the fixed point it reaches.
    bool changed;
    do {
        changed = false;
        for (int e = 0; e < s.nlinks; ++e) {
            const int c = s.link_c[e], d = s.link_d[e];
            if (s.level[c] < s.level[d] - 4) {
                s.level[c] = s.level[d] - 4;
                changed = true;
            }
            if (s.level[d] < s.level[c] - 4) {
                s.level[d] = s.level[c] - 4;
                changed = true;
            }
        }
    } while (changed);
    s.end = 1ull << 52;
    for (int c = 0; c < n; ++c) s.step[c] = 1ull << (52 - s.level[c]);
    return kCtlOk;
}

__host__ __device__ inline unsigned long long sched_time(const SchedCore &s) {
    unsigned long long t = s.next[0];
    for (int c = 1; c < s.n; ++c) t = s.next[c] < t ? s.next[c] : t;
    return t;
}

__host__ __device__ inline int sched_due(const SchedCore &s, unsigned long long tick, int *out) {
    int k = 0;
    for (int c = 0; c < s.n; ++c)
        if (s.next[c] == tick) out[k++] = c;
    return k;
}

__host__ __device__ inline double sched_seconds(const SchedCore &s, unsigned long long tick) {
    return s.horizon * (static_cast<double>(tick) / static_cast<double>(s.end));
}

// local_schedule::adapt (_col_sched.cuh:95-165).  work holds 3 * n ints.
__host__ __device__ inline int sched_adapt(SchedCore &s, unsigned long long tick, const int *groups, int ng,
                                           const double *requested, const unsigned char *passed, int *work) {
    const int n = s.n;
    int *act = work, *cap = work + n, *cand = work + 2 * n;
    for (int c = 0; c < n; ++c) {
        act[c] = 0;
        cand[c] = s.level[c];
    }
    for (int k = 0; k < ng; ++k) act[groups[k]] = 1;
    for (int c = 0; c < n; ++c) cap[c] = act[c] ? 52 : s.level[c];
    bool changed;
    do {
        changed = false;
        for (int e = 0; e < s.nlinks; ++e) {
            const int c = s.link_c[e], d = s.link_d[e];
            if (act[c] && cap[c] > cap[d] + 4) {
                cap[c] = cap[d] + 4;
                changed = true;
            }
            if (act[d] && cap[d] > cap[c] + 4) {
                cap[d] = cap[c] + 4;
                changed = true;
            }
        }
    } while (changed);
    for (int k = 0; k < ng; ++k) {
        const int c = groups[k];
        if (!(requested[c] > 0) || !ctl_finite(requested[c])) return kCtlBadAdaptStep;
        int want = 0;
        double h = s.horizon;
        while (h > requested[c]) {
            if (++want > 52) return kCtlAdaptResolution;
            h *= 0.5;
        }
        cand[c] = passed[c] ? want : ctl_imax(want, s.level[c]);
        while (tick % (1ull << (52 - cand[c]))) ++cand[c];
        cand[c] = ctl_imin(cand[c], cap[c]);
    }
    do {
        changed = false;
        for (int e = 0; e < s.nlinks; ++e) {
            const int c = s.link_c[e], d = s.link_d[e];
            if (act[c] && cand[c] < cand[d] - 4) {
                cand[c] = cand[d] - 4;
                changed = true;
            }
            if (act[d] && cand[d] < cand[c] - 4) {
                cand[d] = cand[c] - 4;
                changed = true;
            }
        }
    } while (changed);
    for (int k = 0; k < ng; ++k) {
        const int c = groups[k];
        s.level[c] = cand[c];
        s.step[c] = 1ull << (52 - s.level[c]);
    }
    return kCtlOk;
}

__host__ __device__ inline void sched_advance(SchedCore &s, const int *groups, int ng) {
    for (int k = 0; k < ng; ++k) s.next[groups[k]] += s.step[groups[k]];
}

// change_limit (_col_bound.cuh:209-220): duration and binding reason (0 horizon, 1 first, 2 second)
__host__ __device__ inline int ctl_change_limit(double A, double B, double epsilon, double horizon, double &duration,
                                                int &reason) {
    if (!ctl_finite(A) || A < 0 || !ctl_finite(B) || B < 0 || !ctl_finite(epsilon) || !(epsilon > 0) ||
        !ctl_finite(horizon) || !(horizon > 0))
        return kCtlBadChangeInputs;
    duration = horizon;
    reason = 0;
    if (A > 0 && epsilon / A < duration) {
        duration = epsilon / A;
        reason = 1;
    }
    if (B > 0 && epsilon * epsilon / B < duration) {
        duration = epsilon * epsilon / B;
        reason = 2;
    }
    if (!(duration > 0)) return kCtlChangeUnderflow;
    return kCtlOk;
}

// _choose_col_bath (_col_bound.cuh:288-310)
__host__ __device__ inline int ctl_choose_bath(const Model &m, const RateBin *bins, int count, double remaining,
                                               double limit_scale, double &out, int *binding) {
    double duration = ctl_min(remaining, m.col_bath_max);
    double tolerance = m.col_bath_eps * limit_scale;
    int reason = 0;
    for (int b = 0; b < count; ++b) {
        const RateBin &v = bins[b];
        if (v.invalid_count) return kCtlBadRateMoments;
        if (!(v.mass > 0)) continue;
        double bound = 0.0;
        int why = 0;
        const int st = ctl_change_limit(v.weighted_change / v.mass, v.weighted_second / v.mass, tolerance, duration,
                                        bound, why);
        if (st) return st;
        if (bound < duration) {
            duration = bound;
            reason = why;
        }
    }
    if (binding) *binding = reason;
    out = duration;
    return kCtlOk;
}

// log(2 c / COL_BATH_ALPHA), the Bernstein confidence of _finish_col_bath for c active bins
inline double ctl_confidence_log(int active_count, double col_bath_alpha) {
    return std::log(2.0 * static_cast<double>(active_count) / col_bath_alpha);
}

// _finish_col_bath (_col_bound.cuh:313-403).  conf_log[c] = ctl_confidence_log(c, alpha), filled by
// the host; the host path may pass nullptr and evaluates it in place.
__host__ __device__ inline int ctl_finish_bath(const Model &m, const AuditBin *bins, int count, BathState &state,
                                               BathResult &result, const double *conf_log) {
    result = BathResult();
    int active_count = 0;
    double total_mass = 0.0;
    for (int b = 0; b < count; ++b) {
        if (bins[b].invalid_count != 0) return kCtlBadAudit;
        if (bins[b].mass > 0.0) active_count++;
        total_mass += bins[b].mass;
    }
    if (!(total_mass > 0.0)) return kCtlNoMass;
    double confidence_log;
#ifdef __CUDA_ARCH__
    confidence_log = conf_log[active_count];
#else
    confidence_log = conf_log ? conf_log[active_count] : ctl_confidence_log(active_count, m.col_bath_alpha);
#endif
    double mass_difference = 0.0;
    for (int b = 0; b < count; ++b) {
        const AuditBin &v = bins[b];
        mass_difference += fabs(v.end_mass - v.mass);
        if (!(v.mass > 0.0)) continue;
        double mass_sq = v.mass * v.mass;
        double predicted_f = v.predicted_f / v.mass;
        double predicted_e = v.predicted_e / v.mass;
        double predicted_g = v.predicted_g / v.mass;
        double touched = v.touched / v.mass;
        double events = v.event_weight / v.mass;
        double growth = v.growth / v.mass;
        double weight_max = v.maximum_weight / v.mass;
        double jump_max = v.maximum_g_jump / v.mass;
        double upper_f = ctl_min(1.0, predicted_f + sqrt(2.0 * v.predicted_var_f / mass_sq * confidence_log) +
                                          weight_max * confidence_log / 3.0);
        double upper_e = predicted_e + sqrt(2.0 * v.predicted_var_e / mass_sq * confidence_log) +
                         weight_max * confidence_log / 3.0;
        double upper_g = predicted_g + sqrt(2.0 * v.predicted_var_g / mass_sq * confidence_log) +
                         jump_max * confidence_log / 3.0;
        result.max_f = ctl_max(result.max_f, predicted_f);
        result.max_e = ctl_max(result.max_e, predicted_e);
        result.max_touched = ctl_max(result.max_touched, touched);
        result.max_events = ctl_max(result.max_events, events);
        result.max_g = ctl_max(result.max_g, growth);
        result.max_g_upper = ctl_max(result.max_g_upper, upper_g);
        result.activity_overshoot = result.activity_overshoot || ctl_min(touched, 1.0) > upper_f || events > upper_e;
        result.distribution_overshoot = result.distribution_overshoot || growth > ctl_max(m.col_bath_eps, upper_g);
    }
    result.d_bath = mass_difference / (2.0 * total_mass);
    result.distribution_overshoot = result.distribution_overshoot || result.d_bath > m.col_bath_eps;
    bool issue = result.activity_overshoot || result.distribution_overshoot;
    bool at_floor = state.limit_scale <= 0.25 * (1.0 + 8.0 * 2.220446049250313e-16);
    if (issue) {
        state.activity_streak++;
        state.quiet_streak = 0;
        state.floor_streak = at_floor ? state.floor_streak + 1 : 0;
    } else {
        state.activity_streak = 0;
        state.quiet_streak++;
        state.floor_streak = 0;
    }
    if (result.distribution_overshoot || state.activity_streak >= 2) {
        state.limit_scale = ctl_max(0.25, 0.5 * state.limit_scale);
        state.activity_streak = 0;
    } else if (state.quiet_streak >= 3) {
        state.limit_scale = ctl_min(1.0, 1.25 * state.limit_scale);
        state.quiet_streak = 0;
    }
    result.persistent_overshoot = state.floor_streak >= 2;
    return kCtlOk;
}

// ------------------------------------------------------------------------------------------------
// The device controller of the collision operator (gd_devctl.cu): the host controller's loop of
// evolve_local_collisions (_col_chain.cuh:215-537) as small single-block kernels between the
// operator's owner kernels, so every decision stays on the device and the waves run as the body of
// a CUDA graph conditional (while) node.
// ------------------------------------------------------------------------------------------------
struct CtlDev {
    WaveInfo wave;          // read by the owner kernels (first member: kernels take &ctl->wave)
    CtlResult res;          // accumulated until the host reads it
    double duration;
    unsigned long long tick;
    int G, S, R, n;
    int operator_count;     // operators since the last controller reset (summary numbering)
    int bath_index;         // baths of the current operator
    int ndue, wt_groups;
    int due[kCtlGroups];    // the groups due at `tick` (empty ones included)
    int group_start[kCtlGroups + 1];
    int wt_start[kCtlGroups], wt_len[kCtlGroups], wt_out[kCtlGroups];  // owner lists of this wave
    double requested[kCtlGroups], current[kCtlGroups], steps_s[kCtlGroups];
    unsigned char passed[kCtlGroups];
    BathState state[kCtlGroups];  // persists across operators until a controller reset
    int work[3 * kCtlGroups];
    SchedCore sched;
    // COL_DIAGNOSTICS bookkeeping of the current operator (_col_chain.cuh:261-289)
    struct GroupStat {
        double published, initial_request, min_request, max_request, max_age, max_ratio, max_growth, max_activity;
        unsigned long long coarsened, refined, constrained, updates;
        int initial_level, binding, overshoots, persistent;
    } gstat[kCtlGroups];
    int previous_level[kCtlGroups];
    unsigned long long log_operator;    // operators since the controller was created (never reset)
    unsigned long long op_updates, op_blocks;
    int op_waves;
    unsigned long long t_begin, t_mark0, t_mark1, t_mark2, t_mark3, chain_ns, audit_ns, rate_ns;
    double clock_sim;
};

// Device pointers the controller kernels read and write (the operator's small scratch).
struct CtlPtrs {
    const int *gcount;
    int *gcursor;
    const unsigned *graph;
    const int *binmap;
    const int *merged;
    const RateBin *ratebin;
    const AuditBin *audit;
    const int *error_flag;
    double *dt;                // bath length per group (seconds), read by the chain kernels
    BathRecord *records;
    int record_capacity;
    const double *conf_log;
    // COL_DIAGNOSTICS (all null when off)
    const int *queued;                    // [2] owners the wave's skip scan queued (front, back)
    OperatorLog *oplog;
    int oplog_capacity;
    const unsigned long long *event_count;
    const double *event_log_mass;
};

// host launchers (gd_devctl.cu)
void ctl_launch_geometry(CtlDev *c, const CtlPtrs &p, int G, cudaStream_t s);
void ctl_launch_reset(CtlDev *c, double duration, const double *duration_dev, double scale, const double *clock_sim,
                      int n, int G, int S, int R, cudaStream_t s);
void ctl_launch_clear(CtlDev *c, cudaStream_t s);
void ctl_launch_begin(CtlDev *c, const Model &m, const CtlPtrs &p, cudaGraphConditionalHandle h, cudaStream_t s);
void ctl_launch_finish(CtlDev *c, const Model &m, const CtlPtrs &p, cudaGraphConditionalHandle h, cudaStream_t s);
void ctl_launch_adapt(CtlDev *c, const Model &m, const CtlPtrs &p, cudaGraphConditionalHandle h, cudaStream_t s);
void ctl_launch_wave_ids(CtlDev *c, const int *sorted, int *ids, int grid, cudaStream_t s);
void ctl_launch_mark(CtlDev *c, int which, cudaStream_t s);  // device-time marks of COL_DIAGNOSTICS

}  // namespace gd
