// Exported host controller (include/gd_b200_controller.h): thin C wrappers over the controller
// arithmetic the collision operator's device controller runs (gd_ctl_core.cuh), here on the host.
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include "../../include/gd_b200_controller.h"
#include "gd_collide.cuh"
#include "gd_ctl_core.cuh"

struct gd_schedule {
    gd::SchedCore s;
};

extern "C" {

int gd_ctl_binmap(int groups, int bins, int bin_min, const int *raw, int *out) {
    if (groups <= 0 || bins <= 0 || !raw || !out) return -1;
    gd::Model m{};
    m.local_groups = groups;
    m.col_bin_s = bins;
    m.col_bin_min = bin_min;
    std::vector<int> rc(raw, raw + groups * bins), map;
    int merged = gd::build_binmap(m, rc, map);
    std::memcpy(out, map.data(), sizeof(int) * map.size());
    return merged;
}

gd_status gd_ctl_choose_bath(const gd_config *cfg, const double *bins, int n, double remaining, double limit_scale,
                             double *out, int *binding) {
    if (!cfg || (!bins && n) || !out || n < 0) return GD_ERR_INVALID_ARGUMENT;
    gd::Model m = gd::make_model(*cfg);
    std::vector<gd::RateBin> v(n);
    for (int b = 0; b < n; ++b) {
        v[b].mass = bins[6 * b + 0];
        v[b].weighted_rate = bins[6 * b + 1];
        v[b].weighted_change = bins[6 * b + 2];
        v[b].weighted_second = bins[6 * b + 3];
        v[b].owner_count = static_cast<int>(bins[6 * b + 4]);
        v[b].invalid_count = static_cast<int>(bins[6 * b + 5]);
    }
    gd::Status s = gd::choose_bath(m, v.data(), n, remaining, limit_scale, *out, binding);
    return s.code;
}

gd_status gd_ctl_finish_bath(const gd_config *cfg, const double *audit, int n, double *state, double *result) {
    if (!cfg || !audit || !state || !result || n < 0) return GD_ERR_INVALID_ARGUMENT;
    gd::Model m = gd::make_model(*cfg);
    std::vector<gd::AuditBin> v(n);
    for (int b = 0; b < n; ++b) {
        const double *a = audit + 15 * b;
        gd::AuditBin &x = v[b];
        x.mass = a[0]; x.predicted_f = a[1]; x.predicted_e = a[2]; x.predicted_var_f = a[3];
        x.predicted_var_e = a[4]; x.predicted_g = a[5]; x.predicted_var_g = a[6]; x.maximum_weight = a[7];
        x.maximum_g_jump = a[8]; x.touched = a[9]; x.event_weight = a[10]; x.growth = a[11]; x.end_mass = a[12];
        x.owner_count = static_cast<int>(a[13]); x.invalid_count = static_cast<int>(a[14]);
    }
    gd::BathState st;
    st.limit_scale = state[0];
    st.activity_streak = static_cast<int>(state[1]);
    st.quiet_streak = static_cast<int>(state[2]);
    st.floor_streak = static_cast<int>(state[3]);
    gd::BathResult r;
    gd::Status s = gd::finish_bath(m, v.data(), n, st, r);
    if (!s) return s.code;
    state[0] = st.limit_scale;
    state[1] = st.activity_streak;
    state[2] = st.quiet_streak;
    state[3] = st.floor_streak;
    const double o[10] = {r.max_f, r.max_e, r.max_touched, r.max_events, r.max_g, r.max_g_upper, r.d_bath,
                          double(r.activity_overshoot), double(r.distribution_overshoot),
                          double(r.persistent_overshoot)};
    std::memcpy(result, o, sizeof(o));
    return GD_OK;
}

gd_schedule *gd_ctl_schedule_create(double horizon, const double *requested, int n, const unsigned *edges,
                                    gd_status *status) {
    if (!requested || !edges || n <= 0 || n > gd::kCtlGroups) {
        if (status) *status = GD_ERR_INVALID_ARGUMENT;
        return nullptr;
    }
    gd_schedule *s = new (std::nothrow) gd_schedule();
    if (!s) {
        if (status) *status = GD_ERR_OUT_OF_MEMORY;
        return nullptr;
    }
    const gd::Status st = gd::ctl_status(gd::sched_init(s->s, horizon, requested, n, edges));
    if (status) *status = st.code;
    if (!st) {
        delete s;
        return nullptr;
    }
    return s;
}

void gd_ctl_schedule_destroy(gd_schedule *s) { delete s; }
unsigned long long gd_ctl_schedule_time(const gd_schedule *s) { return s ? gd::sched_time(s->s) : 0ull; }
unsigned long long gd_ctl_schedule_end(const gd_schedule *s) { return s ? s->s.end : 0ull; }

int gd_ctl_schedule_due(const gd_schedule *s, unsigned long long tick, int *groups) {
    if (!s) return 0;
    int due[gd::kCtlGroups];
    const int k = gd::sched_due(s->s, tick, due);
    if (groups) std::memcpy(groups, due, sizeof(int) * k);
    return k;
}

gd_status gd_ctl_schedule_adapt(gd_schedule *s, unsigned long long tick, const int *groups, int n_groups,
                                const double *requested, const int *passed) {
    if (!s || (!groups && n_groups) || !requested || !passed || n_groups < 0 || n_groups > s->s.n)
        return GD_ERR_INVALID_ARGUMENT;
    const int n = s->s.n;
    std::vector<unsigned char> pass(n);
    for (int c = 0; c < n; ++c) pass[c] = passed[c] != 0;
    std::vector<int> work(3 * static_cast<size_t>(n));
    return gd::ctl_status(gd::sched_adapt(s->s, tick, groups, n_groups, requested, pass.data(), work.data())).code;
}

void gd_ctl_schedule_advance(gd_schedule *s, const int *groups, int n_groups) {
    if (!s || !groups || n_groups < 0) return;
    gd::sched_advance(s->s, groups, n_groups);
}

void gd_ctl_schedule_levels(const gd_schedule *s, int *levels) {
    if (!s || !levels) return;
    for (int c = 0; c < s->s.n; ++c) levels[c] = s->s.level[c];
}

}  // extern "C"
