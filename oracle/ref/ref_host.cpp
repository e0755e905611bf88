// Host entry points over the reference's own collision headers (compiled from the GameDev tree by
// oracle/ref/Makefile), used as golden sources for the oracle and the library's host controller.
// TEST INFRASTRUCTURE ONLY.
#include <cstring>
#include <stdexcept>
#include <vector>

#include <_col_bound.cuh>
#include <_col_event.cuh>
#include <_col_rates.cuh>
#include <_col_sched.cuh>

extern "C" {

int ref_n_k() { return N_K; }

void ref_env(double y, double z, double *out8) {
#ifdef COL_QUERY_ENV_CACHE
    swarm p{};
    p.position.y = y;
    p.position.z = z;
    query_environment e = _cache_query_environment(p);
    const double v[8] = {e.Z, e.omega, e.vn, e.radial, e.strat, e.cs, e.re_inv_sqrt, e.vg_sq};
    std::memcpy(out8, v, sizeof(v));
#else
    (void)y; (void)z;
    for (int k = 0; k < 8; ++k) out8[k] = 0.0;
#endif
}

// _get_col_chain_rate(...) / measure for owner 0 and partner 1, and the pair speed it used
double ref_pair_rate(double yi, double zi, double yj, double zj, double size_i, double size_j, double numr_j,
                     double lambda0, double measure, double *vrel) {
    swarm p[2] = {};
    p[0].position.y = yi;
    p[0].position.z = zi;
    p[1].position.y = yj;
    p[1].position.z = zj;
    double size_old[2] = {size_i, size_j};
    double numr_old[2] = {1.0, numr_j};
#ifdef COL_QUERY_ENV_CACHE
    query_environment env[2] = {_cache_query_environment(p[0]), _cache_query_environment(p[1])};
#else
    query_environment *env = nullptr;
#endif
    double v = 0.0;
    double r = _get_col_chain_rate<static_cast<kernel_type>(COAG_KERNEL)>(p, size_i, size_old, numr_old, 0, 1, 0,
                                                                         lambda0, v, env);
    *vrel = v;
    return r / measure;
}

double ref_outcome_moments(double si, double sj, int high, double *out3) {
    double m = 0, s = 0, x = 0;
    double f = _erosion_outcome_moments(si, sj, high != 0, m, s, x);
    out3[0] = m;
    out3[1] = s;
    out3[2] = x;
    return f;
}

double ref_sample_outcome(double si, double sj, int high, double u) {
    int category;
    double log_mass;
    return _sample_erosion_outcome(si, sj, high != 0, u, category, log_mass);
}

double ref_ball_measure(double y, double z, double radius) { return _get_ball_measure(y, z, radius); }

int ref_raw_count() { return _get_col_raw_count(); }

int ref_binmap(const int *raw, int n, int *out) {
    std::vector<int> rc(raw, raw + n), map;
    int merged = _build_col_binmap(rc, map);
    std::memcpy(out, map.data(), sizeof(int) * n);
    return merged;
}

// bins: [n][6] = mass, weighted_rate, weighted_change, weighted_second, owner_count, invalid_count
int ref_choose_bath(const double *bins, int n, double remaining, double limit_scale, double *out, int *binding) {
    std::vector<col_rate_bin> v(n);
    for (int b = 0; b < n; ++b) {
        v[b].mass = bins[6 * b + 0];
        v[b].weighted_rate = bins[6 * b + 1];
        v[b].weighted_change = bins[6 * b + 2];
        v[b].weighted_second = bins[6 * b + 3];
        v[b].owner_count = static_cast<int>(bins[6 * b + 4]);
        v[b].invalid_count = static_cast<int>(bins[6 * b + 5]);
    }
    try {
        *out = _choose_col_bath(v, n, remaining, limit_scale, binding);
    } catch (const std::exception &) {
        return 1;
    }
    return 0;
}

// audit: [n][15] in col_audit_accum field order; state4: limit_scale, activity, quiet, floor;
// result10: max_f, max_e, max_touched, max_events, max_g, max_g_upper, d_bath, 3 overshoot flags
int ref_finish_bath(const double *audit, int n, double *state4, double *result10) {
    std::vector<col_audit_accum> v(n);
    for (int b = 0; b < n; ++b) {
        const double *a = audit + 15 * b;
        col_audit_accum &x = v[b];
        x.mass = a[0]; x.predicted_f = a[1]; x.predicted_e = a[2]; x.predicted_var_f = a[3];
        x.predicted_var_e = a[4]; x.predicted_g = a[5]; x.predicted_var_g = a[6]; x.maximum_weight = a[7];
        x.maximum_g_jump = a[8]; x.touched = a[9]; x.event_weight = a[10]; x.growth = a[11]; x.end_mass = a[12];
        x.owner_count = static_cast<int>(a[13]); x.invalid_count = static_cast<int>(a[14]);
    }
    col_bath_state st;
    st.limit_scale = state4[0];
    st.activity_streak = static_cast<int>(state4[1]);
    st.quiet_streak = static_cast<int>(state4[2]);
    st.floor_streak = static_cast<int>(state4[3]);
    col_bath_result r;
    try {
        r = _finish_col_bath(v, n, st);
    } catch (const std::exception &) {
        return 1;
    }
    state4[0] = st.limit_scale;
    state4[1] = st.activity_streak;
    state4[2] = st.quiet_streak;
    state4[3] = st.floor_streak;
    const double o[10] = {r.max_f, r.max_e, r.max_touched, r.max_events, r.max_g, r.max_g_upper, r.d_bath,
                          double(r.activity_overshoot), double(r.distribution_overshoot),
                          double(r.persistent_overshoot)};
    std::memcpy(result10, o, sizeof(o));
    return 0;
}

// scheduler: opaque local_schedule
void *ref_schedule_create(double h, const double *requested, int n, const unsigned *edges, int *status) {
    std::vector<double> req(requested, requested + n);
    std::vector<unsigned> e(edges, edges + n * ((n + 31) / 32));
    try {
        *status = 0;
        return new local_schedule(h, req, e);
    } catch (const std::exception &) {
        *status = 1;
        return nullptr;
    }
}
void ref_schedule_destroy(void *s) { delete static_cast<local_schedule *>(s); }
unsigned long long ref_schedule_time(void *s) { return static_cast<local_schedule *>(s)->time(); }
unsigned long long ref_schedule_end(void *s) { return static_cast<local_schedule *>(s)->end; }
int ref_schedule_due(void *s, unsigned long long tick, int *out) {
    auto v = static_cast<local_schedule *>(s)->due(tick);
    for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
    return static_cast<int>(v.size());
}
int ref_schedule_adapt(void *s, unsigned long long tick, const int *groups, int ng, const double *requested,
                       const int *passed) {
    auto *sc = static_cast<local_schedule *>(s);
    const int n = static_cast<int>(sc->level.size());
    std::vector<int> g(groups, groups + ng);
    std::vector<double> req(requested, requested + n);
    std::vector<bool> pass(n);
    for (int c = 0; c < n; ++c) pass[c] = passed[c] != 0;
    try {
        sc->adapt(tick, g, req, pass);
    } catch (const std::exception &) {
        return 1;
    }
    return 0;
}
void ref_schedule_advance(void *s, const int *groups, int ng) {
    static_cast<local_schedule *>(s)->advance(std::vector<int>(groups, groups + ng));
}
void ref_schedule_levels(void *s, int *out) {
    auto *sc = static_cast<local_schedule *>(s);
    for (size_t c = 0; c < sc->level.size(); ++c) out[c] = sc->level[c];
}

}  // extern "C"
