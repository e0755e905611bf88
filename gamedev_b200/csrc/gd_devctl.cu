// The collision operator's controller on the device.  The reference runs it on the host between
// the waves of evolve_local_collisions (_col_chain.cuh:215-537): choose each due group's bath from
// the rate bins, place the groups on the power-of-two schedule, audit the finished baths, adapt the
// schedule and pick the next wave.  Here the same decisions run in single-block kernels between the
// owner kernels, on the same arithmetic (gd_ctl_core.cuh, this file compiled without FMA
// contraction), and the last kernel of each wave sets the CUDA graph conditional that repeats the
// wave body.  Nothing is read back between waves.
#include <cuda_runtime.h>

#include "gd_collide.cuh"
#include "gd_ctl_core.cuh"

namespace gd {

namespace {

constexpr long long kEmptyWaveLimit = 1ll << 20;  // empty waves in a row before the scheduler gives up

__device__ __forceinline__ unsigned long long device_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ void ctl_fail(CtlDev &c, int code, int detail) {
    if (!c.res.error) {
        c.res.error = code;
        c.res.error_detail = detail;
    }
    c.wave.go = 0;
    c.wave.count = 0;
}

// merged rate or audit bins of group g: [first, last)
__device__ __forceinline__ void group_bins(const CtlDev &c, const CtlPtrs &p, int g, int &first, int &last) {
    first = p.binmap[g * c.S];
    last = (g + 1 < c.G) ? p.binmap[(g + 1) * c.S] : *p.merged;
}

// The first wave with owners from the schedule's current time on: groups due with empty owner
// lists are advanced without a bath, as the host loop's `continue` does (_col_chain.cuh:246-252).
__device__ void next_wave(CtlDev &c) {
    for (long long guard = 0;; ++guard) {
        if (guard >= kEmptyWaveLimit) {
            ctl_fail(c, kCtlWaveLimit, 0);
            return;
        }
        const unsigned long long t = sched_time(c.sched);
        if (!(t < c.sched.end)) {
            c.wave.go = 0;
            c.wave.count = 0;
            return;
        }
        c.tick = t;
        c.ndue = sched_due(c.sched, t, c.due);
        // every due group publishes at the wave's time, empty ones too (_col_chain.cuh:296-301)
        const double now = sched_seconds(c.sched, t);
        for (int k = 0; k < c.ndue; ++k) c.gstat[c.due[k]].published = now;
        int count = 0, w = 0;
        for (int k = 0; k < c.ndue; ++k) {
            const int g = c.due[k];
            const int len = c.group_start[g + 1] - c.group_start[g];
            if (len == 0) continue;
            c.wt_start[w] = c.group_start[g];
            c.wt_len[w] = len;
            c.wt_out[w] = count;
            ++w;
            count += len;
        }
        c.wt_groups = w;
        if (count == 0) {
            sched_advance(c.sched, c.due, c.ndue);
            continue;
        }
        c.wave.count = count;
        c.wave.full = count == c.n ? 1 : 0;
        c.wave.go = 1;
        c.wave.need_rates = t != 0 ? 1 : 0;
        if (t != 0) c.wave.publish += 1;  // this wave publishes its reservoir
        return;
    }
}

// COL_DIAGNOSTICS statistics of the wave's nonempty due groups once their bath lengths are set
// (_col_chain.cuh:344-356): the oldest linked reservoir and the bath length over the request.
__device__ void wave_stats(CtlDev &c, const CtlPtrs &p, const double *request) {
    const double now = sched_seconds(c.sched, c.tick);
    const int words = (c.G + 31) / 32;
    for (int k = 0; k < c.ndue; ++k) {
        const int g = c.due[k];
        if (c.group_start[g + 1] == c.group_start[g]) continue;
        CtlDev::GroupStat &st = c.gstat[g];
        for (int d = 0; d < c.G; ++d)
            if (ctl_edge(p.graph, words, g, d)) st.max_age = ctl_max(st.max_age, now - c.gstat[d].published);
        st.max_ratio = ctl_max(st.max_ratio, c.steps_s[g] / request[g]);
    }
}

// the operator's record of the per-operator log (_col_chain.cuh:488-535)
__device__ void write_log(CtlDev &c, const CtlPtrs &p) {
    if (c.res.log_count >= p.oplog_capacity) {
        c.res.log_dropped += 1;
        return;
    }
    OperatorLog &r = p.oplog[c.res.log_count];
    c.res.log_count += 1;
    r.operator_id = ++c.log_operator;
    r.finest_ticks = c.sched.end;
    r.owner_updates = c.op_updates;
    r.chain_blocks = c.op_blocks;
    r.waves = c.op_waves;
    r.chain_launches = c.op_waves;
    r.G = c.G;
    r.pad = 0;
    r.clock_sim = c.clock_sim;
    r.duration = c.duration;
    r.chain_seconds = 1.0e-9 * static_cast<double>(c.chain_ns);
    r.audit_seconds = 1.0e-9 * static_cast<double>(c.audit_ns);
    r.wall_seconds = 1.0e-9 * static_cast<double>(device_ns() - c.t_begin);
    r.rate_seconds = 1.0e-9 * static_cast<double>(c.rate_ns);
    for (int k = 0; k < kEventCategories; ++k) {
        r.event_count[k] = p.event_count ? p.event_count[k] : 0ull;
        r.event_log_mass[k] = p.event_log_mass ? p.event_log_mass[k] : 0.0;
    }
    for (int g = 0; g < c.G; ++g) {
        const CtlDev::GroupStat &st = c.gstat[g];
        OperatorLogGroup &o = r.g[g];
        o.owners = c.group_start[g + 1] - c.group_start[g];
        o.level = c.sched.level[g];
        o.initial_level = st.initial_level;
        o.binding = st.binding;
        o.dt = c.steps_s[g];
        o.min_request = st.min_request;
        o.max_request = st.max_request;
        o.final_request = c.current[g];
        o.initial_request = st.initial_request;
        o.max_age = st.max_age;
        o.max_ratio = st.max_ratio;
        o.max_growth = st.max_growth;
        o.max_activity = st.max_activity;
        o.coarsened = st.coarsened;
        o.refined = st.refined;
        o.constrained = st.constrained;
        o.updates = st.updates;
        o.overshoots = st.overshoots;
        o.persistent = st.persistent;
    }
}

}  // namespace

// owner lists per group from the counting sort's counts (the host's group_start, _col_chain.cuh:162-167)
__global__ void k_ctl_geometry(CtlDev *c, CtlPtrs p, int G) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    int acc = 0;
    for (int g = 0; g < G; ++g) {
        c->group_start[g] = acc;
        p.gcursor[g] = acc;
        acc += p.gcount[g];
    }
    c->group_start[G] = acc;
}

// An operator starts: the tick-0 wave holds every particle and publishes the whole reservoir.  The
// horizon is `duration`, or scale * *duration_dev when the caller's timestep lives on the device.
__global__ void k_ctl_reset(CtlDev *c, double duration, const double *duration_dev, double scale,
                            const double *clock_sim, int n, int G, int S, int R) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (duration_dev) duration = scale * *duration_dev;
    c->clock_sim = clock_sim ? *clock_sim : 0.0;
    c->t_begin = device_ns();
    c->op_updates = c->op_blocks = 0;
    c->op_waves = 0;
    c->chain_ns = c->audit_ns = c->rate_ns = 0;
    c->duration = duration;
    c->n = n;
    c->G = G;
    c->S = S;
    c->R = R;
    c->operator_count += 1;
    c->res.operator_index = c->operator_count;
    c->bath_index = 0;
    c->tick = 0;
    c->wave.count = n;
    c->wave.full = 1;
    c->wave.go = c->res.error ? 0 : 1;  // an earlier unread error stops later operators
    c->wave.need_rates = 1;
    c->wave.publish += 1;
    // the reference's horizon check (_col_sched.cuh:30-33), before any owner kernel runs
    if (c->wave.go && (!(duration > 0) || !ctl_finite(duration))) ctl_fail(*c, kCtlBadHorizon, 0);
}

// an output boundary: default bath states, operators numbered afresh
__global__ void k_ctl_clear(CtlDev *c) {
    for (int g = threadIdx.x; g < kCtlGroups; g += blockDim.x) c->state[g] = BathState();
    if (threadIdx.x == 0) c->operator_count = 0;
}

// the bath-start rates are binned: every group's requested bath, the schedule, the first wave
__global__ void k_ctl_begin(Model m, CtlDev *cp, CtlPtrs p, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    CtlDev &c = *cp;
    if (c.wave.go) {
        int st = kCtlOk;
        for (int g = 0; g < c.G && st == kCtlOk; ++g) {
            int first, last;
            group_bins(c, p, g, first, last);
            c.gstat[g].binding = 0;
            st = ctl_choose_bath(m, p.ratebin + first, last - first, c.duration, c.state[g].limit_scale,
                                 c.requested[g], &c.gstat[g].binding);
        }
        if (st == kCtlOk) st = sched_init(c.sched, c.duration, c.requested, c.G, p.graph);
        if (st != kCtlOk) {
            ctl_fail(c, st, 0);
        } else {
            for (int g = 0; g < c.G; ++g) {
                c.steps_s[g] = sched_seconds(c.sched, c.sched.step[g]);
                c.current[g] = c.requested[g];
                c.passed[g] = 1;
                p.dt[g] = c.steps_s[g];
                CtlDev::GroupStat &gs = c.gstat[g];
                gs.published = 0.0;
                gs.initial_request = gs.min_request = gs.max_request = c.requested[g];
                gs.max_age = gs.max_ratio = gs.max_growth = gs.max_activity = 0.0;
                gs.coarsened = gs.refined = gs.constrained = gs.updates = 0;
                gs.initial_level = c.sched.level[g];
                gs.overshoots = gs.persistent = 0;
            }
            next_wave(c);
            if (c.wave.go && p.oplog) wave_stats(c, p, c.requested);
        }
    }
    cudaGraphSetConditional(h, c.wave.go ? 1u : 0u);
}

// a wave's chains and audit are done: finish its baths, advance the schedule, pick the next wave
__global__ void k_ctl_finish(Model m, CtlDev *cp, CtlPtrs p, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    CtlDev &c = *cp;
    c.res.waves += 1;
    c.res.owner_updates += c.wave.count;
    c.op_waves += 1;
    c.op_updates += c.wave.count;
    if (p.queued) c.op_blocks += static_cast<unsigned long long>(p.queued[0] + p.queued[1]);
    if (p.oplog) {
        c.chain_ns += c.t_mark1 - c.t_mark0;
        c.audit_ns += device_ns() - c.t_mark1;
    }
    const int flag = *p.error_flag;
    if (flag) {
        ctl_fail(c, 100 + flag, flag);
        cudaGraphSetConditional(h, 0u);
        return;
    }
    for (int k = 0; k < c.ndue; ++k) {
        const int g = c.due[k];
        if (c.group_start[g + 1] == c.group_start[g]) continue;
        int first, last;
        group_bins(c, p, g, first, last);
        double mass = 0.0;
        bool bad = false;
        for (int b = first; b < last; ++b) {
            if (p.audit[b].invalid_count) bad = true;
            mass += p.audit[b].mass;
        }
        if (bad) {
            ctl_fail(c, kCtlBadAudit, g);
            cudaGraphSetConditional(h, 0u);
            return;
        }
        if (!(mass > 0)) continue;
        BathResult res;
        const double before = c.state[g].limit_scale;
        const int st = ctl_finish_bath(m, p.audit + first, last - first, c.state[g], res, p.conf_log);
        if (st != kCtlOk) {
            ctl_fail(c, st, g);
            cudaGraphSetConditional(h, 0u);
            return;
        }
        c.passed[g] = !(res.activity_overshoot || res.distribution_overshoot || res.persistent_overshoot);
        CtlDev::GroupStat &gs = c.gstat[g];
        gs.updates += 1;
        gs.overshoots += (res.activity_overshoot || res.distribution_overshoot) ? 1 : 0;
        gs.persistent += res.persistent_overshoot ? 1 : 0;
        gs.max_growth = ctl_max(gs.max_growth, res.max_g);
        gs.max_activity = ctl_max(gs.max_activity, res.max_f);
        c.bath_index += 1;
        if (c.res.rec_count < p.record_capacity) {
            BathRecord &r = p.records[c.res.rec_count];
            r.group_index = g;
            r.operator_index = c.res.operator_index;
            r.bath_index = c.bath_index;
            r.merged_bins = last - first;
            r.continuation_launches = 0;
            r.duration = c.steps_s[g];
            r.limit_before = before;
            r.limit_after = c.state[g].limit_scale;
            r.result = res;
            c.res.rec_count += 1;
        } else {
            c.res.rec_dropped += 1;
        }
    }
    for (int k = 0; k < c.ndue; ++k) {
        const double d = c.steps_s[c.due[k]];
        c.res.min_duration = c.res.min_duration < d ? c.res.min_duration : d;
        c.res.max_duration = c.res.max_duration > d ? c.res.max_duration : d;
    }
    sched_advance(c.sched, c.due, c.ndue);
    next_wave(c);
    // the operator ends normally: its record of the per-operator log
    if (!c.wave.go && !c.res.error && p.oplog) write_log(c, p);
    cudaGraphSetConditional(h, c.wave.go ? 1u : 0u);
}

// a later wave's rates are binned: its groups' baths, the adapted schedule, the bath lengths
__global__ void k_ctl_adapt(Model m, CtlDev *cp, CtlPtrs p, cudaGraphConditionalHandle h) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    CtlDev &c = *cp;
    if (!c.wave.go || !c.wave.need_rates) return;
    int st = kCtlOk;
    for (int k = 0; k < c.ndue && st == kCtlOk; ++k) {
        const int g = c.due[k];
        int first, last;
        group_bins(c, p, g, first, last);
        st = ctl_choose_bath(m, p.ratebin + first, last - first, c.duration, c.state[g].limit_scale, c.current[g],
                             nullptr);
        CtlDev::GroupStat &gs = c.gstat[g];
        gs.min_request = ctl_min(gs.min_request, c.current[g]);
        gs.max_request = ctl_max(gs.max_request, c.current[g]);
        c.previous_level[g] = c.sched.level[g];
    }
    if (st == kCtlOk) st = sched_adapt(c.sched, c.tick, c.due, c.ndue, c.current, c.passed, c.work);
    if (st != kCtlOk) {
        ctl_fail(c, st, 0);
        cudaGraphSetConditional(h, 0u);
        return;
    }
    for (int k = 0; k < c.ndue; ++k) {
        const int g = c.due[k];
        c.steps_s[g] = sched_seconds(c.sched, c.sched.step[g]);
        CtlDev::GroupStat &gs = c.gstat[g];
        gs.coarsened += c.sched.level[g] < c.previous_level[g] ? 1 : 0;
        gs.refined += c.sched.level[g] > c.previous_level[g] ? 1 : 0;
        gs.constrained += c.steps_s[g] > c.current[g] ? 1 : 0;
    }
    for (int g = 0; g < c.G; ++g) p.dt[g] = c.steps_s[g];
    if (p.oplog) {
        wave_stats(c, p, c.current);
        c.rate_ns += c.t_mark3 - c.t_mark2;
    }
}

// device time at the start of a wave's chains (0), of its audit (1), of the next wave's reservoir
// publish and rates (2) and at their end (3)
__global__ void k_ctl_mark(CtlDev *c, int which) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || !c->wave.go) return;
    const unsigned long long t = device_ns();
    if (which == 0) c->t_mark0 = t;
    else if (which == 1) c->t_mark1 = t;
    else if (which == 2) c->t_mark2 = t;
    else c->t_mark3 = t;
}

// the wave's owners: the owner lists of its nonempty due groups, concatenated
__global__ void k_ctl_wave_ids(const CtlDev *c, const int *__restrict__ sorted, int *__restrict__ ids) {
    if (!c->wave.go) return;
    const int total = c->wave.count;
    const int groups = c->wt_groups;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x) {
        int lo = 0, hi = groups - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (c->wt_out[mid] <= q) lo = mid;
            else hi = mid - 1;
        }
        ids[q] = sorted[c->wt_start[lo] + (q - c->wt_out[lo])];
    }
}

void ctl_launch_geometry(CtlDev *c, const CtlPtrs &p, int G, cudaStream_t s) { k_ctl_geometry<<<1, 32, 0, s>>>(c, p, G); }
void ctl_launch_reset(CtlDev *c, double duration, const double *duration_dev, double scale, const double *clock_sim,
                      int n, int G, int S, int R, cudaStream_t s) {
    k_ctl_reset<<<1, 32, 0, s>>>(c, duration, duration_dev, scale, clock_sim, n, G, S, R);
}
void ctl_launch_clear(CtlDev *c, cudaStream_t s) { k_ctl_clear<<<1, 256, 0, s>>>(c); }
void ctl_launch_mark(CtlDev *c, int which, cudaStream_t s) { k_ctl_mark<<<1, 32, 0, s>>>(c, which); }
void ctl_launch_begin(CtlDev *c, const Model &m, const CtlPtrs &p, cudaGraphConditionalHandle h, cudaStream_t s) {
    k_ctl_begin<<<1, 32, 0, s>>>(m, c, p, h);
}
void ctl_launch_finish(CtlDev *c, const Model &m, const CtlPtrs &p, cudaGraphConditionalHandle h, cudaStream_t s) {
    k_ctl_finish<<<1, 32, 0, s>>>(m, c, p, h);
}
void ctl_launch_adapt(CtlDev *c, const Model &m, const CtlPtrs &p, cudaGraphConditionalHandle h, cudaStream_t s) {
    k_ctl_adapt<<<1, 32, 0, s>>>(m, c, p, h);
}
void ctl_launch_wave_ids(CtlDev *c, const int *sorted, int *ids, int grid, cudaStream_t s) {
    k_ctl_wave_ids<<<grid, 256, 0, s>>>(c, sorted, ids);
}

}  // namespace gd
