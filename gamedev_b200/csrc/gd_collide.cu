// Frozen-bath collision operator on sm_100a (evolve_local_collisions, _col_chain.cuh:108-539).
//
// Kernels (reference kernel in brackets):
//   k_env_cache      [col_env_cache, col_env_cache.cu:15-20]     thread per owner
//   k_bath_init      [col_bath_init + col_comp_zero]             thread per owner
//   k_size_*         [col_size_zero/scan/bnds]                   moving log-size bin bounds
//   k_rate_plan      [none: this build keeps unchanged rates]    WARP per 32 owners: whole, changed
//                                                                pairs only, or standing
//   k_bath_rate      [col_bath_rate, col_bath_rate.cu:13-130]    WARP per owner, exact fold order
//   k_pair_eval, k_rate_fold [col_bath_rate's pair terms, fold]  thread per changed pair; WARP per
//                                                                owner folding its stored pairs
//   k_count_bin, k_binmap, k_rate_bins [col_count_bin, _build_col_binmap, col_rate_bins]
//   k_skip_scan      [col_skip_scan, col_skip_scan.cu:13-59]     thread per owner
//   k_chain          [col_chain_run, col_chain_run.cu:21-404]    persistent WARPS over a device queue,
//                                                                each owner run to the end of its bath
//   k_audit_bin      [col_audit_bin, col_audit_bin.cu:13-60]
//   k_group_*, k_dep_graph [host owner lists + col_dep_graph]   device counting sort by group
//
// Differences in mechanism (results per owner are the same):
//   * The reference relaunches col_chain_run with a 32-event cap and a device->host read of the
//     unfinished count after every launch (_col_chain.cuh:379-402).  Its own test shows caps 1 and
//     32 give identical particle and RNG hashes, so here one persistent launch runs every queued
//     owner to its bath end, with a bounded event budget that reports GD_ERR_CONTINUATION_LIMIT.
//   * The queued owner repeats the skip-scan trial draw and restores it (col_chain_run.cu:91-124);
//     that shortcut can only restore the state, so it is not repeated here.
//   * One warp holds one owner: the K frozen partners (size_old, numr_old, vertical scale) are
//     loaded into registers once per owner instead of once per event, the rate folds use the
//     reference's (count+1)/2 pairing in warp-private shared memory, and every lane replays the
//     serial partner walk and the XORWOW draws on an identical RNG copy, so no lane waits.
#include <math_constants.h>

#include <cfloat>
#include <algorithm>
#include <climits>
#include <cmath>
#include <iomanip>
#include <sstream>
#include <cstring>
#include <limits>
#include <memory>
#include <string>

#include "gd_collide.cuh"
#include "gd_ctl_core.cuh"
#include "gd_physics.cuh"

namespace gd {

constexpr int kMaxSlots = kMaxK / 32;  // neighbour slots per lane
constexpr int kMaxGroups = 256;
constexpr int kChainWarps = 4;
constexpr int kChainDoubles = 5;  // doubles per slot of a chain warp's staging: rates and folds
constexpr long long kEventBudget = 1ll << 22;  // events per owner per bath before giving up
constexpr double kHeavyEvents = 16.0;          // expected events that put an owner at the queue's front

// ------------------------------------------------------------------------------------------------
// device scratch layout: one block copied to pinned host memory with one cudaMemcpyAsync
// ------------------------------------------------------------------------------------------------
struct Small {
    size_t merged;       // int
    size_t error_flag;   // int
    size_t queued;       // int: owners the skip scan queued from the front (expected work above the cut)
    size_t light;        // int: owners queued from the back (the rest)
    size_t head;         // int
    size_t events;       // unsigned long long
    size_t pair_count;   // int: changed pairs listed for k_pair_eval this wave
    size_t fold_count;   // int: owners listed for k_rate_fold this wave
    size_t whole_count;  // int: owners listed for k_bath_rate (evaluated whole) this wave
    size_t binmap;       // int[raw]
    size_t ratebin;      // RateBin[raw]
    size_t audit;        // AuditBin[raw]
    size_t counts;       // int[raw]
    size_t dt;           // double[G]
    size_t mmin, mmax;   // u64[G]
    size_t lower, upper; // double[G]
    size_t graph;        // u32[G*words]
    size_t gcount;       // int[G]
    size_t gcursor;      // int[G]
    size_t total;
};

static size_t align256(size_t v) { return (v + 255) / 256 * 256; }

static Small small_layout(const Model &m) {
    Small L;
    const int G = m.local_groups, R = m.raw_bins, W = (G + 31) / 32;
    size_t o = 0;
    L.merged = o; o += 4;
    L.error_flag = o; o += 4;
    L.queued = o; o += 4;
    L.light = o; o += 4;
    L.head = o; o += 4;
    o += 4;
    L.events = o; o += 8;
    L.pair_count = o; o += 4;
    L.fold_count = o; o += 4;
    L.whole_count = o; o += 4;
    o = align256(o);
    L.binmap = o; o = align256(o + 4 * R);
    L.ratebin = o; o = align256(o + sizeof(RateBin) * R);
    L.audit = o; o = align256(o + sizeof(AuditBin) * R);
    L.counts = o; o = align256(o + 4 * R);
    L.dt = o; o = align256(o + 8 * G);
    L.mmin = o; o = align256(o + 8 * G);
    L.mmax = o; o = align256(o + 8 * G);
    L.lower = o; o = align256(o + 8 * G);
    L.upper = o; o = align256(o + 8 * G);
    L.graph = o; o = align256(o + 4 * G * W);
    L.gcount = o; o = align256(o + 4 * G);
    L.gcursor = o; o = align256(o + 4 * G);
    L.total = o;
    return L;
}

template <typename T>
static T *at(DevBuf<unsigned char> &b, size_t off) {
    return reinterpret_cast<T *>(b.ptr + off);
}
template <typename T>
static T *at(unsigned char *b, size_t off) {
    return reinterpret_cast<T *>(b + off);
}

// ------------------------------------------------------------------------------------------------
// small per-owner kernels
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ int owner_at(const int *ids, int slot) { return ids ? ids[slot] : slot; }

__global__ void k_env_cache(Model m, int n, const gd_particle *__restrict__ part, Env *__restrict__ env) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && part[i].position[1] > 0.0) env[i] = make_env(m, part[i].position[1], part[i].position[2]);
}

// R h_g(R) of every particle (the partner term of the N_Z = 1 physical kernel, _col_rates.cuh:205-210),
// once per geometry epoch: positions do not change inside an operator.
__global__ void k_disk_height(Model m, int n, const gd_particle *__restrict__ part, double *__restrict__ height) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double R = cyl_R(m, part[i].position[1], part[i].position[2]);
        height[i] = R * get_hg(m, R);
    }
}

// col_bath_init (col_bath_init.cu:11-23) + col_comp_zero (col_comp_zero.cu:11-19)
__global__ void k_bath_init(const WaveInfo *__restrict__ w, const int *__restrict__ ids,
                            const gd_particle *__restrict__ part, double *__restrict__ size_old,
                            double *__restrict__ numr_old, double *__restrict__ time, int *__restrict__ events,
                            unsigned char *__restrict__ complete, double *__restrict__ hazard,
                            double *__restrict__ jump1, double *__restrict__ jump2, double *__restrict__ jumpmax,
                            int *__restrict__ stamp) {
    if (!w->go || !w->need_rates) return;
    const int count = w->count, publish = w->publish;
    if (w->full) ids = nullptr;
    for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < count; slot += gridDim.x * blockDim.x) {
        const int i = owner_at(ids, slot);
        const double size = part[i].par_size, numr = part[i].par_numr;
        if (!(size_old[i] == size && numr_old[i] == numr)) stamp[i] = publish;  // the reservoir value changes
        size_old[i] = size;
        numr_old[i] = numr;
        time[i] = 0.0;
        events[i] = 0;
        complete[i] = 0;
        hazard[i] = jump1[i] = jump2[i] = jumpmax[i] = 0.0;
    }
}

__global__ void k_size_zero(int G, unsigned long long *mmin, unsigned long long *mmax) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < G) {
        mmin[g] = static_cast<unsigned long long>(__double_as_longlong(CUDART_INF));
        mmax[g] = 0ull;
    }
}

// Warp aggregation of the controller's per-group and per-bin atomics: the lanes holding the same
// key combine their terms with shuffles inside their group and the lowest one updates memory.
__device__ __forceinline__ unsigned int lanes_below() { return (1u << (threadIdx.x & 31)) - 1u; }

__global__ void k_size_scan(const WaveInfo *__restrict__ w, const int *__restrict__ ids,
                            const gd_particle *__restrict__ part, const int32_t *__restrict__ spatial,
                            const unsigned char *__restrict__ active, unsigned long long *mmin,
                            unsigned long long *mmax) {
    if (!w->go || !w->need_rates) return;
    const int count = w->count;
    if (w->full) ids = nullptr;
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    bool on = slot < count;
    int g = 0;
    unsigned long long bits = 0;
    if (on) {
        const int i = owner_at(ids, slot);
        const double size = part[i].par_size;
        on = active[i] && size > 0 && isfinite(size);
        if (on) {
            g = spatial[i];
            bits = static_cast<unsigned long long>(__double_as_longlong(size));
        }
    }
    const unsigned int mask = __ballot_sync(0xffffffffu, on);
    if (!on) return;
    const unsigned int peers = __match_any_sync(mask, g);
    unsigned long long lo = bits, hi = bits;
    for (unsigned int pm = peers; pm; pm &= pm - 1) {
        const unsigned long long v = __shfl_sync(peers, bits, __ffs(pm) - 1);
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
    }
    if ((peers & lanes_below()) == 0) {
        atomicMin(&mmin[g], lo);
        atomicMax(&mmax[g], hi);
    }
}

__global__ void k_size_bnds(int G, const unsigned long long *mmin, const unsigned long long *mmax, double *lower,
                            double *upper) {
    int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < G && mmax[g] != 0) {
        lower[g] = 0.5 * __longlong_as_double(static_cast<long long>(mmin[g]));
        upper[g] = 8.0 * __longlong_as_double(static_cast<long long>(mmax[g]));
    }
}

// _get_col_sizebin (inc/swarm/_col_sizes.cuh:16-21)
__device__ __forceinline__ int size_bin(const Model &m, double size, const double *lower, const double *upper, int g) {
    if (!isfinite(size) || !(size > 0)) return 0;
    double fraction = log(size / lower[g]) / log(upper[g] / lower[g]);
    return max(0, min(m.col_bin_s - 1, static_cast<int>(floor(fraction * m.col_bin_s))));
}

__global__ void k_count_bin(Model m, const WaveInfo *__restrict__ w, const int *__restrict__ ids,
                            int *__restrict__ counts, const gd_particle *__restrict__ part,
                            const int32_t *__restrict__ spatial, const unsigned char *__restrict__ active,
                            const double *lower, const double *upper) {
    if (!w->go || !w->need_rates) return;
    const int count = w->count;
    if (w->full) ids = nullptr;
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    bool on = slot < count;
    int key = 0;
    if (on) {
        const int i = owner_at(ids, slot);
        on = active[i] != 0;
        if (on) {
            const int g = spatial[i];
            key = g * m.col_bin_s + size_bin(m, part[i].par_size, lower, upper, g);
        }
    }
    const unsigned int mask = __ballot_sync(0xffffffffu, on);
    if (!on) return;
    const unsigned int peers = __match_any_sync(mask, key);
    if ((peers & lanes_below()) == 0) atomicAdd(counts + key, __popc(peers));
}

// _build_col_binmap (inc/swarm/_col_bound.cuh:232-285): merge adjacent sparse size bins inside
// every spatial group.  Runs on the host (tests) and in a one-thread kernel.
__host__ __device__ inline int binmap_compute(int groups, int bins, int bin_min, const int *raw_count, int *raw_to_merged) {
    for (int i = 0; i < groups * bins; ++i) raw_to_merged[i] = -1;
    int merged = 0;
    for (int sp = 0; sp < groups; ++sp) {
        int last = -1;
        for (int b = 0; b < bins; ++b)
            if (raw_count[sp * bins + b] > 0) last = b;
        if (last < 0) {
            int id = merged++;
            for (int b = 0; b < bins; ++b) raw_to_merged[sp * bins + b] = id;
            continue;
        }
        int begin = 0, previous = -1;
        while (begin <= last) {
            int end = begin, count = 0;
            while (end <= last && count < bin_min) count += raw_count[sp * bins + end++];
            bool merge_tail = end > last && count < bin_min && previous >= 0;
            int id = merge_tail ? previous : merged++;
            for (int b = begin; b < end; ++b) raw_to_merged[sp * bins + b] = id;
            previous = id;
            begin = end;
        }
        if (last + 1 < bins) {
            int id = merged++;
            for (int b = last + 1; b < bins; ++b) raw_to_merged[sp * bins + b] = id;
        }
    }
    return merged;
}

__global__ void k_binmap(Model m, const WaveInfo *__restrict__ w, const int *counts, int *binmap, int *merged) {
    if (!w->go || !w->need_rates) return;
    if (blockIdx.x == 0 && threadIdx.x == 0) *merged = binmap_compute(m.local_groups, m.col_bin_s, m.col_bin_min, counts, binmap);
}

__global__ void k_rate_bins(Model m, const WaveInfo *__restrict__ w, const int *__restrict__ ids,
                            RateBin *__restrict__ bin, const gd_particle *__restrict__ part,
                            const double *__restrict__ rate, const double *__restrict__ change,
                            const double *__restrict__ second, const int32_t *__restrict__ spatial,
                            const int *__restrict__ binmap, const unsigned char *__restrict__ active,
                            const double *lower, const double *upper) {
    if (!w->go || !w->need_rates) return;
    const int count = w->count;
    if (w->full) ids = nullptr;
    const int slot = blockIdx.x * blockDim.x + threadIdx.x;
    bool on = slot < count;
    int b = 0;
    bool valid = false;
    double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
    if (on) {
        const int i = owner_at(ids, slot);
        on = active[i] != 0;
        if (on) {
            const int g = spatial[i];
            b = binmap[g * m.col_bin_s + size_bin(m, part[i].par_size, lower, upper, g)];
            const double weight = part[i].par_numr * grain_mass(m, part[i].par_size);
            valid = !(!isfinite(weight) || !(weight > 0.0) || !isfinite(rate[i]) || rate[i] < 0.0 ||
                      !isfinite(change[i]) || change[i] < 0 || !isfinite(second[i]) || second[i] < 0);
            if (valid) {
                t0 = weight;
                t1 = weight * rate[i];
                t2 = weight * change[i];
                t3 = weight * second[i];
            }
        }
    }
    const unsigned int mask = __ballot_sync(0xffffffffu, on);
    const unsigned int vmask = __ballot_sync(0xffffffffu, valid);
    if (!on) return;
    const unsigned int peers = __match_any_sync(mask, b);
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    for (unsigned int pm = peers; pm; pm &= pm - 1) {
        const int l = __ffs(pm) - 1;
        s0 += __shfl_sync(peers, t0, l);
        s1 += __shfl_sync(peers, t1, l);
        s2 += __shfl_sync(peers, t2, l);
        s3 += __shfl_sync(peers, t3, l);
    }
    if ((peers & lanes_below()) == 0) {
        atomicAdd(&bin[b].owner_count, __popc(peers));
        const int invalid = __popc(peers & ~vmask);
        if (invalid) atomicAdd(&bin[b].invalid_count, invalid);
        if (peers & vmask) {
            atomicAdd(&bin[b].mass, s0);
            atomicAdd(&bin[b].weighted_rate, s1);
            atomicAdd(&bin[b].weighted_change, s2);
            atomicAdd(&bin[b].weighted_second, s3);
        }
    }
}

// ------------------------------------------------------------------------------------------------
// per-owner context shared by the bath-rate and chain kernels
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ OwnerCtx owner_ctx(const Model &m, const gd_particle *part, const Env *env, int i,
                                              double measure, double lambda0) {
    OwnerCtx o;
    o.y = part[i].position[1];
    o.z = part[i].position[2];
    // the disk height enters only the vertically integrated (N_Z = 1) physical kernel
    o.H_i = 0.0;
    if (m.n_z == 1) {
        const double R = cyl_R(m, o.y, o.z);
        o.H_i = R * get_hg(m, R);
    }
    o.measure = measure;
    o.lambda0 = lambda0;
    if (env && m.coag_kernel == GD_KERNEL_CUSTOM) o.env = env[i];
    return o;
}

// in-place (count+1)/2 fold of a warp-private array (col_bath_rate.cu:105-118)
template <typename F>
__device__ __forceinline__ void warp_fold(int K, int lane, F &&combine) {
    for (int count = K; count > 1; count = (count + 1) / 2) {
        const int half = (count + 1) / 2;
        for (int j = lane; j < count / 2; j += 32) combine(j, j + half);
        __syncwarp();
    }
}

// pair_rate with the partner's disk height (N_Z = 1 physical kernel) read from the per-particle
// array k_disk_height fills, and the owner's Stokes terms of the cached physical kernel passed in
// (evaluated once per owner, or once per event in the chain).  The same operations as pair_rate,
// so the same bits.
// kPhys: the caller knows at compile time that the model is the physical kernel on the cached
// environment, and the synthetic kernels and the direct pair speed are left out of the code.
template <bool kPhys = false>
__device__ __forceinline__ double chain_pair_rate(const Model &m, const OwnerCtx &o, const PairOwner &po,
                                                  double size_i, double size_j, double numr_j, double H_gj,
                                                  double &vrel, const PairPartner *pre = nullptr) {
    if constexpr (kPhys) {
        vrel = pre ? cached_pair_speed_pp(m, o.env, po, *pre) : cached_pair_speed_o(m, o.env, po, size_j);
        double r = numr_j * vrel * M_PI * (size_i + size_j) * (size_i + size_j) / 4.0;
        if (m.n_z == 1) r /= sqrt(2.0 * M_PI * (o.H_i * o.H_i + H_gj * H_gj));
        return r / o.measure;
    }
    vrel = 0.0;
    double r;
    if (m.coag_kernel == GD_KERNEL_CONSTANT) {
        r = o.lambda0 * numr_j;
    } else if (m.coag_kernel == GD_KERNEL_LINEAR) {
        r = o.lambda0 * numr_j * (grain_mass(m, size_i) + grain_mass(m, size_j));
    } else if (m.coag_kernel == GD_KERNEL_PRODUCT) {
        r = o.lambda0 * numr_j * grain_mass(m, size_i) * grain_mass(m, size_j);
    } else {
        if (use_env_cache(m))
            vrel = pre ? cached_pair_speed_pp(m, o.env, po, *pre) : cached_pair_speed_o(m, o.env, po, size_j);
        else
            vrel = direct_pair_speed(m, o.y, o.z, size_i, size_j);
        r = numr_j * vrel * M_PI * (size_i + size_j) * (size_i + size_j) / 4.0;
        if (m.n_z == 1) r /= sqrt(2.0 * M_PI * (o.H_i * o.H_i + H_gj * H_gj));
    }
    return r / o.measure;
}

struct RateArgs {
    const int *ids;
    const double *height;  // R h_g(R) per particle (N_Z = 1 physical kernel), else null
    const WaveInfo *w;  // the wave's owner count and order, and its publish wave
    const gd_particle *part;
    const int32_t *codes;
    const double *measure;
    const unsigned char *active;
    const double *size_old;
    const double *numr_old;
    const Env *env;
    double lambda0;
    double *rate, *change, *second;
    RateMoments *cached;
    const int *stamp;   // publish wave of each particle's last reservoir change
    int *rated;         // publish wave of each owner's stored rates (-1: none)
    // Stored pairs: plane p of `leaf` (planes `plane` = n*K doubles apart) holds each pair's rate,
    // rate*mean, rate*second and maximum (p = 0..3) at owner*K + slot, or null.  With the lists,
    // k_rate_plan sorts the wave's owners first: an owner whose own entry is unchanged has its
    // changed pairs (owner*K + slot) listed in `pairs` and itself in `folds`, for k_pair_eval and
    // k_rate_fold; `whole` lists the owners evaluated whole (their own entry changed, or never
    // rated on this geometry), which k_bath_rate then runs.  Null lists: k_bath_rate checks and
    // evaluates the wave's owners itself.
    double *leaf;
    size_t plane;
    unsigned int *pairs;
    int *pair_count;
    int *folds;
    int *fold_count;
    int *whole;
    int *whole_count;
};

__device__ __forceinline__ void store_pair(const RateArgs &a, size_t e, double r, double c, double sc, double mx) {
    a.leaf[e] = r;
    a.leaf[a.plane + e] = c;
    a.leaf[2 * a.plane + e] = sc;
    a.leaf[3 * a.plane + e] = mx;
}

// The warp's staged pairs of owner i folded in slot order's (count+1)/2 tree and written as its
// stored bath-start rates (col_bath_rate.cu:105-129).
__device__ __forceinline__ void fold_owner(const RateArgs &a, int K, int lane, int i, int publish, double *rate_w,
                                           double *change_w, double *second_w, double *max_w, int *valid_w) {
    __syncwarp();
    warp_fold(K, lane, [&](int j, int h) {
        rate_w[j] += rate_w[h];
        change_w[j] += change_w[h];
        second_w[j] += second_w[h];
        max_w[j] = fmax(max_w[j], max_w[h]);
        valid_w[j] = valid_w[j] && valid_w[h];
    });
    if (lane == 0) {
        RateMoments cm;
        cm.rate = valid_w[0] ? rate_w[0] : -1.0;
        cm.first = change_w[0];
        cm.second = second_w[0];
        cm.maximum = max_w[0];
        a.cached[i] = cm;
        a.rate[i] = rate_w[0];
        a.change[i] = change_w[0];
        a.second[i] = second_w[0];
        a.rated[i] = publish;
    }
    __syncwarp();  // the warp's staging is rewritten by its next owner
}

// col_bath_rate (col_bath_rate.cu:13-130): one warp per owner.  kCached selects, at compile time,
// the physical kernel on the cached environment (owner terms hoisted); the other instantiation
// serves the synthetic kernels and the uncached physical one.  Each lane takes slots s and s + 32
// and issues the gathers of both before the pair arithmetic, so their latencies overlap.  The
// FP64 pair arithmetic is latency-bound: 8 blocks per SM (64 registers, a few spilled) beat 4
// blocks at 128 registers without spills by a fifth on the c3 shapes.
// blocks of 128 per SM the bath-rate kernel is compiled for (its register budget): 8 (64 registers,
// a few spilled) measured best against 6 and 7 on the c3 and c4 shapes
#ifndef GD_RATE_BLOCKS
#define GD_RATE_BLOCKS 8
#endif

// Sorts a wave's owners for the rate pass.  Stored rates stand when neither the owner's reservoir
// entry nor any neighbour's changed since they were evaluated (same geometry and lambda0).  A
// pair's terms depend only on the owner's and the partner's entries, so when the owner's own entry
// is unchanged only the pairs of changed partners need evaluating: they go to the pair list, where
// k_pair_eval evaluates them one per thread (no lane idles on an unchanged pair), and the owner to
// the fold list, where k_rate_fold folds its K stored pairs in the same order.  Owners whose own
// entry changed go to the list k_bath_rate evaluates whole.  The same bits either way.  One warp
// per batch of 32 consecutive owner slots, one reservation per batch in each list (one per owner
// on the same counters serialised the pass).
__global__ void __launch_bounds__(256) k_rate_plan(Model m, RateArgs a) {
    if (!a.w->go || !a.w->need_rates) return;
    const int K = m.n_k;
    const int lane = threadIdx.x & 31;
    const unsigned int below = (1u << lane) - 1u;
    const int count = a.w->count;
    const int *ids = a.w->full ? nullptr : a.ids;
    const int warps = gridDim.x * (blockDim.x >> 5);
    // K <= 64: each owner's changed slots are kept as two ballots from the one scan of its row
    const bool masks = K <= 64;
    for (int base = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; base < count; base += warps * 32) {
        // the batch's owners, one per lane: lane b holds owner b's index, rating and decision
        const bool here = base + lane < count;
        const int my_i = here ? owner_at(ids, base + lane) : 0;
        const int my_rated = here ? a.rated[my_i] : 0;
        const bool my_whole = here && (my_rated < 0 || a.stamp[my_i] > my_rated);
        unsigned int my_m0 = 0u, my_m1 = 0u;  // lane b: owner b's changed slots 0-31 and 32-63
        int my_fresh = 0;
        for (unsigned int left = __ballot_sync(0xffffffffu, here && !my_whole); left; left &= left - 1) {
            const int bo = __ffs(left) - 1;
            const int i = __shfl_sync(0xffffffffu, my_i, bo);
            const int rated = __shfl_sync(0xffffffffu, my_rated, bo);
            int fresh = 0;
            unsigned int m0 = 0u, m1 = 0u;
            for (int s0 = 0; s0 < K; s0 += 32) {
                const int s = s0 + lane;
                bool f = false;
                if (s < K) {
                    const int nb = a.codes[static_cast<size_t>(i) * K + s];
                    f = nb >= 0 && a.stamp[nb / 3] > rated;
                }
                const unsigned int fm = __ballot_sync(0xffffffffu, f);
                fresh += __popc(fm);
                if (s0 == 0) m0 = fm; else m1 = fm;
            }
            if (lane == bo) {
                my_fresh = fresh;
                my_m0 = m0;
                my_m1 = m1;
            }
        }
        const bool my_listed = my_fresh > 0;
        int incl_p = my_fresh, incl_f = my_listed ? 1 : 0, incl_w = my_whole ? 1 : 0;  // lane prefixes
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int vp = __shfl_up_sync(0xffffffffu, incl_p, d);
            const int vf = __shfl_up_sync(0xffffffffu, incl_f, d);
            const int vw = __shfl_up_sync(0xffffffffu, incl_w, d);
            if (lane >= d) {
                incl_p += vp;
                incl_f += vf;
                incl_w += vw;
            }
        }
        int pbase = 0, fbase = 0, wbase = 0;
        if (lane == 31) {
            if (incl_p) pbase = atomicAdd(a.pair_count, incl_p);
            if (incl_f) fbase = atomicAdd(a.fold_count, incl_f);
            if (incl_w) wbase = atomicAdd(a.whole_count, incl_w);
        }
        pbase = __shfl_sync(0xffffffffu, pbase, 31);
        fbase = __shfl_sync(0xffffffffu, fbase, 31);
        wbase = __shfl_sync(0xffffffffu, wbase, 31);
        if (my_whole) a.whole[wbase + incl_w - 1] = my_i;
        if (my_listed) a.folds[fbase + incl_f - 1] = my_i;
        const int my_start = pbase + incl_p - my_fresh;
        for (unsigned int left = __ballot_sync(0xffffffffu, my_listed); left; left &= left - 1) {
            const int bo = __ffs(left) - 1;
            const int i = __shfl_sync(0xffffffffu, my_i, bo);
            int at = __shfl_sync(0xffffffffu, my_start, bo);
            if (masks) {
                const unsigned int m0 = __shfl_sync(0xffffffffu, my_m0, bo);
                const unsigned int m1 = __shfl_sync(0xffffffffu, my_m1, bo);
                if ((m0 >> lane) & 1u) a.pairs[at + __popc(m0 & below)] = static_cast<unsigned int>(i) * K + lane;
                at += __popc(m0);
                if ((m1 >> lane) & 1u) a.pairs[at + __popc(m1 & below)] = static_cast<unsigned int>(i) * K + 32 + lane;
                continue;
            }
            const int rated = __shfl_sync(0xffffffffu, my_rated, bo);
            for (int s0 = 0; s0 < K; s0 += 32) {
                const int s = s0 + lane;
                bool f = false;
                if (s < K) {
                    const int nb = a.codes[static_cast<size_t>(i) * K + s];
                    f = nb >= 0 && a.stamp[nb / 3] > rated;
                }
                const unsigned int fm = __ballot_sync(0xffffffffu, f);
                if (f) a.pairs[at + __popc(fm & below)] = static_cast<unsigned int>(i) * K + s;
                at += __popc(fm);
            }
        }
    }
}

template <bool kCached>
__global__ void __launch_bounds__(128, GD_RATE_BLOCKS) k_bath_rate(Model m, RateArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int K = m.n_k;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    if (!a.w->go || !a.w->need_rates) return;
    const int count = a.w->count, publish = a.w->publish;
    const int *ids = a.w->full ? nullptr : a.ids;
    // with the planner's lists, the owners to evaluate whole; without them, the wave's owners, each
    // checked here
    const bool listed = a.whole != nullptr;
    const int total = listed ? *a.whole_count : count;
    // a persistent grid: each warp takes owners strided by the number of warps
    for (int slot = blockIdx.x * (blockDim.x >> 5) + wib; slot < total; slot += gridDim.x * (blockDim.x >> 5)) {
    double *w = reinterpret_cast<double *>(smem) + static_cast<size_t>(wib) * 4 * K;
    double *rate_w = w, *change_w = w + K, *second_w = w + 2 * K, *max_w = w + 3 * K;
    int *valid_w = reinterpret_cast<int *>(reinterpret_cast<double *>(smem) + static_cast<size_t>(blockDim.x >> 5) * 4 * K) +
                   static_cast<size_t>(wib) * K;
    const int i = listed ? a.whole[slot] : owner_at(ids, slot);
    if (!listed) {
        // stored rates stand when neither the owner's reservoir entry nor any neighbour's changed
        // since they were evaluated (same geometry and lambda0)
        const int rated = a.rated[i];
        bool need = rated < 0 || a.stamp[i] > rated;
        for (int s = lane; s < K && !need; s += 32) {
            const int nb = a.codes[static_cast<size_t>(i) * K + s];
            need = nb >= 0 && a.stamp[nb / 3] > rated;
        }
        if (!__any_sync(0xffffffffu, need)) continue;
    }
    const bool act = a.active[i] != 0;
    const double meas = a.measure[i];
    const OwnerCtx o = owner_ctx(m, a.part, a.env, i, meas, a.lambda0);
    const double size_i = a.size_old[i];
    // the physical kernel on the cached environment: owner terms once per owner
    PairOwner po{0.0, 0.0, 0.0};
    if (kCached) po = cached_owner_terms(m, o.env, size_i);
    const int32_t *row = a.codes + static_cast<size_t>(i) * K;
    for (int s0 = lane; s0 < K; s0 += 64) {
        const int s1 = s0 + 32;
        const int nb0 = row[s0];
        const int nb1 = s1 < K ? row[s1] : -1;
        const bool use0 = act && nb0 >= 0 && meas > 0.0, use1 = act && nb1 >= 0 && meas > 0.0;
        const double sj0 = use0 ? a.size_old[nb0 / 3] : 0.0, nj0 = use0 ? a.numr_old[nb0 / 3] : 0.0;
        const double sj1 = use1 ? a.size_old[nb1 / 3] : 0.0, nj1 = use1 ? a.numr_old[nb1 / 3] : 0.0;
#pragma unroll 1
        for (int t = 0; t < 2; ++t) {
            const int s = t ? s1 : s0;
            if (s >= K) break;
            const bool use = t ? use1 : use0;
            const int j = (t ? nb1 : nb0) / 3;
            const double size_j = t ? sj1 : sj0, numr_j = t ? nj1 : nj0;
            double r = 0.0, c = 0.0, sc = 0.0, mx = 0.0;
            if (use) {
                double vrel;
                const double h_j = a.height ? a.height[j] : 0.0;
                double pr = chain_pair_rate<kCached>(m, o, po, size_i, size_j, numr_j, h_j, vrel);
                double mean = 0.0, sec = 0.0, maxi = 0.0;
                pr *= outcome_moments(m, size_i, size_j, vrel >= m.v_frag, mean, sec, maxi);
                mx = pr > 0.0 ? maxi : 0.0;
                c = pr * mean;
                sc = pr * sec;
                r = pr;
            }
            rate_w[s] = r;
            change_w[s] = c;
            second_w[s] = sc;
            max_w[s] = mx;
            valid_w[s] = isfinite(r) && r >= 0.0;
            if (a.leaf) store_pair(a, static_cast<size_t>(i) * K + s, r, c, sc, mx);
        }
    }
    fold_owner(a, K, lane, i, publish, rate_w, change_w, second_w, max_w, valid_w);
    }
}

// The changed pairs of owners whose own reservoir entry is unchanged (the list k_bath_rate
// appended): one pair per thread, the same operations as k_bath_rate's per-pair evaluation, the
// terms stored in the owner's row.
template <bool kCached>
__global__ void __launch_bounds__(128, GD_RATE_BLOCKS) k_pair_eval(Model m, RateArgs a) {
    if (!a.w->go || !a.w->need_rates) return;
    const int K = m.n_k;
    const int count = *a.pair_count;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < count; e += gridDim.x * blockDim.x) {
        const unsigned int code = a.pairs[e];
        const int i = static_cast<int>(code / static_cast<unsigned int>(K));
        const size_t at = static_cast<size_t>(code);
        const int nb = a.codes[at];
        const double meas = a.measure[i];
        double r = 0.0, c = 0.0, sc = 0.0, mx = 0.0;
        if (a.active[i] && nb >= 0 && meas > 0.0) {
            const OwnerCtx o = owner_ctx(m, a.part, a.env, i, meas, a.lambda0);
            const double size_i = a.size_old[i];
            PairOwner po{0.0, 0.0, 0.0};
            if (kCached) po = cached_owner_terms(m, o.env, size_i);
            const int j = nb / 3;
            const double size_j = a.size_old[j], numr_j = a.numr_old[j];
            const double h_j = a.height ? a.height[j] : 0.0;
            double vrel;
            double pr = chain_pair_rate<kCached>(m, o, po, size_i, size_j, numr_j, h_j, vrel);
            double mean = 0.0, sec = 0.0, maxi = 0.0;
            pr *= outcome_moments(m, size_i, size_j, vrel >= m.v_frag, mean, sec, maxi);
            mx = pr > 0.0 ? maxi : 0.0;
            c = pr * mean;
            sc = pr * sec;
            r = pr;
        }
        store_pair(a, at, r, c, sc, mx);
    }
}

// The owners k_bath_rate listed, folded from their K stored pairs once k_pair_eval has renewed the
// changed ones: one warp per owner, the staging and fold of k_bath_rate.
__global__ void __launch_bounds__(128, GD_RATE_BLOCKS) k_rate_fold(Model m, RateArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (!a.w->go || !a.w->need_rates) return;
    const int K = m.n_k;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int count = *a.fold_count, publish = a.w->publish;
    double *w = reinterpret_cast<double *>(smem) + static_cast<size_t>(wib) * 4 * K;
    double *rate_w = w, *change_w = w + K, *second_w = w + 2 * K, *max_w = w + 3 * K;
    int *valid_w = reinterpret_cast<int *>(reinterpret_cast<double *>(smem) + static_cast<size_t>(blockDim.x >> 5) * 4 * K) +
                   static_cast<size_t>(wib) * K;
    // K = 64, or a power of two up to 32: the fold of warp_fold in registers, the lane's two slots
    // first (a[j] += a[j + 32]), then shuffles (a[j] += a[j + half]), the same additions in the
    // same tree; the validity is an AND, whose order does not matter
    if (K == 64 || (K <= 32 && (K & (K - 1)) == 0)) {
        const int n_slots = K == 64 ? 2 : 1;
        for (int slot = blockIdx.x * (blockDim.x >> 5) + wib; slot < count; slot += gridDim.x * (blockDim.x >> 5)) {
            const int i = a.folds[slot];
            double r = 0.0, c = 0.0, sc = 0.0, mx = 0.0;
            bool valid = true;
            if (lane < K) {
                const size_t e = static_cast<size_t>(i) * K + lane;
                r = a.leaf[e];
                c = a.leaf[a.plane + e];
                sc = a.leaf[2 * a.plane + e];
                mx = a.leaf[3 * a.plane + e];
                valid = isfinite(r) && r >= 0.0;
                if (n_slots == 2) {
                    const double r1 = a.leaf[e + 32];
                    r += r1;
                    c += a.leaf[a.plane + e + 32];
                    sc += a.leaf[2 * a.plane + e + 32];
                    mx = fmax(mx, a.leaf[3 * a.plane + e + 32]);
                    valid = valid && isfinite(r1) && r1 >= 0.0;
                }
            }
            for (int d = K >= 32 ? 16 : K / 2; d >= 1; d >>= 1) {
                r += __shfl_down_sync(0xffffffffu, r, d);
                c += __shfl_down_sync(0xffffffffu, c, d);
                sc += __shfl_down_sync(0xffffffffu, sc, d);
                mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, d));
            }
            valid = __all_sync(0xffffffffu, valid);
            if (lane == 0) {
                RateMoments cm;
                cm.rate = valid ? r : -1.0;
                cm.first = c;
                cm.second = sc;
                cm.maximum = mx;
                a.cached[i] = cm;
                a.rate[i] = r;
                a.change[i] = c;
                a.second[i] = sc;
                a.rated[i] = publish;
            }
        }
        return;
    }
    for (int slot = blockIdx.x * (blockDim.x >> 5) + wib; slot < count; slot += gridDim.x * (blockDim.x >> 5)) {
        const int i = a.folds[slot];
        for (int s = lane; s < K; s += 32) {
            const size_t e = static_cast<size_t>(i) * K + s;
            const double r = a.leaf[e];
            rate_w[s] = r;
            change_w[s] = a.leaf[a.plane + e];
            second_w[s] = a.leaf[2 * a.plane + e];
            max_w[s] = a.leaf[3 * a.plane + e];
            valid_w[s] = isfinite(r) && r >= 0.0;
        }
        fold_owner(a, K, lane, i, publish, rate_w, change_w, second_w, max_w, valid_w);
    }
}

// Per-pair terms of the bath-start rate (the values k_bath_rate folds) against the current
// particle state as reservoir: out[(slot*K + s)*5 + {0..4}] = rate, rate*mean, rate*second,
// maximum, pair speed.  One thread per (owner, neighbour slot).
__global__ void k_pair_rates(Model m, const int *__restrict__ ids, int count, const gd_particle *__restrict__ part,
                             const int32_t *__restrict__ codes, const double *__restrict__ measure,
                             const unsigned char *__restrict__ active, double lambda0, double *__restrict__ out) {
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int K = m.n_k;
    if (t >= static_cast<long long>(count) * K) return;
    const int slot = static_cast<int>(t / K), s = static_cast<int>(t % K);
    const int i = ids[slot];
    double r = 0.0, c = 0.0, sc = 0.0, mx = 0.0, vrel = 0.0;
    const int nb = codes[static_cast<size_t>(i) * K + s];
    const double meas = measure[i];
    if (active[i] && nb >= 0 && meas > 0.0) {
        OwnerCtx o;
        o.y = part[i].position[1];
        o.z = part[i].position[2];
        const double R = cyl_R(m, o.y, o.z);
        o.H_i = R * get_hg(m, R);
        o.measure = meas;
        o.lambda0 = lambda0;
        if (use_env_cache(m) && m.coag_kernel == GD_KERNEL_CUSTOM) o.env = make_env(m, o.y, o.z);
        const int j = nb / 3;
        const double size_i = part[i].par_size, size_j = part[j].par_size;
        double pr = pair_rate(m, o, size_i, size_j, part[j].par_numr, part, j, vrel);
        double mean = 0.0, sec = 0.0, maxi = 0.0;
        pr *= outcome_moments(m, size_i, size_j, vrel >= m.v_frag, mean, sec, maxi);
        mx = pr > 0.0 ? maxi : 0.0;
        c = pr * mean;
        sc = pr * sec;
        r = pr;
    }
    double *o5 = out + static_cast<size_t>(t) * 5;
    o5[0] = r;
    o5[1] = c;
    o5[2] = sc;
    o5[3] = mx;
    o5[4] = vrel;
}

Status pair_rates(const Model &m, const int *ids, int count, const gd_particle *part, const int32_t *codes,
                  const double *measure, const unsigned char *active, double total_dust_mass, int n, double *out,
                  cudaStream_t s) {
    if (count <= 0) return Status::ok();
    const double lambda0 = n / static_cast<double>(m.n_k) / total_dust_mass;
    const long long threads = static_cast<long long>(count) * m.n_k;
    k_pair_rates<<<static_cast<unsigned int>((threads + 255) / 256), 256, 0, s>>>(m, ids, count, part, codes, measure,
                                                                                  active, lambda0, out);
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}

// _get_col_uniform (inc/swarm/_col_rates.cuh:145-149)
__device__ __forceinline__ double col_uniform(curandState *st) {
    return fmin(curand_uniform_double(st), nextafter(1.0, 0.0));
}

struct ChainArgs {
    const int *ids;
    const WaveInfo *w;  // the wave's owner count and order
    curandState *rng;
    const unsigned char *active;
    const double *measure;
    const int32_t *spatial;
    const double *dt;
    const RateMoments *cached;
    double *time, *hazard, *jump1, *jump2, *jumpmax;
    int *events;
    unsigned char *complete;
    int *queue;     // [n]: heavy owners from the front, the rest from the back
    int *queued;    // [2]: owners queued from the front, from the back
    int n;
};

// col_skip_scan (col_skip_scan.cu:13-59)
__global__ void k_skip_scan(ChainArgs a) {
    if (!a.w->go) return;
    const int count = a.w->count;
    const int *ids = a.w->full ? nullptr : a.ids;
    // a persistent grid; every warp of a block runs the same number of passes (ballots below)
    for (int base = blockIdx.x * blockDim.x; base < count; base += gridDim.x * blockDim.x) {
    const int slot = base + threadIdx.x;
    bool enqueue = false, heavy = false;
    int i = 0;
    if (slot < count) {
        i = owner_at(ids, slot);
        const double end = a.dt[a.spatial[i]];
        if (!a.active[i] || !(a.measure[i] > 0.0)) {
            a.time[i] = end;
            a.complete[i] = 1;
        } else if (!a.complete[i]) {
            enqueue = true;
            if (a.time[i] == 0.0 && a.events[i] == 0) {
                const RateMoments c = a.cached[i];
                if (isfinite(c.rate) && c.rate >= 0.0) {
                    if (c.rate == 0.0) {
                        a.time[i] = end;
                        a.complete[i] = 1;
                        enqueue = false;
                    } else {
                        curandState st = a.rng[i];
                        const double wait = -log(col_uniform(&st)) / c.rate;
                        const double remaining = end - a.time[i];
                        heavy = c.rate * remaining >= kHeavyEvents;
                        if (isfinite(wait) && wait > 0.0 && wait >= remaining) {
                            a.hazard[i] += c.rate * remaining;
                            a.jump1[i] += c.first * remaining;
                            a.jump2[i] += c.second * remaining;
                            a.jumpmax[i] = fmax(a.jumpmax[i], c.maximum);
                            a.time[i] = end;
                            a.complete[i] = 1;
                            a.rng[i] = st;
                            enqueue = false;
                        }
                        // otherwise the trial draw stays uncommitted: the chain repeats it
                    }
                }
            }
        }
    }
    // warp-aggregated queue append: owners expecting many events at the front, so that the chain
    // starts its longest owners first (the order of the owners does not change any owner's result)
    const int lane = threadIdx.x & 31;
    const unsigned int hmask = __ballot_sync(0xffffffffu, enqueue && heavy);
    const unsigned int lmask = __ballot_sync(0xffffffffu, enqueue && !heavy);
    if (hmask) {
        int qbase = 0;
        if (lane == __ffs(hmask) - 1) qbase = atomicAdd(&a.queued[0], __popc(hmask));
        qbase = __shfl_sync(0xffffffffu, qbase, __ffs(hmask) - 1);
        if (enqueue && heavy) a.queue[qbase + __popc(hmask & ((1u << lane) - 1u))] = i;
    }
    if (lmask) {
        int qbase = 0;
        if (lane == __ffs(lmask) - 1) qbase = atomicAdd(&a.queued[1], __popc(lmask));
        qbase = __shfl_sync(0xffffffffu, qbase, __ffs(lmask) - 1);
        if (enqueue && !heavy) a.queue[a.n - 1 - (qbase + __popc(lmask & ((1u << lane) - 1u)))] = i;
    }
    }
}

struct ChainRun {
    const double *height;  // R h_g(R) per particle (N_Z = 1 physical kernel), else null
    const gd_particle *part_ro;
    gd_particle *part;
    const int32_t *codes;
    const double *size_old, *numr_old;
    const Env *env;
    double lambda0;
    int *error;
    int *error_flag;
    int *head;
    unsigned long long *events_total;
    unsigned long long *event_count;  // [7] per outcome category (COL_DIAGNOSTICS), or null
    double *event_log_mass;           // [7]
};

// col_chain_run (col_chain_run.cu:21-404): persistent warps, one owner at a time
// kSlots = neighbour slots per lane (2 for K <= 64, 4 for K <= 128, else 8): the owner's partners
// and, for the cached physical kernel, their Stokes terms at the owner's environment stay in
// registers for the whole chain.
// 7 blocks of 4 warps per SM (72 registers, a few spilled): the chains of the C4 operators at
// N = 1e7 ran 1.3% faster than at 6 (80 registers); 1 or 2 blocks with every value in registers
// ran 40% slower, 5 blocks slightly slower
#ifndef GD_CHAIN_BLOCKS
#define GD_CHAIN_BLOCKS 7
#endif
template <int kSlots, bool kPhys>
__global__ void __launch_bounds__(kChainWarps * 32, GD_CHAIN_BLOCKS) k_chain(Model m, ChainArgs a, ChainRun r) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int K = m.n_k;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double *w = reinterpret_cast<double *>(smem) + static_cast<size_t>(wib) * kChainDoubles * K;
    double *prate = w, *tot = w + K, *pj1 = w + 2 * K, *pj2 = w + 3 * K, *pjm = w + 4 * K;
    int *last_w = reinterpret_cast<int *>(reinterpret_cast<double *>(smem) +
                                          static_cast<size_t>(kChainWarps) * kChainDoubles * K) +
                  static_cast<size_t>(wib) * K;
    // per slot: the pair's speed reaches the fragmentation threshold (the event's outcome branch)
    unsigned char *high_w = reinterpret_cast<unsigned char *>(
                                reinterpret_cast<int *>(reinterpret_cast<double *>(smem) +
                                                        static_cast<size_t>(kChainWarps) * kChainDoubles * K) +
                                static_cast<size_t>(kChainWarps) * K) +
                            static_cast<size_t>(wib) * K;
    const int nslot = (K + 31) / 32;
    const int heavy = a.queued[0];
    const int queued = heavy + a.queued[1];

    while (true) {
        int qs = 0;
        if (lane == 0) qs = atomicAdd(r.head, 1);
        qs = __shfl_sync(0xffffffffu, qs, 0);
        if (qs >= queued) break;
        const int i = qs < heavy ? a.queue[qs] : a.queue[a.n - 1 - (qs - heavy)];
        const double bath_end = a.dt[a.spatial[i]];
        const double meas = a.measure[i];

        double size_i = r.part_ro[i].par_size;
        double numr_i = r.part_ro[i].par_numr;
        double time_i = a.time[i];
        double hazard_i = a.hazard[i], jump1_i = a.jump1[i], jump2_i = a.jump2[i], jumpmax_i = a.jumpmax[i];
        curandState rng = a.rng[i];  // every lane holds the same state and draws the same numbers
        int event_count = a.events[i];
        int err = 0;
        bool running = a.complete[i] == 0;
        if (!a.active[i] || !(meas > 0.0)) {
            time_i = bath_end;
            running = false;
        }

        // frozen partners of this owner, kept in registers for every event
        const OwnerCtx o = owner_ctx(m, r.part_ro, r.env, i, meas, r.lambda0);
        int nb[kSlots];
        double sj[kSlots], nj[kSlots], hj[kSlots];
        PairPartner pp[kSlots];
        // kPhys: the physical kernel on the cached environment, known at compile time
        const bool cached = kPhys;
#pragma unroll
        for (int t = 0; t < kSlots; ++t) {
            nb[t] = -1;
            sj[t] = 0.0;
            nj[t] = 0.0;
            hj[t] = 0.0;
            pp[t] = PairPartner{0.0, 0.0, 0.0};
            const int s = lane + 32 * t;
            if (t < nslot && s < K) {
                nb[t] = r.codes[static_cast<size_t>(i) * K + s];
                if (nb[t] >= 0) {
                    const int j = nb[t] / 3;
                    sj[t] = r.size_old[j];
                    nj[t] = r.numr_old[j];
                    if (r.height) hj[t] = r.height[j];  // the partner's disk height (_col_rates.cuh:205-210)
                    if (cached) pp[t] = cached_partner_terms(m, o.env, sj[t]);
                }
            }
        }

        long long accepted = 0;
        while (running) {
            if (accepted >= kEventBudget) {
                err = 7;
                running = false;
                break;
            }
            PairOwner po{0.0, 0.0, 0.0};
            if (cached) po = cached_owner_terms(m, o.env, size_i);
            // one copy of the pair code, not kSlots: the loop body is the kernel's largest, and
            // unrolled it made instruction fetch the leading stall (10% slower chains at N = 1e7)
#pragma unroll 1
            for (int t = 0; t < kSlots; ++t) {
                const int s = lane + 32 * t;
                if (t < nslot && s < K) {
                    double pv = 0.0, j1 = 0.0, j2 = 0.0, jm = 0.0;
                    bool high = false;
                    if (nb[t] >= 0) {
                        double vrel;
                        pv = chain_pair_rate<kPhys>(m, o, po, size_i, sj[t], nj[t], hj[t], vrel,
                                                    cached ? &pp[t] : nullptr);
                        high = vrel >= m.v_frag;
                        double mean = 0.0, sec = 0.0, maxi = 0.0;
                        pv *= outcome_moments(m, size_i, sj[t], high, mean, sec, maxi);
                        j1 = pv * mean;
                        j2 = pv * sec;
                        jm = (pv > 0.0) ? maxi : 0.0;
                    }
                    prate[s] = pv;
                    high_w[s] = high ? 1 : 0;
                    tot[s] = pv;
                    pj1[s] = j1;
                    pj2[s] = j2;
                    pjm[s] = jm;
                    last_w[s] = (!isfinite(pv) || pv < 0.0) ? -2 : (pv > 0.0 ? s : -1);
                }
            }
            __syncwarp();
            warp_fold(K, lane, [&](int j, int h) {
                tot[j] += tot[h];
                pj1[j] += pj1[h];
                pj2[j] += pj2[h];
                pjm[j] = fmax(pjm[j], pjm[h]);
                const int left = last_w[j], right = last_w[h];
                last_w[j] = (left == -2 || right == -2) ? -2 : (left > right ? left : right);
            });
            const double total_rate = tot[0], total_j1 = pj1[0], total_j2 = pj2[0], total_jm = pjm[0];
            const int last_positive = last_w[0];
            __syncwarp();
            // the reference's thread-0 section, replayed identically by every lane
            if (last_positive == -2) {
                err = 1;
                running = false;
            }
            if (running && (!isfinite(total_rate) || total_rate < 0.0)) {
                err = 2;
                running = false;
            }
            if (running && total_rate == 0.0) {
                time_i = bath_end;
                running = false;
            }
            if (!running) break;
            const double wait = -log(col_uniform(&rng)) / total_rate;
            const double remaining = bath_end - time_i;
            if (!isfinite(wait) || !(wait > 0.0)) {
                err = 3;
                break;
            }
            if (wait >= remaining) {
                hazard_i += total_rate * remaining;
                jump1_i += total_j1 * remaining;
                jump2_i += total_j2 * remaining;
                jumpmax_i = fmax(jumpmax_i, total_jm);
                time_i = bath_end;
                break;
            }
            const double event_time = time_i + wait;
            if (!(event_time > time_i)) {
                err = 4;
                break;
            }
            hazard_i += total_rate * wait;
            jump1_i += total_j1 * wait;
            jump2_i += total_j2 * wait;
            jumpmax_i = fmax(jumpmax_i, total_jm);
            // partner: first slot whose cumulative rate exceeds U*total, in slot order.  The sum skips
            // slots without a positive rate, as the reference's does (adding +0 would not change it
            // either); eight slots per step, their loads issued together, the first crossing kept.
            const double target = col_uniform(&rng) * total_rate;
            double cumulative = 0.0;
            int pick = -1;
            for (int s0 = 0; s0 < K && pick < 0; s0 += 8) {
                double pr8[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) pr8[u] = (s0 + u < K) ? prate[s0 + u] : 0.0;
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const bool pos = pr8[u] > 0.0;
                    if (pos) cumulative += pr8[u];
                    if (pick < 0 && pos && cumulative > target) pick = s0 + u;
                }
            }
            if (pick < 0) pick = last_positive;
            if (pick < 0) {
                err = 5;
                break;
            }
            const int code_j = r.codes[static_cast<size_t>(i) * K + pick];
            const double size_j = r.size_old[code_j / 3];
            const double mass_before = numr_i * size_i * size_i * size_i;
            const bool high_speed = high_w[pick] != 0;
            const double sample = high_speed ? col_uniform(&rng) : 0.0;
            const double size_new = sample_outcome(m, size_i, size_j, high_speed, sample);
            if (r.event_count && lane == 0) {
                int cat;
                double lm;
                outcome_category(m, size_i, size_j, high_speed, sample, size_new, cat, lm);
                atomicAdd(&r.event_count[cat], 1ull);
                atomicAdd(&r.event_log_mass[cat], lm);
            }
            numr_i = mass_before / (size_new * size_new * size_new);
            size_i = size_new;
            time_i = event_time;
            ++event_count;
            ++accepted;
            const double mass_after = numr_i * size_i * size_i * size_i;
            const double mass_scale = fmax(fabs(mass_before), fabs(mass_after));
            if (!isfinite(size_i) || !isfinite(numr_i) || !(size_i > 0.0) || !(numr_i > 0.0) ||
                fabs(mass_after - mass_before) > 2.0e-12 * mass_scale) {
                err = 6;
                break;
            }
        }
        if (lane == 0) {
            r.part[i].par_size = size_i;
            r.part[i].par_numr = numr_i;
            a.rng[i] = rng;
            a.time[i] = time_i;
            a.events[i] = event_count;
            a.hazard[i] = hazard_i;
            a.jump1[i] = jump1_i;
            a.jump2[i] = jump2_i;
            a.jumpmax[i] = jumpmax_i;
            a.complete[i] = 1;
            if (err) {
                r.error[i] = err;
                atomicMax(r.error_flag, err);
            }
            if (accepted) atomicAdd(r.events_total, static_cast<unsigned long long>(accepted));
        }
        __syncwarp();
    }
}

// _col_atomic_max (inc/swarm/_col_rates.cuh:152-164)
__device__ __forceinline__ void atomic_max_double(double *address, double value) {
    unsigned long long *p = reinterpret_cast<unsigned long long *>(address);
    unsigned long long old = *p;
    while (value > __longlong_as_double(static_cast<long long>(old))) {
        unsigned long long assumed = old;
        old = atomicCAS(p, assumed, static_cast<unsigned long long>(__double_as_longlong(value)));
        if (old == assumed) break;
    }
}

struct AuditArgs {
    const int *ids;  // the wave's owners, grouped by spatial group (even when the wave holds every one)
    const WaveInfo *w;
    int count;       // set from the wave in the kernel
    AuditBin *bin;
    const gd_particle *part;
    const double *size_old, *numr_old, *rate, *hazard, *jump1, *jump2, *jumpmax;
    const int *events;
    const int32_t *spatial;
    const int *binmap;
    const unsigned char *active;
    const double *dt;
    const double *lower, *upper;
};

// col_audit_bin (col_audit_bin.cu:13-60)
// Audit sums per merged bin.  The lanes of a warp whose owners share a bin combine their terms
// in shared memory and one of them adds them to the bin (owners of one spatial group sit together,
// so a warp mostly feeds one or two bins): one atomic per bin and warp instead of one per owner.
constexpr int kAuditTerms = 13;  // staged doubles per owner besides the two maxima
constexpr int kAuditTPB = 256;   // threads per block of k_audit_bin
// The audit terms of the owner at `slot` (-1: none): whether it is an active owner (`on`), whether
// its terms are valid, its start and stop bins, and the staged terms t.
__device__ __forceinline__ void audit_owner(const Model &m, const AuditArgs &a, int slot, bool &on, bool &valid,
                                            int &start, int &stop, double t[kAuditTerms + 2]) {
    int i = 0;
    on = slot >= 0 && slot < a.count;
    if (on) {
        i = owner_at(a.ids, slot);
        on = a.active[i] != 0;
    }
    start = -1;
    stop = -1;
    valid = false;
#pragma unroll
    for (int f = 0; f < kAuditTerms + 2; ++f) t[f] = 0.0;
    if (on) {
        const int g = a.spatial[i];
        const double duration = a.dt[g];
        start = a.binmap[g * m.col_bin_s + size_bin(m, a.size_old[i], a.lower, a.upper, g)];
        stop = a.binmap[g * m.col_bin_s + size_bin(m, a.part[i].par_size, a.lower, a.upper, g)];
        const double weight = a.numr_old[i] * grain_mass(m, a.size_old[i]);
        const double probability = -expm1(-a.rate[i] * duration);
        const double expected = a.hazard[i];
        const double events = static_cast<double>(a.events[i]);
        valid = !(!isfinite(weight) || !(weight > 0.0) || !isfinite(probability) || !isfinite(expected) ||
                  expected < 0.0 || !isfinite(events) || !isfinite(a.jump1[i]) || a.jump1[i] < 0.0 ||
                  !isfinite(a.jump2[i]) || a.jump2[i] < 0.0 || !isfinite(a.jumpmax[i]) || a.jumpmax[i] < 0.0 ||
                  !isfinite(a.part[i].par_size) || !(a.part[i].par_size > 0.0));
        if (valid) {
            t[0] = weight;
            t[1] = weight * probability;
            t[2] = weight * expected;
            t[3] = weight * weight * probability * (1.0 - probability);
            t[4] = weight * weight * expected;
            t[5] = weight * a.jump1[i];
            t[6] = weight * weight * a.jump2[i];
            t[7] = a.events[i] > 0 ? weight : 0.0;
            t[8] = weight * events;
            t[9] = weight * fabs(log(a.part[i].par_size / a.size_old[i]));
            t[10] = weight;                  // end mass (bin `stop`)
            t[11] = 1.0;                     // valid owner
            t[12] = 0.0;
            t[13] = weight;                  // maximum weight
            t[14] = weight * a.jumpmax[i];   // maximum weighted jump
        }
    }
}

__global__ void __launch_bounds__(kAuditTPB) k_audit_bin(Model m, AuditArgs a_in) {
    if (!a_in.w->go) return;
    AuditArgs a = a_in;
    a.count = a.w->count;
    __shared__ double terms[kAuditTPB / 32][32][kAuditTerms + 2];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    bool on, valid;
    int start, stop;
    double t[kAuditTerms + 2];
    audit_owner(m, a, blockIdx.x * blockDim.x + threadIdx.x, on, valid, start, stop, t);
#pragma unroll
    for (int f = 0; f < kAuditTerms + 2; ++f) terms[wib][lane][f] = t[f];
    const unsigned int on_mask = __ballot_sync(0xffffffffu, on);
    const unsigned int valid_mask = __ballot_sync(0xffffffffu, valid);
    __syncwarp();
    if (!on) return;
    const unsigned int peers = __match_any_sync(on_mask, start);
    if (lane == __ffs(peers) - 1) {
        AuditBin *b = a.bin + start;
        double sum[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
        double mw = 0.0, mg = 0.0;
        int owners = __popc(peers), invalid = __popc(peers & ~valid_mask);
        for (unsigned int pm = peers & valid_mask; pm; pm &= pm - 1) {
            const int l = __ffs(pm) - 1;
#pragma unroll
            for (int f = 0; f < 10; ++f) sum[f] += terms[wib][l][f];
            mw = fmax(mw, terms[wib][l][13]);
            mg = fmax(mg, terms[wib][l][14]);
        }
        atomicAdd(&b->owner_count, owners);
        if (invalid) atomicAdd(&b->invalid_count, invalid);
        if (peers & valid_mask) {
            atomicAdd(&b->mass, sum[0]);
            atomicAdd(&b->predicted_f, sum[1]);
            atomicAdd(&b->predicted_e, sum[2]);
            atomicAdd(&b->predicted_var_f, sum[3]);
            atomicAdd(&b->predicted_var_e, sum[4]);
            atomicAdd(&b->predicted_g, sum[5]);
            atomicAdd(&b->predicted_var_g, sum[6]);
            atomic_max_double(&b->maximum_weight, mw);
            atomic_max_double(&b->maximum_g_jump, mg);
            atomicAdd(&b->touched, sum[7]);
            atomicAdd(&b->event_weight, sum[8]);
            atomicAdd(&b->growth, sum[9]);
        }
    }
    // end mass goes to the bin of the owner's new size
    if (!valid) return;
    const unsigned int speers = __match_any_sync(valid_mask, stop);
    if (lane == __ffs(speers) - 1) {
        double em = 0.0;
        for (unsigned int pm = speers; pm; pm &= pm - 1) em += terms[wib][__ffs(pm) - 1][10];
        atomicAdd(&a.bin[stop].end_mass, em);
    }
}

// The same audit with a second level of aggregation: a block covers kAuditSpan consecutive
// owners (one or two spatial groups, so a handful of bins) and its warps add their per-bin sums
// into a shared-memory copy of the bins; the block then adds each touched bin to global memory
// once.  Used when the raw bin count fits in shared memory (kAuditSmemBins); it turns the
// contended global atomics of the per-warp kernel (all warps hitting the same few hundred bins)
// into about one per bin and block.
constexpr int kAuditPerThread = 16;                          // owners per thread
constexpr int kAuditSpan = kAuditTPB * kAuditPerThread;      // owners per block
constexpr int kAuditSmemBins = 512;
constexpr int kAuditSums = 11;  // the ten start-bin sums, then the end mass
__host__ __device__ constexpr size_t audit_blocked_smem(int bins) {
    return sizeof(double) * (kAuditTPB / 32) * 32 * (kAuditTerms + 2) +
           static_cast<size_t>(bins) * (sizeof(double) * kAuditSums + sizeof(unsigned long long) * 2 + sizeof(int) * 3);
}
__global__ void __launch_bounds__(kAuditTPB) k_audit_bin_blocked(Model m, AuditArgs a_in, int bins) {
    if (!a_in.w->go) return;
    AuditArgs a = a_in;
    a.count = a.w->count;
    if (static_cast<long long>(blockIdx.x) * kAuditSpan >= a.count) return;
    extern __shared__ __align__(16) double sa[];
    double(*terms)[32][kAuditTerms + 2] = reinterpret_cast<double(*)[32][kAuditTerms + 2]>(sa);
    double *bsum = sa + (kAuditTPB / 32) * 32 * (kAuditTerms + 2);                              // [bins][kAuditSums]
    unsigned long long *bmax = reinterpret_cast<unsigned long long *>(bsum + bins * kAuditSums);  // [bins][2]
    int *bcnt = reinterpret_cast<int *>(bmax + bins * 2);  // [bins][3]: owners, invalid owners, end-mass adds
    for (int k = threadIdx.x; k < bins * kAuditSums; k += blockDim.x) bsum[k] = 0.0;
    for (int k = threadIdx.x; k < bins * 2; k += blockDim.x) bmax[k] = 0ull;
    for (int k = threadIdx.x; k < bins * 3; k += blockDim.x) bcnt[k] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long first = static_cast<long long>(blockIdx.x) * kAuditSpan;
    for (int it = 0; it < kAuditPerThread && first + it * kAuditTPB < a.count; ++it) {
        const long long sl = first + it * kAuditTPB + threadIdx.x;
        bool on, valid;
        int start, stop;
        double t[kAuditTerms + 2];
        audit_owner(m, a, sl < a.count ? static_cast<int>(sl) : -1, on, valid, start, stop, t);
#pragma unroll
        for (int f = 0; f < kAuditTerms + 2; ++f) terms[wib][lane][f] = t[f];
        const unsigned int on_mask = __ballot_sync(0xffffffffu, on);
        const unsigned int valid_mask = __ballot_sync(0xffffffffu, valid);
        __syncwarp();
        if (on) {
            const unsigned int peers = __match_any_sync(on_mask, start);
            if (lane == __ffs(peers) - 1) {
                double sum[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
                double mw = 0.0, mg = 0.0;
                for (unsigned int pm = peers & valid_mask; pm; pm &= pm - 1) {
                    const int l = __ffs(pm) - 1;
#pragma unroll
                    for (int f = 0; f < 10; ++f) sum[f] += terms[wib][l][f];
                    mw = fmax(mw, terms[wib][l][13]);
                    mg = fmax(mg, terms[wib][l][14]);
                }
                atomicAdd(&bcnt[start * 3], __popc(peers));
                atomicAdd(&bcnt[start * 3 + 1], __popc(peers & ~valid_mask));
                if (peers & valid_mask) {
#pragma unroll
                    for (int f = 0; f < 10; ++f) atomicAdd(&bsum[start * kAuditSums + f], sum[f]);
                    // non-negative doubles order like their bit patterns
                    atomicMax(&bmax[start * 2], static_cast<unsigned long long>(__double_as_longlong(mw)));
                    atomicMax(&bmax[start * 2 + 1], static_cast<unsigned long long>(__double_as_longlong(mg)));
                }
            }
        }
        if (valid) {
            const unsigned int speers = __match_any_sync(valid_mask, stop);
            if (lane == __ffs(speers) - 1) {
                double em = 0.0;
                for (unsigned int pm = speers; pm; pm &= pm - 1) em += terms[wib][__ffs(pm) - 1][10];
                atomicAdd(&bsum[stop * kAuditSums + 10], em);
                atomicAdd(&bcnt[stop * 3 + 2], 1);
            }
        }
        __syncwarp();  // the staged terms are rewritten by the next owner
    }
    __syncthreads();
    for (int b = threadIdx.x; b < bins; b += blockDim.x) {
        const int owners = bcnt[b * 3], invalid = bcnt[b * 3 + 1], ends = bcnt[b * 3 + 2];
        AuditBin *g = a.bin + b;
        if (owners) {
            atomicAdd(&g->owner_count, owners);
            if (invalid) atomicAdd(&g->invalid_count, invalid);
        }
        if (owners > invalid) {
            const double *v = bsum + b * kAuditSums;
            atomicAdd(&g->mass, v[0]);
            atomicAdd(&g->predicted_f, v[1]);
            atomicAdd(&g->predicted_e, v[2]);
            atomicAdd(&g->predicted_var_f, v[3]);
            atomicAdd(&g->predicted_var_e, v[4]);
            atomicAdd(&g->predicted_g, v[5]);
            atomicAdd(&g->predicted_var_g, v[6]);
            atomic_max_double(&g->maximum_weight, __longlong_as_double(static_cast<long long>(bmax[b * 2])));
            atomic_max_double(&g->maximum_g_jump, __longlong_as_double(static_cast<long long>(bmax[b * 2 + 1])));
            atomicAdd(&g->touched, v[7]);
            atomicAdd(&g->event_weight, v[8]);
            atomicAdd(&g->growth, v[9]);
        }
        if (ends) atomicAdd(&g->end_mass, bsum[b * kAuditSums + 10]);
    }
}

// Blocked forms of the three controller scans, with the aggregation of k_audit_bin_blocked: a block
// covers kAuditSpan consecutive owners, its warps combine per group or bin in shared memory, and
// the block adds each touched entry to global memory once.  The host uses them while the groups
// or bins fit in the default 48 KB of shared memory (kScanSmemEntries).
constexpr int kScanSmemEntries = 1024;

__global__ void __launch_bounds__(kAuditTPB) k_size_scan_blocked(const WaveInfo *__restrict__ w, const int *__restrict__ ids,
                                                                const gd_particle *__restrict__ part,
                                                                const int32_t *__restrict__ spatial,
                                                                const unsigned char *__restrict__ active, int G,
                                                                unsigned long long *mmin, unsigned long long *mmax) {
    if (!w->go || !w->need_rates) return;
    const int count = w->count;
    if (w->full) ids = nullptr;
    if (static_cast<long long>(blockIdx.x) * kAuditSpan >= count) return;
    extern __shared__ __align__(16) unsigned long long smm[];  // [G] minima, [G] maxima (double bits)
    unsigned long long *smin = smm, *smax = smm + G;
    for (int k = threadIdx.x; k < G; k += blockDim.x) {
        smin[k] = ~0ull;
        smax[k] = 0ull;
    }
    __syncthreads();
    const long long first = static_cast<long long>(blockIdx.x) * kAuditSpan;
    for (int it = 0; it < kAuditPerThread && first + it * kAuditTPB < count; ++it) {
        const long long slot = first + it * kAuditTPB + threadIdx.x;
        bool on = slot < count;
        int g = 0;
        unsigned long long bits = 0;
        if (on) {
            const int i = owner_at(ids, static_cast<int>(slot));
            const double size = part[i].par_size;
            on = active[i] && size > 0 && isfinite(size);
            if (on) {
                g = spatial[i];
                bits = static_cast<unsigned long long>(__double_as_longlong(size));
            }
        }
        const unsigned int mask = __ballot_sync(0xffffffffu, on);
        if (on) {
            const unsigned int peers = __match_any_sync(mask, g);
            unsigned long long lo = bits, hi = bits;
            for (unsigned int pm = peers; pm; pm &= pm - 1) {
                const unsigned long long v = __shfl_sync(peers, bits, __ffs(pm) - 1);
                lo = v < lo ? v : lo;
                hi = v > hi ? v : hi;
            }
            if ((peers & lanes_below()) == 0) {
                atomicMin(&smin[g], lo);
                atomicMax(&smax[g], hi);
            }
        }
    }
    __syncthreads();
    for (int g = threadIdx.x; g < G; g += blockDim.x) {
        if (smax[g] != 0ull) {  // touched: positive sizes have non-zero bits
            atomicMin(&mmin[g], smin[g]);
            atomicMax(&mmax[g], smax[g]);
        }
    }
}

__global__ void __launch_bounds__(kAuditTPB) k_count_bin_blocked(Model m, const WaveInfo *__restrict__ w,
                                                                const int *__restrict__ ids,
                                                                int *__restrict__ counts,
                                                                const gd_particle *__restrict__ part,
                                                                const int32_t *__restrict__ spatial,
                                                                const unsigned char *__restrict__ active,
                                                                const double *lower, const double *upper, int R) {
    if (!w->go || !w->need_rates) return;
    const int count = w->count;
    if (w->full) ids = nullptr;
    if (static_cast<long long>(blockIdx.x) * kAuditSpan >= count) return;
    extern __shared__ int scnt[];  // [R]
    for (int k = threadIdx.x; k < R; k += blockDim.x) scnt[k] = 0;
    __syncthreads();
    const long long first = static_cast<long long>(blockIdx.x) * kAuditSpan;
    for (int it = 0; it < kAuditPerThread && first + it * kAuditTPB < count; ++it) {
        const long long slot = first + it * kAuditTPB + threadIdx.x;
        bool on = slot < count;
        int key = 0;
        if (on) {
            const int i = owner_at(ids, static_cast<int>(slot));
            on = active[i] != 0;
            if (on) {
                const int g = spatial[i];
                key = g * m.col_bin_s + size_bin(m, part[i].par_size, lower, upper, g);
            }
        }
        const unsigned int mask = __ballot_sync(0xffffffffu, on);
        if (on) {
            const unsigned int peers = __match_any_sync(mask, key);
            if ((peers & lanes_below()) == 0) atomicAdd(&scnt[key], __popc(peers));
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < R; k += blockDim.x)
        if (scnt[k]) atomicAdd(counts + k, scnt[k]);
}

__global__ void __launch_bounds__(kAuditTPB) k_rate_bins_blocked(Model m, const WaveInfo *__restrict__ w,
                                                                const int *__restrict__ ids,
                                                                RateBin *__restrict__ bin,
                                                                const gd_particle *__restrict__ part,
                                                                const double *__restrict__ rate,
                                                                const double *__restrict__ change,
                                                                const double *__restrict__ second,
                                                                const int32_t *__restrict__ spatial,
                                                                const int *__restrict__ binmap,
                                                                const unsigned char *__restrict__ active,
                                                                const double *lower, const double *upper, int R) {
    if (!w->go || !w->need_rates) return;
    const int count = w->count;
    if (w->full) ids = nullptr;
    if (static_cast<long long>(blockIdx.x) * kAuditSpan >= count) return;
    extern __shared__ __align__(16) double srb[];  // [R][4] sums, then [R][2] owner / invalid counts
    int *sct = reinterpret_cast<int *>(srb + 4 * R);
    for (int k = threadIdx.x; k < 4 * R; k += blockDim.x) srb[k] = 0.0;
    for (int k = threadIdx.x; k < 2 * R; k += blockDim.x) sct[k] = 0;
    __syncthreads();
    const long long first = static_cast<long long>(blockIdx.x) * kAuditSpan;
    for (int it = 0; it < kAuditPerThread && first + it * kAuditTPB < count; ++it) {
        const long long slot = first + it * kAuditTPB + threadIdx.x;
        bool on = slot < count;
        int b = 0;
        bool valid = false;
        double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
        if (on) {
            const int i = owner_at(ids, static_cast<int>(slot));
            on = active[i] != 0;
            if (on) {
                const int g = spatial[i];
                b = binmap[g * m.col_bin_s + size_bin(m, part[i].par_size, lower, upper, g)];
                const double weight = part[i].par_numr * grain_mass(m, part[i].par_size);
                valid = !(!isfinite(weight) || !(weight > 0.0) || !isfinite(rate[i]) || rate[i] < 0.0 ||
                          !isfinite(change[i]) || change[i] < 0 || !isfinite(second[i]) || second[i] < 0);
                if (valid) {
                    t0 = weight;
                    t1 = weight * rate[i];
                    t2 = weight * change[i];
                    t3 = weight * second[i];
                }
            }
        }
        const unsigned int mask = __ballot_sync(0xffffffffu, on);
        const unsigned int vmask = __ballot_sync(0xffffffffu, valid);
        if (on) {
            const unsigned int peers = __match_any_sync(mask, b);
            double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
            for (unsigned int pm = peers; pm; pm &= pm - 1) {
                const int l = __ffs(pm) - 1;
                s0 += __shfl_sync(peers, t0, l);
                s1 += __shfl_sync(peers, t1, l);
                s2 += __shfl_sync(peers, t2, l);
                s3 += __shfl_sync(peers, t3, l);
            }
            if ((peers & lanes_below()) == 0) {
                atomicAdd(&sct[2 * b], __popc(peers));
                const int invalid = __popc(peers & ~vmask);
                if (invalid) atomicAdd(&sct[2 * b + 1], invalid);
                if (peers & vmask) {
                    atomicAdd(&srb[4 * b], s0);
                    atomicAdd(&srb[4 * b + 1], s1);
                    atomicAdd(&srb[4 * b + 2], s2);
                    atomicAdd(&srb[4 * b + 3], s3);
                }
            }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < R; k += blockDim.x) {
        const int owners = sct[2 * k], invalid = sct[2 * k + 1];
        if (!owners) continue;
        atomicAdd(&bin[k].owner_count, owners);
        if (invalid) atomicAdd(&bin[k].invalid_count, invalid);
        if (owners > invalid) {
            atomicAdd(&bin[k].mass, srb[4 * k]);
            atomicAdd(&bin[k].weighted_rate, srb[4 * k + 1]);
            atomicAdd(&bin[k].weighted_change, srb[4 * k + 2]);
            atomicAdd(&bin[k].weighted_second, srb[4 * k + 3]);
        }
    }
}

// owner lists per spatial group (_col_chain.cuh:162-167) by a device counting sort
// Owner lists per spatial group by a counting sort, and the group dependency graph.  Particles
// come in index order, where neighbouring indices belong to unrelated groups, so warp matching
// rarely merges their atomics.  Each block covers kAuditSpan consecutive particles and gathers
// its counts, slot reservations and edges in shared memory first: one global atomic per touched
// group (or edge word) and block instead of one per particle.
constexpr int kGroupTPB = 256;
constexpr int kGroupPerThread = 16;
constexpr int kGroupSpan = kGroupTPB * kGroupPerThread;

__global__ void __launch_bounds__(kGroupTPB) k_group_count(int n, int G, const int32_t *__restrict__ spatial,
                                                          int *__restrict__ gcount) {
    __shared__ int cnt[kMaxGroups];
    for (int g = threadIdx.x; g < G; g += blockDim.x) cnt[g] = 0;
    __syncthreads();
    const long long first = static_cast<long long>(blockIdx.x) * kGroupSpan;
    for (int it = 0; it < kGroupPerThread && first + it * kGroupTPB < n; ++it) {
        const long long i = first + it * kGroupTPB + threadIdx.x;
        const bool on = i < n;
        const int g = on ? spatial[i] : 0;
        const unsigned int mask = __ballot_sync(0xffffffffu, on);
        if (on) {
            const unsigned int peers = __match_any_sync(mask, g);
            if ((peers & lanes_below()) == 0) atomicAdd(&cnt[g], __popc(peers));
        }
    }
    __syncthreads();
    for (int g = threadIdx.x; g < G; g += blockDim.x)
        if (cnt[g]) atomicAdd(&gcount[g], cnt[g]);
}

// Each block reserves one consecutive range per group it touches, then writes its particles
// there at their rank within the block.
__global__ void __launch_bounds__(kGroupTPB) k_group_fill(int n, int G, const int32_t *__restrict__ spatial,
                                                         int *__restrict__ gcursor, int *__restrict__ sorted) {
    __shared__ int cnt[kMaxGroups];
    __shared__ int base[kMaxGroups];
    for (int g = threadIdx.x; g < G; g += blockDim.x) cnt[g] = 0;
    __syncthreads();
    const long long first = static_cast<long long>(blockIdx.x) * kGroupSpan;
    for (int it = 0; it < kGroupPerThread && first + it * kGroupTPB < n; ++it) {
        const long long i = first + it * kGroupTPB + threadIdx.x;
        const bool on = i < n;
        const int g = on ? spatial[i] : 0;
        const unsigned int mask = __ballot_sync(0xffffffffu, on);
        if (on) {
            const unsigned int peers = __match_any_sync(mask, g);
            if ((peers & lanes_below()) == 0) atomicAdd(&cnt[g], __popc(peers));
        }
    }
    __syncthreads();
    for (int g = threadIdx.x; g < G; g += blockDim.x) {
        base[g] = cnt[g] ? atomicAdd(&gcursor[g], cnt[g]) : 0;
        cnt[g] = 0;  // reused as the block's cursor per group
    }
    __syncthreads();
    for (int it = 0; it < kGroupPerThread && first + it * kGroupTPB < n; ++it) {
        const long long i = first + it * kGroupTPB + threadIdx.x;
        const bool on = i < n;
        const int g = on ? spatial[i] : 0;
        const unsigned int mask = __ballot_sync(0xffffffffu, on);
        if (on) {
            const unsigned int peers = __match_any_sync(mask, g);
            const int leader = __ffs(peers) - 1;
            int off = 0;
            if ((threadIdx.x & 31) == leader) off = atomicAdd(&cnt[g], __popc(peers));
            off = __shfl_sync(peers, off, leader);
            sorted[base[g] + off + __popc(peers & lanes_below())] = static_cast<int>(i);
        }
    }
}

// col_dep_graph (col_dep_graph.cu:43-59): edge c->d when an owner in c has a neighbour in d.  A
// warp takes its particles one at a time: the lanes read the owner's codes (coalesced), look up
// the neighbours' groups, and OR-reduce the group bitset across the warp.
__global__ void __launch_bounds__(kGroupTPB) k_dep_graph(int n, int K, int G, int words,
                                                        unsigned int *__restrict__ edges,
                                                        const int32_t *__restrict__ spatial,
                                                        const int32_t *__restrict__ codes,
                                                        const unsigned char *__restrict__ active) {
    __shared__ unsigned int se[kMaxGroups * (kMaxGroups / 32)];
    for (int k = threadIdx.x; k < G * words; k += blockDim.x) se[k] = 0u;
    __syncthreads();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long first = static_cast<long long>(blockIdx.x) * kGroupSpan;
    const long long last = first + kGroupSpan < n ? first + kGroupSpan : n;
    for (long long i = first + wib; i < last; i += kGroupTPB / 32) {
        if (!active[i]) continue;  // warp-uniform: one particle per warp
        unsigned int bits[kMaxGroups / 32];
#pragma unroll
        for (int wd = 0; wd < kMaxGroups / 32; ++wd) bits[wd] = 0u;
        for (int k = lane; k < K; k += 32) {
            const int e = codes[static_cast<size_t>(i) * K + k];
            if (e >= 0) {
                const int c = spatial[e / 3];
#pragma unroll
                for (int wd = 0; wd < kMaxGroups / 32; ++wd)
                    if ((c >> 5) == wd) bits[wd] |= 1u << (c & 31);
            }
        }
        const int gi = spatial[i];
#pragma unroll
        for (int wd = 0; wd < kMaxGroups / 32; ++wd) {
            if (wd >= words) break;
            const unsigned int b = __reduce_or_sync(0xffffffffu, bits[wd]);
            if (lane == 0 && b) atomicOr(&se[gi * words + wd], b);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < G * words; k += blockDim.x)
        if (se[k]) atomicOr(edges + k, se[k]);
}

// ------------------------------------------------------------------------------------------------
// host controller: the shared arithmetic of gd_ctl_core.cuh behind Status
// ------------------------------------------------------------------------------------------------
static Status err(gd_status code, const std::string &msg, long long detail = 0) {
    Status s;
    s.code = code;
    s.msg = msg;
    s.detail = detail;
    return s;
}

Status ctl_status(int code) {
    switch (code) {
    case kCtlOk: return Status::ok();
    case kCtlBadHorizon: return err(GD_ERR_INVALID_ARGUMENT, "invalid local collision horizon");
    case kCtlBadTimestep: return err(GD_ERR_CONTROLLER, "invalid local collision timestep");
    case kCtlTimeResolution: return err(GD_ERR_TIME_RESOLUTION, "local collision timestep exceeds time resolution");
    case kCtlBadAdaptStep: return err(GD_ERR_CONTROLLER, "invalid adaptive collision timestep");
    case kCtlAdaptResolution: return err(GD_ERR_TIME_RESOLUTION, "adaptive collision time resolution exceeded");
    case kCtlBadRateMoments: return err(GD_ERR_CONTROLLER, "invalid change-based rate moments");
    case kCtlBadChangeInputs: return err(GD_ERR_CONTROLLER, "invalid change-based refresh inputs");
    case kCtlChangeUnderflow: return err(GD_ERR_CONTROLLER, "change-based timestep underflow");
    case kCtlBadAudit: return err(GD_ERR_CONTROLLER, "collision bath controller returned an invalid audit state");
    case kCtlNoMass: return err(GD_ERR_CONTROLLER, "collision bath controller found no active represented mass");
    case kCtlWaveLimit: return err(GD_ERR_CONTROLLER, "the collision scheduler found no owners in too many waves");
    default: break;
    }
    if (code == 100 + 7) return err(GD_ERR_CONTINUATION_LIMIT, "local collision continuation limit exceeded", 7);
    if (code > 100) return err(GD_ERR_CHAIN, "local collision chain error " + std::to_string(code - 100), code - 100);
    return err(GD_ERR_CONTROLLER, "unknown controller state " + std::to_string(code), code);
}

int build_binmap(const Model &m, const std::vector<int> &raw_count, std::vector<int> &raw_to_merged) {
    raw_to_merged.assign(raw_count.size(), -1);
    return binmap_compute(m.local_groups, m.col_bin_s, m.col_bin_min, raw_count.data(), raw_to_merged.data());
}

// _choose_col_bath (inc/swarm/_col_bound.cuh:288-310)
Status choose_bath(const Model &m, const RateBin *bins, int count, double remaining, double limit_scale, double &out,
                   int *binding) {
    return ctl_status(ctl_choose_bath(m, bins, count, remaining, limit_scale, out, binding));
}

// _finish_col_bath (inc/swarm/_col_bound.cuh:313-403)
Status finish_bath(const Model &m, const AuditBin *bins, int count, BathState &state, BathResult &result) {
    return ctl_status(ctl_finish_bath(m, bins, count, state, result, nullptr));
}

// ------------------------------------------------------------------------------------------------
// allocation and the operator
// ------------------------------------------------------------------------------------------------
Collider::~Collider() {
    if (host_ctl) cudaFreeHost(host_ctl);
    if (capture_stream) cudaStreamDestroy(capture_stream);
    if (body_stream) cudaStreamDestroy(body_stream);
}

static CtlDev *ctl_of(Collider &c) { return reinterpret_cast<CtlDev *>(c.ctl.ptr); }

// accumulators of a CtlResult the host has read
static CtlResult fresh_result(int operator_index) {
    CtlResult r{};
    r.operator_index = operator_index;
    r.min_duration = HUGE_VAL;
    return r;
}

Status collider_alloc(Collider &c, const Model &m, int n, int record_capacity) {
    if (m.local_groups > kCtlGroups) return err(GD_ERR_INVALID_ARGUMENT, "more than 256 controller groups");
    c.n = n;
    for (DevBuf<double> *b : {&c.size_old, &c.numr_old, &c.time, &c.hazard, &c.jump1, &c.jump2, &c.jumpmax, &c.rate,
                              &c.change_rate, &c.second_rate})
        GD_TRY_CUDA(b->alloc(n));
    GD_TRY_CUDA(c.events.alloc(n));
    GD_TRY_CUDA(c.error.alloc(n));
    GD_TRY_CUDA(c.complete.alloc(n));
    GD_TRY_CUDA(c.env.alloc(static_cast<size_t>(n) * 8));
    GD_TRY_CUDA(c.cached.alloc(static_cast<size_t>(n) * 4));
    if (static_cast<long long>(n) * m.n_k < (1ll << 31)) {
        GD_TRY_CUDA(c.leaf.alloc(static_cast<size_t>(n) * m.n_k * 4));
        GD_TRY_CUDA(c.pairs.alloc(static_cast<size_t>(n) * m.n_k));
        GD_TRY_CUDA(c.folds.alloc(n));
        GD_TRY_CUDA(c.whole.alloc(n));
    }
    GD_TRY_CUDA(c.stamp.alloc(n));
    GD_TRY_CUDA(c.rated.alloc(n));
    GD_TRY_CUDA(cudaMemset(c.stamp.ptr, 0, sizeof(int) * n));
    GD_TRY_CUDA(cudaMemset(c.rated.ptr, 0xff, sizeof(int) * n));
    GD_TRY_CUDA(c.ids.alloc(n));
    GD_TRY_CUDA(c.queue.alloc(n));
    GD_TRY_CUDA(c.group_sorted.alloc(n));
    GD_TRY_CUDA(c.spatial.alloc(n));
    Small L = small_layout(m);
    c.events_offset = L.events;
    GD_TRY_CUDA(c.small.alloc(L.total));
    GD_TRY_CUDA(cudaMemset(c.small.ptr, 0, L.total));
    GD_TRY_CUDA(cudaMemset(c.error.ptr, 0, sizeof(int) * n));
    GD_TRY_CUDA(c.event_count.alloc(kEventCategories));
    GD_TRY_CUDA(c.event_log_mass.alloc(kEventCategories));
    if (m.coag_kernel == GD_KERNEL_CUSTOM && m.n_z == 1) GD_TRY_CUDA(c.height.alloc(n));
    // the device controller: default bath states, no operator yet, empty accumulators
    GD_TRY_CUDA(c.ctl.alloc(sizeof(CtlDev)));
    {
        std::unique_ptr<CtlDev> init(new CtlDev());  // value-initialised: zeros, default bath states
        init->res = fresh_result(0);
        GD_TRY_CUDA(cudaMemcpy(c.ctl.ptr, init.get(), sizeof(CtlDev), cudaMemcpyHostToDevice));
    }
    std::vector<double> logs(static_cast<size_t>(m.raw_bins) + 1);
    for (int k = 0; k <= m.raw_bins; ++k) logs[k] = ctl_confidence_log(k, m.col_bath_alpha);
    GD_TRY_CUDA(c.conf_log.alloc(logs.size()));
    GD_TRY_CUDA(cudaMemcpy(c.conf_log.ptr, logs.data(), sizeof(double) * logs.size(), cudaMemcpyHostToDevice));
    c.record_capacity = record_capacity > 0 ? record_capacity : 1;
    GD_TRY_CUDA(c.records.alloc(c.record_capacity));
    GD_TRY_CUDA(cudaMallocHost(reinterpret_cast<void **>(&c.host_ctl), sizeof(CtlResult) + sizeof(unsigned long long)));
    GD_TRY_CUDA(cudaStreamCreateWithFlags(&c.capture_stream, cudaStreamNonBlocking));
    GD_TRY_CUDA(cudaStreamCreateWithFlags(&c.body_stream, cudaStreamNonBlocking));
    return Status::ok();
}

// The results of the operators run since the last read: error, counters, bath records.  Every
// operator adds to one accumulator on the device, so a graph that holds several operators is read
// once after it ran.  Many colliders are read with three synchronisations in all.
constexpr int kOperatorLogCapacity = 64;  // per-operator log records kept on the device between reads

Status collider_enable_log(Collider &c) {
    if (c.oplog.ptr) return Status::ok();
    GD_TRY_CUDA(c.oplog.alloc(kOperatorLogCapacity));
    c.oplog_capacity = kOperatorLogCapacity;
    return Status::ok();
}

// One line of the per-operator JSONL log, with the keys, order and number format the reference
// writes (_col_chain.cuh:488-535, std::setprecision(17)).
static std::string operator_log_line(const OperatorLog &r) {
    std::ostringstream f;
    f << std::setprecision(17);
    f << "{\"schema\":1,\"method\":\"local_cached_collision\",\"operator\":" << r.operator_id
      << ",\"clock_sim\":" << r.clock_sim << ",\"duration\":" << r.duration << ",\"waves\":" << r.waves
      << ",\"owner_updates\":" << r.owner_updates << ",\"chain_blocks\":" << r.chain_blocks
      << ",\"chain_launches\":" << r.chain_launches << ",\"chain_seconds\":" << r.chain_seconds
      << ",\"audit_seconds\":" << r.audit_seconds << ",\"scheduler_wall_seconds\":" << r.wall_seconds
      << ",\"finest_ticks\":" << r.finest_ticks << ",\"groups\":[";
    for (int g = 0; g < r.G; ++g) {
        const OperatorLogGroup &o = r.g[g];
        if (g) f << ',';
        f << "{\"id\":" << g << ",\"owners\":" << o.owners << ",\"level\":" << o.level << ",\"dt\":" << o.dt
          << ",\"initial_level\":" << o.initial_level << ",\"coarsened_updates\":" << o.coarsened
          << ",\"refined_updates\":" << o.refined << ",\"neighbor_constrained_updates\":" << o.constrained
          << ",\"minimum_requested_dt\":" << o.min_request << ",\"maximum_requested_dt\":" << o.max_request
          << ",\"final_requested_dt\":" << o.final_request << ",\"initial_requested_dt\":" << o.initial_request
          << ",\"initial_binding_constraint\":" << o.binding << ",\"updates\":" << o.updates
          << ",\"overshoots\":" << o.overshoots << ",\"persistent_overshoots\":" << o.persistent
          << ",\"max_snapshot_age_at_start\":" << o.max_age << ",\"max_requested_dt_ratio\":" << o.max_ratio
          << ",\"max_growth\":" << o.max_growth << ",\"max_predicted_activity\":" << o.max_activity << '}';
    }
    f << "],\"event_counts\":[";
    for (int k = 0; k < kEventCategories; ++k) f << (k ? "," : "") << r.event_count[k];
    f << "],\"event_log_mass_sums\":[";
    for (int k = 0; k < kEventCategories; ++k) f << (k ? "," : "") << r.event_log_mass[k];
    f << "]}\n";
    return f.str();
}

Status collider_check_many(Collider *const *cs, int count, cudaStream_t s, int *first_failed) {
    if (first_failed) *first_failed = -1;
    for (int k = 0; k < count; ++k) {
        Collider &c = *cs[k];
        CtlResult *hr = reinterpret_cast<CtlResult *>(c.host_ctl);
        unsigned long long *hev = reinterpret_cast<unsigned long long *>(c.host_ctl + sizeof(CtlResult));
        GD_TRY_CUDA(cudaMemcpyAsync(hr, &ctl_of(c)->res, sizeof(CtlResult), cudaMemcpyDeviceToHost, s));
        GD_TRY_CUDA(cudaMemcpyAsync(hev, c.small.ptr + c.events_offset, sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, s));
    }
    GD_TRY_CUDA(cudaStreamSynchronize(s));
    std::vector<CtlResult> res(count);
    std::vector<unsigned long long> events(count);
    std::vector<std::vector<BathRecord>> recs(count);
    std::vector<std::vector<OperatorLog>> logs(count);
    for (int k = 0; k < count; ++k) {
        Collider &c = *cs[k];
        res[k] = *reinterpret_cast<CtlResult *>(c.host_ctl);
        events[k] = *reinterpret_cast<unsigned long long *>(c.host_ctl + sizeof(CtlResult));
        const int nrec = res[k].rec_count < c.record_capacity ? res[k].rec_count : c.record_capacity;
        if (nrec > 0) {
            recs[k].resize(static_cast<size_t>(nrec));
            GD_TRY_CUDA(cudaMemcpyAsync(recs[k].data(), c.records.ptr, sizeof(BathRecord) * recs[k].size(),
                                        cudaMemcpyDeviceToHost, s));
        }
        const int nlog = res[k].log_count < c.oplog_capacity ? res[k].log_count : c.oplog_capacity;
        if (nlog > 0) {
            logs[k].resize(static_cast<size_t>(nlog));
            GD_TRY_CUDA(cudaMemcpyAsync(logs[k].data(), c.oplog.ptr, sizeof(OperatorLog) * logs[k].size(),
                                        cudaMemcpyDeviceToHost, s));
        }
        CtlResult *hr = reinterpret_cast<CtlResult *>(c.host_ctl);
        *hr = fresh_result(res[k].operator_index);
        GD_TRY_CUDA(cudaMemcpyAsync(&ctl_of(c)->res, hr, sizeof(CtlResult), cudaMemcpyHostToDevice, s));
        GD_TRY_CUDA(cudaMemsetAsync(c.small.ptr + c.events_offset, 0, sizeof(unsigned long long), s));
    }
    GD_TRY_CUDA(cudaStreamSynchronize(s));
    Status first = Status::ok();
    for (int k = 0; k < count; ++k) {
        Collider &c = *cs[k];
        const CtlResult &r = res[k];
        for (const BathRecord &rec : recs[k]) c.summary.record(rec);
        for (const OperatorLog &rec : logs[k]) {
            c.operator_log += operator_log_line(rec);
            c.phase_seconds[0] += rec.rate_seconds;
            c.phase_seconds[1] += rec.chain_seconds;
            c.phase_seconds[2] += rec.audit_seconds;
            c.phase_seconds[3] += rec.wall_seconds;
        }
        c.summary.records_dropped += r.log_dropped;
        // the persistent chain is one launch per wave (the reference relaunches capped chains)
        c.summary.operator_count = r.operator_index;
        c.summary.wave_count += r.waves;
        c.summary.continuation_launches += r.waves;
        c.summary.records_dropped += r.rec_dropped;
        c.stats = gd_operator_stats{};
        c.stats.waves = r.waves;
        c.stats.chain_launches = r.waves;
        c.stats.owner_updates = r.owner_updates;
        c.stats.events = static_cast<long long>(events[k]);
        c.stats.min_duration = r.min_duration;
        c.stats.max_duration = r.max_duration;
        c.launches += c.pending_launches + static_cast<long long>(c.body_launches) * r.waves;
        c.pending_launches = 0;
        c.results_pending = false;
        if (r.error && first) {
            first = ctl_status(r.error);
            if (r.error < 100 && r.error_detail) first.detail = r.error_detail;
            if (first_failed) *first_failed = k;
        }
    }
    return first;
}

Status collider_check(Collider &c, cudaStream_t s) {
    Collider *one = &c;
    return collider_check_many(&one, 1, s, nullptr);
}

// An output boundary: bath states and the summary start afresh (swarm_runtime.cu:490-496); the
// results of operators not read yet are read first.
Status collider_reset_state(Collider &c, cudaStream_t s) {
    Status st = Status::ok();
    if (c.results_pending) st = collider_check(c, s);
    ctl_launch_clear(ctl_of(c), s);
    GD_TRY_CUDA(cudaGetLastError());
    GD_TRY_CUDA(cudaStreamSynchronize(s));
    c.summary = ControllerSummary();
    return st;
}

// _record_col_bath (_col_bound.cuh:219-238)
void ControllerSummary::record(const BathRecord &r) {
    const BathResult &res = r.result;
    bath_count++;
    continuation_launches += r.continuation_launches;
    activity_overshoots += res.activity_overshoot ? 1 : 0;
    distribution_overshoots += res.distribution_overshoot ? 1 : 0;
    persistent_overshoots += res.persistent_overshoot ? 1 : 0;
    minimum_duration = std::min(minimum_duration, r.duration);
    maximum_duration = std::max(maximum_duration, r.duration);
    minimum_limit_scale = std::min(minimum_limit_scale, r.limit_after);
    maximum_f = std::max(maximum_f, res.max_f);
    maximum_e = std::max(maximum_e, res.max_e);
    maximum_touched = std::max(maximum_touched, res.max_touched);
    maximum_events = std::max(maximum_events, res.max_events);
    maximum_g = std::max(maximum_g, res.max_g);
    maximum_g_upper = std::max(maximum_g_upper, res.max_g_upper);
    maximum_d_bath = std::max(maximum_d_bath, res.d_bath);
    baths.push_back(r);
}

// The text save_col_controller writes (_col_bound.cuh:242-299): schema 2, 17 significant digits.
std::string ControllerSummary::json() const {
    std::ostringstream f;
    const double min_dur = std::isfinite(minimum_duration) ? minimum_duration : 0.0;
    f << std::setprecision(17);
    f << "{\n"
      << "  \"schema\": 2,\n"
      << "  \"operator_count\": " << operator_count << ",\n"
      << "  \"bath_count\": " << bath_count << ",\n"
      << "  \"wave_count\": " << wave_count << ",\n"
      << "  \"continuation_launches\": " << continuation_launches << ",\n"
      << "  \"activity_overshoots\": " << activity_overshoots << ",\n"
      << "  \"distribution_overshoots\": " << distribution_overshoots << ",\n"
      << "  \"persistent_overshoots\": " << persistent_overshoots << ",\n"
      << "  \"minimum_duration\": " << min_dur << ",\n"
      << "  \"maximum_duration\": " << maximum_duration << ",\n"
      << "  \"minimum_limit_scale\": " << minimum_limit_scale << ",\n"
      << "  \"maximum_f\": " << maximum_f << ",\n"
      << "  \"maximum_e\": " << maximum_e << ",\n"
      << "  \"maximum_touched\": " << maximum_touched << ",\n"
      << "  \"maximum_events\": " << maximum_events << ",\n"
      << "  \"maximum_g\": " << maximum_g << ",\n"
      << "  \"maximum_g_upper\": " << maximum_g_upper << ",\n"
      << "  \"maximum_d_bath\": " << maximum_d_bath << ",\n"
      << "  \"baths\": [\n";
    for (size_t k = 0; k < baths.size(); ++k) {
        const BathRecord &r = baths[k];
        const BathResult &res = r.result;
        f << "    {\"operator\": " << r.operator_index << ", \"group\": " << r.group_index
          << ", \"bath\": " << r.bath_index << ", \"merged_bins\": " << r.merged_bins
          << ", \"continuation_launches\": " << r.continuation_launches << ", \"duration\": " << r.duration
          << ", \"limit_before\": " << r.limit_before << ", \"limit_after\": " << r.limit_after
          << ", \"max_f\": " << res.max_f << ", \"max_e\": " << res.max_e << ", \"max_touched\": " << res.max_touched
          << ", \"max_events\": " << res.max_events << ", \"max_g\": " << res.max_g
          << ", \"max_g_upper\": " << res.max_g_upper << ", \"d_bath\": " << res.d_bath
          << ", \"activity_overshoot\": " << (res.activity_overshoot ? "true" : "false")
          << ", \"distribution_overshoot\": " << (res.distribution_overshoot ? "true" : "false")
          << ", \"persistent_overshoot\": " << (res.persistent_overshoot ? "true" : "false") << "}"
          << ((k + 1 < baths.size()) ? "," : "") << "\n";
    }
    f << "  ]\n}\n";
    return f.str();
}

// Kernel attributes and persistent grid sizes, once per collider.
static Status collider_setup(Collider &c, const Model &m) {
    if (c.setup_done) return Status::ok();
    const int K = m.n_k, R = m.raw_bins;
    int dev = 0;
    GD_TRY_CUDA(cudaGetDevice(&dev));
    GD_TRY_CUDA(cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, dev));
    if (c.sms <= 0) c.sms = 1;
    c.rate_smem = static_cast<size_t>(4) * (4 * 8 + 4) * K;
    if (c.rate_smem > 48 * 1024) {
        GD_TRY_CUDA(cudaFuncSetAttribute(k_bath_rate<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(c.rate_smem)));
        GD_TRY_CUDA(cudaFuncSetAttribute(k_bath_rate<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(c.rate_smem)));
        GD_TRY_CUDA(cudaFuncSetAttribute(k_rate_fold, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(c.rate_smem)));
    }
    if (R <= kAuditSmemBins)
        GD_TRY_CUDA(cudaFuncSetAttribute(k_audit_bin_blocked, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(audit_blocked_smem(R))));
    c.chain_smem = static_cast<size_t>(kChainWarps) * (kChainDoubles * 8 + 4 + 1) * K;  // doubles, last_w, high_w
    const bool phys = m.coag_kernel == GD_KERNEL_CUSTOM && use_env_cache(m);
    if (phys)
        c.chain_kernel = K <= 64 ? reinterpret_cast<const void *>(&k_chain<2, true>)
                                 : (K <= 128 ? reinterpret_cast<const void *>(&k_chain<4, true>)
                                             : reinterpret_cast<const void *>(&k_chain<8, true>));
    else
        c.chain_kernel = K <= 64 ? reinterpret_cast<const void *>(&k_chain<2, false>)
                                 : (K <= 128 ? reinterpret_cast<const void *>(&k_chain<4, false>)
                                             : reinterpret_cast<const void *>(&k_chain<8, false>));
    if (c.chain_smem > 48 * 1024)
        GD_TRY_CUDA(cudaFuncSetAttribute(c.chain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(c.chain_smem)));
    int per_sm = 0;
    GD_TRY_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, c.chain_kernel, kChainWarps * 32, c.chain_smem));
    c.chain_grid = c.sms * (per_sm < 1 ? 1 : per_sm);
    c.setup_done = true;
    return Status::ok();
}

// The operator's kernels, in stream order on q: the bath-start pass before the loop, then a
// conditional WHILE node whose body, captured on the collider's body stream, is one wave.  q is
// capturing (the collider's own capture or the caller's): no launch here depends on a value the
// host reads back.
static Status enqueue_operator(Collider &c, const Model &m, int n, gd_particle *part, curandState *rng,
                               const int32_t *codes, const double *measure, const unsigned char *active,
                               int32_t *spatial_out, double duration, const double *duration_dev,
                               double duration_scale, const double *clock_sim_dev, double total_dust_mass,
                               cudaStream_t q) {
    const int K = m.n_k;
    const int G = m.local_groups, S = m.col_bin_s, R = m.raw_bins, W = (G + 31) / 32;
    const Small L = small_layout(m);
    int32_t *spatial = c.spatial.ptr;
    const int TPB = 256;
    const int persist = c.sms * 8;  // blocks of the grid-stride kernels
    auto grid_for = [&](long long items, int per_block) {
        return static_cast<int>(std::max(1ll, std::min<long long>((items + per_block - 1) / per_block, persist)));
    };
    CtlDev *ctl = ctl_of(c);
    const WaveInfo *w = &ctl->wave;
    long long pre = 0;
    int body = 0;

    const bool env_on = use_env_cache(m) && m.coag_kernel == GD_KERNEL_CUSTOM;
    if (c.diagnostics) {
        GD_TRY_CUDA(cudaMemsetAsync(c.event_count.ptr, 0, sizeof(unsigned long long) * kEventCategories, q));
        GD_TRY_CUDA(cudaMemsetAsync(c.event_log_mass.ptr, 0, sizeof(double) * kEventCategories, q));
    }
    if (env_on) {
        ++pre;
        k_env_cache<<<(n + TPB - 1) / TPB, TPB, 0, q>>>(m, n, part, reinterpret_cast<Env *>(c.env.ptr));
    }
    CtlPtrs p;
    p.gcount = at<int>(c.small, L.gcount);
    p.gcursor = at<int>(c.small, L.gcursor);
    p.graph = at<unsigned>(c.small, L.graph);
    p.binmap = at<int>(c.small, L.binmap);
    p.merged = at<int>(c.small, L.merged);
    p.ratebin = at<RateBin>(c.small, L.ratebin);
    p.audit = at<AuditBin>(c.small, L.audit);
    p.error_flag = at<int>(c.small, L.error_flag);
    p.dt = at<double>(c.small, L.dt);
    p.records = c.records.ptr;
    p.record_capacity = c.record_capacity;
    p.conf_log = c.conf_log.ptr;
    const bool log_on = c.diagnostics && c.oplog.ptr;
    p.queued = log_on ? at<int>(c.small, L.queued) : nullptr;
    p.oplog = log_on ? c.oplog.ptr : nullptr;
    p.oplog_capacity = log_on ? c.oplog_capacity : 0;
    p.event_count = log_on ? c.event_count.ptr : nullptr;
    p.event_log_mass = log_on ? c.event_log_mass.ptr : nullptr;

    // owner lists and the group dependency graph, once per geometry epoch
    if (!c.local_geometry_valid) {
        GD_TRY(space_bin(m, part, n, spatial, q));
        ++pre;
        if (spatial_out && spatial_out != spatial)
            GD_TRY_CUDA(cudaMemcpyAsync(spatial_out, spatial, sizeof(int32_t) * n, cudaMemcpyDeviceToDevice, q));
        GD_TRY_CUDA(cudaMemsetAsync(c.small.ptr + L.gcount, 0, 4 * G, q));
        GD_TRY_CUDA(cudaMemsetAsync(c.small.ptr + L.graph, 0, 4 * G * W, q));
        pre += 4;
        k_group_count<<<(n + kGroupSpan - 1) / kGroupSpan, kGroupTPB, 0, q>>>(n, G, spatial, at<int>(c.small, L.gcount));
        k_dep_graph<<<(n + kGroupSpan - 1) / kGroupSpan, kGroupTPB, 0, q>>>(n, K, G, W, at<unsigned int>(c.small, L.graph),
                                                                             spatial, codes, active);
        ctl_launch_geometry(ctl, p, G, q);
        k_group_fill<<<(n + kGroupSpan - 1) / kGroupSpan, kGroupTPB, 0, q>>>(n, G, spatial, at<int>(c.small, L.gcursor),
                                                                              c.group_sorted.ptr);
        if (c.height.ptr) {
            ++pre;
            k_disk_height<<<(n + TPB - 1) / TPB, TPB, 0, q>>>(m, n, part, c.height.ptr);
        }
        GD_TRY_CUDA(cudaGetLastError());
        // new neighbour lists and measures: no stored rate stands
        GD_TRY_CUDA(cudaMemsetAsync(c.rated.ptr, 0xff, sizeof(int) * n, q));
        c.local_geometry_valid = true;
    }

    const double lambda0 = n / static_cast<double>(K) / total_dust_mass;
    if (lambda0 != c.rated_lambda0) {
        GD_TRY_CUDA(cudaMemsetAsync(c.rated.ptr, 0xff, sizeof(int) * n, q));
        c.rated_lambda0 = lambda0;
    }
    const Env *env = env_on ? reinterpret_cast<const Env *>(c.env.ptr) : nullptr;
    const bool rate_cached = m.coag_kernel == GD_KERNEL_CUSTOM && use_env_cache(m) && env;

    int *ids = c.ids.ptr;
    double *lower = at<double>(c.small, L.lower), *upper = at<double>(c.small, L.upper);
    double *dt = p.dt;
    int *binmap = at<int>(c.small, L.binmap);
    RateBin *ratebin = at<RateBin>(c.small, L.ratebin);
    AuditBin *audit = at<AuditBin>(c.small, L.audit);

    // publish the reservoir of the wave's owners (kernels skip a wave without new rates)
    auto initialize = [&](cudaStream_t st, int &launches) {
        ++launches;
        k_bath_init<<<grid_for(n, TPB), TPB, 0, st>>>(w, ids, part, c.size_old.ptr, c.numr_old.ptr, c.time.ptr,
                                                       c.events.ptr, c.complete.ptr, c.hazard.ptr, c.jump1.ptr,
                                                       c.jump2.ptr, c.jumpmax.ptr, c.stamp.ptr);
    };
    // rates, size bins and merged rate bins of the wave's owners
    auto rates_and_bins = [&](cudaStream_t st, int &launches) -> Status {
        launches += 7;
        k_size_zero<<<(G + TPB - 1) / TPB, TPB, 0, st>>>(G, at<unsigned long long>(c.small, L.mmin),
                                                          at<unsigned long long>(c.small, L.mmax));
        if (G <= kScanSmemEntries)
            k_size_scan_blocked<<<(n + kAuditSpan - 1) / kAuditSpan, kAuditTPB, sizeof(unsigned long long) * 2 * G,
                                  st>>>(w, ids, part, spatial, active, G, at<unsigned long long>(c.small, L.mmin),
                                        at<unsigned long long>(c.small, L.mmax));
        else
            k_size_scan<<<(n + TPB - 1) / TPB, TPB, 0, st>>>(w, ids, part, spatial, active,
                                                              at<unsigned long long>(c.small, L.mmin),
                                                              at<unsigned long long>(c.small, L.mmax));
        k_size_bnds<<<(G + TPB - 1) / TPB, TPB, 0, st>>>(G, at<unsigned long long>(c.small, L.mmin),
                                                          at<unsigned long long>(c.small, L.mmax), lower, upper);
        RateArgs ra;
        ra.ids = ids;
        ra.height = c.height.ptr;
        ra.w = w;
        ra.part = part;
        ra.codes = codes;
        ra.measure = measure;
        ra.active = active;
        ra.size_old = c.size_old.ptr;
        ra.numr_old = c.numr_old.ptr;
        ra.env = env;
        ra.lambda0 = lambda0;
        ra.rate = c.rate.ptr;
        ra.change = c.change_rate.ptr;
        ra.second = c.second_rate.ptr;
        ra.cached = reinterpret_cast<RateMoments *>(c.cached.ptr);
        ra.stamp = c.stamp.ptr;
        ra.rated = c.rated.ptr;
        const bool stored = c.leaf.ptr != nullptr;
        ra.leaf = c.leaf.ptr;
        ra.plane = static_cast<size_t>(n) * m.n_k;
        ra.pairs = c.pairs.ptr;
        ra.pair_count = at<int>(c.small, L.pair_count);
        ra.folds = c.folds.ptr;
        ra.fold_count = at<int>(c.small, L.fold_count);
        ra.whole = stored ? c.whole.ptr : nullptr;
        ra.whole_count = at<int>(c.small, L.whole_count);
        if (stored) {
            // the wave's owners sorted: evaluated whole, changed pairs only, or standing
            GD_TRY_CUDA(cudaMemsetAsync(c.small.ptr + L.pair_count, 0, 12, st));
            launches += 1;
            k_rate_plan<<<grid_for(n, 256), 256, 0, st>>>(m, ra);
        }
        if (rate_cached)
            k_bath_rate<true><<<grid_for(n, 4), 128, c.rate_smem, st>>>(m, ra);
        else
            k_bath_rate<false><<<grid_for(n, 4), 128, c.rate_smem, st>>>(m, ra);
        if (stored) {
            // the changed pairs of the owners whose own entry is unchanged, then their folds
            launches += 2;
            if (rate_cached)
                k_pair_eval<true><<<grid_for(static_cast<long long>(n) * m.n_k, 128), 128, 0, st>>>(m, ra);
            else
                k_pair_eval<false><<<grid_for(static_cast<long long>(n) * m.n_k, 128), 128, 0, st>>>(m, ra);
            k_rate_fold<<<grid_for(n, 4), 128, c.rate_smem, st>>>(m, ra);
        }
        GD_TRY_CUDA(cudaMemsetAsync(c.small.ptr + L.counts, 0, 4 * R, st));
        if (R <= kScanSmemEntries)
            k_count_bin_blocked<<<(n + kAuditSpan - 1) / kAuditSpan, kAuditTPB, sizeof(int) * R, st>>>(
                m, w, ids, at<int>(c.small, L.counts), part, spatial, active, lower, upper, R);
        else
            k_count_bin<<<(n + TPB - 1) / TPB, TPB, 0, st>>>(m, w, ids, at<int>(c.small, L.counts), part, spatial,
                                                              active, lower, upper);
        GD_TRY_CUDA(cudaMemsetAsync(ratebin, 0, sizeof(RateBin) * R, st));
        k_binmap<<<1, 1, 0, st>>>(m, w, at<int>(c.small, L.counts), binmap, at<int>(c.small, L.merged));
        if (R <= kScanSmemEntries)
            k_rate_bins_blocked<<<(n + kAuditSpan - 1) / kAuditSpan, kAuditTPB,
                                  (sizeof(double) * 4 + sizeof(int) * 2) * R, st>>>(
                m, w, ids, ratebin, part, c.rate.ptr, c.change_rate.ptr, c.second_rate.ptr, spatial, binmap, active,
                lower, upper, R);
        else
            k_rate_bins<<<(n + TPB - 1) / TPB, TPB, 0, st>>>(m, w, ids, ratebin, part, c.rate.ptr, c.change_rate.ptr,
                                                              c.second_rate.ptr, spatial, binmap, active, lower, upper);
        GD_TRY_CUDA(cudaGetLastError());
        return Status::ok();
    };

    // the conditional that repeats the wave body, created in the graph q is capturing into
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t graph = nullptr;
    GD_TRY_CUDA(cudaStreamGetCaptureInfo(q, &cs, nullptr, &graph));
    if (cs != cudaStreamCaptureStatusActive) return err(GD_ERR_CUDA, "collision operator stream is not capturing");
    cudaGraphConditionalHandle handle;
    GD_TRY_CUDA(cudaGraphConditionalHandleCreate(&handle, graph, 0, 0));

    // tick zero: every group starts from the same published reservoir (_col_chain.cuh:175-214)
    int pre_int = 0;
    ctl_launch_reset(ctl, duration, duration_dev, duration_scale, clock_sim_dev, n, G, S, R, q);
    initialize(q, pre_int);
    GD_TRY(rates_and_bins(q, pre_int));
    ctl_launch_begin(ctl, m, p, handle, q);
    ctl_launch_wave_ids(ctl, c.group_sorted.ptr, ids, grid_for(n, TPB), q);
    pre += pre_int + 3;
    GD_TRY_CUDA(cudaGetLastError());

    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    GD_TRY_CUDA(cudaStreamGetCaptureInfo(q, &cs, nullptr, &graph, &deps, &ndeps));
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t loop;
    GD_TRY_CUDA(cudaGraphAddNode(&loop, graph, deps, ndeps, &cp));
    cudaGraph_t wave_graph = cp.conditional.phGraph_out[0];
    GD_TRY_CUDA(cudaStreamUpdateCaptureDependencies(q, &loop, 1, cudaStreamSetCaptureDependencies));

    // the wave body (_col_chain.cuh:215-537): chains, audit, bath finish and schedule advance, then
    // the next wave's owners, reservoir, rates and bath lengths
    cudaStream_t b = c.body_stream;
    GD_TRY_CUDA(cudaStreamBeginCaptureToGraph(b, wave_graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    Status st = [&]() -> Status {
        if (log_on) ctl_launch_mark(ctl, 0, b);
        GD_TRY_CUDA(cudaMemsetAsync(c.small.ptr + L.merged + 4, 0, 16, b));  // error_flag, queued, light, head
        ChainArgs ca;
        // A wave of every group holds every particle once: the skip scan (whose queue order the chain
        // does not depend on) then walks them in index order, with coalesced per-particle loads.
        ca.ids = ids;
        ca.w = w;
        ca.rng = rng;
        ca.active = active;
        ca.measure = measure;
        ca.spatial = spatial;
        ca.dt = dt;
        ca.cached = reinterpret_cast<const RateMoments *>(c.cached.ptr);
        ca.time = c.time.ptr;
        ca.hazard = c.hazard.ptr;
        ca.jump1 = c.jump1.ptr;
        ca.jump2 = c.jump2.ptr;
        ca.jumpmax = c.jumpmax.ptr;
        ca.events = c.events.ptr;
        ca.complete = c.complete.ptr;
        ca.queue = c.queue.ptr;
        ca.queued = at<int>(c.small, L.queued);
        ca.n = n;
        k_skip_scan<<<grid_for(n, TPB), TPB, 0, b>>>(ca);
        ChainRun cr;
        cr.height = c.height.ptr;
        cr.part_ro = part;
        cr.part = part;
        cr.codes = codes;
        cr.size_old = c.size_old.ptr;
        cr.numr_old = c.numr_old.ptr;
        cr.env = env;
        cr.lambda0 = lambda0;
        cr.error = c.error.ptr;
        cr.error_flag = at<int>(c.small, L.error_flag);
        cr.head = at<int>(c.small, L.head);
        cr.events_total = at<unsigned long long>(c.small, L.events);
        cr.event_count = c.diagnostics ? c.event_count.ptr : nullptr;
        cr.event_log_mass = c.diagnostics ? c.event_log_mass.ptr : nullptr;
        const int blocks = std::min(c.chain_grid, (n + kChainWarps - 1) / kChainWarps);
        {
            void *args[] = {const_cast<Model *>(&m), &ca, &cr};
            GD_TRY_CUDA(cudaLaunchKernel(c.chain_kernel, dim3(blocks), dim3(kChainWarps * 32), args, c.chain_smem, b));
        }
        if (log_on) {
            ctl_launch_mark(ctl, 1, b);
            body += 2;
        }
        // audit of the completed baths
        GD_TRY_CUDA(cudaMemsetAsync(audit, 0, sizeof(AuditBin) * R, b));
        AuditArgs aa;
        aa.ids = ids;
        aa.w = w;
        aa.count = 0;
        aa.bin = audit;
        aa.part = part;
        aa.size_old = c.size_old.ptr;
        aa.numr_old = c.numr_old.ptr;
        aa.rate = c.rate.ptr;
        aa.hazard = c.hazard.ptr;
        aa.jump1 = c.jump1.ptr;
        aa.jump2 = c.jump2.ptr;
        aa.jumpmax = c.jumpmax.ptr;
        aa.events = c.events.ptr;
        aa.spatial = spatial;
        aa.binmap = binmap;
        aa.active = active;
        aa.dt = dt;
        aa.lower = lower;
        aa.upper = upper;
        if (R <= kAuditSmemBins)
            k_audit_bin_blocked<<<(n + kAuditSpan - 1) / kAuditSpan, kAuditTPB, audit_blocked_smem(R), b>>>(m, aa, R);
        else
            k_audit_bin<<<(n + kAuditTPB - 1) / kAuditTPB, kAuditTPB, 0, b>>>(m, aa);
        ctl_launch_finish(ctl, m, p, handle, b);
        ctl_launch_wave_ids(ctl, c.group_sorted.ptr, ids, grid_for(n, TPB), b);
        body += 5;
        if (log_on) {
            ctl_launch_mark(ctl, 2, b);
            body += 1;
        }
        initialize(b, body);
        GD_TRY(rates_and_bins(b, body));
        if (log_on) {
            ctl_launch_mark(ctl, 3, b);
            body += 1;
        }
        ctl_launch_adapt(ctl, m, p, handle, b);
        body += 1;
        GD_TRY_CUDA(cudaGetLastError());
        return Status::ok();
    }();
    cudaGraph_t captured = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b, &captured);
    GD_TRY(st);
    GD_TRY_CUDA(e);
    c.pending_launches += pre;
    c.body_launches = body;
    return Status::ok();
}

// col_bath_rate (col_bath_rate.cu:13-130) for every owner, alone and eagerly launched: the
// bath-start rate moments with the current particles as the published reservoir.  Scratch arrays
// hold the reservoir and the stored-rate stamps, so no operator state changes.
Status bath_rates(Collider &c, const Model &m, int n, const gd_particle *part, const int32_t *codes,
                  const double *measure, const unsigned char *active, double total_dust_mass, double *out4,
                  int *launches, cudaStream_t s) {
    if (!(total_dust_mass > 0) || !std::isfinite(total_dust_mass))
        return err(GD_ERR_INVALID_ARGUMENT, "total dust mass must be positive and finite");
    GD_TRY(collider_setup(c, m));
    const int K = m.n_k;
    DevBuf<double> size_old, numr_old, rate, change, second;
    DevBuf<int> stamp, rated;
    DevBuf<WaveInfo> wave;
    GD_TRY_CUDA(size_old.alloc(n));
    GD_TRY_CUDA(numr_old.alloc(n));
    GD_TRY_CUDA(rate.alloc(n));
    GD_TRY_CUDA(change.alloc(n));
    GD_TRY_CUDA(second.alloc(n));
    GD_TRY_CUDA(stamp.alloc(n));
    GD_TRY_CUDA(rated.alloc(n));
    GD_TRY_CUDA(wave.alloc(1));
    const WaveInfo w{n, 1, 1, 1, 1, {0, 0, 0}};
    GD_TRY_CUDA(cudaMemcpyAsync(wave.ptr, &w, sizeof(w), cudaMemcpyHostToDevice, s));
    GD_TRY_CUDA(cudaMemsetAsync(stamp.ptr, 0, sizeof(int) * n, s));
    GD_TRY_CUDA(cudaMemsetAsync(rated.ptr, 0xff, sizeof(int) * n, s));
    GD_TRY_CUDA(cudaMemcpy2DAsync(size_old.ptr, sizeof(double), &part[0].par_size, sizeof(gd_particle), sizeof(double),
                                  n, cudaMemcpyDeviceToDevice, s));
    GD_TRY_CUDA(cudaMemcpy2DAsync(numr_old.ptr, sizeof(double), &part[0].par_numr, sizeof(gd_particle), sizeof(double),
                                  n, cudaMemcpyDeviceToDevice, s));
    const bool env_on = use_env_cache(m) && m.coag_kernel == GD_KERNEL_CUSTOM;
    const int TPB = 256;
    if (env_on) k_env_cache<<<(n + TPB - 1) / TPB, TPB, 0, s>>>(m, n, part, reinterpret_cast<Env *>(c.env.ptr));
    if (c.height.ptr) k_disk_height<<<(n + TPB - 1) / TPB, TPB, 0, s>>>(m, n, part, c.height.ptr);
    RateArgs ra;
    ra.ids = nullptr;
    ra.height = c.height.ptr;
    ra.w = wave.ptr;
    ra.part = part;
    ra.codes = codes;
    ra.measure = measure;
    ra.active = active;
    ra.size_old = size_old.ptr;
    ra.numr_old = numr_old.ptr;
    ra.env = env_on ? reinterpret_cast<const Env *>(c.env.ptr) : nullptr;
    ra.lambda0 = n / static_cast<double>(K) / total_dust_mass;
    ra.rate = rate.ptr;
    ra.change = change.ptr;
    ra.second = second.ptr;
    ra.cached = reinterpret_cast<RateMoments *>(out4);
    ra.leaf = nullptr;  // every owner evaluated whole, nothing stored
    ra.plane = 0;
    ra.pairs = nullptr;
    ra.pair_count = nullptr;
    ra.folds = nullptr;
    ra.fold_count = nullptr;
    ra.whole = nullptr;
    ra.whole_count = nullptr;
    ra.stamp = stamp.ptr;
    ra.rated = rated.ptr;
    const int grid = std::max(1, std::min((n + 3) / 4, c.sms * 8));
    if (env_on)
        k_bath_rate<true><<<grid, 128, c.rate_smem, s>>>(m, ra);
    else
        k_bath_rate<false><<<grid, 128, c.rate_smem, s>>>(m, ra);
    if (launches) *launches += (env_on ? 2 : 1) + (c.height.ptr ? 1 : 0);
    GD_TRY_CUDA(cudaGetLastError());
    GD_TRY_CUDA(cudaStreamSynchronize(s));  // the scratch is freed on return
    return Status::ok();
}

// One frozen bath of `bath` seconds for every owner, launched eagerly: the bath-start rates, the skip
// scan and the chain (col_bath_rate, col_skip_scan, col_chain_run) with the current particles as the
// published reservoir; the particles and RNG streams advance in place.  This is the operator's wave
// when a single bath covers the whole operator (every group due once, dt = bath), outside any graph,
// so the chain can be timed and profiled alone.  Scratch arrays hold the per-owner chain state; the
// collider's operator state is left unchanged.
Status bath_chain(Collider &c, const Model &m, int n, gd_particle *part, curandState *rng, const int32_t *codes,
                  const double *measure, const unsigned char *active, double total_dust_mass, double bath,
                  unsigned long long *events, int *launches, cudaStream_t s) {
    if (!(total_dust_mass > 0) || !std::isfinite(total_dust_mass))
        return err(GD_ERR_INVALID_ARGUMENT, "total dust mass must be positive and finite");
    if (!(bath > 0) || !std::isfinite(bath)) return err(GD_ERR_INVALID_ARGUMENT, "bath duration must be positive and finite");
    GD_TRY(collider_setup(c, m));
    const int K = m.n_k;
    DevBuf<double> size_old, numr_old, rate, change, second, cached, time, hazard, jump1, jump2, jumpmax, dt;
    DevBuf<int> stamp, rated, ev, error, queue, spatial;
    DevBuf<unsigned char> complete, small;
    DevBuf<WaveInfo> wave;
    for (DevBuf<double> *b : {&size_old, &numr_old, &rate, &change, &second, &time, &hazard, &jump1, &jump2, &jumpmax})
        GD_TRY_CUDA(b->alloc(n));
    GD_TRY_CUDA(cached.alloc(static_cast<size_t>(n) * 4));
    GD_TRY_CUDA(dt.alloc(1));
    for (DevBuf<int> *b : {&stamp, &rated, &ev, &error, &queue, &spatial}) GD_TRY_CUDA(b->alloc(n));
    GD_TRY_CUDA(complete.alloc(n));
    GD_TRY_CUDA(small.alloc(32));  // queued [2] at 0, head at 8, error flag at 12, events total at 16
    GD_TRY_CUDA(wave.alloc(1));
    const WaveInfo w{n, 1, 1, 1, 1, {0, 0, 0}};
    GD_TRY_CUDA(cudaMemcpyAsync(wave.ptr, &w, sizeof(w), cudaMemcpyHostToDevice, s));
    GD_TRY_CUDA(cudaMemcpyAsync(dt.ptr, &bath, sizeof(double), cudaMemcpyHostToDevice, s));
    GD_TRY_CUDA(cudaMemsetAsync(stamp.ptr, 0, sizeof(int) * n, s));
    GD_TRY_CUDA(cudaMemsetAsync(rated.ptr, 0xff, sizeof(int) * n, s));
    for (DevBuf<double> *b : {&time, &hazard, &jump1, &jump2, &jumpmax})
        GD_TRY_CUDA(cudaMemsetAsync(b->ptr, 0, sizeof(double) * n, s));
    for (DevBuf<int> *b : {&ev, &error, &spatial}) GD_TRY_CUDA(cudaMemsetAsync(b->ptr, 0, sizeof(int) * n, s));
    GD_TRY_CUDA(cudaMemsetAsync(complete.ptr, 0, n, s));
    GD_TRY_CUDA(cudaMemsetAsync(small.ptr, 0, 32, s));
    GD_TRY_CUDA(cudaMemcpy2DAsync(size_old.ptr, sizeof(double), &part[0].par_size, sizeof(gd_particle), sizeof(double),
                                  n, cudaMemcpyDeviceToDevice, s));
    GD_TRY_CUDA(cudaMemcpy2DAsync(numr_old.ptr, sizeof(double), &part[0].par_numr, sizeof(gd_particle), sizeof(double),
                                  n, cudaMemcpyDeviceToDevice, s));
    const bool env_on = use_env_cache(m) && m.coag_kernel == GD_KERNEL_CUSTOM;
    const Env *env = env_on ? reinterpret_cast<const Env *>(c.env.ptr) : nullptr;
    const int TPB = 256;
    if (env_on) k_env_cache<<<(n + TPB - 1) / TPB, TPB, 0, s>>>(m, n, part, reinterpret_cast<Env *>(c.env.ptr));
    if (c.height.ptr) k_disk_height<<<(n + TPB - 1) / TPB, TPB, 0, s>>>(m, n, part, c.height.ptr);
    RateArgs ra{};
    ra.height = c.height.ptr;
    ra.w = wave.ptr;
    ra.part = part;
    ra.codes = codes;
    ra.measure = measure;
    ra.active = active;
    ra.size_old = size_old.ptr;
    ra.numr_old = numr_old.ptr;
    ra.env = env;
    ra.lambda0 = n / static_cast<double>(K) / total_dust_mass;
    ra.rate = rate.ptr;
    ra.change = change.ptr;
    ra.second = second.ptr;
    ra.cached = reinterpret_cast<RateMoments *>(cached.ptr);
    ra.stamp = stamp.ptr;
    ra.rated = rated.ptr;
    const int grid = std::max(1, std::min((n + 3) / 4, c.sms * 8));
    if (env_on)
        k_bath_rate<true><<<grid, 128, c.rate_smem, s>>>(m, ra);
    else
        k_bath_rate<false><<<grid, 128, c.rate_smem, s>>>(m, ra);
    ChainArgs ca{};
    ca.w = wave.ptr;
    ca.rng = rng;
    ca.active = active;
    ca.measure = measure;
    ca.spatial = spatial.ptr;  // every owner in group 0, whose bath ends at dt[0]
    ca.dt = dt.ptr;
    ca.cached = reinterpret_cast<const RateMoments *>(cached.ptr);
    ca.time = time.ptr;
    ca.hazard = hazard.ptr;
    ca.jump1 = jump1.ptr;
    ca.jump2 = jump2.ptr;
    ca.jumpmax = jumpmax.ptr;
    ca.events = ev.ptr;
    ca.complete = complete.ptr;
    ca.queue = queue.ptr;
    ca.queued = reinterpret_cast<int *>(small.ptr);
    ca.n = n;
    k_skip_scan<<<std::max(1, std::min((n + TPB - 1) / TPB, c.sms * 8)), TPB, 0, s>>>(ca);
    ChainRun cr{};
    cr.height = c.height.ptr;
    cr.part_ro = part;
    cr.part = part;
    cr.codes = codes;
    cr.size_old = size_old.ptr;
    cr.numr_old = numr_old.ptr;
    cr.env = env;
    cr.lambda0 = ra.lambda0;
    cr.error = error.ptr;
    cr.error_flag = reinterpret_cast<int *>(small.ptr + 12);
    cr.head = reinterpret_cast<int *>(small.ptr + 8);
    cr.events_total = reinterpret_cast<unsigned long long *>(small.ptr + 16);
    const int blocks = std::min(c.chain_grid, (n + kChainWarps - 1) / kChainWarps);
    {
        void *args[] = {const_cast<Model *>(&m), &ca, &cr};
        GD_TRY_CUDA(cudaLaunchKernel(c.chain_kernel, dim3(blocks), dim3(kChainWarps * 32), args, c.chain_smem, s));
    }
    if (launches) *launches += 3 + (env_on ? 1 : 0) + (c.height.ptr ? 1 : 0);
    unsigned char host[32];
    GD_TRY_CUDA(cudaMemcpyAsync(host, small.ptr, sizeof(host), cudaMemcpyDeviceToHost, s));
    GD_TRY_CUDA(cudaStreamSynchronize(s));  // the scratch is freed on return
    int flag = 0;
    std::memcpy(&flag, host + 12, sizeof(int));
    unsigned long long total = 0;
    std::memcpy(&total, host + 16, sizeof(total));
    if (events) *events = total;
    if (flag == 7) return err(GD_ERR_CONTINUATION_LIMIT, "an owner's chain exceeded its event budget", flag);
    if (flag) return err(GD_ERR_CHAIN, "event-chain error", flag);
    return Status::ok();
}

Status collision_operator_enqueue(Collider &c, const Model &m, int n, gd_particle *part, curandState *rng,
                                  const int32_t *codes, const double *measure, const unsigned char *active,
                                  double duration, double total_dust_mass, cudaStream_t q) {
    if (!(total_dust_mass > 0) || !std::isfinite(total_dust_mass))
        return err(GD_ERR_INVALID_ARGUMENT, "total dust mass must be positive and finite");
    if (!(duration > 0) || !std::isfinite(duration)) return err(GD_ERR_INVALID_ARGUMENT, "invalid local collision horizon");
    GD_TRY(collider_setup(c, m));
    GD_TRY(enqueue_operator(c, m, n, part, rng, codes, measure, active, nullptr, duration, nullptr, 1.0, nullptr,
                            total_dust_mass, q));
    c.results_pending = true;
    return Status::ok();
}

Status collision_operator(Collider &c, const Model &m, int n, gd_particle *part, curandState *rng, const int32_t *codes,
                          const double *measure, const unsigned char *active, int32_t *spatial_out, double duration,
                          double total_dust_mass, cudaStream_t s, const double *duration_dev, double duration_scale,
                          const double *clock_sim_dev) {
    if (!(total_dust_mass > 0) || !std::isfinite(total_dust_mass))
        return err(GD_ERR_INVALID_ARGUMENT, "total dust mass must be positive and finite");
    // the reference's horizon check (_col_sched.cuh:30-33), made before any work is queued; a
    // horizon on the device is checked by the controller
    if (!duration_dev && (!(duration > 0) || !std::isfinite(duration)))
        return err(GD_ERR_INVALID_ARGUMENT, "invalid local collision horizon");
    GD_TRY(collider_setup(c, m));
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    GD_TRY_CUDA(cudaStreamIsCapturing(s, &cs));
    if (cs == cudaStreamCaptureStatusInvalidated) return err(GD_ERR_CUDA, "the caller's stream capture is invalidated");
    if (cs == cudaStreamCaptureStatusActive) {
        // inside the caller's capture: the operator becomes part of the caller's graph, whose results
        // gd_check_operator (collider_check) reads after it ran
        GD_TRY(enqueue_operator(c, m, n, part, rng, codes, measure, active, spatial_out, duration, duration_dev,
                                duration_scale, clock_sim_dev, total_dust_mass, s));
        c.results_pending = true;
        return Status::ok();
    }
    // eager: capture the operator on the collider's stream, run the graph on s, read the results
    cudaStream_t q = c.capture_stream;
    GD_TRY_CUDA(cudaStreamBeginCapture(q, cudaStreamCaptureModeThreadLocal));
    const Status st = enqueue_operator(c, m, n, part, rng, codes, measure, active, spatial_out, duration,
                                       duration_dev, duration_scale, clock_sim_dev, total_dust_mass, q);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(q, &graph);
    if (!st || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        c.local_geometry_valid = false;
        if (!st) return st;
        GD_TRY_CUDA(e);
    }
    cudaGraphExec_t exec = nullptr;
    cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie == cudaSuccess) ie = cudaGraphLaunch(exec, s);
    if (ie != cudaSuccess) {
        if (exec) cudaGraphExecDestroy(exec);
        c.local_geometry_valid = false;
        c.pending_launches = 0;
        return cuda_status(ie, "collision operator graph");
    }
    c.results_pending = true;
    const Status r = collider_check(c, s);
    cudaGraphExecDestroy(exec);
    return r;
}

}  // namespace gd
