// Radius-bounded exact top-K with one warp per owner (the range query).
//
// gd_knn_bounded receives a proposed search radius r_i for every owner (the learned proposal).
// Inside a well-proposed radius an owner finds a little more than K sites, so its exact top-K is a
// range query followed by a sort: collect every site with d^2 <= lim^2 = min(q_i, r_i)^2, and if
// there are at least K of them, the K smallest (d^2 bits, code) keys among them are the owner's
// exact K nearest within q_i (every other site lies farther than lim >= their K-th distance).
// Owners that find fewer than K sites inside a radius below q_i, or more than the capacity, are
// handed to the per-lane heap query (knn_fallback) with the full q_i, so the rows stay exact by
// construction and equal to the plain query's bit for bit.
//
// Layout of the work.  One warp per bucket of 32 Morton-ordered owners (a leaf of the bucket tree):
//   1. the warp walks the tree breadth-first once for the bucket: internal boxes against the box
//      around all 32 balls, leaf boxes against each lane's own ball, giving the union leaf list;
//   2. then, owner by owner, all 32 lanes serve that one owner: its ball is tested against the
//      union leaves' boxes (32 per instruction), then against the 8-site sub-boxes of the passing
//      leaves, then the passing 8-site groups are scanned four at a time (a lane per site), and the
//      sites inside the ball are appended to the owner's candidate list with a ballot and a
//      population count: no lane walks a list of its own, so nothing diverges;
//   3. the owner's candidates are sorted by a warp-wide bitonic network over 64 or 128 keys held in
//      registers (strided: element j*32 + lane), the first K are its row, written by 16 lanes as
//      coalesced 16-byte stores;
//   4. after the 32 owners, lane o computes owner o's FP64 ball measure from its K-th d^2.
// The per-lane heap kernel keeps each lane's own heap in shared memory and walks its candidates
// serially with half its lanes idle on average; here the only per-owner serial work is the
// warp-wide network.
#include <climits>
#include <cmath>

#include "gd_geom_device.cuh"
#include "gd_internal.cuh"

namespace gd {

namespace {

constexpr int kRangeWarps = 4;       // warps per block
constexpr int kRangeCap = 128;       // candidates an owner may hold (the 128-key network)
constexpr int kRangeFrontier = 128;  // internal nodes of one breadth-first level
constexpr int kRangeList = 256;      // leaves of the bucket's union list
constexpr int kOwnLeaves = 128;      // leaves an owner's ball reaches
constexpr int kOwnGroups = 256;      // 8-site groups an owner's ball reaches
constexpr int kTrim = 8;             // up to this many candidates above 64 are dropped one by one

struct RangeShared {
    int frontier[kRangeFrontier];
    int list[kRangeList];
    int own_leaves[kOwnLeaves];
    int own_groups[kOwnGroups];
    unsigned long long cand[kRangeCap];
    float kth[32];
};

__device__ __forceinline__ unsigned long long umin64(unsigned long long a, unsigned long long b) { return a < b ? a : b; }
__device__ __forceinline__ unsigned long long umax64(unsigned long long a, unsigned long long b) { return a < b ? b : a; }

// Ascending bitonic sort of 32*J keys held strided across the warp (element j*32 + lane in v[j]).
template <int J>
__device__ __forceinline__ void warp_bitonic(unsigned long long (&v)[J], int lane) {
#pragma unroll
    for (int k = 2; k <= 32 * J; k <<= 1) {
#pragma unroll
        for (int s = k >> 1; s > 0; s >>= 1) {
            if (s >= 32) {
                const int sj = s >> 5;
#pragma unroll
                for (int j = 0; j < J; ++j) {
                    if (j & sj) continue;
                    const int jp = j | sj;
                    const bool asc = ((j * 32) & k) == 0;
                    const unsigned long long lo = umin64(v[j], v[jp]), hi = umax64(v[j], v[jp]);
                    v[j] = asc ? lo : hi;
                    v[jp] = asc ? hi : lo;
                }
            } else {
                const bool lower = (lane & s) == 0;
#pragma unroll
                for (int j = 0; j < J; ++j) {
                    const unsigned long long other = __shfl_xor_sync(0xffffffffu, v[j], s);
                    const bool asc = (((j * 32) | lane) & k) == 0;
                    v[j] = (lower == asc) ? umin64(v[j], other) : umax64(v[j], other);
                }
            }
        }
    }
}

// Writes an owner's row from its sorted keys (element e = j*32 + lane): slot e < K gets the code of
// element e if e < len, else -1.  Returns the K-th kept d^2 (0 for an empty row) on every lane.
template <int J>
__device__ __forceinline__ float write_row(const unsigned long long (&v)[J], int lane, int len, int K, int32_t *row) {
    const int keep = len < K ? len : K;
#pragma unroll
    for (int j = 0; j < J; ++j) {
        const int e = j * 32 + lane;
        if (row && e < K) row[e] = e < keep ? static_cast<int>(static_cast<unsigned int>(v[j])) : -1;
    }
    float kth = 0.0f;
    if (keep > 0) {  // warp-uniform
        const int e = keep - 1;
        unsigned long long sel = v[0];
#pragma unroll
        for (int j = 1; j < J; ++j)
            if (j == (e >> 5)) sel = v[j];
        const unsigned long long kv = __shfl_sync(0xffffffffu, sel, e & 31);
        kth = __uint_as_float(static_cast<unsigned int>(kv >> 32));
    }
    return kth;
}

}  // namespace

struct RangeArgs {
    const float4 *sorted, *lo, *hi, *sub_lo, *sub_hi;
    const float *qrad, *radius;
    const int *counters;
    const gd_particle *part;
    int leaf_slots, k;
    int32_t *codes;
    double *measure;
    float *kth;
    unsigned long long *stats;  // optional: 8-site groups scanned, tree nodes tested, candidates, fallbacks
    int *fb_count;              // buckets with owners left to the heap query
    int *fb_leaf;               // their bucket (leaf) indices
    unsigned int *fb_mask;      // and which lanes
};

__global__ void __launch_bounds__(kRangeWarps * 32, 8) k_knn_range(Model m, RangeArgs a) {
    __shared__ RangeShared sh_all[kRangeWarps];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    RangeShared &sh = sh_all[wib];
    const int leaf = blockIdx.x * kRangeWarps + wib;
    const int n_act = a.counters[0];
    const int n_leaves = (n_act + kLeaf - 1) / kLeaf;
    if (leaf >= n_leaves) return;
    const int K = a.k;
    const unsigned int lt = (1u << lane) - 1u;

    // this lane's owner
    const int i = leaf * kLeaf + lane;
    const float4 me = a.sorted[i];
    const bool valid = i < n_act;
    const int idx = valid ? __float_as_int(me.w) / 3 : 0;
    const float qr = valid ? a.qrad[idx] : 0.0f;
    const float q2 = qr * qr;
    float lim2 = q2;
    if (valid) {
        const float r = a.radius[idx];
        if (r >= 0.0f && r < qr) lim2 = r * r;  // a negative or NaN proposal bounds nothing
    }
    const float cut = valid ? lim2 : -1.0f;
    const float3 qp = make_float3(me.x, me.y, me.z);
    long long st_groups = 0, st_nodes = 0, st_cand = 0;

    // 1. Leaf lists by a breadth-first walk: internal boxes against an axis-aligned box around the
    //    balls (the heap query's conservative inflation), leaf boxes exactly against each ball.
    //    single < 0: the union of the 32 lanes' balls; single = o: owner o's ball of squared radius
    //    sbound alone.  Returns the number of leaves written to out (at most cap), or -1 when a
    //    level or the list outgrows its buffer.
    const int levels = 31 - __clz(a.leaf_slots);
    const int first_leaf = a.leaf_slots - 1;
    auto walk = [&](int single, float sbound, int *out, int cap) -> int {
        const float3 sq = single < 0 ? qp
                                     : make_float3(__shfl_sync(0xffffffffu, qp.x, single),
                                                   __shfl_sync(0xffffffffu, qp.y, single),
                                                   __shfl_sync(0xffffffffu, qp.z, single));
        const float scut = single < 0 ? cut : sbound;
        const bool in_box = single < 0 ? valid : true;
        const float rr = in_box ? sqrtf(scut) * 1.0001f + (fabsf(sq.x) + fabsf(sq.y) + fabsf(sq.z)) * 1.0e-6f : 0.f;
        float ulx = in_box ? sq.x - rr : CUDART_INF_F_, uly = in_box ? sq.y - rr : CUDART_INF_F_,
              ulz = in_box ? sq.z - rr : CUDART_INF_F_;
        float uhx = in_box ? sq.x + rr : -CUDART_INF_F_, uhy = in_box ? sq.y + rr : -CUDART_INF_F_,
              uhz = in_box ? sq.z + rr : -CUDART_INF_F_;
        if (single < 0) {
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                ulx = fminf(ulx, __shfl_xor_sync(0xffffffffu, ulx, off));
                uly = fminf(uly, __shfl_xor_sync(0xffffffffu, uly, off));
                ulz = fminf(ulz, __shfl_xor_sync(0xffffffffu, ulz, off));
                uhx = fmaxf(uhx, __shfl_xor_sync(0xffffffffu, uhx, off));
                uhy = fmaxf(uhy, __shfl_xor_sync(0xffffffffu, uhy, off));
                uhz = fmaxf(uhz, __shfl_xor_sync(0xffffffffu, uhz, off));
            }
        }
        auto overlaps = [&](const float4 &l, const float4 &h) {
            return l.x <= uhx && h.x >= ulx && l.y <= uhy && h.y >= uly && l.z <= uhz && h.z >= ulz;
        };
        if (levels == 0) {
            out[0] = 0;
            return 1;
        }
        int fr[kRangeFrontier / 32];
        fr[0] = 0;
        int nf = 1, nl = 0;
        for (int d = 0; d < levels; ++d) {
            const bool to_leaves = (d + 1 == levels);
            int nnext = 0;
#pragma unroll
            for (int r = 0; r < kRangeFrontier / 32; ++r) {
                if (r * 32 >= nf) break;
                const bool has = r * 32 + lane < nf;
                const int node = has ? fr[r] : 0;
                const int c0 = 2 * node + 1, c1 = c0 + 1;
                float4 l0 = make_float4(0.f, 0.f, 0.f, 0.f), h0 = l0, l1 = l0, h1 = l0;
                if (has) {
                    l0 = a.lo[c0];
                    h0 = a.hi[c0];
                    l1 = a.lo[c1];
                    h1 = a.hi[c1];
                }
                st_nodes += has ? 2 : 0;
                bool p0 = has && overlaps(l0, h0);
                bool p1 = has && overlaps(l1, h1);
                // leaves: exact against a single owner's ball; the union list keeps every leaf the
                // union box reaches, since each owner tests the listed leaves against its own ball
                if (to_leaves && single >= 0) {
                    p0 = p0 && box_dist2(sq, l0, h0) <= scut;
                    p1 = p1 && box_dist2(sq, l1, h1) <= scut;
                }
                const unsigned int b0 = __ballot_sync(0xffffffffu, p0), b1 = __ballot_sync(0xffffffffu, p1);
                const int tot = __popc(b0) + __popc(b1);
                int kk = __popc(b0 & lt) + __popc(b1 & lt);
                if (to_leaves) {
                    if (nl + tot > cap) return -1;
                    kk += nl;
                    if (p0) out[kk++] = c0 - first_leaf;
                    if (p1) out[kk] = c1 - first_leaf;
                    nl += tot;
                } else {
                    if (nnext + tot > kRangeFrontier) return -1;
                    kk += nnext;
                    if (p0) sh.frontier[kk++] = c0;
                    if (p1) sh.frontier[kk] = c1;
                    nnext += tot;
                }
            }
            __syncwarp();
            if (!to_leaves) {
#pragma unroll
                for (int r = 0; r < kRangeFrontier / 32; ++r)
                    if (r * 32 + lane < nnext) fr[r] = sh.frontier[r * 32 + lane];
                nf = nnext;
                __syncwarp();
                if (nf == 0) break;
            }
        }
        return nl;
    };
    // the bucket's union list, walked once for all 32 owners; when the bucket's sites lie far apart
    // (a jump of the Morton curve) the union outgrows the buffers and each owner walks alone
    const int union_leaves = walk(-1, 0.0f, sh.list, kRangeList);
    const bool list_ok = union_leaves >= 0;
    const int nleaf = list_ok ? union_leaves : 0;
    __syncwarp();

    // 2-3. owner by owner
    const unsigned int valid_mask = __ballot_sync(0xffffffffu, valid);
    unsigned int fb_mask = 0u;  // lanes left to the heap query
    for (unsigned int todo = valid_mask; todo; todo &= todo - 1) {
        const int o = __ffs(todo) - 1;
        const float oc = __shfl_sync(0xffffffffu, cut, o);
        const float oq2 = __shfl_sync(0xffffffffu, q2, o);
        const int oidx = __shfl_sync(0xffffffffu, idx, o);
        const float3 oq = make_float3(__shfl_sync(0xffffffffu, qp.x, o), __shfl_sync(0xffffffffu, qp.y, o),
                                      __shfl_sync(0xffffffffu, qp.z, o));
        int ngroup = 0;
        // The leaves (into own_leaves) and then the 8-site groups (into own_groups) the owner's ball
        // of squared radius `bound` reaches: from the bucket's union list when the first bound is
        // the one that list was walked with, else by a walk of the owner's own.  False when a list
        // outgrows its buffer.
        auto gather = [&](float bound, bool from_union) -> bool {
            int nown = 0;
            if (from_union) {
                for (int b = 0; b < nleaf; b += 32) {
                    const bool has = b + lane < nleaf;
                    const int lf = has ? sh.list[b + lane] : 0;
                    const bool pass = has && box_dist2(oq, a.lo[first_leaf + lf], a.hi[first_leaf + lf]) <= bound;
                    const unsigned int bal = __ballot_sync(0xffffffffu, pass);
                    if (nown + __popc(bal) > kOwnLeaves) return false;
                    if (pass) sh.own_leaves[nown + __popc(bal & lt)] = lf;
                    nown += __popc(bal);
                }
            } else {
                nown = walk(o, bound, sh.own_leaves, kOwnLeaves);
                if (nown < 0) return false;
            }
            __syncwarp();
            // eight leaves per pass, a lane per sub-box
            ngroup = 0;
            for (int b = 0; b < nown; b += 8) {
                const int li = b + (lane >> 2);
                const bool has = li < nown;
                const int g = has ? sh.own_leaves[li] * kSubs + (lane & 3) : 0;
                const bool pass = has && box_dist2(oq, a.sub_lo[g], a.sub_hi[g]) <= bound;
                const unsigned int bal = __ballot_sync(0xffffffffu, pass);
                if (ngroup + __popc(bal) > kOwnGroups) return false;
                if (pass) sh.own_groups[ngroup + __popc(bal & lt)] = g;
                ngroup += __popc(bal);
            }
            __syncwarp();
            return true;
        };
        // the groups' sites, four groups (32 sites) per pass: candidates with d^2 <= bound
        auto collect = [&](float bound) {
            int cnt = 0;
            // eight groups (two sites per lane, both loads in flight) per pass
            for (int b = 0; b < ngroup; b += 8) {
                const int g0 = b + (lane >> 3), g1 = g0 + 4;
                const float4 inf4 = make_float4(CUDART_INF_F_, CUDART_INF_F_, CUDART_INF_F_, 0.f);
                const float4 p0 = g0 < ngroup ? a.sorted[sh.own_groups[g0] * kSub + (lane & 7)] : inf4;
                const float4 p1 = g1 < ngroup ? a.sorted[sh.own_groups[g1] * kSub + (lane & 7)] : inf4;
                // padding sites of a partly filled leaf lie at +inf too
                const float d0 = dist2(oq, make_float3(p0.x, p0.y, p0.z));
                const float d1 = dist2(oq, make_float3(p1.x, p1.y, p1.z));
                const bool in0 = d0 <= bound, in1 = d1 <= bound;
                const unsigned int bal0 = __ballot_sync(0xffffffffu, in0), bal1 = __ballot_sync(0xffffffffu, in1);
                const int pos0 = cnt + __popc(bal0 & lt), pos1 = cnt + __popc(bal0) + __popc(bal1 & lt);
                if (in0 && pos0 < kRangeCap)
                    sh.cand[pos0] = (static_cast<unsigned long long>(__float_as_uint(d0)) << 32) |
                                    static_cast<unsigned int>(__float_as_int(p0.w));
                if (in1 && pos1 < kRangeCap)
                    sh.cand[pos1] = (static_cast<unsigned long long>(__float_as_uint(d1)) << 32) |
                                    static_cast<unsigned int>(__float_as_int(p1.w));
                cnt += __popc(bal0) + __popc(bal1);
            }
            __syncwarp();
            st_groups += ngroup;
            st_cand += cnt;
            return cnt;
        };
        // More candidates than the network holds: the K-th smallest d^2 among the first kRangeCap
        // collected is a bound that at least K sites meet, so the true K nearest lie inside it;
        // rescan with it (six rounds at most).
        auto shrink = [&](int cnt) {
            for (int round = 0; round < 6 && cnt > kRangeCap; ++round) {
                unsigned long long v[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) v[j] = sh.cand[j * 32 + lane];
                __syncwarp();
                warp_bitonic<4>(v, lane);
                const int e = K - 1;
                unsigned long long sel = v[0];
#pragma unroll
                for (int j = 1; j < 4; ++j)
                    if (j == (e >> 5)) sel = v[j];
                const float bound =
                    __uint_as_float(static_cast<unsigned int>(__shfl_sync(0xffffffffu, sel, e & 31) >> 32));
                cnt = collect(bound);
            }
            return cnt;
        };
        float bound = oc;
        bool ok = gather(bound, list_ok);
        int count = ok ? shrink(collect(bound)) : 0;
        if (ok && count < K && bound < oq2) {
            // fewer than K inside a proposal below q: a short proposal, or an owner whose row is not
            // full even at q (a sparse region).  Search the whole q ball, which the range query can
            // hold when the region is sparse.
            bound = oq2;
            ok = gather(bound, false);
            count = ok ? shrink(collect(bound)) : 0;
        }
        if (!ok || count > kRangeCap) {
            fb_mask |= 1u << o;  // warp-uniform: the heap query takes this owner
            __syncwarp();
            continue;
        }
        __syncwarp();
        int32_t *row = a.codes ? a.codes + static_cast<size_t>(oidx) * K : nullptr;
        float kth;
        // up to kTrim candidates above 64: drop the largest one at a time, then a 64-key network
        int len = count;
        if (len > 64 && len <= 64 + kTrim) {
            for (; len > 64; --len) {
                unsigned long long best = 0;
                int where = -1;
                for (int e = lane; e < len; e += 32) {
                    const unsigned long long v = sh.cand[e];
                    if (where < 0 || v > best) {
                        best = v;
                        where = e;
                    }
                }
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    const unsigned long long ov = __shfl_xor_sync(0xffffffffu, best, off);
                    const int ow = __shfl_xor_sync(0xffffffffu, where, off);
                    if (ow >= 0 && (where < 0 || ov > best)) {
                        best = ov;
                        where = ow;
                    }
                }
                __syncwarp();
                if (lane == 0 && where != len - 1) sh.cand[where] = sh.cand[len - 1];
                __syncwarp();
            }
        }
        if (len <= 64) {
            unsigned long long v[2];
#pragma unroll
            for (int j = 0; j < 2; ++j) v[j] = (j * 32 + lane < len) ? sh.cand[j * 32 + lane] : ~0ull;
            warp_bitonic<2>(v, lane);
            kth = write_row<2>(v, lane, len, K, row);
        } else {
            unsigned long long v[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = (j * 32 + lane < len) ? sh.cand[j * 32 + lane] : ~0ull;
            warp_bitonic<4>(v, lane);
            kth = write_row<4>(v, lane, len, K, row);
        }
        if (lane == 0) sh.kth[o] = kth;
        __syncwarp();
    }
    __syncwarp();

    // 4. per-lane outputs of the owners served here
    const bool served = valid && !((fb_mask >> lane) & 1u);
    if (served) {
        const float kd2 = sh.kth[lane];
        if (a.kth) a.kth[idx] = kd2;
        if (a.measure) {
            const double y = a.part[idx].position[1];
            const double z = a.part[idx].position[2];
            a.measure[idx] = ball_measure(m, y, z, sqrt(static_cast<double>(kd2)));
        }
    }
    if (fb_mask && lane == 0) {
        const int slot = atomicAdd(a.fb_count, 1);
        a.fb_leaf[slot] = leaf;
        a.fb_mask[slot] = fb_mask;
    }
    if (a.stats) {
        if (lane == 0) {
            atomicAdd(&a.stats[0], static_cast<unsigned long long>(st_groups));
            atomicAdd(&a.stats[1], static_cast<unsigned long long>(st_nodes));
            atomicAdd(&a.stats[2], static_cast<unsigned long long>(st_cand));
        }
        if ((fb_mask >> lane) & 1u) atomicAdd(&a.stats[3], 1ull);
    }
}

bool knn_range_eligible(const Model &m, int K) { return !m.wedge && K >= 1 && K <= 64; }

Status knn_range(Geometry &g, const Model &m, const gd_particle *dev_particle, int32_t *codes, double *measure,
                 float *kth_d2, cudaStream_t s, const float *radius, unsigned long long *stats, const Tuning &tune) {
    RangeArgs ra;
    ra.sorted = g.sorted.ptr;
    ra.lo = g.node_lo.ptr;
    ra.hi = g.node_hi.ptr;
    ra.sub_lo = g.sub_lo.ptr;
    ra.sub_hi = g.sub_hi.ptr;
    ra.qrad = g.q.ptr;
    ra.radius = radius;
    ra.counters = g.counters.ptr;
    ra.part = dev_particle;
    ra.leaf_slots = g.leaf_slots;
    ra.k = m.n_k;
    ra.codes = codes;
    ra.measure = measure;
    ra.kth = kth_d2;
    ra.stats = stats;
    ra.fb_count = g.fb_count.ptr;
    ra.fb_leaf = g.fb_leaf.ptr;
    ra.fb_mask = g.fb_mask.ptr;
    GD_TRY_CUDA(cudaMemsetAsync(g.fb_count.ptr, 0, sizeof(int), s));
    const int max_leaves = (g.n_sites + kLeaf - 1) / kLeaf;
    g.launches += 1;
    k_knn_range<<<(max_leaves + kRangeWarps - 1) / kRangeWarps, kRangeWarps * 32, 0, s>>>(m, ra);
    GD_TRY_CUDA(cudaGetLastError());
    // the owners left over: the per-lane heap query with the full q, over the listed buckets only
    GD_TRY(knn_fallback(g, m, dev_particle, codes, measure, kth_d2, s, stats, tune));
    return Status::ok();
}

}  // namespace gd
