// Geometry stage of the swarm collision path on sm_100a:
//   col_site_init (src/swarm/col_site_init.cu:17-119)  -> k_site_init
//   index build (kdtree::buildTree, builder.h:109-152 / morton_index::build,
//                morton_index.cuh:168-229)              -> Morton keys + LSD radix sort + bucket tree
//   col_cache_get (inc/swarm/_col_cache.cuh:15-159)      -> k_knn_query (exact top-K + measure)
//   colstate_flag (src/swarm/colstate_flag.cu:13-29)     -> k_state_screen
//   col_space_bin (src/swarm/col_space_bin.cu:11-35)     -> k_space_bin
//
// Design.  Sites are kept as 16-byte float4 records (x, y, z, code bits) so every site read is
// one 128-bit load.  Active sites are ordered along a 63-bit Morton curve by a hand-written
// 8-bit-digit LSD radix sort, cut into buckets of 32 consecutive sites, and covered by an
// implicit complete binary tree of axis-aligned boxes.  A query warp owns one bucket: each lane
// is one owner, the warp walks the tree once for all 32 owners, and every candidate bucket is
// staged once in shared memory and read by all 32 lanes, so one 512-byte tile load serves 1024
// distance tests.  Each lane keeps its exact top-K as a 4-ary max-heap of packed (d^2 bits, code) keys
// in shared memory, the same key the reference heap uses (kdtree/index_heap.cuh:59-69), so the
// kept set is the reference's set; a final in-place heap sort yields ascending (d^2, code), the
// order of the reference Morton search (morton_types.cuh:68-72).
#include <cfloat>
#include <climits>
#include <cmath>

#include "gd_internal.cuh"
#include "gd_geom_device.cuh"

namespace gd {

// ------------------------------------------------------------------------------------------------
// col_site_init (col_site_init.cu:17-55 / 78-118) fused with the Morton key generation
// (morton_keygen, morton_index.cuh:41-60).  One thread per particle; threads past the sites write
// the sort padding.  Site i is particle i; with a wedge, sites n + i and 2n + i are its images
// rotated by -width (image 1) and +width (image 2), active when the particle is.
// ------------------------------------------------------------------------------------------------
__global__ void k_site_init(Model m, int n, int n_sites, const gd_particle *__restrict__ part,
                            float4 *__restrict__ site, float *__restrict__ qrad,
                            unsigned char *__restrict__ active, unsigned long long *__restrict__ key,
                            unsigned int *__restrict__ val, int n_sort, int *__restrict__ counters) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_sort) return;
    if (i >= n) {
        if (i >= n_sites) {  // sort padding: sorts after every active site
            key[i] = ~0ull;
            val[i] = static_cast<unsigned int>(i);
        }
        return;
    }
    const double2 *rec = reinterpret_cast<const double2 *>(part + i);
    double2 a = rec[0], b = rec[1], c = rec[2], d = rec[3];  // 4 x 128-bit loads of the 64 B record
    double x = a.x, y = a.y, z = b.x;
    bool finite = isfinite(a.x) && isfinite(a.y) && isfinite(b.x) && isfinite(b.y) && isfinite(c.x) &&
                  isfinite(c.y) && isfinite(d.x) && isfinite(d.y);
    unsigned long long k = ~0ull;
    float4 s = make_float4(0.f, 0.f, 0.f, __int_as_float(3 * i));
    float qi = 0.f;
    bool act = false;
    if (!finite) {
        atomicMin(&counters[1], i);
    } else {
        act = site_active(m, y, z);
        double R = cyl_R(m, y, z);
        double Z = cyl_Z(m, y, z);
        float3 p = (m.n_x == 1 && m.n_z == 1)
                       ? make_float3(static_cast<float>(R), 0.0f, 0.0f)
                       : make_float3(static_cast<float>(R * cos(x)), static_cast<float>(R * sin(x)),
                                     static_cast<float>(Z));
        s.x = p.x;
        s.y = p.y;
        s.z = p.z;
        if (act) {
            qi = static_cast<float>(m.h_search * get_hg(m, R) * R);
            k = morton_key(m, p);
        }
    }
    site[i] = s;
    qrad[i] = qi;
    active[i] = act ? 1 : 0;
    key[i] = k;
    val[i] = static_cast<unsigned int>(i);
    if (m.wedge) {
        // both rotated images, rounded as each search's reference kernel rounds them (KD:
        // col_site_init.cu:58-76; Morton ghosts: morton_ghost.cuh:60-82).  Which product of each
        // coordinate the reference's compiled code fuses was measured against its records, so the
        // Morton forms are written out; the KD loop keeps the reference kernel's own expression.
        float sin_width, cos_width;
        sincosf(m.wedge_width, &sin_width, &cos_width);
        float3 img[2];
        if (!m.morton_images) {
            for (int image = 0; image < 2; image++) {
                float sin_angle = (image == 0) ? -sin_width : sin_width;
                img[image] = make_float3(cos_width * s.x - sin_angle * s.y, sin_angle * s.x + cos_width * s.y, s.z);
            }
        } else {
            // image 2 (+width): x' = cos x - sin y, y' = sin x + cos y
            img[1] = make_float3(__fmaf_rn(cos_width, s.x, -__fmul_rn(sin_width, s.y)),
                                 __fmaf_rn(sin_width, s.x, __fmul_rn(cos_width, s.y)), s.z);
            // image 1 (-width): x' = cos x + sin y, y' = -sin x + cos y
            img[0] = make_float3(__fmaf_rn(cos_width, s.x, __fmul_rn(sin_width, s.y)),
                                 __fmaf_rn(cos_width, s.y, -__fmul_rn(sin_width, s.x)), s.z);
        }
#pragma unroll
        for (int image = 0; image < 2; ++image) {
            const int t = (image + 1) * n + i;
            site[t] = make_float4(img[image].x, img[image].y, img[image].z, __int_as_float(3 * i + image + 1));
            key[t] = act ? morton_key(m, img[image]) : ~0ull;
            val[t] = static_cast<unsigned int>(t);
        }
        // the largest search radius, for the Morton search's one dedup decision
        // (swarm_runtime.cu:413-415); q >= 0, so its bits order as the values do
        if (act) atomicMax(&counters[2], __float_as_int(qi));
    }
    // count active sites with one atomic per warp
    unsigned int ballot = __ballot_sync(__activemask(), act);
    if ((threadIdx.x & 31) == (__ffs(__activemask()) - 1) && ballot)
        atomicAdd(&counters[0], __popc(ballot) * (m.wedge ? 3 : 1));
}

// Distance from a site to the radial plane a rotation of `offset` radians carries it across: the
// perpendicular distance R|sin(offset)| while that plane lies ahead of the site (cos >= 0), else the
// site's cylindrical radius (_get_morton_seam_dist, morton_ghost.cuh:28-35, the same float steps).
__device__ __forceinline__ float seam_distance(float x, float y, float offset) {
    const float R = hypotf(x, y);
    return (cosf(offset) >= 0.0f) ? R * fabsf(sinf(offset)) : R;
}

// The Morton search's ghost rule (morton_gcount / morton_gwrite, morton_ghost.cuh:38-88, called
// with the largest search radius, swarm_runtime.cu:413-421): a rotated image is indexed only when
// the seam it stands for lies within q_max of the physical site.  Image 2 (+width) stands for the
// x_min seam, image 1 (-width) for the x_max seam.  k_site_init wrote both images and q_max; this
// pass, run once the radius maximum is complete, drops the images the rule rejects: their keys
// become all ones (sorted past the indexed sites, like inactive ones) and their codes -1, and the
// indexed-site count loses them.  Images of inactive particles are marked too (the reference
// writes ghost records for every finite particle), but were never indexed.
__global__ void k_morton_ghosts(Model m, int n, const gd_particle *__restrict__ part,
                                const unsigned char *__restrict__ active, float4 *__restrict__ site,
                                unsigned long long *__restrict__ key, int *__restrict__ counters) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int dropped = 0;
    if (i < n) {
        const float q_max = __int_as_float(counters[2]);
        const float x_min = static_cast<float>(m.x_min), x_max = static_cast<float>(m.x_max);
        const float posx = static_cast<float>(part[i].position[0]);
        const float4 s = site[i];
        const bool keep[2] = {seam_distance(s.x, s.y, x_max - posx) <= q_max,   // image 1
                              seam_distance(s.x, s.y, posx - x_min) <= q_max};  // image 2
#pragma unroll
        for (int image = 0; image < 2; ++image) {
            if (keep[image]) continue;
            const int t = (image + 1) * n + i;
            site[t].w = __int_as_float(-1);
            key[t] = ~0ull;
            dropped += active[i] ? 1 : 0;
        }
    }
    // one atomic per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dropped += __shfl_xor_sync(0xffffffffu, dropped, o);
    if ((threadIdx.x & 31) == 0 && dropped) atomicSub(&counters[0], dropped);
}

// colstate_flag (colstate_flag.cu:13-29): non-finite screen when the geometry is reused.
__global__ void k_state_screen(int n, const gd_particle *__restrict__ part, int *__restrict__ counters) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double2 *rec = reinterpret_cast<const double2 *>(part + i);
    double2 a = rec[0], b = rec[1], c = rec[2], d = rec[3];
    bool finite = isfinite(a.x) && isfinite(a.y) && isfinite(b.x) && isfinite(b.y) && isfinite(c.x) &&
                  isfinite(c.y) && isfinite(d.x) && isfinite(d.y);
    if (!finite) atomicMin(&counters[1], i);
}

// ------------------------------------------------------------------------------------------------
// LSD radix sort of (u64 key, u32 value), 8-bit digits, stable.  Per digit: per-tile digit
// histogram, exclusive scan over [digit][tile] (chunk-local scans, then the chunk totals), stable
// scatter.
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kRadixThreads) k_radix_hist(const unsigned long long *__restrict__ key,
                                                              int shift, int tiles,
                                                              unsigned int *__restrict__ hist) {
    __shared__ unsigned int h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const unsigned long long *tk = key + static_cast<size_t>(blockIdx.x) * kRadixTile;
#pragma unroll
    for (int it = 0; it < kRadixItems; ++it) {
        unsigned int dg = static_cast<unsigned int>(tk[it * kRadixThreads + threadIdx.x] >> shift) & 255u;
        atomicAdd(&h[dg], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive scan of the 4096-entry chunk `chunk` of cnt[0..len) in place, 256 threads owning 16
// consecutive entries each; `carry` is added to every entry.  Returns the chunk total to all threads.
__device__ __forceinline__ unsigned int scan_chunk(unsigned int *__restrict__ cnt, int len, long long chunk,
                                                   unsigned int carry) {
    __shared__ unsigned int warp_tot[kRadixThreads / 32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const long long first = chunk * kScanChunk + static_cast<long long>(t) * kScanItems;
    unsigned int v[kScanItems];
    unsigned int sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = (first + i < len) ? cnt[first + i] : 0u;
        sum += v[i];
    }
    unsigned int x = sum;  // inclusive scan of the per-thread sums across the warp
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const unsigned int y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    unsigned int before = 0, total = 0;
#pragma unroll
    for (int j = 0; j < kRadixThreads / 32; ++j) {
        const unsigned int wt = warp_tot[j];
        before += (j < w) ? wt : 0u;
        total += wt;
    }
    unsigned int run = carry + before + x - sum;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (first + i < len) cnt[first + i] = run;
        run += v[i];
    }
    __syncthreads();  // warp_tot is reused by the next chunk
    return total;
}

// Chunk-local exclusive scans of cnt[0..len); chunk totals to part[] (null when one chunk covers
// cnt, which then holds the full exclusive scan).
__global__ void __launch_bounds__(kRadixThreads) k_scan_chunks(unsigned int *__restrict__ cnt, int len,
                                                               unsigned int *__restrict__ part) {
    const unsigned int total = scan_chunk(cnt, len, blockIdx.x, 0u);
    if (part && threadIdx.x == 0) part[blockIdx.x] = total;
}

// Exclusive scan of the chunk totals part[0..n) in place, one block, 4096 entries at a time.
__global__ void __launch_bounds__(kRadixThreads) k_scan_parts(unsigned int *__restrict__ part, int n) {
    unsigned int carry = 0;
    for (long long c = 0; c * kScanChunk < n; ++c) carry += scan_chunk(part, n, c, carry);
}

__global__ void __launch_bounds__(kRadixThreads)
    k_radix_scatter(const unsigned long long *__restrict__ kin, const unsigned int *__restrict__ vin,
                    unsigned long long *__restrict__ kout, unsigned int *__restrict__ vout, int shift,
                    int tiles, const unsigned int *__restrict__ offs, const unsigned int *__restrict__ part) {
    constexpr int kWarps = kRadixThreads / 32;
    __shared__ unsigned int wcnt[kWarps][256];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j = threadIdx.x; j < kWarps * 256; j += kRadixThreads) (&wcnt[0][0])[j] = 0;
    __syncthreads();
    // warp w ranks tile elements [w*512, w*512+512) in 16 rounds of 32: element order inside the
    // tile is (warp, round, lane), so the ranks are stable.
    size_t base = static_cast<size_t>(blockIdx.x) * kRadixTile + warp * (kRadixItems * 32);
    unsigned long long k[kRadixItems];
    unsigned int rank[kRadixItems];
    unsigned int lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < kRadixItems; ++r) {
        k[r] = kin[base + r * 32 + lane];
        unsigned int dg = static_cast<unsigned int>(k[r] >> shift) & 255u;
        unsigned int peers = __match_any_sync(0xffffffffu, dg);
        unsigned int before = wcnt[warp][dg];
        __syncwarp();
        rank[r] = before + __popc(peers & lt);
        if ((peers & lt) == 0) wcnt[warp][dg] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // exclusive prefix over warps for every digit, plus the tile's global digit offset (the
    // chunk-local scan of [digit][tile] plus its chunk's offset)
    {
        int dg = threadIdx.x;  // kRadixThreads == 256
        const int at = dg * tiles + blockIdx.x;
        unsigned int run = offs[at] + (part ? part[at / kScanChunk] : 0u);
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            unsigned int c = wcnt[w][dg];
            wcnt[w][dg] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kRadixItems; ++r) {
        unsigned int dg = static_cast<unsigned int>(k[r] >> shift) & 255u;
        unsigned int dst = wcnt[warp][dg] + rank[r];
        kout[dst] = k[r];
        vout[dst] = vin[base + r * 32 + lane];
    }
}

// ------------------------------------------------------------------------------------------------
// Bucket tree: gather Morton-ordered sites, leaf boxes, then internal boxes level by level.
// ------------------------------------------------------------------------------------------------
__global__ void k_gather_sorted(int n_slots, const int *__restrict__ counters, const unsigned int *__restrict__ val,
                                const float4 *__restrict__ site, float4 *__restrict__ sorted) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_slots) return;
    int n_act = counters[0];
    int n_pad = (n_act + kLeaf - 1) / kLeaf * kLeaf;
    if (i >= n_pad) return;
    float4 s;
    if (i < n_act) {
        s = site[val[i]];
    } else {
        s = make_float4(CUDART_INF_F_, CUDART_INF_F_, CUDART_INF_F_, __int_as_float(-1));
    }
    sorted[i] = s;
}

// one warp per leaf slot: four 8-site sub-boxes (8-lane reductions) and their union
__global__ void k_leaf_bounds(int leaf_slots, const int *__restrict__ counters, const float4 *__restrict__ sorted,
                              float4 *__restrict__ lo, float4 *__restrict__ hi, float4 *__restrict__ sub_lo,
                              float4 *__restrict__ sub_hi) {
    int leaf = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (leaf >= leaf_slots) return;
    int n_act = counters[0];
    int i = leaf * kLeaf + lane;
    float3 a = make_float3(CUDART_INF_F_, CUDART_INF_F_, CUDART_INF_F_);
    float3 b = make_float3(-CUDART_INF_F_, -CUDART_INF_F_, -CUDART_INF_F_);
    if (i < n_act) {
        float4 s = sorted[i];
        a = make_float3(s.x, s.y, s.z);
        b = a;
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        if (off == kSub) {
            // lanes 0, 8, 16, 24 now hold their sub-box
            if ((lane & (kSub - 1)) == 0) {
                sub_lo[leaf * kSubs + lane / kSub] = make_float4(a.x, a.y, a.z, 0.f);
                sub_hi[leaf * kSubs + lane / kSub] = make_float4(b.x, b.y, b.z, 0.f);
            }
        }
        a.x = fminf(a.x, __shfl_xor_sync(0xffffffffu, a.x, off));
        a.y = fminf(a.y, __shfl_xor_sync(0xffffffffu, a.y, off));
        a.z = fminf(a.z, __shfl_xor_sync(0xffffffffu, a.z, off));
        b.x = fmaxf(b.x, __shfl_xor_sync(0xffffffffu, b.x, off));
        b.y = fmaxf(b.y, __shfl_xor_sync(0xffffffffu, b.y, off));
        b.z = fmaxf(b.z, __shfl_xor_sync(0xffffffffu, b.z, off));
    }
    if (lane == 0) {
        int node = leaf_slots - 1 + leaf;
        lo[node] = make_float4(a.x, a.y, a.z, 0.f);
        hi[node] = make_float4(b.x, b.y, b.z, 0.f);
    }
}

// internal nodes [first, first+count) from their two children
__global__ void k_tree_level(int first, int count, float4 *__restrict__ lo, float4 *__restrict__ hi) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    int node = first + t;
    float4 l0 = lo[2 * node + 1], l1 = lo[2 * node + 2];
    float4 h0 = hi[2 * node + 1], h1 = hi[2 * node + 2];
    lo[node] = make_float4(fminf(l0.x, l1.x), fminf(l0.y, l1.y), fminf(l0.z, l1.z), 0.f);
    hi[node] = make_float4(fmaxf(h0.x, h1.x), fmaxf(h0.y, h1.y), fmaxf(h0.z, h1.z), 0.f);
}

// ------------------------------------------------------------------------------------------------
// Exact top-K query.  One warp per bucket of 32 Morton-ordered active owners.
// ------------------------------------------------------------------------------------------------
struct QueryArgs {
    const float4 *sorted;
    const float4 *lo;
    const float4 *hi;
    const float4 *sub_lo;   // 8-site sub-boxes of every leaf
    const float4 *sub_hi;
    const float *qrad;      // by particle index
    const int *counters;
    const gd_particle *part;
    int leaf_slots;
    int k;
    int32_t *codes;         // may be null
    double *measure;        // may be null
    float *kth;             // may be null
    const float *radius;    // proposed search radius by particle index, or null for the plain query
    int prescan;            // Morton-neighbour buckets scanned on each side before the walk
    int bfs;                // breadth-first (1) or depth-first (0) walk
    unsigned long long *stats;  // optional counters: leaves scanned, nodes tested, offers, fallbacks
};

// Per-lane 4-ary max-heaps of 64-bit keys (d^2 bits << 32 | code).  Lane-major: lane l's n
// entries start at entry l * heap_stride(K).  The root (slot 0) has children 1..3, every other slot
// i has children 4i..4i+3, so a node's children form one 32-byte aligned group that two 16-byte
// loads fetch.  A depth-3 heap holds 64 entries.  heap_stride keeps the stride an odd number of 16-byte
// chunks, so eight lanes reading the same slot group hit eight different bank groups.
__host__ __device__ constexpr int heap_stride(int K) { return ((K + 3) & ~3) + 2; }

// Sifts `key` down from slot i of a heap of n entries.
__device__ __forceinline__ void heap_sift(unsigned long long *hp, unsigned long long key, int i, int n) {
    while (true) {
        const int c0 = i ? 4 * i : 1;  // first child
        if (c0 >= n) break;
        const int gb = c0 & ~3;        // the group holding the children (the root's holds the root too)
        const ulonglong2 lo = *reinterpret_cast<const ulonglong2 *>(hp + gb);
        const ulonglong2 hi = *reinterpret_cast<const ulonglong2 *>(hp + gb + 2);
        const unsigned long long v[4] = {lo.x, lo.y, hi.x, hi.y};
        unsigned long long bv = 0;
        int bj = -1;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int sl = gb + j;
            if (sl >= c0 && sl < n && (bj < 0 || v[j] > bv)) {
                bv = v[j];
                bj = sl;
            }
        }
        if (bv < key) break;
        hp[i] = bv;
        i = bj;
    }
    hp[i] = key;
}

// Floyd heap construction over the first n entries of one lane's heap
__device__ __forceinline__ void heap_build(unsigned long long *hp, int n) {
    for (int i = (n - 1) / 4; i >= 0 && n > 1; --i) heap_sift(hp, hp[i], i, n);
}

__device__ __forceinline__ float key_d2(unsigned long long k) { return __uint_as_float(static_cast<unsigned int>(k >> 32)); }

// Per-warp shared memory of k_knn_query: the heaps of 32 lanes (heap_stride(K) entries each), a
// 32-site tile (also the breadth-first frontier staging, kFrontier ints), and the leaf list /
// depth-first stack.
constexpr int kFrontier = 128;   // internal nodes of one breadth-first level
constexpr int kListInts = 352;   // leaves of the breadth-first walk (also the depth-first stack)
__host__ __device__ constexpr size_t knn_heap_bytes(int K) { return static_cast<size_t>(heap_stride(K)) * 32 * 8; }
__host__ __device__ constexpr size_t knn_warp_bytes(int K) { return knn_heap_bytes(K) + 32 * 16 + kListInts * 4; }
// Entries a lane may hold.  Inside a well-proposed radius a lane finds a little more than K sites
// (about 1.2 K at c3); a radius-bounded lane gets 3K/8 extra slots (rounded up to 8), appends them
// all and selects the K nearest once at the end, instead of building its heap mid-walk (in as many
// batches as the warp has fill times) and sifting every later candidate.  At K = 64: 88 slots;
// 72, 80 and 96 were slower (fewer spare slots build more heaps, more cost residency).
__host__ __device__ constexpr int knn_capacity(int K, bool bounded) {
    return bounded ? K + (((3 * K) / 8 + 7) & ~7) : K;
}

// Loads of one leaf: this lane's site of the 32-site tile and the four 8-site sub-boxes.
struct LeafLoad {
    float4 site;
    float4 sl[kSubs], sh[kSubs];
};

// The slot of this lane's entry for the same particle as code `code` among its first `len` entries,
// or -1: the duplicate-image scan of idx_old_heap::processCandidate (kdtree/index_heap.cuh:118-131).
__device__ __forceinline__ int same_particle(const unsigned long long *hp, int len, int code) {
    const int base = code - code % 3;  // 3 * particle
    for (int j = 0; j < len; ++j)
        if (static_cast<unsigned int>(static_cast<int>(static_cast<unsigned int>(hp[j])) - base) < 3u) return j;
    return -1;
}

// The exact top-K of the 32 owners of bucket (leaf) `leaf` of one swarm, by one warp.  `wbase` is
// the warp's shared memory laid out for up to kcap neighbours (knn_warp_bytes(kcap)).  kImages: the
// sites include wedge images, so only image-0 lanes are owners, and an owner whose search ball can
// reach two images of one particle keeps only the nearer (the dedup of index_heap.cuh:118-136).
template <bool kImages>
__device__ __forceinline__ void knn_bucket(const Model &m, const QueryArgs &a, int leaf, unsigned char *wbase,
                                           int kcap, unsigned int lanes = 0xffffffffu) {
    const int lane = threadIdx.x & 31;
    const int K = a.k;
    const int cap = knn_capacity(K, a.radius != nullptr);  // entries a lane may hold (<= kcap)
    unsigned long long *hp = reinterpret_cast<unsigned long long *>(wbase) + lane * heap_stride(cap);
    float4 *tile = reinterpret_cast<float4 *>(wbase + knn_heap_bytes(kcap));
    // the breadth-first walk stages its next frontier in the tile buffer (no leaf is scanned then)
    int *staging = reinterpret_cast<int *>(tile);
    // leaf list of the breadth-first walk; the depth-first walk's stack (never live together)
    int *stack = reinterpret_cast<int *>(wbase + knn_heap_bytes(kcap) + 32 * 16);
    int *leaf_list = stack;

    const int n_act = a.counters[0];
    const int n_leaves = (n_act + kLeaf - 1) / kLeaf;
    if (leaf >= n_leaves) return;

    const int i = leaf * kLeaf + lane;
    const float4 me = a.sorted[i];
    const float3 qp = make_float3(me.x, me.y, me.z);
    const int code = __float_as_int(me.w);
    // with wedge images only the physical sites (image 0) query (_col_cache.cuh:22)
    const bool valid = i < n_act && (!kImages || code % 3 == 0) && ((lanes >> lane) & 1u);
    const int idx = valid ? code / 3 : 0;
    const float qr = valid ? a.qrad[idx] : 0.f;
    // dedup_needed = !unique_ids (_col_cache.cuh:38-39 per owner for KD; the largest q for Morton,
    // swarm_runtime.cu:413-415)
    bool dd = false;
    if (kImages && valid) {
        const float qd = m.morton_images ? __int_as_float(a.counters[2]) : qr;
        dd = !(m.image_dist_min < 0.0f || m.image_dist_min > 2.0f * qd);
    }
    // Reference acceptance: key < (q^2 bits, 0xffffffff), i.e. d^2 <= q^2 with the float q^2 the
    // reference heap is seeded with (kdtree/index_heap.cuh:58-61, morton_index.cuh:276).
    const float q2 = qr * qr;
    // Radius-bounded pass: accept d^2 <= lim2 = min(q, r)^2.  Finding K sites there proves they are
    // the K nearest overall; otherwise the lane repeats the walk with lim2 = q^2.
    float lim2 = q2;
    if (a.radius && valid) {
        const float r = a.radius[idx];
        if (r >= 0.0f && r < qr) lim2 = r * r;  // a negative or NaN proposal bounds nothing
    }
    int cnt = 0;                              // real entries held by this lane (fill phase below K)
    float cut = valid ? lim2 : -1.0f;         // d^2 bound of an acceptable candidate
    long long st_leaves = 0, st_nodes = 0, st_offers = 0;

    const int depth_leaves = a.leaf_slots;  // leaves under the root (a power of two)

    bool built = false;  // this lane's cap entries have been arranged into a max-heap

    auto load_leaf = [&](int lf, LeafLoad &L) {
        L.site = a.sorted[lf * kLeaf + lane];
#pragma unroll
        for (int gq = 0; gq < kSubs; ++gq) {
            L.sl[gq] = a.sub_lo[lf * kSubs + gq];
            L.sh[gq] = a.sub_hi[lf * kSubs + gq];
        }
    };

    auto process_leaf = [&](int lf, const LeafLoad &L) {
        const int base = lf * kLeaf;
        // which 8-site groups of this leaf can hold a candidate for some lane
        unsigned int groups = 0;
#pragma unroll
        for (int gq = 0; gq < kSubs; ++gq)
            if (__any_sync(0xffffffffu, box_dist2(qp, L.sl[gq], L.sh[gq]) <= cut)) groups |= 1u << gq;
        if (!groups) return;
        tile[lane] = L.site;
        __syncwarp();
        const int ncand = min(kLeaf, n_act - base);
        // the distances of every needed group first (independent work), then this lane's accepted
        // candidates only
        unsigned int mask = 0;
#pragma unroll
        for (int gq = 0; gq < kSubs; ++gq) {
            if (!(groups & (1u << gq))) continue;
#pragma unroll
            for (int c8 = 0; c8 < kSub; ++c8) {
                const int c = gq * kSub + c8;
                const float4 p = tile[c];
                const float d2 = dist2(qp, make_float3(p.x, p.y, p.z));
                mask |= ((c < ncand) && (d2 <= cut)) ? (1u << c) : 0u;
            }
            st_leaves += 1;
        }
        // Fill phase: a lane with fewer than cap entries appends without ordering work.  A lane
        // that reaches cap stops and keeps the rest of its mask; the lanes that filled up in this
        // leaf then build their heaps together (in step, instead of one lane after another).
        if constexpr (kImages) {
            // one candidate per pass; a second image of a held particle replaces it when nearer
            while (mask && cnt < cap) {
                const int c = __ffs(mask) - 1;
                mask &= mask - 1;
                const float4 p = tile[c];
                const float d2 = dist2(qp, make_float3(p.x, p.y, p.z));
                if (d2 <= cut) {
                    ++st_offers;
                    const int cc = __float_as_int(p.w);
                    const unsigned long long key =
                        (static_cast<unsigned long long>(__float_as_uint(d2)) << 32) | static_cast<unsigned int>(cc);
                    const int slot = dd ? same_particle(hp, cnt, cc) : -1;
                    if (slot < 0) hp[cnt++] = key;
                    else if (key < hp[slot]) hp[slot] = key;
                }
            }
        }
        // two candidates per pass: half the divergent trips, two independent distance chains
        while (!kImages && mask && cnt < cap) {
            const int c0 = __ffs(mask) - 1;
            mask &= mask - 1;
            const bool two = mask && cnt + 1 < cap;
            const int c1 = two ? __ffs(mask) - 1 : c0;
            if (two) mask &= mask - 1;
            const float4 p0 = tile[c0], p1 = tile[c1];
            const float d0 = dist2(qp, make_float3(p0.x, p0.y, p0.z));
            const float d1 = dist2(qp, make_float3(p1.x, p1.y, p1.z));
            if (d0 <= cut) {
                ++st_offers;
                hp[cnt] = (static_cast<unsigned long long>(__float_as_uint(d0)) << 32) |
                          static_cast<unsigned int>(__float_as_int(p0.w));
                ++cnt;
            }
            if (two && d1 <= cut) {
                ++st_offers;
                hp[cnt] = (static_cast<unsigned long long>(__float_as_uint(d1)) << 32) |
                          static_cast<unsigned int>(__float_as_int(p1.w));
                ++cnt;
            }
        }
        const bool build_now = cnt == cap && !built;
        if (__any_sync(0xffffffffu, build_now)) {
            if (build_now) {
                heap_build(hp, cap);
                cut = key_d2(hp[0]);
                built = true;
            }
        }
        // heap phase: a candidate below the heap's largest key replaces it (with images: a nearer
        // image of a held particle replaces that particle's entry instead, index_heap.cuh:133-141)
        while (mask) {
            const int c = __ffs(mask) - 1;
            mask &= mask - 1;
            const float4 p = tile[c];
            const float d2 = dist2(qp, make_float3(p.x, p.y, p.z));
            if (d2 <= cut) {
                ++st_offers;
                const unsigned long long key = (static_cast<unsigned long long>(__float_as_uint(d2)) << 32) |
                                               static_cast<unsigned int>(__float_as_int(p.w));
                const int slot = (kImages && dd) ? same_particle(hp, cap, __float_as_int(p.w)) : -1;
                if (slot >= 0) {
                    if (key < hp[slot]) {
                        heap_sift(hp, key, slot, cap);
                        cut = key_d2(hp[0]);
                    }
                } else if (key < hp[0]) {
                    heap_sift(hp, key, 0, cap);
                    cut = key_d2(hp[0]);
                }
            }
        }
        __syncwarp();
    };

    auto scan_leaf = [&](int lf) {
        LeafLoad L;
        load_leaf(lf, L);
        process_leaf(lf, L);
    };

    // Scans leaves id(0..count-1) (warp-uniform ids, -1 = skip), loading the next leaf while the
    // current one is processed.
    auto scan_sequence = [&](auto id, int count) {
        LeafLoad cur, nxt;
        int i = 0, lf = -1;
        while (i < count && (lf = id(i)) < 0) ++i;
        if (lf < 0) return;
        load_leaf(lf, cur);
        while (true) {
            int j = i + 1, nf = -1;
            while (j < count && (nf = id(j)) < 0) ++j;
            if (nf >= 0) load_leaf(nf, nxt);
            process_leaf(lf, cur);
            if (nf < 0) break;
            cur = nxt;
            lf = nf;
            i = j;
        }
    };

    // own bucket and its Morton neighbours: they hold near sites, so the heaps fill and the bounds
    // tighten before the tree walk
    auto prescan = [&]() {
        scan_sequence(
            [&](int t) {
                const int lf = (t == 0) ? leaf : ((t & 1) ? leaf - (t + 1) / 2 : leaf + t / 2);
                return (lf >= 0 && lf < n_leaves) ? lf : -1;
            },
            2 * a.prescan + 1);
    };
    auto prescanned = [&](int lf) { return lf >= leaf - a.prescan && lf <= leaf + a.prescan; };

    // Depth-first walk.  A node's box is tested when its parent is expanded: both children's
    // boxes are loaded together and only children that can hold a candidate for some lane are
    // pushed, so a pop needs no load.  The stack holds at most one pending sibling per tree level
    // plus the node being expanded.
    auto walk_dfs = [&]() {
        int sp = 0;
        {
            const float4 rl = a.lo[0], rh = a.hi[0];
            st_nodes += 1;
            if (__any_sync(0xffffffffu, box_dist2(qp, rl, rh) <= cut)) stack[sp++] = 0;
        }
        while (sp > 0) {
            const int node = stack[--sp];
            if (node >= a.leaf_slots - 1) {
                const int lf = node - (a.leaf_slots - 1);
                if (!prescanned(lf)) scan_leaf(lf);
                continue;
            }
            const int c0 = 2 * node + 1, c1 = 2 * node + 2;
            const float4 l0 = a.lo[c0], h0 = a.hi[c0], l1 = a.lo[c1], h1 = a.hi[c1];
            st_nodes += 2;
            const bool p0 = __any_sync(0xffffffffu, box_dist2(qp, l0, h0) <= cut);
            const bool p1 = __any_sync(0xffffffffu, box_dist2(qp, l1, h1) <= cut);
            // Visit first the child whose leaf range lies closer, in Morton order, to the warp's
            // own bucket: its sites are the nearer ones.
            const int depth = 31 - __clz(node + 1);
            const int span = depth_leaves >> depth;  // leaves under this node
            const int start = (node + 1 - (1 << depth)) * span;
            const bool left_near = leaf < start + (span >> 1);
            const int near = left_near ? c0 : c1, far = left_near ? c1 : c0;
            const bool pn = left_near ? p0 : p1, pf = left_near ? p1 : p0;
            if (pf) stack[sp++] = far;
            if (pn) stack[sp++] = near;
            __syncwarp();
        }
    };

    // Breadth-first walk for the lanes in `part`: one level of the tree per memory round trip, up
    // to 32 nodes tested at once (one per lane).  Internal nodes are pruned against the
    // axis-aligned box around every participating lane's ball; leaves against each lane's own ball
    // (d^2 bound `cut`).  The passing leaves are then scanned in one pipelined sequence.  Returns
    // false (nothing scanned) when a level or the leaf list exceeds its capacity.
    auto walk_bfs = [&](bool part) -> bool {
        const int levels = 31 - __clz(a.leaf_slots);  // leaves sit at this depth
        if (levels == 0) return true;                 // a single leaf: the prescan covered it
        // conservative union box: radius inflated by 1e-4 and by the rounding of q +- r
        const float rr = part ? sqrtf(cut) * 1.0001f + (fabsf(qp.x) + fabsf(qp.y) + fabsf(qp.z)) * 1.0e-6f : 0.f;
        float ulx = part ? qp.x - rr : CUDART_INF_F_, uly = part ? qp.y - rr : CUDART_INF_F_,
              ulz = part ? qp.z - rr : CUDART_INF_F_;
        float uhx = part ? qp.x + rr : -CUDART_INF_F_, uhy = part ? qp.y + rr : -CUDART_INF_F_,
              uhz = part ? qp.z + rr : -CUDART_INF_F_;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            ulx = fminf(ulx, __shfl_xor_sync(0xffffffffu, ulx, off));
            uly = fminf(uly, __shfl_xor_sync(0xffffffffu, uly, off));
            ulz = fminf(ulz, __shfl_xor_sync(0xffffffffu, ulz, off));
            uhx = fmaxf(uhx, __shfl_xor_sync(0xffffffffu, uhx, off));
            uhy = fmaxf(uhy, __shfl_xor_sync(0xffffffffu, uhy, off));
            uhz = fmaxf(uhz, __shfl_xor_sync(0xffffffffu, uhz, off));
        }
        auto overlaps = [&](const float4 &l, const float4 &h) {
            return l.x <= uhx && h.x >= ulx && l.y <= uhy && h.y >= uly && l.z <= uhz && h.z >= ulz;
        };
        // a lane outside `part` tests against an empty ball
        const float pcut = part ? cut : -1.0f;
        const unsigned int lt = (1u << lane) - 1u;
        const int first_leaf = a.leaf_slots - 1;
        int fr[kFrontier / 32];
        fr[0] = 0;  // the root, held by lane 0
        int nf = 1, nleaf = 0;
        for (int d = 0; d < levels; ++d) {
            const bool to_leaves = (d + 1 == levels);
            int nnext = 0;
#pragma unroll
            for (int r = 0; r < kFrontier / 32; ++r) {
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
                if (to_leaves) {
                    p0 = p0 && !prescanned(c0 - first_leaf);
                    p1 = p1 && !prescanned(c1 - first_leaf);
                    if (__any_sync(0xffffffffu, p0 || p1)) {
                        // exact: some participating lane's own ball reaches the leaf box
                        bool e0 = false, e1 = false;
                        for (int o = 0; o < 32; ++o) {
                            const float ox = __shfl_sync(0xffffffffu, qp.x, o);
                            const float oy = __shfl_sync(0xffffffffu, qp.y, o);
                            const float oz = __shfl_sync(0xffffffffu, qp.z, o);
                            const float oc = __shfl_sync(0xffffffffu, pcut, o);
                            const float3 oq = make_float3(ox, oy, oz);
                            e0 = e0 || (p0 && box_dist2(oq, l0, h0) <= oc);
                            e1 = e1 || (p1 && box_dist2(oq, l1, h1) <= oc);
                        }
                        p0 = e0;
                        p1 = e1;
                    }
                }
                const unsigned int b0 = __ballot_sync(0xffffffffu, p0), b1 = __ballot_sync(0xffffffffu, p1);
                const int tot = __popc(b0) + __popc(b1);
                int k = __popc(b0 & lt) + __popc(b1 & lt);
                if (to_leaves) {
                    if (nleaf + tot > kListInts) return false;
                    k += nleaf;
                    if (p0) leaf_list[k++] = c0 - first_leaf;
                    if (p1) leaf_list[k] = c1 - first_leaf;
                    nleaf += tot;
                } else {
                    if (nnext + tot > kFrontier) return false;
                    k += nnext;
                    if (p0) staging[k++] = c0;
                    if (p1) staging[k] = c1;
                    nnext += tot;
                }
            }
            __syncwarp();
            if (!to_leaves) {
#pragma unroll
                for (int r = 0; r < kFrontier / 32; ++r)
                    if (r * 32 + lane < nnext) fr[r] = staging[r * 32 + lane];
                nf = nnext;
                __syncwarp();
                if (nf == 0) break;
            }
        }
        // the listed leaves, by this walk's lanes only (the others see them in their own walk)
        const float keep = cut;
        if (!part) cut = -1.0f;
        scan_sequence([&](int t) { return leaf_list[t]; }, nleaf);
        if (!part) cut = keep;
        __syncwarp();
        return true;
    };

    auto walk = [&]() {
        prescan();
        if (!a.bfs) {
            walk_dfs();
            return;
        }
        // lanes whose heap is not yet full still search the whole q ball: they walk depth-first
        // after the others, so that their ball does not widen the breadth-first union box
        const bool deferred = valid && cut >= 0.0f && cnt < K && !(lim2 < q2);
        const bool part = valid && cut >= 0.0f && !deferred;
        const bool bfs_ok = __any_sync(0xffffffffu, part) ? walk_bfs(part) : true;
        if (!bfs_ok) {
            walk_dfs();  // nothing was scanned past the prescan: every lane walks depth-first
            return;
        }
        if (__any_sync(0xffffffffu, deferred)) {
            const float keep = cut;
            if (!deferred) cut = -1.0f;
            walk_dfs();
            if (!deferred) cut = keep;
        }
    };

    walk();
    bool fell_back = false;
    if (a.radius) {
        // lanes that found fewer than K sites inside a radius shorter than q repeat the walk with q
        const bool need_fb = valid && lim2 < q2 && cnt < K;
        if (__any_sync(0xffffffffu, need_fb)) {
            if (need_fb) {
                lim2 = q2;
                cnt = 0;
                cut = q2;
                fell_back = true;
            } else {
                cut = -1.0f;  // this lane's heap is final: keep it out of the second walk
            }
            walk();
        }
    }

    // the K nearest of the held entries, ascending (d^2 bits, code): drop the largest beyond K,
    // then heap sort
    if (!built) heap_build(hp, cnt);
    for (; cnt > K; --cnt) heap_sift(hp, hp[cnt - 1], 0, cnt - 1);
    for (int end = cnt - 1; end > 0; --end) {
        const unsigned long long top = hp[0];
        const unsigned long long last = hp[end];
        hp[end] = top;
        heap_sift(hp, last, 0, end);
    }
    if (a.stats && lane == 0) {
        atomicAdd(&a.stats[0], static_cast<unsigned long long>(st_leaves));
        atomicAdd(&a.stats[1], static_cast<unsigned long long>(st_nodes));
    }
    if (a.stats) {
        unsigned long long offers = static_cast<unsigned long long>(st_offers);
        if (valid) atomicAdd(&a.stats[2], offers);
        if (fell_back) atomicAdd(&a.stats[3], 1ull);
    }
    if (!valid) return;

    const float maxd2 = cnt > 0 ? key_d2(hp[cnt - 1]) : 0.f;
    int32_t *row = a.codes ? a.codes + static_cast<size_t>(idx) * K : nullptr;
    if (row) {
        if ((K & 3) == 0) {
            for (int s = 0; s < K; s += 4) {
                // slots s..s+3 are one 32-byte aligned group of this lane's heap
                const ulonglong2 lo = *reinterpret_cast<const ulonglong2 *>(hp + s);
                const ulonglong2 hi = *reinterpret_cast<const ulonglong2 *>(hp + s + 2);
                int4 v;
                v.x = (s < cnt) ? static_cast<int>(static_cast<unsigned int>(lo.x)) : -1;
                v.y = (s + 1 < cnt) ? static_cast<int>(static_cast<unsigned int>(lo.y)) : -1;
                v.z = (s + 2 < cnt) ? static_cast<int>(static_cast<unsigned int>(hi.x)) : -1;
                v.w = (s + 3 < cnt) ? static_cast<int>(static_cast<unsigned int>(hi.y)) : -1;
                reinterpret_cast<int4 *>(row)[s >> 2] = v;
            }
        } else {
            for (int s = 0; s < K; ++s)
                row[s] = (s < cnt) ? static_cast<int>(static_cast<unsigned int>(hp[s])) : -1;
        }
    }
    if (a.kth) a.kth[idx] = maxd2;
    if (a.measure) {
        const double y = a.part[idx].position[1];
        const double z = a.part[idx].position[2];
        a.measure[idx] = ball_measure(m, y, z, sqrt(static_cast<double>(maxd2)));
    }
}

template <bool kImages>
__global__ void k_knn_query(Model m, QueryArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int wib = threadIdx.x >> 5;
    const int kcap = knn_capacity(a.k, a.radius != nullptr);
    knn_bucket<kImages>(m, a, blockIdx.x * (blockDim.x >> 5) + wib, smem + wib * knn_warp_bytes(kcap), kcap);
}

// The owners the range query (k_knn_range) left over: the listed buckets, only the listed lanes of
// each, by the per-lane heap query with the full q.  A persistent grid walks the list, whose
// length the range query left in device memory.
__global__ void k_knn_fallback(Model m, QueryArgs a, const int *__restrict__ fb_count, const int *__restrict__ fb_leaf,
                               const unsigned int *__restrict__ fb_mask) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int wib = threadIdx.x >> 5, warps = blockDim.x >> 5;
    const int kcap = knn_capacity(a.k, false);
    unsigned char *wbase = smem + wib * knn_warp_bytes(kcap);
    const int total = *fb_count;
    for (int w = blockIdx.x * warps + wib; w < total; w += gridDim.x * warps) {
        knn_bucket<false>(m, a, fb_leaf[w], wbase, kcap, fb_mask[w]);
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------------------------
// Many swarms in one persistent launch.  Every warp takes (swarm, bucket) items from a device
// counter until none is left and runs the same knn_bucket as the one-swarm kernel, so each swarm's
// rows are bit-identical to its solo query.  Items are numbered swarm by swarm
// (leaf_prefix[s] .. leaf_prefix[s + 1]).
// ------------------------------------------------------------------------------------------------
__global__ void k_knn_batch(Model m, const BatchSwarm *__restrict__ tab, const int *__restrict__ leaf_prefix, int S,
                            int *__restrict__ next, const gd_particle *__restrict__ part, int32_t *__restrict__ codes,
                            double *__restrict__ measure, float *__restrict__ kth, int kcap, int prescan,
                            int bfs) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    unsigned char *wbase = smem + wib * knn_warp_bytes(kcap);
    const int total = leaf_prefix[S];
    while (true) {
        int item = 0;
        if (lane == 0) item = atomicAdd(next, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= total) break;
        int lo = 0, hi = S;  // the swarm s with leaf_prefix[s] <= item < leaf_prefix[s + 1]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (leaf_prefix[mid] <= item) lo = mid;
            else hi = mid;
        }
        const BatchSwarm &b = tab[lo];
        QueryArgs a;
        a.sorted = b.sorted;
        a.lo = b.lo;
        a.hi = b.hi;
        a.sub_lo = b.sub_lo;
        a.sub_hi = b.sub_hi;
        a.qrad = b.qrad;
        a.counters = b.counters;
        a.part = part + b.part_off;
        a.leaf_slots = b.leaf_slots;
        a.k = b.k;
        a.codes = codes + b.codes_off;
        a.measure = measure + b.part_off;
        a.kth = kth + b.part_off;
        a.radius = nullptr;
        a.stats = nullptr;
        a.prescan = prescan;
        a.bfs = bfs;
        knn_bucket<false>(m, a, item - leaf_prefix[lo], wbase, kcap);
        __syncwarp();
    }
}

// inactive owners of every swarm of a batch: a row of -1 and zero measure
__global__ void k_batch_inactive_rows(const BatchSwarm *__restrict__ tab, const long long *__restrict__ part_prefix,
                                      int S, long long total, int32_t *__restrict__ codes, double *__restrict__ measure,
                                      float *__restrict__ kth) {
    const long long g = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= total) return;
    int lo = 0, hi = S;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (part_prefix[mid] <= g) lo = mid;
        else hi = mid;
    }
    const BatchSwarm &b = tab[lo];
    const long long i = g - b.part_off;
    if (b.active[i]) return;
    for (int s = 0; s < b.k; ++s) codes[b.codes_off + i * b.k + s] = -1;
    measure[g] = 0.0;
    kth[g] = 0.f;
}

Status knn_batch_query(const Model &m, const BatchSwarm *dev_tab, const int *dev_leaf_prefix,
                       const long long *dev_part_prefix, int S, long long n_total, int kcap, int *dev_next,
                       const gd_particle *part, int32_t *codes, double *measure, float *kth, cudaStream_t s,
                       long long *launches, const Tuning &tune) {
    const size_t per_warp = knn_warp_bytes(kcap);
    int best_res = 0;
    const int warps = knn_block_warps(kcap, tune, &best_res);
    if (warps == 0) return Status{GD_ERR_INVALID_ARGUMENT, "warps per block do not fit in shared memory", 0};
    const size_t smem = per_warp * warps;
    static int smem_set[64] = {};
    int dev = 0, sms = 0;
    GD_TRY_CUDA(cudaGetDevice(&dev));
    GD_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (dev < 0 || dev >= 64 || smem_set[dev] < static_cast<int>(smem)) {
        GD_TRY_CUDA(cudaFuncSetAttribute(k_knn_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem)));
        if (dev >= 0 && dev < 64) smem_set[dev] = static_cast<int>(smem);
    }
    // persistent grid: every resident warp slot of every SM, each pulling items until none is left
    const int blocks = sms * (best_res / warps);
    GD_TRY_CUDA(cudaMemsetAsync(dev_next, 0, sizeof(int), s));
    k_knn_batch<<<blocks, warps * 32, smem, s>>>(m, dev_tab, dev_leaf_prefix, S, dev_next, part, codes, measure, kth,
                                                 kcap, tune.prescan, tune.bfs);
    k_batch_inactive_rows<<<static_cast<unsigned int>((n_total + 255) / 256), 256, 0, s>>>(
        dev_tab, dev_part_prefix, S, n_total, codes, measure, kth);
    if (launches) *launches += 2;
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}

// inactive owners: a row of -1 and zero measure (_col_cache.cuh:26-34)
__global__ void k_inactive_rows(int n, int K, const unsigned char *__restrict__ active, int32_t *__restrict__ codes,
                                double *__restrict__ measure, float *__restrict__ kth) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || active[i]) return;
    if (codes)
        for (int s = 0; s < K; ++s) codes[static_cast<size_t>(i) * K + s] = -1;
    if (measure) measure[i] = 0.0;
    if (kth) kth[i] = 0.f;
}

// Keplerian azimuthal advance phi += Omega_K(R) dt, wrapped into [x_min, x_max)
__global__ void k_drift_keplerian(Model m, int n, gd_particle *__restrict__ part, double dt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double y = part[i].position[1], z = part[i].position[2];
    if (!site_active(m, y, z)) return;
    const double R = cyl_R(m, y, z);
    const double width = m.x_max - m.x_min;
    double x = part[i].position[0] + sqrt(m.G * m.M_S / R / R / R) * dt;
    x = m.x_min + fmod(x - m.x_min, width);
    if (x < m.x_min) x += width;
    part[i].position[0] = x;
}

Status drift_keplerian(const Model &m, int n, gd_particle *part, double dt, cudaStream_t s) {
    k_drift_keplerian<<<(n + 255) / 256, 256, 0, s>>>(m, n, part, dt);
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}

// col_space_bin (col_space_bin.cu:11-35)
__global__ void k_space_bin(Model m, int n, const gd_particle *__restrict__ part, int32_t *__restrict__ spatial) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double x = part[i].position[0], y = part[i].position[1], z = part[i].position[2];
    int bx = 0, bz = 0;
    int by = static_cast<int>(floor((y - m.y_min) / (m.y_max - m.y_min) * m.col_bin_y));
    if (m.n_x > 1) bx = static_cast<int>(floor((x - m.x_min) / (m.x_max - m.x_min) * m.col_bin_x));
    if (m.n_z > 1) bz = static_cast<int>(floor((z - m.z_min) / (m.z_max - m.z_min) * m.col_bin_z));
    bx = bx < 0 ? 0 : (bx >= m.col_bin_x ? m.col_bin_x - 1 : bx);
    by = by < 0 ? 0 : (by >= m.col_bin_y ? m.col_bin_y - 1 : by);
    bz = bz < 0 ? 0 : (bz >= m.col_bin_z ? m.col_bin_z - 1 : bz);
    int cx = (m.n_x > 1) ? m.col_bin_x : 1;
    spatial[i] = bx + cx * (by + m.col_bin_y * bz);
}

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------
static int next_pow2(int v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}

Status geometry_alloc(Geometry &g, const Model &m, int n) {
    g.n = n;
    g.n_sites = m.wedge ? 3 * n : n;
    g.n_sort = (g.n_sites + kRadixTile - 1) / kRadixTile * kRadixTile;
    int leaves = (g.n_sites + kLeaf - 1) / kLeaf;
    g.leaf_slots = next_pow2(leaves < 1 ? 1 : leaves);
    g.key_bits = 21 * m.dim;
    int tiles = g.n_sort / kRadixTile;
    GD_TRY_CUDA(g.site.alloc(g.n_sites));
    GD_TRY_CUDA(g.q.alloc(n));
    GD_TRY_CUDA(g.active.alloc(n));
    GD_TRY_CUDA(g.key_a.alloc(g.n_sort));
    GD_TRY_CUDA(g.key_b.alloc(g.n_sort));
    GD_TRY_CUDA(g.val_a.alloc(g.n_sort));
    GD_TRY_CUDA(g.val_b.alloc(g.n_sort));
    // [digit][tile] counts, then the chunk totals of their scan when it spans several chunks
    const size_t hist_len = static_cast<size_t>(256) * tiles;
    const size_t chunks = (hist_len + kScanChunk - 1) / kScanChunk;
    GD_TRY_CUDA(g.hist.alloc(hist_len + (chunks > 1 ? chunks : 0)));
    GD_TRY_CUDA(g.sorted.alloc(static_cast<size_t>(g.leaf_slots) * kLeaf));
    GD_TRY_CUDA(g.node_lo.alloc(2 * static_cast<size_t>(g.leaf_slots)));
    GD_TRY_CUDA(g.node_hi.alloc(2 * static_cast<size_t>(g.leaf_slots)));
    GD_TRY_CUDA(g.sub_lo.alloc(static_cast<size_t>(g.leaf_slots) * kSubs));
    GD_TRY_CUDA(g.sub_hi.alloc(static_cast<size_t>(g.leaf_slots) * kSubs));
    GD_TRY_CUDA(g.counters.alloc(4));
    GD_TRY_CUDA(g.fb_leaf.alloc(static_cast<size_t>(g.leaf_slots)));
    GD_TRY_CUDA(g.fb_mask.alloc(static_cast<size_t>(g.leaf_slots)));
    GD_TRY_CUDA(g.fb_count.alloc(1));
    return Status::ok();
}

// counters: [0] active sites, [1] first non-finite index (INT_MAX if none), [2..3] zero
__global__ void k_counters_reset(int *counters) {
    if (threadIdx.x < 4) counters[threadIdx.x] = (threadIdx.x == 1) ? INT_MAX : 0;
}

static Status read_counters(Geometry &g, cudaStream_t s, int out[2]) {
    GD_TRY_CUDA(cudaMemcpyAsync(out, g.counters.ptr, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    GD_TRY_CUDA(cudaStreamSynchronize(s));
    return Status::ok();
}

Status geometry_build(Geometry &g, const Model &m, const gd_particle *dev_particle, cudaStream_t s) {
    const int n = g.n;
    g.launches += 2;
    k_counters_reset<<<1, 32, 0, s>>>(g.counters.ptr);
    k_site_init<<<(g.n_sort + 255) / 256, 256, 0, s>>>(m, n, g.n_sites, dev_particle, g.site.ptr, g.q.ptr,
                                                        g.active.ptr, g.key_a.ptr, g.val_a.ptr, g.n_sort,
                                                        g.counters.ptr);
    GD_TRY_CUDA(cudaGetLastError());
    if (m.wedge && m.morton_images) {
        g.launches += 1;
        k_morton_ghosts<<<(n + 255) / 256, 256, 0, s>>>(m, n, dev_particle, g.active.ptr, g.site.ptr,
                                                         g.key_a.ptr, g.counters.ptr);
        GD_TRY_CUDA(cudaGetLastError());
    }
    // the reference stops on the first non-finite particle before building (swarm_runtime.cu:382-393);
    // a deferred screen is read by geometry_check instead (non-finite particles are inactive and
    // carry the all-ones key, so the rest of the build and the query run safely past them)
    if (!g.deferred_check) GD_TRY(geometry_check(g, s));
    // radix sort over the bits that carry key information (inactive keys are all ones)
    const int tiles = g.n_sort / kRadixTile;
    const int bits = (g.sort_bits > 0 && g.sort_bits < g.key_bits) ? g.sort_bits : g.key_bits;
    const int passes = (bits + 7) / 8;
    const int shift0 = g.key_bits - 8 * passes > 0 ? g.key_bits - 8 * passes : 0;  // the top `bits`
    unsigned long long *kin = g.key_a.ptr, *kout = g.key_b.ptr;
    unsigned int *vin = g.val_a.ptr, *vout = g.val_b.ptr;
    const int hist_len = 256 * tiles;
    const int chunks = (hist_len + kScanChunk - 1) / kScanChunk;
    unsigned int *part = chunks > 1 ? g.hist.ptr + hist_len : nullptr;
    for (int p = 0; p < passes; ++p) {
        const int shift = shift0 + 8 * p;
        g.launches += part ? 4 : 3;
        k_radix_hist<<<tiles, kRadixThreads, 0, s>>>(kin, shift, tiles, g.hist.ptr);
        k_scan_chunks<<<chunks, kRadixThreads, 0, s>>>(g.hist.ptr, hist_len, part);
        if (part) k_scan_parts<<<1, kRadixThreads, 0, s>>>(part, chunks);
        k_radix_scatter<<<tiles, kRadixThreads, 0, s>>>(kin, vin, kout, vout, shift, tiles, g.hist.ptr, part);
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    GD_TRY_CUDA(cudaGetLastError());
    g.sorted_val = vin;
    g.sorted_key = kin;
    const int slots = g.leaf_slots * kLeaf;
    g.launches += 2;
    k_gather_sorted<<<(slots + 255) / 256, 256, 0, s>>>(slots, g.counters.ptr, vin, g.site.ptr, g.sorted.ptr);
    k_leaf_bounds<<<(g.leaf_slots * 32 + 255) / 256, 256, 0, s>>>(g.leaf_slots, g.counters.ptr, g.sorted.ptr,
                                                                  g.node_lo.ptr, g.node_hi.ptr, g.sub_lo.ptr,
                                                                  g.sub_hi.ptr);
    for (int count = g.leaf_slots / 2; count >= 1; count /= 2) {
        const int first = count - 1;
        g.launches += 1;
        k_tree_level<<<(count + 255) / 256, 256, 0, s>>>(first, count, g.node_lo.ptr, g.node_hi.ptr);
    }
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}

// ------------------------------------------------------------------------------------------------
// Batched geometry (BatchGeometry): every stage of geometry_build once over all swarms.
// ------------------------------------------------------------------------------------------------
// the last s in [0, S) with prefix[s] <= x (prefix[0] = 0, ascending)
__device__ __forceinline__ int segment_of(const long long *__restrict__ prefix, int S, long long x) {
    int lo = 0, hi = S - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= x) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

__global__ void k_batch_counters_reset(int S, int *counters) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 2 * S) counters[t] = (t & 1) ? INT_MAX : 0;
}

// k_site_init over the batch: key = swarm id above the top `mbits` Morton bits; an inactive or
// non-finite site carries an all-ones Morton field, so it sorts after its swarm's active sites
__global__ void k_batch_site_init(Model m, int S, const long long *__restrict__ part_prefix, long long n_total,
                                  long long n_sort, const gd_particle *__restrict__ part, float4 *__restrict__ site,
                                  float *__restrict__ qrad, unsigned char *__restrict__ active,
                                  unsigned long long *__restrict__ key, unsigned int *__restrict__ val, int mbits,
                                  int mshift, int *__restrict__ counters) {
    const long long g = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= n_sort) return;
    if (g >= n_total) {  // sort padding: after every swarm
        key[g] = ~0ull;
        val[g] = static_cast<unsigned int>(g);
        return;
    }
    const int sw = segment_of(part_prefix, S, g);
    const int i = static_cast<int>(g - part_prefix[sw]);
    const double2 *rec = reinterpret_cast<const double2 *>(part + g);
    const double2 a = rec[0], b = rec[1], c = rec[2], d = rec[3];
    const bool finite = isfinite(a.x) && isfinite(a.y) && isfinite(b.x) && isfinite(b.y) && isfinite(c.x) &&
                        isfinite(c.y) && isfinite(d.x) && isfinite(d.y);
    const unsigned long long ones = (mbits >= 64) ? ~0ull : ((1ull << mbits) - 1ull);
    unsigned long long field = ones;
    float4 st = make_float4(0.f, 0.f, 0.f, __int_as_float(3 * i));
    float qi = 0.f;
    bool act = false;
    if (!finite) {
        atomicMin(&counters[2 * sw + 1], i);
    } else {
        const double x = a.x, y = a.y, z = b.x;
        act = site_active(m, y, z);
        const double R = cyl_R(m, y, z);
        const double Z = cyl_Z(m, y, z);
        const float3 pt = (m.n_x == 1 && m.n_z == 1)
                              ? make_float3(static_cast<float>(R), 0.0f, 0.0f)
                              : make_float3(static_cast<float>(R * cos(x)), static_cast<float>(R * sin(x)),
                                            static_cast<float>(Z));
        st.x = pt.x;
        st.y = pt.y;
        st.z = pt.z;
        if (act) {
            qi = static_cast<float>(m.h_search * get_hg(m, R) * R);
            field = morton_key(m, pt) >> mshift;
            if (field == ones) field = ones - 1;  // strictly before the swarm's inactive sites
        }
    }
    site[g] = st;
    qrad[g] = qi;
    active[g] = act ? 1 : 0;
    key[g] = (static_cast<unsigned long long>(sw) << mbits) | field;
    val[g] = static_cast<unsigned int>(g);
    // one atomic per swarm present among the warp's active lanes
    const unsigned int am = __ballot_sync(__activemask(), act);
    if (act) {
        const unsigned int peers = __match_any_sync(am, sw);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&counters[2 * sw], __popc(peers));
    }
}

// k_gather_sorted over the batch: global sorted slot j of swarm s is its slot j - 32 * leaf_prefix[s]
__global__ void k_batch_gather(int S, long long n_slots, const long long *__restrict__ leaf_prefix,
                               const long long *__restrict__ part_prefix, const int *__restrict__ counters,
                               const unsigned int *__restrict__ val, const float4 *__restrict__ site,
                               float4 *__restrict__ sorted) {
    const long long j = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= n_slots) return;
    const int sw = segment_of(leaf_prefix, S, j / kLeaf);
    const long long l = j - leaf_prefix[sw] * kLeaf;
    const int n_act = counters[2 * sw];
    const long long n_pad = (n_act + kLeaf - 1) / kLeaf * kLeaf;
    if (l >= n_pad) return;
    sorted[j] = (l < n_act) ? site[val[part_prefix[sw] + l]]
                            : make_float4(CUDART_INF_F_, CUDART_INF_F_, CUDART_INF_F_, __int_as_float(-1));
}

// k_leaf_bounds over the batch: one warp per leaf slot of every swarm
__global__ void k_batch_leaf_bounds(int S, long long n_leaves, const long long *__restrict__ leaf_prefix,
                                    const long long *__restrict__ node_off, const int *__restrict__ counters,
                                    const float4 *__restrict__ sorted, float4 *__restrict__ lo, float4 *__restrict__ hi,
                                    float4 *__restrict__ sub_lo, float4 *__restrict__ sub_hi) {
    const long long L = (static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (L >= n_leaves) return;
    const int sw = segment_of(leaf_prefix, S, L);
    const long long leaf = L - leaf_prefix[sw];
    const long long slots = leaf_prefix[sw + 1] - leaf_prefix[sw];
    const int n_act = counters[2 * sw];
    const long long i = leaf * kLeaf + lane;
    float3 a = make_float3(CUDART_INF_F_, CUDART_INF_F_, CUDART_INF_F_);
    float3 b = make_float3(-CUDART_INF_F_, -CUDART_INF_F_, -CUDART_INF_F_);
    if (i < n_act) {
        const float4 st = sorted[leaf_prefix[sw] * kLeaf + i];
        a = make_float3(st.x, st.y, st.z);
        b = a;
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        if (off == kSub && (lane & (kSub - 1)) == 0) {
            sub_lo[L * kSubs + lane / kSub] = make_float4(a.x, a.y, a.z, 0.f);
            sub_hi[L * kSubs + lane / kSub] = make_float4(b.x, b.y, b.z, 0.f);
        }
        a.x = fminf(a.x, __shfl_xor_sync(0xffffffffu, a.x, off));
        a.y = fminf(a.y, __shfl_xor_sync(0xffffffffu, a.y, off));
        a.z = fminf(a.z, __shfl_xor_sync(0xffffffffu, a.z, off));
        b.x = fmaxf(b.x, __shfl_xor_sync(0xffffffffu, b.x, off));
        b.y = fmaxf(b.y, __shfl_xor_sync(0xffffffffu, b.y, off));
        b.z = fmaxf(b.z, __shfl_xor_sync(0xffffffffu, b.z, off));
    }
    if (lane == 0) {
        const long long node = node_off[sw] + slots - 1 + leaf;
        lo[node] = make_float4(a.x, a.y, a.z, 0.f);
        hi[node] = make_float4(b.x, b.y, b.z, 0.f);
    }
}

// k_tree_level over the batch: rows (node offset, first node, count, running count) of one level
__global__ void k_batch_tree_level(const int4 *__restrict__ rows, int n_rows, int n_nodes, float4 *__restrict__ lo,
                                   float4 *__restrict__ hi) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_nodes) return;
    int r0 = 0, r1 = n_rows - 1;
    while (r0 < r1) {
        const int mid = (r0 + r1 + 1) >> 1;
        if (rows[mid].w <= t) r0 = mid;
        else r1 = mid - 1;
    }
    const int4 row = rows[r0];
    const long long base = row.x;
    const int node = row.y + (t - row.w);
    const float4 l0 = lo[base + 2 * node + 1], l1 = lo[base + 2 * node + 2];
    const float4 h0 = hi[base + 2 * node + 1], h1 = hi[base + 2 * node + 2];
    lo[base + node] = make_float4(fminf(l0.x, l1.x), fminf(l0.y, l1.y), fminf(l0.z, l1.z), 0.f);
    hi[base + node] = make_float4(fmaxf(h0.x, h1.x), fmaxf(h0.y, h1.y), fmaxf(h0.z, h1.z), 0.f);
}

Status batch_geometry_alloc(BatchGeometry &g, const Model &m, int S, const int *n_p, int sort_bits) {
    g.S = S;
    g.h_part_prefix.assign(S + 1, 0);
    g.h_leaf_prefix.assign(S + 1, 0);
    g.h_node_off.assign(S + 1, 0);
    g.leaf_slots.assign(S, 0);
    for (int s = 0; s < S; ++s) {
        const int leaves = (n_p[s] + kLeaf - 1) / kLeaf;
        g.leaf_slots[s] = next_pow2(leaves < 1 ? 1 : leaves);
        g.h_part_prefix[s + 1] = g.h_part_prefix[s] + n_p[s];
        g.h_leaf_prefix[s + 1] = g.h_leaf_prefix[s] + g.leaf_slots[s];
        g.h_node_off[s + 1] = g.h_node_off[s] + 2 * static_cast<long long>(g.leaf_slots[s]);
    }
    g.n_total = g.h_part_prefix[S];
    if (g.n_total >= 0xffffffffLL || g.h_node_off[S] >= 0x7fffffffLL)
        return Status{GD_ERR_INVALID_ARGUMENT, "batch too large for 32-bit site and node indices", 0};
    g.n_sort = (g.n_total + kRadixTile - 1) / kRadixTile * kRadixTile;
    const int key_bits = 21 * m.dim;
    g.sbits = 0;
    while ((1LL << g.sbits) < S) ++g.sbits;
    if (g.sbits > 32) return Status{GD_ERR_INVALID_ARGUMENT, "too many swarms for the sort key", 0};
    // by default the top Morton bits that fit beside the swarm id (the lists are exact for any key)
    g.mbits = (sort_bits > 0 && sort_bits < key_bits) ? sort_bits : key_bits;
    if (sort_bits == 0 && g.mbits + g.sbits > 64) g.mbits = 64 - g.sbits;
    g.mshift = key_bits - g.mbits;
    if (g.mbits + g.sbits > 64) return Status{GD_ERR_INVALID_ARGUMENT, "too many swarms for the sort key", 0};
    const long long tiles = g.n_sort / kRadixTile;
    const size_t hist_len = static_cast<size_t>(256) * tiles;
    const size_t chunks = (hist_len + kScanChunk - 1) / kScanChunk;
    const long long L = g.h_leaf_prefix[S];
    GD_TRY_CUDA(g.site.alloc(g.n_total));
    GD_TRY_CUDA(g.q.alloc(g.n_total));
    GD_TRY_CUDA(g.active.alloc(g.n_total));
    GD_TRY_CUDA(g.key_a.alloc(g.n_sort));
    GD_TRY_CUDA(g.key_b.alloc(g.n_sort));
    GD_TRY_CUDA(g.val_a.alloc(g.n_sort));
    GD_TRY_CUDA(g.val_b.alloc(g.n_sort));
    GD_TRY_CUDA(g.hist.alloc(hist_len + (chunks > 1 ? chunks : 0)));
    GD_TRY_CUDA(g.sorted.alloc(static_cast<size_t>(L) * kLeaf));
    GD_TRY_CUDA(g.node_lo.alloc(g.h_node_off[S]));
    GD_TRY_CUDA(g.node_hi.alloc(g.h_node_off[S]));
    GD_TRY_CUDA(g.sub_lo.alloc(static_cast<size_t>(L) * kSubs));
    GD_TRY_CUDA(g.sub_hi.alloc(static_cast<size_t>(L) * kSubs));
    GD_TRY_CUDA(g.counters.alloc(2 * static_cast<size_t>(S)));
    GD_TRY_CUDA(g.part_prefix.alloc(S + 1));
    GD_TRY_CUDA(g.leaf_prefix.alloc(S + 1));
    GD_TRY_CUDA(g.node_off.alloc(S + 1));
    GD_TRY_CUDA(cudaMemcpy(g.part_prefix.ptr, g.h_part_prefix.data(), sizeof(long long) * (S + 1),
                           cudaMemcpyHostToDevice));
    GD_TRY_CUDA(cudaMemcpy(g.leaf_prefix.ptr, g.h_leaf_prefix.data(), sizeof(long long) * (S + 1),
                           cudaMemcpyHostToDevice));
    GD_TRY_CUDA(cudaMemcpy(g.node_off.ptr, g.h_node_off.data(), sizeof(long long) * (S + 1), cudaMemcpyHostToDevice));
    // tree level rows: level t covers the nodes t levels above each swarm's leaves
    int depth_max = 0;
    for (int s = 0; s < S; ++s) {
        int d = 0;
        while ((1 << d) < g.leaf_slots[s]) ++d;
        depth_max = d > depth_max ? d : depth_max;
    }
    std::vector<int4> rows;
    g.level_row0.assign(depth_max + 1, 0);
    g.level_rows.assign(depth_max + 1, 0);
    g.level_nodes.assign(depth_max + 1, 0);
    for (int t = 1; t <= depth_max; ++t) {
        g.level_row0[t] = static_cast<int>(rows.size());
        int run = 0;
        for (int s = 0; s < S; ++s) {
            const int count = g.leaf_slots[s] >> t;
            if (count < 1) continue;
            rows.push_back(make_int4(static_cast<int>(g.h_node_off[s]), count - 1, count, run));
            run += count;
        }
        g.level_rows[t] = static_cast<int>(rows.size()) - g.level_row0[t];
        g.level_nodes[t] = run;
    }
    GD_TRY_CUDA(g.level_tab.alloc(rows.size()));
    if (!rows.empty())
        GD_TRY_CUDA(cudaMemcpy(g.level_tab.ptr, rows.data(), sizeof(int4) * rows.size(), cudaMemcpyHostToDevice));
    return Status::ok();
}

Status batch_geometry_build(BatchGeometry &g, const Model &m, const gd_particle *dev_particle, cudaStream_t s) {
    const int S = g.S;
    g.launches += 2;
    k_batch_counters_reset<<<(2 * S + 255) / 256, 256, 0, s>>>(S, g.counters.ptr);
    k_batch_site_init<<<static_cast<unsigned int>((g.n_sort + 255) / 256), 256, 0, s>>>(
        m, S, g.part_prefix.ptr, g.n_total, g.n_sort, dev_particle, g.site.ptr, g.q.ptr, g.active.ptr, g.key_a.ptr,
        g.val_a.ptr, g.mbits, g.mshift, g.counters.ptr);
    GD_TRY_CUDA(cudaGetLastError());
    // one LSD radix sort over the swarm id and the kept Morton bits
    const int tiles = static_cast<int>(g.n_sort / kRadixTile);
    const int passes = (g.mbits + g.sbits + 7) / 8;
    unsigned long long *kin = g.key_a.ptr, *kout = g.key_b.ptr;
    unsigned int *vin = g.val_a.ptr, *vout = g.val_b.ptr;
    const int hist_len = 256 * tiles;
    const int chunks = (hist_len + kScanChunk - 1) / kScanChunk;
    unsigned int *part = chunks > 1 ? g.hist.ptr + hist_len : nullptr;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        g.launches += part ? 4 : 3;
        k_radix_hist<<<tiles, kRadixThreads, 0, s>>>(kin, shift, tiles, g.hist.ptr);
        k_scan_chunks<<<chunks, kRadixThreads, 0, s>>>(g.hist.ptr, hist_len, part);
        if (part) k_scan_parts<<<1, kRadixThreads, 0, s>>>(part, chunks);
        k_radix_scatter<<<tiles, kRadixThreads, 0, s>>>(kin, vin, kout, vout, shift, tiles, g.hist.ptr, part);
        std::swap(kin, kout);
        std::swap(vin, vout);
    }
    const long long L = g.h_leaf_prefix[S];
    const long long slots = L * kLeaf;
    g.launches += 2;
    k_batch_gather<<<static_cast<unsigned int>((slots + 255) / 256), 256, 0, s>>>(
        S, slots, g.leaf_prefix.ptr, g.part_prefix.ptr, g.counters.ptr, vin, g.site.ptr, g.sorted.ptr);
    k_batch_leaf_bounds<<<static_cast<unsigned int>((L * 32 + 255) / 256), 256, 0, s>>>(
        S, L, g.leaf_prefix.ptr, g.node_off.ptr, g.counters.ptr, g.sorted.ptr, g.node_lo.ptr, g.node_hi.ptr,
        g.sub_lo.ptr, g.sub_hi.ptr);
    for (size_t t = 1; t < g.level_rows.size(); ++t) {
        if (g.level_nodes[t] == 0) continue;
        g.launches += 1;
        k_batch_tree_level<<<(g.level_nodes[t] + 255) / 256, 256, 0, s>>>(
            g.level_tab.ptr + g.level_row0[t], g.level_rows[t], g.level_nodes[t], g.node_lo.ptr, g.node_hi.ptr);
    }
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}

Status batch_geometry_check(BatchGeometry &g, cudaStream_t s, int *swarm) {
    std::vector<int> c(2 * static_cast<size_t>(g.S));
    GD_TRY_CUDA(cudaMemcpyAsync(c.data(), g.counters.ptr, sizeof(int) * c.size(), cudaMemcpyDeviceToHost, s));
    GD_TRY_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < g.S; ++k) {
        if (c[2 * k + 1] != INT_MAX) {
            if (swarm) *swarm = k;
            Status st;
            st.code = GD_ERR_NONFINITE;
            st.detail = g.h_part_prefix[k] + c[2 * k + 1];
            st.msg = "non-finite particle state before collision search at particle " + std::to_string(st.detail) +
                     " (swarm " + std::to_string(k) + ")";
            return st;
        }
    }
    return Status::ok();
}

Status geometry_check(Geometry &g, cudaStream_t s) {
    int cnt[2];
    GD_TRY(read_counters(g, s, cnt));
    if (cnt[1] != INT_MAX) {
        Status st;
        st.code = GD_ERR_NONFINITE;
        st.detail = cnt[1];
        st.msg = "non-finite particle state before collision search at particle " + std::to_string(cnt[1]);
        return st;
    }
    return Status::ok();
}

size_t knn_smem_per_warp(int K) { return knn_warp_bytes(K); }

int knn_block_warps(int K, const Tuning &tune, int *resident) {
    // the per-lane heaps bound residency: by default pick the block width that keeps the most
    // warps per SM (227 KB of shared memory per SM, at most 8 warps per block)
    const size_t per_warp = knn_smem_per_warp(K);
    const size_t sm_bytes = 227 * 1024;
    auto res_of = [&](int w) { return static_cast<int>(sm_bytes / (per_warp * w + 1024)) * w; };
    if (tune.warps > 0) {
        if (tune.warps > 32 || per_warp * tune.warps > sm_bytes) return 0;
        if (resident) *resident = res_of(tune.warps);
        return tune.warps;
    }
    int best = 1, best_res = 0;
    for (int w = 1; w <= 8; ++w) {
        if (per_warp * w > sm_bytes) break;
        const int res = res_of(w);
        if (res > best_res) {
            best_res = res;
            best = w;
        }
    }
    if (resident) *resident = best_res;
    return best;
}

Status knn_fallback(Geometry &g, const Model &m, const gd_particle *dev_particle, int32_t *codes, double *measure,
                    float *kth_d2, cudaStream_t s, unsigned long long *stats, const Tuning &tune) {
    const int K = m.n_k;
    const int kcap = knn_capacity(K, false);
    int resident = 0;
    const int warps = knn_block_warps(kcap, tune, &resident);
    if (warps == 0) return Status{GD_ERR_INVALID_ARGUMENT, "warps per block do not fit in shared memory", 0};
    const size_t smem = knn_smem_per_warp(kcap) * warps;
    static int smem_set[64] = {};
    int dev = 0, sms = 0;
    GD_TRY_CUDA(cudaGetDevice(&dev));
    GD_TRY_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (dev < 0 || dev >= 64 || smem_set[dev] < static_cast<int>(smem)) {
        GD_TRY_CUDA(cudaFuncSetAttribute(k_knn_fallback, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem)));
        if (dev >= 0 && dev < 64) smem_set[dev] = static_cast<int>(smem);
    }
    QueryArgs qa;
    qa.sorted = g.sorted.ptr;
    qa.lo = g.node_lo.ptr;
    qa.hi = g.node_hi.ptr;
    qa.sub_lo = g.sub_lo.ptr;
    qa.sub_hi = g.sub_hi.ptr;
    qa.qrad = g.q.ptr;
    qa.counters = g.counters.ptr;
    qa.part = dev_particle;
    qa.leaf_slots = g.leaf_slots;
    qa.k = K;
    qa.codes = codes;
    qa.measure = measure;
    qa.kth = kth_d2;
    qa.radius = nullptr;
    qa.stats = stats;
    qa.prescan = tune.prescan;
    qa.bfs = tune.bfs;
    // one block per SM's worth of resident warps: the list is short (owners whose proposal missed)
    const int blocks = sms * (resident / warps > 0 ? resident / warps : 1);
    g.launches += 1;
    k_knn_fallback<<<blocks, warps * 32, smem, s>>>(m, qa, g.fb_count.ptr, g.fb_leaf.ptr, g.fb_mask.ptr);
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}

Status knn_query(Geometry &g, const Model &m, const gd_particle *dev_particle, int32_t *codes, double *measure,
                 float *kth_d2, cudaStream_t s, const float *radius, unsigned long long *stats, const Tuning &tune) {
    const int K = m.n_k;
    if (radius && tune.range && knn_range_eligible(m, K)) {
        // a proposed radius: the warp-per-owner range query (gd_range.cu), its leftovers by the heap query
        GD_TRY(knn_range(g, m, dev_particle, codes, measure, kth_d2, s, radius, stats, tune));
        g.launches += 1;
        k_inactive_rows<<<(g.n + 255) / 256, 256, 0, s>>>(g.n, K, g.active.ptr, codes, measure, kth_d2);
        GD_TRY_CUDA(cudaGetLastError());
        return Status::ok();
    }
    const int kcap = knn_capacity(K, radius != nullptr);
    const size_t per_warp = knn_smem_per_warp(kcap);
    const int warps = knn_block_warps(kcap, tune, nullptr);
    if (warps == 0) return Status{GD_ERR_INVALID_ARGUMENT, "warps per block do not fit in shared memory", 0};
    const size_t smem = per_warp * warps;
    // raise the kernel's shared-memory limit only when a larger one is needed, so that a step
    // enqueued under stream capture after a first eager call makes no attribute call
    static int smem_set[2][64] = {};
    int dev = 0;
    GD_TRY_CUDA(cudaGetDevice(&dev));
    const int wi = m.wedge ? 1 : 0;
    if (dev < 0 || dev >= 64 || smem_set[wi][dev] < static_cast<int>(smem)) {
        GD_TRY_CUDA(cudaFuncSetAttribute(m.wedge ? k_knn_query<true> : k_knn_query<false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
        if (dev >= 0 && dev < 64) smem_set[wi][dev] = static_cast<int>(smem);
    }
    QueryArgs qa;
    qa.sorted = g.sorted.ptr;
    qa.lo = g.node_lo.ptr;
    qa.hi = g.node_hi.ptr;
    qa.sub_lo = g.sub_lo.ptr;
    qa.sub_hi = g.sub_hi.ptr;
    qa.qrad = g.q.ptr;
    qa.counters = g.counters.ptr;
    qa.part = dev_particle;
    qa.leaf_slots = g.leaf_slots;
    qa.k = K;
    qa.codes = codes;
    qa.measure = measure;
    qa.kth = kth_d2;
    qa.radius = radius;
    qa.stats = stats;
    qa.prescan = tune.prescan;
    qa.bfs = tune.bfs;
    const int max_leaves = (g.n_sites + kLeaf - 1) / kLeaf;
    const int blocks = (max_leaves + warps - 1) / warps;
    g.launches += 2;
    if (m.wedge) k_knn_query<true><<<blocks, warps * 32, smem, s>>>(m, qa);
    else k_knn_query<false><<<blocks, warps * 32, smem, s>>>(m, qa);
    k_inactive_rows<<<(g.n + 255) / 256, 256, 0, s>>>(g.n, K, g.active.ptr, codes, measure, kth_d2);
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}

// clears only the first-bad-index counter: the screen keeps the built geometry's active-site count
// and largest q, which a later query on the same geometry reads
__global__ void k_bad_index_reset(int *counters) {
    if (threadIdx.x == 0) counters[1] = INT_MAX;
}

Status state_screen(Geometry &g, const Model &m, const gd_particle *dev_particle, cudaStream_t s) {
    (void)m;
    g.launches += 2;
    k_bad_index_reset<<<1, 32, 0, s>>>(g.counters.ptr);
    k_state_screen<<<(g.n + 255) / 256, 256, 0, s>>>(g.n, dev_particle, g.counters.ptr);
    GD_TRY_CUDA(cudaGetLastError());
    if (g.deferred_check) return Status::ok();  // read by geometry_check later
    int cnt[2];
    GD_TRY(read_counters(g, s, cnt));
    if (cnt[1] != INT_MAX) {
        Status st;
        st.code = GD_ERR_NONFINITE;
        st.detail = cnt[1];
        st.msg = "non-finite particle state before collision search at particle " + std::to_string(cnt[1]);
        return st;
    }
    return Status::ok();
}

// keeps the first failed screen of a captured step: a later build of the same step resets the
// geometry's counter, and the reference stops at the first screen that fails
__global__ void k_screen_keep(const int *counters, int *first) {
    if (threadIdx.x == 0 && *first == INT_MAX && counters[1] != INT_MAX) *first = counters[1];
}

Status screen_keep(Geometry &g, int *first, cudaStream_t s) {
    g.launches += 1;
    k_screen_keep<<<1, 32, 0, s>>>(g.counters.ptr, first);
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}

Status space_bin(const Model &m, const gd_particle *dev_particle, int n, int32_t *spatial, cudaStream_t s) {
    k_space_bin<<<(n + 255) / 256, 256, 0, s>>>(m, n, dev_particle, spatial);
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}

}  // namespace gd
