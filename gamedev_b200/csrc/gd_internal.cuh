// Internal declarations shared by the translation units of libgd_b200.
//
// Layout in HBM (one handle, n_p particles, K = n_k):
//   caller-owned  : gd_particle[n_p] (64 B AoS, the reference `struct swarm`), curandState[n_p]
//   geometry      : site[n_p] float4 (x, y, z, code bits), q[n_p] float search radius,
//                   active[n_p] u8, key/val ping-pong [n_sort] u64/u32 (radix sort),
//                   sorted[n_pad] float4 (Morton order, w = code), node lo/hi [2*leaf_slots] float4
//   neighbour cache: codes[n_p*K] int32 owner-major, measure[n_p] f64, kth_d2[n_p] f32
//   controller    : SoA owner state f64 (size_old, numr_old, time, hazard, jump1/2/max, rates),
//                   query_environment[n_p] (8 x f64), group/bin scratch
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/gd_b200.h"

namespace gd {

// Leaf width of the bucket tree: one Morton-ordered bucket of 32 sites is one warp's query tile
// and one candidate tile.
constexpr int kLeaf = 32;
constexpr int kSub = 8;              // sites per leaf sub-box
constexpr int kSubs = kLeaf / kSub;  // sub-boxes per leaf
constexpr int kPrescan = 2;          // Morton-neighbour buckets scanned on each side before the walk
constexpr int kMaxK = 256;
constexpr int kRadixThreads = 256;
constexpr int kRadixItems = 16;
constexpr int kRadixTile = kRadixThreads * kRadixItems;  // 4096 keys per sort tile
constexpr int kScanItems = 16;                            // histogram entries per scan thread
constexpr int kScanChunk = kRadixThreads * kScanItems;    // 4096 entries per scan block

// Device copy of the model constants, passed by value to kernels.
struct Model {
    double G, M_S, R_0, S_0;
    int n_x, n_y, n_z;
    double x_min, x_max, y_min, y_max, z_min, z_max;
    double sigma_0, aspr_0, idx_p, idx_q;
    int const_nu;
    double nu, alpha;
    int code_unit;
    double reynolds_0, m_mol, x_sec;
    int half_disk, const_st;
    double stokes_0, rho_0;
    int coag_kernel, n_k;
    double h_search, v_frag;
    int col_event_cap, col_bin_x, col_bin_y, col_bin_z, col_bin_s, col_bin_min;
    double col_bath_max, col_bath_eps, col_bath_alpha;
    double init_smin, init_smax;
    // derived
    int dim;          // 2 when the polar direction is collapsed, else 3
    int local_groups; // spatial controller groups (_col_types.cuh:463)
    int raw_bins;     // local_groups * col_bin_s (_col_bound.cuh:223-229)
    // Azimuthal wedge: X_WEDGE (const_defs.cuh:56-57), n_x > 1 and an azimuth shorter than 2 pi.
    // Every particle then has two more sites, rotated by -width (image 1) and +width (image 2).
    int wedge;
    int morton_images;     // 1: the Morton search's rotation, width and dedup decision; 0: KD's
    float wedge_width;     // KD: float(x_max - x_min) (col_site_init.cu:60);
                           // Morton: float(x_max) - float(x_min) (morton_ghost.cuh:62)
    float image_dist_min;  // _get_image_dist_min (param_grid.cuh:86-89); -1 without a wedge
};

Model make_model(const gd_config &c);

// Status carried out of a call: code, message, numeric detail.
struct Status {
    gd_status code = GD_OK;
    std::string msg;
    long long detail = 0;
    static Status ok() { return {}; }
    explicit operator bool() const { return code == GD_OK; }
};

Status cuda_status(cudaError_t e, const char *what);
// Caller-owned device arrays must sit on their element's alignment: particle records and RNG states
// (doubles inside) on 8 bytes, codes on 4.  A misaligned pointer would fault the first kernel that
// loads through it, so the entry points reject one as GD_ERR_INVALID_ARGUMENT.
inline bool aligned_to(const void *p, size_t a) { return reinterpret_cast<uintptr_t>(p) % a == 0; }

#define GD_TRY_CUDA(expr)                                              \
    do {                                                               \
        cudaError_t gd_e_ = (expr);                                    \
        if (gd_e_ != cudaSuccess) return ::gd::cuda_status(gd_e_, #expr); \
    } while (0)

#define GD_TRY(expr)                   \
    do {                               \
        ::gd::Status gd_s_ = (expr);   \
        if (!gd_s_) return gd_s_;      \
    } while (0)

// Owned device allocation.
template <typename T>
struct DevBuf {
    T *ptr = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    cudaError_t alloc(size_t count) {
        release();
        n = count;
        if (count == 0) return cudaSuccess;
        return cudaMalloc(reinterpret_cast<void **>(&ptr), sizeof(T) * count);
    }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        n = 0;
    }
};

// Geometry (index) state of one swarm.
struct Geometry {
    int n = 0;              // particles
    int n_sites = 0;        // sites: n, or 3n with wedge images (site n*image + i)
    int n_sort = 0;         // n_sites rounded up to the sort tile
    int leaf_slots = 0;     // power of two >= ceil(n / kLeaf)
    int key_bits = 0;       // Morton bits sorted (3*21 or 2*21)
    DevBuf<float4> site;    // by site index
    DevBuf<float> q;        // search radius by particle index
    DevBuf<unsigned char> active;
    DevBuf<unsigned long long> key_a, key_b;
    DevBuf<unsigned int> val_a, val_b;
    DevBuf<unsigned int> hist;    // [256][tiles]
    DevBuf<float4> sorted;        // [leaf_slots*kLeaf] Morton-ordered sites, w = code bits
    DevBuf<float4> node_lo, node_hi;  // implicit tree, 2*leaf_slots-1 nodes
    DevBuf<float4> sub_lo, sub_hi;    // four 8-site sub-boxes per leaf, [leaf_slots*4]
    DevBuf<int> counters;         // [0] active sites, [1] first bad index (INT_MAX if none),
                                  // [2] bits of the largest q (wedges only)
    unsigned int *sorted_val = nullptr;  // points into val_a or val_b after the sort
    unsigned long long *sorted_key = nullptr;  // points into key_a or key_b after the sort
    long long launches = 0;              // kernels launched by this geometry (reported by the ABI)
    // Deferred screen: the build enqueues everything without waiting for the non-finite screen,
    // and geometry_check reads it later (what stream capture into a CUDA graph needs).
    bool deferred_check = false;
    int sort_bits = 0;  // top Morton key bits the radix sort orders by (0: all)
    // owners the radius-bounded range query leaves to the heap query: bucket, lanes, count
    DevBuf<int> fb_leaf;
    DevBuf<unsigned int> fb_mask;
    DevBuf<int> fb_count;
};

// Speed-only settings of the neighbour search (every setting gives the same exact lists).
struct Tuning {
    int warps = 0;            // warps per block of the top-K kernel; 0 = the most resident warps
    int prescan = kPrescan;   // Morton-neighbour buckets scanned on each side before the walk
    int bfs = 1;              // breadth-first walk (1) or depth-first walk (0)
    int sort_bits = 0;        // top Morton key bits the radix sort orders by (0: all)
    int range = 1;            // radius-bounded query: warp-per-owner range query (1) or per-lane heaps (0)
};

Status geometry_alloc(Geometry &g, const Model &m, int n);
// col_site_init + Morton keys + radix sort + bucket tree.  Returns GD_ERR_NONFINITE with the
// smallest bad index when a particle is non-finite.
Status geometry_build(Geometry &g, const Model &m, const gd_particle *dev_particle, cudaStream_t s);
// The non-finite screen of the last build: GD_ERR_NONFINITE with the smallest bad index, if any.
// Synchronises the stream.
Status geometry_check(Geometry &g, cudaStream_t s);
// *first = the first bad index of the latest screen, unless an earlier one was kept (INT_MAX: none)
Status screen_keep(Geometry &g, int *first, cudaStream_t s);
// Exact top-K over the bucket tree.  Writes codes/measure/kth (any may be null).
// With `radius` (per particle, may be null) the walk is first bounded by min(q, radius) and falls
// back to q for owners that find fewer than K sites inside; `stats` (may be null) accumulates
// [8-site leaf groups scanned, nodes tested, candidate offers, fallbacks].
Status knn_query(Geometry &g, const Model &m, const gd_particle *dev_particle, int32_t *codes,
                 double *measure, float *kth_d2, cudaStream_t s, const float *radius = nullptr,
                 unsigned long long *stats = nullptr, const Tuning &tune = Tuning());
// Warps per block of the top-K kernel for K neighbours under `tune` (0 when infeasible), and the
// resident warps per SM it gives.
int knn_block_warps(int K, const Tuning &tune, int *resident);
// The radius-bounded range query (gd_range.cu) and the heap query over its leftover owners.
bool knn_range_eligible(const Model &m, int K);
Status knn_range(Geometry &g, const Model &m, const gd_particle *dev_particle, int32_t *codes, double *measure,
                 float *kth_d2, cudaStream_t s, const float *radius, unsigned long long *stats, const Tuning &tune);
Status knn_fallback(Geometry &g, const Model &m, const gd_particle *dev_particle, int32_t *codes, double *measure,
                    float *kth_d2, cudaStream_t s, unsigned long long *stats, const Tuning &tune);
// One swarm of a batch as the persistent batch query sees it: its geometry and the offsets of its
// rows in the caller's concatenated particle (part_off) and code (codes_off) buffers.
struct BatchSwarm {
    const float4 *sorted, *lo, *hi, *sub_lo, *sub_hi;
    const float *qrad;
    const unsigned char *active;
    const int *counters;
    int leaf_slots;
    int k;
    long long part_off;
    long long codes_off;
};
// The geometry of many swarms built together: one launch per stage for all of them.  Sites are
// concatenated in swarm order (particle g of the batch is particle g - part_prefix[s] of swarm s);
// one LSD radix sort orders (swarm id, top Morton bits) keys, so each swarm's sites come out
// contiguous and Morton-ordered; per-swarm sorted tiles, trees and sub-boxes sit at the offsets
// below, and the BatchSwarm table points into them.
struct BatchGeometry {
    int S = 0;
    long long n_total = 0, n_sort = 0;
    int mbits = 0, mshift = 0, sbits = 0;  // Morton bits kept, low Morton bits dropped, swarm id bits
    DevBuf<float4> site;                   // [n_total], w = code bits of the swarm-local index
    DevBuf<float> q;
    DevBuf<unsigned char> active;
    DevBuf<unsigned long long> key_a, key_b;
    DevBuf<unsigned int> val_a, val_b, hist;
    DevBuf<float4> sorted, node_lo, node_hi, sub_lo, sub_hi;
    DevBuf<int> counters;                  // [2S]: active count, first non-finite local index
    DevBuf<long long> part_prefix, leaf_prefix, node_off;  // [S+1] particles, leaf slots; [S] nodes
    std::vector<long long> h_part_prefix, h_leaf_prefix, h_node_off;
    std::vector<int> leaf_slots;           // per swarm, a power of two
    // tree levels bottom-up: level t holds, for each swarm with at least t levels, the nodes t
    // levels above its leaves as (node offset, first node, count, running count) rows; the rows of
    // all levels are concatenated in level_tab, level t's starting at level_row0[t]
    DevBuf<int4> level_tab;
    std::vector<int> level_row0, level_rows, level_nodes;
    long long launches = 0;
};
Status batch_geometry_alloc(BatchGeometry &g, const Model &m, int S, const int *n_p, int sort_bits);
Status batch_geometry_build(BatchGeometry &g, const Model &m, const gd_particle *dev_particle, cudaStream_t s);
// The non-finite screen of the last build: GD_ERR_NONFINITE with the smallest bad index of the
// first swarm that has one (as a batch index); synchronises the stream.
Status batch_geometry_check(BatchGeometry &g, cudaStream_t s, int *swarm);

// Top-K of every swarm of a batch in one persistent launch (plus the inactive rows): dev_tab[S],
// dev_leaf_prefix[S + 1] (buckets of swarm s are items leaf_prefix[s] ..), dev_part_prefix[S + 1],
// kcap = the largest K.  dev_next is a device counter the call resets.
Status knn_batch_query(const Model &m, const BatchSwarm *dev_tab, const int *dev_leaf_prefix,
                       const long long *dev_part_prefix, int S, long long n_total, int kcap, int *dev_next,
                       const gd_particle *part, int32_t *codes, double *measure, float *kth, cudaStream_t s,
                       long long *launches, const Tuning &tune = Tuning());
// Learned-radius features of every owner (gd_radius.cu).
Status radius_features(const Geometry &g, const Model &m, const gd_particle *part, const float *prev_kth,
                       double total_mass, float *feat, cudaStream_t s);
// colstate_flag: non-finite screen only.
Status state_screen(Geometry &g, const Model &m, const gd_particle *dev_particle, cudaStream_t s);
// Keplerian azimuthal advance of the active particles
Status drift_keplerian(const Model &m, int n, gd_particle *part, double dt, cudaStream_t s);
// col_space_bin
Status space_bin(const Model &m, const gd_particle *dev_particle, int n, int32_t *spatial,
                 cudaStream_t s);

}  // namespace gd
