// C ABI of libgd_b200: handle lifecycle and the entry points declared in include/gd_b200.h.
#include <curand_kernel.h>

#include <climits>
#include <cmath>
#include <cstring>
#include <new>

#include "gd_collide.cuh"
#include "gd_internal.cuh"
#include "gd_transport.cuh"

namespace gd {

// Order-independent 64-bit digest of a neighbour cache: every code mixed with its position, and
// every kept d^2 with its owner (a sum modulo 2^64, so the block order does not matter).
__global__ void k_codes_digest(const int32_t *codes, size_t n_codes, const float *kth, int n,
                               unsigned long long *out) {
    unsigned long long acc = 0;
    const size_t stride = static_cast<size_t>(gridDim.x) * blockDim.x;
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_codes; i += stride) {
        unsigned long long v = static_cast<unsigned long long>(static_cast<unsigned int>(codes[i])) + 1ull;
        v = (v * 0x9E3779B97F4A7C15ull) ^ ((i + 1) * 0xBF58476D1CE4E5B9ull);
        acc += v ^ (v >> 31);
    }
    for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < static_cast<size_t>(n); i += stride) {
        unsigned long long v = static_cast<unsigned long long>(__float_as_uint(kth[i])) + 0x5851F42D4C957F2Dull;
        v = (v * 0x94D049BB133111EBull) ^ ((i + 7) * 0x9E3779B97F4A7C15ull);
        acc += v ^ (v >> 29);
    }
    for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

Status cuda_status(cudaError_t e, const char *what) {
    Status s;
    s.code = (e == cudaErrorMemoryAllocation) ? GD_ERR_OUT_OF_MEMORY : GD_ERR_CUDA;
    s.detail = static_cast<long long>(e);
    s.msg = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError();  // clear a sticky launch error so the handle stays usable
    return s;
}

Model make_model(const gd_config &c) {
    Model m;
    m.G = c.G; m.M_S = c.M_S; m.R_0 = c.R_0; m.S_0 = c.S_0;
    m.n_x = c.n_x; m.n_y = c.n_y; m.n_z = c.n_z;
    m.x_min = c.x_min; m.x_max = c.x_max; m.y_min = c.y_min; m.y_max = c.y_max;
    m.z_min = c.z_min; m.z_max = c.z_max;
    m.sigma_0 = c.sigma_0; m.aspr_0 = c.aspr_0; m.idx_p = c.idx_p; m.idx_q = c.idx_q;
    m.const_nu = c.const_nu; m.nu = c.nu; m.alpha = c.alpha;
    m.code_unit = c.code_unit; m.reynolds_0 = c.reynolds_0; m.m_mol = c.m_mol; m.x_sec = c.x_sec;
    m.half_disk = c.half_disk; m.const_st = c.const_st;
    m.stokes_0 = c.stokes_0; m.rho_0 = c.rho_0;
    m.coag_kernel = c.coag_kernel; m.n_k = c.n_k; m.h_search = c.h_search; m.v_frag = c.v_frag;
    m.col_event_cap = c.col_event_cap;
    m.col_bin_x = c.col_bin_x; m.col_bin_y = c.col_bin_y; m.col_bin_z = c.col_bin_z;
    m.col_bin_s = c.col_bin_s; m.col_bin_min = c.col_bin_min;
    m.col_bath_max = c.col_bath_max; m.col_bath_eps = c.col_bath_eps; m.col_bath_alpha = c.col_bath_alpha;
    m.init_smin = c.init_smin; m.init_smax = c.init_smax;
    m.dim = (c.n_z > 1) ? 3 : 2;
    m.local_groups = ((c.n_x > 1) ? c.col_bin_x : 1) * c.col_bin_y * ((c.n_z > 1) ? c.col_bin_z : 1);
    m.raw_bins = m.local_groups * c.col_bin_s;
    // X_WEDGE (const_defs.cuh:56-57) and _get_image_dist_min (param_grid.cuh:86-89, evaluated on
    // the host as swarm_runtime.cu:334-339 does)
    const float fx_min = static_cast<float>(c.x_min), fx_max = static_cast<float>(c.x_max);
    m.wedge = (c.n_x > 1 && fx_max - fx_min < 6.28318530717958647692f - 1.0e-06f) ? 1 : 0;
    m.morton_images = (c.search == GD_SEARCH_MORTON) ? 1 : 0;
    m.wedge_width = m.morton_images ? fx_max - fx_min : static_cast<float>(c.x_max - c.x_min);
    m.image_dist_min = -1.0f;
    if (m.wedge) {
        const float y_min = static_cast<float>(c.y_min), z_min = static_cast<float>(c.z_min),
                    z_max = static_cast<float>(c.z_max);
        m.image_dist_min = 2.0f * y_min * fminf(sinf(z_min), sinf(z_max)) * fabsf(sinf(0.5f * (fx_max - fx_min)));
    }
    return m;
}

// rngstate_init (src/swarm/rngstate_init.cu:11-18)
__global__ void k_rng_init(curandState *st, int n, unsigned long long seed) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) curand_init(seed, static_cast<unsigned long long>(i), 0ull, &st[i]);
}

// _get_col_uniform (_col_rates.cuh:145-149) replayed on a copy of each state
__global__ void k_rng_uniforms(const curandState *st, int n, int count, double *out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    curandState s = st[i];
    for (int k = 0; k < count; ++k)
        out[static_cast<size_t>(i) * count + k] = fmin(curand_uniform_double(&s), nextafter(1.0, 0.0));
}

}  // namespace gd

struct gd_handle {
    gd_config cfg;
    gd::Model m;
    int n = 0;
    cudaStream_t stream = nullptr;
    gd::Geometry geo;
    gd::DevBuf<int32_t> codes;
    gd::DevBuf<double> measure;
    gd::DevBuf<float> kth;
    gd::DevBuf<int32_t> spatial;
    gd::Collider col;
    gd::Tuning tune;
    bool geom_valid = false;   // col_geom_valid (swarm_runtime.cu:332)
    bool cache_valid = false;
    std::string err;
    long long detail = 0;
    // the Strang step: device clocks and optical depth, and the learned proposal's buffers
    gd::DynState dyn;
    gd::DevBuf<float> step_features, step_radius, step_prev_kth;
    bool step_prev_valid = false;  // step_prev_kth holds the last search's K-th d^2
    gd::DevBuf<int> step_screen;   // first failed screen of the captured steps since the last check
};

static gd_status fail(gd_handle *h, const gd::Status &s) {
    if (h) {
        h->err = s.msg;
        h->detail = s.detail;
    }
    return s.code;
}

static gd_status fail(gd_handle *h, gd_status code, const std::string &msg, long long detail = 0) {
    gd::Status s;
    s.code = code;
    s.msg = msg;
    s.detail = detail;
    return fail(h, s);
}

static gd_status done(gd_handle *h, const gd::Status &s) {
    if (!s) return fail(h, s);
    h->err.clear();
    h->detail = 0;
    return GD_OK;
}

extern "C" {

size_t gd_rng_state_bytes(void) { return sizeof(curandState); }

void gd_config_default(gd_config *c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->G = 1.0; c->M_S = 1.0; c->R_0 = 1.0; c->S_0 = 1.0;
    c->n_x = 100; c->n_y = 100; c->n_z = 1;
    c->x_min = -M_PI; c->x_max = M_PI; c->y_min = 0.5; c->y_max = 1.5;
    c->z_min = 0.5 * M_PI; c->z_max = 0.5 * M_PI;
    c->sigma_0 = 1.0e-2; c->aspr_0 = 0.05; c->idx_p = -1.0; c->idx_q = -0.4;
    c->const_nu = 0; c->nu = 1.0e-5; c->alpha = 1.0e-4;
    c->code_unit = 0; c->reynolds_0 = 1.0e8; c->m_mol = 2.3 * 1.66054e-24; c->x_sec = 2.0e-15;
    c->half_disk = 0; c->const_st = 0;
    c->stokes_0 = 1.0e-3; c->rho_0 = 1.0;
    c->coag_kernel = GD_KERNEL_CONSTANT; c->n_k = 200; c->h_search = 1.0; c->v_frag = 1.0;
    c->col_event_cap = 32;
    c->col_bin_x = 8; c->col_bin_y = 4; c->col_bin_z = 2; c->col_bin_s = 8; c->col_bin_min = 64;
    c->col_bath_max = 0.05; c->col_bath_eps = 0.02; c->col_bath_alpha = 1.0e-3;
    c->init_smin = 1.0; c->init_smax = 1.0;
    c->search = GD_SEARCH_KDTREE;
    c->morton_leaf_target = 128; c->morton_max_level = 20;
}

static std::string validate(const gd_config &c, int n) {
    if (n <= 0) return "particle count must be positive";
    if (static_cast<long long>(n) * 3 > INT_MAX) return "particle count too large for packed neighbour codes";
    if (c.n_k < 1 || c.n_k > gd::kMaxK) return "n_k must be in 1..256";
    if (c.n_x < 1 || c.n_y < 1 || c.n_z < 1) return "grid counts must be positive";
    if (!(c.y_max > c.y_min) || !(c.y_min >= 0)) return "invalid radial domain";
    if (c.coag_kernel < 0 || c.coag_kernel > 3) return "coag_kernel must be 0..3";
    if (c.col_bin_x < 1 || c.col_bin_y < 1 || c.col_bin_z < 1 || c.col_bin_s < 1) return "controller bins must be positive";
    if (c.search != GD_SEARCH_KDTREE && c.search != GD_SEARCH_MORTON) return "unknown search";
    // the index addresses at most 2^30 sites (its leaf slots times 32 in int); a wedge has three per
    // particle
    if (gd::make_model(c).wedge && 3LL * n > (1LL << 30))
        return "a wedge's three sites per particle exceed the 2^30 sites the index addresses";
    return std::string();
}

gd_status gd_create(const gd_config *cfg, int n_p, gd_handle **out) {
    if (!cfg || !out) return GD_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    std::string why = validate(*cfg, n_p);
    if (!why.empty()) return GD_ERR_INVALID_ARGUMENT;
    gd_handle *h = new (std::nothrow) gd_handle();
    if (!h) return GD_ERR_OUT_OF_MEMORY;
    h->cfg = *cfg;
    h->m = gd::make_model(*cfg);
    h->n = n_p;
    gd::Status s = gd::geometry_alloc(h->geo, h->m, n_p);
    cudaError_t e = cudaSuccess;
    if (s) e = h->codes.alloc(static_cast<size_t>(n_p) * cfg->n_k);
    if (s && e == cudaSuccess) e = h->measure.alloc(n_p);
    if (s && e == cudaSuccess) e = h->kth.alloc(n_p);
    if (s && e == cudaSuccess) e = h->spatial.alloc(n_p);
    if (s && e != cudaSuccess) s = gd::cuda_status(e, "allocate neighbour cache");
    if (s) s = gd::collider_alloc(h->col, h->m, n_p);
    if (!s) {
        gd_status code = s.code;
        delete h;
        return code;
    }
    *out = h;
    return GD_OK;
}

void gd_destroy(gd_handle *h) { delete h; }

gd_status gd_set_stream(gd_handle *h, void *stream) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    h->stream = static_cast<cudaStream_t>(stream);
    return GD_OK;
}

size_t gd_last_error(const gd_handle *h, char *buf, size_t len) {
    if (!h) return 0;
    if (buf && len) {
        size_t k = h->err.size() < len - 1 ? h->err.size() : len - 1;
        std::memcpy(buf, h->err.data(), k);
        buf[k] = '\0';
    }
    return h->err.size();
}

long long gd_error_detail(const gd_handle *h) { return h ? h->detail : 0; }

gd_status gd_rng_init(void *dev_rng, int n, unsigned long long seed, void *stream) {
    if (!dev_rng || n < 0 || !gd::aligned_to(dev_rng, alignof(curandState))) return GD_ERR_INVALID_ARGUMENT;
    if (n == 0) return GD_OK;
    gd::k_rng_init<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<curandState *>(dev_rng), n, seed);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}

gd_status gd_geometry_build(gd_handle *h, const gd_particle *dev_particle) {
    if (!h || !dev_particle) return fail(h, GD_ERR_INVALID_ARGUMENT, "null handle or particle pointer");
    if (!gd::aligned_to(dev_particle, 8)) return fail(h, GD_ERR_INVALID_ARGUMENT, "misaligned particle pointer");
    h->geom_valid = false;
    h->cache_valid = false;
    h->geo.sort_bits = h->tune.sort_bits;
    gd::Status s = gd::geometry_build(h->geo, h->m, dev_particle, h->stream);
    if (s) h->geom_valid = true;
    return done(h, s);
}

static bool tuning_ok(const gd::Model &m, const gd_tuning &t) {
    const int full = 21 * m.dim;
    return t.warps_per_block >= 0 && t.warps_per_block <= 32 && t.prescan >= 0 && t.prescan <= 8 &&
           (t.walk_breadth_first == 0 || t.walk_breadth_first == 1) &&
           (t.sort_bits == 0 || (t.sort_bits >= 16 * m.dim && t.sort_bits <= full)) &&
           (t.range_query == 0 || t.range_query == 1);
}

static gd::Tuning to_tuning(const gd_tuning &t) {
    gd::Tuning u;
    u.warps = t.warps_per_block;
    u.prescan = t.prescan;
    u.bfs = t.walk_breadth_first;
    u.sort_bits = t.sort_bits;
    u.range = t.range_query;
    return u;
}

static gd_tuning from_tuning(const gd::Tuning &u) {
    gd_tuning t;
    t.warps_per_block = u.warps;
    t.prescan = u.prescan;
    t.walk_breadth_first = u.bfs;
    t.sort_bits = u.sort_bits;
    t.range_query = u.range;
    return t;
}

gd_status gd_get_tuning(const gd_handle *h, gd_tuning *out) {
    if (!h || !out) return GD_ERR_INVALID_ARGUMENT;
    *out = from_tuning(h->tune);
    return GD_OK;
}

gd_status gd_set_tuning(gd_handle *h, const gd_tuning *t) {
    if (!h || !t) return GD_ERR_INVALID_ARGUMENT;
    if (!tuning_ok(h->m, *t)) return fail(h, GD_ERR_INVALID_ARGUMENT, "tuning out of range");
    if (t->warps_per_block > 0 && gd::knn_block_warps(h->m.n_k, to_tuning(*t), nullptr) == 0)
        return fail(h, GD_ERR_INVALID_ARGUMENT, "warps per block do not fit in shared memory");
    h->tune = to_tuning(*t);
    return GD_OK;
}

gd_status gd_autotune(gd_handle *h, const gd_particle *dev_particle, const float *dev_radius, int tune_sort,
                      gd_tuning *out_best, double *out_ms) {
    if (!h || !dev_particle) return fail(h, GD_ERR_INVALID_ARGUMENT, "null handle or particle pointer");
    if (!gd::aligned_to(dev_particle, 8)) return fail(h, GD_ERR_INVALID_ARGUMENT, "misaligned particle pointer");
    const bool deferred = h->geo.deferred_check;
    h->geo.deferred_check = false;  // the tuner screens its input once, eagerly
    cudaEvent_t a = nullptr, b = nullptr;
    gd::DevBuf<unsigned long long> digest;
    gd::Status st;
    auto cuda = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && st) st = gd::cuda_status(e, what);
        return static_cast<bool>(st);
    };
    cuda(digest.alloc(1), "autotune digest");
    if (st) cuda(cudaEventCreate(&a), "autotune event");
    if (st) cuda(cudaEventCreate(&b), "autotune event");
    // one timed run (best of three): optional geometry build, then the query; returns ms and a
    // digest of the codes and kept d^2, which every tuning must reproduce bit for bit
    auto run = [&](const gd::Tuning &t, bool build, float &ms, unsigned long long &dig) {
        ms = 1e30f;
        for (int rep = 0; rep < 3 && st; ++rep) {
            cuda(cudaEventRecord(a, h->stream), "autotune record");
            if (st && build) {
                h->geo.sort_bits = t.sort_bits;
                st = gd::geometry_build(h->geo, h->m, dev_particle, h->stream);
            }
            if (st)
                st = gd::knn_query(h->geo, h->m, dev_particle, h->codes.ptr, h->measure.ptr, h->kth.ptr, h->stream,
                                   dev_radius, nullptr, t);
            if (st) cuda(cudaEventRecord(b, h->stream), "autotune record");
            if (st) cuda(cudaEventSynchronize(b), "autotune run");
            float e = 0.f;
            if (st) cuda(cudaEventElapsedTime(&e, a, b), "autotune time");
            if (st && e < ms) ms = e;
        }
        if (!st) return;
        cuda(cudaMemsetAsync(digest.ptr, 0, sizeof(unsigned long long), h->stream), "autotune digest");
        gd::k_codes_digest<<<592, 256, 0, h->stream>>>(h->codes.ptr, static_cast<size_t>(h->n) * h->m.n_k, h->kth.ptr,
                                                       h->n, digest.ptr);
        cuda(cudaGetLastError(), "autotune digest");
        if (st) cuda(cudaMemcpy(&dig, digest.ptr, sizeof(dig), cudaMemcpyDeviceToHost), "autotune digest");
    };
    gd::Tuning best = h->tune;
    float best_ms = 0.f, ms = 0.f;
    unsigned long long ref = 0, dig = 0;
    run(best, true, best_ms, ref);
    auto consider = [&](const gd::Tuning &t, bool build) {
        if (!st) return;
        run(t, build, ms, dig);
        if (!st) return;
        if (dig != ref) {
            st = gd::Status{GD_ERR_CONTROLLER, "autotune: a tuning changed the neighbour lists", 0};
            return;
        }
        // a setting must beat the current one by 2%: near-equal settings differ by about that much
        // from one timing to the next, and a pick made on noise costs the replayed step as much
        if (ms < 0.98f * best_ms) {
            best_ms = ms;
            best = t;
        }
    };
    if (st && tune_sort) {
        // sort order: all Morton bits, or the top 16 per axis (fewer radix passes, coarser buckets)
        for (int sb : {0, 16 * h->m.dim}) {
            if (sb == best.sort_bits) continue;
            gd::Tuning t = best;
            t.sort_bits = sb;
            consider(t, true);
        }
    }
    if (st) {
        // the query alone from here on, on the geometry of the chosen sort order
        const gd::Tuning base = best;
        run(base, true, best_ms, dig);
        if (st && dig != ref) st = gd::Status{GD_ERR_CONTROLLER, "autotune: a tuning changed the neighbour lists", 0};
        if (st) run(base, false, best_ms, dig);
    }
    for (int bfs = 1; bfs >= 0 && st; --bfs)
        for (int pre = 1; pre <= 3 && st; ++pre) {
            gd::Tuning t = best;
            t.bfs = bfs;
            t.prescan = pre;
            if (t.bfs == best.bfs && t.prescan == best.prescan) continue;
            consider(t, false);
        }
    if (st && dev_radius && gd::knn_range_eligible(h->m, h->m.n_k)) {
        // the radius-bounded query: warp-per-owner range query or per-lane heaps
        gd::Tuning t = best;
        t.range = best.range ? 0 : 1;
        consider(t, false);
    }
    for (int w : {1, 2, 4, 8}) {
        if (!st) break;
        gd::Tuning t = best;
        t.warps = w;
        if (gd::knn_block_warps(h->m.n_k, t, nullptr) == 0 || t.warps == best.warps) continue;
        consider(t, false);
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    h->geo.deferred_check = deferred;
    if (!st) {
        h->geom_valid = false;
        h->cache_valid = false;
        return fail(h, st);
    }
    // leave the handle built and cached with the chosen tuning
    h->tune = best;
    h->geo.sort_bits = best.sort_bits;
    gd::Status s2 = gd::geometry_build(h->geo, h->m, dev_particle, h->stream);
    if (s2) s2 = gd::knn_query(h->geo, h->m, dev_particle, h->codes.ptr, h->measure.ptr, h->kth.ptr, h->stream,
                               dev_radius, nullptr, best);
    h->geom_valid = static_cast<bool>(s2);
    h->cache_valid = static_cast<bool>(s2) && !dev_radius;
    h->col.local_geometry_valid = false;
    if (!s2) return fail(h, s2);
    if (out_best) *out_best = from_tuning(best);
    if (out_ms) *out_ms = best_ms;
    return done(h, s2);
}

gd_status gd_set_deferred_checks(gd_handle *h, int on) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    h->geo.deferred_check = on != 0;
    return GD_OK;
}

gd_status gd_check_geometry(gd_handle *h) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    if (!h->geo.sorted_key) return fail(h, GD_ERR_NOT_READY, "gd_check_geometry called before gd_geometry_build");
    // the screen of the most recent build on the stream, eager or replayed from a captured graph
    gd::Status s = gd::geometry_check(h->geo, h->stream);
    h->geom_valid = static_cast<bool>(s);
    if (!s) h->cache_valid = false;
    return done(h, s);
}

gd_status gd_knn(gd_handle *h, const gd_particle *dev_particle, int32_t *dev_codes, double *dev_measure,
                 float *dev_kth_d2) {
    if (!h || !dev_particle) return fail(h, GD_ERR_INVALID_ARGUMENT, "null handle or particle pointer");
    if (!gd::aligned_to(dev_particle, 8)) return fail(h, GD_ERR_INVALID_ARGUMENT, "misaligned particle pointer");
    if (!h->geom_valid) return fail(h, GD_ERR_NOT_READY, "gd_knn called before gd_geometry_build");
    const bool own = !dev_codes && !dev_measure;
    int32_t *codes = dev_codes ? dev_codes : h->codes.ptr;
    double *measure = dev_measure ? dev_measure : h->measure.ptr;
    float *kth = dev_kth_d2 ? dev_kth_d2 : h->kth.ptr;
    gd::Status s = gd::knn_query(h->geo, h->m, dev_particle, codes, measure, kth, h->stream, nullptr, nullptr, h->tune);
    if (s && own) {
        h->cache_valid = true;
        h->col.local_geometry_valid = false;
    }
    return done(h, s);
}

gd_status gd_knn_bounded(gd_handle *h, const gd_particle *dev_particle, const float *dev_radius, int32_t *dev_codes,
                         double *dev_measure, float *dev_kth_d2, unsigned long long *dev_stats) {
    if (!h || !dev_particle) return fail(h, GD_ERR_INVALID_ARGUMENT, "null handle or particle pointer");
    if (!gd::aligned_to(dev_particle, 8)) return fail(h, GD_ERR_INVALID_ARGUMENT, "misaligned particle pointer");
    if (!h->geom_valid) return fail(h, GD_ERR_NOT_READY, "gd_knn_bounded called before gd_geometry_build");
    const bool own = !dev_codes && !dev_measure;
    int32_t *codes = dev_codes ? dev_codes : h->codes.ptr;
    double *measure = dev_measure ? dev_measure : h->measure.ptr;
    float *kth = dev_kth_d2 ? dev_kth_d2 : h->kth.ptr;
    gd::Status s = gd::knn_query(h->geo, h->m, dev_particle, codes, measure, kth, h->stream, dev_radius, dev_stats,
                                 h->tune);
    if (s && own) {
        h->cache_valid = true;
        h->col.local_geometry_valid = false;
    }
    return done(h, s);
}

gd_status gd_pair_rates(gd_handle *h, const gd_particle *dev_particle, const int32_t *dev_owner_ids, int count,
                        double total_dust_mass, double *dev_out) {
    if (!h || !dev_particle || !dev_owner_ids || !dev_out || count < 0 || !(total_dust_mass > 0))
        return fail(h, GD_ERR_INVALID_ARGUMENT, "null pointer, negative count or non-positive mass");
    if (!h->cache_valid) return fail(h, GD_ERR_NOT_READY, "gd_pair_rates needs a neighbour cache");
    return done(h, gd::pair_rates(h->m, dev_owner_ids, count, dev_particle, h->codes.ptr, h->measure.ptr,
                                  h->geo.active.ptr, total_dust_mass, h->n, dev_out, h->stream));
}

gd_status gd_bath_rates(gd_handle *h, const gd_particle *dev_particle, double total_dust_mass, double *dev_cached4) {
    if (!h || !dev_particle || !dev_cached4) return fail(h, GD_ERR_INVALID_ARGUMENT, "null pointer");
    if (!gd::aligned_to(dev_particle, 8) || !gd::aligned_to(dev_cached4, 8))
        return fail(h, GD_ERR_INVALID_ARGUMENT, "misaligned particle or output pointer");
    if (!h->cache_valid) return fail(h, GD_ERR_NOT_READY, "gd_bath_rates needs a neighbour cache");
    int launches = 0;
    gd::Status s = gd::bath_rates(h->col, h->m, h->n, dev_particle, h->codes.ptr, h->measure.ptr, h->geo.active.ptr,
                                  total_dust_mass, dev_cached4, &launches, h->stream);
    h->col.launches += launches;
    return done(h, s);
}

gd_status gd_bath_chain(gd_handle *h, gd_particle *dev_particle, void *dev_rngstate, double total_dust_mass,
                        double bath, unsigned long long *events) {
    if (!h || !dev_particle || !dev_rngstate) return fail(h, GD_ERR_INVALID_ARGUMENT, "null pointer");
    if (!gd::aligned_to(dev_particle, 8) || !gd::aligned_to(dev_rngstate, 8))
        return fail(h, GD_ERR_INVALID_ARGUMENT, "misaligned particle or RNG pointer");
    if (!h->cache_valid) return fail(h, GD_ERR_NOT_READY, "gd_bath_chain needs a neighbour cache");
    int launches = 0;
    gd::Status s = gd::bath_chain(h->col, h->m, h->n, dev_particle, static_cast<curandState *>(dev_rngstate),
                                  h->codes.ptr, h->measure.ptr, h->geo.active.ptr, total_dust_mass, bath, events,
                                  &launches, h->stream);
    h->col.launches += launches;
    return done(h, s);
}

gd_status gd_drift_keplerian(gd_handle *h, gd_particle *dev_particle, double dt) {
    if (!h || !dev_particle || !std::isfinite(dt)) return fail(h, GD_ERR_INVALID_ARGUMENT, "null pointer or bad dt");
    h->geo.launches += 1;
    gd::Status s = gd::drift_keplerian(h->m, h->n, dev_particle, dt, h->stream);
    h->geom_valid = false;
    h->cache_valid = false;
    h->col.local_geometry_valid = false;
    return done(h, s);
}

gd_status gd_radius_features(gd_handle *h, const gd_particle *dev_particle, const float *dev_prev_kth_d2,
                             double total_mass, float *dev_features) {
    if (!h || !dev_particle || !dev_features || !(total_mass > 0))
        return fail(h, GD_ERR_INVALID_ARGUMENT, "null pointer or non-positive mass");
    if (!h->geom_valid) return fail(h, GD_ERR_NOT_READY, "gd_radius_features called before gd_geometry_build");
    return done(h, gd::radius_features(h->geo, h->m, dev_particle, dev_prev_kth_d2, total_mass, dev_features,
                                       h->stream));
}

gd_status gd_get_sites(gd_handle *h, float *dev_site4, float *dev_q, unsigned char *dev_active) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    if (!h->geom_valid) return fail(h, GD_ERR_NOT_READY, "geometry not built");
    cudaError_t e = cudaSuccess;
    if (dev_site4)
        e = cudaMemcpyAsync(dev_site4, h->geo.site.ptr, sizeof(float4) * h->geo.n_sites, cudaMemcpyDeviceToDevice,
                            h->stream);
    if (e == cudaSuccess && dev_q)
        e = cudaMemcpyAsync(dev_q, h->geo.q.ptr, sizeof(float) * h->n, cudaMemcpyDeviceToDevice, h->stream);
    if (e == cudaSuccess && dev_active)
        e = cudaMemcpyAsync(dev_active, h->geo.active.ptr, h->n, cudaMemcpyDeviceToDevice, h->stream);
    if (e != cudaSuccess) return fail(h, gd::cuda_status(e, "copy sites"));
    return GD_OK;
}

int gd_site_count(const gd_handle *h) { return h ? h->geo.n_sites : 0; }

gd_status gd_wedge_info(const gd_config *cfg, int *wedge, float *width, float *image_dist_min) {
    if (!cfg) return GD_ERR_INVALID_ARGUMENT;
    const gd::Model m = gd::make_model(*cfg);
    if (wedge) *wedge = m.wedge;
    if (width) *width = m.wedge ? m.wedge_width : 0.0f;
    if (image_dist_min) *image_dist_min = m.image_dist_min;
    return GD_OK;
}

gd_status gd_get_cache(gd_handle *h, int32_t *dev_codes, double *dev_measure) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    if (!h->cache_valid) return fail(h, GD_ERR_NOT_READY, "neighbour cache not built");
    cudaError_t e = cudaSuccess;
    if (dev_codes)
        e = cudaMemcpyAsync(dev_codes, h->codes.ptr, sizeof(int32_t) * h->codes.n, cudaMemcpyDeviceToDevice, h->stream);
    if (e == cudaSuccess && dev_measure)
        e = cudaMemcpyAsync(dev_measure, h->measure.ptr, sizeof(double) * h->n, cudaMemcpyDeviceToDevice, h->stream);
    if (e != cudaSuccess) return fail(h, gd::cuda_status(e, "copy neighbour cache"));
    return GD_OK;
}

gd_status gd_set_cache(gd_handle *h, const int32_t *dev_codes, const double *dev_measure) {
    if (!h || !dev_codes || !dev_measure) return fail(h, GD_ERR_INVALID_ARGUMENT, "null cache pointer");
    cudaError_t e = cudaMemcpyAsync(h->codes.ptr, dev_codes, sizeof(int32_t) * h->codes.n,
                                    cudaMemcpyDeviceToDevice, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h->measure.ptr, dev_measure, sizeof(double) * h->n, cudaMemcpyDeviceToDevice, h->stream);
    if (e != cudaSuccess) return fail(h, gd::cuda_status(e, "set neighbour cache"));
    h->cache_valid = true;
    h->col.local_geometry_valid = false;
    return GD_OK;
}

gd_status gd_space_bin(gd_handle *h, const gd_particle *dev_particle, int32_t *dev_spatial) {
    if (!h || !dev_particle) return fail(h, GD_ERR_INVALID_ARGUMENT, "null pointer");
    if (!gd::aligned_to(dev_particle, 8)) return fail(h, GD_ERR_INVALID_ARGUMENT, "misaligned particle pointer");
    return done(h, gd::space_bin(h->m, dev_particle, h->n, dev_spatial ? dev_spatial : h->spatial.ptr, h->stream));
}

gd_status gd_invalidate_geometry(gd_handle *h) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    h->geom_valid = false;
    h->cache_valid = false;
    h->col.local_geometry_valid = false;
    return GD_OK;
}

gd_status gd_reset_controller(gd_handle *h) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    return done(h, gd::collider_reset_state(h->col, h->stream));
}

gd_status gd_check_operator(gd_handle *h) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    return done(h, gd::collider_check(h->col, h->stream));
}

gd_status gd_set_diagnostics(gd_handle *h, int on) {
    if (!h || (on != 0 && on != 1)) return GD_ERR_INVALID_ARGUMENT;
    if (on) {
        gd::Status s = gd::collider_enable_log(h->col);
        if (!s) return fail(h, s);
    }
    h->col.diagnostics = on != 0;
    return GD_OK;
}

gd_status gd_operator_phase_seconds(const gd_handle *h, double *out4) {
    if (!h || !out4) return GD_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 4; ++k) out4[k] = h->col.phase_seconds[k];
    return GD_OK;
}

size_t gd_operator_log(const gd_handle *h, char *buf, size_t len) {
    if (!h) return 0;
    const std::string &text = h->col.operator_log;
    if (buf && len) {
        const size_t k = text.size() < len - 1 ? text.size() : len - 1;
        std::memcpy(buf, text.data(), k);
        buf[k] = '\0';
    }
    return text.size();
}

gd_status gd_event_totals(gd_handle *h, unsigned long long *counts, double *log_mass) {
    if (!h || !counts || !log_mass) return GD_ERR_INVALID_ARGUMENT;
    if (!h->col.diagnostics) return fail(h, GD_ERR_NOT_READY, "diagnostics are off (gd_set_diagnostics)");
    if (cudaMemcpyAsync(counts, h->col.event_count.ptr, sizeof(unsigned long long) * gd::kEventCategories,
                        cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaMemcpyAsync(log_mass, h->col.event_log_mass.ptr, sizeof(double) * gd::kEventCategories,
                        cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess)
        return fail(h, GD_ERR_CUDA, "copy of the event totals");
    return GD_OK;
}

size_t gd_controller_summary(const gd_handle *h, char *buf, size_t len) {
    if (!h) return 0;
    const std::string text = h->col.summary.json();
    if (buf && len) {
        const size_t k = text.size() < len - 1 ? text.size() : len - 1;
        std::memcpy(buf, text.data(), k);
        buf[k] = '\0';
    }
    return text.size();
}

gd_status gd_collision_operator(gd_handle *h, gd_particle *dev_particle, void *dev_rng, double duration,
                                double total_dust_mass) {
    if (!h || !dev_particle || !dev_rng) return fail(h, GD_ERR_INVALID_ARGUMENT, "null pointer");
    if (!gd::aligned_to(dev_particle, 8) || !gd::aligned_to(dev_rng, alignof(curandState)))
        return fail(h, GD_ERR_INVALID_ARGUMENT, "misaligned particle or RNG pointer");
    if (!h->cache_valid) return fail(h, GD_ERR_NOT_READY, "collision operator needs a neighbour cache");
    gd::Status s = gd::collision_operator(h->col, h->m, h->n, dev_particle, static_cast<curandState *>(dev_rng),
                                          h->codes.ptr, h->measure.ptr, h->geo.active.ptr, h->spatial.ptr,
                                          duration, total_dust_mass, h->stream);
    return done(h, s);
}

gd_status gd_evolve_collisions(gd_handle *h, gd_particle *dev_particle, void *dev_rng, double duration,
                               double total_dust_mass) {
    if (!h || !dev_particle || !dev_rng) return fail(h, GD_ERR_INVALID_ARGUMENT, "null pointer");
    if (!gd::aligned_to(dev_particle, 8) || !gd::aligned_to(dev_rng, alignof(curandState)))
        return fail(h, GD_ERR_INVALID_ARGUMENT, "misaligned particle or RNG pointer");
    gd::Status s;
    if (h->geom_valid && h->cache_valid) {
        s = gd::state_screen(h->geo, h->m, dev_particle, h->stream);
    } else {
        h->geom_valid = false;
        h->cache_valid = false;
        h->geo.sort_bits = h->tune.sort_bits;
        s = gd::geometry_build(h->geo, h->m, dev_particle, h->stream);
        if (s) {
            h->geom_valid = true;
            s = gd::knn_query(h->geo, h->m, dev_particle, h->codes.ptr, h->measure.ptr, h->kth.ptr, h->stream, nullptr,
                              nullptr, h->tune);
        }
        if (s) s = gd::space_bin(h->m, dev_particle, h->n, h->spatial.ptr, h->stream);
        if (s) {
            h->cache_valid = true;
            h->col.local_geometry_valid = false;
        }
    }
    if (!s) return fail(h, s);
    return gd_collision_operator(h, dev_particle, dev_rng, duration, total_dust_mass);
}

long long gd_launch_count(const gd_handle *h) { return h ? h->geo.launches + h->col.launches : 0; }

gd_status gd_rng_uniforms(const void *dev_rng, int n, int count, double *dev_out, void *stream) {
    if (!dev_rng || !dev_out || n < 0 || count < 0 || !gd::aligned_to(dev_rng, alignof(curandState)) ||
        !gd::aligned_to(dev_out, 8))
        return GD_ERR_INVALID_ARGUMENT;
    if (n == 0 || count == 0) return GD_OK;
    gd::k_rng_uniforms<<<(n + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const curandState *>(dev_rng), n, count, dev_out);
    return cudaGetLastError() == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}

gd_status gd_get_owner_state(gd_handle *h, double *dev_cached4, double *dev_time, int32_t *dev_events,
                             double *dev_size_old, double *dev_numr_old) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    const size_t n = static_cast<size_t>(h->n);
    cudaError_t e = cudaSuccess;
    auto cp = [&](void *dst, const void *src, size_t bytes) {
        if (dst && e == cudaSuccess) e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, h->stream);
    };
    cp(dev_cached4, h->col.cached.ptr, sizeof(double) * 4 * n);
    cp(dev_time, h->col.time.ptr, sizeof(double) * n);
    cp(dev_events, h->col.events.ptr, sizeof(int) * n);
    cp(dev_size_old, h->col.size_old.ptr, sizeof(double) * n);
    cp(dev_numr_old, h->col.numr_old.ptr, sizeof(double) * n);
    if (e != cudaSuccess) return fail(h, gd::cuda_status(e, "copy owner state"));
    return GD_OK;
}

gd_status gd_last_operator_stats(const gd_handle *h, gd_operator_stats *out) {
    if (!h || !out) return GD_ERR_INVALID_ARGUMENT;
    *out = h->col.stats;
    return GD_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// gd_knn_static: the neighbour search (site init + Morton radix sort + bucket tree + exact top-K)
// for swarms of at most kStaticParticles particles, with every scratch array carved from one fixed
// device array instead of a handle's allocations.  It serves callers that cannot allocate device
// memory while they run: hosts that hand the whole device to their own memory pool at start-up and
// allow no allocation outside it, and time loops that cannot afford the device-wide
// synchronisation cudaMalloc/cudaFree can imply.  The build and query kernels are the ones
// gd_geometry_build/gd_knn run; only where their scratch lives differs.
// ---------------------------------------------------------------------------------------------
#include <mutex>

namespace gd {
namespace {

constexpr int kStaticParticles = 1 << 16;  // maximum n_p of gd_knn_static
constexpr int kStaticSort = (kStaticParticles + kRadixTile - 1) / kRadixTile * kRadixTile;
constexpr int kStaticLeafSlots = kStaticParticles / kLeaf;  // a power of two: 2048
static_assert((kStaticLeafSlots & (kStaticLeafSlots - 1)) == 0, "leaf slots must be a power of two");

constexpr size_t round256(size_t b) { return (b + 255) / 256 * 256; }

// Fixed layout of the scratch at the maximum size; a smaller swarm uses a prefix of each array.
constexpr size_t kOffSite = 0;
constexpr size_t kOffQ = kOffSite + round256(sizeof(float4) * kStaticParticles);
constexpr size_t kOffActive = kOffQ + round256(sizeof(float) * kStaticParticles);
constexpr size_t kOffKeyA = kOffActive + round256(kStaticParticles);
constexpr size_t kOffKeyB = kOffKeyA + round256(sizeof(unsigned long long) * kStaticSort);
constexpr size_t kOffValA = kOffKeyB + round256(sizeof(unsigned long long) * kStaticSort);
constexpr size_t kOffValB = kOffValA + round256(sizeof(unsigned int) * kStaticSort);
constexpr size_t kOffHist = kOffValB + round256(sizeof(unsigned int) * kStaticSort);
constexpr size_t kOffSorted = kOffHist + round256(sizeof(unsigned int) * 256 * (kStaticSort / kRadixTile));
constexpr size_t kOffNodeLo = kOffSorted + round256(sizeof(float4) * kStaticLeafSlots * kLeaf);
constexpr size_t kOffNodeHi = kOffNodeLo + round256(sizeof(float4) * 2 * kStaticLeafSlots);
constexpr size_t kOffSubLo = kOffNodeHi + round256(sizeof(float4) * 2 * kStaticLeafSlots);
constexpr size_t kOffSubHi = kOffSubLo + round256(sizeof(float4) * kStaticLeafSlots * kSubs);
constexpr size_t kOffCounters = kOffSubHi + round256(sizeof(float4) * kStaticLeafSlots * kSubs);
constexpr size_t kStaticBytes = kOffCounters + round256(sizeof(int) * 4);  // 4,407,552 bytes
static_assert(kStaticBytes == 4407552, "scratch size stated in gd_b200.h");
// The histogram region holds the [digit][tile] counts of one scan chunk and no chunk totals:
// geometry_build's chunked scan needs a chunk-total area only when the counts span more than one
// chunk, which this bound rules out for every swarm that fits the scratch.
static_assert(256 * (kStaticSort / kRadixTile) <= kScanChunk,
              "raising kStaticParticles past one scan chunk needs room for the chunk totals");

constexpr int kStaticMaxDevices = 64;

}  // namespace

// The scratch.  Every device that loads this library holds it until the process exits.  In host
// code this name is only a host-side stand-in: kernels receive the device address resolved below.
static __device__ __align__(256) unsigned char g_knn_scratch[kStaticBytes];

namespace {

std::mutex g_scratch_mu;
unsigned char *g_scratch_addr[kStaticMaxDevices] = {};

// Device address of g_knn_scratch on the current device, resolved once per device with that device
// current (the first call on a device may load this library's device code there).  The address is
// kept for the life of the process: after the host resets a device (cudaDeviceReset) this entry
// point must not be called on it again.
Status static_scratch(unsigned char **out) {
    int dev = -1;
    GD_TRY_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kStaticMaxDevices) {
        Status st;
        st.code = GD_ERR_CAPACITY;
        st.detail = dev;
        st.msg = "gd_knn_static supports device ordinals below 64";
        return st;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_knn_scratch);
        if (e != cudaSuccess) return cuda_status(e, "resolve the gd_knn_static scratch");
        g_scratch_addr[dev] = static_cast<unsigned char *>(p);
    }
    *out = g_scratch_addr[dev];
    return Status::ok();
}

// Points a Geometry's buffers into the fixed scratch and detaches them again on scope exit, so
// that the DevBuf destructors never free memory they do not own.
struct BorrowedGeometry {
    Geometry g;
    BorrowedGeometry(const Model &m, int n, unsigned char *base) {
        g.n = n;
        g.n_sites = n;  // gd_knn_static rejects wedges
        g.n_sort = (n + kRadixTile - 1) / kRadixTile * kRadixTile;
        const int leaves = (n + kLeaf - 1) / kLeaf;
        int slots = 1;
        while (slots < leaves) slots <<= 1;
        g.leaf_slots = slots;
        g.key_bits = 21 * m.dim;
        bind(g.site, base + kOffSite, n);
        bind(g.q, base + kOffQ, n);
        bind(g.active, base + kOffActive, n);
        bind(g.key_a, base + kOffKeyA, g.n_sort);
        bind(g.key_b, base + kOffKeyB, g.n_sort);
        bind(g.val_a, base + kOffValA, g.n_sort);
        bind(g.val_b, base + kOffValB, g.n_sort);
        bind(g.hist, base + kOffHist, static_cast<size_t>(256) * (g.n_sort / kRadixTile));
        bind(g.sorted, base + kOffSorted, static_cast<size_t>(g.leaf_slots) * kLeaf);
        bind(g.node_lo, base + kOffNodeLo, 2 * static_cast<size_t>(g.leaf_slots));
        bind(g.node_hi, base + kOffNodeHi, 2 * static_cast<size_t>(g.leaf_slots));
        bind(g.sub_lo, base + kOffSubLo, static_cast<size_t>(g.leaf_slots) * kSubs);
        bind(g.sub_hi, base + kOffSubHi, static_cast<size_t>(g.leaf_slots) * kSubs);
        bind(g.counters, base + kOffCounters, 4);
    }
    ~BorrowedGeometry() {
        detach(g.site); detach(g.q); detach(g.active);
        detach(g.key_a); detach(g.key_b); detach(g.val_a); detach(g.val_b); detach(g.hist);
        detach(g.sorted); detach(g.node_lo); detach(g.node_hi); detach(g.sub_lo); detach(g.sub_hi);
        detach(g.counters);
    }
    BorrowedGeometry(const BorrowedGeometry &) = delete;
    BorrowedGeometry &operator=(const BorrowedGeometry &) = delete;

  private:
    template <typename T>
    static void bind(DevBuf<T> &b, unsigned char *at, size_t count) {
        b.ptr = reinterpret_cast<T *>(at);
        b.n = count;
    }
    template <typename T>
    static void detach(DevBuf<T> &b) {
        b.ptr = nullptr;
        b.n = 0;
    }
};

gd_status static_fail(const Status &s, long long *detail, char *msg, size_t msg_len) {
    if (detail) *detail = s.detail;
    if (msg && msg_len) {
        const size_t k = s.msg.size() < msg_len - 1 ? s.msg.size() : msg_len - 1;
        std::memcpy(msg, s.msg.data(), k);
        msg[k] = '\0';
    }
    return s.code;
}

}  // namespace
}  // namespace gd

extern "C" gd_status gd_knn_static(const gd_config *cfg, const gd_particle *dev_particle, int n_p,
                                   int32_t *dev_codes, double *dev_measure, float *dev_kth_d2, void *stream,
                                   long long *detail, char *msg, size_t msg_len) {
    using gd::Status;
    if (detail) *detail = 0;
    if (msg && msg_len) msg[0] = '\0';
    Status st;
    if (!cfg || !dev_particle || !dev_codes || !dev_measure || !dev_kth_d2) {
        st.code = GD_ERR_INVALID_ARGUMENT;
        st.msg = "gd_knn_static: null configuration, particle or output pointer";
        return gd::static_fail(st, detail, msg, msg_len);
    }
    if (n_p > gd::kStaticParticles) {
        st.code = GD_ERR_CAPACITY;
        st.detail = n_p;
        st.msg = "gd_knn_static: " + std::to_string(n_p) + " particles exceed its fixed scratch of " +
                 std::to_string(gd::kStaticParticles) + " particles; use gd_create/gd_geometry_build/gd_knn";
        return gd::static_fail(st, detail, msg, msg_len);
    }
    std::string why = validate(*cfg, n_p);
    if (why.empty() && gd::make_model(*cfg).wedge)
        why = "azimuthal wedges (three sites per particle) need gd_create/gd_geometry_build/gd_knn";
    if (!why.empty()) {
        st.code = GD_ERR_INVALID_ARGUMENT;
        st.msg = "gd_knn_static: " + why;
        return gd::static_fail(st, detail, msg, msg_len);
    }
    unsigned char *base = nullptr;
    st = gd::static_scratch(&base);
    if (!st) return gd::static_fail(st, detail, msg, msg_len);
    const gd::Model m = gd::make_model(*cfg);
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    gd::BorrowedGeometry bg(m, n_p, base);
    // The scratch keeps whatever the previous call left.  geometry_build resets the four counters
    // (active count, first bad index, two spare) on the stream before any kernel reads them; every
    // other scratch array is written in full before it is read.
    st = gd::geometry_build(bg.g, m, dev_particle, s);
    if (st) st = gd::knn_query(bg.g, m, dev_particle, dev_codes, dev_measure, dev_kth_d2, s);
    if (!st) return gd::static_fail(st, detail, msg, msg_len);
    return GD_OK;
}

// ---------------------------------------------------------------------------------------------
// The Strang step of the reference's time loop (src/swarm/swarm_runtime.cu:504-601)
// ---------------------------------------------------------------------------------------------
namespace {

// The geometry and the handle's neighbour cache for the current positions: the plain query, or,
// with a radius model and a previous search, the learned proposal seeded by the previous K-th
// distances (the rows are the plain query's either way).
gd::Status step_search(gd_handle *h, gd_particle *part, double total_mass, gd_radius_model *model) {
    h->geom_valid = false;
    h->cache_valid = false;
    h->col.local_geometry_valid = false;
    h->geo.sort_bits = h->tune.sort_bits;
    GD_TRY(gd::geometry_build(h->geo, h->m, part, h->stream));
    h->geom_valid = true;
    const float *radius = nullptr;
    if (model && h->step_prev_valid) {
        GD_TRY(gd::radius_features(h->geo, h->m, part, h->step_prev_kth.ptr, total_mass, h->step_features.ptr,
                                   h->stream));
        if (gd_radius_model_predict(model, h->step_features.ptr, h->n, h->step_radius.ptr, h->stream) != GD_OK)
            return gd::Status{GD_ERR_CUDA, "radius model prediction failed", 0};
        radius = h->step_radius.ptr;
    }
    GD_TRY(gd::knn_query(h->geo, h->m, part, h->codes.ptr, h->measure.ptr, h->kth.ptr, h->stream, radius, nullptr,
                         h->tune));
    GD_TRY(gd::space_bin(h->m, part, h->n, h->spatial.ptr, h->stream));
    if (h->step_prev_kth.ptr) {
        GD_TRY_CUDA(cudaMemcpyAsync(h->step_prev_kth.ptr, h->kth.ptr, sizeof(float) * h->n, cudaMemcpyDeviceToDevice,
                                    h->stream));
        h->step_prev_valid = true;
    }
    h->cache_valid = true;
    return gd::Status::ok();
}

void invalidate(gd_handle *h) {
    h->geom_valid = false;
    h->cache_valid = false;
    h->col.local_geometry_valid = false;
}

gd::Status step_prepare(gd_handle *h, const gd_run_info *run, gd_particle *part, void *rng, gd::Dyn &d) {
    if (!run || !part || !rng) return gd::Status{GD_ERR_INVALID_ARGUMENT, "null pointer", 0};
    if (!gd::aligned_to(part, 8) || !gd::aligned_to(rng, alignof(curandState)))
        return gd::Status{GD_ERR_INVALID_ARGUMENT, "misaligned particle or RNG pointer", 0};
    GD_TRY(gd::dyn_validate(h->m, *run));
    d = gd::make_dyn(*run);
    GD_TRY(gd::dyn_alloc(h->dyn, h->m));
    return gd::Status::ok();
}

// the dynamics of one step: D(dt/2) T(dt) D(dt/2) on the step's device timestep
gd::Status step_dynamics(gd_handle *h, const gd::Dyn &d, gd_particle *part, void *rng, long long *launches) {
    curandState *st = static_cast<curandState *>(rng);
    GD_TRY(gd::dyn_diffuse(h->dyn, h->m, d, h->n, part, st, h->stream, launches));
    GD_TRY(gd::dyn_transport(h->dyn, h->m, d, h->n, part, h->stream, launches));
    GD_TRY(gd::dyn_diffuse(h->dyn, h->m, d, h->n, part, st, h->stream, launches));
    invalidate(h);
    return gd::Status::ok();
}

}  // namespace

extern "C" {

gd_status gd_set_clock(gd_handle *h, double clock_sim, double clock_out, double dt_out) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    if (!std::isfinite(clock_sim) || !std::isfinite(clock_out) || !(dt_out > 0) || !std::isfinite(dt_out))
        return fail(h, GD_ERR_INVALID_ARGUMENT, "invalid clocks");
    gd::Status s = gd::dyn_alloc(h->dyn, h->m);
    if (s) s = gd::dyn_set_clock(h->dyn, clock_sim, clock_out, dt_out, h->stream);
    return done(h, s);
}

gd_status gd_get_clock(gd_handle *h, double *clock_sim, double *clock_out, double *dt_last, int *steps) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    if (!h->dyn.clock.ptr) return fail(h, GD_ERR_NOT_READY, "gd_get_clock before gd_set_clock");
    gd::StepClock c{};
    gd::Status s = gd::dyn_read_clock(h->dyn, c, h->stream);
    if (!s) return fail(h, s);
    if (clock_sim) *clock_sim = c.clock_sim;
    if (clock_out) *clock_out = c.clock_out;
    if (dt_last) *dt_last = c.dt;
    if (steps) *steps = c.count_dyn;
    return done(h, s);
}

gd_status gd_dynamics_step(gd_handle *h, const gd_run_info *run, gd_particle *dev_particle, void *dev_rng) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    gd::Dyn d;
    gd::Status s = step_prepare(h, run, dev_particle, dev_rng, d);
    if (s && !h->dyn.clock.ptr) s = gd::Status{GD_ERR_NOT_READY, "gd_dynamics_step before gd_set_clock", 0};
    long long launches = 0;
    if (s) s = gd::dyn_timestep(h->dyn, h->m, d, h->n, dev_particle, h->stream, &launches);
    if (s) s = step_dynamics(h, d, dev_particle, dev_rng, &launches);
    if (s) s = gd::dyn_clock_advance(h->dyn, h->stream, &launches);
    h->geo.launches += launches;
    return done(h, s);
}

gd_status gd_step(gd_handle *h, const gd_run_info *run, gd_particle *dev_particle, void *dev_rng,
                  double total_dust_mass, gd_radius_model *radius_model) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(h->stream, &cs) != cudaSuccess || cs == cudaStreamCaptureStatusInvalidated)
        return fail(h, GD_ERR_CUDA, "the handle's stream capture is invalid");
    const bool captured = cs == cudaStreamCaptureStatusActive;
    // a captured step allocates nothing and reads nothing back: the buffers come from an eager step
    if (captured && (!h->dyn.clock.ptr || !h->col.setup_done || !h->step_screen.ptr ||
                     (radius_model && !h->step_features.ptr)))
        return fail(h, GD_ERR_NOT_READY, "capture gd_step after one eager gd_step with the same radius model");
    gd::Dyn d;
    gd::Status s = step_prepare(h, run, dev_particle, dev_rng, d);
    if (s && !h->dyn.clock.ptr) s = gd::Status{GD_ERR_NOT_READY, "gd_step before gd_set_clock", 0};
    if (s && !(total_dust_mass > 0)) s = gd::Status{GD_ERR_INVALID_ARGUMENT, "total dust mass must be positive", 0};
    const bool deferred = h->geo.deferred_check;
    if (captured) h->geo.deferred_check = true;  // the screens are read by gd_check_step
    if (s && !h->step_screen.ptr) {
        const int none = INT_MAX;
        cudaError_t e = h->step_screen.alloc(1);
        if (e == cudaSuccess) e = cudaMemcpy(h->step_screen.ptr, &none, sizeof(int), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) s = gd::cuda_status(e, "gd_step screen buffer");
    }
    if (s && radius_model && !h->step_features.ptr) {
        cudaError_t e = h->step_features.alloc(static_cast<size_t>(h->n) * GD_RADIUS_FEATURES);
        if (e == cudaSuccess) e = h->step_radius.alloc(h->n);
        if (e == cudaSuccess) e = h->step_prev_kth.alloc(h->n);
        if (e != cudaSuccess) s = gd::cuda_status(e, "gd_step radius buffers");
        h->step_prev_valid = false;
    }
    long long launches = 0;
    // dt = min(DT_MAX, 1 / max rate, dt_out - clock_out), on the device; the collision halves read
    // dt / 2 there (the operator's controller rejects a non-positive or non-finite one)
    if (s) s = gd::dyn_timestep(h->dyn, h->m, d, h->n, dev_particle, h->stream, &launches);
    const double *dt_dev = h->dyn.clock.ptr ? &h->dyn.clock.ptr->dt : nullptr;
    const double *clock_sim_dev = h->dyn.clock.ptr ? &h->dyn.clock.ptr->clock_sim : nullptr;
    // C(dt/2): the geometry stays while the positions have not moved
    if (s) {
        if (h->geom_valid && h->cache_valid) s = gd::state_screen(h->geo, h->m, dev_particle, h->stream);
        else s = step_search(h, dev_particle, total_dust_mass, radius_model);
    }
    if (s && captured) s = gd::screen_keep(h->geo, h->step_screen.ptr, h->stream);
    if (s) s = gd::collision_operator(h->col, h->m, h->n, dev_particle, static_cast<curandState *>(dev_rng),
                                      h->codes.ptr, h->measure.ptr, h->geo.active.ptr, h->spatial.ptr, 0.0,
                                      total_dust_mass, h->stream, dt_dev, 0.5, clock_sim_dev);
    // D(dt/2) T(dt) D(dt/2), then C(dt/2) on the moved positions
    if (s) s = step_dynamics(h, d, dev_particle, dev_rng, &launches);
    if (s) s = step_search(h, dev_particle, total_dust_mass, radius_model);
    if (s && captured) s = gd::screen_keep(h->geo, h->step_screen.ptr, h->stream);
    if (s) s = gd::collision_operator(h->col, h->m, h->n, dev_particle, static_cast<curandState *>(dev_rng),
                                      h->codes.ptr, h->measure.ptr, h->geo.active.ptr, h->spatial.ptr, 0.0,
                                      total_dust_mass, h->stream, dt_dev, 0.5, clock_sim_dev);
    if (s) s = gd::dyn_clock_advance(h->dyn, h->stream, &launches);
    h->geo.launches += launches;
    h->geo.deferred_check = deferred;
    return done(h, s);
}

gd_status gd_check_step(gd_handle *h) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    // the operators' results (this also clears their accumulators), then the first failed
    // non-finite screen of the steps, which the reference meets before the operator that follows it
    gd::Status op = gd::collider_check(h->col, h->stream);
    int first = INT_MAX;
    if (h->step_screen.ptr) {
        const int none = INT_MAX;
        if (cudaMemcpyAsync(&first, h->step_screen.ptr, sizeof(int), cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
            cudaMemcpyAsync(h->step_screen.ptr, &none, sizeof(int), cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
            cudaStreamSynchronize(h->stream) != cudaSuccess)
            return fail(h, GD_ERR_CUDA, "read of the step screen");
    }
    if (first != INT_MAX) {
        invalidate(h);
        gd::Status st{GD_ERR_NONFINITE,
                      "non-finite particle state before collision search at particle " + std::to_string(first), first};
        return fail(h, st);
    }
    return done(h, op);
}

}  // extern "C"
