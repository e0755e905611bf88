// Batched neighbour search: many independent swarms of uneven size (and K) per call.  No
// counterpart in the reference, which runs one swarm per process.
//
// One BatchGeometry indexes every swarm with one launch per stage: site init over the
// concatenated particles, one radix sort of (swarm id, Morton) keys (each swarm's sites come out
// contiguous), gather, leaf bounds and one launch per tree level across swarms.  One persistent
// launch then runs the top-K of every bucket of every swarm (knn_batch_query).  The non-finite
// screen is deferred to gd_batch_check, so a call makes no host synchronisation and can be
// captured into a CUDA graph: about fifty kernels per call, whatever the number of swarms.
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "gd_collide.cuh"
#include "gd_internal.cuh"

// operators of one batch run side by side on this many forked streams (graph branches)
constexpr int kBatchOperatorStreams = 16;
// bath records each swarm's controller keeps between two reads
constexpr int kBatchRecordCapacity = 1024;

struct gd_batch {
    gd_config cfg;
    int S = 0;
    std::vector<int> n, k;
    std::vector<long long> part_off, codes_off;
    long long n_total = 0, codes_total = 0;
    int kcap = 0;
    std::vector<gd::Model> models;
    gd::BatchGeometry geo;
    gd::DevBuf<gd::BatchSwarm> tab;
    gd::DevBuf<int> leaf_prefix;
    gd::DevBuf<long long> part_prefix;
    gd::DevBuf<int> next;
    cudaStream_t stream = nullptr;
    long long launches = 0;
    gd::Tuning tune;
    std::string err;
    long long detail = 0;
    // the batched collision operator: one collider per swarm, allocated at its first call
    std::vector<std::unique_ptr<gd::Collider>> col;
    cudaStream_t capture = nullptr;
    cudaStream_t fork[kBatchOperatorStreams] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kBatchOperatorStreams] = {};
    bool collide_pending = false;
    ~gd_batch() {
        for (int i = 0; i < kBatchOperatorStreams; ++i) {
            if (fork[i]) cudaStreamDestroy(fork[i]);
            if (ev_join[i]) cudaEventDestroy(ev_join[i]);
        }
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (capture) cudaStreamDestroy(capture);
    }
};

namespace {

gd_status batch_fail(gd_batch *b, const gd::Status &s) {
    if (b) {
        b->err = s.msg;
        b->detail = s.detail;
    }
    return s.code;
}

gd_status batch_fail(gd_batch *b, gd_status code, const std::string &msg, long long detail = 0) {
    gd::Status s;
    s.code = code;
    s.msg = msg;
    s.detail = detail;
    return batch_fail(b, s);
}

}  // namespace

extern "C" {

gd_status gd_batch_create(const gd_config *cfg, int S, const int *n_p, const int *n_k, gd_batch **out) {
    if (!cfg || !n_p || !n_k || !out || S <= 0) return GD_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    std::unique_ptr<gd_batch> b(new (std::nothrow) gd_batch());
    if (!b) return GD_ERR_OUT_OF_MEMORY;
    b->cfg = *cfg;
    b->S = S;
    b->n.assign(n_p, n_p + S);
    b->k.assign(n_k, n_k + S);
    // the segmented geometry holds one site per particle: wedges (three) take the one-swarm path
    if (gd::make_model(*cfg).wedge) return GD_ERR_INVALID_ARGUMENT;
    std::vector<int> leaf_prefix(S + 1, 0);
    std::vector<long long> part_prefix(S + 1, 0);
    for (int s = 0; s < S; ++s) {
        if (n_p[s] <= 0 || static_cast<long long>(n_p[s]) * 3 > 0x7fffffffLL || n_k[s] < 1 || n_k[s] > gd::kMaxK)
            return GD_ERR_INVALID_ARGUMENT;
        gd_config c = *cfg;
        c.n_k = n_k[s];
        b->models.push_back(gd::make_model(c));
        b->part_off.push_back(b->n_total);
        b->codes_off.push_back(b->codes_total);
        b->n_total += n_p[s];
        b->codes_total += static_cast<long long>(n_p[s]) * n_k[s];
        b->kcap = n_k[s] > b->kcap ? n_k[s] : b->kcap;
        leaf_prefix[s + 1] = leaf_prefix[s] + (n_p[s] + gd::kLeaf - 1) / gd::kLeaf;
        part_prefix[s + 1] = b->n_total;
    }
    gd::Status st = gd::batch_geometry_alloc(b->geo, b->models[0], S, n_p, b->tune.sort_bits);
    if (!st) return st.code;
    gd::BatchGeometry &g = b->geo;
    std::vector<gd::BatchSwarm> tab(S);
    for (int s = 0; s < S; ++s) {
        gd::BatchSwarm &t = tab[s];
        t.sorted = g.sorted.ptr + g.h_leaf_prefix[s] * gd::kLeaf;
        t.lo = g.node_lo.ptr + g.h_node_off[s];
        t.hi = g.node_hi.ptr + g.h_node_off[s];
        t.sub_lo = g.sub_lo.ptr + g.h_leaf_prefix[s] * gd::kSubs;
        t.sub_hi = g.sub_hi.ptr + g.h_leaf_prefix[s] * gd::kSubs;
        t.qrad = g.q.ptr + b->part_off[s];
        t.active = g.active.ptr + b->part_off[s];
        t.counters = g.counters.ptr + 2 * s;
        t.leaf_slots = g.leaf_slots[s];
        t.k = n_k[s];
        t.part_off = b->part_off[s];
        t.codes_off = b->codes_off[s];
    }
    if (b->tab.alloc(S) != cudaSuccess || b->leaf_prefix.alloc(S + 1) != cudaSuccess ||
        b->part_prefix.alloc(S + 1) != cudaSuccess || b->next.alloc(1) != cudaSuccess)
        return GD_ERR_OUT_OF_MEMORY;
    if (cudaMemcpy(b->tab.ptr, tab.data(), sizeof(gd::BatchSwarm) * S, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->leaf_prefix.ptr, leaf_prefix.data(), sizeof(int) * (S + 1), cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemcpy(b->part_prefix.ptr, part_prefix.data(), sizeof(long long) * (S + 1), cudaMemcpyHostToDevice) !=
            cudaSuccess)
        return GD_ERR_CUDA;
    *out = b.release();
    return GD_OK;
}

void gd_batch_destroy(gd_batch *b) { delete b; }

gd_status gd_batch_set_stream(gd_batch *b, void *stream) {
    if (!b) return GD_ERR_INVALID_ARGUMENT;
    b->stream = static_cast<cudaStream_t>(stream);
    return GD_OK;
}

gd_status gd_batch_knn(gd_batch *b, const gd_particle *dev_particle, int32_t *dev_codes, double *dev_measure,
                       float *dev_kth_d2) {
    if (!b || !dev_particle || !dev_codes || !dev_measure || !dev_kth_d2)
        return batch_fail(b, GD_ERR_INVALID_ARGUMENT, "null batch, particle or output pointer");
    if (!gd::aligned_to(dev_particle, 8) || !gd::aligned_to(dev_codes, 4) || !gd::aligned_to(dev_measure, 8) ||
        !gd::aligned_to(dev_kth_d2, 4))
        return batch_fail(b, GD_ERR_INVALID_ARGUMENT, "misaligned particle or output pointer");
    const long long before = b->geo.launches;
    gd::Status st = gd::batch_geometry_build(b->geo, b->models[0], dev_particle, b->stream);
    b->launches += b->geo.launches - before;
    if (!st) return batch_fail(b, st);
    st = gd::knn_batch_query(b->models[0], b->tab.ptr, b->leaf_prefix.ptr, b->part_prefix.ptr, b->S, b->n_total,
                             b->kcap, b->next.ptr, dev_particle, dev_codes, dev_measure, dev_kth_d2, b->stream,
                             &b->launches, b->tune);
    if (!st) return batch_fail(b, st);
    for (auto &c : b->col) c->local_geometry_valid = false;  // new rows: the operators' owner lists follow
    b->err.clear();
    b->detail = 0;
    return GD_OK;
}

// the colliders' results since the last read; detail of an error = the swarm index
static gd::Status batch_collide_check(gd_batch *b) {
    std::vector<gd::Collider *> cs;
    for (auto &c : b->col) cs.push_back(c.get());
    int failed = -1;
    gd::Status st = gd::collider_check_many(cs.data(), static_cast<int>(cs.size()), b->stream, &failed);
    b->collide_pending = false;
    if (!st) {
        st.msg = "swarm " + std::to_string(failed) + ": " + st.msg;
        st.detail = failed;
    }
    return st;
}

gd_status gd_batch_check(gd_batch *b) {
    if (!b) return GD_ERR_INVALID_ARGUMENT;
    int swarm = -1;
    gd::Status st = gd::batch_geometry_check(b->geo, b->stream, &swarm);
    if (!st) return batch_fail(b, st);
    if (b->collide_pending) {
        st = batch_collide_check(b);
        if (!st) return batch_fail(b, st);
    }
    b->err.clear();
    b->detail = 0;
    return GD_OK;
}

// The operators of all swarms enqueued on q (capturing): forked onto the batch's streams after q's
// work so far, joined back into q.
static gd::Status batch_collide_enqueue(gd_batch *b, gd_particle *part, curandState *rng, const int32_t *codes,
                                        const double *measure, const double *durations, const double *masses,
                                        cudaStream_t q) {
    const int F = b->S < kBatchOperatorStreams ? b->S : kBatchOperatorStreams;
    GD_TRY_CUDA(cudaEventRecord(b->ev_fork, q));
    for (int i = 0; i < F; ++i) GD_TRY_CUDA(cudaStreamWaitEvent(b->fork[i], b->ev_fork, 0));
    gd::Status st = gd::Status::ok();
    for (int s = 0; s < b->S && st; ++s) {
        st = gd::collision_operator_enqueue(*b->col[s], b->models[s], b->n[s], part + b->part_off[s],
                                            rng + b->part_off[s], codes + b->codes_off[s], measure + b->part_off[s],
                                            b->geo.active.ptr + b->part_off[s], durations[s], masses[s],
                                            b->fork[s % F]);
    }
    // join every forked stream, whatever happened, so that the capture can end
    for (int i = 0; i < F; ++i) {
        cudaEventRecord(b->ev_join[i], b->fork[i]);
        cudaStreamWaitEvent(q, b->ev_join[i], 0);
    }
    GD_TRY(st);
    GD_TRY_CUDA(cudaGetLastError());
    return gd::Status::ok();
}

gd_status gd_batch_collide(gd_batch *b, gd_particle *dev_particle, void *dev_rng, const int32_t *dev_codes,
                           const double *dev_measure, const double *durations, const double *total_dust_masses) {
    if (!b || !dev_particle || !dev_rng || !dev_codes || !dev_measure || !durations || !total_dust_masses)
        return batch_fail(b, GD_ERR_INVALID_ARGUMENT, "null batch, particle, RNG, cache or argument pointer");
    if (!gd::aligned_to(dev_particle, 8) || !gd::aligned_to(dev_rng, alignof(curandState)) ||
        !gd::aligned_to(dev_codes, 4) || !gd::aligned_to(dev_measure, 8))
        return batch_fail(b, GD_ERR_INVALID_ARGUMENT, "misaligned particle, RNG or cache pointer");
    for (int s = 0; s < b->S; ++s)
        if (!(durations[s] > 0) || !std::isfinite(durations[s]) || !(total_dust_masses[s] > 0) ||
            !std::isfinite(total_dust_masses[s]))
            return batch_fail(b, GD_ERR_INVALID_ARGUMENT, "invalid operator length or dust mass", s);
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(b->stream, &cs) != cudaSuccess || cs == cudaStreamCaptureStatusInvalidated)
        return batch_fail(b, GD_ERR_CUDA, "the batch stream's capture is invalid");
    const bool outer = cs == cudaStreamCaptureStatusActive;
    if (b->col.empty()) {
        if (outer) return batch_fail(b, GD_ERR_NOT_READY, "run gd_batch_collide once before capturing it");
        for (int s = 0; s < b->S; ++s) {
            std::unique_ptr<gd::Collider> c(new (std::nothrow) gd::Collider());
            if (!c) return batch_fail(b, GD_ERR_OUT_OF_MEMORY, "batch colliders");
            gd::Status st = gd::collider_alloc(*c, b->models[s], b->n[s], kBatchRecordCapacity);
            if (!st) {
                b->col.clear();
                return batch_fail(b, st);
            }
            b->col.push_back(std::move(c));
        }
        bool ok = cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking) == cudaSuccess &&
                  cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) == cudaSuccess;
        for (int i = 0; i < kBatchOperatorStreams && ok; ++i)
            ok = cudaStreamCreateWithFlags(&b->fork[i], cudaStreamNonBlocking) == cudaSuccess &&
                 cudaEventCreateWithFlags(&b->ev_join[i], cudaEventDisableTiming) == cudaSuccess;
        if (!ok) return batch_fail(b, GD_ERR_CUDA, "batch operator streams");
    }
    gd_particle *part = dev_particle;
    curandState *rng = static_cast<curandState *>(dev_rng);
    if (outer) {
        gd::Status st = batch_collide_enqueue(b, part, rng, dev_codes, dev_measure, durations, total_dust_masses,
                                              b->stream);
        if (!st) return batch_fail(b, st);
        b->collide_pending = true;
        return GD_OK;
    }
    // eager: one graph of every swarm's operator, run on the batch's stream, results read
    if (cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return batch_fail(b, GD_ERR_CUDA, "batch operator capture");
    gd::Status st = batch_collide_enqueue(b, part, rng, dev_codes, dev_measure, durations, total_dust_masses,
                                          b->capture);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->capture, &graph);
    if (!st || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        for (auto &c : b->col) c->local_geometry_valid = false;
        if (!st) return batch_fail(b, st);
        return batch_fail(b, gd::cuda_status(e, "batch operator capture"));
    }
    cudaGraphExec_t exec = nullptr;
    cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie == cudaSuccess) ie = cudaGraphLaunch(exec, b->stream);
    if (ie != cudaSuccess) {
        if (exec) cudaGraphExecDestroy(exec);
        for (auto &c : b->col) c->local_geometry_valid = false;
        return batch_fail(b, gd::cuda_status(ie, "batch operator graph"));
    }
    st = batch_collide_check(b);
    cudaGraphExecDestroy(exec);
    if (!st) return batch_fail(b, st);
    b->err.clear();
    b->detail = 0;
    return GD_OK;
}

gd_status gd_batch_reset_controller(gd_batch *b) {
    if (!b) return GD_ERR_INVALID_ARGUMENT;
    for (size_t s = 0; s < b->col.size(); ++s) {
        gd::Status st = gd::collider_reset_state(*b->col[s], b->stream);
        if (!st) {
            st.msg = "swarm " + std::to_string(s) + ": " + st.msg;
            st.detail = static_cast<long long>(s);
            return batch_fail(b, st);
        }
    }
    b->collide_pending = false;
    return GD_OK;
}

gd_status gd_batch_invalidate(gd_batch *b) {
    if (!b) return GD_ERR_INVALID_ARGUMENT;
    for (auto &c : b->col) c->local_geometry_valid = false;
    return GD_OK;
}

gd_status gd_batch_operator_stats(const gd_batch *b, int s, gd_operator_stats *out) {
    if (!b || !out || s < 0 || s >= b->S) return GD_ERR_INVALID_ARGUMENT;
    if (b->col.empty()) return GD_ERR_NOT_READY;
    *out = b->col[s]->stats;
    return GD_OK;
}

gd_status gd_batch_set_tuning(gd_batch *b, const gd_tuning *t) {
    if (!b || !t) return GD_ERR_INVALID_ARGUMENT;
    const int dim = b->models[0].dim;
    const bool ok = t->warps_per_block >= 0 && t->warps_per_block <= 32 && t->prescan >= 0 && t->prescan <= 8 &&
                    (t->walk_breadth_first == 0 || t->walk_breadth_first == 1) &&
                    (t->sort_bits == 0 || (t->sort_bits >= 16 * dim && t->sort_bits <= 21 * dim));
    if (!ok) return batch_fail(b, GD_ERR_INVALID_ARGUMENT, "tuning out of range");
    gd::Tuning u;
    u.warps = t->warps_per_block;
    u.prescan = t->prescan;
    u.bfs = t->walk_breadth_first;
    u.sort_bits = t->sort_bits;
    if (u.warps > 0 && gd::knn_block_warps(b->kcap, u, nullptr) == 0)
        return batch_fail(b, GD_ERR_INVALID_ARGUMENT, "warps per block do not fit in shared memory");
    // the Morton bits the next build keeps under the swarm id
    const int key_bits = 21 * dim;
    int mbits = (u.sort_bits > 0 && u.sort_bits < key_bits) ? u.sort_bits : key_bits;
    if (u.sort_bits == 0 && mbits + b->geo.sbits > 64) mbits = 64 - b->geo.sbits;
    if (mbits + b->geo.sbits > 64) return batch_fail(b, GD_ERR_INVALID_ARGUMENT, "too many swarms for the sort key");
    b->geo.mbits = mbits;
    b->geo.mshift = key_bits - mbits;
    b->tune = u;
    return GD_OK;
}

size_t gd_batch_last_error(const gd_batch *b, char *buf, size_t len) {
    if (!b) return 0;
    if (buf && len) {
        size_t k = b->err.size() < len - 1 ? b->err.size() : len - 1;
        std::memcpy(buf, b->err.data(), k);
        buf[k] = '\0';
    }
    return b->err.size();
}

long long gd_batch_error_detail(const gd_batch *b) { return b ? b->detail : 0; }

long long gd_batch_launch_count(const gd_batch *b) { return b ? b->launches : 0; }

}  // extern "C"
