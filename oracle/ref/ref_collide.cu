// Reference-GPU collision step: the reference's own evolve_collisions glue
// (src/swarm/swarm_runtime.cu:357-471: col_site_init, KD or Morton index, col_cache_get,
// col_space_bin) and evolve_local_collisions (inc/swarm/_col_chain.cuh:108-539) with its kernels
// (src/swarm/col_*.cu, rngstate_init.cu), compiled from the GameDev tree where it lies, against a
// generated model header, by oracle/ref/Makefile into oracle/_ref/collide_<model>_<n>/ref_collide.
// TEST INFRASTRUCTURE ONLY: it pins the B200 collision operator against the reference's CUDA
// build (statistically, and per particle where the neighbour order is the same) and times it.
//
//   ref_collide <in.bin> <out.bin> <seed> <duration> <total_dust_mass> <operators> [<summary.json>]
//   in.bin : int32 n (= N_P), then n particle records (the 64 B struct swarm)
//   out.bin: the n records after `operators` calls of evolve_collisions(duration) on one geometry
//   stdout : one JSON line {"n", "operators", "geometry_ms", "operator_ms": [...], "total_ms"}
//   GD_REF_SITES=<file> (environment): also writes the search's records (KD nodes, or the Morton
//            index's points and periodic ghosts), int32 count, count x (float32 x, y, z, int32 code)
//   GD_REF_NEIGHBOURS=<file> (environment): also writes the neighbour cache of the geometry,
//            int32 n, int32 K, int32 codes[n][K] (col_cache_get's order), float64 measure[n]
//   GD_REF_STEPS=<s> (environment): repeat the whole sequence s times (default 1), as a swarm step
//            of the reference's runtime does it (swarm_runtime.cu:504-601 without transport): rebuild
//            the geometry (col_site_init, index, col_cache_get, col_space_bin; the owner lists are
//            invalidated), then `operators` evolve_collisions(duration) calls, each after the first
//            preceded by the colstate_flag screen the reference runs on a valid geometry
//            (swarm_runtime.cu:361-373); stdout then also holds "steps": [[geometry_ms, op_ms...]...]
//            and the dumps below describe the first step's geometry
//   summary.json (builds with COL_DIAGNOSTICS only): the controller summary of the operators as
//            the reference's save_col_controller writes it (_col_bound.cuh:242-299); those builds
//            also write their per-operator log, collision_local_<stamp>.jsonl, to the working
//            directory
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <gpu.cuh>

#include <thrust/device_ptr.h>
#include <thrust/extrema.h>

#include <swarm_kern.cuh>

#include <_col_chain.cuh>
#ifdef COLLISION_MORTON
#include <morton/morton_ghost.cuh>
#endif

namespace {

void check(gpuError_t e, const char *what) {
    if (e != gpuSuccess) throw std::runtime_error(std::string(what) + ": " + gpuGetErrorString(e));
}

template <typename T>
T *dev_alloc(std::size_t count, const char *what) {
    T *p = nullptr;
    check(gpuMalloc(reinterpret_cast<void **>(&p), sizeof(T) * (count ? count : 1)), what);
    return p;
}

void check_bad(int *dev_bad_part) {
    int bad = 0;
    check(gpuMemcpy(&bad, dev_bad_part, sizeof(int), gpuMemcpyDeviceToHost), "read bad particle");
    if (bad != 0) throw std::runtime_error("non-finite particle " + std::to_string(bad - 1));
}

}  // namespace

int main(int argc, char **argv) {
    try {
        if (argc != 7 && argc != 8)
            throw std::runtime_error("usage: ref_collide <in> <out> <seed> <duration> <mass> <operators> [<summary>]");
        static_assert(sizeof(swarm) == 64, "MULTISIZE particle record");
        std::ifstream in(argv[1], std::ios::binary);
        int n = 0;
        in.read(reinterpret_cast<char *>(&n), 4);
        if (!in || n != N_P) throw std::runtime_error("particle count differs from the model's N_P");
        std::vector<swarm> particle(N_P);
        in.read(reinterpret_cast<char *>(particle.data()), sizeof(swarm) * N_P);
        if (!in) throw std::runtime_error("short input");
        const int seed = std::atoi(argv[3]);
        const real duration = std::atof(argv[4]);
        const real total_dust_mass = std::atof(argv[5]);
        const int operators = std::atoi(argv[6]);

        // the device state swarm_runtime.cu:120-184 allocates for COLLISION
        swarm *dev_particle = dev_alloc<swarm>(N_P, "particles");
        check(gpuMemcpy(dev_particle, particle.data(), sizeof(swarm) * N_P, gpuMemcpyHostToDevice), "copy particles");
        unsigned char *dev_col_active = dev_alloc<unsigned char>(N_P, "active");
        int *dev_bad_part = dev_alloc<int>(1, "bad particle");
#ifdef COLLISION_KDTREE
        kdtree_boxf *dev_kdtree_box = dev_alloc<kdtree_boxf>(1, "kd box");
        kdtree_node *dev_kdtree_node = dev_alloc<kdtree_node>(N_T, "kd nodes");
#else
        float3 *dev_morton_point = dev_alloc<float3>(N_P, "morton points");
        float *dev_morton_posx = dev_alloc<float>(N_P, "morton posx");
        float *dev_search_dist = dev_alloc<float>(N_P, "search distance");
        unsigned int *dev_morton_overflow = dev_alloc<unsigned int>(N_P, "morton overflow");
        morton_ghost_index morton_owner;
#endif
        real *dev_size_old = dev_alloc<real>(N_P, "size_old");
        real *dev_numr_old = dev_alloc<real>(N_P, "numr_old");
        real *dev_col_rate = dev_alloc<real>(N_P, "rate");
        int *dev_col_neighbor = dev_alloc<int>(static_cast<std::size_t>(N_P) * N_K, "neighbours");
        real *dev_col_measure = dev_alloc<real>(N_P, "measure");
        const int col_raw_count = _get_col_raw_count();
        int *dev_col_events = dev_alloc<int>(N_P, "events");
        int *dev_col_spatial = dev_alloc<int>(N_P, "spatial");
        int *dev_col_count = dev_alloc<int>(col_raw_count, "bin counts");
        int *dev_col_binmap = dev_alloc<int>(col_raw_count, "bin map");
        int *dev_col_error = dev_alloc<int>(N_P, "errors");
        int *dev_col_unfinished = dev_alloc<int>(1, "unfinished");
        real *dev_col_time = dev_alloc<real>(N_P, "clock");
        real *dev_col_hazard = dev_alloc<real>(N_P, "hazard");
        real *dev_col_jump1_int = dev_alloc<real>(N_P, "jump1");
        real *dev_col_jump2_int = dev_alloc<real>(N_P, "jump2");
        real *dev_col_jumpmax_int = dev_alloc<real>(N_P, "jumpmax");
        unsigned char *dev_col_complete = dev_alloc<unsigned char>(N_P, "complete");
        col_rate_bin *dev_col_ratebin = dev_alloc<col_rate_bin>(col_raw_count, "rate bins");
        col_audit_accum *dev_col_audit = dev_alloc<col_audit_accum>(col_raw_count, "audit bins");
        check(gpuMemset(dev_col_error, 0, sizeof(int) * N_P), "clear errors");
        curs *dev_rngstate = dev_alloc<curs>(N_P, "rng");
        rngstate_init<<<NB_P, TPB>>>(dev_rngstate, seed);
        check(gpuGetLastError(), "rngstate_init");

        float image_dist_min = -1.0f;
        if (X_WEDGE)
            image_dist_min = _get_image_dist_min(static_cast<float>(X_MIN), static_cast<float>(X_MAX),
                                                 static_cast<float>(Y_MIN), static_cast<float>(Z_MIN),
                                                 static_cast<float>(Z_MAX));
        // the COL_DIAGNOSTICS build writes its per-operator log (collision_local_<stamp>.jsonl) here
        local_workspace local("./");
        bool local_geometry_valid = false;
        real clock_dyn = 0.0, dt_col = 0.0;
        int count_col = 0;
#ifdef COL_DIAGNOSTICS
        col_controller_summary col_summary;
        const real clock_sim = 0.0;
#endif

        gpuEvent_t a, b;
        check(gpuEventCreate(&a), "event");
        check(gpuEventCreate(&b), "event");
        float geometry_ms = 0.0f;
        std::vector<float> op_ms;
        int steps = 1;
        if (const char *env = std::getenv("GD_REF_STEPS")) steps = std::atoi(env);
        if (steps < 1) throw std::runtime_error("GD_REF_STEPS must be positive");
        std::vector<std::vector<float>> step_ms;

        for (int step = 0; step < steps; ++step) {
        // geometry once per step (positions do not change between the operators of a step)
        local_geometry_valid = false;
        clock_dyn = 0.0;
        count_col = 0;
        check(gpuDeviceSynchronize(), "setup");
        check(gpuEventRecord(a, 0), "record");
        check(gpuMemset(dev_bad_part, 0, sizeof(int)), "clear bad particle");
#ifdef COLLISION_KDTREE
        col_site_init<<<NB_P, TPB>>>(dev_kdtree_node, dev_col_active, dev_particle, dev_bad_part);
        check(gpuGetLastError(), "col_site_init");
        check_bad(dev_bad_part);
        kdtree::buildTree<kdtree_node, kdtree_traits>(dev_kdtree_node, N_T, dev_kdtree_box);
        col_cache_get<<<(N_T + kdtree_heap::threads - 1) / kdtree_heap::threads, kdtree_heap::threads>>>(
            dev_col_neighbor, dev_col_measure, dev_kdtree_node, dev_kdtree_box, dev_col_active, dev_particle,
            image_dist_min);
        check(gpuGetLastError(), "col_cache_get");
#else
        col_site_init<<<NB_P, TPB>>>(dev_morton_point, dev_morton_posx, dev_search_dist, dev_col_active,
                                       dev_particle, dev_bad_part);
        check(gpuGetLastError(), "col_site_init");
        check_bad(dev_bad_part);
        thrust::device_ptr<const float> search_dist_ptr(dev_search_dist);
        const float max_search_dist = *thrust::max_element(search_dist_ptr, search_dist_ptr + N_P);
        const bool unique_ids = image_dist_min < 0.0f || image_dist_min > 2.0f * max_search_dist;
        morton_owner.build(dev_morton_point, dev_morton_posx, N_P, max_search_dist, static_cast<float>(X_MIN),
                           static_cast<float>(X_MAX), static_cast<float>(Y_MAX), X_WEDGE, unique_ids,
                           (N_Z > 1) ? 3 : 2, MORTON_LEAF_TARGET, MORTON_MAX_LEVEL);
        col_cache_get<<<N_P, MORTON_TPB>>>(dev_col_neighbor, dev_col_measure, dev_morton_overflow, dev_morton_point,
                                            dev_col_active, dev_particle, morton_owner.view(),
                                            morton_owner.unique_ids());
        check(gpuGetLastError(), "col_cache_get");
        thrust::device_ptr<const unsigned int> overflow_ptr(dev_morton_overflow);
        if (*thrust::max_element(overflow_ptr, overflow_ptr + N_P) != 0)
            throw std::runtime_error("Morton traversal stack overflow in col_cache_get");
#endif
        col_space_bin<<<NB_P, TPB>>>(dev_col_spatial, dev_particle);
        check(gpuGetLastError(), "col_space_bin");
        check(gpuEventRecord(b, 0), "record");
        check(gpuEventSynchronize(b), "geometry");
        check(gpuEventElapsedTime(&geometry_ms, a, b), "elapsed");
        // the search's records (KD tree nodes, or the Morton index's points with its periodic ghosts),
        // when GD_REF_SITES names a file: int32 count, then count x (float x, y, z, int32 code)
        const char *sites_path = step == 0 ? std::getenv("GD_REF_SITES") : nullptr;
        if (const char *path = sites_path) {
            std::vector<float> rec;
#ifdef COLLISION_KDTREE
            std::vector<kdtree_node> node(N_T);
            check(gpuMemcpy(node.data(), dev_kdtree_node, sizeof(kdtree_node) * N_T, gpuMemcpyDeviceToHost),
                  "copy kd nodes");
            for (const kdtree_node &t : node) {
                const int code = _encode_col_neighbor(t.idx_old, t.image);
                float c;
                std::memcpy(&c, &code, 4);
                rec.insert(rec.end(), {t.cartesian.x, t.cartesian.y, t.cartesian.z, c});
            }
#else
            const morton_view view = morton_owner.view();
            std::vector<morton_point> pts(view.point_count);
            check(gpuMemcpy(pts.data(), view.dev_point, sizeof(morton_point) * pts.size(), gpuMemcpyDeviceToHost),
                  "copy Morton points");
            for (const morton_point &t : pts) {
                float c;
                std::memcpy(&c, &t.idx_old, 4);
                rec.insert(rec.end(), {t.cartesian.x, t.cartesian.y, t.cartesian.z, c});
            }
#endif
            std::ofstream sf(path, std::ios::binary);
            const int count = static_cast<int>(rec.size() / 4);
            sf.write(reinterpret_cast<const char *>(&count), 4);
            sf.write(reinterpret_cast<const char *>(rec.data()), sizeof(float) * rec.size());
            if (!sf) throw std::runtime_error("cannot write the search records");
        }
        // the neighbour cache col_cache_get wrote, when GD_REF_NEIGHBOURS names a file
        const char *neighbours_path = step == 0 ? std::getenv("GD_REF_NEIGHBOURS") : nullptr;
        if (const char *path = neighbours_path) {
            std::vector<int> codes(static_cast<std::size_t>(N_P) * N_K);
            std::vector<real> measure(N_P);
            check(gpuMemcpy(codes.data(), dev_col_neighbor, sizeof(int) * codes.size(), gpuMemcpyDeviceToHost),
                  "copy neighbours");
            check(gpuMemcpy(measure.data(), dev_col_measure, sizeof(real) * N_P, gpuMemcpyDeviceToHost),
                  "copy measures");
            std::ofstream nb(path, std::ios::binary);
            const int header[2] = {N_P, N_K};
            nb.write(reinterpret_cast<const char *>(header), sizeof(header));
            nb.write(reinterpret_cast<const char *>(codes.data()), sizeof(int) * codes.size());
            nb.write(reinterpret_cast<const char *>(measure.data()), sizeof(real) * measure.size());
            if (!nb) throw std::runtime_error("cannot write the neighbour cache");
        }

        std::vector<float> this_step{geometry_ms};
        for (int op = 0; op < operators; ++op) {
            check(gpuEventRecord(a, 0), "record");
            if (op > 0) {
                // the non-finite screen evolve_collisions runs when the geometry is still valid
                check(gpuMemset(dev_bad_part, 0, sizeof(int)), "clear bad particle");
                colstate_flag<<<NB_P, TPB>>>(dev_particle, dev_bad_part);
                check(gpuGetLastError(), "colstate_flag");
                check_bad(dev_bad_part);
            }
            evolve_local_collisions(local, local_geometry_valid, duration, total_dust_mass, clock_dyn, dt_col,
                                    count_col, col_raw_count, dev_particle, dev_rngstate, dev_col_spatial,
                                    dev_col_neighbor, dev_col_events, dev_col_count, dev_col_binmap, dev_col_error,
                                    dev_col_unfinished, dev_col_active, dev_col_complete, dev_size_old,
                                    dev_numr_old, dev_col_time, dev_col_rate, dev_col_hazard, dev_col_jump1_int,
                                    dev_col_jump2_int, dev_col_jumpmax_int, dev_col_measure, dev_col_ratebin,
                                    dev_col_audit
#ifdef COL_DIAGNOSTICS
                                    , clock_sim, col_summary
#endif
            );
            check(gpuEventRecord(b, 0), "record");
            check(gpuEventSynchronize(b), "operator");
            float ms = 0.0f;
            check(gpuEventElapsedTime(&ms, a, b), "elapsed");
            this_step.push_back(ms);
        }
        if (step == 0) op_ms.assign(this_step.begin() + 1, this_step.end());
        step_ms.push_back(this_step);
        }
        check(gpuMemcpy(particle.data(), dev_particle, sizeof(swarm) * N_P, gpuMemcpyDeviceToHost), "copy back");
#ifdef COL_DIAGNOSTICS
        if (argc == 8 && !save_col_controller(argv[7], col_summary))
            throw std::runtime_error("cannot write the controller summary");
#endif
        std::ofstream out(argv[2], std::ios::binary);
        out.write(reinterpret_cast<const char *>(&n), 4);
        out.write(reinterpret_cast<const char *>(particle.data()), sizeof(swarm) * N_P);
        if (!out) throw std::runtime_error("cannot write output");
        float total = step_ms[0][0];
        std::string ops;
        for (std::size_t i = 0; i < op_ms.size(); ++i) {
            total += op_ms[i];
            ops += (i ? ", " : "") + std::to_string(op_ms[i]);
        }
        std::string all;
        for (std::size_t s = 0; s < step_ms.size(); ++s) {
            all += s ? ", [" : "[";
            for (std::size_t k = 0; k < step_ms[s].size(); ++k) all += (k ? ", " : "") + std::to_string(step_ms[s][k]);
            all += "]";
        }
        std::printf("{\"n\": %d, \"operators\": %d, \"geometry_ms\": %.4f, \"operator_ms\": [%s], \"total_ms\": %.4f, "
                    "\"steps\": [%s]}\n",
                    N_P, operators, step_ms[0][0], ops.c_str(), total, all.c_str());
        return 0;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_collide: %s\n", e.what());
        return 1;
    }
}
