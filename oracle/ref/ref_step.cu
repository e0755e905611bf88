// Reference-GPU dynamics of the Strang step: the reference's own dyn_rate_calc, diffusion_pos,
// ssa_transport or ssa_substep_1 + optdepth_* + ssa_substep_2 (src/swarm/*.cu), compiled from the
// GameDev tree where it lies, against a generated model header, by oracle/ref/Makefile into
// oracle/_ref/step_<model>_<n>/ref_step, and driven the way swarm_runtime.cu:504-600 drives them
// without the collision halves:
//     dt = min(DT_MAX, min(1 / max rate, DT_OUT - clock_out))
//     diffusion_pos(dt/2); transport(dt); diffusion_pos(dt/2); clocks += dt
// TEST INFRASTRUCTURE ONLY: it pins the B200 dynamics (gd_dynamics_step) against the reference.
//
//   ref_step <in.bin> <out.bin> <seed> <steps> <total_dust_mass> <clock_sim> <clock_out>
//   in.bin : int32 n (= N_P), then n particle records (the 64 B struct swarm)
//   out.bin: int32 n, the n records after `steps` steps, then the n curand states
//   stdout : one JSON line {"n", "steps", "dt": [...], "ms": [...] (each step, host clock around the
//            synchronised step, as the reference loop synchronises), "clock_sim", "clock_out"}
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <gpu.cuh>

#include <thrust/device_ptr.h>
#include <thrust/extrema.h>

#include <swarm_kern.cuh>

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

}  // namespace

int main(int argc, char **argv) {
    try {
        if (argc != 8) throw std::runtime_error("usage: ref_step <in> <out> <seed> <steps> <mass> <clock_sim> <clock_out>");
        std::ifstream in(argv[1], std::ios::binary);
        int n = 0;
        in.read(reinterpret_cast<char *>(&n), 4);
        if (!in || n != N_P) throw std::runtime_error("particle count differs from the model's N_P");
        std::vector<swarm> particle(N_P);
        in.read(reinterpret_cast<char *>(particle.data()), sizeof(swarm) * N_P);
        if (!in) throw std::runtime_error("short input");
        const int seed = std::atoi(argv[3]);
        const int steps = std::atoi(argv[4]);
        const real total_dust_mass = std::atof(argv[5]);
        real clock_sim = std::atof(argv[6]);
        real clock_out = std::atof(argv[7]);

        swarm *dev_particle = dev_alloc<swarm>(N_P, "particles");
        check(gpuMemcpy(dev_particle, particle.data(), sizeof(swarm) * N_P, gpuMemcpyHostToDevice), "copy particles");
        curs *dev_rngstate = dev_alloc<curs>(N_P, "rng");
        rngstate_init<<<NB_P, TPB>>>(dev_rngstate, seed);
        check(gpuGetLastError(), "rngstate_init");
        real *dev_dyn_rate = dev_alloc<real>(N_P, "dyn rate");
#ifdef RADIATION
        real *dev_optdepth = dev_alloc<real>(N_G, "optdepth");
#endif
        (void)total_dust_mass;
        std::string dts, mss;
        check(gpuDeviceSynchronize(), "setup");
        for (int step = 0; step < steps; ++step) {
            const auto t0 = std::chrono::steady_clock::now();
            // swarm_runtime.cu:504-514
            dyn_rate_calc<<<NB_P, TPB>>>(dev_dyn_rate, dev_particle);
            check(gpuGetLastError(), "dyn_rate_calc");
            thrust::device_ptr<const real> dt_rate_ptr(dev_dyn_rate);
            const real max_dt_rate = *thrust::max_element(dt_rate_ptr, dt_rate_ptr + N_P);
            const real dt_dyn = std::fmin(DT_MAX, std::fmin(1.0 / max_dt_rate, DT_OUT - clock_out));
#ifdef DIFFUSION
            diffusion_pos<<<NB_P, TPB>>>(dev_particle, dev_rngstate, 0.5 * dt_dyn);
            check(gpuGetLastError(), "diffusion_pos");
#endif
#ifdef RADIATION
            // swarm_runtime.cu:548-579
            ssa_substep_1<<<NB_P, TPB>>>(dev_particle, dt_dyn);
            check(gpuGetLastError(), "ssa_substep_1");
            optdepth_init<<<NB_G, TPB>>>(dev_optdepth);
            optdepth_depo<<<NB_P, TPB>>>(dev_optdepth, dev_particle, total_dust_mass);
            optdepth_calc<<<NB_G, TPB>>>(dev_optdepth);
            optdepth_csum<<<NB_Y, TPB>>>(dev_optdepth);
            check(gpuGetLastError(), "optdepth");
            real taper = (T_BETA > 0.0) ? (clock_sim + 0.5 * dt_dyn) / T_BETA : 1.0;
            taper = std::fmin(std::fmax(taper, 0.0), 1.0);
            const real beta_taper = taper * taper * (3.0 - 2.0 * taper);
            ssa_substep_2<<<NB_P, TPB>>>(dev_particle, dev_optdepth, beta_taper, dt_dyn);
            check(gpuGetLastError(), "ssa_substep_2");
#else
            ssa_transport<<<NB_P, TPB>>>(dev_particle, dt_dyn);
            check(gpuGetLastError(), "ssa_transport");
#endif
#ifdef DIFFUSION
            diffusion_pos<<<NB_P, TPB>>>(dev_particle, dev_rngstate, 0.5 * dt_dyn);
            check(gpuGetLastError(), "diffusion_pos");
#endif
            check(gpuDeviceSynchronize(), "step");
            const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            clock_sim += dt_dyn;
            clock_out += dt_dyn;
            char buf[64];
            std::snprintf(buf, sizeof(buf), "%s%.17g", step ? ", " : "", dt_dyn);
            dts += buf;
            std::snprintf(buf, sizeof(buf), "%s%.6g", step ? ", " : "", ms);
            mss += buf;
        }
        check(gpuMemcpy(particle.data(), dev_particle, sizeof(swarm) * N_P, gpuMemcpyDeviceToHost), "copy back");
        std::vector<curs> rng(N_P);
        check(gpuMemcpy(rng.data(), dev_rngstate, sizeof(curs) * N_P, gpuMemcpyDeviceToHost), "copy rng");
        std::ofstream out(argv[2], std::ios::binary);
        out.write(reinterpret_cast<const char *>(&n), 4);
        out.write(reinterpret_cast<const char *>(particle.data()), sizeof(swarm) * N_P);
        out.write(reinterpret_cast<const char *>(rng.data()), sizeof(curs) * N_P);
        if (!out) throw std::runtime_error("cannot write output");
        std::printf("{\"n\": %d, \"steps\": %d, \"dt\": [%s], \"ms\": [%s], \"clock_sim\": %.17g, "
                    "\"clock_out\": %.17g}\n", N_P, steps, dts.c_str(), mss.c_str(), clock_sim, clock_out);
        return 0;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_step: %s\n", e.what());
        return 1;
    }
}
