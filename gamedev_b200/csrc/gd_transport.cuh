// Dynamics of the Strang step (gd_transport.cu): the run settings the kernels read, the device
// clock of the time loop and the host entry points.
#pragma once

#include <curand_kernel.h>

#include "gd_internal.cuh"

namespace gd {

// The gd_run_info settings of the dynamics (the model directory's TRANSPORT, DIFFUSION, RADIATION,
// PR_EFFECT and VISC_FLOW flags and the constants they bring in).
struct Dyn {
    int transport, diffusion, radiation, pr_effect, visc_flow;
    double schmidt_x, schmidt_r, schmidt_z;
    double beta_0, kappa_0, t_beta, c_light;
    double dt_max, cfl_dyn;
};
Dyn make_dyn(const gd_run_info &r);

// The time loop's clocks in device memory (swarm_runtime.cu:475-600): a step reads its timestep
// from here, so it enqueues without reading anything back.
struct StepClock {
    double clock_sim, clock_out, dt_out;
    double dt, half_dt, beta_taper;
    unsigned long long max_rate_bits;  // the step's largest inverse timestep, as double bits
    int count_dyn;
};

struct DynState {
    DevBuf<StepClock> clock;
    DevBuf<double> optdepth;  // N_X * N_Y * N_Z optical depth of the radiation field
};

Status dyn_validate(const Model &m, const gd_run_info &r);
Status dyn_alloc(DynState &s, const Model &m);
Status dyn_set_clock(DynState &s, double clock_sim, double clock_out, double dt_out, cudaStream_t st);
// dyn_rate_calc + the max reduction + the step's dt and radiation taper (device)
Status dyn_timestep(DynState &s, const Model &m, const Dyn &d, int n, const gd_particle *part, cudaStream_t st,
                    long long *launches);
// diffusion_pos over half the step's dt
Status dyn_diffuse(DynState &s, const Model &m, const Dyn &d, int n, gd_particle *part, curandState *rng,
                   cudaStream_t st, long long *launches);
// ssa_transport, or ssa_substep_1 + optical depth + ssa_substep_2 with radiation
Status dyn_transport(DynState &s, const Model &m, const Dyn &d, int n, gd_particle *part, cudaStream_t st,
                     long long *launches);
Status dyn_clock_advance(DynState &s, cudaStream_t st, long long *launches);
Status dyn_read_clock(DynState &s, StepClock &out, cudaStream_t st);

}  // namespace gd
