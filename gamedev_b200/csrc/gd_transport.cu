// The dynamics operators of the reference's Strang step on sm_100a: the dynamics timestep, the
// staggered semi-analytic drag/gravity transport, radiation pressure with Poynting-Robertson drag
// through the radial optical depth, and Ito diffusion.  The reference's time loop
// (src/swarm/swarm_runtime.cu:504-601) composes them with the collision operator as
//     dt = min(DT_MAX, 1 / max rate, dt_out - clock_out)            dyn_rate_calc + max_element
//     C(dt/2)  D(dt/2)  T(dt)  D(dt/2)  C(dt/2)
// with T = ssa_transport, or with radiation ssa_substep_1 + optical depth + ssa_substep_2.
//
// Kernels (reference kernel in brackets), one thread per particle unless said otherwise:
//   k_dyn_rate       [dyn_rate_calc, dyn_rate_calc.cu:24-196] + a warp max and one atomic max per
//                    warp (the reference reduces with thrust::max_element on the host's side)
//   k_dyn_dt         the timestep and the radiation start-up taper, on the device (one thread)
//   k_ssa_transport  [ssa_transport, ssa_transport.cu:13-62]
//   k_ssa_substep_1  [ssa_substep_1, ssa_substep_1.cu:13-33]
//   k_optdepth_depo / _calc / _csum  [optdepth_depo.cu, optdepth_calc.cu, optdepth_csum.cu]
//   k_ssa_substep_2  [ssa_substep_2, ssa_substep_2.cu:13-63]
//   k_diffuse        [diffusion_pos, diffusion_pos.cu:21-201] through the cuRAND device API
//
// The timestep, the taper and the clocks live in device memory (StepClock), so a whole step
// enqueues without a host synchronisation.  The arithmetic follows the reference's expressions
// operation by operation (the FP64 state is what the physics conserves), with the model constants
// read at run time instead of compiled in.
#include <curand_kernel.h>

#include <cfloat>
#include <cmath>

#include "gd_collide.cuh"
#include "gd_geom_device.cuh"
#include "gd_internal.cuh"
#include "gd_physics.cuh"
#include "gd_transport.cuh"

namespace gd {

Dyn make_dyn(const gd_run_info &r) {
    Dyn d;
    d.transport = r.transport;
    d.diffusion = r.diffusion;
    d.radiation = r.radiation;
    d.pr_effect = r.pr_effect;
    d.visc_flow = r.visc_flow;
    d.schmidt_x = r.schmidt_x;
    d.schmidt_r = r.schmidt_r;
    d.schmidt_z = r.schmidt_z;
    d.beta_0 = r.beta_0;
    d.kappa_0 = r.kappa_0;
    d.t_beta = r.t_beta;
    d.c_light = r.c_light;
    d.dt_max = r.dt_max;
    d.cfl_dyn = r.cfl_dyn;
    return d;
}

namespace {

// ------------------------------------------------------------------------------------------------
// mesh primitives (inc/swarm/param_grid.cuh:13-108)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ double mesh_dx(const Model &m) { return (m.x_max - m.x_min) / static_cast<double>(m.n_x); }
__device__ __forceinline__ double mesh_dy(const Model &m) { return pow(m.y_max / m.y_min, 1.0 / static_cast<double>(m.n_y)); }
__device__ __forceinline__ double mesh_dz(const Model &m) { return (m.z_max - m.z_min) / static_cast<double>(m.n_z); }
__device__ __forceinline__ double yface(const Model &m, int iy) { return m.y_min * pow(mesh_dy(m), static_cast<double>(iy)); }
__device__ __forceinline__ double zface(const Model &m, int iz) { return m.z_min + mesh_dz(m) * static_cast<double>(iz); }
__device__ __forceinline__ double mesh_dim(const Model &m) { return 2.0 + static_cast<double>(m.n_z > 1); }
__device__ __forceinline__ double vol_x(const Model &m) {
    double v = mesh_dx(m);
    return (m.n_x > 1) ? v : 2.0 * M_PI;
}
__device__ __forceinline__ double vol_y(const Model &m, int iy) {
    double md = mesh_dim(m);
    return pow(yface(m, iy), md) * (pow(mesh_dy(m), md) - 1.0) / md;
}
__device__ __forceinline__ double vol_z(const Model &m, int iz) {
    double v = cos(zface(m, iz)) - cos(zface(m, iz + 1));
    return (m.n_z > 1) ? v : 1.0;
}
__device__ __forceinline__ double loc_x(const Model &m, double x) { return (m.n_x > 1) ? (x - m.x_min) / mesh_dx(m) : 0.0; }
__device__ __forceinline__ double loc_y(const Model &m, double y) {
    return (m.n_y > 1) ? log(y / m.y_min) / log(mesh_dy(m)) : 0.0;
}
__device__ __forceinline__ double loc_z(const Model &m, double z) { return (m.n_z > 1) ? (z - m.z_min) / mesh_dz(m) : 0.0; }
__device__ __forceinline__ bool in_bounds(const Model &m, double lx, double ly, double lz) {
    bool in_x = lx >= 0.0 && lx < static_cast<double>(m.n_x);
    bool in_y = ly >= 0.0 && ly < static_cast<double>(m.n_y);
    bool in_z = lz >= 0.0 && lz < static_cast<double>(m.n_z);
    return in_x && in_y && in_z;
}

// ------------------------------------------------------------------------------------------------
// trilinear stencil (inc/swarm/swarm_grid.cuh:21-196): periodic azimuth, logarithmic radius
// (cell centroids, or radial outer faces for the optical depth), clamped polar angle
// ------------------------------------------------------------------------------------------------
struct Stencil {
    int next_x, next_y, next_z;
    double frac_x, frac_y, frac_z;
};

__device__ __forceinline__ void interp_x(const Model &m, double lx, double deci, double &frac, int &next) {
    if (m.n_x == 1) {
        frac = 0.0;
        next = 0;
        return;
    }
    const double ref = 0.5;
    const bool bound = lx < ref || lx > static_cast<double>(m.n_x) + ref - 1.0;
    if (deci == ref) {
        frac = 0.0;
        next = 0;
    } else if (!bound) {
        if (deci > ref) {
            frac = deci - ref;
            next = 1;
        } else {
            frac = ref - deci;
            next = -1;
        }
    } else {
        if (deci >= ref) {
            frac = deci - ref;
            next = 1 - m.n_x;
        } else {
            frac = ref - deci;
            next = m.n_x - 1;
        }
    }
}

__device__ __forceinline__ void interp_y(const Model &m, double ly, double deci, double &frac, int &next, bool outer) {
    if (m.n_y == 1) {
        frac = 0.0;
        next = 0;
        return;
    }
    const double dy = mesh_dy(m);
    double ref;
    if (outer) {
        ref = 1.0;
    } else {
        const double md = mesh_dim(m);
        ref = log((md / (md + 1.0)) * (pow(dy, md + 1.0) - 1.0) / (pow(dy, md) - 1.0)) / log(dy);
    }
    const bool bound = outer ? ly < ref || ly > static_cast<double>(m.n_y) + ref - 1.0
                             : ly <= ref || ly >= static_cast<double>(m.n_y) + ref - 1.0;
    if (outer) {
        frac = (dy - pow(dy, deci)) / (dy - 1.0);
        next = bound ? 0 : -m.n_x;
    } else if (!bound) {
        if (deci >= ref) {
            frac = (pow(dy, deci - ref) - 1.0) / (dy - 1.0);
            next = m.n_x;
        } else {
            frac = (pow(dy, deci - ref) - 1.0) / (1.0 / dy - 1.0);
            next = -m.n_x;
        }
    } else {
        frac = 0.0;
        next = 0;
    }
}

__device__ __forceinline__ void interp_z(const Model &m, double lz, double deci, double &frac, int &next) {
    if (m.n_z == 1) {
        frac = 0.0;
        next = 0;
        return;
    }
    const double ref = 0.5;
    const bool bound = lz <= ref || lz >= static_cast<double>(m.n_z) + ref - 1.0;
    if (!bound) {
        if (deci >= ref) {
            frac = deci - ref;
            next = m.n_x * m.n_y;
        } else {
            frac = ref - deci;
            next = -m.n_x * m.n_y;
        }
    } else {
        frac = 0.0;
        next = 0;
    }
}

__device__ __forceinline__ Stencil stencil(const Model &m, double lx, double ly, double lz, bool outer) {
    Stencil t;
    const double dx = lx - floor(lx), dy = ly - floor(ly), dz = lz - floor(lz);
    interp_x(m, lx, dx, t.frac_x, t.next_x);
    interp_y(m, ly, dy, t.frac_y, t.next_y, outer);
    interp_z(m, lz, dz, t.frac_z, t.next_z);
    return t;
}

// _interp_field (swarm_grid.cuh:205-243)
__device__ __forceinline__ double interp_field(const Model &m, const double *f, double lx, double ly, double lz,
                                               bool outer) {
    if (m.half_disk) lz = fmin(lz, static_cast<double>(m.n_z) - 1.0e-06);
    if (outer) {
        if (ly < 0) return 0.0;
        if (!in_bounds(m, lx, ly, lz)) return DBL_MAX;
    } else if (!in_bounds(m, lx, ly, lz)) {
        return 0.0;
    }
    const int ix = static_cast<int>(lx), iy = static_cast<int>(ly), iz = static_cast<int>(lz);
    const int c = ix + iy * m.n_x + iz * m.n_x * m.n_y;
    const Stencil t = stencil(m, lx, ly, lz, outer);
    double v = 0.0;
    v += f[c] * (1.0 - t.frac_x) * (1.0 - t.frac_y) * (1.0 - t.frac_z);
    v += f[c + t.next_x] * t.frac_x * (1.0 - t.frac_y) * (1.0 - t.frac_z);
    v += f[c + t.next_y] * (1.0 - t.frac_x) * t.frac_y * (1.0 - t.frac_z);
    v += f[c + t.next_x + t.next_y] * t.frac_x * t.frac_y * (1.0 - t.frac_z);
    v += f[c + t.next_z] * (1.0 - t.frac_x) * (1.0 - t.frac_y) * t.frac_z;
    v += f[c + t.next_x + t.next_z] * t.frac_x * (1.0 - t.frac_y) * t.frac_z;
    v += f[c + t.next_y + t.next_z] * (1.0 - t.frac_x) * t.frac_y * t.frac_z;
    v += f[c + t.next_x + t.next_y + t.next_z] * t.frac_x * t.frac_y * t.frac_z;
    if (outer && ly < 1.0) v *= 1.0 - t.frac_y;
    return v;
}

// _deposit_field (swarm_grid.cuh:249-279)
__device__ __forceinline__ void deposit_field(const Model &m, double *g, const gd_particle &p, double weight) {
    double lx = loc_x(m, p.position[0]);
    double ly = loc_y(m, p.position[1]);
    double lz = loc_z(m, p.position[2]);
    if (m.half_disk) lz = fmin(lz, static_cast<double>(m.n_z) - 1.0e-06);
    if (!in_bounds(m, lx, ly, lz)) return;
    const int ix = static_cast<int>(lx), iy = static_cast<int>(ly), iz = static_cast<int>(lz);
    const int c = ix + iy * m.n_x + iz * m.n_x * m.n_y;
    const Stencil t = stencil(m, lx, ly, lz, false);
    atomicAdd(&g[c], (1.0 - t.frac_x) * (1.0 - t.frac_y) * (1.0 - t.frac_z) * weight);
    atomicAdd(&g[c + t.next_x], t.frac_x * (1.0 - t.frac_y) * (1.0 - t.frac_z) * weight);
    atomicAdd(&g[c + t.next_y], (1.0 - t.frac_x) * t.frac_y * (1.0 - t.frac_z) * weight);
    atomicAdd(&g[c + t.next_x + t.next_y], t.frac_x * t.frac_y * (1.0 - t.frac_z) * weight);
    atomicAdd(&g[c + t.next_z], (1.0 - t.frac_x) * (1.0 - t.frac_y) * t.frac_z * weight);
    atomicAdd(&g[c + t.next_x + t.next_z], t.frac_x * (1.0 - t.frac_y) * t.frac_z * weight);
    atomicAdd(&g[c + t.next_y + t.next_z], (1.0 - t.frac_x) * t.frac_y * t.frac_z * weight);
    atomicAdd(&g[c + t.next_x + t.next_y + t.next_z], t.frac_x * t.frac_y * t.frac_z * weight);
}

// ------------------------------------------------------------------------------------------------
// gas profiles (inc/swarm/param_phys.cuh:100-161)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ double get_nu(const Model &m, double R, double h) {
    if (m.const_nu) return m.nu;
    double nu = m.alpha * h * h * R * R * omega_k(m, R);
    return nu;
}

__device__ __forceinline__ double visc_vel(const Model &m, double R, double Z, double h) {
    double nu = get_nu(m, R, h);
    double grad_nu_R = m.const_nu ? 0.0 : m.idx_q + 1.5;
    if (m.n_z == 1) return -3.0 * nu * (grad_nu_R + m.idx_p + 0.5) / R;
    double y = sqrt(R * R + Z * Z);
    double cyl_frac = R / y;
    double strat = (cyl_frac - 1.0) / (h * h);
    double grad_strat_R = cyl_frac * (1.0 - cyl_frac * cyl_frac) / (h * h) - (m.idx_q + 1.0) * strat;
    double grad_strat_Z = -cyl_frac * (1.0 - cyl_frac * cyl_frac) / (h * h);
    double grad_rhog_R = m.idx_p - 0.5 * (m.idx_q + 3.0) + grad_strat_R;
    double grad_rhog_Z = grad_strat_Z;
    double term_R = 3.0 * nu * (grad_nu_R + grad_rhog_R + 0.5);
    double term_Z = m.idx_q * nu * (1.0 + grad_rhog_Z);
    return -(term_R - term_Z) / R;
}

// ------------------------------------------------------------------------------------------------
// boundaries (inc/swarm/_transport.cuh:37-146)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void periodic_x(const Model &m, double &x) {
    if (m.n_x == 1) {
        x = 0.5 * (m.x_min + m.x_max);
    } else {
        while (x >= m.x_max) x -= m.x_max - m.x_min;
        while (x < m.x_min) x += m.x_max - m.x_min;
    }
}

__device__ __forceinline__ void absorb(double &y, double &z, double &lx, double &vy, double &lz) {
    y = 0.0;
    z = 0.5 * M_PI;
    lx = 0.0;
    vy = 0.0;
    lz = 0.0;
}

__device__ __forceinline__ void transport_boundary(const Model &m, double &x, double &y, double &z, double &lx,
                                                   double &vy, double &lz) {
    periodic_x(m, x);
    if (m.n_z == 1) {
        z = 0.5 * M_PI;
        lz = 0.0;
    }
    if (y < m.y_min || y >= m.y_max) {
        absorb(y, z, lx, vy, lz);
        return;
    }
    if (m.half_disk && m.n_z > 1 && z > m.z_max) {
        z = M_PI - z;
        lz = -lz;
    }
    const bool polar_exit = m.half_disk ? (m.n_z > 1 && (z < m.z_min || z > m.z_max))
                                        : (m.n_z > 1 && (z < m.z_min || z >= m.z_max));
    if (polar_exit) absorb(y, z, lx, vy, lz);
}

__device__ __forceinline__ void diffusion_boundary(const Model &m, double &x, double &y, double &z) {
    periodic_x(m, x);
    while (y < m.y_min || y > m.y_max) {
        if (y < m.y_min) y = 2.0 * m.y_min - y;
        if (y > m.y_max) y = 2.0 * m.y_max - y;
    }
    if (y >= m.y_max) y = m.y_max - 1.0e-12 * (m.y_max - m.y_min);
    if (m.n_z == 1) {
        z = 0.5 * M_PI;
    } else {
        while (z < m.z_min || z > m.z_max) {
            if (z < m.z_min) z = 2.0 * m.z_min - z;
            if (z > m.z_max) z = 2.0 * m.z_max - z;
        }
        if (z >= m.z_max) z = m.z_max - 1.0e-12 * (m.z_max - m.z_min);
    }
}

// ------------------------------------------------------------------------------------------------
// staggered semi-analytic transport (inc/swarm/_transport.cuh:152-339)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void ssa_half_drift(const Model &m, double dt, double x_i, double y_i, double z_i, double lx_i,
                                               double vy_i, double lz_i, double &x_1, double &y_1, double &z_1) {
    y_1 = y_i + 0.5 * vy_i * dt;
    if (m.n_z == 1) {
        z_1 = 0.5 * M_PI;
        x_1 = (m.n_x > 1) ? x_i + 0.5 * lx_i * dt / y_i / y_1 : 0.5 * (m.x_min + m.x_max);
        return;
    }
    z_1 = z_i + 0.5 * lz_i * dt / y_i / y_1;
    x_1 = x_i + 0.5 * lx_i * dt / y_i / y_1 / sin(z_i) / sin(z_1);
}

__device__ __forceinline__ void force_term(const Model &m, double y, double z, double R, double lx, double lz,
                                           double beta, double &grav_y, double &cent_y, double &torq_z) {
    grav_y = -(1.0 - beta) * omega_k(m, y) * omega_k(m, y) * y;
    cent_y = lx * lx / R / R / y + lz * lz / y / y / y;
    torq_z = (m.n_z > 1) ? lx * lx / R / R / sin(z) * cos(z) : 0.0;
}

__device__ __forceinline__ void ssa_advance(const Model &m, const Dyn &d, double dt, double ts_1, double lx_g1,
                                            double vy_g1, double lz_g1, double beta, double lx_i, double vy_i,
                                            double lz_i, double x_1, double y_1, double z_1, double &x_j, double &y_j,
                                            double &z_j, double &lx_j, double &vy_j, double &lz_j) {
    double R_1 = cyl_R(m, y_1, z_1);
    double grav_y1, cent_y1, torq_z1;
    force_term(m, y_1, z_1, R_1, lx_i, lz_i, beta, grav_y1, cent_y1, torq_z1);
    double lx_1, vy_1, lz_1;
    double inv_ts1 = 0.0, rate_x1 = 0.0, rate_y1 = 0.0, rate_z1 = 0.0, tau_1 = 0.0;
    if (d.pr_effect) {
        inv_ts1 = 1.0 / ts_1;
        double pr_rate1 = beta * m.G * m.M_S / (d.c_light * y_1 * y_1);
        rate_x1 = inv_ts1 + pr_rate1;
        rate_y1 = inv_ts1 + 2.0 * pr_rate1;
        rate_z1 = inv_ts1 + pr_rate1;
        double relax_x1 = -expm1(-0.5 * rate_x1 * dt);
        double relax_y1 = -expm1(-0.5 * rate_y1 * dt);
        double relax_z1 = -expm1(-0.5 * rate_z1 * dt);
        double resp_x1 = relax_x1 / rate_x1;
        double resp_y1 = relax_y1 / rate_y1;
        double resp_z1 = relax_z1 / rate_z1;
        lx_1 = (1.0 - relax_x1) * lx_i + resp_x1 * inv_ts1 * lx_g1;
        vy_1 = (1.0 - relax_y1) * vy_i + resp_y1 * (inv_ts1 * vy_g1 + grav_y1 + cent_y1);
        lz_1 = (1.0 - relax_z1) * lz_i + resp_z1 * (inv_ts1 * lz_g1 + torq_z1);
    } else {
        tau_1 = dt / ts_1;
        lx_1 = lx_i + (lx_g1 - lx_i) * (1.0 - exp(-0.5 * tau_1));
        vy_1 = vy_i + ((grav_y1 + cent_y1) * ts_1 + vy_g1 - vy_i) * (1.0 - exp(-0.5 * tau_1));
        lz_1 = lz_i + (torq_z1 * ts_1 + lz_g1 - lz_i) * (1.0 - exp(-0.5 * tau_1));
    }
    (void)vy_1;  // the midpoint radial speed does not enter the second force evaluation
    double grav_y2, cent_y2, torq_z2;
    force_term(m, y_1, z_1, R_1, lx_1, lz_1, beta, grav_y2, cent_y2, torq_z2);
    if (d.pr_effect) {
        double relax_xj = -expm1(-rate_x1 * dt);
        double relax_yj = -expm1(-rate_y1 * dt);
        double relax_zj = -expm1(-rate_z1 * dt);
        double resp_xj = relax_xj / rate_x1;
        double resp_yj = relax_yj / rate_y1;
        double resp_zj = relax_zj / rate_z1;
        lx_j = (1.0 - relax_xj) * lx_i + resp_xj * inv_ts1 * lx_g1;
        vy_j = (1.0 - relax_yj) * vy_i + resp_yj * (inv_ts1 * vy_g1 + grav_y2 + cent_y2);
        lz_j = (1.0 - relax_zj) * lz_i + resp_zj * (inv_ts1 * lz_g1 + torq_z2);
    } else {
        lx_j = lx_i + (lx_g1 - lx_i) * (1.0 - exp(-tau_1));
        vy_j = vy_i + ((grav_y2 + cent_y2) * ts_1 + vy_g1 - vy_i) * (1.0 - exp(-tau_1));
        lz_j = lz_i + (torq_z2 * ts_1 + lz_g1 - lz_i) * (1.0 - exp(-tau_1));
    }
    y_j = y_1 + 0.5 * vy_j * dt;
    if (m.n_z == 1) {
        z_j = 0.5 * M_PI;
        lz_j = 0.0;
        x_j = (m.n_x > 1) ? x_1 + 0.5 * lx_j * dt / y_1 / y_j : 0.5 * (m.x_min + m.x_max);
        return;
    }
    z_j = z_1 + 0.5 * lz_j * dt / y_1 / y_j;
    x_j = x_1 + 0.5 * lx_j * dt / y_1 / y_j / sin(z_1) / sin(z_j);
}

__device__ __forceinline__ void ssa_complete(const Model &m, const Dyn &d, double dt, double size, double beta,
                                             double lx_i, double vy_i, double lz_i, double x_1, double y_1, double z_1,
                                             double &x_j, double &y_j, double &z_j, double &lx_j, double &vy_j,
                                             double &lz_j) {
    double R_1 = cyl_R(m, y_1, z_1);
    double Z_1 = cyl_Z(m, y_1, z_1);
    double h_g = get_hg(m, R_1);
    double omega = omega_k(m, R_1);
    double eta = get_eta(m, R_1, Z_1, h_g);
    double lx_g1 = sqrt(fmax(1.0 - 2.0 * eta, 0.0)) * omega * R_1 * R_1;
    double vy_g1 = 0.0, lz_g1 = 0.0;
    if (d.visc_flow) {
        double vR_g = visc_vel(m, R_1, Z_1, h_g);
        vy_g1 = (m.n_z > 1) ? vR_g * sin(z_1) : vR_g;
        lz_g1 = (m.n_z > 1) ? y_1 * vR_g * cos(z_1) : 0.0;
    }
    double ts_1 = stokes_at(m, R_1, Z_1, h_g, size) / omega;
    ssa_advance(m, d, dt, ts_1, lx_g1, vy_g1, lz_g1, beta, lx_i, vy_i, lz_i, x_1, y_1, z_1, x_j, y_j, z_j, lx_j, vy_j,
                lz_j);
}

__device__ __forceinline__ void load_particle(const gd_particle &p, double &x, double &y, double &z, double &lx,
                                              double &vy, double &lz) {
    x = p.position[0];
    y = p.position[1];
    z = p.position[2];
    lx = p.velocity[0];
    vy = p.velocity[1];
    lz = p.velocity[2];
}
__device__ __forceinline__ void save_particle(gd_particle &p, double x, double y, double z, double lx, double vy,
                                              double lz) {
    p.position[0] = x;
    p.position[1] = y;
    p.position[2] = z;
    p.velocity[0] = lx;
    p.velocity[1] = vy;
    p.velocity[2] = lz;
}

// ------------------------------------------------------------------------------------------------
// dust diffusion (inc/swarm/_diffusion.cuh:9-119, analytic gas, density diffusion)
// ------------------------------------------------------------------------------------------------
struct DustDiffusion {
    double nu, drift_R_per_D, drift_Z_per_D, drift_phi_per_D;
};

__device__ __forceinline__ DustDiffusion dust_diffusion(const Model &m, double y, double z, double size) {
    double R = cyl_R(m, y, z);
    double Z = cyl_Z(m, y, z);
    double h = get_hg(m, R);
    double st = stokes_at(m, R, Z, h, size);
    double f = 1.0 / (1.0 + st * st);
    double gy, gz;
    if (m.n_z == 1) {
        gy = m.idx_p / R;
    } else {
        double r = sqrt(R * R + Z * Z);
        gy = (m.idx_p - 0.5 * m.idx_q - 1.5) / R + (Z * Z / (r * r * r) - (m.idx_q + 1.0) * (R / r - 1.0) / R) / (h * h);
    }
    gz = (m.n_z > 1) ? -R * Z / (h * h * pow(R * R + Z * Z, 1.5)) : 0.0;
    double st_R = (m.n_z > 1) ? -gy - (m.idx_q + 3.0) / (2.0 * R) : -gy;
    double st_Z = -gz;
    double st_phi = -0.0;
    if (m.const_st) st_R = st_Z = st_phi = 0.0;
    double factor_grad = 2.0 * (1.0 - f);
    // the diffusion drift D/R plus dD/dR (_get_diff_drift_R): constant nu, or alpha with nu ~ R^(q + 3/2)
    double drift_R = m.const_nu ? 1.0 / R : 1.0 * (m.idx_q + 2.5) / R;
    DustDiffusion out;
    out.nu = get_nu(m, R, h) * f;
    out.drift_R_per_D = drift_R - factor_grad * st_R + 0.0 * gy;
    out.drift_Z_per_D = -factor_grad * st_Z + 0.0 * gz;
    out.drift_phi_per_D = -factor_grad * st_phi + 0.0 * 0.0;
    return out;
}

}  // namespace

// ------------------------------------------------------------------------------------------------
// kernels
// ------------------------------------------------------------------------------------------------
// dyn_rate_calc (dyn_rate_calc.cu:24-196, analytic gas), reduced to the largest rate: rates are
// non-negative, so their bit patterns order as the values do and one 64-bit atomic max per warp
// keeps the maximum
__global__ void k_dyn_rate(Model m, Dyn d, int n, const gd_particle *__restrict__ part, StepClock *clk) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    double rate = 0.0;
    if (idx < n) {
        const gd_particle p = part[idx];
        double y = p.position[1], z = p.position[2];
        if (site_active(m, y, z)) {
            double lx = p.velocity[0], vy = p.velocity[1], lz = p.velocity[2];
            double R = cyl_R(m, y, z);
            double dx = mesh_dx(m);
            double dy = mesh_dy(m);
            double dz = mesh_dz(m);
            int iy = static_cast<int>(log(y / m.y_min) / log(dy));
            iy = (iy >= m.n_y) ? m.n_y - 1 : iy;
            double dr = yface(m, iy) * (dy - 1.0);
            double omega = omega_k(m, R);
            rate = omega / d.cfl_dyn;
            if (m.n_x > 1) rate = fmax(rate, omega / (dx * d.cfl_dyn));
            if (m.n_x > 1) rate = fmax(rate, fabs(lx) / (R * R * dx * d.cfl_dyn));
            if (m.n_y > 1) rate = fmax(rate, fabs(vy) / (dr * d.cfl_dyn));
            if (m.n_z > 1) rate = fmax(rate, fabs(lz) / (y * y * dz * d.cfl_dyn));
            double beta = 0.0;
            if (d.radiation) {
                double size = p.par_size;
                // the strongest permitted radiation force after fragmentation (COLLISION and MULTISIZE)
                size = fmin(size, m.init_smin);
                beta = d.beta_0 / (size / m.S_0);
            }
            double grav_y = -(1.0 - beta) * m.G * m.M_S / (y * y);
            double cent_y = lx * lx / (R * R * y) + lz * lz / (y * y * y);
            double accel_y = fabs(grav_y + cent_y);
            rate = fmax(rate, sqrt(accel_y / (2.0 * d.cfl_dyn * dr)));
            if (m.n_z > 1) {
                double torq_z = lx * lx / (R * R) * cos(z) / sin(z);
                double accel_z = fabs(torq_z) / y;
                rate = fmax(rate, sqrt(accel_z / (2.0 * d.cfl_dyn * y * dz)));
            }
            if (d.visc_flow) {
                double h_g = get_hg(m, R);
                double vR_g = visc_vel(m, R, cyl_Z(m, y, z), h_g);
                if (m.n_y > 1) rate = fmax(rate, fabs((m.n_z > 1) ? vR_g * sin(z) : vR_g) / (dr * d.cfl_dyn));
                if (m.n_z > 1) rate = fmax(rate, fabs(vR_g * cos(z)) / (y * dz * d.cfl_dyn));
            }
            if (d.diffusion) {
                const DustDiffusion df = dust_diffusion(m, y, z, p.par_size);
                double nu = df.nu;
                double diff_x = nu / d.schmidt_x;
                double diff_R = nu / d.schmidt_r;
                double diff_Z = (m.n_z > 1) ? nu / d.schmidt_z : 0.0;
                double drift_x = diff_x * df.drift_phi_per_D / (R * R);
                double drift_R = diff_R * df.drift_R_per_D;
                double drift_Z = diff_Z * df.drift_Z_per_D;
                double sin_z = (m.n_z > 1) ? sin(z) : 1.0;
                double cos_z = (m.n_z > 1) ? cos(z) : 0.0;
                double diff_y = diff_R * sin_z * sin_z + diff_Z * cos_z * cos_z;
                double drift_y = drift_R * sin_z + drift_Z * cos_z;
                rate = fmax(rate, 2.0 * diff_y / (d.cfl_dyn * d.cfl_dyn * dr * dr));
                rate = fmax(rate, fabs(drift_y) / (d.cfl_dyn * dr));
                if (m.n_x > 1) {
                    double cell_x = R * dx;
                    rate = fmax(rate, 2.0 * diff_x / (d.cfl_dyn * d.cfl_dyn * cell_x * cell_x));
                    rate = fmax(rate, fabs(drift_x) / (d.cfl_dyn * dx));
                }
                if (m.n_z > 1) {
                    double cell_z = y * dz;
                    double diff_z = diff_R * cos_z * cos_z + diff_Z * sin_z * sin_z;
                    double drift_z = drift_R * cos_z - drift_Z * sin_z;
                    rate = fmax(rate, 2.0 * diff_z / (d.cfl_dyn * d.cfl_dyn * cell_z * cell_z));
                    rate = fmax(rate, fabs(drift_z) / (d.cfl_dyn * cell_z));
                }
            }
        }
    }
    unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(rate));
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long o = __shfl_xor_sync(0xffffffffu, bits, off);
        bits = o > bits ? o : bits;
    }
    if ((threadIdx.x & 31) == 0 && bits) atomicMax(&clk->max_rate_bits, bits);
}

// dt_dyn = min(DT_MAX, min(1 / max rate, dt_out - clock_out)) (swarm_runtime.cu:512-514) and the
// smooth radiation start-up of the step's midpoint (:564-566)
__global__ void k_dyn_dt(Dyn d, StepClock *clk) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double max_rate = __longlong_as_double(static_cast<long long>(clk->max_rate_bits));
    const double dt = fmin(d.dt_max, fmin(1.0 / max_rate, clk->dt_out - clk->clock_out));
    clk->dt = dt;
    clk->half_dt = 0.5 * dt;
    double taper = (d.t_beta > 0.0) ? (clk->clock_sim + 0.5 * dt) / d.t_beta : 1.0;
    taper = fmin(fmax(taper, 0.0), 1.0);
    clk->beta_taper = taper * taper * (3.0 - 2.0 * taper);
    clk->max_rate_bits = 0ull;  // ready for the next step's reduction
}

// the clocks after the step (swarm_runtime.cu:598-600)
__global__ void k_clock_advance(StepClock *clk) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    clk->clock_sim += clk->dt;
    clk->clock_out += clk->dt;
    clk->count_dyn += 1;
}

// ssa_transport (ssa_transport.cu:13-62): the whole step without a radiation field
__global__ void k_ssa_transport(Model m, Dyn d, int n, gd_particle *__restrict__ part, const StepClock *clk) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const double dt = clk->dt;
    double x_i, y_i, z_i, lx_i, vy_i, lz_i;
    load_particle(part[idx], x_i, y_i, z_i, lx_i, vy_i, lz_i);
    if (!site_active(m, y_i, z_i)) return;
    double x_1, y_1, z_1;
    ssa_half_drift(m, dt, x_i, y_i, z_i, lx_i, vy_i, lz_i, x_1, y_1, z_1);
    transport_boundary(m, x_1, y_1, z_1, lx_i, vy_i, lz_i);
    if (!site_active(m, y_1, z_1)) {
        save_particle(part[idx], x_1, y_1, z_1, lx_i, vy_i, lz_i);
        return;
    }
    const double size = part[idx].par_size;
    const double beta = 0.0;
    double x_j, y_j, z_j, lx_j, vy_j, lz_j;
    ssa_complete(m, d, dt, size, beta, lx_i, vy_i, lz_i, x_1, y_1, z_1, x_j, y_j, z_j, lx_j, vy_j, lz_j);
    transport_boundary(m, x_j, y_j, z_j, lx_j, vy_j, lz_j);
    save_particle(part[idx], x_j, y_j, z_j, lx_j, vy_j, lz_j);
}

// ssa_substep_1 (ssa_substep_1.cu:13-33): drift to the midpoint positions
__global__ void k_ssa_substep_1(Model m, int n, gd_particle *__restrict__ part, const StepClock *clk) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const double dt = clk->dt;
    double x_i, y_i, z_i, lx_i, vy_i, lz_i;
    load_particle(part[idx], x_i, y_i, z_i, lx_i, vy_i, lz_i);
    if (!site_active(m, y_i, z_i)) return;
    double x_1, y_1, z_1;
    ssa_half_drift(m, dt, x_i, y_i, z_i, lx_i, vy_i, lz_i, x_1, y_1, z_1);
    transport_boundary(m, x_1, y_1, z_1, lx_i, vy_i, lz_i);
    save_particle(part[idx], x_1, y_1, z_1, lx_i, vy_i, lz_i);
}

// optdepth_depo (optdepth_depo.cu:12-43): extinction cross sections onto the cell-centred grid
__global__ void k_optdepth_depo(Model m, Dyn d, int n, const gd_particle *__restrict__ part, double *grid) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    if (!site_active(m, part[idx].position[1], part[idx].position[2])) return;
    double size = part[idx].par_size;
    double weight = grain_mass(m, size) * part[idx].par_numr;
    weight *= d.kappa_0 / (size / m.S_0);
    if (m.n_z == 1) {
        double R = cyl_R(m, part[idx].position[1], part[idx].position[2]);
        double H_g = get_hg(m, R) * R;
        weight /= sqrt(2.0 * M_PI) * H_g;
    }
    deposit_field(m, grid, part[idx], weight);
}

// optdepth_calc (optdepth_calc.cu:12-27): cross section per cell volume times the radial cell width
__global__ void k_optdepth_calc(Model m, double *grid) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m.n_x * m.n_y * m.n_z) return;
    const int iy = (c / m.n_x) % m.n_y;
    const int iz = c / (m.n_x * m.n_y);
    double cell_measure = vol_x(m) * vol_y(m, iy) * vol_z(m, iz);
    double dr = yface(m, iy) * (mesh_dy(m) - 1.0);
    grid[c] /= cell_measure;
    grid[c] *= dr;
}

// optdepth_csum (optdepth_csum.cu:12-27): one radial ray per thread, from the inner boundary out
__global__ void k_optdepth_csum(Model m, double *grid) {
    const int ray = blockIdx.x * blockDim.x + threadIdx.x;
    if (ray >= m.n_x * m.n_z) return;
    const int ix = ray % m.n_x;
    const int iz = ray / m.n_x;
    for (int iy = 1; iy < m.n_y; iy++) {
        const int c = ix + iy * m.n_x + iz * m.n_x * m.n_y;
        grid[c] += grid[c - m.n_x];
    }
}

// ssa_substep_2 (ssa_substep_2.cu:13-63): drag, gravity and radiation pressure at the midpoint
__global__ void k_ssa_substep_2(Model m, Dyn d, int n, gd_particle *__restrict__ part, const double *__restrict__ grid,
                                const StepClock *clk) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const double dt = clk->dt;
    double x_1, y_1, z_1, lx_i, vy_i, lz_i;
    load_particle(part[idx], x_1, y_1, z_1, lx_i, vy_i, lz_i);
    if (!site_active(m, y_1, z_1)) return;
    double lx_ = loc_x(m, x_1), ly_ = loc_y(m, y_1), lz_ = loc_z(m, z_1);
    double optdepth = interp_field(m, grid, lx_, ly_, lz_, true);
    double size = part[idx].par_size;
    double beta = clk->beta_taper * d.beta_0 * exp(-optdepth) / (size / m.S_0);
    double x_j, y_j, z_j, lx_j, vy_j, lz_j;
    ssa_complete(m, d, dt, size, beta, lx_i, vy_i, lz_i, x_1, y_1, z_1, x_j, y_j, z_j, lx_j, vy_j, lz_j);
    transport_boundary(m, x_j, y_j, z_j, lx_j, vy_j, lz_j);
    save_particle(part[idx], x_j, y_j, z_j, lx_j, vy_j, lz_j);
}

// diffusion_pos (diffusion_pos.cu:21-201): one cylindrical Ito step of half the step's dt keeping
// the physical Cartesian velocity, with the particle's own cuRAND stream (normal draws, the device API)
__global__ void k_diffuse(Model m, Dyn d, int n, gd_particle *__restrict__ part, curandState *__restrict__ rng,
                          const StepClock *clk) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const double dt = clk->half_dt;
    double x = part[idx].position[0];
    double y = part[idx].position[1];
    double z = part[idx].position[2];
    if (!site_active(m, y, z)) return;
    double R = cyl_R(m, y, z);
    double Z = cyl_Z(m, y, z);
    double lx = part[idx].velocity[0];
    double vy = part[idx].velocity[1];
    double lz = part[idx].velocity[2];
    if (m.n_z == 1) {
        double vx = lx / R;
        double vR = vy;
        double vx_cart = vR * cos(x) - vx * sin(x);
        double vy_cart = vR * sin(x) + vx * cos(x);
        const DustDiffusion df = dust_diffusion(m, y, z, part[idx].par_size);
        double nu = df.nu;
        curandState st = rng[idx];
        double delta_x = 0.0;
        if (m.n_x > 1) {
            double diff_x = nu / d.schmidt_x;
            double avg_x = dt * diff_x * df.drift_phi_per_D / (R * R);
            double std_x = sqrt(2.0 * dt * diff_x) / R;
            delta_x = avg_x + std_x * curand_normal_double(&st);
        }
        double diff_R = nu / d.schmidt_r;
        double avg_R = dt * diff_R * df.drift_R_per_D;
        double std_R = sqrt(2.0 * dt * diff_R);
        double x_new = x + delta_x;
        double R_new = R + avg_R + std_R * curand_normal_double(&st);
        double z_new = 0.5 * M_PI;
        double x_basis = x_new;
        diffusion_boundary(m, x_new, R_new, z_new);
        double vR_new = vx_cart * cos(x_basis) + vy_cart * sin(x_basis);
        double vx_new = vy_cart * cos(x_basis) - vx_cart * sin(x_basis);
        part[idx].position[0] = x_new;
        part[idx].position[1] = R_new;
        part[idx].position[2] = 0.5 * M_PI;
        part[idx].velocity[0] = R_new * vx_new;
        part[idx].velocity[1] = vR_new;
        part[idx].velocity[2] = 0.0;
        rng[idx] = st;
        return;
    }
    double vx = lx / R;
    double vz = lz / y;
    double vR = vy * sin(z) + vz * cos(z);
    double vZ = vy * cos(z) - vz * sin(z);
    double vx_cart = vR * cos(x) - vx * sin(x);
    double vy_cart = vR * sin(x) + vx * cos(x);
    const DustDiffusion df = dust_diffusion(m, y, z, part[idx].par_size);
    double nu = df.nu;
    curandState st = rng[idx];
    double delta_x = 0.0, delta_R = 0.0, delta_Z = 0.0;
    if (m.n_x > 1) {
        double diff_x = nu / d.schmidt_x;
        double avg_x = dt * diff_x * df.drift_phi_per_D / (R * R);
        double std_x = sqrt(2.0 * dt * diff_x) / R;
        delta_x = avg_x + std_x * curand_normal_double(&st);
    }
    if (m.n_y > 1) {
        double diff_R = nu / d.schmidt_r;
        double avg_R = dt * diff_R * df.drift_R_per_D;
        double std_R = sqrt(2.0 * dt * diff_R);
        delta_R = avg_R + std_R * curand_normal_double(&st);
    }
    if (m.n_z > 1) {
        double diff_Z = nu / d.schmidt_z;
        double avg_Z = dt * diff_Z * df.drift_Z_per_D;
        double std_Z = sqrt(2.0 * dt * diff_Z);
        delta_Z = avg_Z + std_Z * curand_normal_double(&st);
    }
    double x_new = x + delta_x;
    double R_new = R + delta_R;
    double Z_new = Z + delta_Z;
    if (R_new < 0.0) {
        R_new = -R_new;
        x_new += M_PI;
    }
    double y_new = sqrt(R_new * R_new + Z_new * Z_new);
    double z_new = atan2(R_new, Z_new);
    double x_basis = x_new;
    diffusion_boundary(m, x_new, y_new, z_new);
    R_new = cyl_R(m, y_new, z_new);
    Z_new = cyl_Z(m, y_new, z_new);
    double sinz_new = R_new / y_new;
    double cosz_new = Z_new / y_new;
    double vR_new = vx_cart * cos(x_basis) + vy_cart * sin(x_basis);
    double vx_new = vy_cart * cos(x_basis) - vx_cart * sin(x_basis);
    lx = vx_new * R_new;
    vy = vR_new * sinz_new + vZ * cosz_new;
    lz = (vR_new * cosz_new - vZ * sinz_new) * y_new;
    part[idx].position[0] = x_new;
    part[idx].position[1] = y_new;
    part[idx].position[2] = z_new;
    part[idx].velocity[0] = lx;
    part[idx].velocity[1] = vy;
    part[idx].velocity[2] = lz;
    rng[idx] = st;
}

__global__ void k_clock_set(StepClock *clk, double clock_sim, double clock_out, double dt_out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    clk->clock_sim = clock_sim;
    clk->clock_out = clock_out;
    clk->dt_out = dt_out;
    clk->dt = clk->half_dt = 0.0;
    clk->beta_taper = 0.0;
    clk->max_rate_bits = 0ull;
    clk->count_dyn = 0;
}

// ------------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------------
Status dyn_validate(const Model &m, const gd_run_info &r) {
    if (r.importgas) return Status{GD_ERR_INVALID_ARGUMENT, "imported gas fields are not supported by the dynamics", 0};
    if (!r.transport) return Status{GD_ERR_INVALID_ARGUMENT, "the dynamics step needs TRANSPORT", 0};
    if (!(r.cfl_dyn > 0) || !(r.dt_max > 0)) return Status{GD_ERR_INVALID_ARGUMENT, "invalid CFL_DYN or DT_MAX", 0};
    if (r.diffusion && (!(r.schmidt_x > 0) || !(r.schmidt_r > 0) || !(r.schmidt_z > 0)))
        return Status{GD_ERR_INVALID_ARGUMENT, "invalid Schmidt numbers", 0};
    if (r.pr_effect && !(r.c_light > 0)) return Status{GD_ERR_INVALID_ARGUMENT, "invalid C_LIGHT", 0};
    if (m.n_z > 1 && !r.diffusion) return Status{GD_ERR_INVALID_ARGUMENT, "a 3D model needs DIFFUSION", 0};
    return Status::ok();
}

Status dyn_alloc(DynState &s, const Model &m) {
    if (!s.clock.ptr) {
        GD_TRY_CUDA(s.clock.alloc(1));
        GD_TRY_CUDA(cudaMemset(s.clock.ptr, 0, sizeof(StepClock)));
    }
    const size_t cells = static_cast<size_t>(m.n_x) * m.n_y * m.n_z;
    if (s.optdepth.n != cells) GD_TRY_CUDA(s.optdepth.alloc(cells));
    return Status::ok();
}

Status dyn_set_clock(DynState &s, double clock_sim, double clock_out, double dt_out, cudaStream_t st) {
    k_clock_set<<<1, 32, 0, st>>>(s.clock.ptr, clock_sim, clock_out, dt_out);
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}

Status dyn_timestep(DynState &s, const Model &m, const Dyn &d, int n, const gd_particle *part, cudaStream_t st,
                    long long *launches) {
    const int tpb = 256;
    k_dyn_rate<<<(n + tpb - 1) / tpb, tpb, 0, st>>>(m, d, n, part, s.clock.ptr);
    k_dyn_dt<<<1, 32, 0, st>>>(d, s.clock.ptr);
    if (launches) *launches += 2;
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}

Status dyn_diffuse(DynState &s, const Model &m, const Dyn &d, int n, gd_particle *part, curandState *rng,
                   cudaStream_t st, long long *launches) {
    if (!d.diffusion) return Status::ok();
    const int tpb = 128;
    k_diffuse<<<(n + tpb - 1) / tpb, tpb, 0, st>>>(m, d, n, part, rng, s.clock.ptr);
    if (launches) *launches += 1;
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}

Status dyn_transport(DynState &s, const Model &m, const Dyn &d, int n, gd_particle *part, cudaStream_t st,
                     long long *launches) {
    const int tpb = 128;
    const int blocks = (n + tpb - 1) / tpb;
    if (!d.radiation) {
        k_ssa_transport<<<blocks, tpb, 0, st>>>(m, d, n, part, s.clock.ptr);
        if (launches) *launches += 1;
        GD_TRY_CUDA(cudaGetLastError());
        return Status::ok();
    }
    const int cells = m.n_x * m.n_y * m.n_z;
    k_ssa_substep_1<<<blocks, tpb, 0, st>>>(m, n, part, s.clock.ptr);
    GD_TRY_CUDA(cudaMemsetAsync(s.optdepth.ptr, 0, sizeof(double) * cells, st));
    k_optdepth_depo<<<blocks, tpb, 0, st>>>(m, d, n, part, s.optdepth.ptr);
    k_optdepth_calc<<<(cells + 255) / 256, 256, 0, st>>>(m, s.optdepth.ptr);
    k_optdepth_csum<<<(m.n_x * m.n_z + 127) / 128, 128, 0, st>>>(m, s.optdepth.ptr);
    k_ssa_substep_2<<<blocks, tpb, 0, st>>>(m, d, n, part, s.optdepth.ptr, s.clock.ptr);
    if (launches) *launches += 5;
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}

Status dyn_clock_advance(DynState &s, cudaStream_t st, long long *launches) {
    k_clock_advance<<<1, 32, 0, st>>>(s.clock.ptr);
    if (launches) *launches += 1;
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}

Status dyn_read_clock(DynState &s, StepClock &out, cudaStream_t st) {
    GD_TRY_CUDA(cudaMemcpyAsync(&out, s.clock.ptr, sizeof(StepClock), cudaMemcpyDeviceToHost, st));
    GD_TRY_CUDA(cudaStreamSynchronize(st));
    return Status::ok();
}

}  // namespace gd
