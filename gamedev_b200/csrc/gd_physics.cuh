// FP64 pair physics of the collision operator, evaluated per (owner, neighbour slot).
// Every function restates the reference formula named in its comment, with the same operation
// order, so only the libm/libdevice rounding of transcendental calls can separate the two.
#pragma once

#include <cuda_runtime.h>

#include "gd_geom_device.cuh"
#include "gd_internal.cuh"

namespace gd {

// query_environment (inc/swarm/_col_types.cuh:355-358)
struct Env {
    double Z, omega, vn, radial, strat, cs, re_inv_sqrt, vg_sq;
};

// cached_rate_moments (inc/swarm/_col_types.cuh:366)
struct RateMoments {
    double rate, first, second, maximum;
};

// param_phys.cuh:16-18
__device__ __forceinline__ double grain_mass(const Model &m, double size) {
    return M_PI * m.rho_0 * size * size * size / 6.0;
}
// param_phys.cuh:66-68
__device__ __forceinline__ double omega_k(const Model &m, double R) { return sqrt(m.G * m.M_S / R / R / R); }
// param_phys.cuh:75-77
__device__ __forceinline__ double get_eta(const Model &m, double R, double Z, double h) {
    return -0.5 * ((m.idx_p + 0.5 * m.idx_q - 1.5) * h * h + m.idx_q * (1.0 - R / sqrt(R * R + Z * Z)));
}
// param_phys.cuh:80-82
__device__ __forceinline__ double gas_strat(double R, double Z, double h) {
    return exp((R / sqrt(R * R + Z * Z) - 1.0) / (h * h));
}
// param_phys.cuh:85-87
__device__ __forceinline__ double sigma_g(const Model &m, double R) { return m.sigma_0 * pow(R / m.R_0, m.idx_p); }
// param_phys.cuh:95-97
__device__ __forceinline__ double sound_speed(const Model &m, double R, double h) { return h * omega_k(m, R) * R; }
// param_phys.cuh:113-122
__device__ __forceinline__ double get_alpha(const Model &m, double R, double h) {
    if (m.const_nu) return m.nu / (h * h * R * R * omega_k(m, R));
    return m.alpha;
}
// _get_re_inv_sqrt (inc/swarm/_collision.cuh:137-150)
__device__ __forceinline__ double re_inv_sqrt(const Model &m, double R, double alpha, double sig) {
    double reynolds;
    if (m.code_unit) {
        double alpha_0 = get_alpha(m, m.R_0, m.aspr_0);
        reynolds = m.reynolds_0 * (alpha / alpha_0) * (sig / m.sigma_0);
    } else {
        reynolds = 0.5 * alpha * sig * m.x_sec / m.m_mol;
    }
    return 1.0 / sqrt(reynolds);
}
// _get_stokes for analytic gas (param_phys.cuh:163-210)
__device__ __forceinline__ double stokes_at(const Model &m, double R, double Z, double h, double size) {
    double st = m.stokes_0 * (size / m.S_0);
    if (!m.const_st) {
        st /= pow(R / m.R_0, m.idx_p);
        st /= gas_strat(R, Z, h);
    }
    return st;
}

// Ormel-Cuzzi turbulent relative speed from the regime algebra shared by _get_vrel_t
// (_collision.cuh:153-273) and _cached_turbulence (_col_rates.cuh:34-124).
__device__ __forceinline__ double oc07_speed(double stokes_i, double stokes_j, double re_inv, double vg_sq) {
    double sl, ss;
    if (stokes_i >= stokes_j) {
        sl = stokes_i;
        ss = stokes_j;
    } else {
        sl = stokes_j;
        ss = stokes_i;
    }
    double eps = ss / sl;
    double y_a = 1.6;
    double y_s = 1.6015125;
    y_s += -0.63119577 * sl;
    y_s += 0.32938936 * sl * sl;
    y_s += -0.29847604 * sl * sl * sl;
    double v2 = 0.0;
    if (sl < 0.2 * re_inv) {
        v2 = vg_sq * (sl - ss) * (sl - ss) / re_inv;
    } else if (sl < re_inv / y_a) {
        v2 = vg_sq * (sl - ss) / (sl + ss);
        v2 *= (sl / (1.0 + re_inv / sl) - ss / (1.0 + re_inv / ss));
    } else if (sl < 5.0 * re_inv) {
        double c = (sl - ss) / (sl + ss);
        c *= (sl / (1.0 + y_a) - ss * ss / (ss + y_a * sl));
        c += 2.0 * (y_a * sl - re_inv) + sl / (1.0 + y_a);
        c -= sl * sl / (sl + re_inv);
        c += ss * ss / (y_a * sl + ss);
        c -= ss * ss / (ss + re_inv);
        v2 = vg_sq * c;
    } else if (sl < 0.2) {
        v2 = vg_sq * sl;
        v2 *= (2.0 * y_a - (1.0 + eps) + 2.0 / (1.0 + eps) * (1.0 / (1.0 + y_a) + eps * eps * eps / (y_a + eps)));
    } else if (sl < 1.0) {
        v2 = vg_sq * sl;
        v2 *= (2.0 * y_s - (1.0 + eps) + 2.0 / (1.0 + eps) * (1.0 / (1.0 + y_s) + eps * eps * eps / (y_s + eps)));
    } else {
        v2 = vg_sq * (1.0 / (1.0 + sl) + 1.0 / (1.0 + ss));
    }
    // the reference asserts on a negative square (_collision.cuh:266-270); NaN propagates here and
    // is reported by the chain's invalid-rate checks instead of trapping the GPU
    return sqrt(v2);
}

// si*fi - sj*fj of the radial drift (_collision.cuh:305, _col_rates.cuh:133), with the contraction
// pinned to one fused multiply-add: fma(si, fi, -(sj*fj)).  Under FMA contraction this difference is
// not zero for identical grains (it is the rounding residual of sj*fj), which gives a self pair a
// tiny positive speed; pinning it makes the host oracle reproduce the device value exactly.
__device__ __forceinline__ double drift_difference(double si, double fi, double sj, double fj) {
    return __fma_rn(si, fi, -__dmul_rn(sj, fj));
}

// _cache_query_environment (inc/swarm/_col_rates.cuh:13-24)
__device__ __forceinline__ Env make_env(const Model &m, double y, double z) {
    double R = cyl_R(m, y, z);
    double Z = cyl_Z(m, y, z);
    double h = get_hg(m, R);
    double omega = omega_k(m, R);
    double cs = sound_speed(m, R, h);
    double alpha = get_alpha(m, R, h);
    double strat = gas_strat(R, Z, h);
    Env e;
    e.Z = Z;
    e.omega = omega;
    e.vn = -get_eta(m, R, Z, h) * R * omega;
    e.radial = pow(R / m.R_0, m.idx_p);
    e.strat = strat;
    e.cs = cs;
    e.re_inv_sqrt = re_inv_sqrt(m, R, alpha, sigma_g(m, R) * strat);
    e.vg_sq = 1.5 * alpha * cs * cs;
    return e;
}

// Owner terms of _cached_pair_velocity (inc/swarm/_col_rates.cuh:127-141): the owner's Stokes
// number, drag factor and grain mass, the same for all of its pairs.
struct PairOwner {
    double si, fi, mi;
};

__device__ __forceinline__ PairOwner cached_owner_terms(const Model &m, const Env &e, double size_i) {
    PairOwner o;
    double si = m.stokes_0 * (size_i / m.S_0);
    si /= e.radial;
    si /= e.strat;
    o.si = si;
    o.fi = 1.0 / (1.0 + si * si);
    o.mi = grain_mass(m, size_i);
    return o;
}

// The partner's terms of _cached_pair_velocity at the owner's environment: its Stokes number, drag
// factor and grain mass.  They depend on the partner's frozen reservoir and the owner's position
// only, so a chain evaluates them once per owner instead of once per event.
struct PairPartner {
    double sj, fj, mj;
};

__device__ __forceinline__ PairPartner cached_partner_terms(const Model &m, const Env &e, double size_j) {
    PairPartner p;
    double sj = m.stokes_0 * (size_j / m.S_0);
    sj /= e.radial;
    sj /= e.strat;
    p.sj = sj;
    p.fj = 1.0 / (1.0 + sj * sj);
    p.mj = grain_mass(m, size_j);
    return p;
}

// _cached_pair_velocity from the owner's and the partner's terms (the same operations as below)
__device__ __forceinline__ double cached_pair_speed_pp(const Model &m, const Env &e, const PairOwner &o,
                                                       const PairPartner &p) {
    const double si = o.si, fi = o.fi, mi = o.mi;
    const double sj = p.sj, fj = p.fj, mj = p.mj;
    double dvr = 2.0 * e.vn * drift_difference(si, fi, sj, fj);
    double dvphi = e.vn * (fi - fj);
    double dvz = e.Z * e.omega * (fmin(si, 0.5) - fmin(sj, 0.5));
    double vt = oc07_speed(si, sj, e.re_inv_sqrt, e.vg_sq);
    double vb = fmin(sqrt(8.0 * e.cs * e.cs * m.m_mol * (mi + mj) / (M_PI * mi * mj)), e.cs);
    return sqrt(dvr * dvr + dvphi * dvphi + dvz * dvz + vt * vt + vb * vb);
}

// _cached_pair_velocity with the owner terms evaluated once
__device__ __forceinline__ double cached_pair_speed_o(const Model &m, const Env &e, const PairOwner &o,
                                                      double size_j) {
    return cached_pair_speed_pp(m, e, o, cached_partner_terms(m, e, size_j));
}

// _cached_pair_velocity (inc/swarm/_col_rates.cuh:127-141): physical units, analytic gas
__device__ __forceinline__ double cached_pair_speed(const Model &m, const Env &e, double size_i, double size_j) {
    return cached_pair_speed_o(m, e, cached_owner_terms(m, e, size_i), size_j);
}

// _get_vrel_pair (inc/swarm/_collision.cuh:277-325) for analytic gas: code units or CONST_ST
__device__ __forceinline__ double direct_pair_speed(const Model &m, double y, double z, double size_i, double size_j) {
    double R = cyl_R(m, y, z);
    double Z = cyl_Z(m, y, z);
    double h = get_hg(m, R);
    double omega = omega_k(m, R);
    double si = stokes_at(m, R, Z, h, size_i);
    double sj = stokes_at(m, R, Z, h, size_j);
    double vn = -get_eta(m, R, Z, h) * R * omega;
    double fi = 1.0 / (1.0 + si * si);
    double fj = 1.0 / (1.0 + sj * sj);
    double dvr = 2.0 * vn * drift_difference(si, fi, sj, fj);
    double dvphi = vn * (fi - fj);
    double dvz = Z * omega * (fmin(si, 0.5) - fmin(sj, 0.5));
    double sigma_local = sigma_g(m, R) * gas_strat(R, Z, h);
    // _get_vrel_t (_collision.cuh:153-273)
    double cs = sound_speed(m, R, h);
    double alpha = get_alpha(m, R, h);
    double rinv = re_inv_sqrt(m, R, alpha, sigma_local);
    double vt = oc07_speed(si, sj, rinv, 1.5 * alpha * cs * cs);
    double vb = 0.0;
    if (!m.code_unit) {
        // _get_vrel_b (_collision.cuh:119-133)
        double c = sound_speed(m, R, h);
        double mi = grain_mass(m, size_i);
        double mj = grain_mass(m, size_j);
        double v = sqrt(8.0 * c * c * m.m_mol * (mi + mj) / (M_PI * mi * mj));
        vb = fmin(v, c);
    }
    return sqrt(dvr * dvr + dvphi * dvphi + dvz * dvz + vt * vt + vb * vb);
}

// The environment cache is valid for analytic gas in physical units (_col_types.cuh:359-362).
__host__ __device__ __forceinline__ bool use_env_cache(const Model &m) { return !m.code_unit && !m.const_st; }

// Per-owner constants of one pair-rate evaluation.
struct OwnerCtx {
    double y, z;        // owner position (spherical radius, polar angle)
    double H_i;         // R_i * h_g(R_i), used by the vertically integrated physical kernel
    double measure;
    double lambda0;
    Env env;
};

// _get_col_chain_rate (inc/swarm/_col_rates.cuh:167-223) divided by the owner measure;
// vrel receives the pair speed for the fragmentation test (0 for synthetic kernels).
__device__ __forceinline__ double pair_rate(const Model &m, const OwnerCtx &o, double size_i, double size_j,
                                            double numr_j, const gd_particle *part, int j, double &vrel) {
    vrel = 0.0;
    double r;
    if (m.coag_kernel == GD_KERNEL_CONSTANT) {
        r = o.lambda0 * numr_j;
    } else if (m.coag_kernel == GD_KERNEL_LINEAR) {
        r = o.lambda0 * numr_j * (grain_mass(m, size_i) + grain_mass(m, size_j));
    } else if (m.coag_kernel == GD_KERNEL_PRODUCT) {
        r = o.lambda0 * numr_j * grain_mass(m, size_i) * grain_mass(m, size_j);
    } else {
        vrel = use_env_cache(m) ? cached_pair_speed(m, o.env, size_i, size_j)
                                : direct_pair_speed(m, o.y, o.z, size_i, size_j);
        r = numr_j * vrel * M_PI * (size_i + size_j) * (size_i + size_j) / 4.0;
        if (m.n_z == 1) {
            double R_j = cyl_R(m, part[j].position[1], part[j].position[2]);
            double H_gj = R_j * get_hg(m, R_j);
            r /= sqrt(2.0 * M_PI * (o.H_i * o.H_i + H_gj * H_gj));
        }
    }
    return r / o.measure;
}

// pair_rate for the physical kernel on the cached environment, with the owner terms evaluated once
__device__ __forceinline__ double pair_rate_cached(const Model &m, const OwnerCtx &o, const PairOwner &po,
                                                   double size_i, double size_j, double numr_j,
                                                   const gd_particle *part, int j, double &vrel) {
    vrel = cached_pair_speed_o(m, o.env, po, size_j);
    double r = numr_j * vrel * M_PI * (size_i + size_j) * (size_i + size_j) / 4.0;
    if (m.n_z == 1) {
        double R_j = cyl_R(m, part[j].position[1], part[j].position[2]);
        double H_gj = R_j * get_hg(m, R_j);
        r /= sqrt(2.0 * M_PI * (o.H_i * o.H_i + H_gj * H_gj));
    }
    return r / o.measure;
}

// _sticking_packet, _sticking_mass_ratio (inc/swarm/_col_event.cuh:242-252)
__device__ __forceinline__ double sticking_packet(double q) {
    return q > 0.0 && q <= 1.0e-06 ? fmax(1.0, floor(1.0e-04 / q)) : 1.0;
}
__device__ __forceinline__ double mass_ratio(double size_i, double size_j) {
    double ratio = size_j / size_i;
    return ratio * ratio * ratio;
}

// _erosion_outcome_moments (inc/swarm/_col_event.cuh:258-301)
__device__ __forceinline__ double outcome_moments(const Model &m, double si, double sj, bool high_speed, double &mean,
                                                  double &second, double &maximum) {
    double q = mass_ratio(si, sj);
    double G = sticking_packet(q);
    if (!high_speed) {
        mean = log1p(G * q) / 3.0;
        second = mean * mean;
        maximum = mean;
        return 1.0 / G;
    }
    if (q <= 0.1) {
        double remnant = (1.0 - q) / G;
        double debris = q;
        double factor = remnant + debris;
        double jr = -log1p(-G * q) / 3.0;
        double jd = -log(q) / 3.0;
        mean = (remnant * jr + debris * jd) / factor;
        second = (remnant * jr * jr + debris * jd * jd) / factor;
        maximum = fmax(jr, jd);
        return factor;
    }
    double L = 0.5 * log(si / m.init_smin);
    if (L < 1.0e-03) {
        mean = L - L * L / 6.0 + L * L * L * L / 360.0;
        second = L * L * (4.0 / 3.0 - L / 3.0 + L * L / 90.0 + L * L * L / 180.0);
    } else {
        double tail = exp(-L) / (-expm1(-L));
        mean = 2.0 * (1.0 - L * tail);
        second = 8.0 - (4.0 * L * L + 8.0 * L) * tail;
    }
    maximum = 2.0 * L;
    return 1.0;
}

// The COL_DIAGNOSTICS bookkeeping of one sampled outcome (_sample_erosion_outcome and
// _record_event_work, inc/swarm/_col_event.cuh:9-13, :306-336): category 0..3 sticking with
// q <= 1e-6, 1e-4, 1e-2 or above, 4 catastrophic fragmentation, 5 remnant erosion, 6 debris; and
// the event's log mass change.  si is the owner's diameter before the event, size_new after it.
__device__ __forceinline__ void outcome_category(const Model &m, double si, double sj, bool high_speed, double u,
                                                 double size_new, int &category, double &log_mass) {
    (void)m;
    const double q = mass_ratio(si, sj);
    const double G = sticking_packet(q);
    if (!high_speed) {
        category = q <= 1.0e-06 ? 0 : q <= 1.0e-04 ? 1 : q <= 1.0e-02 ? 2 : 3;
        log_mass = log1p(G * q);
        return;
    }
    if (q <= 0.1) {
        const double factor = (1.0 - q) / G + q;
        if (u < q / factor) {
            category = 6;
            log_mass = log(q);
        } else {
            category = 5;
            log_mass = log1p(-G * q);
        }
        return;
    }
    category = 4;
    log_mass = 3.0 * log(size_new / si);
}

// _sample_erosion_outcome (inc/swarm/_col_event.cuh:306-336): the new owner diameter
__device__ __forceinline__ double sample_outcome(const Model &m, double si, double sj, bool high_speed, double u) {
    double q = mass_ratio(si, sj);
    double G = sticking_packet(q);
    if (!high_speed) return cbrt(si * si * si + G * sj * sj * sj);
    if (q <= 0.1) {
        double factor = (1.0 - q) / G + q;
        if (u < q / factor) return sj;
        return si * cbrt(1.0 - G * q);
    }
    double lower = sqrt(m.init_smin);
    double root = lower + u * (sqrt(si) - lower);
    return fmin(si, fmax(m.init_smin, root * root));
}

}  // namespace gd
