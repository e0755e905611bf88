// gd_bridge.cuh -- drop-in bridge from a GameDev model directory to libgd_b200.
//
// A model that wants the B200 collision path adds this directory and ../../include to
// MODEL_INCLUDE_DIRS, links libgd_b200 (see flags.mk beside this file), and in its model-local
// swarm_runtime.cu (the reference already lets a model replace that translation unit,
// Makefile:302-309) replaces the body of the evolve_collisions lambda
// (src/swarm/swarm_runtime.cu:357-471) with
//
//     gd_bridge_evolve_collisions(dev_particle, dev_rngstate, duration, total_dust_mass,
//                                 col_geom_valid);
//
// and the controller reset at output boundaries (swarm_runtime.cu:490-496) with
// gd_bridge_reset_controller().  invalidate_col_geometry() keeps its meaning: it sets
// col_geom_valid = false, which the bridge forwards as gd_invalidate_geometry().
//
// Everything the bridge reads comes from the model's own const_defs.cuh (the reference's
// compile-time interface), so one model directory drives both the reference build and this one.
// Errors keep the reference's behaviour: a non-finite particle prints the reference's message and
// exits (swarm_runtime.cu:382-393); chain and controller errors throw std::runtime_error with the
// reference's wording (_col_chain.cuh:381-405).
#pragma once

#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <string>

#include <gd_b200.h>

// gd_config from the model's constexprs (inc/swarm/const_defs.cuh names)
inline gd_config gd_bridge_config() {
    gd_config c;
    gd_config_default(&c);
    c.G = G;
    c.M_S = M_S;
    c.R_0 = R_0;
    c.S_0 = S_0;
    c.n_x = N_X;
    c.n_y = N_Y;
    c.n_z = N_Z;
    c.x_min = X_MIN;
    c.x_max = X_MAX;
    c.y_min = Y_MIN;
    c.y_max = Y_MAX;
    c.z_min = Z_MIN;
    c.z_max = Z_MAX;
    c.sigma_0 = SIGMA_0;
    c.aspr_0 = ASPR_0;
    c.idx_p = IDX_P;
    c.idx_q = IDX_Q;
#ifdef CONST_NU
    c.const_nu = 1;
    c.nu = NU;
#else
    c.const_nu = 0;
    c.alpha = ALPHA;
#endif
#ifdef CODE_UNIT
    c.code_unit = 1;
    c.reynolds_0 = REYNOLDS_0;
#else
    c.code_unit = 0;
    c.m_mol = M_MOL;
    c.x_sec = X_SEC;
#endif
#ifdef HALF_DISK
    c.half_disk = 1;
#endif
#ifdef CONST_ST
    c.const_st = 1;
#endif
    c.stokes_0 = STOKES_0;
    c.rho_0 = RHO_0;
    c.coag_kernel = COAG_KERNEL;
    c.n_k = N_K;
    c.h_search = H_SEARCH;
    c.v_frag = V_FRAG;
    c.col_event_cap = COL_EVENT_CAP;
    c.col_bin_x = COL_BIN_X;
    c.col_bin_y = COL_BIN_Y;
    c.col_bin_z = COL_BIN_Z;
    c.col_bin_s = COL_BIN_S;
    c.col_bin_min = COL_BIN_MIN;
    c.col_bath_max = COL_BATH_MAX;
    c.col_bath_eps = COL_BATH_EPS;
    c.col_bath_alpha = COL_BATH_ALPHA;
#ifdef MULTISIZE
    c.init_smin = INIT_SMIN;
    c.init_smax = INIT_SMAX;
#endif
#ifdef COLLISION_MORTON
    c.search = GD_SEARCH_MORTON;
    c.morton_leaf_target = MORTON_LEAF_TARGET;
    c.morton_max_level = MORTON_MAX_LEVEL;
#else
    c.search = GD_SEARCH_KDTREE;
#endif
    return c;
}

// the handle lives for the process, like the reference's local_workspace (swarm_runtime.cu:341)
inline gd_handle *&gd_bridge_handle_slot() {
    static gd_handle *h = nullptr;
    return h;
}

inline gd_handle *gd_bridge_handle() {
    gd_handle *&h = gd_bridge_handle_slot();
    if (!h) {
        gd_config c = gd_bridge_config();
        gd_status st = gd_create(&c, N_P, &h);
        if (st != GD_OK) {
            std::cerr << "Error: libgd_b200 could not create the collision handle (status " << st << ")" << std::endl;
            std::exit(EXIT_FAILURE);
        }
    }
    return h;
}

inline std::string gd_bridge_message(gd_handle *h) {
    char buf[512];
    gd_last_error(h, buf, sizeof(buf));
    return std::string(buf);
}

// reference error behaviour for a failed call
inline void gd_bridge_raise(gd_handle *h, gd_status st) {
    if (st == GD_OK) return;
    long long detail = gd_error_detail(h);
    switch (st) {
    case GD_ERR_NONFINITE:
        std::cerr << "Error: non-finite particle state before collision search at particle " << detail << std::endl;
        std::exit(EXIT_FAILURE);
    case GD_ERR_CHAIN:
        throw std::runtime_error("local collision chain error " + std::to_string(detail));
    case GD_ERR_CONTINUATION_LIMIT:
        throw std::runtime_error("local collision continuation limit exceeded");
    case GD_ERR_TIME_RESOLUTION:
    case GD_ERR_CONTROLLER:
    case GD_ERR_INVALID_ARGUMENT:
        throw std::runtime_error(gd_bridge_message(h));
    default:
        std::cerr << "Error: CUDA failure in libgd_b200: " << gd_bridge_message(h) << std::endl;
        std::exit(EXIT_FAILURE);
    }
}

// evolve_collisions(duration) (swarm_runtime.cu:357-471): col_geom_valid is the caller's geometry
// epoch flag; it is false after any position update and true once the bridge rebuilt the index.
template <typename Particle, typename RngState>
inline void gd_bridge_evolve_collisions(Particle *dev_particle, RngState *dev_rngstate, double duration,
                                        double total_dust_mass, bool &col_geom_valid) {
    static_assert(sizeof(Particle) == sizeof(gd_particle), "the bridge needs the MULTISIZE swarm record");
    gd_handle *h = gd_bridge_handle();
    if (!col_geom_valid) gd_invalidate_geometry(h);
    gd_status st = gd_evolve_collisions(h, reinterpret_cast<gd_particle *>(dev_particle),
                                        static_cast<void *>(dev_rngstate), duration, total_dust_mass);
    gd_bridge_raise(h, st);
    col_geom_valid = true;
}

// restart the per-group controller memory at output boundaries (swarm_runtime.cu:490-496)
inline void gd_bridge_reset_controller() { gd_reset_controller(gd_bridge_handle()); }

inline void gd_bridge_release() {
    gd_handle *&h = gd_bridge_handle_slot();
    if (h) gd_destroy(h);
    h = nullptr;
}
