// Checkpoint I/O in the reference's on-disk formats, so that a run driven through this library
// writes and resumes the files GameDev writes and reads (inc/swarm/swarm_host.cuh:776-914,
// 1142-1205):
//   <prefix>particle_<frame>.dat   n 64-byte particle records, velocities as linear speeds;
//   <prefix>rngstate_<frame>.dat   n raw per-particle cuRAND XORWOW states.
// The frame number is zero padded to max(5, digits of save_max) (frame_num, :906-913).  Files are
// written and read in 64 MB chunks through a bounded host buffer and a read checks the exact file
// size first, as load_host_binary / load_device_binary do.  Host code only.
// Also the run's parameter file, variables.txt, as save_variable writes it (:989-1143).
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include "gd_geom_device.cuh"
#include "gd_internal.cuh"

namespace {

constexpr size_t kChunkBytes = 64ull << 20;

std::string frame_name(int idx_file, int save_max) {
    std::string num = std::to_string(idx_file);
    const size_t width = std::max<size_t>(5, std::to_string(save_max).size());
    if (num.size() < width) num.insert(0, width - num.size(), '0');
    return num;
}

// save_sam_as_velocity (swarm_host.cuh:864-880): R from the stored (y, z) first, then the inactive
// coordinates are pinned and the angular velocities become linear speeds
void to_file_layout(const gd::Model &m, gd_particle *p, int n) {
    for (int i = 0; i < n; ++i) {
        const double y = p[i].position[1];
        const double z = p[i].position[2];
        const double R = gd::cyl_R(m, y, z);
        if (m.n_x == 1) p[i].position[0] = 0.5 * (m.x_min + m.x_max);
        if (m.n_z == 1) p[i].position[2] = 0.5 * M_PI;
        p[i].velocity[0] = (R > 0.0) ? p[i].velocity[0] / R : 0.0;
        p[i].velocity[2] = (m.n_z > 1 && y > 0.0) ? p[i].velocity[2] / y : 0.0;
    }
}

// load_velocity_as_sam (swarm_host.cuh:883-899): the inactive coordinates are pinned first, then
// R from the pinned (y, z) turns the linear speeds back into angular velocities
void from_file_layout(const gd::Model &m, gd_particle *p, int n) {
    for (int i = 0; i < n; ++i) {
        if (m.n_x == 1) p[i].position[0] = 0.5 * (m.x_min + m.x_max);
        if (m.n_z == 1) p[i].position[2] = 0.5 * M_PI;
        const double y = p[i].position[1];
        const double z = p[i].position[2];
        const double R = gd::cyl_R(m, y, z);
        p[i].velocity[0] *= R;
        p[i].velocity[2] = (m.n_z > 1) ? p[i].velocity[2] * y : 0.0;
    }
}

bool file_size_is(std::FILE *f, size_t bytes) {
    if (std::fseek(f, 0, SEEK_END) != 0) return false;
    const long long sz = static_cast<long long>(std::ftell(f));
    if (std::fseek(f, 0, SEEK_SET) != 0) return false;
    return sz == static_cast<long long>(bytes);
}

// device buffer -> file, through a bounded host buffer
gd_status save_device(const std::string &name, const void *dev, size_t bytes) {
    std::FILE *f = std::fopen(name.c_str(), "wb");
    if (!f) return GD_ERR_IO;
    std::vector<unsigned char> buf(std::min(bytes, kChunkBytes));
    gd_status st = GD_OK;
    for (size_t off = 0; off < bytes && st == GD_OK; off += kChunkBytes) {
        const size_t len = std::min(kChunkBytes, bytes - off);
        if (cudaMemcpy(buf.data(), static_cast<const unsigned char *>(dev) + off, len, cudaMemcpyDeviceToHost) !=
            cudaSuccess)
            st = GD_ERR_CUDA;
        else if (std::fwrite(buf.data(), 1, len, f) != len)
            st = GD_ERR_IO;
    }
    if (std::fclose(f) != 0 && st == GD_OK) st = GD_ERR_IO;
    return st;
}

// file -> device buffer, after the exact size check
gd_status load_device(const std::string &name, void *dev, size_t bytes) {
    std::FILE *f = std::fopen(name.c_str(), "rb");
    if (!f) return GD_ERR_IO;
    gd_status st = file_size_is(f, bytes) ? GD_OK : GD_ERR_IO;
    std::vector<unsigned char> buf(std::min(bytes, kChunkBytes));
    for (size_t off = 0; off < bytes && st == GD_OK; off += kChunkBytes) {
        const size_t len = std::min(kChunkBytes, bytes - off);
        if (std::fread(buf.data(), 1, len, f) != len)
            st = GD_ERR_IO;
        else if (cudaMemcpy(static_cast<unsigned char *>(dev) + off, buf.data(), len, cudaMemcpyHostToDevice) !=
                 cudaSuccess)
            st = GD_ERR_CUDA;
    }
    std::fclose(f);
    return st;
}

}  // namespace

extern "C" {

gd_status gd_frame_name(int idx_file, int save_max, char *buf, size_t len) {
    if (idx_file < 0 || !buf || len == 0) return GD_ERR_INVALID_ARGUMENT;
    const std::string s = frame_name(idx_file, save_max);
    if (s.size() + 1 > len) return GD_ERR_INVALID_ARGUMENT;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return GD_OK;
}

gd_status gd_particles_to_file_layout(const gd_config *cfg, gd_particle *host, int n) {
    if (!cfg || !host || n < 0) return GD_ERR_INVALID_ARGUMENT;
    to_file_layout(gd::make_model(*cfg), host, n);
    return GD_OK;
}

gd_status gd_particles_from_file_layout(const gd_config *cfg, gd_particle *host, int n) {
    if (!cfg || !host || n < 0) return GD_ERR_INVALID_ARGUMENT;
    from_file_layout(gd::make_model(*cfg), host, n);
    return GD_OK;
}

gd_status gd_save_checkpoint(const gd_config *cfg, const char *prefix, int idx_file, int save_max,
                             const gd_particle *dev_particle, int n, const void *dev_rng) {
    if (!cfg || !prefix || !dev_particle || n <= 0 || idx_file < 0) return GD_ERR_INVALID_ARGUMENT;
    const gd::Model m = gd::make_model(*cfg);
    const std::string frame = frame_name(idx_file, save_max);
    // SAVE_PARTICLE_TO_FILE (swarm_host.cuh:1148-1175): the whole array to the host, converted
    std::vector<gd_particle> host(static_cast<size_t>(n));
    if (cudaMemcpy(host.data(), dev_particle, sizeof(gd_particle) * host.size(), cudaMemcpyDeviceToHost) !=
        cudaSuccess)
        return GD_ERR_CUDA;
    to_file_layout(m, host.data(), n);
    const std::string pname = std::string(prefix) + "particle_" + frame + ".dat";
    std::FILE *f = std::fopen(pname.c_str(), "wb");
    if (!f) return GD_ERR_IO;
    const size_t total = sizeof(gd_particle) * host.size();
    const unsigned char *bytes = reinterpret_cast<const unsigned char *>(host.data());
    gd_status st = GD_OK;
    for (size_t off = 0; off < total && st == GD_OK; off += kChunkBytes) {
        const size_t len = std::min(kChunkBytes, total - off);
        if (std::fwrite(bytes + off, 1, len, f) != len) st = GD_ERR_IO;
    }
    if (std::fclose(f) != 0 && st == GD_OK) st = GD_ERR_IO;
    if (st != GD_OK || !dev_rng) return st;
    return save_device(std::string(prefix) + "rngstate_" + frame + ".dat", dev_rng,
                       sizeof(curandState) * static_cast<size_t>(n));
}

gd_status gd_load_checkpoint(const gd_config *cfg, const char *prefix, int idx_file, int save_max,
                             gd_particle *dev_particle, int n, void *dev_rng) {
    if (!cfg || !prefix || !dev_particle || n <= 0 || idx_file < 0) return GD_ERR_INVALID_ARGUMENT;
    const gd::Model m = gd::make_model(*cfg);
    const std::string frame = frame_name(idx_file, save_max);
    // LOAD_PARTICLE_TO_VRAM (swarm_host.cuh:1178-1205)
    const std::string pname = std::string(prefix) + "particle_" + frame + ".dat";
    std::FILE *f = std::fopen(pname.c_str(), "rb");
    if (!f) return GD_ERR_IO;
    std::vector<gd_particle> host(static_cast<size_t>(n));
    const size_t total = sizeof(gd_particle) * host.size();
    gd_status st = file_size_is(f, total) ? GD_OK : GD_ERR_IO;
    unsigned char *bytes = reinterpret_cast<unsigned char *>(host.data());
    for (size_t off = 0; off < total && st == GD_OK; off += kChunkBytes) {
        const size_t len = std::min(kChunkBytes, total - off);
        if (std::fread(bytes + off, 1, len, f) != len) st = GD_ERR_IO;
    }
    std::fclose(f);
    if (st != GD_OK) return st;
    from_file_layout(m, host.data(), n);
    if (cudaMemcpy(dev_particle, host.data(), total, cudaMemcpyHostToDevice) != cudaSuccess) return GD_ERR_CUDA;
    if (!dev_rng) return GD_OK;
    return load_device(std::string(prefix) + "rngstate_" + frame + ".dat", dev_rng,
                       sizeof(curandState) * static_cast<size_t>(n));
}

// save_variable (inc/swarm/swarm_host.cuh:989-1143) for a collision build.  The file is read by the
// reference's Python tools, so its keys, spacing and number formats are the reference's: one
// stream, with the same format flags set in the same order, so that a value printed without its own
// manipulator (the INACTIVE_* lines) takes the state the previous line left, as it does there.
gd_status gd_save_variables(const gd_config *cfg, const gd_run_info *run, int n_p, double total_dust_mass,
                            const char *path) {
    if (!cfg || !run || !path || n_p <= 0 || cfg->n_k <= 0 || !(total_dust_mass > 0)) return GD_ERR_INVALID_ARGUMENT;
    const gd_config &c = *cfg;
    const gd_run_info &r = *run;
    std::ofstream f(path);
    if (!f) return GD_ERR_IO;
    auto sci = [&](const char *key, auto v) { f << key << std::scientific << std::setprecision(8) << v << '\n'; };
    auto dfl = [&](const char *key, auto v) { f << key << std::defaultfloat << std::setprecision(8) << v << '\n'; };
    f << "[PARAMETERS]\n\n";
    // gas
    sci("SIGMA_0     = ", c.sigma_0);
    sci("METAL_Z     = ", r.metal_z);
    dfl("ASPR_0      = ", c.aspr_0);
    dfl("IDX_P       = ", c.idx_p);
    dfl("IDX_Q       = ", c.idx_q);
    if (c.const_nu) sci("NU          = ", c.nu);
    else sci("ALPHA       = ", c.alpha);
    if (r.visc_flow) f << "VISC_FLOW   = " << std::defaultfloat << 1 << '\n';
    if (c.code_unit) {
        sci("REYNOLDS_0        = ", c.reynolds_0);
    } else {
        sci("M_MOL       = ", c.m_mol);
        sci("X_SEC       = ", c.x_sec);
    }
    f << '\n';
    // dust
    sci("STOKES_0    = ", c.stokes_0);
    sci("TOTAL_DUST_MASS = ", total_dust_mass);
    sci("RHO_0       = ", c.rho_0);
    if (r.radiation) {
        sci("BETA_0      = ", r.beta_0);
        sci("KAPPA_0     = ", r.kappa_0);
        sci("T_BETA      = ", r.t_beta);
        if (r.pr_effect) sci("C_LIGHT     = ", r.c_light);
    }
    if (r.diffusion) {
        sci("SCHMIDT_X   = ", r.schmidt_x);
        sci("SCHMIDT_R   = ", r.schmidt_r);
    }
    sci("SCHMIDT_Z   = ", r.schmidt_z);
    // collision
    sci("LAMBDA_0    = ", n_p / static_cast<double>(c.n_k) / total_dust_mass);
    sci("V_FRAG      = ", c.v_frag);
    dfl("COAG_KERNEL = ", c.coag_kernel);
    dfl("N_K         = ", c.n_k);
    dfl("H_SEARCH    = ", c.h_search);
    f << "COL_BATH_TPB  = " << r.col_bath_tpb << '\n';
    f << "COL_EVENT_CAP  = " << c.col_event_cap << '\n';
    sci("COL_BATH_MAX   = ", c.col_bath_max);
    sci("COL_BATH_EPS   = ", c.col_bath_eps);
    sci("COL_BATH_ALPHA = ", c.col_bath_alpha);
    f << "COL_CONTROLLER_AUDIT = path_integrated\n";
    f << "COL_CONTROLLER_FAILURE = two_consecutive_minimum_scale_overshoots\n";
    f << "COL_CONTROLLER_BINS = " << c.col_bin_x << " " << c.col_bin_y << " " << c.col_bin_z << " " << c.col_bin_s
      << '\n';
    f << "COL_BIN_MIN    = " << c.col_bin_min << '\n';
    f << "COL_SIZE_BIN_POLICY = moving_per_group\n";
    f << "COL_SIZE_RANGE_FACTORS = 0.5 8\n";
    f << "RNG_STREAM_POLICY = shared_per_particle\n";
    if (c.search == GD_SEARCH_MORTON) {
        f << "COLLISION_SEARCH = morton\n";
        f << "MORTON_LEAF_TARGET = " << c.morton_leaf_target << '\n';
        f << "MORTON_MAX_LEVEL   = " << c.morton_max_level << '\n';
    } else {
        f << "COLLISION_SEARCH = kdtree\n";
    }
    f << '\n';
    // mesh
    sci("N_P         = ", n_p);
    f << '\n';
    dfl("N_X         = ", c.n_x);
    dfl("X_MIN       = ", c.x_min);
    dfl("X_MAX       = ", c.x_max);
    f << '\n';
    dfl("N_Y         = ", c.n_y);
    dfl("Y_MIN       = ", c.y_min);
    dfl("Y_MAX       = ", c.y_max);
    f << '\n';
    dfl("N_Z         = ", c.n_z);
    dfl("Z_MIN       = ", c.z_min);
    dfl("Z_MAX       = ", c.z_max);
    f << '\n';
    sci("N_G         = ", c.n_x * c.n_y * c.n_z);
    f << '\n';
    if (c.n_x == 1 && c.n_z == 1) f << "GEOMETRY    = radial\n";
    if (c.n_x > 1 && c.n_z == 1) f << "GEOMETRY    = radial_azimuthal\n";
    if (c.n_x == 1 && c.n_z > 1) f << "GEOMETRY    = radial_polar\n";
    if (c.n_x > 1 && c.n_z > 1) f << "GEOMETRY    = full_3d\n";
    f << "DUST_DENSITY_KIND = " << ((c.n_z == 1) ? "surface" : "volume") << '\n';
    if (r.importgas) {
        f << "GAS_DENSITY_KIND  = " << ((c.n_z == 1) ? "surface" : "volume") << '\n';
        f << "IMPORTED_EPSILON_NORMALIZATION = shape_only\n";
    }
    if (c.n_x == 1) f << "INACTIVE_X  = " << 0.5 * (c.x_min + c.x_max) << '\n';
    if (c.n_z == 1) f << "INACTIVE_Z  = " << 0.5 * M_PI << '\n';
    if (c.n_x == 1 && c.n_z == 1) f << "DYNAMICAL_CLOSURE = midplane\n";
    f << '\n';
    // initial sizes
    if (r.multisize) {
        sci("INIT_SMIN   = ", c.init_smin);
        sci("INIT_SMAX   = ", c.init_smax);
    }
    f << '\n';
    // output cadence
    dfl("SAVE_MAX    = ", r.save_max);
    if (r.log_output) dfl("LOG_BASE    = ", r.out_base);
    else dfl("LIN_BASE    = ", r.out_base);
    sci("DT_OUT      = ", r.dt_out);
    if (r.transport) {
        sci("DT_MAX      = ", r.dt_max);
        dfl("CFL_DYN     = ", r.cfl_dyn);
    }
    f << '\n';
    // the particle record with linear velocities, as a configparser section of NumPy dtypes
    f << "[SWARM_DTYPE]\n";
    for (const char *name : {"position_x", "position_y", "position_z", "velocity_x", "velocity_y", "velocity_z"})
        f << name << " = f8\n";
    if (r.multisize) f << "par_size   = f8\npar_numr   = f8\n";
    f.flush();
    return f.good() ? GD_OK : GD_ERR_IO;
}

}  // extern "C"
