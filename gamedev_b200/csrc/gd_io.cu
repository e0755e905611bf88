// Checkpoint I/O in the reference's on-disk formats, so that a run driven through this library
// writes and resumes the files GameDev writes and reads (inc/swarm/swarm_host.cuh:776-914,
// 1142-1205):
//   <prefix>particle_<frame>.dat   n 64-byte particle records, velocities as linear speeds;
//   <prefix>rngstate_<frame>.dat   n raw per-particle cuRAND XORWOW states.
// The frame number is zero padded to max(5, digits of save_max) (frame_num, :906-913).  Files are
// written and read in 64 MB chunks through a bounded host buffer and a read checks the exact file
// size first, as load_host_binary / load_device_binary do.  Host code only.
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
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

}  // extern "C"
