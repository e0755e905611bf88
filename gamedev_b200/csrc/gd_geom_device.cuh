// Device helpers of the geometry stage: active test, cylindrical coordinates, search radius,
// Morton keys, pinned single-precision distances and the FP64 ball measure.
#pragma once

#include <cuda_runtime.h>

#include "gd_internal.cuh"

namespace gd {

#define CUDART_INF_F_ __int_as_float(0x7f800000)

// _is_particle_active (inc/swarm/_transport.cuh:37-48)
__device__ __forceinline__ bool site_active(const Model &m, double y, double z) {
    if (y < m.y_min || y >= m.y_max) return false;
    if (m.n_z > 1) {
        if (m.half_disk) {
            if (z < m.z_min || z > m.z_max) return false;
        } else {
            if (z < m.z_min || z >= m.z_max) return false;
        }
    }
    return true;
}

// _get_cyl_R / _get_cyl_Z (inc/swarm/param_grid.cuh:236-241)
__host__ __device__ __forceinline__ double cyl_R(const Model &m, double y, double z) {
    return (m.n_z > 1) ? y * sin(z) : y;
}
__host__ __device__ __forceinline__ double cyl_Z(const Model &m, double y, double z) {
    return (m.n_z > 1) ? y * cos(z) : 0.0;
}

// _get_hg (inc/swarm/param_phys.cuh:70-72): aspect ratio h_g(R)
__host__ __device__ __forceinline__ double get_hg(const Model &m, double R) {
    return m.aspr_0 * pow(R / m.R_0, 0.5 * (m.idx_q + 1.0));
}

// Single-precision squared distance with the contraction pinned to the evaluation nvcc gives the
// reference's dx*dx + dy*dy + dz*dz (morton_types.cuh:76-82, kdtree/math.h:110-111,227-228) under
// its default -fmad=true: the first product of dx*dx + dy*dy is fused (fma(dx, dx, dy*dy)), then
// dz*dz is fused onto that sum.  The reference's compiled KD search on a B200 returns these bits
// (checked neighbour by neighbour by the reference-GPU parity test).  The host oracle evaluates
// the same fmaf chain.
__device__ __forceinline__ float dist2(const float3 &q, const float3 &p) {
    const float dx = __fsub_rn(q.x, p.x);
    const float dy = __fsub_rn(q.y, p.y);
    const float dz = __fsub_rn(q.z, p.z);
    return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
}

// Lower bound of dist2 over a box, with the same operation chain: every per-axis gap is at most
// the corresponding |q - p| of a contained site and rounding is monotone, so the bound never
// exceeds the computed dist2 of any site inside the box.  Empty boxes (lo = +inf) give +inf.
__device__ __forceinline__ float box_dist2(const float3 &q, const float4 &lo, const float4 &hi) {
    const float dx = fmaxf(fmaxf(__fsub_rn(lo.x, q.x), 0.0f), __fsub_rn(q.x, hi.x));
    const float dy = fmaxf(fmaxf(__fsub_rn(lo.y, q.y), 0.0f), __fsub_rn(q.y, hi.y));
    const float dz = fmaxf(fmaxf(__fsub_rn(lo.z, q.z), 0.0f), __fsub_rn(q.z, hi.z));
    return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
}

// Spread the low 21 bits of v so that bit b lands on bit 3b.
__device__ __forceinline__ unsigned long long spread3(unsigned int v) {
    unsigned long long x = v & 0x1fffffu;
    x = (x | (x << 32)) & 0x1f00000000ffffull;
    x = (x | (x << 16)) & 0x1f0000ff0000ffull;
    x = (x | (x << 8)) & 0x100f00f00f00f00full;
    x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
    x = (x | (x << 2)) & 0x1249249249249249ull;
    return x;
}

// 63-bit Morton key of a site on 2^21 cells per axis over the cube of half-width 1.0001*Y_MAX
// centred on the star (the reference's root cell, morton_ghost.cuh:176-183).  The key only orders
// sites for locality; results do not depend on it.
__device__ __forceinline__ unsigned long long morton_key(const Model &m, const float3 &p) {
    const float half = static_cast<float>(1.0001 * m.y_max);
    const float scale = 2097152.0f / (2.0f * half);
    const int top = 2097151;
    int ix = min(top, max(0, static_cast<int>((p.x + half) * scale)));
    int iy = min(top, max(0, static_cast<int>((p.y + half) * scale)));
    int iz = (m.dim == 2) ? 0 : min(top, max(0, static_cast<int>((p.z + half) * scale)));
    return spread3(ix) | (spread3(iy) << 1) | (spread3(iz) << 2);
}

// _get_ball_measure (inc/swarm/_collision.cuh:65-115): the part of the KNN ball inside the radial
// and polar domain bounds, revolved around the ring when the azimuth is collapsed.
__device__ __forceinline__ double ball_measure(const Model &m, double y, double z, double radius) {
    if (radius <= 0.0) return 0.0;
    if (m.n_x == 1 && m.n_z == 1) {
        double R_lo = fmax(m.y_min, y - radius);
        double R_hi = fmin(m.y_max, y + radius);
        return (R_hi > R_lo) ? M_PI * (R_hi * R_hi - R_lo * R_lo) : 0.0;
    }
    int dim = 1 + static_cast<int>(m.n_x > 1) + static_cast<int>(m.n_z > 1);
    double measure = (dim == 1) ? 2.0 * radius
                     : (dim == 2) ? M_PI * radius * radius
                                  : 4.0 * M_PI * radius * radius * radius / 3.0;
    double distances[4] = {y - m.y_min, m.y_max - y, 1.0e+100, 1.0e+100};
    if (m.n_z > 1) {
        distances[2] = y * (z - m.z_min);
        distances[3] = y * (m.z_max - z);
    }
    int bounds = (m.n_z > 1) ? 4 : 2;
    for (int b = 0; b < bounds; ++b) {
        double d = fmax(0.0, distances[b]);
        if (d >= radius) continue;
        if (dim == 1) {
            measure *= 0.5 * (1.0 + d / radius);
        } else if (dim == 2) {
            double cap = radius * radius * acos(d / radius) - d * sqrt(radius * radius - d * d);
            measure *= 1.0 - cap / (M_PI * radius * radius);
        } else {
            double cap = M_PI * (radius - d) * (radius - d) * (2.0 * radius + d) / 3.0;
            measure *= 1.0 - cap / (4.0 * M_PI * radius * radius * radius / 3.0);
        }
    }
    if (m.n_x == 1) measure *= 2.0 * M_PI * cyl_R(m, y, z);
    return measure;
}

}  // namespace gd
