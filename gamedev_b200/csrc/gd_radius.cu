// Learned search-radius proposal: per-owner features, an 8 -> 64 -> 64 -> 1 GELU network with
// BF16 weights and FP32 accumulation, its forward / backward / Adam kernels, residual calibration
// and radius prediction.  The network predicts the CHANGE of the log K-th distance since the
// previous step: the proposal is feature 7 (that previous log distance, raw) plus the network's
// output.  Its output layer starts at zero, so an untrained network proposes the previous distance
// itself.  It is trained with the pinball loss of the kQuantile quantile, so it learns an upper
// bound per owner (how far that owner's K-th distance can move, which the local shear sets) rather
// than the mean; calibration then adds one global margin for the 0.999 coverage.  The proposal only seeds gd_knn_bounded, whose fallback keeps the
// neighbour lists identical to the plain query, so the network never changes a result.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "gd_geom_device.cuh"
#include "gd_internal.cuh"

namespace gd {

constexpr int kF = GD_RADIUS_FEATURES;  // 8
constexpr int kH = 64;
constexpr int kNP = GD_RADIUS_PARAMS;   // 4801
// flat parameter layout
constexpr int oW1 = 0;                  // [kH][kF]
constexpr int oB1 = oW1 + kH * kF;      // [kH]
constexpr int oW2 = oB1 + kH;           // [kH][kH], row = output unit
constexpr int oB2 = oW2 + kH * kH;      // [kH]
constexpr int oW3 = oB2 + kH;           // [kH]
constexpr int oB3 = oW3 + kH;           // scalar
static_assert(oB3 + 1 == kNP, "parameter layout");
constexpr int kTile = 128;              // samples per training block
constexpr float kQuantile = 0.99f;      // the quantile the pinball loss trains for
constexpr int kHistBins = 8192;
constexpr float kHistLo = -4.0f, kHistHi = 4.0f;
// Morton levels of the occupancy features: cells of 2^-9, 2^-12 and 2^-15 of the root cube
constexpr int kMortonLevel0 = 9, kMortonLevel1 = 12, kMortonLevel2 = 15;

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * __expf(-0.5f * x * x);
}
__device__ __forceinline__ bool is_weight(int p) {
    return (p >= oW1 && p < oB1) || (p >= oW2 && p < oB2) || (p >= oW3 && p < oB3);
}

// splitmix64: counter-based sampling and initialisation
__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

struct RadiusModel {
    double R_0 = 1.0;
    unsigned long long seed = 0;
    bool normalised = false;
    long long step = 0;
    DevBuf<float> params, grad, adam_m, adam_v;  // [kNP]
    DevBuf<__nv_bfloat16> wq;                    // bf16 weights (biases kept in fp32)
    DevBuf<float> norm;                          // mean[8], inv_scale[8], margin, target_mean
    DevBuf<double> acc;                          // reductions: loss, stats
    DevBuf<unsigned int> hist;                   // residual histogram
    DevBuf<int> err;                             // set by a tensor-core forward whose wait timed out
};

}  // namespace gd

struct gd_radius_model {
    gd::RadiusModel m;
};

namespace gd {

// ---------------------------------------------------------------------------------------------
// features (one warp per bucket of the handle's Morton order)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ int morton_run_count(const unsigned long long *key, int n, int i, int shift) {
    const unsigned long long p = key[i] >> shift;
    // gallop outwards, then bisect, for the run of keys sharing the prefix
    int lo = i, step = 1;
    while (lo - step >= 0 && (key[lo - step] >> shift) == p) {
        lo -= step;
        step <<= 1;
    }
    int a = lo - step < 0 ? 0 : lo - step, b = lo;  // key[b] matches, key[a] may not
    while (a < b) {
        int mid = (a + b) >> 1;
        if ((key[mid] >> shift) == p) b = mid;
        else a = mid + 1;
    }
    const int first = b;
    int hi = i;
    step = 1;
    while (hi + step < n && (key[hi + step] >> shift) == p) {
        hi += step;
        step <<= 1;
    }
    a = hi;
    b = hi + step >= n ? n - 1 : hi + step;  // key[a] matches
    while (a < b) {
        int mid = (a + b + 1) >> 1;
        if ((key[mid] >> shift) == p) a = mid;
        else b = mid - 1;
    }
    return a - first + 1;
}

__global__ void k_features(Model m, int slots, const int *__restrict__ counters, const float4 *__restrict__ sorted,
                           const unsigned long long *__restrict__ key, const gd_particle *__restrict__ part,
                           const float *__restrict__ prev_kth, double w_mean, float *__restrict__ feat) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= slots) return;  // whole warps: slots is a multiple of 32
    const int n_act = counters[0];
    const bool valid = i < n_act;
    int idx = 0, image = 0;
    double w = 0.0, y = 0.0, z = 0.0, size = 1.0;
    if (valid) {
        const int code = __float_as_int(sorted[i].w);
        idx = code / 3;
        image = code % 3;
        y = part[idx].position[1];
        z = part[idx].position[2];
        size = part[idx].par_size;
        w = part[idx].par_numr * M_PI * m.rho_0 * size * size * size / 6.0;
    }
    double wsum = w;
    int cnt = valid ? 1 : 0;
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        wsum += __shfl_xor_sync(0xffffffffu, wsum, off);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
    }
    if (!valid || image != 0) return;  // a wedge image's particle row is written by its own site
    float f[kF];
#pragma unroll
    for (int l = 0; l < 3; ++l) {
        const int level = (l == 0) ? kMortonLevel0 : (l == 1) ? kMortonLevel1 : kMortonLevel2;
        const int shift = 3 * (21 - level);
        f[l] = log2f(1.0f + static_cast<float>(morton_run_count(key, n_act, i, shift)));
    }
    const double R = cyl_R(m, y, z);
    f[3] = static_cast<float>(log(y / m.R_0));
    f[4] = (m.n_z > 1) ? static_cast<float>((z - 0.5 * M_PI) / get_hg(m, R)) : 0.0f;
    f[5] = static_cast<float>(log(size / m.S_0));
    f[6] = static_cast<float>(log(wsum / (cnt * w_mean)));
    float pk = 0.0f;
    if (prev_kth) {
        const float d2 = prev_kth[idx];
        pk = d2 > 0.0f ? static_cast<float>(0.5 * log(static_cast<double>(d2)) - log(m.R_0)) : 0.0f;
    }
    f[7] = pk;
    float4 *o = reinterpret_cast<float4 *>(feat + static_cast<size_t>(idx) * kF);
    o[0] = make_float4(f[0], f[1], f[2], f[3]);
    o[1] = make_float4(f[4], f[5], f[6], f[7]);
}

// ---------------------------------------------------------------------------------------------
// network
// ---------------------------------------------------------------------------------------------
__global__ void k_init_params(float *params, float *m1, float *m2, float *grad, unsigned long long seed) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kNP) return;
    float v = 0.0f;
    if (is_weight(p) && p < oW3) {  // the output layer W3 starts at zero
        const int fan_in = (p < oB1) ? kF : kH;
        // Box-Muller normal from two hashed uniforms, He-style scale
        const unsigned long long a = mix64(seed * 0x100000001b3ull + 2ull * p), b = mix64(a + 1ull);
        const double u1 = (static_cast<double>(a >> 11) + 1.0) * (1.0 / 9007199254740992.0);
        const double u2 = static_cast<double>(b >> 11) * (1.0 / 9007199254740992.0);
        v = static_cast<float>(sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2) * sqrt(2.0 / fan_in));
    }
    params[p] = v;
    m1[p] = 0.0f;
    m2[p] = 0.0f;
    grad[p] = 0.0f;
}

__global__ void k_quantise(const float *params, __nv_bfloat16 *wq) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < kNP) wq[p] = __float2bfloat16_rn(params[p]);
}

__device__ __forceinline__ float target_of(float kth_d2, double R_0) {
    return static_cast<float>(0.5 * log(static_cast<double>(kth_d2)) - log(R_0));
}
// the skip term of the output: the raw previous log K-th distance (feature 7; 0 when unknown)
__device__ __forceinline__ float base_of(const float *feat, size_t r) { return feat[r * kF + kF - 1]; }

// feature and target moments over rows with a valid target: acc[0..7] sum, [8..15] sum sq,
// [16] target sum, [17] count
__global__ void k_stats(const float *__restrict__ feat, const float *__restrict__ kth, int n, double R_0, double *acc) {
    __shared__ double part[18];
    if (threadIdx.x < 18) part[threadIdx.x] = 0.0;
    __syncthreads();
    double loc[18] = {};
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        if (!(kth[r] > 0.0f)) continue;
        for (int k = 0; k < kF; ++k) {
            const double x = feat[static_cast<size_t>(r) * kF + k];
            loc[k] += x;
            loc[kF + k] += x * x;
        }
        loc[16] += target_of(kth[r], R_0) - base_of(feat, static_cast<size_t>(r));
        loc[17] += 1.0;
    }
    for (int k = 0; k < 18; ++k) atomicAdd(&part[k], loc[k]);
    __syncthreads();
    if (threadIdx.x < 18) atomicAdd(&acc[threadIdx.x], part[threadIdx.x]);
}

__global__ void k_set_norm(const double *acc, float *norm, float *params) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double cnt = acc[17] > 0 ? acc[17] : 1.0;
    for (int k = 0; k < kF; ++k) {
        const double mean = acc[k] / cnt;
        const double var = acc[kF + k] / cnt - mean * mean;
        norm[k] = static_cast<float>(mean);
        norm[kF + k] = static_cast<float>(var > 1e-12 ? 1.0 / sqrt(var) : 1.0);
    }
    norm[2 * kF] = 0.0f;  // margin
    params[oB3] = static_cast<float>(acc[16] / cnt);
}

// weights of one block in shared memory: W1, b1, W2, b2, W3, b3 as float (weights from bf16)
__device__ __forceinline__ void load_net(float *sw, const float *params, const __nv_bfloat16 *wq) {
    for (int p = threadIdx.x; p < kNP; p += blockDim.x) sw[p] = is_weight(p) ? __bfloat162float(wq[p]) : params[p];
}

__device__ __forceinline__ void load_x(const float *feat, size_t r, const float *norm, float x[kF]) {
    const float4 *f = reinterpret_cast<const float4 *>(feat + r * kF);
    const float4 a = f[0], b = f[1];
    const float raw[kF] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
    for (int k = 0; k < kF; ++k) x[k] = (raw[k] - norm[k]) * norm[kF + k];
}

// Forward and backward of one tile of rows; accumulates the summed gradient of
// (1/norm_count) * sum pinball(y - t) into grad and the summed pinball loss into acc[0].
// rows: sample_mode 0 -> rows base..base+kTile-1 (bounded by n); 1 -> hashed uniform draws.
__global__ void __launch_bounds__(kTile) k_grad_tile(const float *__restrict__ params, const __nv_bfloat16 *__restrict__ wq,
                                                     const float *__restrict__ norm, const float *__restrict__ feat,
                                                     const float *__restrict__ kth, int n, double R_0, int sample_mode,
                                                     unsigned long long seed, long long step, float scale,
                                                     float *__restrict__ grad, double *__restrict__ acc) {
    extern __shared__ __align__(16) float sm[];
    float *sw = sm;                                   // kNP
    float *sx = sw + ((kNP + 3) & ~3);                // [kTile][kF]
    float *sh1 = sx + kTile * kF;                     // [kTile][kH + 1]
    float *sd1 = sh1 + kTile * (kH + 1);              // [kTile][kH + 1]
    float *sd2 = sd1 + kTile * (kH + 1);              // [kTile][kH + 1]
    float *sh2 = sd2 + kTile * (kH + 1);              // [kTile][kH + 1]
    float *sdy = sh2 + kTile * (kH + 1);              // [kTile]
    load_net(sw, params, wq);
    __syncthreads();
    const int t = threadIdx.x;
    const long long row_id = static_cast<long long>(blockIdx.x) * kTile + t;
    long long r = -1;
    if (sample_mode == 0) {
        if (row_id < n) r = row_id;
    } else {
        r = static_cast<long long>(mix64(seed ^ mix64(static_cast<unsigned long long>(step) * 0x9e3779b97f4a7c15ull +
                                                      static_cast<unsigned long long>(row_id))) %
                                   static_cast<unsigned long long>(n));
    }
    float x[kF] = {};
    float target = 0.0f, base = 0.0f;
    bool valid = false;
    if (r >= 0) {
        const float d2 = kth[r];
        valid = d2 > 0.0f;
        if (valid) {
            load_x(feat, static_cast<size_t>(r), norm, x);
            target = target_of(d2, R_0);
            base = base_of(feat, static_cast<size_t>(r));
        }
    }
    float *h1 = sh1 + t * (kH + 1), *d1 = sd1 + t * (kH + 1), *d2 = sd2 + t * (kH + 1), *h2 = sh2 + t * (kH + 1);
    for (int j = 0; j < kH; ++j) {
        float a = sw[oB1 + j];
#pragma unroll
        for (int k = 0; k < kF; ++k) a = fmaf(sw[oW1 + j * kF + k], x[k], a);
        h1[j] = gelu(a);
        d1[j] = gelu_grad(a);  // holds gelu'(a1) until the backward pass
    }
    float y = sw[oB3] + base;
    for (int o = 0; o < kH; ++o) {
        float a = sw[oB2 + o];
        for (int j = 0; j < kH; ++j) a = fmaf(sw[oW2 + o * kH + j], h1[j], a);
        const float g = gelu(a);
        h2[o] = g;
        d2[o] = gelu_grad(a);
        y = fmaf(sw[oW3 + o], g, y);
    }
    // pinball loss of the kQuantile quantile: tau * (t - y) above the output, (1 - tau) * (y - t) below
    const float err = valid ? (y - target) : 0.0f;
    const float dy = valid ? (err >= 0.0f ? (1.0f - kQuantile) : -kQuantile) * scale : 0.0f;
    const float pin = valid ? (err >= 0.0f ? (1.0f - kQuantile) * err : -kQuantile * err) : 0.0f;
    sdy[t] = dy;
    for (int o = 0; o < kH; ++o) d2[o] *= dy * sw[oW3 + o];
    for (int j = 0; j < kH; ++j) {
        float s = 0.0f;
        for (int o = 0; o < kH; ++o) s = fmaf(sw[oW2 + o * kH + j], d2[o], s);
        d1[j] *= s;
    }
#pragma unroll
    for (int k = 0; k < kF; ++k) sx[t * kF + k] = x[k];
    // pinball-loss sum of the tile
    float e2 = pin;
#pragma unroll
    for (int off = 16; off; off >>= 1) e2 += __shfl_xor_sync(0xffffffffu, e2, off);
    if ((t & 31) == 0) atomicAdd(&acc[0], static_cast<double>(e2));
    __syncthreads();
    // tile reductions: each thread owns a strided set of parameters
    for (int p = t; p < kNP; p += kTile) {
        float g = 0.0f;
        if (p < oB1) {
            const int j = p / kF, k = p % kF;
            for (int s = 0; s < kTile; ++s) g = fmaf(sd1[s * (kH + 1) + j], sx[s * kF + k], g);
        } else if (p < oW2) {
            const int j = p - oB1;
            for (int s = 0; s < kTile; ++s) g += sd1[s * (kH + 1) + j];
        } else if (p < oB2) {
            const int o = (p - oW2) / kH, j = (p - oW2) % kH;
            for (int s = 0; s < kTile; ++s) g = fmaf(sd2[s * (kH + 1) + o], sh1[s * (kH + 1) + j], g);
        } else if (p < oW3) {
            const int o = p - oB2;
            for (int s = 0; s < kTile; ++s) g += sd2[s * (kH + 1) + o];
        } else if (p < oB3) {
            const int o = p - oW3;
            for (int s = 0; s < kTile; ++s) g = fmaf(sdy[s], sh2[s * (kH + 1) + o], g);
        } else {
            for (int s = 0; s < kTile; ++s) g += sdy[s];
        }
        atomicAdd(&grad[p], g);
    }
}

__global__ void k_adam(float *params, float *grad, float *m1, float *m2, __nv_bfloat16 *wq, float lr, long long step) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kNP) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float g = grad[p];
    const float a = b1 * m1[p] + (1.0f - b1) * g;
    const float v = b2 * m2[p] + (1.0f - b2) * g * g;
    m1[p] = a;
    m2[p] = v;
    const float ah = a / (1.0f - powf(b1, static_cast<float>(step)));
    const float vh = v / (1.0f - powf(b2, static_cast<float>(step)));
    const float np = params[p] - lr * ah / (sqrtf(vh) + eps);
    params[p] = np;
    wq[p] = __float2bfloat16_rn(np);
    grad[p] = 0.0f;
}

// ---------------------------------------------------------------------------------------------
// Tensor-core forward on sm_100a (tcgen05).  One block of 128 threads per 128-row tile (a
// persistent loop over tiles); thread t owns row t of the tile.
//   1. Layer 1 (8 -> 64) and GELU on the CUDA cores.  Each FP32 activation h is split into two
//      BF16 parts, hi = bf16(h) and lo = bf16(h - hi), stored in shared memory as two A operands
//      (K-major, no swizzle): hi + lo carries about 16 significant bits, so the tensor-core layer
//      matches the FP32 forward to ~1e-5 instead of the ~1e-3 that BF16 activations alone give.
//   2. Layer 2 (64 x 64) as eight tcgen05.mma.kind::f16 (M = 128, N = 64, K = 16 each; hi and lo
//      times the same B): B = W2 (BF16 weights, exact), stored once per block, FP32 accumulator in
//      64 TMEM columns, issued by one thread and committed to an mbarrier.
//   3. Every warp reads its 32 accumulator rows (tcgen05.ld 32x32b, lane = row), adds b2, applies
//      GELU and the 64 -> 1 output layer on the CUDA cores.
// The waits are bounded: a commit that does not arrive within about a second stops the block,
// which sets *err, frees its TMEM and returns (gd_radius_model_check reports it).
// Operand layout (SWIZZLE_NONE canonical K-major): element (row, k) of a 64-column BF16 operand
// lies at (row / 8) * 1024 + (k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2 bytes: 8-row x 16-byte
// core matrices, K-adjacent ones 128 B apart (leading byte offset), 8-row groups 1024 B apart
// (stride byte offset).  One MMA consumes two K-adjacent core matrices (K = 16), so step ks starts
// 256 * ks bytes in.
// ---------------------------------------------------------------------------------------------
constexpr int kTcRows = 128;  // rows per tile = threads per block = TMEM lanes
constexpr int kTcCols = 64;   // TMEM columns of the FP32 accumulator (N)
// instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), A and B BF16 (bits 7-9,
// 10-12 = 1), both K-major (bits 15, 16 = 0), N / 8 in bits 17-22, M / 16 in bits 24-28
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24);
constexpr int kTcB = 0;                           // W2 (N = 64 rows x K = 64), 8 KB
constexpr int kTcA = 8192;                        // activations, hi part (128 rows x K = 64), 16 KB
constexpr int kTcAlo = kTcA + 16384;              // activations, lo part, 16 KB
constexpr int kTcW = kTcAlo + 16384;              // floats: W1 [512], b1 [64], b2 [64], W3 [64], b3, margin
constexpr int kTcWFloats = kH * kF + 3 * kH + 2;
constexpr int kTcBar = kTcW + ((kTcWFloats * 4 + 15) & ~15);  // mbarrier (8 B), TMEM address (4 B)
constexpr int kTcSmem = kTcBar + 16;

__host__ __device__ constexpr int tc_offset(int row, int k) {
    return (row >> 3) * 1024 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor: start address, leading byte offset 128, stride byte offset
// 1024 (all in 16-byte units), descriptor version 1 (bit 46), base offset 0, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3fffu) | (static_cast<uint64_t>(128 >> 4) << 16) |
           (static_cast<uint64_t>(1024 >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// waits for the completion of phase `parity` of the mbarrier at `bar`, for at most ~2^31 cycles
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity) {
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t"
            "}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > (1ll << 31)) return false;
    }
}

// 64 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_load64(uint32_t taddr, uint32_t v[64]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, %48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31]), "=r"(v[32]), "=r"(v[33]), "=r"(v[34]), "=r"(v[35]), "=r"(v[36]), "=r"(v[37]), "=r"(v[38]), "=r"(v[39]), "=r"(v[40]), "=r"(v[41]), "=r"(v[42]), "=r"(v[43]), "=r"(v[44]), "=r"(v[45]), "=r"(v[46]), "=r"(v[47]), "=r"(v[48]), "=r"(v[49]), "=r"(v[50]), "=r"(v[51]), "=r"(v[52]), "=r"(v[53]), "=r"(v[54]), "=r"(v[55]), "=r"(v[56]), "=r"(v[57]), "=r"(v[58]), "=r"(v[59]), "=r"(v[60]), "=r"(v[61]), "=r"(v[62]), "=r"(v[63])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__global__ void __launch_bounds__(kTcRows, 4) k_mlp_tc(const float *__restrict__ params,
                                                       const __nv_bfloat16 *__restrict__ wq,
                                                       const float *__restrict__ norm, const float *__restrict__ feat,
                                                       int n, double R_0, float *__restrict__ radius,
                                                       const float *__restrict__ kth, unsigned int *hist, int *err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int t = threadIdx.x, warp = t >> 5;
    float *sw = reinterpret_cast<float *>(smem + kTcW);
    float *w1 = sw, *b1 = sw + kH * kF, *b2 = b1 + kH, *w3 = b2 + kH;
    for (int p = t; p < kH * kF; p += kTcRows) w1[p] = __bfloat162float(wq[oW1 + p]);
    for (int j = t; j < kH; j += kTcRows) {
        b1[j] = params[oB1 + j];
        b2[j] = params[oB2 + j];
        w3[j] = __bfloat162float(wq[oW3 + j]);
    }
    if (t == 0) {
        w3[kH] = params[oB3];
        w3[kH + 1] = norm[2 * kF];  // margin
    }
    for (int p = t; p < kH * kH; p += kTcRows)  // W2[o][j]: row o of B (N), column j (K)
        *reinterpret_cast<__nv_bfloat16 *>(smem + kTcB + tc_offset(p / kH, p % kH)) = wq[oW2 + p];
    const uint32_t bar = smem_u32(smem + kTcBar);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + kTcBar + 8);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (t == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // W2 was written through the generic proxy: make it visible to the tensor core
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t a_addr = smem_u32(smem + kTcA), alo_addr = smem_u32(smem + kTcAlo), b_addr = smem_u32(smem + kTcB);
    const float b3 = w3[kH], margin = w3[kH + 1];
    const int tiles = (n + kTcRows - 1) / kTcRows;
    uint32_t parity = 0;
    bool failed = false;
    for (int tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const int r = tile * kTcRows + t;
        float x[kF];
#pragma unroll
        for (int k = 0; k < kF; ++k) x[k] = 0.0f;
        float base = 0.0f;
        if (r < n) {
            load_x(feat, static_cast<size_t>(r), norm, x);
            base = base_of(feat, static_cast<size_t>(r));
        }
#pragma unroll 1
        for (int kc = 0; kc < kH / 8; ++kc) {
            uint32_t ph[4], pl[4];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                float hi2[2], lo2[2];
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int j = kc * 8 + h * 2 + e;
                    float a = b1[j];
#pragma unroll
                    for (int k = 0; k < kF; ++k) a = fmaf(w1[j * kF + k], x[k], a);
                    const float v = gelu(a);
                    hi2[e] = __bfloat162float(__float2bfloat16_rn(v));
                    lo2[e] = v - hi2[e];  // exact in FP32
                }
                const __nv_bfloat162 bh = __floats2bfloat162_rn(hi2[0], hi2[1]);
                const __nv_bfloat162 bl = __floats2bfloat162_rn(lo2[0], lo2[1]);
                ph[h] = *reinterpret_cast<const uint32_t *>(&bh);
                pl[h] = *reinterpret_cast<const uint32_t *>(&bl);
            }
            *reinterpret_cast<uint4 *>(smem + kTcA + tc_offset(t, kc * 8)) = make_uint4(ph[0], ph[1], ph[2], ph[3]);
            *reinterpret_cast<uint4 *>(smem + kTcAlo + tc_offset(t, kc * 8)) = make_uint4(pl[0], pl[1], pl[2], pl[3]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_fence_before();
        __syncthreads();
        if (t == 0) {
            tc_fence_after();
#pragma unroll
            for (int ks = 0; ks < kH / 16; ++ks) {
                tc_mma(tmem, tc_desc(a_addr + 256 * ks), tc_desc(b_addr + 256 * ks), kTcIdesc, ks > 0 ? 1u : 0u);
                tc_mma(tmem, tc_desc(alo_addr + 256 * ks), tc_desc(b_addr + 256 * ks), kTcIdesc, 1u);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                         : "memory");
        }
        const bool ok = tc_wait(bar, parity);
        parity ^= 1u;
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        tc_fence_after();
        uint32_t acc[kTcCols];
        tc_load64(tmem + (static_cast<uint32_t>(warp * 32) << 16), acc);
        float y = b3 + base;
#pragma unroll
        for (int o = 0; o < kH; ++o) y = fmaf(w3[o], gelu(__uint_as_float(acc[o]) + b2[o]), y);
        if (r < n) {
            if (hist) {
                if (kth[r] > 0.0f) {
                    const float res = target_of(kth[r], R_0) - y;
                    int b = static_cast<int>(floorf((res - kHistLo) / (kHistHi - kHistLo) * kHistBins));
                    b = b < 0 ? 0 : (b >= kHistBins ? kHistBins + 1 : b + 1);  // [0] under, [bins+1] over
                    atomicAdd(&hist[b], 1u);
                }
            } else {
                radius[r] = static_cast<float>(R_0 * exp(static_cast<double>(y + margin)));
            }
        }
        // every row's accumulator is read before the next tile's MMA overwrites it
        tc_fence_before();
        __syncthreads();
    }
    if (failed && t == 0) atomicExch(err, 1);
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
}

static size_t tile_smem() {
    return sizeof(float) * (((kNP + 3) & ~3) + kTile * kF + 4 * kTile * (kH + 1) + kTile);
}

}  // namespace gd

using gd::RadiusModel;

namespace {

// The tensor-core forward over n rows: radii into `radius`, or (with `hist`) the residual histogram
// against kth.  A persistent grid of up to 4 blocks per SM (the launch bound; 4 x 64 TMEM columns).
cudaError_t launch_mlp(RadiusModel &m, const float *feat, int n, float *radius, const float *kth, unsigned int *hist,
                       cudaStream_t s) {
    static int sms[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!sms[dev]) {
        e = cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
    }
    const int tiles = (n + gd::kTcRows - 1) / gd::kTcRows;
    const int grid = tiles < 4 * sms[dev] ? tiles : 4 * sms[dev];
    gd::k_mlp_tc<<<grid, gd::kTcRows, gd::kTcSmem, s>>>(m.params.ptr, m.wq.ptr, m.norm.ptr, feat, n, m.R_0, radius, kth,
                                                       hist, m.err.ptr);
    return cudaGetLastError();
}

}  // namespace

extern "C" {

gd_status gd_radius_model_create(unsigned long long seed, double R_0, gd_radius_model **out) {
    if (!out || !(R_0 > 0)) return GD_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    gd_radius_model *h = new (std::nothrow) gd_radius_model();
    if (!h) return GD_ERR_OUT_OF_MEMORY;
    RadiusModel &m = h->m;
    m.R_0 = R_0;
    m.seed = seed;
    cudaError_t e = m.params.alloc(gd::kNP);
    if (e == cudaSuccess) e = m.grad.alloc(gd::kNP);
    if (e == cudaSuccess) e = m.adam_m.alloc(gd::kNP);
    if (e == cudaSuccess) e = m.adam_v.alloc(gd::kNP);
    if (e == cudaSuccess) e = m.wq.alloc(gd::kNP);
    if (e == cudaSuccess) e = m.norm.alloc(2 * gd::kF + 2);
    if (e == cudaSuccess) e = m.acc.alloc(32);
    if (e == cudaSuccess) e = m.hist.alloc(gd::kHistBins + 2);
    if (e == cudaSuccess) e = m.err.alloc(1);
    if (e == cudaSuccess) e = cudaMemset(m.err.ptr, 0, sizeof(int));
    if (e == cudaSuccess) {
        std::vector<float> norm(2 * gd::kF + 2, 0.0f);
        for (int k = 0; k < gd::kF; ++k) norm[gd::kF + k] = 1.0f;
        e = cudaMemcpy(m.norm.ptr, norm.data(), sizeof(float) * norm.size(), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) {
        gd::k_init_params<<<(gd::kNP + 255) / 256, 256>>>(m.params.ptr, m.adam_m.ptr, m.adam_v.ptr, m.grad.ptr, seed);
        gd::k_quantise<<<(gd::kNP + 255) / 256, 256>>>(m.params.ptr, m.wq.ptr);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) e = cudaFuncSetAttribute(gd::k_grad_tile, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(gd::tile_smem()));
    if (e != cudaSuccess) {
        delete h;
        return e == cudaErrorMemoryAllocation ? GD_ERR_OUT_OF_MEMORY : GD_ERR_CUDA;
    }
    *out = h;
    return GD_OK;
}

void gd_radius_model_destroy(gd_radius_model *m) { delete m; }

static gd_status ensure_norm(RadiusModel &m, const float *feat, const float *kth, int n, cudaStream_t s) {
    if (m.normalised) return GD_OK;
    if (cudaMemsetAsync(m.acc.ptr, 0, sizeof(double) * 32, s) != cudaSuccess) return GD_ERR_CUDA;
    gd::k_stats<<<592, 256, 0, s>>>(feat, kth, n, m.R_0, m.acc.ptr);
    gd::k_set_norm<<<1, 32, 0, s>>>(m.acc.ptr, m.norm.ptr, m.params.ptr);
    gd::k_quantise<<<(gd::kNP + 255) / 256, 256, 0, s>>>(m.params.ptr, m.wq.ptr);
    if (cudaGetLastError() != cudaSuccess) return GD_ERR_CUDA;
    m.normalised = true;
    return GD_OK;
}

gd_status gd_radius_model_train(gd_radius_model *h, const float *dev_features, const float *dev_kth_d2, int n,
                                int iterations, int batch, float lr, float *loss, void *stream) {
    if (!h || !dev_features || !dev_kth_d2 || n <= 0 || iterations < 0 || batch < gd::kTile || !(lr > 0))
        return GD_ERR_INVALID_ARGUMENT;
    RadiusModel &m = h->m;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    gd_status st = ensure_norm(m, dev_features, dev_kth_d2, n, s);
    if (st != GD_OK) return st;
    const int tiles = batch / gd::kTile;
    const float scale = 1.0f / static_cast<float>(tiles * gd::kTile);
    for (int it = 0; it < iterations; ++it) {
        ++m.step;
        if (it == iterations - 1 && cudaMemsetAsync(m.acc.ptr, 0, sizeof(double), s) != cudaSuccess) return GD_ERR_CUDA;
        gd::k_grad_tile<<<tiles, gd::kTile, gd::tile_smem(), s>>>(m.params.ptr, m.wq.ptr, m.norm.ptr, dev_features,
                                                                  dev_kth_d2, n, m.R_0, 1, m.seed, m.step, scale,
                                                                  m.grad.ptr, m.acc.ptr);
        gd::k_adam<<<(gd::kNP + 255) / 256, 256, 0, s>>>(m.params.ptr, m.grad.ptr, m.adam_m.ptr, m.adam_v.ptr,
                                                         m.wq.ptr, lr, m.step);
    }
    if (cudaGetLastError() != cudaSuccess) return GD_ERR_CUDA;
    if (loss) {
        double l = 0.0;
        if (cudaMemcpyAsync(&l, m.acc.ptr, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return GD_ERR_CUDA;
        *loss = static_cast<float>(l * scale);
    }
    return GD_OK;
}

gd_status gd_radius_model_gradient(gd_radius_model *h, const float *dev_features, const float *dev_kth_d2, int n,
                                   float *dev_grad, float *loss, void *stream) {
    if (!h || !dev_features || !dev_kth_d2 || n <= 0 || !dev_grad) return GD_ERR_INVALID_ARGUMENT;
    RadiusModel &m = h->m;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    gd_status st = ensure_norm(m, dev_features, dev_kth_d2, n, s);
    if (st != GD_OK) return st;
    if (cudaMemsetAsync(dev_grad, 0, sizeof(float) * gd::kNP, s) != cudaSuccess ||
        cudaMemsetAsync(m.acc.ptr, 0, sizeof(double), s) != cudaSuccess)
        return GD_ERR_CUDA;
    const int tiles = (n + gd::kTile - 1) / gd::kTile;
    const float scale = 1.0f / static_cast<float>(n);
    gd::k_grad_tile<<<tiles, gd::kTile, gd::tile_smem(), s>>>(m.params.ptr, m.wq.ptr, m.norm.ptr, dev_features,
                                                              dev_kth_d2, n, m.R_0, 0, m.seed, 0, scale, dev_grad,
                                                              m.acc.ptr);
    if (cudaGetLastError() != cudaSuccess) return GD_ERR_CUDA;
    if (loss) {
        double l = 0.0;
        if (cudaMemcpyAsync(&l, m.acc.ptr, sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return GD_ERR_CUDA;
        *loss = static_cast<float>(l * scale);
    }
    return GD_OK;
}

gd_status gd_radius_model_calibrate(gd_radius_model *h, const float *dev_features, const float *dev_kth_d2, int n,
                                    double quantile, float *margin, void *stream) {
    if (!h || !dev_features || !dev_kth_d2 || n <= 0 || !(quantile > 0) || !(quantile < 1))
        return GD_ERR_INVALID_ARGUMENT;
    RadiusModel &m = h->m;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    gd_status st = ensure_norm(m, dev_features, dev_kth_d2, n, s);
    if (st != GD_OK) return st;
    if (cudaMemsetAsync(m.hist.ptr, 0, sizeof(unsigned int) * (gd::kHistBins + 2), s) != cudaSuccess)
        return GD_ERR_CUDA;
    if (launch_mlp(m, dev_features, n, nullptr, dev_kth_d2, m.hist.ptr, s) != cudaSuccess) return GD_ERR_CUDA;
    std::vector<unsigned int> hist(gd::kHistBins + 2);
    if (cudaMemcpyAsync(hist.data(), m.hist.ptr, sizeof(unsigned int) * hist.size(), cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return GD_ERR_CUDA;
    const gd_status chk = gd_radius_model_check(h);
    if (chk != GD_OK) return chk;
    unsigned long long total = 0;
    for (unsigned int v : hist) total += v;
    if (total == 0) return GD_ERR_INVALID_ARGUMENT;
    // smallest bin upper edge that leaves at most (1 - quantile) of the residuals above it
    const unsigned long long need = static_cast<unsigned long long>(std::ceil(quantile * static_cast<double>(total)));
    unsigned long long run = 0;
    float mg = gd::kHistHi;
    for (int b = 0; b < gd::kHistBins + 2; ++b) {
        run += hist[b];
        if (run >= need) {
            if (b == 0) mg = gd::kHistLo;
            else if (b <= gd::kHistBins)
                mg = gd::kHistLo + (gd::kHistHi - gd::kHistLo) * static_cast<float>(b) / gd::kHistBins;
            else mg = 1e30f;  // residuals beyond the histogram: propose no bound
            break;
        }
    }
    if (cudaMemcpyAsync(m.norm.ptr + 2 * gd::kF, &mg, sizeof(float), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return GD_ERR_CUDA;
    if (margin) *margin = mg;
    return GD_OK;
}

gd_status gd_radius_model_predict(gd_radius_model *h, const float *dev_features, int n, float *dev_radius,
                                  void *stream) {
    if (!h || !dev_features || !dev_radius || n <= 0) return GD_ERR_INVALID_ARGUMENT;
    RadiusModel &m = h->m;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    return launch_mlp(m, dev_features, n, dev_radius, nullptr, nullptr, s) == cudaSuccess ? GD_OK : GD_ERR_CUDA;
}

gd_status gd_radius_model_check(gd_radius_model *h) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    int e = 0;
    if (cudaMemcpy(&e, h->m.err.ptr, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return GD_ERR_CUDA;
    return e ? GD_ERR_TIMEOUT : GD_OK;
}

gd_status gd_radius_model_get(const gd_radius_model *h, float *params, float *norm17) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    const RadiusModel &m = h->m;
    if (params && cudaMemcpy(params, m.params.ptr, sizeof(float) * gd::kNP, cudaMemcpyDeviceToHost) != cudaSuccess)
        return GD_ERR_CUDA;
    if (norm17 && cudaMemcpy(norm17, m.norm.ptr, sizeof(float) * (2 * gd::kF + 1), cudaMemcpyDeviceToHost) != cudaSuccess)
        return GD_ERR_CUDA;
    return GD_OK;
}

gd_status gd_radius_model_set(gd_radius_model *h, const float *params, const float *norm17) {
    if (!h) return GD_ERR_INVALID_ARGUMENT;
    RadiusModel &m = h->m;
    if (params) {
        if (cudaMemcpy(m.params.ptr, params, sizeof(float) * gd::kNP, cudaMemcpyHostToDevice) != cudaSuccess)
            return GD_ERR_CUDA;
        gd::k_quantise<<<(gd::kNP + 255) / 256, 256>>>(m.params.ptr, m.wq.ptr);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return GD_ERR_CUDA;
    }
    if (norm17) {
        if (cudaMemcpy(m.norm.ptr, norm17, sizeof(float) * (2 * gd::kF + 1), cudaMemcpyHostToDevice) != cudaSuccess)
            return GD_ERR_CUDA;
        m.normalised = true;
    }
    return GD_OK;
}

}  // extern "C"

// features need the handle's geometry: implemented beside the other geometry entry points
namespace gd {
Status radius_features(const Geometry &g, const Model &m, const gd_particle *part, const float *prev_kth,
                       double total_mass, float *feat, cudaStream_t s) {
    if (!g.sorted_key) return Status{GD_ERR_NOT_READY, "geometry not built", 0};
    const int slots = g.leaf_slots * kLeaf;
    // the mean bucket weight uses all n sites; inactive sites are a vanishing fraction
    const double w_mean = total_mass / static_cast<double>(g.n);
    k_features<<<(slots + 255) / 256, 256, 0, s>>>(m, slots, g.counters.ptr, g.sorted.ptr, g.sorted_key, part,
                                                   prev_kth, w_mean, feat);
    GD_TRY_CUDA(cudaGetLastError());
    return Status::ok();
}
}  // namespace gd
