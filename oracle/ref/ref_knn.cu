// Reference-GPU neighbour cache over given sites: the reference's own KD builder
// (kdtree::buildTree, inc/swarm/kdtree/builder.h:109-152) and its top-K heap and traversal
// (kdtree/index_heap.cuh:16-177, kdtree::cct::knn in kdtree/knn.h:429-442), driven the way
// col_cache_get drives them (inc/swarm/_col_cache.cuh:15-71: one thread per tree node, search
// distance q_i, active filter, codes in heap order).  Compiled from the GameDev tree where it lies by
// oracle/ref/Makefile into oracle/_ref/ref_knn.  TEST INFRASTRUCTURE ONLY: it pins the B200 search
// against the reference's own CUDA build on the same GPU and times that build.
//
//   ref_knn <in.bin> <out.bin|-> <repeats>
//   in.bin : int32 n, int32 K, float32 site[n][4] (x, y, z, unused), float32 q[n], uint8 active[n]
//   out.bin: int32 codes[n][K], float32 d2[n][K] (heap order, as col_cache_get writes them)
//   stdout : one JSON line {"n", "k", "build_ms", "query_ms", "queries"}; query_ms is the mean of
//            `repeats` timed launches after one untimed launch.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include <gpu.cuh>

#include <kdtree/builder.h>
#include <kdtree/knn.h>

#include <knn_types.cuh>

namespace {

using ref_box = kdtree::box_t<float3>;

void check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

__global__ void init_nodes(kdtree_point *node, const float4 *site, int n) {
    int i = threadIdx.x + blockDim.x * blockIdx.x;
    if (i >= n) return;
    node[i].cartesian = make_float3(site[i].x, site[i].y, site[i].z);
    node[i].idx_old = i;
    node[i].split_dim = 0;
    node[i].image = 0;
}

template <int K>
__global__ void cache_get(int *codes, float *d2, const kdtree_point *node, const ref_box *box,
                          const unsigned char *active, const float *q, int n, int write) {
    int t = threadIdx.x + blockDim.x * blockIdx.x;
    if (t >= n) return;
    int i = node[t].idx_old;
    if (active[i] == 0) {
        if (write)
            for (int k = 0; k < K; ++k) {
                codes[static_cast<size_t>(i) * K + k] = -1;
                d2[static_cast<size_t>(i) * K + k] = 0.0f;
            }
        return;
    }
    kdtree_heap<K> heap(q[i], node, false, active);
    kdtree::cct::knn<kdtree_heap<K>, kdtree_point, kdtree_traits>(heap, node[t].cartesian, *box, node, n);
    if (write) {
        for (int k = 0; k < K; ++k) {
            codes[static_cast<size_t>(i) * K + k] = heap.returnNeighbor(k);
            d2[static_cast<size_t>(i) * K + k] = heap.returnDist2(k);
        }
    } else {
        // keep the heap live without the output traffic (the reference's KNN harness times its
        // queries the same way, val/swarm/mod/test_knn/knn_benchmark.cu:122-145)
        float s = 0.0f;
        for (int k = 0; k < K; ++k) s += heap.returnDist2(k);
        d2[i] = s;
    }
}

template <int K>
float run(int *codes, float *d2, const kdtree_point *node, const ref_box *box, const unsigned char *active,
          const float *q, int n, int write, int repeats) {
    const int tpb = kdtree_heap<K>::threads;
    const int blocks = (n + tpb - 1) / tpb;
    cache_get<K><<<blocks, tpb>>>(codes, d2, node, box, active, q, n, write);
    check(cudaGetLastError(), "launch cache_get");
    check(cudaDeviceSynchronize(), "run cache_get");
    cudaEvent_t a, b;
    check(cudaEventCreate(&a), "event");
    check(cudaEventCreate(&b), "event");
    float total = 0.0f;
    for (int r = 0; r < repeats; ++r) {
        check(cudaEventRecord(a), "record");
        cache_get<K><<<blocks, tpb>>>(codes, d2, node, box, active, q, n, write);
        check(cudaEventRecord(b), "record");
        check(cudaEventSynchronize(b), "sync");
        float ms = 0.0f;
        check(cudaEventElapsedTime(&ms, a, b), "elapsed");
        total += ms;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return repeats > 0 ? total / repeats : 0.0f;
}

}  // namespace

int main(int argc, char **argv) {
    try {
        if (argc != 4) throw std::runtime_error("usage: ref_knn <in.bin> <out.bin|-> <repeats>");
        std::ifstream in(argv[1], std::ios::binary);
        if (!in) throw std::runtime_error("cannot open input");
        int n = 0, K = 0;
        in.read(reinterpret_cast<char *>(&n), 4);
        in.read(reinterpret_cast<char *>(&K), 4);
        if (n <= 0 || K <= 0) throw std::runtime_error("bad header");
        std::vector<float> site(static_cast<size_t>(n) * 4), q(n);
        std::vector<unsigned char> active(n);
        in.read(reinterpret_cast<char *>(site.data()), site.size() * 4);
        in.read(reinterpret_cast<char *>(q.data()), q.size() * 4);
        in.read(reinterpret_cast<char *>(active.data()), active.size());
        if (!in) throw std::runtime_error("short input");
        const bool write = std::strcmp(argv[2], "-") != 0;
        const int repeats = std::atoi(argv[3]);

        float4 *d_site = nullptr;
        float *d_q = nullptr, *d_d2 = nullptr;
        unsigned char *d_active = nullptr;
        int *d_codes = nullptr;
        kdtree_point *d_node = nullptr;
        ref_box *d_box = nullptr;
        const size_t rows = static_cast<size_t>(n) * K;
        check(cudaMalloc(&d_site, sizeof(float4) * n), "alloc sites");
        check(cudaMalloc(&d_q, sizeof(float) * n), "alloc q");
        check(cudaMalloc(&d_active, n), "alloc active");
        check(cudaMalloc(&d_node, sizeof(kdtree_point) * n), "alloc nodes");
        check(cudaMalloc(&d_box, sizeof(ref_box)), "alloc box");
        check(cudaMalloc(&d_d2, sizeof(float) * (write ? rows : static_cast<size_t>(n))), "alloc d2");
        if (write) check(cudaMalloc(&d_codes, sizeof(int) * rows), "alloc codes");
        check(cudaMemcpy(d_site, site.data(), sizeof(float4) * n, cudaMemcpyHostToDevice), "copy sites");
        check(cudaMemcpy(d_q, q.data(), sizeof(float) * n, cudaMemcpyHostToDevice), "copy q");
        check(cudaMemcpy(d_active, active.data(), n, cudaMemcpyHostToDevice), "copy active");

        cudaEvent_t a, b;
        check(cudaEventCreate(&a), "event");
        check(cudaEventCreate(&b), "event");
        check(cudaEventRecord(a), "record");
        init_nodes<<<(n + 255) / 256, 256>>>(d_node, d_site, n);
        check(cudaGetLastError(), "launch init_nodes");
        kdtree::buildTree<kdtree_point, kdtree_traits>(d_node, n, d_box);
        check(cudaEventRecord(b), "record");
        check(cudaEventSynchronize(b), "build");
        float build_ms = 0.0f;
        check(cudaEventElapsedTime(&build_ms, a, b), "elapsed");

        float query_ms = 0.0f;
        const int w = write ? 1 : 0;
        switch (K) {
        case 8: query_ms = run<8>(d_codes, d_d2, d_node, d_box, d_active, d_q, n, w, repeats); break;
        case 12: query_ms = run<12>(d_codes, d_d2, d_node, d_box, d_active, d_q, n, w, repeats); break;
        case 16: query_ms = run<16>(d_codes, d_d2, d_node, d_box, d_active, d_q, n, w, repeats); break;
        case 20: query_ms = run<20>(d_codes, d_d2, d_node, d_box, d_active, d_q, n, w, repeats); break;
        case 24: query_ms = run<24>(d_codes, d_d2, d_node, d_box, d_active, d_q, n, w, repeats); break;
        case 32: query_ms = run<32>(d_codes, d_d2, d_node, d_box, d_active, d_q, n, w, repeats); break;
        case 64: query_ms = run<64>(d_codes, d_d2, d_node, d_box, d_active, d_q, n, w, repeats); break;
        case 200: query_ms = run<200>(d_codes, d_d2, d_node, d_box, d_active, d_q, n, w, repeats); break;
        case 256: query_ms = run<256>(d_codes, d_d2, d_node, d_box, d_active, d_q, n, w, repeats); break;
        default: throw std::runtime_error("K not instantiated: " + std::to_string(K));
        }
        if (write) {
            std::vector<int> codes(rows);
            std::vector<float> d2(rows);
            check(cudaMemcpy(codes.data(), d_codes, sizeof(int) * rows, cudaMemcpyDeviceToHost), "copy codes");
            check(cudaMemcpy(d2.data(), d_d2, sizeof(float) * rows, cudaMemcpyDeviceToHost), "copy d2");
            std::ofstream out(argv[2], std::ios::binary);
            out.write(reinterpret_cast<const char *>(codes.data()), rows * 4);
            out.write(reinterpret_cast<const char *>(d2.data()), rows * 4);
            if (!out) throw std::runtime_error("cannot write output");
        }
        long long queries = 0;
        for (unsigned char v : active) queries += v ? 1 : 0;
        std::printf("{\"n\": %d, \"k\": %d, \"build_ms\": %.4f, \"query_ms\": %.4f, \"queries\": %lld}\n", n, K,
                    build_ms, query_ms, queries);
        cudaFree(d_site); cudaFree(d_q); cudaFree(d_active); cudaFree(d_node); cudaFree(d_box); cudaFree(d_d2);
        if (d_codes) cudaFree(d_codes);
        return 0;
    } catch (const std::exception &e) {
        std::fprintf(stderr, "ref_knn: %s\n", e.what());
        return 1;
    }
}
