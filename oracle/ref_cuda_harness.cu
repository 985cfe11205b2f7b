// Baseline only (never part of the product): the reference renderer's own GPU traversal,
// BVH::intersectRay through BVH::IntersectRayFunctor and thrust::transform — the kernel of its
// BVH::intersectRaysGpu (cuda_libraries/BVH.cu:541-584, 355-448) — compiled with the flags of
// its own build script (compile.sh: -O3 --use_fast_math -maxrregcount=64). The tree is the
// reference's: Morton sort + generateHierarchy + computeBoundingBoxes with its own member
// functions on the host (as ref_harness.cu does), then copied to the device with the
// triangles pointing at device vertex arrays, which is what its BVH constructor produces.
#include <thrust/device_vector.h>
#include <thrust/host_vector.h>
#include <thrust/sort.h>
#include <thrust/transform.h>
#include <thrust/sequence.h>
#include <thrust/random.h>
#include <thrust/functional.h>
#include <iostream>
#include <vector>
#include <random>
#include <string>
#include <fstream>
#include <thread>
#include <atomic>
#include <mutex>
#include <cmath>
#include <algorithm>
#include <unordered_map>
#include <sstream>
#include <queue>
#include <memory>
#include <functional>
#include <filesystem>
#include <chrono>
#include <bit>
#include <array>
#include <tuple>
#include <utility>
#include <cstdint>
#include <curand_kernel.h>
#include <math_constants.h>

#define swap ref_swap_
#include "cuda_libraries/types.h"
#include "shapes/Triangle.cu"
#include "cuda_libraries/BVH.cu"
#undef swap

#define REFG_API extern "C" __attribute__((visibility("default")))

namespace {
struct RefGpuBvh {
    uint32_t root = 0, ntri = 0;
    thrust::device_vector<Point3f> vertices;
    TriangleMeshData *d_mesh = nullptr;
    thrust::device_vector<Triangle> triangles;
    thrust::device_vector<BVH::Node> nodes;
    ~RefGpuBvh()
    {
        if (d_mesh) cudaFree(d_mesh);
    }
};
thread_local std::string g_error;
}  // namespace

REFG_API const char *refg_error() { return g_error.c_str(); }

// Builds the reference tree over one mesh and uploads it. Returns null on failure.
REFG_API void *refg_build(const float *xyz, uint32_t nv, const uint32_t *idx, uint32_t ntri)
{
    if (ntri < 2) {
        g_error = "need at least two triangles";
        return nullptr;
    }
    try {
        std::vector<Point3f> hv(nv);
        for (uint32_t i = 0; i < nv; i++) hv[i] = Point3f(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
        TriangleMeshData hmesh;
        hmesh.vertices = hv.data();
        thrust::host_vector<Triangle> tris(ntri);
        for (uint32_t t = 0; t < ntri; t++) {
            int vi[3] = {(int)idx[3 * t], (int)idx[3 * t + 1], (int)idx[3 * t + 2]};
            Triangle tri(vi);
            tri.mesh = &hmesh;
            tri.meshId = 0;
            tri.isTransparent = false;
            tris[t] = tri;
        }
        Bound3f world = Bound3f();
        for (uint32_t t = 0; t < ntri; t++) world = world + triangleWorldBoundFunctor()(tris[t]);
        Morton3DFunctor morton(world);
        std::vector<std::pair<unsigned int, unsigned int>> keyed(ntri);
        for (uint32_t t = 0; t < ntri; t++) keyed[t] = {morton(tris[t]), t};
        std::sort(keyed.begin(), keyed.end());
        thrust::host_vector<unsigned int> codes(ntri), sorted(ntri);
        for (uint32_t t = 0; t < ntri; t++) {
            codes[t] = keyed[t].first;
            sorted[t] = keyed[t].second;
        }
        thrust::host_vector<BVH::Node> nodes(2 * ntri - 1);
        for (uint32_t i = 0; i < ntri; i++) BVH::initializeLeaf(i, nodes.data(), tris.data(), sorted.data());
        alignas(BVH) static unsigned char storage[sizeof(BVH)];
        BVH *shell = reinterpret_cast<BVH *>(storage);
        RefGpuBvh *b = new RefGpuBvh();
        b->root = shell->generateHierarchy(codes, sorted, nodes, ntri);
        shell->computeBoundingBoxes(nodes, ntri);
        b->ntri = ntri;
        b->vertices = thrust::device_vector<Point3f>(hv.begin(), hv.end());
        TriangleMeshData dmesh;
        dmesh.vertices = b->vertices.data().get();
        if (cudaMalloc(&b->d_mesh, sizeof dmesh) != cudaSuccess ||
            cudaMemcpy(b->d_mesh, &dmesh, sizeof dmesh, cudaMemcpyHostToDevice) != cudaSuccess) {
            delete b;
            g_error = "device mesh upload failed";
            return nullptr;
        }
        for (uint32_t t = 0; t < ntri; t++) tris[t].mesh = b->d_mesh;
        b->triangles = tris;
        b->nodes = nodes;
        return b;
    } catch (const std::exception &e) {
        g_error = e.what();
        return nullptr;
    }
}

REFG_API void refg_free(void *h) { delete static_cast<RefGpuBvh *>(h); }

// Traces n rays (origin xyz, direction xyz per ray) with the reference's GPU traversal.
// out_ids: its hit ids (-1: miss). ms_kernel: average time of the transform over `reps`
// launches with the rays resident on the device; ms_api: average time of the reference's
// per-call path (rays copied to the device, transform, ids copied back), as
// BVH::intersectRaysGpu does it. Returns 0, or 1 with refg_error() set.
REFG_API int refg_trace(void *h, const float *od, uint64_t n, int32_t reps, int32_t *out_ids, float *ms_kernel,
                        float *ms_api)
{
    RefGpuBvh *b = static_cast<RefGpuBvh *>(h);
    try {
        thrust::host_vector<Ray> rays(n);
        for (uint64_t i = 0; i < n; i++)
            rays[i] = Ray(Point3f(od[6 * i], od[6 * i + 1], od[6 * i + 2]),
                          Vector3f(od[6 * i + 3], od[6 * i + 4], od[6 * i + 5]));
        auto functor = BVH::IntersectRayFunctor(b->root, b->nodes.data().get(), b->triangles.data().get(), false);
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        thrust::device_vector<Ray> d_rays(rays);
        thrust::device_vector<int> d_ids(n);
        thrust::transform(d_rays.begin(), d_rays.end(), d_ids.begin(), functor);  // warm-up
        cudaDeviceSynchronize();
        cudaEventRecord(e0);
        for (int r = 0; r < reps; r++) thrust::transform(d_rays.begin(), d_rays.end(), d_ids.begin(), functor);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        *ms_kernel = ms / (float)reps;
        thrust::host_vector<int> ids;
        cudaEventRecord(e0);
        for (int r = 0; r < reps; r++) {
            thrust::device_vector<Ray> s(rays);
            thrust::device_vector<int> o(n);
            thrust::transform(s.begin(), s.end(), o.begin(), functor);
            ids = o;
        }
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        *ms_api = ms / (float)reps;
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        for (uint64_t i = 0; i < n; i++) out_ids[i] = ids[i];
        cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) {
            g_error = cudaGetErrorString(err);
            return 1;
        }
        return 0;
    } catch (const std::exception &e) {
        g_error = e.what();
        return 1;
    }
}
