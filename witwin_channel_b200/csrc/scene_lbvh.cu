// Device BVH rebuild: a linear BVH from Morton codes of the face centroids,
// built entirely on the GPU (Karras, "Maximizing Parallelism in the
// Construction of BVHs, Octrees, and k-d Trees", HPG 2012), then boxed
// bottom-up by the refit's kernel.  The tree has the compiled scene's layout
// (F-1 internal nodes of 64 bytes, one triangle per leaf, leaves in tree
// order), so every traversal kernel uses it unchanged.
//
// The host SAH build of the compile gives faster traversal on most scenes; this
// rebuild replaces it without a host round trip, e.g. after refits that moved
// the geometry far enough to degrade the tree.

#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"
#include "scene.cuh"

namespace wcb {

namespace lbvh {

constexpr int kB = 256;

// centroid bounds of all faces (one block)
__global__ void k_centroid_bounds(const float* v, const int* faces, int F, float* bounds) {
    __shared__ float slo[3][kB], shi[3][kB];
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int f = threadIdx.x; f < F; f += blockDim.x)
        for (int k = 0; k < 3; ++k) {
            const float c = (v[3 * faces[3 * f] + k] + v[3 * faces[3 * f + 1] + k] + v[3 * faces[3 * f + 2] + k]) *
                             (1.0f / 3.0f);
            lo[k] = fminf(lo[k], c);
            hi[k] = fmaxf(hi[k], c);
        }
    for (int k = 0; k < 3; ++k) {
        slo[k][threadIdx.x] = lo[k];
        shi[k][threadIdx.x] = hi[k];
    }
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
            for (int k = 0; k < 3; ++k) {
                slo[k][threadIdx.x] = fminf(slo[k][threadIdx.x], slo[k][threadIdx.x + s]);
                shi[k][threadIdx.x] = fmaxf(shi[k][threadIdx.x], shi[k][threadIdx.x + s]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 3; ++k) {
            bounds[k] = slo[k][0];
            bounds[3 + k] = shi[k][0];
        }
}

// 10 bits spread to every third bit
WCB_D unsigned spread10(unsigned x) {
    x = (x * 0x00010001u) & 0xFF0000FFu;
    x = (x * 0x00000101u) & 0x0F00F00Fu;
    x = (x * 0x00000011u) & 0xC30C30C3u;
    x = (x * 0x00000005u) & 0x49249249u;
    return x;
}

// key = 30-bit Morton code of the normalised centroid << 32 | face index
// (unique keys, so the tree is fully determined)
__global__ void k_morton(const float* v, const int* faces, int F, const float* bounds, unsigned long long* keys,
                         int* vals) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= F) return;
    unsigned q[3];
    for (int k = 0; k < 3; ++k) {
        const float c = (v[3 * faces[3 * f] + k] + v[3 * faces[3 * f + 1] + k] + v[3 * faces[3 * f + 2] + k]) *
                        (1.0f / 3.0f);
        const float ext = bounds[3 + k] - bounds[k];
        const float u = ext > 0.0f ? (c - bounds[k]) / ext : 0.0f;
        q[k] = unsigned(fminf(fmaxf(u * 1024.0f, 0.0f), 1023.0f));
    }
    const unsigned code = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
    keys[f] = (static_cast<unsigned long long>(code) << 32) | static_cast<unsigned>(f);
    vals[f] = f;
}

WCB_D int common_prefix(const unsigned long long* keys, int F, long long a, long long b) {
    if (b < 0 || b >= F) return -1;
    return __clzll(keys[a] ^ keys[b]);
}

// internal node i of the radix tree over the sorted keys: its range, its
// split and its two children (internal index, or ~leaf slot)
__global__ void k_karras(const unsigned long long* keys, int F, BvhNode* nodes, int* leaf_parent, int* node_parent) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F - 1) return;
    const int d = common_prefix(keys, F, i, i + 1) - common_prefix(keys, F, i, i - 1) >= 0 ? 1 : -1;
    const int dmin = common_prefix(keys, F, i, (long long)i - d);
    long long lmax = 2;
    while (common_prefix(keys, F, i, i + lmax * d) > dmin) lmax <<= 1;
    long long l = 0;
    for (long long t = lmax >> 1; t >= 1; t >>= 1)
        if (common_prefix(keys, F, i, i + (l + t) * d) > dmin) l += t;
    const long long j = i + l * d;
    const int dnode = common_prefix(keys, F, i, j);
    long long s = 0;
    for (long long div = 2;; div <<= 1) {
        const long long t = (l + div - 1) / div;
        if (common_prefix(keys, F, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    const int gamma = int(i + s * d + (d < 0 ? -1 : 0));
    const int lo = int(min((long long)i, j)), hi = int(max((long long)i, j));
    const int left = lo == gamma ? ~gamma : gamma;
    const int right = hi == gamma + 1 ? ~(gamma + 1) : gamma + 1;
    nodes[i].d = make_int4(left, right, 0, 0);
    if (left >= 0) node_parent[left] = (i << 1) | 0;
    else leaf_parent[~left] = (i << 1) | 0;
    if (right >= 0) node_parent[right] = (i << 1) | 1;
    else leaf_parent[~right] = (i << 1) | 1;
    if (i == 0) node_parent[0] = -1;
}

// depth of every leaf (internal nodes above it); a walk longer than F steps
// (a malformed tree) sets *bad instead of looping
__global__ void k_depth(const int* leaf_parent, const int* node_parent, int F, int* max_depth, int* bad) {
    const int sl = blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= F) return;
    int ref = leaf_parent[sl];
    int depth = 0;
    while (ref >= 0 && depth <= F) {
        ++depth;
        ref = node_parent[ref >> 1];
    }
    if (depth > F) atomicOr(bad, 1);
    atomicMax(max_depth, depth);
}

// the leaf triangles in tree order: v0 | face, v1 | group, v2
__global__ void k_leaves(const float* v, const int* faces, const int* face_group, const int* order, int F,
                         float4* tri) {
    const int sl = blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= F) return;
    const int f = order[sl];
    const float* a = v + 3 * faces[3 * f];
    const float* b = v + 3 * faces[3 * f + 1];
    const float* c = v + 3 * faces[3 * f + 2];
    tri[3 * sl + 0] = make_float4(a[0], a[1], a[2], __int_as_float(f));
    tri[3 * sl + 1] = make_float4(b[0], b[1], b[2], __int_as_float(face_group[f]));
    tri[3 * sl + 2] = make_float4(c[0], c[1], c[2], 0.0f);
}

}  // namespace lbvh

int scene_rebuild_bvh(SceneHandle* h, int* depth_out, cudaStream_t stream) {
    using namespace lbvh;
    if (h == nullptr) return 1;
    SceneDev& sd = h->dev;
    const int F = sd.num_faces;
    if (F < 2) {
        if (depth_out) *depth_out = sd.max_depth;
        return 0;
    }
    // scratch: keys and values (in and out), the new tree, its parent links,
    // the bounds, the depth and the sort's temporary storage
    size_t sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, static_cast<unsigned long long*>(nullptr),
                                    static_cast<unsigned long long*>(nullptr), static_cast<int*>(nullptr),
                                    static_cast<int*>(nullptr), F, 0, 64, stream);
    auto up16 = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t o_keys = 0;
    const size_t o_keys2 = o_keys + up16(size_t(F) * 8);
    const size_t o_vals = o_keys2 + up16(size_t(F) * 8);
    const size_t o_vals2 = o_vals + up16(size_t(F) * 4);
    const size_t o_nodes = o_vals2 + up16(size_t(F) * 4);
    const size_t o_lp = o_nodes + up16(size_t(F - 1) * sizeof(BvhNode));
    const size_t o_np = o_lp + up16(size_t(F) * 4);
    const size_t o_misc = o_np + up16(size_t(F - 1) * 4);
    const size_t o_sort = o_misc + 256;
    const size_t total = o_sort + up16(sort_bytes);
    unsigned char* buf = nullptr;
    if (cudaMalloc(&buf, total) != cudaSuccess) return 2;
    auto* keys = reinterpret_cast<unsigned long long*>(buf + o_keys);
    auto* keys2 = reinterpret_cast<unsigned long long*>(buf + o_keys2);
    int* vals = reinterpret_cast<int*>(buf + o_vals);
    int* vals2 = reinterpret_cast<int*>(buf + o_vals2);
    BvhNode* nodes = reinterpret_cast<BvhNode*>(buf + o_nodes);
    int* lp = reinterpret_cast<int*>(buf + o_lp);
    int* np = reinterpret_cast<int*>(buf + o_np);
    float* bounds = reinterpret_cast<float*>(buf + o_misc);
    int* stats = reinterpret_cast<int*>(buf + o_misc + 32);  // [0] max depth, [1] malformed
    bool ok = cudaMemsetAsync(stats, 0, 8, stream) == cudaSuccess;
    ok = ok && cudaMemsetAsync(nodes, 0, size_t(F - 1) * sizeof(BvhNode), stream) == cudaSuccess;
    const int grid = (F + kB - 1) / kB;
    k_centroid_bounds<<<1, kB, 0, stream>>>(sd.vertices, sd.faces, F, bounds);
    k_morton<<<grid, kB, 0, stream>>>(sd.vertices, sd.faces, F, bounds, keys, vals);
    ok = ok && cub::DeviceRadixSort::SortPairs(buf + o_sort, sort_bytes, keys, keys2, vals, vals2, F, 0, 64,
                                               stream) == cudaSuccess;
    k_karras<<<(F - 1 + kB - 1) / kB, kB, 0, stream>>>(keys2, F, nodes, lp, np);
    k_depth<<<grid, kB, 0, stream>>>(lp, np, F, stats, stats + 1);
    int host_stats[2] = {0, 0};
    ok = ok && cudaGetLastError() == cudaSuccess;
    ok = ok && cudaMemcpyAsync(host_stats, stats, 8, cudaMemcpyDeviceToHost, stream) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(stream) == cudaSuccess;
    note_launch(5);
    if (!ok || host_stats[1] != 0) {
        cudaFree(buf);
        return 2;
    }
    const int depth = host_stats[0];
    if (depth + 2 > kStackDepth) {  // the old tree stays
        cudaFree(buf);
        return 4;
    }
    // commit in place: the node links, the parent links and the leaf
    // triangles, then the boxes bottom-up
    ok = cudaMemcpyAsync(const_cast<BvhNode*>(sd.nodes), nodes, size_t(F - 1) * sizeof(BvhNode),
                         cudaMemcpyDeviceToDevice, stream) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(h->leaf_parent, lp, size_t(F) * 4, cudaMemcpyDeviceToDevice, stream) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(h->node_parent, np, size_t(F - 1) * 4, cudaMemcpyDeviceToDevice, stream) ==
                   cudaSuccess;
    k_leaves<<<grid, kB, 0, stream>>>(sd.vertices, sd.faces, sd.face_group, vals2, F, const_cast<float4*>(sd.tri));
    ok = ok && cudaMemsetAsync(h->bvh_counter, 0, size_t(F - 1) * sizeof(int), stream) == cudaSuccess;
    ok = ok && refit_boxes(h, stream) == 0;
    ok = ok && cudaGetLastError() == cudaSuccess;
    ok = ok && cudaStreamSynchronize(stream) == cudaSuccess;
    note_launch(1);
    cudaFree(buf);
    if (!ok) return 2;
    sd.root = 0;
    sd.max_depth = depth;
    sd.stack_entries = std::max(8, std::min(kStackDepth, depth + 2));
    if (depth_out) *depth_out = depth;
    return 0;
}

}  // namespace wcb
