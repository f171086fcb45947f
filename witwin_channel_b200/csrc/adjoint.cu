// Fixed-topology VJP of the path fields (the drop-in for the reference's
// deterministic AD: the field Functions of witwin/channel/kernels/fields.py
// :1087-2140 and the frozen-winner geometry re-solve of
// witwin/channel/propagation/geometry.py:214-286).
//
// The forward solve froze every path's interaction sequence in a 48-byte
// record (faces per bounce, edge id).  The backward pass stores no
// intermediates: each record is re-evaluated from the raw scene values
// (vertex coordinates, per-material eps_r / sigma, frequency, Tx and Rx
// positions) in FP64 dual numbers.  A record touches a handful of scalars
// (its faces' vertices and materials, the endpoints, the frequency); they are
// enumerated per record, deduplicated, and pushed through the field
// evaluation N at a time as dual tangent lanes.  With the incoming per-record
// cotangents (of path gain and the complex path field) each lane gives one
// (parameter id, contribution) pair.  The pairs are stably radix-sorted by
// parameter id and summed per id in record order, so the gradient is
// deterministic bit for bit, with one write per parameter.
//
// Geometry of the re-solve: a reflection's hit points come from the image
// method over the planes of the record's own faces (unit normal of
// (b - a) x (c - a), anchor a), a transmission's walls from their face
// normals, a diffraction's edge frame from its end vertices and the two faces
// whose normals bound the wedge.
#include <algorithm>
#include <climits>
#include <cstring>

#include "adjoint.cuh"

namespace wcb {
namespace adj {

// per record: its parameter count, its (component, depth) grouping key and
// the per-component record counts
// per-component record counts: one atomic per warp and component (the
// launches use whole warps; lanes past the end vote for no component)
WCB_D void count_component(int* comp_counts, int rank) {
    for (int r = 0; r < 4; ++r) {
        const unsigned b = __ballot_sync(0xffffffffu, rank == r);
        if ((threadIdx.x & 31) == 0 && b) atomicAdd(comp_counts + r, __popc(b));
    }
}

__global__ void k_vjp_count(AdjParams p, int* keys, int* idx) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int rank = -1;
    if (i < p.count) {
        const RowRec row = p.rows[p.selected[i]];
        p.counts[i] = row.component == 2 ? diffraction_params(p, row).count : face_record_param_count(p, row);
        keys[i] = order_key(p, row);
        idx[i] = int(i);
        rank = component_rank(row.component);
    }
    count_component(p.comp_counts, rank);
}

// The execution-order keys alone (wcb_rows_order)
__global__ void k_order_keys(AdjParams p, int* keys, int* idx, int* comp_counts) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int rank = -1;
    if (i < p.count) {
        const RowRec row = p.rows[p.selected[i]];
        keys[i] = order_key(p, row);
        idx[i] = int(i);
        rank = component_rank(row.component);
    }
    count_component(comp_counts, rank);
}

// Ordered per-id sums of the id-sorted pairs (a parameter's contributions
// form one run).  A run is cut into chunks of kChunk entries in record order;
// one block sums a chunk (each thread a fixed strided subset, then a
// fixed-shape block tree) and one thread then sums a run's chunk partials in
// chunk order.  The partition depends only on the run lengths, never on
// timing, so the gradient is deterministic bit for bit, and a parameter that
// every record touches (a Tx coordinate, a material value) is summed by many
// blocks instead of one.  Parameters without a run stay zero.
constexpr int kReduceBlock = 256;
constexpr int kChunk = 16384;

__global__ void k_run_chunks(const int* run_counts, const int* num_runs, int cap, int* chunk_n) {
    const int runs = *num_runs;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < cap; r += gridDim.x * blockDim.x)
        chunk_n[r] = r < runs ? (run_counts[r] + kChunk - 1) / kChunk : 0;
}

__global__ void __launch_bounds__(kReduceBlock) k_reduce_chunks(const int* run_counts, const long long* run_offsets,
                                                                const int* num_runs, const int* chunk_base,
                                                                const int* chunk_n, int cap, const double* vals,
                                                                double* chunk_sums) {
    typedef cub::BlockReduce<double, kReduceBlock> Reduce;
    __shared__ typename Reduce::TempStorage tmp;
    const int runs = *num_runs;
    const int total = chunk_base[cap - 1] + chunk_n[cap - 1];
    for (int c = blockIdx.x; c < total; c += gridDim.x) {
        // the run holding chunk c: the last run whose first chunk is at or before c
        int lo = 0, hi = runs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (chunk_base[mid] <= c) lo = mid;
            else hi = mid - 1;
        }
        const int j = c - chunk_base[lo];
        const long long beg = run_offsets[lo] + (long long)j * kChunk;
        const int n = min(kChunk, run_counts[lo] - j * kChunk);
        double s = 0.0;
        for (int q = threadIdx.x; q < n; q += kReduceBlock) s += vals[beg + q];
        const double sum = Reduce(tmp).Sum(s);
        if (threadIdx.x == 0) chunk_sums[c] = sum;
        __syncthreads();
    }
}

__global__ void k_reduce_run_chunks(const unsigned* run_ids, const int* num_runs, const int* chunk_base,
                                    const int* chunk_n, const double* chunk_sums, double* grad) {
    const int runs = *num_runs;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < runs; r += gridDim.x * blockDim.x) {
        double s = 0.0;
        const int b = chunk_base[r];
        for (int k = 0; k < chunk_n[r]; ++k) s += chunk_sums[b + k];
        grad[run_ids[r]] = s;
    }
}

size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

// Workspace: the per-record counts, offsets and scan scratch (sized by the
// record count) come first; the (id, contribution) pairs and the sort scratch
// (sized by the pair count) follow.
struct VjpLayout {
    size_t counts, offsets, comp_counts, keys, keys2, order, order2, scan_tmp, scan_bytes, ids, ids2, vals, vals2,
        run_ids, run_counts, run_offsets, num_runs, sort_tmp, sort_bytes, total;
};

VjpLayout vjp_layout(long long K, long long pairs) {
    VjpLayout L;
    const size_t k = size_t(std::max<long long>(K, 1));
    const size_t m = size_t(std::max<long long>(pairs, 1));
    size_t o = 0;
    auto take = [&](size_t b) { const size_t a = o; o = a256(o + b); return a; };
    L.counts = take(k * 4);
    L.offsets = take(k * 8);
    L.comp_counts = take(16);
    L.keys = take(k * 4);
    L.keys2 = take(k * 4);
    L.order = take(k * 4);
    L.order2 = take(k * 4);
    size_t scan_b = 0, group_b = 0, work_b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_b, (int*)nullptr, (long long*)nullptr, int(k));
    cub::DeviceRadixSort::SortPairs(nullptr, group_b, (int*)nullptr, (int*)nullptr, (int*)nullptr, (int*)nullptr,
                                    int(k), 0, 5);
    cub::DeviceScan::ExclusiveSum(nullptr, work_b, (int*)nullptr, (int*)nullptr, int(k));
    L.scan_bytes = std::max(std::max(scan_b, group_b), work_b);
    L.scan_tmp = take(L.scan_bytes);
    L.ids = take(m * 4);
    L.ids2 = take(m * 4);
    L.vals = take(m * 8);
    L.vals2 = take(m * 8);
    L.run_ids = take(m * 4);
    L.run_counts = take(m * 4);
    L.run_offsets = take(m * 8);
    L.num_runs = take(16);
    size_t sort_b = 0, rle_b = 0, roff_b = 0;
    const int mi = int(std::min<size_t>(m, INT_MAX));
    cub::DeviceRadixSort::SortPairs(nullptr, sort_b, (unsigned*)nullptr, (unsigned*)nullptr, (double*)nullptr,
                                    (double*)nullptr, mi, 0, 32);
    cub::DeviceRunLengthEncode::Encode(nullptr, rle_b, (const unsigned*)nullptr, (unsigned*)nullptr, (int*)nullptr,
                                       (int*)nullptr, mi);
    cub::DeviceScan::ExclusiveSum(nullptr, roff_b, (int*)nullptr, (long long*)nullptr, mi);
    size_t chunk_b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, chunk_b, (int*)nullptr, (int*)nullptr, mi);
    L.sort_bytes = std::max(std::max(sort_b, chunk_b), std::max(rle_b, roff_b));
    L.sort_tmp = take(L.sort_bytes);
    L.total = o;
    return L;
}

long long max_params_per_row(int max_depth, int max_layers) {
    const int d = std::max(1, std::min(max_depth, kMaxDepth));
    const int l = std::max(1, std::min(max_layers, kMaxLayersPerMaterial));
    const long long refl = 7 + d * (9 + 2);
    const long long trans = 7 + d * (9 + 2 * l);
    const long long diff = 7 + 15 + 4;
    return std::min<long long>(kMaxParams, std::max(refl, std::max(trans, diff)));
}

// Scene, endpoint, material (at freq_index) and parameter-layout fields of
// the derivative kernels' parameters.
void fill_params(AdjParams& p, const SceneHandle* h, const wcb_solve_desc* desc, const wcb_materials* materials,
                 int freq_index, const void* rows, const int64_t* selected, long long K, const int64_t* layout) {
    std::memset(&p, 0, sizeof(p));
    p.sc = h->dev;
    p.edge_slot = h->edge_slot;
    p.edge_topo = h->edge_topo;
    p.tx_pos = desc->tx_pos;
    p.tx_power = desc->tx_power;
    p.tx_pol = desc->tx_pol;
    p.rx_kind = desc->rx_kind;
    p.rx_pos = desc->rx_pos;
    for (int i = 0; i < 3; ++i) {
        p.grid_origin[i] = desc->grid_origin[i];
        p.grid_x[i] = desc->grid_x_axis[i];
        p.grid_y[i] = desc->grid_y_axis[i];
    }
    p.grid_rows = desc->grid_rows;
    p.grid_cols = desc->grid_cols;
    p.grid_spacing[0] = desc->grid_spacing[0];
    p.grid_spacing[1] = desc->grid_spacing[1];
    p.rx_pol = desc->rx_pol;
    p.rx_pol_stride = desc->rx_pol_stride;
    p.freq = desc->frequency_hz[freq_index];
    const int M = materials->num_materials;
    const int NL = materials->num_layers;
    p.num_materials = M;
    p.eps_r = materials->eps_r + (long long)freq_index * M;
    p.sigma_e = materials->sigma_e + (long long)freq_index * M;
    p.mu_r = materials->mu_r + (long long)freq_index * M;
    p.gain = materials->gain + (long long)freq_index * M;
    p.thickness = materials->thickness + (long long)freq_index * M;
    p.num_layers = NL;
    p.layer_offset = materials->layer_offset;
    p.layer_count = materials->layer_count;
    p.layer_thickness = materials->layer_thickness + (long long)freq_index * NL;
    p.layer_eps_r = materials->layer_eps_r + (long long)freq_index * NL;
    p.layer_sigma_e = materials->layer_sigma_e + (long long)freq_index * NL;
    p.layer_mu_r = materials->layer_mu_r + (long long)freq_index * NL;
    p.rows = static_cast<const RowRec*>(rows);
    p.selected = reinterpret_cast<const long long*>(selected);
    p.count = K;
    p.base_meps = int(layout[1]);
    p.base_msig = int(layout[2]);
    p.base_leps = int(layout[3]);
    p.base_lsig = int(layout[4]);
    p.gid_freq = int(layout[5]);
    p.base_tx = int(layout[6]);
    p.base_rx = int(layout[7]);
}

}  // namespace adj
}  // namespace wcb

struct wcb_scene {
    wcb::SceneHandle* h;
};

extern "C" {

int wcb_rows_vjp_layout(const wcb_scene* scene, const wcb_solve_desc* desc, const wcb_materials* materials,
                        int64_t* layout) {
    if (scene == nullptr || desc == nullptr || materials == nullptr || layout == nullptr)
        return WCB_ERR_INVALID_ARGUMENT;
    const long long V = scene->h->dev.num_vertices;
    const long long M = materials->num_materials;
    const long long Ly = materials->num_layers;
    const long long T = desc->num_tx;
    const long long R = desc->rx_kind == 0 ? desc->num_rx : 0;
    layout[0] = 0;                    // vertices (V,3)
    layout[1] = 3 * V;                // material eps_r (M)
    layout[2] = layout[1] + M;        // material sigma_e (M)
    layout[3] = layout[2] + M;        // layer eps_r (L)
    layout[4] = layout[3] + Ly;       // layer sigma_e (L)
    layout[5] = layout[4] + Ly;       // frequency (1)
    layout[6] = layout[5] + 1;        // tx positions (T,3)
    layout[7] = layout[6] + 3 * T;    // rx positions (R,3), point receivers only
    layout[8] = layout[7] + 3 * R;    // total
    return layout[8] < INT_MAX ? WCB_OK : WCB_ERR_NOT_SUPPORTED;
}

int wcb_rows_vjp_workspace_size(int64_t num_selected, int32_t max_depth, int32_t max_layers, int64_t* bytes) {
    if (bytes == nullptr || num_selected < 0) return WCB_ERR_INVALID_ARGUMENT;
    const long long pairs = num_selected * wcb::adj::max_params_per_row(max_depth, max_layers);
    if (pairs >= INT_MAX) return WCB_ERR_NOT_SUPPORTED;
    *bytes = int64_t(wcb::adj::vjp_layout(num_selected, pairs).total);
    return WCB_OK;
}

int wcb_rows_vjp(const wcb_scene* scene, const wcb_solve_desc* desc, const wcb_materials* materials,
                 int32_t freq_index, const void* rows, const int64_t* selected, int64_t num_selected,
                 const double* grad_path_gain, const double* grad_field_real, const double* grad_field_imag,
                 int32_t want, const uint8_t* vertex_mask, double* grad_out, int64_t grad_size, double* row_field,
                 const int32_t* order, const int64_t* comp_counts_in, void* workspace, int64_t workspace_bytes,
                 void* stream) {
    if (scene == nullptr || desc == nullptr || materials == nullptr || grad_out == nullptr || num_selected < 0)
        return WCB_ERR_INVALID_ARGUMENT;
    if (num_selected > 0 && (rows == nullptr || selected == nullptr)) return WCB_ERR_INVALID_ARGUMENT;
    if (freq_index < 0 || freq_index >= desc->num_freq || desc->frequency_hz == nullptr)
        return WCB_ERR_INVALID_ARGUMENT;
    int64_t layout[9];
    int rc = wcb_rows_vjp_layout(scene, desc, materials, layout);
    if (rc != WCB_OK) return rc;
    if (grad_size < layout[8]) return WCB_ERR_CAPACITY;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long long K = num_selected;
    const long long P = layout[8];
    if (K == 0) {
        return cudaMemsetAsync(grad_out, 0, size_t(P) * 8, s) == cudaSuccess ? WCB_OK : WCB_ERR_CUDA;
    }
    wcb::adj::VjpLayout L = wcb::adj::vjp_layout(K, 1);
    if (workspace == nullptr || workspace_bytes < (long long)L.ids) return WCB_ERR_CAPACITY;
    char* b = static_cast<char*>(workspace);
    wcb::adj::AdjParams p;
    wcb::adj::fill_params(p, scene->h, desc, materials, freq_index, rows, selected, K, layout);
    p.g_gain = grad_path_gain;
    p.g_re = grad_field_real;
    p.g_im = grad_field_imag;
    p.want = want;
    p.vertex_mask = vertex_mask;
    p.counts = reinterpret_cast<int*>(b + L.counts);
    long long* offsets = reinterpret_cast<long long*>(b + L.offsets);
    p.offsets = offsets;
    p.row_field = row_field;
    p.comp_counts = reinterpret_cast<int*>(b + L.comp_counts);
    int* keys = reinterpret_cast<int*>(b + L.keys);
    int* keys2 = reinterpret_cast<int*>(b + L.keys2);
    int* idx = reinterpret_cast<int*>(b + L.order);
    int* order2 = reinterpret_cast<int*>(b + L.order2);
    const int grid = int((K + wcb::adj::kBlock - 1) / wcb::adj::kBlock);
    cudaMemsetAsync(p.comp_counts, 0, 16, s);
    wcb::adj::k_vjp_count<<<grid, wcb::adj::kBlock, 0, s>>>(p, keys, idx);
    size_t tb = L.scan_bytes;
    if (cub::DeviceScan::ExclusiveSum(b + L.scan_tmp, tb, p.counts, offsets, int(K), s) != cudaSuccess)
        return WCB_ERR_CUDA;
    // records grouped by component, depth and diffraction edge (wcb_rows_order's
    // key), record order kept within a group; or the caller's order
    if (order == nullptr) {
        tb = L.scan_bytes;
        if (cub::DeviceRadixSort::SortPairs(b + L.scan_tmp, tb, keys, keys2, idx, order2, int(K), 0, 31, s) !=
            cudaSuccess)
            return WCB_ERR_CUDA;
    }
    wcb::note_launch(3);
    long long last_off = 0;
    int last_cnt = 0;
    int comp_counts[4] = {0, 0, 0, 0};
    cudaMemcpyAsync(&last_off, offsets + K - 1, 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&last_cnt, p.counts + K - 1, 4, cudaMemcpyDeviceToHost, s);
    if (order == nullptr) cudaMemcpyAsync(comp_counts, p.comp_counts, 16, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return WCB_ERR_CUDA;
    if (order != nullptr) {
        for (int r = 0; r < 4; ++r) comp_counts[r] = int(comp_counts_in ? comp_counts_in[r] : 0);
        p.order = order;
    } else {
        p.order = order2;
    }
    const long long pairs = last_off + last_cnt;
    if (pairs >= INT_MAX) return WCB_ERR_NOT_SUPPORTED;
    L = wcb::adj::vjp_layout(K, pairs);
    if (workspace_bytes < (long long)L.total) return WCB_ERR_CAPACITY;
    p.out_ids = reinterpret_cast<unsigned*>(b + L.ids);
    p.out_vals = reinterpret_cast<double*>(b + L.vals);
    {
        // one launch per component over its dense range of the grouped order
        const int cids[4] = {0, 1, 5, 2};
        long long begin = 0;
        for (int r = 0; r < 4; ++r) {
            p.order_begin = begin;
            p.order_count = comp_counts[r];
            begin += comp_counts[r];
            if (p.order_count <= 0) continue;
            const unsigned g = unsigned((p.order_count + wcb::adj::kBlock - 1) / wcb::adj::kBlock);
            switch (cids[r]) {
                case 0: wcb::adj::k_vjp_rows<wcb::adj::kLanes, 0><<<g, wcb::adj::kBlock, 0, s>>>(p); break;
                case 1: wcb::adj::k_vjp_rows<wcb::adj::kLanes, 1><<<g, wcb::adj::kBlock, 0, s>>>(p); break;
                case 5: wcb::adj::k_vjp_rows<wcb::adj::kLanes, 5><<<g, wcb::adj::kBlock, 0, s>>>(p); break;
                default: {
                    wcb::ProfileState& prof = wcb::profile_state();
                    cudaEvent_t e0 = nullptr, e1 = nullptr;
                    if (prof.enabled) {
                        cudaEventCreate(&e0);
                        cudaEventCreate(&e1);
                        cudaEventRecord(e0, s);
                    }
                    wcb::adj::launch_vjp_diffraction(p, s);
                    if (prof.enabled) {
                        float ms = 0.f;
                        cudaEventRecord(e1, s);
                        if (cudaEventSynchronize(e1) == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) {
                            prof.acc_vjp_diff_ms += ms;
                            prof.acc_vjp_diff_records += p.order_count;
                            prof.acc_vjp_diff_launches += 1;
                        }
                        cudaEventDestroy(e0);
                        cudaEventDestroy(e1);
                    }
                    break;
                }
            }
            wcb::note_launch();
        }
    }
    unsigned* ids2 = reinterpret_cast<unsigned*>(b + L.ids2);
    double* vals2 = reinterpret_cast<double*>(b + L.vals2);
    int end_bit = 1;
    while (end_bit < 31 && (P >> end_bit) != 0) ++end_bit;
    if (pairs > 0) {
        tb = L.sort_bytes;
        if (cub::DeviceRadixSort::SortPairs(b + L.sort_tmp, tb, p.out_ids, ids2, p.out_vals, vals2, int(pairs), 0,
                                            end_bit, s) != cudaSuccess)
            return WCB_ERR_CUDA;
        wcb::note_launch();
    }
    cudaMemsetAsync(grad_out, 0, size_t(P) * 8, s);
    if (pairs > 0) {
        unsigned* run_ids = reinterpret_cast<unsigned*>(b + L.run_ids);
        int* run_counts = reinterpret_cast<int*>(b + L.run_counts);
        long long* run_offsets = reinterpret_cast<long long*>(b + L.run_offsets);
        int* num_runs = reinterpret_cast<int*>(b + L.num_runs);
        tb = L.sort_bytes;
        if (cub::DeviceRunLengthEncode::Encode(b + L.sort_tmp, tb, ids2, run_ids, run_counts, num_runs, int(pairs), s) !=
            cudaSuccess)
            return WCB_ERR_CUDA;
        tb = L.sort_bytes;
        if (cub::DeviceScan::ExclusiveSum(b + L.sort_tmp, tb, run_counts, run_offsets, int(std::min<long long>(pairs, P)),
                                          s) != cudaSuccess)
            return WCB_ERR_CUDA;
        // chunk counts and bases reuse the unsorted-id and sorted-id buffers, the
        // chunk partials the unsorted values (all free once sorted and encoded)
        const int cap = int(std::min<long long>(pairs, P));
        int* chunk_n = reinterpret_cast<int*>(p.out_ids);
        int* chunk_base = reinterpret_cast<int*>(ids2);
        double* chunk_sums = p.out_vals;
        const int tgrid = int(std::min<long long>((cap + 255) / 256, 4096));
        wcb::adj::k_run_chunks<<<tgrid, 256, 0, s>>>(run_counts, num_runs, cap, chunk_n);
        tb = L.sort_bytes;
        if (cub::DeviceScan::ExclusiveSum(b + L.sort_tmp, tb, chunk_n, chunk_base, cap, s) != cudaSuccess)
            return WCB_ERR_CUDA;
        wcb::adj::k_reduce_chunks<<<148 * 8, wcb::adj::kReduceBlock, 0, s>>>(run_counts, run_offsets, num_runs,
                                                                            chunk_base, chunk_n, cap, vals2,
                                                                            chunk_sums);
        wcb::adj::k_reduce_run_chunks<<<tgrid, 256, 0, s>>>(run_ids, num_runs, chunk_base, chunk_n, chunk_sums,
                                                           grad_out);
        wcb::note_launch(6);
    }
    rc = cudaGetLastError() == cudaSuccess ? WCB_OK : WCB_ERR_CUDA;
    return rc;
}

int wcb_rows_jvp(const wcb_scene* scene, const wcb_solve_desc* desc, const wcb_materials* materials,
                 int32_t freq_index, const void* rows, const int64_t* selected, int64_t num_selected,
                 const double* tangent, int64_t tangent_size, double* row_field, double* row_field_tangent,
                 const int32_t* order, const int64_t* comp_counts, void* stream) {
    if (scene == nullptr || desc == nullptr || materials == nullptr || num_selected < 0)
        return WCB_ERR_INVALID_ARGUMENT;
    if (num_selected > 0 && (rows == nullptr || selected == nullptr)) return WCB_ERR_INVALID_ARGUMENT;
    // no tangent: the FP64 fields alone (plain evaluation, no dual lane)
    if (tangent == nullptr ? row_field == nullptr : row_field_tangent == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    if (desc->frequency_hz == nullptr || desc->num_freq < 1) return WCB_ERR_INVALID_ARGUMENT;
    if (freq_index == -1) {
        // every frequency of the desc, fields only: row_field (NF, K, 2);
        // diffraction records form their UTD geometry once for all of them
        if (tangent != nullptr) return WCB_ERR_INVALID_ARGUMENT;
        int64_t layout_all[9];
        const int rc_all = wcb_rows_vjp_layout(scene, desc, materials, layout_all);
        if (rc_all != WCB_OK) return rc_all;
        if (num_selected == 0) return WCB_OK;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const int NF = desc->num_freq;
        const int cids[4] = {0, 1, 5, 2};
        long long begin = 0;
        for (int r = 0; r < 4; ++r) {
            const long long count = order ? (comp_counts ? comp_counts[r] : 0) : num_selected;
            const long long at = order ? begin : 0;
            begin += count;
            if (count <= 0) continue;
            const unsigned g = unsigned((count + wcb::adj::kBlock - 1) / wcb::adj::kBlock);
            wcb::adj::AdjParams p;
            if (cids[r] == 2 && NF <= 4) {
                wcb::adj::fill_params(p, scene->h, desc, materials, 0, rows, selected, num_selected, layout_all);
                p.order = order;
                p.order_begin = at;
                p.order_count = count;
                wcb::adj::FreqSet fs{};
                for (int c = 0; c < NF; ++c) fs.f[c] = desc->frequency_hz[c];
                wcb::adj::launch_field64_diffraction_multi(p, NF, fs, row_field, s);
                wcb::note_launch();
                continue;
            }
            for (int c = 0; c < NF; ++c) {
                wcb::adj::fill_params(p, scene->h, desc, materials, c, rows, selected, num_selected, layout_all);
                p.order = order;
                p.order_begin = at;
                p.order_count = count;
                double* out = row_field + 2 * num_selected * (long long)c;
                switch (cids[r]) {
                    case 0: wcb::adj::k_field64_rows<0><<<g, wcb::adj::kBlock, 0, s>>>(p, out); break;
                    case 1: wcb::adj::k_field64_rows<1><<<g, wcb::adj::kBlock, 0, s>>>(p, out); break;
                    case 5: wcb::adj::k_field64_rows<5><<<g, wcb::adj::kBlock, 0, s>>>(p, out); break;
                    default: wcb::adj::launch_field64_diffraction(p, out, s); break;
                }
                wcb::note_launch();
            }
        }
        return cudaGetLastError() == cudaSuccess ? WCB_OK : WCB_ERR_CUDA;
    }
    if (freq_index < 0 || freq_index >= desc->num_freq) return WCB_ERR_INVALID_ARGUMENT;
    int64_t layout[9];
    const int rc = wcb_rows_vjp_layout(scene, desc, materials, layout);
    if (rc != WCB_OK) return rc;
    if (tangent != nullptr && tangent_size < layout[8]) return WCB_ERR_CAPACITY;
    if (num_selected == 0) return WCB_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    wcb::adj::AdjParams p;
    wcb::adj::fill_params(p, scene->h, desc, materials, freq_index, rows, selected, num_selected, layout);
    // one launch per component: over its dense range of the execution order
    // (wcb_rows_order), or over every record when no order is given
    const int cids[4] = {0, 1, 5, 2};
    long long begin = 0;
    p.order = order;
    for (int r = 0; r < 4; ++r) {
        p.order_begin = order ? begin : 0;
        p.order_count = order ? (comp_counts ? comp_counts[r] : 0) : num_selected;
        begin += p.order_count;
        if (p.order_count <= 0) continue;
        const unsigned g = unsigned((p.order_count + wcb::adj::kBlock - 1) / wcb::adj::kBlock);
        if (tangent == nullptr) {
            switch (cids[r]) {
                case 0: wcb::adj::k_field64_rows<0><<<g, wcb::adj::kBlock, 0, s>>>(p, row_field); break;
                case 1: wcb::adj::k_field64_rows<1><<<g, wcb::adj::kBlock, 0, s>>>(p, row_field); break;
                case 5: wcb::adj::k_field64_rows<5><<<g, wcb::adj::kBlock, 0, s>>>(p, row_field); break;
                default: wcb::adj::launch_field64_diffraction(p, row_field, s); break;
            }
        } else {
            switch (cids[r]) {
                case 0: wcb::adj::k_jvp_rows<0><<<g, wcb::adj::kBlock, 0, s>>>(p, tangent, row_field, row_field_tangent); break;
                case 1: wcb::adj::k_jvp_rows<1><<<g, wcb::adj::kBlock, 0, s>>>(p, tangent, row_field, row_field_tangent); break;
                case 5: wcb::adj::k_jvp_rows<5><<<g, wcb::adj::kBlock, 0, s>>>(p, tangent, row_field, row_field_tangent); break;
                default: wcb::adj::launch_jvp_diffraction(p, tangent, row_field, row_field_tangent, s); break;
            }
        }
        wcb::note_launch();
    }
    return cudaGetLastError() == cudaSuccess ? WCB_OK : WCB_ERR_CUDA;
}

int wcb_rows_order_workspace_size(int64_t num_selected, int64_t* bytes) {
    if (bytes == nullptr || num_selected < 0) return WCB_ERR_INVALID_ARGUMENT;
    const size_t k = size_t(std::max<int64_t>(num_selected, 1));
    size_t sort_b = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_b, (int*)nullptr, (int*)nullptr, (int*)nullptr, (int*)nullptr,
                                    int(k), 0, 31);
    *bytes = int64_t(wcb::adj::a256(k * 4) * 3 + wcb::adj::a256(16) + wcb::adj::a256(sort_b));
    return WCB_OK;
}

int wcb_rows_order(const wcb_scene* scene, const void* rows, const int64_t* selected, int64_t num_selected,
                   int32_t* order, int64_t* comp_counts, void* workspace, int64_t workspace_bytes, void* stream) {
    if (scene == nullptr || order == nullptr || comp_counts == nullptr || num_selected < 0)
        return WCB_ERR_INVALID_ARGUMENT;
    if (num_selected > 0 && (rows == nullptr || selected == nullptr)) return WCB_ERR_INVALID_ARGUMENT;
    for (int r = 0; r < 4; ++r) comp_counts[r] = 0;
    if (num_selected == 0) return WCB_OK;
    if (num_selected >= INT_MAX) return WCB_ERR_NOT_SUPPORTED;
    int64_t need = 0;
    wcb_rows_order_workspace_size(num_selected, &need);
    if (workspace == nullptr || workspace_bytes < need) return WCB_ERR_CAPACITY;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t k = size_t(num_selected);
    char* b = static_cast<char*>(workspace);
    int* keys = reinterpret_cast<int*>(b);
    int* keys2 = reinterpret_cast<int*>(b + wcb::adj::a256(k * 4));
    int* idx = reinterpret_cast<int*>(b + 2 * wcb::adj::a256(k * 4));
    int* counts = reinterpret_cast<int*>(b + 3 * wcb::adj::a256(k * 4));
    void* tmp = b + 3 * wcb::adj::a256(k * 4) + wcb::adj::a256(16);
    size_t tb = size_t(need) - (3 * wcb::adj::a256(k * 4) + wcb::adj::a256(16));
    wcb::adj::AdjParams p;
    std::memset(&p, 0, sizeof(p));
    p.sc = scene->h->dev;
    p.edge_slot = scene->h->edge_slot;
    p.rows = static_cast<const wcb::RowRec*>(rows);
    p.selected = reinterpret_cast<const long long*>(selected);
    p.count = num_selected;
    bool ok = cudaMemsetAsync(counts, 0, 16, s) == cudaSuccess;
    wcb::adj::k_order_keys<<<unsigned((k + wcb::adj::kBlock - 1) / wcb::adj::kBlock), wcb::adj::kBlock, 0, s>>>(
        p, keys, idx, counts);
    ok = ok && cub::DeviceRadixSort::SortPairs(tmp, tb, keys, keys2, idx, order, int(k), 0, 31, s) == cudaSuccess;
    int host[4] = {0, 0, 0, 0};
    ok = ok && cudaMemcpyAsync(host, counts, 16, cudaMemcpyDeviceToHost, s) == cudaSuccess;
    ok = ok && cudaStreamSynchronize(s) == cudaSuccess;
    wcb::note_launch(2);
    if (!ok) return WCB_ERR_CUDA;
    for (int r = 0; r < 4; ++r) comp_counts[r] = host[r];
    return WCB_OK;
}

}  // extern "C"
