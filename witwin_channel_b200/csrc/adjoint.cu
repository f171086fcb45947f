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

__global__ void k_vjp_count(AdjParams p) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= p.count) return;
    ParamList pl;
    build_params(p, p.rows[p.selected[i]], pl);
    p.counts[i] = pl.n;
}

// one thread per parameter: its contributions are a contiguous run of the
// id-sorted pairs, summed in record order
__global__ void k_vjp_reduce(long long params, long long n, const unsigned* ids, const double* vals, double* grad) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (g >= params) return;
    long long lo = 0, hi = n;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if ((long long)ids[mid] < g) lo = mid + 1;
        else hi = mid;
    }
    double s = 0.0;
    for (long long q = lo; q < n && (long long)ids[q] == g; ++q) s += vals[q];
    grad[g] = s;
}

size_t a256(size_t x) { return (x + 255) & ~size_t(255); }

// Workspace: the per-record counts, offsets and scan scratch (sized by the
// record count) come first; the (id, contribution) pairs and the sort scratch
// (sized by the pair count) follow.
struct VjpLayout {
    size_t counts, offsets, scan_tmp, scan_bytes, ids, ids2, vals, vals2, sort_tmp, sort_bytes, total;
};

VjpLayout vjp_layout(long long K, long long pairs) {
    VjpLayout L;
    const size_t k = size_t(std::max<long long>(K, 1));
    const size_t m = size_t(std::max<long long>(pairs, 1));
    size_t o = 0;
    auto take = [&](size_t b) { const size_t a = o; o = a256(o + b); return a; };
    L.counts = take(k * 4);
    L.offsets = take(k * 8);
    L.scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, L.scan_bytes, (int*)nullptr, (long long*)nullptr, int(k));
    L.scan_tmp = take(L.scan_bytes);
    L.ids = take(m * 4);
    L.ids2 = take(m * 4);
    L.vals = take(m * 8);
    L.vals2 = take(m * 8);
    L.sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, L.sort_bytes, (unsigned*)nullptr, (unsigned*)nullptr, (double*)nullptr,
                                    (double*)nullptr, int(std::min<size_t>(m, INT_MAX)), 0, 32);
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
                 void* workspace, int64_t workspace_bytes, void* stream) {
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
    const wcb::SceneHandle* h = scene->h;
    const long long K = num_selected;
    const long long P = layout[8];
    if (K == 0) {
        return cudaMemsetAsync(grad_out, 0, size_t(P) * 8, s) == cudaSuccess ? WCB_OK : WCB_ERR_CUDA;
    }
    wcb::adj::VjpLayout L = wcb::adj::vjp_layout(K, 1);
    if (workspace == nullptr || workspace_bytes < (long long)L.ids) return WCB_ERR_CAPACITY;
    char* b = static_cast<char*>(workspace);
    wcb::adj::AdjParams p;
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
    p.rows = static_cast<const wcb::RowRec*>(rows);
    p.selected = reinterpret_cast<const long long*>(selected);
    p.count = K;
    p.g_gain = grad_path_gain;
    p.g_re = grad_field_real;
    p.g_im = grad_field_imag;
    p.want = want;
    p.vertex_mask = vertex_mask;
    p.base_meps = int(layout[1]);
    p.base_msig = int(layout[2]);
    p.base_leps = int(layout[3]);
    p.base_lsig = int(layout[4]);
    p.gid_freq = int(layout[5]);
    p.base_tx = int(layout[6]);
    p.base_rx = int(layout[7]);
    p.counts = reinterpret_cast<int*>(b + L.counts);
    long long* offsets = reinterpret_cast<long long*>(b + L.offsets);
    p.offsets = offsets;
    p.row_field = row_field;
    const int grid = int((K + wcb::adj::kBlock - 1) / wcb::adj::kBlock);
    wcb::adj::k_vjp_count<<<grid, wcb::adj::kBlock, 0, s>>>(p);
    size_t tb = L.scan_bytes;
    if (cub::DeviceScan::ExclusiveSum(b + L.scan_tmp, tb, p.counts, offsets, int(K), s) != cudaSuccess)
        return WCB_ERR_CUDA;
    wcb::note_launch(2);
    long long last_off = 0;
    int last_cnt = 0;
    cudaMemcpyAsync(&last_off, offsets + K - 1, 8, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(&last_cnt, p.counts + K - 1, 4, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return WCB_ERR_CUDA;
    const long long pairs = last_off + last_cnt;
    if (pairs >= INT_MAX) return WCB_ERR_NOT_SUPPORTED;
    L = wcb::adj::vjp_layout(K, pairs);
    if (workspace_bytes < (long long)L.total) return WCB_ERR_CAPACITY;
    p.out_ids = reinterpret_cast<unsigned*>(b + L.ids);
    p.out_vals = reinterpret_cast<double*>(b + L.vals);
    wcb::adj::k_vjp_rows<wcb::adj::kLanes, 0><<<grid, wcb::adj::kBlock, 0, s>>>(p);
    wcb::adj::k_vjp_rows<wcb::adj::kLanes, 1><<<grid, wcb::adj::kBlock, 0, s>>>(p);
    wcb::adj::k_vjp_rows<wcb::adj::kLanes, 5><<<grid, wcb::adj::kBlock, 0, s>>>(p);
    wcb::adj::launch_vjp_diffraction(p, grid, s);
    wcb::note_launch(4);
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
    wcb::adj::k_vjp_reduce<<<int((P + 255) / 256), 256, 0, s>>>(P, pairs, ids2, vals2, grad_out);
    wcb::note_launch();
    rc = cudaGetLastError() == cudaSuccess ? WCB_OK : WCB_ERR_CUDA;
    return rc;
}

}  // extern "C"
