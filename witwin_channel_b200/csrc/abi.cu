// extern "C" entry points of libwcb200.so.  Thin wrappers: argument checks,
// status mapping and stream casting; the work lives in scene.cu, solve.cu and
// rows.cu.
#include <atomic>
#include <cstdio>
#include <cstring>

#include "../../include/witwin_channel_b200.h"
#include "internal.h"
#include "solve.h"

namespace wcb {
std::atomic<long long> g_launch_count{0};
}

struct wcb_scene {
    wcb::SceneHandle* h;
};

static cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

extern "C" {

int wcb_scene_create(const float* vertices, int64_t num_vertices, const int32_t* faces, int64_t num_faces,
                     const int32_t* face_surface, const int32_t* face_structure, const int32_t* face_material,
                     int32_t boundary_half_plane, int32_t vertical_only, double vertical_ratio, void* stream,
                     wcb_scene** out) {
    if (out == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (num_faces > 0 && (vertices == nullptr || faces == nullptr || face_surface == nullptr ||
                          face_structure == nullptr || face_material == nullptr))
        return WCB_ERR_INVALID_ARGUMENT;
    wcb::SceneHandle* h = nullptr;
    const int rc = wcb::scene_create(vertices, num_vertices, faces, num_faces, face_surface, face_structure,
                                     face_material, boundary_half_plane, vertical_only, vertical_ratio,
                                     as_stream(stream), &h);
    if (rc != 0) return rc;
    *out = new wcb_scene{h};
    return WCB_OK;
}

int wcb_scene_destroy(wcb_scene* scene) {
    if (scene == nullptr) return WCB_OK;
    wcb::scene_destroy(scene->h);
    delete scene;
    return WCB_OK;
}

int wcb_scene_refit(wcb_scene* scene, const float* vertices, int64_t num_vertices, int32_t* topology_changed,
                    void* stream) {
    if (scene == nullptr || topology_changed == nullptr || num_vertices < 0) return WCB_ERR_INVALID_ARGUMENT;
    int changed = 0;
    const int rc = wcb::scene_refit(scene->h, vertices, num_vertices, &changed, as_stream(stream));
    *topology_changed = changed;
    return rc;
}

int wcb_scene_info(const wcb_scene* scene, int64_t* counts) {
    if (scene == nullptr || counts == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    const wcb::SceneDev& d = scene->h->dev;
    counts[0] = d.num_faces;
    counts[1] = d.num_groups;
    counts[2] = d.num_edges;
    counts[3] = d.max_depth;
    counts[4] = scene->h->num_nodes;
    counts[5] = scene->h->num_edges_total;
    return WCB_OK;
}

int wcb_scene_groups(const wcb_scene* scene, int32_t* face_group, int32_t* group_rep, void* stream) {
    if (scene == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    const wcb::SceneDev& d = scene->h->dev;
    if (face_group && d.num_faces)
        cudaMemcpyAsync(face_group, d.face_group, size_t(d.num_faces) * 4, cudaMemcpyDeviceToDevice, as_stream(stream));
    if (group_rep && d.num_groups)
        cudaMemcpyAsync(group_rep, d.group_rep, size_t(d.num_groups) * 4, cudaMemcpyDeviceToDevice, as_stream(stream));
    return cudaGetLastError() == cudaSuccess ? WCB_OK : WCB_ERR_CUDA;
}

int wcb_scene_edges(const wcb_scene* scene, int32_t* edge_id, void* stream) {
    if (scene == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    const wcb::SceneDev& d = scene->h->dev;
    if (edge_id && d.num_edges)
        cudaMemcpyAsync(edge_id, scene->h->edge_ids, size_t(d.num_edges) * 4, cudaMemcpyDeviceToDevice, as_stream(stream));
    return cudaGetLastError() == cudaSuccess ? WCB_OK : WCB_ERR_CUDA;
}

int wcb_solve_workspace_size(const wcb_scene* scene, const wcb_solve_desc* desc, int64_t* bytes) {
    if (scene == nullptr || desc == nullptr || bytes == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    return wcb::solve_workspace_size(scene->h, desc, bytes);
}

int wcb_solve(const wcb_scene* scene, const wcb_solve_desc* desc, const wcb_materials* materials,
              const wcb_outputs* outputs, void* workspace, int64_t workspace_bytes, void* stream) {
    if (scene == nullptr || desc == nullptr || materials == nullptr || outputs == nullptr)
        return WCB_ERR_INVALID_ARGUMENT;
    if (desc->max_depth < 0 || desc->max_depth > 5) return WCB_ERR_INVALID_ARGUMENT;
    if (desc->num_freq < 1 || desc->frequency_hz == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < desc->num_freq; ++i)
        if (!(desc->frequency_hz[i] > 0.0)) return WCB_ERR_INVALID_ARGUMENT;
    if (desc->num_tx > 0 && (desc->tx_pos == nullptr || desc->tx_power == nullptr || desc->tx_pol == nullptr))
        return WCB_ERR_INVALID_ARGUMENT;
    if (desc->rx_kind == 0 && desc->num_rx > 0 && desc->rx_pos == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    if (desc->rx_pol == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    const int rc = wcb::solve(scene->h, desc, materials, outputs, workspace, workspace_bytes, as_stream(stream));
    if (rc != 0) return rc;
    if (outputs->rows != nullptr && outputs->row_count != nullptr) {
        int64_t n = 0;
        cudaMemcpyAsync(&n, outputs->row_count, 8, cudaMemcpyDeviceToHost, as_stream(stream));
        if (cudaStreamSynchronize(as_stream(stream)) != cudaSuccess) return WCB_ERR_CUDA;
        if (n > outputs->row_capacity) return WCB_ERR_CAPACITY;
    }
    return WCB_OK;
}

int wcb_rows_decode(const void* rows, const int64_t* selected, int64_t num_selected, int32_t* tx_id, int32_t* rx_id,
                    int32_t* component_id, int32_t* depth, int32_t* primitive_sequence, int32_t* edge_id,
                    float* length, void* stream) {
    return wcb::rows_decode(rows, selected, num_selected, tx_id, rx_id, component_id, depth, primitive_sequence,
                            edge_id, length, as_stream(stream));
}

int wcb_rows_select_workspace_size(int64_t num_rows, int64_t* bytes) {
    if (bytes == nullptr || num_rows < 0) return WCB_ERR_INVALID_ARGUMENT;
    return wcb::rows_select_workspace(num_rows, bytes);
}

int wcb_rows_select(const void* rows, int64_t num_rows, int32_t width, int64_t max_paths, int32_t scope,
                    int64_t* selected, int64_t* num_selected, void* workspace, int64_t workspace_bytes, void* stream) {
    if (num_selected == nullptr || (num_rows > 0 && (rows == nullptr || selected == nullptr)))
        return WCB_ERR_INVALID_ARGUMENT;
    if (width < 0 || width > 5 || (scope != 0 && scope != 1)) return WCB_ERR_INVALID_ARGUMENT;
    return wcb::rows_select(rows, num_rows, width, max_paths, scope, selected, num_selected, workspace,
                            workspace_bytes, as_stream(stream));
}

int wcb_rows_evaluate(const wcb_scene* scene, const wcb_solve_desc* desc, const wcb_materials* materials,
                      int32_t freq_index, const void* rows, const int64_t* selected, int64_t num_selected,
                      int32_t width, const wcb_row_fields* out, void* stream) {
    if (scene == nullptr || desc == nullptr || materials == nullptr || out == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    if (width < 0 || width > 5) return WCB_ERR_INVALID_ARGUMENT;
    return wcb::rows_evaluate(scene->h, desc, materials, freq_index, rows, selected, num_selected, width, out,
                              as_stream(stream));
}

int wcb_rows_accumulate(const void* rows, const int64_t* selected, int64_t num_selected, const float* path_gain,
                        const float* path_field, const float* field_xyz, const float* tx_power, int32_t num_tx,
                        int32_t num_rx, int32_t coherent, const wcb_outputs* outputs, void* stream) {
    if (outputs == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    return wcb::rows_accumulate(rows, selected, num_selected, path_gain, path_field, field_xyz, tx_power, num_tx,
                                num_rx, coherent, outputs, as_stream(stream));
}

int wcb_field_free_space(int64_t n, const float* source, const float* target, const float* tx_power,
                         const float* tx_pol, const float* rx_pol, double frequency_hz, float* field_vector,
                         float* coefficient, float* path_field, float* path_gain, float* path_length, float* delay,
                         float* direction, void* stream) {
    if (!(frequency_hz > 0.0)) return WCB_ERR_INVALID_ARGUMENT;
    return wcb::field_free_space(n, source, target, tx_power, tx_pol, rx_pol, frequency_hz, field_vector, coefficient,
                                 path_field, path_gain, path_length, delay, direction, as_stream(stream));
}

int wcb_scene_rebuild_bvh(wcb_scene* scene, int32_t* depth, void* stream) {
    if (scene == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    int d = 0;
    const int rc = wcb::scene_rebuild_bvh(scene->h, &d, as_stream(stream));
    if (depth) *depth = d;
    if (rc == 4) return WCB_ERR_BVH_DEPTH;
    return rc == 0 ? WCB_OK : (rc == 1 ? WCB_ERR_INVALID_ARGUMENT : WCB_ERR_CUDA);
}

int wcb_rows_replay(const wcb_scene* scene, const wcb_frozen_rows* rows, const wcb_endpoint_batch* sources,
                    const wcb_endpoint_batch* sinks, int64_t slot_count, const wcb_materials* materials,
                    const double* frequencies, int32_t num_columns, int32_t test_visibility,
                    const wcb_replay_outputs* out, int32_t* status, void* stream) {
    if (scene == nullptr || rows == nullptr || sources == nullptr || sinks == nullptr || materials == nullptr ||
        out == nullptr || status == nullptr)
        return WCB_ERR_INVALID_ARGUMENT;
    if (rows->num_rows < 0 || rows->width < 0 || rows->width > 5 || slot_count < 1 || num_columns < 1 ||
        sources->count < 0 || sinks->count < 0 || sources->count % slot_count != 0 || sinks->count % slot_count != 0)
        return WCB_ERR_INVALID_ARGUMENT;
    if (sources->count > 0 && sinks->count > INT64_MAX / sources->count) return WCB_ERR_INVALID_ARGUMENT;
    if (rows->num_rows > 0) {
        if (rows->component_id == nullptr || rows->depth == nullptr || rows->source_index == nullptr ||
            rows->sink_index == nullptr || (rows->width > 0 && rows->primitive_sequence == nullptr) ||
            sources->count == 0 || sinks->count == 0 || sources->positions == nullptr ||
            sources->polarizations == nullptr || sinks->positions == nullptr || sinks->polarizations == nullptr ||
            frequencies == nullptr)
            return WCB_ERR_INVALID_ARGUMENT;
        if ((rows->source_id != nullptr && sources->stable_ids == nullptr) ||
            (rows->sink_id != nullptr && sinks->stable_ids == nullptr))
            return WCB_ERR_INVALID_ARGUMENT;
        if (out->jones != nullptr && (sources->polarization_basis == nullptr || sinks->polarization_basis == nullptr))
            return WCB_ERR_INVALID_ARGUMENT;
        if (materials->num_materials > 0 && (materials->eps_r == nullptr || materials->sigma_e == nullptr ||
                                              materials->mu_r == nullptr || materials->gain == nullptr ||
                                              materials->thickness == nullptr))
            return WCB_ERR_INVALID_ARGUMENT;
    }
    if (out->pair_offsets != nullptr && rows->num_rows > 0 && out->pair_index == nullptr)
        return WCB_ERR_INVALID_ARGUMENT;
    return wcb::rows_replay(scene->h, rows, sources, sinks, slot_count, materials, frequencies, num_columns,
                            test_visibility, out, status, as_stream(stream));
}

int wcb_los_jones(const int64_t* pair_index, int64_t num_rows, const float* source_positions, int64_t num_sources,
                  const float* sink_positions, int64_t num_sinks, const float* source_reference_basis,
                  const float* sink_reference_basis, double frequency_hz, float* matrix, float* source_basis,
                  float* sink_basis, int32_t* status, void* stream) {
    if (num_rows < 0 || !(frequency_hz > 0.0)) return WCB_ERR_INVALID_ARGUMENT;
    if (num_rows == 0) return WCB_OK;
    if (pair_index == nullptr || source_positions == nullptr || sink_positions == nullptr ||
        source_reference_basis == nullptr || sink_reference_basis == nullptr || matrix == nullptr ||
        source_basis == nullptr || sink_basis == nullptr || num_sources <= 0 || num_sinks <= 0 ||
        num_sources > INT64_MAX / num_sinks)
        return WCB_ERR_INVALID_ARGUMENT;
    return wcb::los_jones(num_rows, pair_index, source_positions, num_sources, sink_positions, num_sinks,
                          source_reference_basis, sink_reference_basis, frequency_hz, matrix, source_basis, sink_basis,
                          status, as_stream(stream));
}

int wcb_field_reflection_sequence(int64_t n, int32_t depth, const float* source, const float* target,
                                  const float* positions, const float* normals, const float* tx_power,
                                  const float* tx_pol, const float* rx_pol, const float* eps_r, const float* sigma_e,
                                  const float* mu_r, const float* gain, const float* thickness, double frequency_hz,
                                  float* field_vector, float* coefficient, float* path_field, float* path_gain,
                                  float* path_length, float* delay, float* direction, void* stream) {
    if (!(frequency_hz > 0.0)) return WCB_ERR_INVALID_ARGUMENT;
    return wcb::field_reflection(n, depth, source, target, positions, normals, tx_power, tx_pol, rx_pol, eps_r, sigma_e,
                                 mu_r, gain, thickness, frequency_hz, field_vector, coefficient, path_field, path_gain,
                                 path_length, delay, direction, as_stream(stream));
}

int wcb_field_transmission_sequence(int64_t n, int32_t depth, const float* source, const float* target,
                                    const float* normals, const int32_t* material_ids, const int32_t* wall_count,
                                    const float* tx_power, const float* tx_pol, const float* rx_pol,
                                    const wcb_materials* materials, double frequency_hz, float* field_vector,
                                    float* coefficient, float* path_field, float* path_gain, float* path_length,
                                    float* delay, float* direction, void* stream) {
    if (!(frequency_hz > 0.0) || materials == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    return wcb::field_transmission(n, depth, source, target, normals, material_ids, wall_count, tx_power, tx_pol,
                                   rx_pol, materials, frequency_hz, field_vector, coefficient, path_field, path_gain,
                                   path_length, delay, direction, as_stream(stream));
}

int wcb_field_project_complex3(int64_t n, const float* field_vector, const float* direction, const float* rx_pol,
                               float* coefficient, float* path_gain, void* stream) {
    return wcb::field_project(n, field_vector, direction, rx_pol, coefficient, path_gain, as_stream(stream));
}

int wcb_profile_enable(int32_t enabled) {
    wcb::ProfileState& st = wcb::profile_state();
    st.enabled = enabled != 0;
    if (st.enabled) {
        st.acc_rays = 0;
        st.acc_vjp_diff_ms = 0.0;
        st.acc_vjp_diff_records = 0;
        st.acc_vjp_diff_launches = 0;
    }
    return WCB_OK;
}

int wcb_profile_read(double* values) {
    if (values == nullptr) return WCB_ERR_INVALID_ARGUMENT;
    const wcb::ProfileState& st = wcb::profile_state();
    values[0] = st.main_ms;
    values[1] = st.prep_ms;
    values[2] = double(st.rays);
    values[3] = double(st.main_launches);
    values[4] = double(st.prep_rays);
    for (int i = 0; i < 4; ++i) values[5 + i] = st.kernel_ms[i];
    for (int i = 0; i < 3; ++i) values[9 + i] = double(st.kernel_rays[i]);
    for (int i = 0; i < 5; ++i) values[12 + i] = double(st.chains[i]);
    values[17] = double(st.edges);
    values[18] = st.diffract_vis_ms;
    values[19] = double(st.acc_rays);
    values[20] = st.acc_vjp_diff_ms;
    values[21] = double(st.acc_vjp_diff_records);
    values[22] = double(st.acc_vjp_diff_launches);
    return WCB_OK;
}

int wcb_build_info(char* buffer, int64_t capacity) {
    if (buffer == nullptr || capacity <= 0) return WCB_ERR_INVALID_ARGUMENT;
    std::snprintf(buffer, size_t(capacity), "witwin_channel_b200 sm_100a cuda %d", CUDART_VERSION);
    return WCB_OK;
}

int64_t wcb_launch_count(void) { return wcb::g_launch_count.load(); }

}  // extern "C"
