// Library-internal declarations shared by the CUDA translation units.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <vector>

#include "scene.cuh"
#include "../../include/witwin_channel_b200.h"

namespace wcb {

struct SceneHandle {
    SceneDev dev;
    std::vector<void*> owned;
    int* edge_ids = nullptr;     // (E) device, reference edge id of each selected edge
    int* edge_slot = nullptr;    // (edges total) device, selected index of each reference edge or -1
    int* edge_topo = nullptr;    // (E,4) device: va, vb (edge direction vb - va), fn0, fn1 (-1: half-plane)
    std::vector<int> group_rep_host;
    std::vector<int> face_group_host;
    int num_edges_total = 0;
    int num_nodes = 0;
    // device caches of the compile's discrete decisions (for scene_refit)
    int* face_surface = nullptr;         // (F)
    long long* face_keys = nullptr;      // (F,5) coplanar group keys (refit scratch)
    int4* edge_rec = nullptr;            // (NE) v0, v1, f0, f1 of every edge record
    unsigned char* edge_state = nullptr; // (NE) bit 0 wedge order, 1 coplanar, 2 selected before merges, 3 final
    long long* edge_qkey = nullptr;      // (NE,6) quantised endpoints of shared-boundary candidates (refit scratch)
    int* edge_qhead = nullptr;           // (NE) first record of a candidate's endpoint class; -1 not a candidate
    int* key_table = nullptr;            // open-addressing table of class keys for the refit's distinctness check
    int key_table_slots = 0;             // power of two, at least twice the classes
    int* edge_partner = nullptr;         // (NE) merged partner of a pair head; -2 merged away; -1 none
    int* leaf_parent = nullptr;          // (F) parent node << 1 | side (-1: none)
    int* node_parent = nullptr;          // (F-1) parent node << 1 | side (-1: root)
    int* bvh_counter = nullptr;          // (F-1) refit arrival counters
    int* refit_flag = nullptr;           // (1)
    double* diagonal_dev = nullptr;      // (1)
    int half_plane_policy = 1;
    int vertical_only_policy = 0;
    double vertical_ratio = 0.7;
};

int scene_create(const float* vertices, int64_t nv, const int32_t* faces, int64_t nf, const int32_t* surface,
                 const int32_t* structure, const int32_t* material, int boundary_half_plane, int vertical_only,
                 double vertical_ratio, cudaStream_t stream, SceneHandle** out);
void scene_destroy(SceneHandle* h);
int scene_refit(SceneHandle* h, const float* d_vertices, int64_t nv, int* topology_changed, cudaStream_t stream);

int rows_select_workspace(int64_t n, int64_t* bytes);
int rows_decode(const void* rows, const int64_t* selected, int64_t n, int32_t* tx, int32_t* rx, int32_t* component,
                int32_t* depth, int32_t* seq, int32_t* edge, float* length, cudaStream_t stream);
int rows_select(const void* rows, int64_t n, int width, int64_t max_paths, int scope, int64_t* selected,
                int64_t* num_selected, void* ws, int64_t ws_bytes, cudaStream_t stream);
int rows_evaluate(const SceneHandle* h, const wcb_solve_desc* d, const wcb_materials* m, int fi, const void* rows,
                  const int64_t* selected, int64_t count, int width, const wcb_row_fields* out, cudaStream_t stream);
int rows_accumulate(const void* rows, const int64_t* selected, int64_t n, const float* path_gain, const float* path_field,
                    const float* field_xyz, const float* tx_power, int num_tx, int num_rx, int coherent,
                    const wcb_outputs* out, cudaStream_t stream);
int field_free_space(int64_t n, const float* s, const float* t, const float* pw, const float* tp, const float* rp, double f,
                     float* fv, float* c, float* pf, float* pg, float* pl, float* dl, float* dr, cudaStream_t stream);
int refit_boxes(SceneHandle* h, cudaStream_t stream);
int scene_rebuild_bvh(SceneHandle* h, int* depth_out, cudaStream_t stream);
int rows_replay(const SceneHandle* h, const wcb_frozen_rows* rows, const wcb_endpoint_batch* src,
                const wcb_endpoint_batch* snk, int64_t slot_count, const wcb_materials* m, const double* freqs,
                int num_columns, int visibility, const wcb_replay_outputs* out, int* status, cudaStream_t stream);
int los_jones(int64_t n, const int64_t* pair, const float* src, int64_t num_src, const float* snk, int64_t num_snk,
              const float* src_ref, const float* snk_ref, double f, float* matrix, float* src_basis, float* snk_basis,
              int* status, cudaStream_t stream);
int field_reflection(int64_t n, int depth, const float* s, const float* t, const float* pos, const float* nrm, const float* pw,
                     const float* tp, const float* rp, const float* eps, const float* sig, const float* mu, const float* gain,
                     const float* th, double f, float* fv, float* c, float* pf, float* pg, float* pl, float* dl, float* dr,
                     cudaStream_t stream);
int field_transmission(int64_t n, int depth, const float* s, const float* t, const float* nrm, const int* mids,
                       const int* counts, const float* pw, const float* tp, const float* rp, const wcb_materials* m,
                       double f, float* fv, float* c, float* pf, float* pg, float* pl, float* dl, float* dr,
                       cudaStream_t stream);
int field_project(int64_t n, const float* fv, const float* dir, const float* rp, float* c, float* pg, cudaStream_t stream);

extern std::atomic<long long> g_launch_count;
inline void note_launch(int n = 1) { g_launch_count.fetch_add(n, std::memory_order_relaxed); }

}  // namespace wcb
