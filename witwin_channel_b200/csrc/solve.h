// Kernel parameter blocks shared by the solve and row translation units.
#pragma once

#include <stdint.h>

#include "../../include/witwin_channel_b200.h"
#include "scene.cuh"

namespace wcb {

// Device layout of wcb_row (48 bytes).
struct RowRec {
    int tx;
    int rx;
    short component;
    short depth;
    int seq[5];
    int edge;
    float length;
    int pad;
    int pad2;
};
static_assert(sizeof(RowRec) == 48, "RowRec must match wcb_row");
static_assert(sizeof(wcb_row) == 48, "wcb_row must be 48 bytes");

struct MainParams {
    SceneDev sc;
    int num_tx, num_rx;
    int rx_kind;
    const float* rx_pos;
    float grid_origin[3], grid_x[3], grid_y[3];
    int grid_rows, grid_cols;
    float grid_spacing[2];
    const float* rx_pol;
    int rx_pol_stride;
    const float* tx_pos;
    const float* tx_power;
    const float* tx_pol;
    // frequencies of this launch (chunk of at most four)
    double freq[4];
    double k[4];
    int freq_base;
    int num_freq_total;
    // materials (already offset to this chunk's first frequency)
    int num_materials;
    const float* mat_eps_r;
    const float* mat_sigma_e;
    const float* mat_mu_r;
    const float* mat_gain;
    const float* mat_thickness;
    const int* mat_volumetric;
    int num_layers;
    const int* layer_offset;
    const int* layer_count;
    const float* layer_thickness;
    const float* layer_eps_r;
    const float* layer_sigma_e;
    const float* layer_mu_r;
    int components;
    int max_depth;
    int coherent;
    // candidates
    const int* chain_count;          // (T, 5)
    const long long* chain_offset;   // (T, 5) in chain-int units
    const int* chain_groups;
    const double* chain_planes;
    const double* chain_images;
    const float4* chain_pre;         // per chain: last plane (n, offset) and last image (xyz, group) in FP32
    const int* edge_count;           // (T)
    const int* edge_list;            // (T, E)
    // outputs
    void* out_path_gain;
    void* out_field;
    void* out_comp_power;
    void* out_comp_field;
    void* out_diff_vec_power;
    RowRec* rows;
    long long row_capacity;
    unsigned long long* row_counter;
    int* status;
    unsigned long long* overflow_counter;
    unsigned long long* ray_counter;  // segment/ray queries traced (optional)
};

// Optional measurement of the main kernel: CUDA events bracket each launch
// and the ray counter is read back after the solve.
struct ProfileState {
    bool enabled = false;
    double main_ms = 0.0;        // summed time of the per-cell kernels of the last solve
    double prep_ms = 0.0;        // candidate preparation time of the last solve
    long long rays = 0;          // rays traced by the per-cell kernels in the last solve
    long long prep_rays = 0;     // rays traced while preparing candidates (discovery, edge prefilter)
    long long main_launches = 0;
    double kernel_ms[4] = {0, 0, 0, 0};       // los+transmission, reflection, diffraction, finalize
    double diffract_vis_ms = 0.0;             // the visibility part of the diffraction time
    long long kernel_rays[3] = {0, 0, 0};     // los+transmission, reflection, diffraction
    long long chains[5] = {0, 0, 0, 0, 0};    // reflection candidates per depth (first transmitter)
    long long edges = 0;                      // diffraction edges kept by the prefilter (first transmitter)
    // accumulated since profiling was last enabled (over every solve and VJP)
    long long acc_rays = 0;                   // rays traced by all solves (preparation and per-cell kernels)
    double acc_vjp_diff_ms = 0.0;             // reverse-mode diffraction VJP kernel time
    long long acc_vjp_diff_records = 0;       // diffraction records it processed
    long long acc_vjp_diff_launches = 0;
};
ProfileState& profile_state();

struct SceneHandle;
int solve_workspace_size(const SceneHandle* h, const wcb_solve_desc* d, int64_t* bytes);
int solve(const SceneHandle* h, const wcb_solve_desc* d, const wcb_materials* m, const wcb_outputs* out, void* ws,
          int64_t ws_bytes, cudaStream_t stream);

}  // namespace wcb
