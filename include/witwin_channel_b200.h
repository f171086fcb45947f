/*
 * witwin_channel_b200 -- C ABI of the B200 deterministic radiomap/path engine.
 *
 * Plain pointers, sizes and a cudaStream_t (passed as void*); no C++ or
 * framework types.  Every entry point returns a wcb_status; device-side
 * failures are reported through a status word the host reads, never by a
 * device trap.  The caller owns every buffer passed in; scene handles own
 * their scene tables.
 *
 * Reference interfaces replaced (paths within witwin-ai/witwin-channel):
 *   wcb_scene_create   <- scene/compiler.py:1306-1450 (compile) +
 *                         scene/resources.py:169-240 (RayD scene build) +
 *                         propagation/geometry.py:128-161 (coplanar groups) +
 *                         native/channel/kernels/diffraction.cu:803-900 and
 *                         scene/resources.py:356-405 (edge selection/refinement)
 *   wcb_solve          <- deterministic.py:786-949 (_solve_pipeline) through
 *                         propagation/enumerated.py:549-836 and the native ops
 *                         it calls (los.cu:74-125, paths.cu:317-361,
 *                         rayd/reflection.cpp:24-57, rayd/diffraction.cpp,
 *                         rayd/geometry.cpp:188-212, fields.cu:36-204,
 *                         deterministic.cu:829-970)
 *   wcb_rows_*         <- evaluated_paths.cu:560-760 (canonical sort, dedup,
 *                         max_paths) + deterministic.py:461-514 (path table)
 *   wcb_field_*        <- kernels/fields.py facades over fields.cu:36-204 and
 *                         RayD's field_transmission_sequence
 *   wcb_accumulate_flat* <- kernels/deterministic.py:23-367 over
 *                         deterministic.cu:829-1262 (forward, adjoint, JVP)
 *   wcb_rows_vjp       <- the field AD Functions in kernels/fields.py:1087-2140 and
 *                         the frozen-winner re-solve of propagation/geometry.py:214-286
 */
#ifndef WITWIN_CHANNEL_B200_H
#define WITWIN_CHANNEL_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    WCB_OK = 0,
    WCB_ERR_INVALID_ARGUMENT = 1,
    WCB_ERR_CUDA = 2,
    WCB_ERR_CAPACITY = 3,        /* a caller buffer is too small; *_needed reports the size */
    WCB_ERR_BVH_DEPTH = 4,       /* traversal stack would overflow */
    WCB_ERR_NOT_SUPPORTED = 5,
    WCB_ERR_DEVICE_STATUS = 6    /* a kernel reported a failure bit */
} wcb_status;

/* Component bits. */
#define WCB_COMPONENT_LOS 1
#define WCB_COMPONENT_REFLECTION 2
#define WCB_COMPONENT_DIFFRACTION 4
#define WCB_COMPONENT_TRANSMISSION 8

/* Precision modes. */
#define WCB_PRECISION_MIXED 0 /* FP32 traversal/fields, FP64 image solve, length and phase */
#define WCB_PRECISION_FP64 1  /* every stage in FP64 */

typedef struct wcb_scene wcb_scene;

/* Scene build.  All pointers are device pointers.
 * vertices (V,3) f32; faces (F,3) i32; face_surface, face_structure,
 * face_material (F) i32.  boundary_half_plane: keep boundary edges as
 * half-planes; vertical_only with vertical_ratio filters edges by |dz|/length. */
int wcb_scene_create(const float* vertices, int64_t num_vertices, const int32_t* faces, int64_t num_faces,
                     const int32_t* face_surface, const int32_t* face_structure, const int32_t* face_material,
                     int32_t boundary_half_plane, int32_t vertical_only, double vertical_ratio, void* stream,
                     wcb_scene** out);
int wcb_scene_destroy(wcb_scene* scene);
/* Moves a compiled scene's vertices in place (the reference recompiles the
 * scene when its mesh changes: scene/compiler.py:1306-1450 behind the compile
 * cache of deterministic.py:960-971).  `vertices` (V,3) f32 device, V as at
 * create.  The compile's discrete decisions (coplanar groups, edge selection
 * and wedge order, shared-boundary merges, the edge policy) are recomputed
 * from the new vertices and compared with the compiled ones first; if any
 * differs, nothing is changed and *topology_changed (host) is set to 1: the
 * caller must create the scene again.  Otherwise face planes, group planes
 * and boxes, edge frames, leaf triangles and the BVH boxes are recomputed on
 * the device (the BVH topology is kept) and *topology_changed is 0.  Reads
 * back two small values (one stream synchronisation); the mesh stays on the
 * device. */
int wcb_scene_refit(wcb_scene* scene, const float* vertices, int64_t num_vertices, int32_t* topology_changed,
                    void* stream);
/* counts[0..5] = faces, groups, selected edges, bvh depth, bvh nodes, representative faces */
/* Rebuilds the compiled scene's BVH on the device from its current vertices
 * (a linear BVH from 30-bit Morton codes of the face
 * centroids, radix-sorted, the radix tree of Karras (HPG 2012), boxes
 * bottom-up); no reference counterpart (the reference builds its BVH inside
 * RayD on the host at compile, scene/compiler.py:1306-1450).  Same node
 * layout as the compile's SAH tree, so every kernel traverses it unchanged;
 * the discrete compile decisions (groups, edges) are untouched.  *depth
 * (may be NULL) receives the tree depth.  A tree deeper than the traversal
 * stack returns WCB_ERR_BVH_DEPTH and leaves the old tree in place.
 * Synchronises `stream`; no solve on this scene may run meanwhile. */
int wcb_scene_rebuild_bvh(wcb_scene* scene, int32_t* depth, void* stream);
int wcb_scene_info(const wcb_scene* scene, int64_t* counts);
/* Group table export: face_group (F) i32, group_rep (G) i32 (device). */
int wcb_scene_groups(const wcb_scene* scene, int32_t* face_group, int32_t* group_rep, void* stream);
/* Selected edge export: edge_id (E) i32 (device). */
int wcb_scene_edges(const wcb_scene* scene, int32_t* edge_id, void* stream);

/* Material tables at each solve frequency.  Per-material arrays are (NF, M)
 * row-major; layer arrays are (NF, L) with a CSR (offset, count) per material
 * shared across frequencies. */
typedef struct {
    int32_t num_materials;
    const float* eps_r;
    const float* sigma_e;
    const float* mu_r;
    const float* gain;
    const float* thickness;
    const int32_t* volumetric; /* (M) */
    int32_t num_layers;
    const int32_t* layer_offset; /* (M) */
    const int32_t* layer_count;  /* (M) */
    const float* layer_thickness;
    const float* layer_eps_r;
    const float* layer_sigma_e;
    const float* layer_mu_r;
} wcb_materials;

/* Endpoints and solve options. */
typedef struct {
    int32_t num_tx;
    const float* tx_pos;    /* (T,3) device */
    const float* tx_power;  /* (T)   device */
    const float* tx_pol;    /* (T,3) device */
    int32_t rx_kind;        /* 0: points, 1: grid */
    int32_t num_rx;
    const float* rx_pos;    /* (R,3) device; points only */
    float grid_origin[3];
    float grid_x_axis[3];
    float grid_y_axis[3];
    int32_t grid_rows;
    int32_t grid_cols;
    float grid_spacing[2];
    const float* rx_pol;     /* (R,3) or (1,3) device */
    int32_t rx_pol_stride;   /* 3 for per-receiver polarization, 0 for one shared vector */
    int32_t num_freq;
    const double* frequency_hz; /* host array (NF) */
    int32_t components;      /* WCB_COMPONENT_* bits */
    int32_t max_depth;
    int32_t coherent;
    int32_t precision;       /* WCB_PRECISION_* */
    int32_t discovery_rays;  /* 0 selects the default 262144 */
    int32_t stack_entries;   /* traversal stack entries per thread; 0 = the scene's BVH depth + 2.  A smaller
                                value makes descents that need more drop the far subtree and set status bit 0
                                (a failure-path test hook: results are then incomplete) */
} wcb_solve_desc;

/* Per-cell outputs, all device, NF-major:
 *   path_gain (NF,T,R) f32, field (NF,T,R) complex64 (interleaved f32 pairs),
 *   comp_power (6,NF,T,R) f32, comp_field (6,NF,T,R) complex64,
 *   diff_vec_power (NF,T,R) f32 (sum over xyz of |sum_paths E|^2).
 * Any pointer may be NULL to skip that output.  In FP64 precision mode the
 * same outputs are float64 / complex128.
 * rows: optional compact path records (wcb_row, 48 bytes each); row_count is
 * a device int64 that receives the number of valid paths (it may exceed
 * row_capacity, in which case the call returns WCB_ERR_CAPACITY).
 * status: device int32 receiving device failure bits (bit 0: a traversal
 * stack overflowed).
 * transmission_overflow: optional device int64 receiving the number of
 * transmitter-receiver segments that cross more than max_depth walls; such a
 * segment yields no transmission path (the reference flags it in its capacity
 * failure state, runtime.py:1280-1290 SEGMENT_PENETRATION_FAILURE). */
typedef struct {
    void* path_gain;
    void* field;
    void* comp_power;
    void* comp_field;
    void* diff_vec_power;
    void* rows;
    int64_t row_capacity;
    int64_t* row_count;
    int32_t* status;
    int64_t* transmission_overflow;
} wcb_outputs;

/* Compact path record (the frozen topology of one path). */
typedef struct {
    int32_t tx;
    int32_t rx;
    int16_t component;  /* 0 LoS, 1 reflection, 2 diffraction, 5 transmission */
    int16_t depth;
    int32_t seq[5];     /* resolved face ids, -1 padded */
    int32_t edge;       /* reference edge id for diffraction, else -1 */
    float length;       /* path length (m) */
    int32_t reserved[2];
} wcb_row;

/* Scratch bytes a wcb_solve call needs for `desc`. */
int wcb_solve_workspace_size(const wcb_scene* scene, const wcb_solve_desc* desc, int64_t* bytes);

/* Full fused solve on one scene. */
int wcb_solve(const wcb_scene* scene, const wcb_solve_desc* desc, const wcb_materials* materials,
              const wcb_outputs* outputs, void* workspace, int64_t workspace_bytes, void* stream);

/* Canonical order of path records: sorts, removes duplicate identities
 * (shortest kept, NaN drops the group) and applies max_paths (-1 = none;
 * scope 0 global, 1 per pair).  Writes the selected record indices in
 * canonical order to `selected` (capacity num_rows) and their count to
 * *num_selected (host).  The sort key keeps every field at full width (any
 * number of sources, sinks and object ids).  Reads counts back and
 * synchronises `stream` before returning. */
int wcb_rows_select(const void* rows, int64_t num_rows, int32_t width, int64_t max_paths, int32_t scope,
                    int64_t* selected, int64_t* num_selected, void* workspace, int64_t workspace_bytes, void* stream);
int wcb_rows_select_workspace_size(int64_t num_rows, int64_t* bytes);

/* Integer columns of selected records (the record-to-table unpacking of
 * propagation/topology.py:408-466 evaluated_paths_from_block): per selected
 * index i, tx_id, rx_id, component_id, depth, primitive_sequence (5 per row),
 * edge_id and length of rows[selected[i]].  One pass; any output may be NULL.
 * No host sync. */
int wcb_rows_decode(const void* rows, const int64_t* selected, int64_t num_selected, int32_t* tx_id, int32_t* rx_id,
                    int32_t* component_id, int32_t* depth, int32_t* primitive_sequence, int32_t* edge_id,
                    float* length, void* stream);

/* wcb_rows_select without a caller workspace and without any allocation (no
 * counterpart in the reference, whose selection allocates through torch).
 * For callers that may not allocate device memory at call time: code inside
 * an out-of-memory handler, real-time loops where a cudaMalloc would
 * synchronise the device, hosts with pools frozen after start-up.  The
 * scratch is a fixed WCB_ROWS_SELECT_NOALLOC_SCRATCH_BYTES array in the
 * library's device image; inputs whose wcb_rows_select_workspace_size exceeds
 * it (above 597,120 records) return WCB_ERR_CAPACITY before any work.  Every
 * call looks up the array's address on the current device; the first lookup
 * on a device may load the library's module there, so make the first call on
 * a device before any stream capture begins.  The call reads its counts back
 * and synchronises `stream` before returning, so it blocks the calling
 * thread.  All calls on a device share
 * the array (each call rewrites what it reads), so calls that overlap in time
 * race: serialise them. */
#define WCB_ROWS_SELECT_NOALLOC_SCRATCH_BYTES (32ll << 20)
int wcb_rows_select_noalloc(const void* rows, int64_t num_rows, int32_t width, int64_t max_paths, int32_t scope,
                            int64_t* selected, int64_t* num_selected, void* stream);

/* Field evaluation of selected path records at one frequency (index freq
 * into the materials tables).  Writes the path-table columns; any output
 * pointer may be NULL. */
typedef struct {
    float* path_length_m;   /* (K) */
    float* delay_s;         /* (K) */
    float* path_gain;       /* (K) */
    float* path_field;      /* (K) complex64 */
    float* coefficient;     /* (K) complex64 */
    float* field_xyz;       /* (K,3) complex64, unit excitation */
    float* field_direction; /* (K,3) */
    float* interaction_positions; /* (K,W,3) */
    float* interaction_normals;   /* (K,W,3) */
    float* phase_rad;       /* (K) */
} wcb_row_fields;

int wcb_rows_evaluate(const wcb_scene* scene, const wcb_solve_desc* desc, const wcb_materials* materials,
                      int32_t freq_index, const void* rows, const int64_t* selected, int64_t num_selected,
                      int32_t width, const wcb_row_fields* out, void* stream);

/* Per-cell accumulation of evaluated rows (selected, canonical order):
 * per-slot coherent sums and gains written like wcb_outputs for one
 * frequency (NF = 1).  Deterministic: every cell sums its rows in canonical
 * order. */
int wcb_rows_accumulate(const void* rows, const int64_t* selected, int64_t num_selected,
                        const float* path_gain, const float* path_field, const float* field_xyz,
                        const float* tx_power, int32_t num_tx, int32_t num_rx, int32_t coherent,
                        const wcb_outputs* outputs, void* stream);

/* Flat accumulation of evaluated paths (replaces the reference op
 * deterministic_accumulate_flat: kernels/deterministic.py:23-102 over
 * native/channel/kernels/deterministic.cu:829-970).  Per path: valid flag
 * (1 byte), tx, rx, component id (0 los, 1 reflection, 2 diffraction,
 * 3/4/7 coupled, 5 transmission, 6 scattering), gain and field (real, imag)
 * in `dtype`.  Paths with an out-of-range tx/rx or an unknown component are
 * dropped.  Outputs: power_total, field_total_real/imag (T,R) and
 * component_power, component_field_real/imag (6,T,R), all in `dtype`, each
 * element written once.  Every slot sums its paths in path index order, so
 * results are bit-reproducible. */
#define WCB_DTYPE_F32 0
#define WCB_DTYPE_F64 1
typedef struct {
    void* power_total;
    void* field_total_real;
    void* field_total_imag;
    void* component_power;
    void* component_field_real;
    void* component_field_imag;
} wcb_accumulate_outputs;
int wcb_accumulate_flat_workspace_size(int64_t num_paths, int64_t* bytes);
int wcb_accumulate_flat(const uint8_t* valid, const int32_t* tx_id, const int32_t* rx_id, const int32_t* component_id,
                        const void* path_gain, const void* field_real, const void* field_imag, int64_t num_paths,
                        int32_t num_tx, int32_t num_rx, int32_t coherent, int32_t scattering_coherent, int32_t dtype,
                        const wcb_accumulate_outputs* outputs, void* workspace, int64_t workspace_bytes,
                        void* stream);
/* Pushforward of wcb_accumulate_flat (replaces deterministic_accumulate_flat_jvp,
 * kernels/deterministic.py:155-185): tangents of gain/field per path (any
 * NULL = zero) give the tangents of all six outputs in `tangent_out`,
 * linearised at the forward outputs in `saved`. */
int wcb_accumulate_flat_jvp_workspace_size(int64_t num_paths, int32_t dtype, int64_t* bytes);
int wcb_accumulate_flat_jvp(const uint8_t* valid, const int32_t* tx_id, const int32_t* rx_id,
                            const int32_t* component_id, const void* tangent_path_gain, const void* tangent_field_real,
                            const void* tangent_field_imag, int64_t num_paths, int32_t num_tx, int32_t num_rx,
                            int32_t coherent, int32_t scattering_coherent, int32_t dtype,
                            const wcb_accumulate_outputs* saved, const wcb_accumulate_outputs* tangent_out,
                            void* workspace, int64_t workspace_bytes, void* stream);
/* Adjoint of wcb_accumulate_flat (replaces deterministic_accumulate_flat_backward,
 * kernels/deterministic.py:115-152): `saved` holds the forward outputs, `grads`
 * their cotangents (any member NULL = zero).  Writes per-path gradients of
 * gain and field (real, imag); dropped paths get zeros. */
int wcb_accumulate_flat_backward(const uint8_t* valid, const int32_t* tx_id, const int32_t* rx_id,
                                 const int32_t* component_id, int64_t num_paths, int32_t num_tx, int32_t num_rx,
                                 int32_t coherent, int32_t scattering_coherent, int32_t dtype,
                                 const wcb_accumulate_outputs* saved, const wcb_accumulate_outputs* grads,
                                 void* grad_path_gain, void* grad_field_real, void* grad_field_imag, void* stream);

/* Fixed-topology VJP of selected path records (replaces the reference's
 * deterministic AD: kernels/fields.py:1087-2140 field Functions and the
 * frozen-winner re-solve of propagation/geometry.py:214-286).  Given per-record
 * cotangents of path gain and path field (real, imag; FP64, any NULL = 0),
 * writes the dense FP64 gradient `grad_out` over the layout of
 * wcb_rows_vjp_layout: layout[0..7] are the offsets of vertices (V,3),
 * material eps_r (M), material sigma_e (M), layer eps_r (L), layer sigma_e
 * (L), frequency (1), Tx positions (T,3) and point-receiver positions (R,3);
 * layout[8] is the total.  `want` bits: 1 Tx, 2 Rx, 4 frequency, 8 vertices,
 * 16 materials (unrequested parts are written as zeros); vertex_mask (V bytes,
 * NULL = all) limits the vertex gradient to the vertices marked nonzero.  Records are
 * re-evaluated from raw scene values in FP64 (no stored intermediates): LoS,
 * reflection and transmission records in dual numbers, diffraction records by
 * a reverse-mode sweep; the per-parameter sums are deterministic.  row_field
 * (optional, (K,2) FP64) receives each record's re-evaluated path field.
 * order / comp_counts (optional, from wcb_rows_order on the same selection)
 * replace the call's own grouping of the records. */
int wcb_rows_vjp_layout(const wcb_scene* scene, const wcb_solve_desc* desc, const wcb_materials* materials,
                        int64_t* layout);
int wcb_rows_vjp_workspace_size(int64_t num_selected, int32_t max_depth, int32_t max_layers, int64_t* bytes);
int wcb_rows_vjp(const wcb_scene* scene, const wcb_solve_desc* desc, const wcb_materials* materials,
                 int32_t freq_index, const void* rows, const int64_t* selected, int64_t num_selected,
                 const double* grad_path_gain, const double* grad_field_real, const double* grad_field_imag,
                 int32_t want, const uint8_t* vertex_mask, double* grad_out, int64_t grad_size, double* row_field,
                 const int32_t* order, const int64_t* comp_counts, void* workspace, int64_t workspace_bytes,
                 void* stream);

/* Fixed-topology JVP of selected path records (replaces the reference's
 * forward-mode companions run inside the forward pass for ad_mode="jvp":
 * deterministic.py:733-742, kernels/fields.py field Functions' jvp,
 * native/channel/kernels/fields.cu:1193-1356 and :2183).  `tangent` is a dense
 * FP64 tangent vector over the layout of wcb_rows_vjp_layout (tangent_size >=
 * layout[8]); each record is re-evaluated once in FP64 with one dual lane
 * seeded by it.  Writes row_field_tangent (K,2) FP64, the directional
 * derivative of each record's powered path field (real, imag), and optionally
 * row_field (K,2) FP64, the re-evaluated field.  With tangent NULL only
 * row_field is written (a plain FP64 evaluation, no dual lane): the records'
 * fields the derivatives are linearised at.  order / comp_counts (optional,
 * from wcb_rows_order) run each component's records in that order.
 * freq_index -1 (tangent NULL): the fields at every frequency of the desc,
 * row_field (NF,K,2); diffraction records form their frequency-independent
 * UTD geometry once for up to 4 frequencies.  No workspace, no host sync. */
int wcb_rows_jvp(const wcb_scene* scene, const wcb_solve_desc* desc, const wcb_materials* materials,
                 int32_t freq_index, const void* rows, const int64_t* selected, int64_t num_selected,
                 const double* tangent, int64_t tangent_size, double* row_field, double* row_field_tangent,
                 const int32_t* order, const int64_t* comp_counts, void* stream);

/* Execution order of selected records for the derivative kernels (no
 * reference counterpart: it only reorders their work).  order (K int32)
 * receives the selection indices grouped by component (LoS, reflection,
 * transmission, diffraction), then depth, diffraction records by edge,
 * selection order kept within a group; comp_counts (host, 4 int64) the group
 * sizes.  Warps of one edge share the wedge and most branches of the UTD.
 * The result depends only on the records, so one order serves every
 * frequency and pass over them.  Synchronises its stream.  Workspace:
 * wcb_rows_order_workspace_size bytes. */
int wcb_rows_order_workspace_size(int64_t num_selected, int64_t* bytes);
int wcb_rows_order(const wcb_scene* scene, const void* rows, const int64_t* selected, int64_t num_selected,
                   int32_t* order, int64_t* comp_counts, void* workspace, int64_t workspace_bytes, void* stream);

/* Channel frequency response of path records (replaces PathResult.cfr,
 * path.py:646-656): per (tx, rx) cell and subcarrier k,
 * H_k = sum_p a_p exp(-j 2 pi (tau_p - tau_min) f_k), tau_min the cell's
 * smallest delay when normalize_delays (else 0).  Records (tx, rx, delay,
 * complex coefficient a) must be grouped by cell in (rx, tx) order (the
 * canonical order).  Subcarriers: f0 + k df for df != 0, else the device
 * array `frequencies` (num_freq, FP64).  out: (T,R,num_freq) complex64, every
 * element written once.  Workspace: wcb_cfr_workspace_size bytes. */
int wcb_cfr_workspace_size(int32_t num_tx, int32_t num_rx, int64_t* bytes);
int wcb_cfr(const int32_t* tx_id, const int32_t* rx_id, const float* delay_s, const float* path_field,
            int64_t num_paths, int32_t num_tx, int32_t num_rx, int32_t num_freq, double f0, double df,
            const double* frequencies, int32_t normalize_delays, float* out, void* workspace,
            int64_t workspace_bytes, void* stream);

/* Standalone field operators (reference kernels/fields.py facades).  All
 * arrays are device f32; complex outputs interleaved.  N rows. */
int wcb_field_free_space(int64_t n, const float* source, const float* target, const float* tx_power,
                         const float* tx_pol, const float* rx_pol, double frequency_hz, float* field_vector,
                         float* coefficient, float* path_field, float* path_gain, float* path_length,
                         float* delay, float* direction, void* stream);
int wcb_field_reflection_sequence(int64_t n, int32_t depth, const float* source, const float* target,
                                  const float* positions, const float* normals, const float* tx_power,
                                  const float* tx_pol, const float* rx_pol, const float* eps_r,
                                  const float* sigma_e, const float* mu_r, const float* gain,
                                  const float* thickness, double frequency_hz, float* field_vector,
                                  float* coefficient, float* path_field, float* path_gain, float* path_length,
                                  float* delay, float* direction, void* stream);
/* Straight thin-sheet chain: normals (N,D,3), material ids (N,D) i32 and
 * per-row wall count (N) i32; materials as in wcb_materials (NF = 1). */
int wcb_field_transmission_sequence(int64_t n, int32_t depth, const float* source, const float* target,
                                    const float* normals, const int32_t* material_ids, const int32_t* wall_count,
                                    const float* tx_power, const float* tx_pol, const float* rx_pol,
                                    const wcb_materials* materials, double frequency_hz, float* field_vector,
                                    float* coefficient, float* path_field, float* path_gain, float* path_length,
                                    float* delay, float* direction, void* stream);
int wcb_field_project_complex3(int64_t n, const float* field_vector, const float* direction, const float* rx_pol,
                               float* coefficient, float* path_gain, void* stream);

/* Line-of-sight Jones operator between per-endpoint transverse frames
 * (replaces consumer_los_jones, witwin/channel/propagation/consumer.py:2037-2093,
 * and its kernel native/channel/kernels/los.cu:2001-2078).  Row i takes pair
 * p = pair_index[i]: source p % num_sources, sink p / num_sources.  Reference
 * bases are (num_sources,2,3) and (num_sinks,2,3) f32; each endpoint's frame
 * is its first vector made transverse to the LoS direction and unit, and
 * direction x that vector turned to the side of its second vector.  Outputs
 * (N rows): matrix (N,2,2) complex64 interleaved, matrix[i][a][b] the
 * unit-excitation response of sink frame vector a to source frame vector b;
 * source_basis, sink_basis (N,2,3) the frames used.  A pair outside
 * [0, num_sources*num_sinks) writes NaN to its row and sets bit 0 of *status
 * (status may be NULL). */
int wcb_los_jones(const int64_t* pair_index, int64_t num_rows, const float* source_positions, int64_t num_sources,
                  const float* sink_positions, int64_t num_sinks, const float* source_reference_basis,
                  const float* sink_reference_basis, double frequency_hz, float* matrix, float* source_basis,
                  float* sink_basis, int32_t* status, void* stream);

/* Fixed-topology replay of frozen line-of-sight and reflection records at new
 * endpoint positions (replaces reevaluate and its bucket replay,
 * witwin/channel/propagation/consumer.py:3846-4110, with prepared_row_gather
 * :2375-2449, _los_inputs / _reflection_inputs :2734-2811, evaluate_prepared
 * :3029-3096 and the direct-plane EPC re-solve propagation/geometry.py:214-264).
 * One launch replays every record and every frequency column, plus one launch
 * for the pair segmentation; no host synchronisation.
 *
 * Records (wcb_frozen_rows, all device, K rows): component_id 0 (LoS, depth 0)
 * or 1 (reflection, depth 1..width); primitive_sequence (K,width) the faces of
 * the bounces; source_index / sink_index into the endpoint batches;
 * source_id / sink_id the stable ids the records were discovered with (NULL:
 * no identity check); order (NULL: row order) a permutation of the rows that
 * sets the execution order only.
 * Endpoints (wcb_endpoint_batch, device): positions (N,3), polarizations (N,3),
 * stable_ids (N) i64, powers (N) (sources), polarization_basis (N,2,3) (only
 * read when out->jones is set).
 * slot_count >= 1: pair p of row i is sink*num_sources+source for one slot and
 * the block-diagonal layout slot*ss*ks + (sink-slot*ks)*ss + (source-slot*ss)
 * otherwise (ss, ks the per-slot counts; the slot is the source's).
 * materials: num_columns frequency columns (column c at frequencies[c],
 * a device FP64 array), as wcb_materials with NF = num_columns.
 * test_visibility: re-test each LoS record's segment and each reflection
 * record's plane crossings, containment in its faces' coplanar groups and
 * legs against the scene, as discovery does (FP32 segment tests); a record
 * that fails is published with row_valid 0 and zero field, length, delay and
 * direction.  With 0 every record is evaluated as valid.
 *
 * status (device int32[2], caller-zeroed): status[0] the contract bits of the
 * reference's validation mask, 1 a source or sink index outside its batch, 2
 * in-bounds rows not in non-decreasing pair order, 16 a stable id that differs
 * from the batch's, 32 a slot-batched row whose sink lies outside its
 * source's slot; status[1] engine bits, 1 traversal stack overflow, 2 a
 * record whose component or depth this replay does not take, 4 a face id
 * outside the scene.  A row with any bit is written as invalid zeros.
 * Any output pointer may be NULL. */
typedef struct {
    int64_t num_rows;
    int32_t width;
    const int32_t* component_id;
    const int32_t* depth;
    const int32_t* primitive_sequence;
    const int32_t* source_index;
    const int32_t* sink_index;
    const int64_t* source_id;
    const int64_t* sink_id;
    const int32_t* order;
} wcb_frozen_rows;

typedef struct {
    int64_t count;
    const float* positions;
    const float* polarizations;
    const int64_t* stable_ids;
    const float* powers;
    const float* polarization_basis;
} wcb_endpoint_batch;

typedef struct {
    float* coefficient;          /* (K) complex64, column 0: receiver-projected, sqrt(power) */
    float* coefficient_offsets;  /* (K,C-1) complex64, columns 1.. */
    float* field;                /* (K,3) complex64, column 0: world-Cartesian, sqrt(power) */
    float* field_offsets;        /* (K,C-1,3) complex64 */
    float* path_length_m;        /* (K) */
    float* delay_s;              /* (K) */
    float* direction;            /* (K,3) arrival direction */
    float* interaction_positions; /* (K,width,3) */
    float* interaction_normals;  /* (K,width,3) */
    uint8_t* row_valid;          /* (K) */
    float* jones;                /* (K,2,2) complex64, column 0, unit excitation */
    float* source_basis;         /* (K,2,3) */
    float* sink_basis;           /* (K,2,3) */
    int64_t* pair_index;         /* (K) */
    int64_t* pair_offsets;       /* (P+1), P = slot_count * per-slot sources * per-slot sinks */
} wcb_replay_outputs;

int wcb_rows_replay(const wcb_scene* scene, const wcb_frozen_rows* rows, const wcb_endpoint_batch* sources,
                    const wcb_endpoint_batch* sinks, int64_t slot_count, const wcb_materials* materials,
                    const double* frequencies, int32_t num_columns, int32_t test_visibility,
                    const wcb_replay_outputs* out, int32_t* status, void* stream);

/* Measurement: when enabled, wcb_solve brackets its candidate preparation and
 * its main kernel with CUDA events on the solve stream and counts the rays
 * (segment visibility / penetration queries) the main kernel traces.
 * wcb_profile_read returns the last solve's figures: values[0] main-kernel ms,
 * values[1] preparation ms, values[2] main-kernel rays, values[3] main-kernel
 * launches, values[4] preparation rays (discovery bounces, edge prefilter),
 * values[5..8] ms of the LoS+transmission, reflection, diffraction and
 * finalize kernels, values[9..11] rays of the first three, values[12..16]
 * reflection candidates per depth, values[17] prefiltered diffraction
 * edges (both for the first transmitter) and values[18] the ms of the
 * diffraction visibility kernel (part of values[7]).  Accumulated since the
 * last wcb_profile_enable(1): values[19] rays of every solve (preparation and
 * main kernels), values[20] ms of the reverse-mode diffraction VJP kernel
 * (wcb_rows_vjp brackets it with events and synchronises its stream),
 * values[21] the diffraction records it processed, values[22] its launches.
 * `values` holds 23 doubles. */
int wcb_profile_enable(int32_t enabled);
int wcb_profile_read(double* values);

/* Runtime info: writes a NUL-terminated description (architecture, build). */
int wcb_build_info(char* buffer, int64_t capacity);
/* Number of kernel launches issued by this library since load. */
int64_t wcb_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* WITWIN_CHANNEL_B200_H */
