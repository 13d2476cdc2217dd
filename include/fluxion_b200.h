/*
 * fluxion_b200.h -- C ABI of the B200-native HAPR placement hot path.
 *
 * This header is the drop-in boundary. Each entry point names the reference
 * interface it replaces (paths are relative to the reference project:
 * H/ = HAPR_fluxion_v4/, O/ = neon_old_codebase/).
 *
 * Conventions
 *   - Every call returns an int status: FX_OK (0) or a negative FX_E* code.
 *     No exception or abort crosses this boundary. fx_last_error() returns a
 *     thread-local message describing the most recent failure.
 *   - Host arrays are caller-owned. They are read-only unless the parameter
 *     name starts with out_ or the comment says "in/out".
 *   - Device state lives behind opaque handles (fx_ctx, fx_design). One
 *     context is driven by one host thread at a time; distinct contexts may
 *     run on distinct host threads.
 *   - Netlists are flat index arrays: net e connects the gates
 *     net_gate[net_ptr[e] .. net_ptr[e+1]-1]. This is the reference's
 *     Circuit::net_gate_indices (H/src/data/circuit.rs:62) flattened to CSR.
 *   - Positions are SoA float32 x[N], y[N] (H/src/data/placement.rs:9-13).
 */
#ifndef FLUXION_B200_H_
#define FLUXION_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define FX_OK        0
#define FX_EINVAL   -1 /* bad argument, malformed CSR, out-of-range index     */
#define FX_ENOMEM   -2 /* device or host allocation failed                    */
#define FX_ECUDA    -3 /* a CUDA runtime/driver call failed                   */
#define FX_ETIMEOUT -4 /* a bounded device-side wait gave up                  */
#define FX_EADMIT   -5 /* serving admission refused (HBM budget exceeded)     */
#define FX_ENODEV   -6 /* no usable sm_100 device                             */

typedef struct fx_ctx fx_ctx;
typedef struct fx_design fx_design;

/* Thread-local description of the last failure on this thread. */
const char *fx_last_error(void);
/* Library version string ("fluxion_b200 <major>.<minor>"). */
const char *fx_version(void);

/* ---- context ----------------------------------------------------------- */
/* Creates a context on CUDA device `device` (an sm_100 B200). Replaces
 * GpuContext::new (H/src/gpu/context.rs:17-70); unlike the reference there is
 * no CPU fallback: a missing device is FX_ENODEV. */
int fx_ctx_create(fx_ctx **out_ctx, int device);
int fx_ctx_destroy(fx_ctx *ctx);
/* Turns per-stage CUDA-event timing on (1) or off (0). */
int fx_ctx_set_profiling(fx_ctx *ctx, int enable);
/* Limits the timing to the stages whose bit (1 << FX_STAGE_*) is set in
 * stage_mask (all stages by default). Each timed stage adds two events to
 * its stream, so a long timed run can time only the stages it reports. */
int fx_ctx_set_profiling_stages(fx_ctx *ctx, uint32_t stage_mask);
/* Per-stage timing accumulated since the last reset, in milliseconds:
 * out_ms[s] total device time and out_calls[s] launches of stage s
 * (FX_STAGE_*). n = capacity of both arrays. */
int fx_ctx_stage_times(fx_ctx *ctx, double *out_ms, int64_t *out_calls, int n);
int fx_ctx_reset_stage_times(fx_ctx *ctx);
/* Number of kernels this library has launched on the context. */
int64_t fx_ctx_kernel_launches(fx_ctx *ctx);
/* Device-side timing on the context's main stream: fx_ctx_mark records
 * event `slot` (0..15); fx_ctx_elapsed waits for both and returns the
 * milliseconds between two recorded slots. */
int fx_ctx_mark(fx_ctx *ctx, int slot);
int fx_ctx_elapsed(fx_ctx *ctx, int slot_a, int slot_b, float *out_ms);
/* Waits until all work queued on the context has finished. */
int fx_ctx_synchronize(fx_ctx *ctx);

/* Stage identifiers for fx_ctx_stage_times. */
#define FX_STAGE_ATTRACT_INTEGRATE 0 /* rows A+E fused                        */
#define FX_STAGE_BH_KEYS           1 /* row B: Morton keys                    */
#define FX_STAGE_BH_SORT           2 /* row B: radix sort                     */
#define FX_STAGE_BH_TREE           3 /* row B: radix tree + mass sums         */
#define FX_STAGE_BH_WALK           4 /* row B: warp-cooperative walk          */
#define FX_STAGE_DENSITY           5 /* row C: scatter + DCT GEMMs + field    */
#define FX_STAGE_CONGESTION        6 /* rows D+F: bbox, counting, HPWL        */
#define FX_STAGE_LEAF              7 /* row H: batched leaf placer            */
#define FX_STAGE_FIEDLER           8 /* row G: power iteration                */
#define FX_STAGE_ATTENTION         9 /* (f.4) attention scores of a level     */
#define FX_STAGE_COUNT             10

/* ---- designs (device-resident netlists) -------------------------------- */
/* Uploads a netlist and builds every device structure the hot path needs
 * (net CSR, gate->net incidence CSR, the deduplicated clique-expansion
 * adjacency of H/src/data/circuit.rs:154-171). Replaces the upload half of
 * dispatch_forces / dispatch_congestion (H/src/gpu/dispatch.rs:31-45,
 * 115-139). gate_w/gate_h may be NULL (reference defaults 2 x 10,
 * H/src/parser/blif.rs:49). Positions start at (0,0) as in Placement::new
 * (H/src/data/placement.rs:28-37). */
int fx_design_load(fx_ctx *ctx, int32_t n_gates, int32_t n_nets,
                   const int32_t *net_ptr, const int32_t *net_gate,
                   const float *gate_w, const float *gate_h,
                   float chip_w, float chip_h, fx_design **out_design);
int fx_design_free(fx_design *design);
/* Sizes: gates, nets, pins, directed adjacency entries. */
int fx_design_sizes(const fx_design *design, int64_t *out_n, int64_t *out_m,
                    int64_t *out_p, int64_t *out_a);
/* Host copy of the device adjacency CSR (out_adj_ptr[N+1], out_adj_idx[A]).
 * Each list holds the same neighbour set as circuit.rs:154-171. */
int fx_design_adjacency(const fx_design *design, int32_t *out_adj_ptr,
                        int32_t *out_adj_idx);
/* Host <-> device copies of the resident positions (and velocities, which
 * are zeroed by set_positions). */
int fx_design_set_positions(fx_design *design, const float *x, const float *y);
int fx_design_get_positions(fx_design *design, float *out_x, float *out_y);
/* Device-side checkpoint of the placement state (positions and velocities):
 * save_state copies the current state into a second device buffer set
 * (allocated on the first call), restore_state copies it back. Both are
 * stream-ordered device copies on the context's stream; restore before a
 * save fails with FX_EINVAL. No counterpart in the reference (its state
 * lives in host Vec<f32>s that the caller clones). */
int fx_design_save_state(fx_design *design);
int fx_design_restore_state(fx_design *design);
/* Device bytes held by the design (netlist + positions + workspaces). */
int64_t fx_design_device_bytes(const fx_design *design);

/* ---- rows D + F: congestion counting and HPWL --------------------------- */
/* Mirrors compute_congestion_cpu (H/src/algorithm/congestion.rs:11-62) with
 * the grid geometry of RoutingGrid::new / cell_at (H/src/data/grid.rs:25-62):
 * every net with >= 2 gate entries adds +1 to each cell of its bounding box
 * in both the h and v grids. The two grids are identical, so one uint32
 * count grid (rows x cols, row-major) is returned; h[i] == v[i] ==
 * (float)out_counts[i] exactly. Also returns the HPWL of
 * Placement::compute_hpwl (H/src/data/placement.rs:48-74) summed in FP64,
 * and the FP64 sum / f32 max of max(0, h+v-capacity) (grid.rs:71-91).
 * x/y: host positions, or NULL to use the design's resident positions.
 * Any out pointer may be NULL. */
int fx_congestion(fx_ctx *ctx, fx_design *design, const float *x,
                  const float *y, int32_t cols, int32_t rows,
                  uint32_t *out_counts, double *out_hpwl,
                  double *out_total_overflow, float *out_max_overflow);

/* Congestion without any device allocation. No counterpart in the reference
 * (its congestion runs on host Vecs); this is an extra entry point beside
 * fx_congestion for callers that may not allocate device memory during the
 * call: fx_congestion allocates its workspace on first use and again when
 * the grid changes size, which can fail when the caller's own memory pool
 * holds the HBM, and cudaFree waits for the whole device. Same kernels and
 * results as fx_congestion (bit-identical counts, HPWL and overflow).
 *
 * Scratch: one fixed 8 MiB device array per device inside the library;
 * the difference array needs (rows+1)*(cols+1)*4 bytes of it, so grids up to
 * 2,080,000 such entries (about 1440 x 1440) are accepted and larger ones
 * are rejected with FX_EINVAL (use fx_congestion for those).
 * Inputs and outputs are DEVICE pointers owned by the caller:
 *   d_x, d_y           positions (n_gates floats each), or both NULL to use
 *                      the design's resident positions;
 *   d_counts           rows*cols uint32 (required);
 *   d_hpwl_overflow    2 doubles {HPWL, total overflow}, or NULL;
 *   d_max_overflow     1 float, or NULL.
 * The work is enqueued on the context's stream and the call returns without
 * waiting; results are ready after fx_ctx_synchronize (or anything ordered
 * after that stream). The first call on a device sets the scratch up
 * (cudaGetSymbolAddress, then a zeroing on the context's stream that the
 * call waits for before it launches anything), so make that first call
 * before any stream capture begins. Calls share the scratch: two calls
 * that overlap on one device (different contexts, streams or host threads)
 * race and corrupt each other's counts; order them. */
int fx_congestion_noalloc(fx_ctx *ctx, const fx_design *design, const float *d_x,
                          const float *d_y, int32_t cols, int32_t rows,
                          uint32_t *d_counts, double *d_hpwl_overflow,
                          float *d_max_overflow);

/* ---- (f.2) hierarchy build: recursive spectral bisection ---------------- */
/* Mirrors build_hierarchy (H/src/algorithm/partitioner.rs:36-100, with
 * compute_fiedler_vector :106-185 and split_by_fiedler :189-213) and the
 * region pass of hapr_placement (H/src/algorithm/placer.rs:40-63,111-141):
 * returns the leaves in HierarchyTree::leaves() order (hierarchy.rs:176-190)
 * with their gates, regions (cx, cy, w, h) and depths. All clusters of one
 * depth run on the device together. */
#define FX_PART_EXACT 0 /* the reference's f32 iteration; identical leaves       */
#define FX_PART_FP64 1  /* FP64 norms / Rayleigh quotient, stop at tol           */
typedef struct fx_part_cfg {
  int32_t max_leaf_size;    /* PartitionConfig (partitioner.rs:24-32): 64        */
  int32_t min_cluster_size; /* 8                                                 */
  float balance_factor;     /* 0.4, in [0, 0.5]                                  */
  int32_t power_iterations; /* 30 (main.rs:80); EXACT runs exactly this many,    */
                            /* FP64 at most this many                            */
  int32_t mode;             /* FX_PART_*                                         */
  int32_t reserved0;
  double tol;               /* FP64: relative change of the Rayleigh quotient    */
} fx_part_cfg;
typedef struct fx_part_stats {
  int32_t n_leaves, n_nodes, max_depth, levels;
  int64_t power_iterations; /* summed over the bisected clusters                 */
} fx_part_stats;
int fx_part_cfg_default(fx_part_cfg *cfg);
/* out_leaf_ptr[leaf_capacity+1], out_leaf_gate[n_gates],
 * out_region[4*leaf_capacity], out_leaf_depth[leaf_capacity]; any may be NULL.
 * FX_EINVAL if the tree has more leaves than leaf_capacity. */
int fx_partition(fx_ctx *ctx, fx_design *design, const fx_part_cfg *cfg,
                 int32_t leaf_capacity, int32_t *out_leaf_ptr, int32_t *out_leaf_gate,
                 float *out_region, int32_t *out_leaf_depth, fx_part_stats *out_stats);

/* ---- (f.4) attention scores between the clusters of one level ------------ */
/* Mirrors compute_level_attention (H/src/algorithm/attention.rs:50-88) for
 * the clusters of one hierarchy level, given as a CSR over gates (disjoint;
 * gates in no cluster are ignored): score(A -> B) = |nets touching A and B| /
 * |nets touching A| in f32, and per cluster the top_k clusters by score
 * (descending, ties by smaller index, zero scores dropped; unused slots -1).
 * out_topk[n * top_k] and the dense out_scores[n * n] (row A, column B) are
 * host buffers and may be NULL. At most 65535 clusters. */
int fx_attention(fx_ctx *ctx, fx_design *design, int32_t n_clusters,
                 const int32_t *cluster_ptr, const int32_t *cluster_gate, int32_t top_k,
                 int32_t *out_topk, float *out_scores);
/* Mirrors compute_all_attention (H/src/algorithm/attention.rs:33-48) for a
 * hierarchy given as its leaves in DFS order (leaf_ptr[L+1] over leaf_gate,
 * leaf_depth[L], depths <= 62; every internal node has two children, as
 * build_hierarchy makes them): every depth with at least two clusters
 * (clusters_at_depth, hierarchy.rs:134-159), in depth order. Per level:
 * out_level_depth[v], out_level_clusters[v] (n_v, <= 65535) and n_v * top_k
 * top-k entries appended to out_topk (-1 padded; NULL to size the call).
 * FX_EINVAL when max_levels or topk_capacity is too small (the error text
 * gives the sizes); sum n_v <= 2 L. */
int fx_attention_tree(fx_ctx *ctx, fx_design *design, int32_t n_leaves,
                      const int32_t *leaf_ptr, const int32_t *leaf_gate,
                      const int32_t *leaf_depth, int32_t top_k, int32_t max_levels,
                      int32_t *out_n_levels, int32_t *out_level_depth,
                      int32_t *out_level_clusters, int64_t topk_capacity, int32_t *out_topk);

/* ---- rows A..F: the plain composite force iteration -------------------- */
typedef struct fx_iter_cfg {
  float attract_weight;  /* spring k (placer.rs:250, default 1.0)            */
  float repel_weight;    /* Barnes-Hut k (placer.rs:264, default 0.5)        */
  float min_dist;        /* distance floor (placer.rs:263, default 0.1)      */
  float theta;           /* opening angle (BarnesHutTree.cpp:16, 0.5)        */
  float density_weight;  /* weight of the DCT Poisson force (0 disables)     */
  float target_density;  /* rho_target (force_electrostatic.py:37)           */
  int32_t density_bins;  /* G: G x G density grid, G % 128 == 0 (0 = off)    */
  int32_t dct_precision; /* FX_DCT_*                                         */
  int32_t cong_cols;     /* congestion grid (0 = off)                        */
  int32_t cong_rows;
  float damping;         /* placer.rs:276 (0.9)                              */
  float dt;              /* placer.rs:276-279 (0.1)                          */
  int32_t bh_walk;       /* FX_BH_* (default FX_BH_FAST)                     */
} fx_iter_cfg;

/* Barnes-Hut walk. Both give every point the interaction list of the
 * reference's per-point opening rule (BarnesHutTree.cpp:145-167) on the
 * same tree and add its terms in the same order; they differ in the
 * inverse square root. */
#define FX_BH_FAST  0 /* hardware rsqrt; single points share the cell code:   */
                      /* forces within f32 rounding of the exact walk         */
#define FX_BH_EXACT 1 /* reproducible rsqrt (bit-level estimate + 3 Newton    */
                      /* steps): forces bit-identical to the oracle's f32 walk */

#define FX_DCT_FP32  0 /* 3xTF32 split on the tensor cores; its error grows   */
                       /* with G (6.6e-4 at 256, 4.4e-3 at 2048 measured):  */
                       /* FP32 inputs, not FP32 accuracy                     */
#define FX_DCT_TF32  1 /* single-pass TF32 inputs, FP32 accumulate           */
#define FX_DCT_BF16  2 /* BF16 inputs, FP32 accumulate                       */
#define FX_DCT_SIMT  3 /* FP32 CUDA-core GEMM (no tensor cores)              */
#define FX_DCT_I8    4 /* tensor cores, FP32-accurate: each operand row split */
                       /* into six exact 8-bit slices under a power-of-two    */
                       /* scale, slice products accumulated exactly in int32  */
                       /* (tcgen05 kind::i8), classes combined in FP64: the   */
                       /* iteration's default                                  */

typedef struct fx_iter_stats {
  double hpwl;            /* FP64 HPWL after the last iteration              */
  double total_overflow;  /* FP64 sum of congestion overflow                 */
  float max_overflow;     /* max cell overflow                               */
  float pad0;
  double density_energy;  /* 0.5 * sum q*phi at the gates (FP64)             */
  int64_t iterations;     /* iterations run                                  */
  int64_t bh_nodes;       /* internal nodes of the last Barnes-Hut tree      */
} fx_iter_stats;

/* Fills cfg with the defaults (H/config/default.yaml placement section plus
 * the Barnes-Hut and density defaults above). */
int fx_iter_cfg_default(fx_iter_cfg *cfg);

/* Runs `iters` plain composite iterations: F = attraction (placer.rs:243-255
 * over the full adjacency) + Barnes-Hut repulsion (law of placer.rs:258-272,
 * tree rules of O/src/cpp/BarnesHutTree.cpp) + DCT Poisson density force
 * (O/src/python/fluxion/force_electrostatic.py:47-150); then the damped
 * Euler step clamped to the die (placer.rs:275-280); then congestion + HPWL
 * on the new positions. Replaces dispatch_forces (H/src/gpu/dispatch.rs:
 * 18-106). x/y are in/out host arrays (NULL = run on resident positions and
 * leave them on the device). stats may be NULL. */
int fx_force_iterate(fx_ctx *ctx, fx_design *design, const fx_iter_cfg *cfg,
                     int32_t iters, float *x, float *y, fx_iter_stats *stats);

/* Force trace (no reference counterpart; a parity and diagnosis aid for
 * fx_force_iterate). While enabled, every plain iteration also stores, per
 * gate, the total f32 force its damped step integrated (attraction +
 * Barnes-Hut + density, exactly the value placer.rs:276-277 multiplies by
 * dt) and the positions and velocities it started from;
 * fx_design_trace_get returns those of the last iteration run (host
 * arrays of n_gates floats, each may be NULL). */
int fx_design_trace(fx_design *design, int enable);
/* With the trace enabled, fx_hapr_place_leaves also records each slot's
 * total force (springs + repulsion) of the first iteration, at the leaf's
 * deterministic start positions (placer.rs:226-227); this returns those of
 * the last batch, in leaf_gate order (out arrays of the batch's slot count,
 * each may be NULL). */
int fx_design_leaf_trace_get(fx_design *design, float *out_fx, float *out_fy);
int fx_design_trace_get(fx_design *design, float *out_fx, float *out_fy, float *out_x0,
                        float *out_y0, float *out_vx0, float *out_vy0);

/* Single-stage entry points on the resident positions (used by the parity
 * tests; each writes float32 forces to host arrays). */
/* Row A: out_f = k * sum_{j in adj(i)} (p_j - p_i)  (placer.rs:243-255). */
int fx_stage_attraction(fx_ctx *ctx, fx_design *design, float k,
                        float *out_fx, float *out_fy);
/* Row B: Barnes-Hut repulsion. Also returns the Morton keys in gate order
 * (out_keys[N]), the stable key order (out_perm[s] = gate at sorted
 * position s) and the root square (out_root[3] = {x_min, y_min, size});
 * any of the three may be NULL. */
int fx_stage_barnes_hut(fx_ctx *ctx, fx_design *design, float k, float theta,
                        float min_dist, float *out_fx, float *out_fy,
                        uint32_t *out_keys, int32_t *out_perm,
                        float *out_root);
/* The same with the walk chosen (FX_BH_*; fx_stage_barnes_hut is
 * FX_BH_EXACT). FX_BH_FAST can also return each gate's interaction count
 * (out_terms[N], NULL to skip): single points plus accepted cells. */
int fx_stage_barnes_hut_walk(fx_ctx *ctx, fx_design *design, float k, float theta,
                             float min_dist, int32_t walk, float *out_fx, float *out_fy,
                             uint32_t *out_keys, int32_t *out_perm, float *out_root,
                             int32_t *out_terms);
/* Row C: DCT Poisson density force. Optional grids (G*G, row-major, may be
 * NULL): out_rho (charge density rho - rho_target), out_phi, out_ex,
 * out_ey. */
int fx_stage_density(fx_ctx *ctx, fx_design *design, int32_t bins,
                     float target_density, float weight, int32_t precision,
                     float *out_fx, float *out_fy, float *out_rho,
                     float *out_phi, float *out_ex, float *out_ey,
                     double *out_energy);

/* ---- row H: batched leaf placement --------------------------------------- */
typedef struct fx_leaf_cfg {
  int32_t force_iterations; /* PlacerConfig::force_iterations (default 50)    */
  float attract_weight;     /* placer.rs:250 (1.0)                            */
  float repel_weight;       /* placer.rs:264 (0.5)                            */
  float damping;            /* placer.rs:276 (0.9)                            */
  float dt;                 /* placer.rs:276-279 (0.1)                        */
  int32_t schedule;         /* FX_LEAF_*                                      */
  int32_t precision;        /* FX_LEAF_IEEE (default) or FX_LEAF_FAST         */
  int32_t reserved1;
} fx_leaf_cfg;

/* Arithmetic of the pair repulsion term (placer.rs:258-272). */
#define FX_LEAF_IEEE 0 /* the reference's sqrt and three divisions: positions  */
                       /* bit-identical to place_gates_in_leaf                 */
#define FX_LEAF_FAST 1 /* repel * d * rsqrt(max(|d|^2, 0.01))^3, hardware      */
                       /* rsqrt: forces within f32 rounding of the IEEE form   */

#define FX_LEAF_AUTO        0 /* time the schedules once, keep the fastest   */
#define FX_LEAF_WARP        1 /* one warp per leaf, 8 leaves per block        */
#define FX_LEAF_CTA64       2 /* 64 threads per leaf                          */
#define FX_LEAF_CTA128      3 /* 128 threads per leaf                         */
#define FX_LEAF_CTA256      4 /* one 256-thread block per leaf                */
#define FX_LEAF_PER_CLUSTER 5 /* baseline: one kernel launch per leaf         */
#define FX_LEAF_PAIR64      6 /* pair-triangle, 64 threads per leaf (<= 128 gates) */
#define FX_LEAF_PAIR128     7 /* pair-triangle, 128 threads per leaf (<= 128 gates) */
#define FX_LEAF_PAIR256     8 /* pair-triangle, 256 threads per leaf (<= 128 gates) */

int fx_leaf_cfg_default(fx_leaf_cfg *cfg);

/* Places every leaf with place_gates_in_leaf (H/src/algorithm/placer.rs:
 * 210-287) -- the leaf loop of hapr_placement (placer.rs:65-69) -- in one
 * persistent launch. Leaf l holds the gates leaf_gate[leaf_ptr[l] ..
 * leaf_ptr[l+1]-1] (at most 512) and the region (cx, cy, w, h) =
 * region[4l..4l+3]. Attraction uses the design's adjacency restricted to the
 * leaf. Results are bit-identical to the reference's f32 loop. out_x/out_y
 * (length N) are in/out: leaf gates are overwritten, other gates keep their
 * values. out_schedule (may be NULL) receives the schedule used. */
int fx_hapr_place_leaves(fx_ctx *ctx, fx_design *design, int32_t n_leaves,
                         const int32_t *leaf_ptr, const int32_t *leaf_gate,
                         const float *region, const fx_leaf_cfg *cfg,
                         float *out_x, float *out_y, int32_t *out_schedule);

/* ---- row G: batched power iteration ------------------------------------- */
/* Runs compute_fiedler_vector (H/src/algorithm/partitioner.rs:106-185) for
 * every cluster at once: cluster c is the gate list cluster_gate[
 * cluster_ptr[c] .. cluster_ptr[c+1]-1] (clusters must not share gates);
 * its induced Laplacian uses the design's adjacency. The start vector is the
 * reference's sin(i * 2.71828), normalised; each iteration applies L, removes
 * the mean (deflation against the constant vector) and normalises.
 * tol = 0 runs exactly max_iters iterations (the reference uses 30,
 * H/src/main.rs:80) with the reference's f32 mean and norm (sequential
 * folds), so the vectors are bit-identical to compute_fiedler_vector's;
 * tol > 0 takes the mean and norm in FP64 and stops a cluster once its
 * Rayleigh quotient changes by at most tol relative. out_v[G] receives each
 * cluster's vector (same order as cluster_gate); out_iters[C] and
 * out_lambda[C] (may be NULL) the iterations run and the Rayleigh quotient
 * v^T L v / v^T v of the returned vector, in FP64. */
int fx_fiedler(fx_ctx *ctx, fx_design *design, int32_t n_clusters,
               const int32_t *cluster_ptr, const int32_t *cluster_gate,
               int32_t max_iters, double tol, float *out_v,
               int32_t *out_iters, double *out_lambda);

/* ---- congestion refinement (the loop of the next pipeline stage) -------- */
typedef struct fx_refine_cfg {
  int32_t max_iterations;   /* RefineConfig::max_iterations (100)            */
  float move_distance;      /* max move per step (5.0)                       */
  float overflow_threshold; /* hot-cell threshold and stop level (1.0 in the
                               default YAML, H/config/default.yaml:37)       */
  int32_t grid_cols;        /* routing grid (256 x 256)                       */
  int32_t grid_rows;
  int32_t reserved0;
} fx_refine_cfg;

typedef struct fx_refine_stats {
  int64_t iterations;       /* iterations that moved gates                   */
  int64_t moves;            /* gate moves in total                           */
  float total_overflow;     /* final f32 total overflow (grid.rs:86-91)      */
  float max_overflow;       /* final max overflow -> Placement::max_congestion */
  double hpwl;              /* final HPWL (FP64)                             */
} fx_refine_stats;

int fx_refine_cfg_default(fx_refine_cfg *cfg);

/* refine_placement (H/src/algorithm/refiner.rs:34-126): repeat congestion ->
 * f32 total overflow -> stop when <= threshold or after 10 stalled
 * iterations (change < 1 %) -> move every gate of a hot cell toward the
 * first least-congested cell within radius 3, clamped to move_distance and
 * the die. Positions end bit-identical to the reference loop. x/y: in/out
 * host positions, or NULL to refine the resident positions. out_counts
 * (rows x cols, may be NULL) receives the final congestion counts. */
int fx_refine(fx_ctx *ctx, fx_design *design, const fx_refine_cfg *cfg,
              float *x, float *y, fx_refine_stats *stats, uint32_t *out_counts);

/* ---- serving: continuous batching of placement and ECO jobs ------------- */
/* A request server on one GPU (continuous batching; the reference
 * has no server: FluxionEngine.place runs one placement per process,
 * H/python/fluxion/engine.py:25-50). Jobs:
 *   FX_JOB_PLACE  the reference's main.rs flow (H/src/main.rs:74-111) on a
 *                 netlist: fx_partition -> fx_hapr_place_leaves -> fx_refine;
 *                 the placed design can stay resident for later ECO jobs;
 *   FX_JOB_ECO    on a resident design: move the given gates (clamped to the
 *                 die; each gate listed at most once, else the job fails with
 *                 FX_EINVAL), then `iterations` plain iterations (fx_force_iterate).
 * Up to `slots` jobs run at once, each on its own worker thread and context
 * (own streams), so their kernels overlap on the device. A queued job is
 * admitted when a slot is free and its estimated device footprint fits in
 * what the budget has left (resident designs count at their actual size);
 * jobs that fit may pass a larger one waiting at the head of the queue, but
 * jobs on one design run in submission order. A job whose estimate exceeds
 * the whole budget, or a full queue, is refused at submit with FX_EADMIT.
 * Every job computes exactly what it would compute alone (own buffers and
 * streams, fixed reduction orders, no atomics shared between jobs). */
typedef struct fx_server fx_server;
#define FX_JOB_PLACE 0
#define FX_JOB_ECO 1
typedef struct fx_serve_cfg {
  int32_t device;
  int32_t slots;            /* jobs on the GPU at once (default 8)                */
  int32_t queue_capacity;   /* queued jobs before FX_EADMIT (default 65536)       */
  int32_t reserved0;
  int64_t hbm_budget_bytes; /* admission budget; 0 = 80 % of free memory at start */
} fx_serve_cfg;
typedef struct fx_job_desc {
  int32_t kind;             /* FX_JOB_*                                            */
  int32_t keep_resident;    /* PLACE: keep the placed design for ECO jobs          */
  int64_t design_id;        /* ECO: job id of the PLACE job that made the design   */
  int32_t n_gates, n_nets;  /* PLACE: the netlist, copied at submit                */
  const int32_t *net_ptr, *net_gate;
  const float *gate_w, *gate_h;
  float chip_w, chip_h;
  int32_t n_moves;          /* ECO: gate moves, copied at submit                   */
  int32_t iterations;       /* ECO: plain iterations after the moves               */
  const int32_t *move_gate;
  const float *move_dx, *move_dy;
  const fx_part_cfg *part;  /* stage configurations; NULL = defaults (PLACE: the   */
  const fx_leaf_cfg *leaf;  /* leaf default with FX_LEAF_FAST; ECO: the iteration  */
  const fx_refine_cfg *refine; /* default with a G x G density grid, G the         */
  const fx_iter_cfg *iter;  /* multiple of 128 nearest sqrt(n) in [128, 1024],     */
                            /* FX_DCT_SIMT below G = 1024, and a 256 x 256         */
                            /* congestion grid)                                    */
} fx_job_desc;
typedef struct fx_job_result {
  int64_t job_id, design_id;
  int32_t kind, status;     /* status: FX_OK or the failing FX_* code              */
  int32_t n_gates, n_leaves;
  int32_t iterations;       /* refine (PLACE) or plain (ECO) iterations run        */
  float max_overflow;
  double hpwl;              /* FP64 HPWL of the final positions                    */
  double total_overflow;
  double submit_s, start_s, end_s; /* server clock, seconds since creation         */
  int64_t est_bytes;        /* admission estimate                                  */
  char error[160];
} fx_job_result;
int fx_serve_cfg_default(fx_serve_cfg *cfg);
/* Host-only admission estimate of a job (ECO: uses n_gates of the design). */
int fx_serve_estimate(const fx_job_desc *job, int64_t *out_bytes);
int fx_serve_create(const fx_serve_cfg *cfg, fx_server **out);
/* Waits for the running jobs; queued jobs are dropped; frees resident designs. */
int fx_serve_destroy(fx_server *server);
int fx_serve_submit(fx_server *server, const fx_job_desc *job, int64_t *out_job_id);
/* Next finished job in completion order: 1 when *out was filled, 0 when none
 * finished within wait_ms (wait_ms < 0 waits until one does or nothing is
 * queued or running). */
int fx_serve_poll(fx_server *server, int32_t wait_ms, fx_job_result *out);
/* Positions of a resident design (waits while a job runs on it). */
int fx_serve_positions(fx_server *server, int64_t design_id, float *out_x, float *out_y);
int fx_serve_release(fx_server *server, int64_t design_id);
int fx_serve_stats(fx_server *server, int64_t *out_reserved_bytes, int32_t *out_queued,
                   int32_t *out_running, int32_t *out_resident, int64_t *out_launches);

/* ---- host-only helpers (no GPU needed) ---------------------------------- */
/* Builds the deduplicated clique-expansion adjacency of
 * Circuit::build_adjacency (H/src/data/circuit.rs:154-171) in the
 * reference's insertion order: out_adj_ptr[N+1], out_adj_idx[A]. Returns A
 * (the full count even when it exceeds cap; at most cap entries are
 * written; out_adj_idx may be NULL to query A) or a negative FX_E* code. */
int64_t fx_adjacency_build(int32_t n_gates, int32_t n_nets,
                           const int32_t *net_ptr, const int32_t *net_gate,
                           int32_t *out_adj_ptr, int32_t *out_adj_idx,
                           int64_t cap);

/* ---- synthetic netlists (host-only; no GPU needed) ---------------------- */
typedef struct fx_netlist fx_netlist;
/* Plain generator: n gates in leaf_size-gate leaves of a binary cluster
 * tree, widths U{1..4} x 1, n_nets nets whose degree is 2 (p=0.6), 3
 * (p=0.2) or power-law alpha=2.5 on [2,64]; pins from the driver's leaf
 * (0.7), its sibling leaf (0.2) or anywhere (0.1); positions uniform on the
 * die. Deterministic in seed (SplitMix64). */
int fx_synth_plain(uint64_t seed, int32_t n_gates, int32_t n_nets,
                   float die_w, float die_h, int32_t leaf_size,
                   fx_netlist **out);
/* Batched-leaf generator: n_clusters clusters of log-uniform size in
 * [min_size, max_size]; per cluster round(nets_per_gate * n) intra-cluster
 * nets of degree 2 + Geometric(0.5) capped at 8. Every cluster gets the unit
 * box region. */
int fx_synth_leaves(uint64_t seed, int32_t n_clusters, int32_t min_size,
                    int32_t max_size, float nets_per_gate, fx_netlist **out);
int fx_netlist_sizes(const fx_netlist *nl, int64_t *out_n, int64_t *out_m,
                     int64_t *out_p, int64_t *out_leaves);
/* Copies the arrays out; any pointer may be NULL. Leaves are contiguous
 * gate ranges: out_leaf_ptr[L+1]; out_region[4L] = (cx, cy, w, h). */
int fx_netlist_copy(const fx_netlist *nl, int32_t *out_net_ptr,
                    int32_t *out_net_gate, float *out_w, float *out_h,
                    float *out_x, float *out_y, float *out_die,
                    int32_t *out_leaf_ptr, float *out_region);
int fx_netlist_free(fx_netlist *nl);

/* ---- (f.3) netlist ingestion and DEF output (host-only) ----------------- */
/* Mirrors parser::blif::parse (H/src/parser/blif.rs:12-116): one gate per
 * .names / .latch / .gate line, named g0, g1, ... (width 2, height 10; die
 * 1000 x 1000); a net joins the driver of a signal (the last token of
 * .names, the output of .latch, the O= / Y= pin of .gate) and its readers,
 * in reading order; signals read by several gates but driven by none
 * (primary inputs) form nets of their readers; one-gate nets are dropped.
 * The reference collects nets by iterating HashMaps, whose order is seeded
 * randomly per process; here nets come in first-appearance order of their
 * signal names (driven signals first, then undriven ones), which fixes the
 * netlist for a file. design_name (may be NULL) receives the file stem
 * (Circuit::name) truncated to name_cap - 1 bytes. */
int fx_blif_read(const char *path, fx_netlist **out, char *design_name, int32_t name_cap);
/* Mirrors parser::def::write_def (H/src/parser/def.rs:11-43): DIEAREA and
 * PLACED coordinates are (v * 1000.0f32) as i64 (truncation, saturating,
 * NaN -> 0). names: n NUL-terminated gate names laid end to end, or NULL for
 * g0, g1, ... */
int fx_def_write(const char *path, const char *design_name, int32_t n, const float *x,
                 const float *y, float chip_w, float chip_h, const char *names);

#ifdef __cplusplus
}
#endif
#endif /* FLUXION_B200_H_ */
