/*
 * chiaro_depth.h — C ABI of the B200 multi-view depth stage.
 *
 * This library is a drop-in for chiaro-fusion's calibrated multi-view depth
 * stage, `refine_multiview_depth` (crates/chiaro-fusion/src/depth.rs:312-580).
 * Every entry point takes plain pointers and sizes; no C++ or torch types cross
 * the boundary. A Rust `-sys` crate, a ctypes module or a C caller binds these
 * declarations directly.
 *
 * Units and conventions (identical to the reference):
 *   - depths are calibration distance units (millimetres on the L16);
 *   - pixel coordinates are calibration-raster pixels, x right, y down;
 *   - luminance planes are the half-resolution f32 log-luminance planes of
 *     `Mosaic::luminance_half` (crates/chiaro-fusion/src/image.rs:401-428);
 *     plane pixel (i, j) is centred at raster (2i + 0.5, 2j + 0.5);
 *   - warps map reference-raster pixels to target-raster pixels on a regular
 *     grid, NaN marking undefined nodes (crates/chiaro-fusion/src/align.rs:34-45).
 *
 * Status codes: every function returns one of CHIARO_OK .. CHIARO_ERR_*.
 * CHIARO_INVALID is the C form of the reference's `None` return.
 */
#ifndef CHIARO_DEPTH_H
#define CHIARO_DEPTH_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CHIARO_DEPTH_ABI_VERSION 1

enum chiaro_status {
    CHIARO_OK = 0,
    CHIARO_INVALID = 1,       /* reference returns None (depth.rs:318-324)      */
    CHIARO_ERR_CUDA = 2,      /* a CUDA runtime call failed                      */
    CHIARO_ERR_TIMEOUT = 3,   /* a bounded device wait gave up                   */
    CHIARO_ERR_CAPACITY = 4,  /* a caller buffer is smaller than the result     */
    CHIARO_ERR_ARGUMENT = 5   /* NULL pointer or inconsistent sizes             */
};

/* DepthOptions (depth.rs:39-91). usize fields are 64-bit like Rust's usize. */
typedef struct chiaro_depth_options {
    int32_t enabled;
    int32_t _pad0;
    uint64_t grid_step;
    double near_depth;
    double far_depth;
    uint64_t planes;
    uint64_t patch_radius;
    uint64_t minimum_support;
    uint64_t best_view_count;
    float minimum_score;
    float minimum_margin;
    float minimum_improvement;
    int32_t _pad1;
    uint64_t minimum_neighbour_support;
    uint64_t completion_iterations;
} chiaro_depth_options;

/* Resolved camera (geometry.rs:31-62). Matrices are row-major m[row*3+col].
 * flip: 0 = no mirror flip, 1 = flip_img_around_x == true, 2 == false
 * (geometry.rs:129-136). pose_kind: 0 = Canonical, 1 = Mirror
 * (geometry.rs:50-62). Missing distortion coefficients are zero
 * (geometry.rs:310-312). */
typedef struct chiaro_camera {
    uint64_t width;
    uint64_t height;
    double k[9];
    double k_inverse[9];
    int32_t has_distortion;
    int32_t flip;
    double distortion_center[2];
    double distortion_normalization[2];
    double distortion_coeffs[5];
    int32_t pose_kind;
    int32_t _pad0;
    double rotation_wc[9];
    double rotation_cw[9];
    double translation_wc[3];
    double center[3];
    double real_cw[9];
    double reflect[9];
    double virtual_center[3];
    double orientation_correction[9];
} chiaro_camera;

/* One module's input (AlignInput, align.rs:246-257) plus its global alignment
 * (ModuleAlignment.warp / report.accepted, align.rs:148-157). */
typedef struct chiaro_warp {
    uint64_t step;
    uint64_t columns;
    uint64_t rows;
    float *points;       /* 2 * columns * rows, (x, y) interleaved; NaN = undefined */
    float *confidence;   /* columns * rows (may be NULL on input)                    */
    uint64_t capacity;   /* node capacity of points/confidence when used as output  */
} chiaro_warp;

typedef struct chiaro_view {
    const float *luminance;   /* luma_width * luma_height, row-major */
    uint64_t luma_width;
    uint64_t luma_height;
    uint64_t width;           /* raster width  (AlignInput.width)  */
    uint64_t height;          /* raster height (AlignInput.height) */
    int32_t has_camera;       /* AlignInput.camera.is_some()        */
    int32_t accepted;         /* ModuleAlignment.report.accepted    */
    chiaro_camera camera;
    chiaro_warp warp;         /* ModuleAlignment.warp (input)       */
} chiaro_view;

/* DepthProvenance (depth.rs:115-121). */
enum chiaro_provenance {
    CHIARO_UNSUPPORTED = 0,
    CHIARO_GLOBAL = 1,
    CHIARO_MEASURED = 2,
    CHIARO_REGULARIZED = 3
};

/* DenseDepthMap (depth.rs:133-141); caller-owned arrays of `capacity` nodes.
 * depth is NaN where the reference holds None. */
typedef struct chiaro_depth_map {
    uint64_t columns;
    uint64_t rows;
    uint64_t step;
    double near_depth;
    double far_depth;
    uint64_t capacity;
    double *depth;
    float *confidence;
    uint8_t *provenance;
} chiaro_depth_map;

/* DepthAlignmentReport (depth.rs:93-113); `present` mirrors report.depth.is_some(). */
typedef struct chiaro_depth_report {
    int32_t present;
    int32_t has_median_depth;
    uint64_t tested_nodes;
    uint64_t measured_nodes;
    uint64_t regularized_nodes;
    uint64_t fallback_nodes;
    uint64_t refined_nodes;
    uint64_t occluded_nodes;
    uint64_t boundary_nodes;
    float reconstructed_fraction;
    float refined_fraction;
    float occluded_fraction;
    int32_t has_median_score_improvement;
    double median_depth;
    float median_score_improvement;
    int32_t _pad0;
} chiaro_depth_report;

/* Optional host buffers receiving intermediate stage results (any may be NULL).
 * Sizes: coarse N = coarse_columns*coarse_rows, D = planes + 1, fine M =
 * columns*rows of the output grid. Per-target arrays are [n_views][M]. */
typedef struct chiaro_depth_debug {
    float *coarse_scores;          /* N*D  CostVolume.scores     (depth.rs:1233) */
    float *coarse_costs;           /* N*D  CostVolume.costs      (depth.rs:1236) */
    float *coarse_guidance;        /* N                                         */
    uint8_t *coarse_tested;        /* N                                         */
    float *regularised;            /* N*D  semi_global_costs     (depth.rs:1279) */
    uint8_t *coarse_has;           /* N    select_depths field   (depth.rs:1385) */
    double *coarse_depth;          /* N                                         */
    float *coarse_confidence;      /* N                                         */
    float *coarse_improvement;     /* N                                         */
    uint8_t *coarse_regularized;   /* N                                         */
    uint8_t *coarse_fillable;      /* N                                         */
    uint8_t *direct_has;           /* M    measure_direct_depths (depth.rs:715)  */
    double *direct_depth;          /* M                                         */
    float *direct_confidence;      /* M                                         */
    float *direct_improvement;     /* M                                         */
    uint8_t *direct_regularized;   /* M                                         */
    float *direct_guidance;        /* M                                         */
    uint8_t *direct_tested;        /* M                                         */
    uint8_t *isolated_has;         /* M    after reject_isolated (depth.rs:881)  */
    uint8_t *component_has;        /* M    after components      (depth.rs:933)  */
    double *fitted_depth;          /* M    after plane fit       (depth.rs:995)  */
    uint8_t *decision_kind;        /* n_views*M NodeWarp kind after boundaries   */
} chiaro_depth_debug;

/* NodeWarp kinds (depth.rs:256-271). */
enum chiaro_node_warp {
    CHIARO_NW_UNDEFINED = 0,
    CHIARO_NW_GLOBAL = 1,
    CHIARO_NW_REFINED = 2,
    CHIARO_NW_OCCLUDED = 3,
    CHIARO_NW_BOUNDARY = 4
};

typedef struct chiaro_depth_ctx chiaro_depth_ctx;

/* ---- pinned host memory ---------------------------------------------------- */

/* No counterpart in the reference: page-locked host buffers for the inputs and
 * outputs of the host-buffer entry points, which then move at the full
 * host-link rate (about 50 GB/s here, against about 19 GB/s for pageable
 * memory) and overlap the stage's kernels. Allocation is slow (it pins pages),
 * so callers keep and reuse these buffers. */
int chiaro_host_alloc(uint64_t bytes, void **out);
void chiaro_host_free(void *ptr);

/* ---- context ------------------------------------------------------------ */

/* Create a context bound to CUDA device `device` with its own stream. One
 * context per host thread; calls on one context are synchronous. */
int chiaro_depth_ctx_create(int device, chiaro_depth_ctx **out);
void chiaro_depth_ctx_destroy(chiaro_depth_ctx *ctx);
const char *chiaro_depth_last_error(const chiaro_depth_ctx *ctx);
int chiaro_depth_abi_version(void);

/* DepthOptions::default() (depth.rs:69-91). */
void chiaro_depth_options_default(chiaro_depth_options *out);
/* valid_options (depth.rs:1879-1891): 1 when valid. */
int chiaro_depth_options_valid(const chiaro_depth_options *options);

/* Output grid of the stage for a reference raster: the direct-pass grid
 * (depth.rs:326-328, depth.rs:726-728). Also reports the coarse grid. */
int chiaro_depth_output_shape(uint64_t width, uint64_t height,
                              const chiaro_depth_options *options,
                              uint64_t *columns, uint64_t *rows, uint64_t *step,
                              uint64_t *coarse_columns, uint64_t *coarse_rows,
                              uint64_t *coarse_step);

/* ---- the stage ---------------------------------------------------------- */

/* refine_multiview_depth (depth.rs:312-580).
 * views[n_views]: every module's input and global warp (host memory).
 * refined[n_views]: caller-owned output warps. For every target that the
 * reference would rewrite (accepted, has a camera, not the reference;
 * depth.rs:420-426) the library writes step/columns/rows, points and
 * confidence, and sets reports[t].present = 1; other entries are untouched
 * except reports[t].present = 0.
 * out_map: the DenseDepthMap. debug may be NULL.
 * Returns CHIARO_INVALID where the reference returns None. */
int chiaro_refine_multiview_depth(chiaro_depth_ctx *ctx,
                                  const chiaro_view *views, size_t n_views,
                                  size_t reference_index,
                                  const chiaro_depth_options *options,
                                  chiaro_warp *refined,
                                  chiaro_depth_report *reports,
                                  chiaro_depth_map *out_map,
                                  const chiaro_depth_debug *debug);

/* Same stage with every array pointer in `views` (luminance, warp points and
 * confidence), in `refined` and in `out_map` referring to device memory of the
 * context's device; nothing is copied across PCIe. Used when inputs are
 * already resident in HBM. Reports are host structs. */
int chiaro_refine_multiview_depth_device(chiaro_depth_ctx *ctx,
                                         const chiaro_view *views, size_t n_views,
                                         size_t reference_index,
                                         const chiaro_depth_options *options,
                                         chiaro_warp *refined,
                                         chiaro_depth_report *reports,
                                         chiaro_depth_map *out_map);

/* Whole-stage CUDA graph of chiaro_refine_multiview_depth_device (no counterpart in
 * the reference; off by default). When enabled, a device-buffer call whose views
 * (pointers, sizes, flags, cameras), reference, options and output pointers equal the
 * previous call's is captured into a graph on its second occurrence and replayed from
 * the third on: the stage's ~35 launches become one, and a replay reads the current
 * contents of the same buffers. Any other call, or any buffer the context reallocates
 * (another entry point on a larger size, for instance), voids the graph and the next
 * calls run, capture and replay afresh. Calls with debug arrays or host buffers never
 * use it. The first call of a key should not come during another stream capture.
 * Switching it off drops the graph and switching it on starts afresh; setting the
 * current value again changes nothing. */
int chiaro_depth_set_stage_graph(chiaro_depth_ctx *ctx, int32_t enabled);
/* What the last device-buffer stage call did: 0 launched its kernels, 1 captured and
 * launched the graph, 2 replayed it. */
int chiaro_depth_stage_graph_state(const chiaro_depth_ctx *ctx);

/* No counterpart in the reference (whose CPU union-find is a depth-first search
 * with no retries): the bound on the compare-and-swap attempts of one union-find
 * join in the connected-components filter (depth.rs:933-989), on the GPU. A
 * negative value, the default, bounds a join by the grid's node count plus one,
 * which cannot run out (each failed attempt means another join succeeded). A
 * smaller bound may run out (0 allows no attempt, so every join gives up); the
 * call then returns CHIARO_ERR_TIMEOUT instead of a result with a join left out,
 * and the context stays usable. */
int chiaro_depth_set_union_retry_limit(chiaro_depth_ctx *ctx, int32_t retries);

/* No counterpart in the reference: a cap on the device memory the context's
 * buffers may hold (0, the default: no cap), for hosts that give this library a
 * fixed budget. A call that would grow its buffers past the cap returns
 * CHIARO_ERR_CUDA (out of memory, with the message in chiaro_depth_last_error)
 * before allocating; buffers already held are kept, and the context stays usable.
 * chiaro_depth_memory_held reports the bytes held now. */
int chiaro_depth_set_memory_limit(chiaro_depth_ctx *ctx, uint64_t bytes);
uint64_t chiaro_depth_memory_held(const chiaro_depth_ctx *ctx);

/* No counterpart in the reference: launch-shape autotuning. With mode 1 (the default),
 * the first cost-volume launch of each (targets, labels scored, patch radius) bucket with
 * at least 4096 nodes, outside any stream capture, times every candidate CTA size (64, 96,
 * 128, 160 and 192 threads per node) and keeps the fastest for the context's later launches.
 * Every size gives the same bits. Mode 0 runs the default of 128 threads; mode 64, 96, 128,
 * 160 or 192 runs that size everywhere; both forget the choices made. Other modes return
 * CHIARO_ERR_ARGUMENT. chiaro_depth_tuning writes up to `capacity` choices, each a bucket
 * key ((targets << 24) | (labels scored << 8) | radius) and its threads, and returns how
 * many the context holds. */
int chiaro_depth_set_autotune(chiaro_depth_ctx *ctx, int32_t mode);
int chiaro_depth_tuning(const chiaro_depth_ctx *ctx, uint64_t *keys, int32_t *threads, int capacity);

/* Device time in milliseconds of each stage of the last call on this context:
 * [0] cost volume, [1] SGM, [2] select, [3] direct pass, [4] filters,
 * [5] per-target decisions, [6] whole stage. Returns the count written. */
int chiaro_depth_last_timings(const chiaro_depth_ctx *ctx, float *ms, int capacity);

/* Number of this library's kernel launches in the last stage call. */
int chiaro_depth_last_launches(const chiaro_depth_ctx *ctx);

/* The context's CUDA stream (a cudaStream_t), for callers that order their
 * own work or timing events with the library's. */
void *chiaro_depth_ctx_stream(const chiaro_depth_ctx *ctx);

/* ---- individual operators (host buffers) -------------------------------- */

/* semi_global_costs (depth.rs:1279-1311): eight-path SGM over a label-minor
 * [columns*rows][labels] f32 cost volume with per-node guidance. Output order
 * of summation is the reference's, so results are bit-identical. */
int chiaro_sgm_aggregate(chiaro_depth_ctx *ctx, const float *costs,
                         const float *guidance, uint64_t columns, uint64_t rows,
                         uint64_t labels, float *out);

/* Same operator on device pointers (stream of the context). */
int chiaro_sgm_aggregate_device(chiaro_depth_ctx *ctx, const float *costs,
                                const float *guidance, uint64_t columns,
                                uint64_t rows, uint64_t labels, float *out);

/* select_depths (depth.rs:1385-1467) with sublabel_depth (depth.rs:1469-1488).
 * labels[n_labels]: label depths, NaN for label 0 (the global warp). */
int chiaro_select_depths(chiaro_depth_ctx *ctx, const double *labels,
                         uint64_t n_labels, const float *scores,
                         const float *regularised, const uint8_t *tested,
                         uint64_t n_nodes, const chiaro_depth_options *options,
                         uint8_t *has, double *depth, float *confidence,
                         float *improvement, uint8_t *regularized,
                         uint8_t *fillable);

/* reject_isolated_direct_depths (depth.rs:881-924), in place on has[]. */
int chiaro_reject_isolated(chiaro_depth_ctx *ctx, uint8_t *has, const double *depth,
                           const float *confidence, const float *guidance,
                           uint64_t columns, uint64_t rows, double inverse_tolerance);

/* reject_small_direct_components (depth.rs:933-989), in place on has[]. */
int chiaro_reject_small_components(chiaro_depth_ctx *ctx, uint8_t *has,
                                   const double *depth, const float *guidance,
                                   uint64_t columns, uint64_t rows,
                                   double inverse_tolerance, uint64_t minimum_nodes);

/* fit_local_depth_planes (depth.rs:995-1060), in place on depth[]. */
int chiaro_fit_local_planes(chiaro_depth_ctx *ctx, const uint8_t *has, double *depth,
                            const float *confidence, const float *guidance,
                            uint64_t columns, uint64_t rows, double inverse_tolerance);

/* enforce_warp_consensus (depth.rs:582-618) then, when `boundaries` is set,
 * suppress_warp_boundaries (depth.rs:620-672), in place. kind[] uses
 * chiaro_node_warp; global/point are 2 floats per node. */
int chiaro_warp_decisions_filter(chiaro_depth_ctx *ctx, uint8_t *kind, float *global,
                                 float *point, const uint8_t *measured,
                                 const float *guidance, uint64_t columns,
                                 uint64_t rows, int consensus, int boundaries);

/* ---- quantised SGM ---------------------------------------------------------- */

/* No counterpart in the reference: the quantised performance mode of
 * semi_global_costs (depth.rs:1279-1383). Costs (f32 [N][D], the stage's range
 * [0, 2.25]; NaN counts as 2.25) become u16 fixed point at 2048 per unit, the
 * edge penalties are the reference's f32 p1, p2 quantised the same way, and the
 * 8-path recurrence and sum run in exact 16-bit integers on label pairs (a path
 * cost is at most 5530, the sum at most 44240). Outputs, each optional: the
 * u16 aggregate [N][D] and the winner over labels 1..D-1 per node (first
 * minimum). Half the bytes of the f32 path per cell; the winner agrees with the
 * f32 path's within one plane. labels <= 256. The _device form takes device
 * pointers. */
int chiaro_sgm_aggregate_u16(chiaro_depth_ctx *ctx, const float *costs, const float *guidance,
                             uint64_t columns, uint64_t rows, uint64_t labels, uint16_t *aggregate,
                             uint16_t *best);
int chiaro_sgm_aggregate_u16_device(chiaro_depth_ctx *ctx, const float *costs,
                                    const float *guidance, uint64_t columns, uint64_t rows,
                                    uint64_t labels, uint16_t *aggregate, uint16_t *best);

/* ---- batched SGM -------------------------------------------------------------- */

/* One SGM instance of a batch: every array in device memory of the context's
 * device. out receives semi_global_costs of (costs, guidance), bit-identical to
 * chiaro_sgm_aggregate_device on the same instance. */
typedef struct chiaro_sgm_instance {
    const float *costs;     /* [columns * rows][labels] */
    const float *guidance;  /* [columns * rows] */
    float *out;             /* [columns * rows][labels] */
    uint64_t columns, rows, labels;
} chiaro_sgm_instance;

enum {
    CHIARO_BATCH_GRAPH = 1,    /* capture the batch in a CUDA graph; replay it while the batch is unchanged */
    CHIARO_BATCH_AUTOTUNE = 2  /* time the launch shapes once per size bucket and keep the fastest */
};

/* No counterpart in the reference (which runs each grouping's SGM on its own):
 * all reference/source groupings of a capture, or of many captures, as one
 * batch of SGM instances of uneven sizes and label counts (labels <= 256). A
 * persistent kernel walks every path of every direction of every instance from
 * a work list (longest paths first), then one kernel forms each instance's
 * ordered sum. Each instance needs 8 x its volume of path scratch; instances
 * run in waves whose scratch fits in scratch_bytes (0: 16 GiB), and an
 * instance larger than that returns CHIARO_ERR_CAPACITY. flags: see above. A
 * captured graph refers to the context's scratch and the instances' pointers:
 * it is replayed only while both are unchanged, and re-captured otherwise. */
int chiaro_sgm_aggregate_batch_device(chiaro_depth_ctx *ctx, const chiaro_sgm_instance *instances,
                                      uint64_t n_instances, uint64_t scratch_bytes, int flags);

/* How the last batch ran: warps per CTA of the persistent kernel, number of
 * waves, and whether a captured graph was replayed (1) rather than launched or
 * captured (0). Any pointer may be NULL. */
int chiaro_sgm_batch_report(const chiaro_depth_ctx *ctx, int *warps_per_cta, int *waves, int *replayed);

/* ---- banded SGM ------------------------------------------------------------------ */

/* No counterpart in the reference: the band-limited SGM of the learned-band
 * design. The grid is cut into tiles of tile x tile nodes; tile t's nodes
 * aggregate only the labels [tile_offsets[t], tile_offsets[t] + band)
 * (1 <= offset <= labels - band, band <= 32; tiles row-major, ceil(columns /
 * tile) per row) with the recurrence of semi_global_costs (depth.rs:1363-1381),
 * the band shifting between tiles along each path. winner[node] is the label of
 * the first minimum over the band. A tile whose winner sits on a band edge at
 * any node, with labels beyond that edge (not at label 1 or labels - 1), falls
 * back (fallback[t] = 1). Fallback tiles are grouped into rectangles (in raster
 * order: the widest run of fallback tiles, then as many rows of that run as are
 * all fallback tiles); the full-range SGM over each rectangle grown by `margin`
 * nodes decides its nodes' winners (labels 1..labels-1). The _device form takes
 * device pointers. */
int chiaro_sgm_banded(chiaro_depth_ctx *ctx, const float *costs, const float *guidance, uint64_t columns,
                      uint64_t rows, uint64_t labels, const int32_t *tile_offsets, uint64_t tile,
                      uint64_t band, uint64_t margin, int32_t *winner, uint8_t *fallback);
int chiaro_sgm_banded_device(chiaro_depth_ctx *ctx, const float *costs, const float *guidance,
                             uint64_t columns, uint64_t rows, uint64_t labels,
                             const int32_t *tile_offsets, uint64_t tile, uint64_t band,
                             uint64_t margin, int32_t *winner, uint8_t *fallback);

/* The number of fallback windows (rectangles) of the last banded SGM. */
int chiaro_sgm_banded_report(const chiaro_depth_ctx *ctx, int *windows);

/* ---- learned band proposal ------------------------------------------------------- */

/* No counterpart in the reference (which uses no learned model): the band
 * proposal network of the banded SGM. Six 3x3 convolutions of 32 channels on
 * the coarse grid (one pixel per node), bf16 tensor-core kernels with fp32
 * accumulation. Inputs per node: the reference luminance (guidance), the costs
 * of 16 sampled labels spread over the finite ones (labels >= 19), the first
 * sampled label at their minimum and that minimum cost. Parameters are
 * chiaro_bandnet_parameter_count() fp32 values: per layer the weights
 * [tap][co][ci] then the 32 biases. All arrays below are device memory; costs
 * [images][nodes][cost_stride]: full rows (cost_stride = labels) or the
 * pre-pass's rows (cost_stride = 17, chiaro_band_prepass_device); guidance
 * [images][nodes], winners (the target labels, e.g. the full-range SGM's) and
 * mask (1 for nodes to learn from) [images][nodes]. */
uint64_t chiaro_bandnet_parameter_count(void);

/* Band offsets per tile (as chiaro_sgm_banded takes them): the band centred on
 * the mean predicted label of the tile's nodes, clamped to [1, labels - band];
 * centres (optional, [nodes]) receives each node's normalised prediction. */
int chiaro_bandnet_propose_device(chiaro_depth_ctx *ctx, const float *params, const float *costs,
                                  const float *guidance, uint64_t columns, uint64_t rows,
                                  uint64_t labels, uint64_t cost_stride, uint64_t tile, uint64_t band,
                                  int32_t *tile_offsets, float *centres);

/* `steps` full-batch Adam steps (numbered from first_step + 1) of the Huber loss
 * between the normalised prediction and (winner - 1) / (labels - 2) on the
 * masked nodes; losses (host, optional) receives each step's loss. adam_m and
 * adam_v hold the optimiser state (zero before the first step). */
int chiaro_bandnet_train_device(chiaro_depth_ctx *ctx, float *params, float *adam_m, float *adam_v,
                                uint64_t first_step, uint64_t steps, const float *costs,
                                const float *guidance, const int32_t *winners, const uint8_t *mask,
                                uint64_t images, uint64_t columns, uint64_t rows, uint64_t labels,
                                uint64_t cost_stride, float learning_rate, float *losses);

/* One forward and backward pass: the loss (host) and its gradient (device,
 * the parameters' layout). */
int chiaro_bandnet_gradient_device(chiaro_depth_ctx *ctx, const float *params, const float *costs,
                                   const float *guidance, const int32_t *winners, const uint8_t *mask,
                                   uint64_t images, uint64_t columns, uint64_t rows, uint64_t labels,
                                   uint64_t cost_stride, float *grads, float *loss);

/* ---- coarse depth search ------------------------------------------------------- */

/* The learned-band form of the coarse search (no counterpart in the reference, which
 * searches every label). params: the band network's parameters in device memory
 * (chiaro_bandnet_parameter_count() floats), or NULL for the band without learning
 * (per tile, the median of its nodes' lowest sampled labels). A tile is tile x tile
 * coarse nodes (1..8); band finite labels per tile (1..32, at most planes); margin nodes
 * of full-range context around each fallback rectangle; a tile also falls back when
 * more than contradicted_fraction of its tested nodes fail the cross-view check (1 or
 * more: never). */
typedef struct chiaro_band_options {
    const float *params;
    uint64_t tile;
    uint64_t band;
    uint64_t margin;
    float contradicted_fraction;
    int32_t _pad0;
} chiaro_band_options;

/* What a coarse search did. Tiles whose winner sat on a band edge (edge_tiles), that
 * failed the cross-view check (consistency_tiles), either (fallback_tiles); the fallback
 * windows and the nodes whose full-range costs they computed; device milliseconds of
 * [0] the shared set-up (geometry, tap lattice, quad planes), [1] the pre-pass, [2] the
 * band proposal, [3] the cost volume (banded or full), [4] the SGM and winners (with the
 * fallback flags), [5] the fallback (host round trip included), [6] the whole search. */
typedef struct chiaro_band_report {
    uint64_t tiles;
    uint64_t edge_tiles;
    uint64_t consistency_tiles;
    uint64_t fallback_tiles;
    uint64_t windows;
    uint64_t window_nodes;
    float ms[7];
    int32_t _pad0;
} chiaro_band_report;

/* The coarse depth search of refine_multiview_depth on the reference's coarse grid
 * (depth.rs:326-328): build_cost_volume (depth.rs:1187-1277), semi_global_costs
 * (depth.rs:1279-1383) and each node's winning label over the finite labels, the first
 * minimum as select_depths takes it (depth.rs:1406-1413). views as for
 * chiaro_refine_multiview_depth_device (device memory). winner [N] (device) receives
 * each coarse node's label; tested [N] (device, optional) the cost volume's tested flags.
 * band == NULL: the plain search, bit-identical to the stage's. Otherwise the learned-band
 * search (no counterpart in the reference): a pre-pass scores label 0 and 16 sampled
 * labels at every node, the band proposal picks each tile's band, the cost volume scores
 * label 0 and the band, the banded SGM picks winners, and tiles whose winner sits on a
 * band edge or that fail the cross-view check (a node's aggregated score at its winner
 * more than 0.12 below its score under the global warp, the threshold of depth.rs:
 * 458-485) are searched again at full range in windows around them. tile_offsets and
 * tile_fallback ([tiles], device, optional) receive each tile's band start and fallback
 * flag; report (host, optional) what the search did. */
int chiaro_coarse_depth_device(chiaro_depth_ctx *ctx, const chiaro_view *views, size_t n_views,
                               size_t reference_index, const chiaro_depth_options *options,
                               const chiaro_band_options *band, int32_t *winner, uint8_t *tested,
                               int32_t *tile_offsets, uint8_t *tile_fallback, chiaro_band_report *report);

/* The learned-band search's pre-pass alone (no counterpart in the reference): per coarse
 * node, the costs of label 0 and of the 16 sampled labels ([N][17], device), the
 * guidance and the tested flag ([N], device, optional): the band network's inputs, for
 * training it. The sampled labels are 1 + (b (planes - 1) + 7) / 15, b = 0..15. */
int chiaro_band_prepass_device(chiaro_depth_ctx *ctx, const chiaro_view *views, size_t n_views,
                               size_t reference_index, const chiaro_depth_options *options, float *sampled_costs,
                               float *guidance, uint8_t *tested);

/* ---- input plane --------------------------------------------------------- */

/* VignettingMesh (calibration.rs:354-358): a columns x rows grid of flat-field
 * gains over the sensor raster, row-major. columns or rows below 2 (or a NULL
 * mesh) means flat field 1 (Mosaic::flat_field, image.rs:145-150). */
typedef struct chiaro_vignetting {
    uint64_t columns, rows;
    const float *gains;
} chiaro_vignetting;

/* Mosaic::luminance_half (image.rs:401-428): the width x height u16 Q6 mosaic
 * (row-major, calibration raster) becomes the (width / 2) x (height / 2) f32
 * plane ln(1 + 1000 * linear), linear = max((mean of the 2x2 cell - black_q6) /
 * max(white_q6 - black_q6, 1), 0) * flat_field(2i + 0.5, 2j + 0.5), ready to be
 * a chiaro_view's luminance. Everything before the log is the reference's f32
 * arithmetic bit for bit; the log is the correctly rounded one (f64 log rounded
 * to f32), within 1 ulp of the host logf the reference calls. The _device
 * form takes device pointers (samples, gains, out); the other
 * takes host buffers and copies. */
int chiaro_luminance_half(chiaro_depth_ctx *ctx, const uint16_t *samples, uint64_t width,
                          uint64_t height, float black_q6, float white_q6,
                          const chiaro_vignetting *mesh, float *out);
int chiaro_luminance_half_device(chiaro_depth_ctx *ctx, const uint16_t *samples, uint64_t width,
                                 uint64_t height, float black_q6, float white_q6,
                                 const chiaro_vignetting *mesh, float *out);

/* ---- consumers of the stage's outputs ------------------------------------------- */

/* Warp::map and Warp::confidence (crates/chiaro-fusion/src/align.rs:84-131), the
 * per-pixel warp lookups of synthesize (synth.rs:591-700), at n reference-raster
 * points xy (2n floats, (x, y) interleaved). Every array is device memory of the
 * context's device, warp->points and warp->confidence included (confidence may be
 * NULL: every confidence is then 0, as for the reference's length mismatch).
 * mapped (2n) receives the target point, NaN for None; confidence (n, may be NULL)
 * the bilinear confidence. Bit-identical to the reference. */
int chiaro_warp_sample_device(chiaro_depth_ctx *ctx, const chiaro_warp *warp, const float *xy, uint64_t n,
                              float *mapped, float *confidence);

/* DenseDepthMap::sample_nearest (depth.rs:152-159) at n reference-raster points xy
 * (device memory, as are map's arrays and the outputs): node (may be NULL) receives
 * the nearest node's index or -1 for None; depth / confidence / provenance (each may
 * be NULL) the node's fields (NaN / 0 / 0 for None). */
int chiaro_depth_sample_nearest_device(chiaro_depth_ctx *ctx, const chiaro_depth_map *map, const float *xy,
                                       uint64_t n, double *depth, float *confidence, uint8_t *provenance,
                                       int64_t *node);

/* ---- global alignment ------------------------------------------------------------- */

/* AlignInput (crates/chiaro-fusion/src/align.rs:246-257). */
typedef struct chiaro_align_input {
    const float *luminance;   /* half-resolution log luminance, luma_width * luma_height */
    uint64_t luma_width;
    uint64_t luma_height;
    uint64_t width;           /* raster */
    uint64_t height;
    int32_t has_camera;       /* camera.is_some() */
    chiaro_camera camera;
    double nominal_focal_px;  /* used without cameras */
} chiaro_align_input;

/* AlignOptions (align.rs:205-243) without the depth options. */
typedef struct chiaro_align_options {
    uint64_t grid_step;      /* 32 */
    uint64_t patch;          /* 32 */
    uint64_t coarse_radius;  /* 12 */
    float min_score;         /* 0.5 */
    float inlier_px;         /* 3.0 */
    float min_inlier_ratio;  /* 0.45 */
    int32_t refine;          /* 1 */
} chiaro_align_options;

/* AlignmentReport.initialised_from and .status (align.rs:290-300, 463-477). */
enum chiaro_align_initialisation {
    CHIARO_INIT_REFERENCE = 0,
    CHIARO_INIT_SEED = 1,
    CHIARO_INIT_CALIBRATION = 2,
    CHIARO_INIT_NOMINAL_FOCAL_GROUP = 3
};
enum chiaro_align_status {
    CHIARO_ALIGN_REFERENCE = 0,
    CHIARO_ALIGN_REJECTED = 1,      /* "rejected: NN% correspondence consensus" (inlier_ratio) */
    CHIARO_ALIGN_FACTORY_MODEL = 2,
    CHIARO_ALIGN_REFINED = 3,
    CHIARO_ALIGN_WEAK_REFINEMENT = 4,
    CHIARO_ALIGN_NO_SUPPORT = 5     /* "no correlation support; factory model kept" */
};

#define CHIARO_ALIGN_MAX_LEVELS 24

/* LevelReport (align.rs:202-207). */
typedef struct chiaro_align_level {
    uint64_t scale;
    uint64_t patches;
    uint64_t inliers;
    float median_residual_px;  /* NaN when the level had no fit */
} chiaro_align_level;

/* The alignment fields of AlignmentReport (align.rs:160-200); the camera name,
 * focus fields and the depth report belong to other stages. */
typedef struct chiaro_alignment_report {
    int32_t initialised_from;  /* enum chiaro_align_initialisation */
    int32_t status;            /* enum chiaro_align_status */
    int32_t accepted;
    float coverage;
    float correction_median_px[2];
    uint64_t inliers;
    uint64_t patches;
    float residual_median_px;
    float residual_p90_px;
    float inlier_ratio;
    uint64_t n_levels;         /* coarsest first, as the reference pushes them */
    chiaro_align_level levels[CHIARO_ALIGN_MAX_LEVELS];
} chiaro_alignment_report;

/* AlignOptions::default() (align.rs:231-244), without the depth options. */
void chiaro_align_options_default(chiaro_align_options *options);

/* Replaces align_module / align_module_seeded (align.rs:281-519), called per module
 * by the pipeline before the depth stage. target_is_reference stands for the
 * reference's name comparison (the reference aligns to itself with an identity
 * warp); seed (NULL for none) is the externally predicted warp. The target plane
 * is matched against the reference over both luminance pyramids: the rendering
 * through the current homography, the patch searches and the RANSAC inlier counts
 * run on the GPU, the homography fits and the report on the host. out_warp (host
 * memory, step options->grid_step, capacity >= columns * rows; step, columns and
 * rows are set on return) receives the warp, gain the photometric gain. Returns
 * CHIARO_INVALID where the reference returns Err (no correlation in the
 * no-calibration search), with its message in chiaro_depth_last_error. A level's
 * patch search keeps the window and its scores in shared memory: (patch^2 +
 * (2 radius + 1)^2) * 4 bytes must fit 200 KiB (a patch up to 226 at the fine
 * levels' radius 3; the default 32 with radius 12 takes 6.5 KiB), else
 * CHIARO_ERR_ARGUMENT. */
int chiaro_align_module(chiaro_depth_ctx *ctx, const chiaro_align_input *reference,
                        const chiaro_align_input *target, int32_t target_is_reference,
                        const chiaro_align_options *options, const chiaro_warp *seed,
                        chiaro_warp *out_warp, float *gain, chiaro_alignment_report *report);

/* ---- resolution-domain local warp refinement ------------------------------------ */

/* ResolutionAlignmentReport (crates/chiaro-fusion/src/resolution.rs:88-100). */
typedef struct chiaro_resolution_report {
    float verified_fraction;     /* control nodes with a coherent, verified match  */
    float supported_fraction;    /* verified or completed from coherent neighbours */
    float median_correction_px;  /* median verified correction, reference pixels   */
    float mean_confidence;       /* mean confidence of the verified nodes          */
} chiaro_resolution_report;

/* Replaces refine_resolution_warp (crates/chiaro-fusion/src/resolution.rs:232-439),
 * called per target module at pipeline.rs:1185 and chiaro-stack/src/fusion.rs:384.
 * reference and target are half-resolution luminance planes (Plane, row-major f32,
 * host memory); base is the target's warp from the reference raster (width x
 * height) into the target raster (host memory). The target is resampled to the
 * reference plane through base (a Gaussian footprint when base magnifies it more
 * than 1.15x), a 12 x 12 patch is matched around every node of a 32 px grid (radius
 * 2, or 5 when base magnifies more than 1.35x), and the matches are median-filtered
 * and completed over the grid. out (host memory) receives the refined warp: step 32,
 * columns = ceil(width / 32) + 1, rows = ceil(height / 32) + 1 (set on return, also
 * when out->capacity is too small, which returns CHIARO_ERR_CAPACITY); points and
 * confidence of columns * rows nodes (confidence may be NULL). Bit-identical to the
 * reference's result. */
int chiaro_refine_resolution_warp(chiaro_depth_ctx *ctx, const float *reference, uint64_t reference_width,
                                  uint64_t reference_height, const float *target, uint64_t target_width,
                                  uint64_t target_height, const chiaro_warp *base, uint64_t width,
                                  uint64_t height, chiaro_warp *out, chiaro_resolution_report *report);
/* The same with reference and target in device memory of the context's device (the
 * warps and the report stay host memory): a pipeline that keeps the modules' planes
 * in HBM refines every target without uploading them. */
int chiaro_refine_resolution_warp_device(chiaro_depth_ctx *ctx, const float *reference,
                                         uint64_t reference_width, uint64_t reference_height,
                                         const float *target, uint64_t target_width,
                                         uint64_t target_height, const chiaro_warp *base, uint64_t width,
                                         uint64_t height, chiaro_warp *out, chiaro_resolution_report *report);

/* ---- allocation-free operator --------------------------------------------- */

/* No counterpart in the reference: an allocation-free form of
 * chiaro_reject_small_components for callers that cannot allocate device
 * memory (a host with a fixed memory budget, a plugin whose framework owns the
 * allocator, code that wraps its own buffers in a CUDA graph). All pointers are
 * device memory of the current device; has_out may not alias has. The work is
 * queued on `stream` (a cudaStream_t, NULL for the default stream) and the
 * call returns without synchronising. Its union-find scratch lives in a static
 * device array of 2^20 nodes (8 MiB per GPU, held until exit): grids with more
 * nodes return CHIARO_ERR_CAPACITY. The first call on a device looks up that
 * array's address; make it before any stream capture. That address is kept
 * per device index for the life of the process, so do not use this call across
 * cudaDeviceReset. Calls share the array, so calls that overlap on the GPU race.
 * Nothing here calls cudaMalloc. */
int chiaro_reject_small_components_noalloc(void *stream, const uint8_t *has, const double *depth,
                                           const float *guidance, uint64_t columns, uint64_t rows,
                                           double inverse_tolerance, uint64_t minimum_nodes,
                                           uint8_t *has_out);

#ifdef __cplusplus
}
#endif

#endif /* CHIARO_DEPTH_H */
