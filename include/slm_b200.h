/* slm_b200.h -- C ABI of the B200 streamline tracer (libslm_b200.so).
 *
 * Drop-in boundary for the OpenCL kernels of atthecodeface/slm's `streamlines`
 * package.  The reference builds one OpenCL program per launch with every
 * scalar as a -D macro (python/streamlines/pocl.py:178-299) and passes only
 * __global buffers, in the insertion order of each wrapper's array_dict
 * (pocl.py:538-539).  Each entry point here takes:
 *   - `const slm_params*`: the macro values as a host struct (field = macro name
 *     in lower case; built by slm_b200/params.py exactly as the reference
 *     formats its macros);
 *   - the same buffers as the reference kernel, in the same order, as DEVICE
 *     pointers owned by the caller (nothing here allocates device memory);
 *   - a CUDA stream (`void*`, cudaStream_t; NULL = legacy default stream).
 * Calls are asynchronous and stream-ordered.  They return 0 on success or an
 * SLM_ERR_* code; slm_last_error() gives the message of the calling thread's
 * last failure.  No exception or device trap crosses this boundary.
 *
 * Accumulators that the reference keeps as wrapping uint32 (slt, slc) are
 * uint64 here; the low 32 bits equal the reference's values.
 */
#ifndef SLM_B200_H
#define SLM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SLM_OK 0
#define SLM_ERR_ARGS 1          /* bad pointer, size or parameter */
#define SLM_ERR_CUDA 2          /* a CUDA runtime call failed */
#define SLM_ERR_CAPACITY 3      /* a buffer or work queue is too small */
#define SLM_ERR_ITERATION_CAP 4 /* a bounded device loop hit its cap (see message) */
#define SLM_ERR_UNSUPPORTED 5   /* option not built into this library */

/* Kernel parameters: one field per -D macro of pocl.set_compile_options
 * (pocl.py:197-277); the last two carry the DO_MEASURE_HSL_FROM_RIDGES flag
 * and the KDF_IS_<shape> selector (0 tophat, 1 triangle, 2 epanechnikov,
 * 3 cosine, 4 gaussian). */
typedef struct slm_params {
    uint32_t n_seed_points, downup_sign;
    float integrator_step_factor, max_integration_step_error, adjusted_max_error,
          integration_halt_threshold, max_length, pixel_size;
    uint32_t pad_width;
    float pad_width_pp5;
    uint32_t nx_padded, ny_padded, nxy_padded;
    float nxf_mp5, nyf_mp5, grid_scale, combo_factor, dt_max;
    uint32_t max_n_steps, trajectory_resolution, seeds_chunk_offset,
             subpixel_seed_point_density;
    float subpixel_seed_halfspan, subpixel_seed_step, jitter_magnitude;
    uint32_t interchannel_max_n_steps, left_flank_addition;
    uint32_t is_channel, is_thinchannel, is_interchannel, is_channelhead,
             is_channeltail, is_majorconfluence, is_minorconfluence,
             is_majorinflow, is_minorinflow, is_leftflank, is_rightflank,
             is_midslope, is_ridge, was_channelhead, is_subsegmenthead, is_loop,
             is_blockage;
    uint32_t segmentation_threshold;
    float bandwidth;
    uint32_t n_data, n_hist_bins, n_pdf_points;
    float logx_min, logx_max, logx_range, bin_dx, pdf_dx, kdf_width_x;
    uint32_t n_kdf_part_points_x;
    float logy_min, logy_max, logy_range, bin_dy, pdf_dy, kdf_width_y;
    uint32_t n_kdf_part_points_y;
    uint32_t do_measure_hsl_from_ridges, kdf_kind;
} slm_params;

/* Integrator order used by the tracing entry points. */
#define SLM_RK2 2   /* the reference's integrator (opencl/computestep.cl:42-106) */
#define SLM_RK4 4   /* classical 4-stage extension; same quantisation and dt rule */

/* Launch shape of the field tracer. */
#define SLM_SCHED_PLAIN 0       /* one thread per (seed, sub-pixel) trajectory */
#define SLM_SCHED_PERSISTENT 1  /* persistent warps refilled from a work queue */

typedef struct slm_launch {
    int32_t schedule;        /* SLM_SCHED_* */
    int32_t integrator;      /* SLM_RK2 or SLM_RK4 */
    int32_t block_threads;   /* threads per block (multiple of 32); 0 = default */
    int32_t blocks_per_sm;   /* persistent schedule: resident blocks per SM; 0 = default */
    int32_t chunk;           /* persistent schedule: a warp takes new trajectories from the
                                queue once at least this many of its lanes are idle (or all
                                are); 1 = as soon as one lane is idle; 0 = default (4) */
    int32_t reserved[3];
} slm_launch;

/* One DTM tile of a batched field trace (no counterpart in the reference: it
 * traces each grid with its own kernel launch).  A tile's grids are the
 * reference's padded (nx_padded x ny_padded, x-major) arrays, stored
 * back to back with the other tiles' in shared uv / mask / slc / slt
 * buffers; its seeds (tile-local, unpadded coordinates as the reference's
 * seed_point array) are a contiguous range of the shared seed array.  The
 * three float fields are the tile's GRID_SCALE, COMBO_FACTOR (signed by the
 * direction) and DT_MAX as pocl.set_compile_options derives them. */
typedef struct slm_tile {
    uint64_t grid_offset;          /* first padded pixel of the tile */
    uint32_t nx_padded, ny_padded;
    uint32_t seed_begin, n_seeds;  /* seed_point[seed_begin .. seed_begin + n_seeds) */
    float grid_scale, combo_factor, dt_max;
    uint32_t reserved;
} slm_tile;

const char* slm_version(void);
const char* slm_last_error(void);
int slm_device_count(void);

/* Words of device scratch the field tracer needs (queue head and counters);
 * the caller allocates slm_fields_workspace_words() uint64 words. */
size_t slm_fields_workspace_words(void);

/* integrate_fields: d*d jittered sub-pixel trajectories per seed, downstream
 * or upstream (sign carried in combo_factor / downup_sign), accumulating per
 * pixel the streamline count slc (+1 per visit) and the rounded running length
 * slt (+ (uint)(l+0.5)).  Replaces kernel integrate_fields
 * (opencl/integratefields.cl:60-114, jittertrajectory.cl:42-88) bound by
 * Fields.gpu_integrate (python/streamlines/fields.py:217-260).
 *   seed_point [n_seed_points] float2 (x,y) in unpadded pixel units
 *   mask       [nxy_padded] uint8 (nonzero = masked)
 *   uv         [nxy_padded] float2, x-major (idx = ny_padded*x + y)
 *   mapping    unused by the kernel (kept for argument-order parity); may be NULL
 *   slc, slt   [nxy_padded] uint64 accumulators (added to, not cleared)
 *   workspace  [slm_fields_workspace_words()] uint64; on return word 1 holds
 *              the number of RK steps and word 2 the number of trajectories
 *              traced by this call (stream-ordered).
 * Seeds seeds_chunk_offset .. n_seed_points-1 are traced (the whole list when
 * seeds_chunk_offset is 0). */
int slm_integrate_fields(const slm_params* p, const slm_launch* launch,
                         const float* seed_point, const uint8_t* mask, const float* uv,
                         uint32_t* mapping, uint64_t* slc, uint64_t* slt,
                         uint64_t* workspace, void* stream);

/* slm_integrate_fields_scheduled: slm_integrate_fields with two options for
 * the scheduler (no counterpart in the reference; neither changes a result):
 *   seed_order  [n_seed_points] uint32 or NULL: queue position j traces seed
 *               seed_order[j] (its RNG stream still follows the seed index),
 *               so trajectories can be issued e.g. longest first;
 *   item_steps  [(n_seed_points - seeds_chunk_offset) * d*d] uint16 or NULL:
 *               RK steps of each trajectory (saturated at 65535), indexed by
 *               queue position * d*d + sub-pixel index -- the training data of
 *               the learned length scheduler. */
int slm_integrate_fields_scheduled(const slm_params* p, const slm_launch* launch,
                                   const float* seed_point, const uint8_t* mask, const float* uv,
                                   uint32_t* mapping, uint64_t* slc, uint64_t* slt,
                                   uint64_t* workspace, const uint32_t* seed_order,
                                   uint16_t* item_steps, void* stream);

/* slm_integrate_fields_pair -- no counterpart in the reference (which runs
 * one integrate_fields launch per direction): both directions of one grid in
 * one persistent launch, so one direction's long last trajectories overlap
 * the other's bulk.  p_down / p_up: the two directions' parameter blocks
 * (they may differ only in COMBO_FACTOR's sign and DOWNUP_SIGN); slc, slt:
 * the downstream uint64 arrays, the upstream ones up_stride elements further
 * (>= nxy_padded), each direction's equal to slm_integrate_fields of that
 * direction; workspace words 1, 2 count both directions' steps and
 * trajectories, word 3 the upstream direction's steps; seed_order as in
 * slm_integrate_fields_scheduled for the downstream queue; seed_order_up the
 * upstream queue's order (NULL: seed_order serves both directions). */
int slm_integrate_fields_pair(const slm_params* p_down, const slm_params* p_up, const slm_launch* launch,
                              const float* seed_point, const uint8_t* mask, const float* uv, uint64_t* slc,
                              uint64_t* slt, uint64_t up_stride, uint64_t* workspace,
                              const uint32_t* seed_order, const uint32_t* seed_order_up, void* stream);

/* slm_integrate_fields_batched -- no counterpart in the reference (which
 * launches integrate_fields once per grid).  Traces every tile of a batch in
 * one persistent work-queue launch; each tile's slc/slt equal those of
 * slm_integrate_fields on that tile alone (same trajectories: the RNG stream
 * of the tile-local seed index).
 *   p        shared parameters (direction, step factor, errors, MAX_LENGTH,
 *            MAX_N_STEPS, pad, d, jitter, resolution); its grid fields and
 *            n_seed_points / seeds_chunk_offset are not used
 *   tiles    [n_tiles] DEVICE array, sorted by seed_begin, seed ranges
 *            contiguous from 0 and summing to n_seeds; all tiles share pad
 *            width and pixel size; total padded pixels < 2^32
 *   seed_order [n_seeds] or NULL: queue position j traces global seed
 *            seed_order[j]; item_steps [n_seeds*d*d] or NULL as in
 *            slm_integrate_fields_scheduled
 *   workspace  slm_fields_workspace_words() uint64; word 3 becomes 1 if a
 *            seed fell outside its tile (an inconsistent table). */
int slm_integrate_fields_batched(const slm_params* p, const slm_launch* launch, const slm_tile* tiles,
                                 uint32_t n_tiles, uint32_t n_seeds, const float* seed_point,
                                 const uint8_t* mask, const float* uv, uint64_t* slc, uint64_t* slt,
                                 uint64_t* workspace, const uint32_t* seed_order, uint16_t* item_steps,
                                 void* stream);

/* slm_integrate_fields_noalloc -- no counterpart in the reference.
 * For callers that cannot call cudaMalloc: a host application that hands a
 * plugin only its own pre-allocated device buffers, or a binding of the
 * reference's six-buffer integrate_fields signature, which has no workspace
 * argument.  Same field trace and results as slm_integrate_fields, but it
 * allocates nothing: its scratch (work-queue head, step and trajectory
 * counters) lives in a static device array of SLM_NOALLOC_SCRATCH_WORDS uint64
 * words inside this library, which every GPU that loads the library holds
 * until the process exits.  The caller still passes every input and output.
 * Every call looks up the array's device address in the current context
 * (cudaGetSymbolAddress), so a cudaDeviceReset or a change of context between
 * calls is safe; the first call on a device may load the module there, so
 * make it before any stream capture.  All calls share the one array and each call
 * clears the words it uses: calls that overlap on the GPU (several streams or
 * host threads) race on it, so the caller must serialise them.  The step and
 * trajectory counters are not returned.  Returns SLM_ERR_CAPACITY if the
 * tracer ever needs more scratch than the array holds. */
#define SLM_NOALLOC_SCRATCH_WORDS 64
int slm_integrate_fields_noalloc(const slm_params* p, const slm_launch* launch,
                                 const float* seed_point, const uint8_t* mask, const float* uv,
                                 uint32_t* mapping, uint64_t* slc, uint64_t* slt, void* stream);

/* slm_selftest_div6 -- no counterpart in the reference: checks on the
 * device, over all 2^32 float bit patterns, that the tracer's x / 6 (the
 * RK4 step's weighted sum; a product by a two-float constant where that is
 * exact, else a division) equals the IEEE quotient.  counts:
 * two device uint64 words; [0] receives the number of inputs that differ
 * (NaN equals NaN), [1] the largest such bit pattern plus one (0: none). */
int slm_selftest_div6(uint64_t* counts, void* stream);

/* slm_selftest_cvt_i8 -- no counterpart in the reference: checks on the
 * device, over all 2^32 float bit patterns, that the tracer's float -> char
 * conversion (one range test around the device's saturating conversion)
 * equals the x86 conversion the reference's compress/approximate follow
 * (essentials.cl:71-109): truncation in range, INT32_MIN's low byte (0)
 * for NaN and out of range.  counts: DEVICE [2] uint64: mismatches, and the
 * largest mismatching bit pattern + 1 (0: none).  Asynchronous. */
int slm_selftest_cvt_i8(uint64_t* counts, void* stream);

/* slm_fields_finish: the host arithmetic of Fields.integrate
 * (fields.py:146-167, 293-310) on the device, so only the finished fields
 * leave the GPU.  acc [2 directions][slc, slt][nxy_padded] uint64 raw sums
 * (as accumulated by slm_integrate_fields); ds_scale_* = mean ds / pixel
 * size per direction (the trajectory statistics).  Outputs [nxy_padded][2]
 * (direction innermost, the (nxp, nyp, 2) arrays): slc float64, slt and
 * sla float32.  The same NumPy promotion order as the reference (raw sums
 * wrapped to uint32 unless exact); slc's pow(x, 2/3) is taken from
 * slc_table[count] when count < table_len (a table the caller computes with
 * the reference expression, for bit-identical values), else computed here
 * (within 2 ulp). */
int slm_fields_finish(const uint64_t* acc, uint32_t nxy_padded, uint32_t density,
                      double ds_scale_down, double ds_scale_up, int exact,
                      const double* slc_table, uint32_t table_len, double* slc_out,
                      float* slt_out, float* sla_out, void* stream);

/* integrate_trajectory: one un-jittered trajectory per seed of the chunk
 * seeds_chunk_offset .. seeds_chunk_offset+n_chunk-1 (clipped to
 * n_seed_points), recording each step as a char2 at 1/trajectory_resolution
 * px, the step count (uint16) and the length in px (float).  Replaces kernel
 * integrate_trajectory (opencl/integratetraj.cl:54-97, trajectory.cl:41-80)
 * bound by Trajectories.gpu_compute_trajectories
 * (python/streamlines/trajectories.py:196-317).
 *   trajectories [n_chunk * max_n_steps] int8x2, row g = chunk-local seed g
 *   nsteps       [n_chunk] uint16
 *   length       [n_chunk] float */
int slm_integrate_trajectory(const slm_params* p, int32_t integrator, uint32_t n_chunk,
                             const float* seed_point, const uint8_t* mask, const float* uv,
                             uint32_t* mapping, int8_t* trajectories, uint16_t* nsteps,
                             float* length, void* stream);


/* ---- kernel-density estimation (log-distributions) ----
 * Histograms are added to (zero them first); the smoothing passes overwrite.
 * kdf_kind selects the kernel shape (KDF_IS_<shape>); n_hist_bins must be a
 * multiple of n_pdf_points (the reference assumes so, opencl/kde.cl:438). */

/* histogram_univariate (opencl/kde.cl:383-394) as run by kde.gpu_compute
 * (python/streamlines/kde.py:196-293) for estimate_univariate_pdf (kde.py:116-194).
 *   sl [n_data] float log-values; hist [n_hist_bins] uint32 */
int slm_histogram_univariate(const slm_params* p, const float* sl, uint32_t n_data,
                             uint32_t* hist, void* stream);

/* pdf_univariate (opencl/kde.cl:426-526): hist [n_hist_bins] -> pdf [n_pdf_points] */
int slm_pdf_univariate(const slm_params* p, const uint32_t* hist, float* pdf, void* stream);

/* histogram_bivariate (opencl/kde.cl:109-123) for estimate_bivariate_pdf (kde.py:35-114).
 *   sl [n_data] float2 (x,y); hist [n_hist_bins^2] uint32, index y + n_hist_bins*x */
int slm_histogram_bivariate(const slm_params* p, const float* sl, uint32_t n_data,
                            uint32_t* hist, void* stream);

/* pdf_bivariate_rows (opencl/kde.cl:144-228): hist -> partial [n_hist_bins^2] float */
int slm_pdf_bivariate_rows(const slm_params* p, const uint32_t* hist, float* partial, void* stream);

/* pdf_bivariate_cols (opencl/kde.cl:249-361): partial -> pdf [n_pdf_points^2] float */
int slm_pdf_bivariate_cols(const slm_params* p, const float* partial, float* pdf, void* stream);

/* ---- channel / segment / hillslope mapping ----
 * One entry point per reference mapping kernel, same buffers in the same
 * order after (params, n_seeds, seed_point).  Results equal the reference's
 * work-items run one after another in ascending global id (the reference
 * races in count_downchannels, flag_downchannels, segment_downchannels,
 * prune_channel_heads and fix_*_flanks; this is the schedule its results are
 * pinned to).  `status` is a device word cleared by the call: bit 0 = a loop
 * cap the reference would exceed was hit, bit 1 = an out-of-grid neighbour
 * was skipped.  Entry points with a workspace run a counting pass first: with
 * too small a workspace they return SLM_ERR_CAPACITY and write the bytes
 * needed to *required_bytes (host pointer); fix_*_flanks and
 * count_downchannels synchronise the stream. */

/* connect_channels (opencl/connect.cl:26-108; connect.py:32-79);
 * interchannel_max_n_steps must be <= 256 */
int slm_connect_channels(const slm_params* p, uint32_t n_seeds, const float* seed_point,
                         const uint8_t* mask, const float* uv, uint32_t* mapping,
                         uint32_t* status, void* stream);
/* map_channel_heads (opencl/channelheads.cl:32-93; channelheads.py:33-80) */
int slm_map_channel_heads(const slm_params* p, uint32_t n_seeds, const float* seed_point,
                          const uint8_t* mask, const float* uv, uint32_t* mapping, void* stream);
/* prune_channel_heads (opencl/channelheads.cl:143-199; channelheads.py:82-118) */
int slm_prune_channel_heads(const slm_params* p, uint32_t n_seeds, const float* seed_point,
                            const uint8_t* mask, const float* uv, uint32_t* mapping, void* stream);
/* count_downchannels (opencl/countlink.cl:34-114; countlink.py:36-81) */
size_t slm_count_downchannels_workspace(uint32_t n_seeds, uint64_t n_path_events);
int slm_count_downchannels(const slm_params* p, uint32_t n_seeds, const float* seed_point,
                           const uint8_t* mask, const float* uv, uint32_t* mapping, uint32_t* count,
                           uint32_t* link, void* workspace, size_t workspace_bytes,
                           uint64_t* required_bytes, void* stream);
/* flag_downchannels (opencl/countlink.cl:134-210; countlink.py:83-130), the
 * heads' walks all at once with the result of the sequential order; the
 * workspace (slm_flag_downchannels_workspace bytes; SLM_ERR_CAPACITY with
 * *required_bytes otherwise) holds four per-pixel and three per-seed arrays */
size_t slm_flag_downchannels_workspace(uint32_t n_seeds, uint32_t nxy_padded);
int slm_flag_downchannels(const slm_params* p, uint32_t n_seeds, const float* seed_point,
                          const uint8_t* mask, const float* uv, uint32_t* mapping, uint32_t* count,
                          const uint32_t* link, void* workspace, size_t workspace_bytes,
                          uint64_t* required_bytes, void* stream);
/* label_confluences (opencl/label.cl:49-134; label.py:33-78); slt = downstream slt, float */
int slm_label_confluences(const slm_params* p, uint32_t n_seeds, const float* seed_point,
                          const uint8_t* mask, const float* uv, const float* slt, uint32_t* mapping,
                          const uint32_t* count, const uint32_t* link, void* stream);
/* segment_downchannels (opencl/segment.cl:38-107; segment.py:34-93) */
int slm_segment_downchannels(const slm_params* p, uint32_t n_seeds, const float* seed_point,
                             const uint8_t* mask, const float* uv, uint32_t* mapping,
                             const uint32_t* count, const uint32_t* link, uint32_t* label,
                             uint32_t* status, void* stream);
/* segment_hillslopes (opencl/segment.cl:133-188; segment.py:95-146) */
int slm_segment_hillslopes(const slm_params* p, uint32_t n_seeds, const float* seed_point,
                           const uint8_t* mask, const float* uv, const uint32_t* mapping,
                           const uint32_t* count, const uint32_t* link, uint32_t* label, void* stream);
/* subsegment_channel_edges (opencl/segment.cl:195-334; segment.py:148-195) */
int slm_subsegment_channel_edges(const slm_params* p, uint32_t n_seeds, const float* seed_point,
                                 const uint8_t* mask, const float* uv, uint32_t* mapping,
                                 const uint32_t* channel_label, const uint32_t* link,
                                 uint32_t* label, uint32_t* status, void* stream);
/* subsegment_flanks (opencl/segment.cl:360-414; segment.py:197-208) */
int slm_subsegment_flanks(const slm_params* p, uint32_t n_seeds, const float* seed_point,
                          const uint8_t* mask, const float* uv, const uint32_t* mapping,
                          const uint32_t* channel_label, const uint32_t* link, uint32_t* label,
                          void* stream);
/* slm_exclusive_scan_u64 -- no counterpart in the reference (the prefix sum
 * behind the mapping kernels' stored walks): out[i] = in[0] + ... + in[i-1]
 * for i <= n (out[n] = the total).  in [n], out [n+1], scratch
 * [slm_exclusive_scan_u64_scratch(n) bytes]: DEVICE, 8-byte aligned.
 * Asynchronous. */
size_t slm_exclusive_scan_u64_scratch(uint32_t n);
int slm_exclusive_scan_u64(const uint64_t* in, uint32_t n, uint64_t* out, void* scratch, size_t scratch_bytes,
                           void* stream);

/* slm_fmm_lengths -- the fast-marching distances behind pass 2's hillslope
 * lengths (python/streamlines/mapping.py:841-900, Mapping.fmm_lengths, which
 * calls scikit-fmm's skfmm.distance per fine subsegment).  One problem per
 * subsegment[i] (an absolute label value): the window pixels with |label| ==
 * subsegment[i], grown by one pixel (4-neighbour), are the domain; the
 * domain's own-label pixels whose flags hold all of thin_bit take phi = -1,
 * the rest +1; the signed distance from phi's zero contour is marched over
 * the domain (second-order fast marching when order == 2, first-order when
 * 1; unit grid, times dx).  Per problem: sum[i] and count[i] of the reached
 * distances (the reference's mean is sum / count), n_phi[i] (own-label
 * pixels), n_channel[i] (own-label thin-channel pixels) and status[i]: 0 ok,
 * 1 no channel pixel (nothing marched), 2 no zero contour, 3 heap full
 * (internal), 4 box or workspace out of range (the problem is skipped).
 * box[4i..4i+3] = x0, x1, y0, y1 (inclusive) must hold the domain (the
 * own-label pixels' box grown by one, clipped to the window); offset[i] is
 * the problem's first pixel in the workspaces, which hold total pixels:
 * val_ws [total] (on return the signed distance times dx on reached pixels,
 * else 0), st_ws [total] (bits 0-1: 2 = reached, 3 = outside the domain;
 * bit 2: phi < 0), hkey_ws [4 total], hidx_ws [4 total].
 * label, flags [nx*ny] row-major; every pointer is DEVICE.  Asynchronous. */
int slm_fmm_lengths(const int32_t* label, const uint32_t* flags, int nx, int ny, uint32_t thin_bit,
                    const int32_t* subsegment, const int32_t* box, const int64_t* offset, int n, int64_t total,
                    int order, double dx, double* val_ws, uint8_t* st_ws, double* hkey_ws, int32_t* hidx_ws,
                    double* sum, int64_t* count, int64_t* n_phi, int64_t* n_channel, int32_t* status,
                    void* stream);

/* fix_right_flanks / fix_left_flanks (opencl/segment.cl:441-504, 530-594;
 * segment.py:210-232), with the result of the items run in ascending order.
 * The walks are traced in parallel, once, into linked blocks of the path
 * store (the workspace beyond the minimum slm_fix_flanks_workspace(n, nxy,
 * 0)), then settled in one persistent launch that takes items in ascending
 * order and waits (bounded) for the final label of a lower-index item whose
 * pixel it reads.  When the store is too small the walks are traced again
 * into index-ordered contiguous chunks of it (SLM_ERR_CAPACITY with
 * *required_bytes when one path does not fit) and settled chunk by chunk.
 * If a wait runs out, or when the environment variable SLM_FLANK_ROUNDS is
 * nonzero, the labels are restored and the items resolve in rounds
 * instead. */
size_t slm_fix_flanks_workspace(uint32_t n_seeds, uint32_t nxy_padded, uint64_t n_path_steps);
int slm_fix_right_flanks(const slm_params* p, uint32_t n_seeds, const float* seed_point,
                         const uint8_t* mask, const float* uv, const uint32_t* mapping,
                         const uint32_t* channel_label, const uint32_t* link, uint32_t* label,
                         void* workspace, size_t workspace_bytes, uint64_t* required_bytes,
                         void* stream);
int slm_fix_left_flanks(const slm_params* p, uint32_t n_seeds, const float* seed_point,
                        const uint8_t* mask, const float* uv, const uint32_t* mapping,
                        const uint32_t* channel_label, const uint32_t* link, uint32_t* label,
                        void* workspace, size_t workspace_bytes, uint64_t* required_bytes,
                        void* stream);
/* hillslopes (opencl/hillslopes.cl:31-91; hillslopes.py:32-80) */
int slm_hillslopes(const slm_params* p, uint32_t n_seeds, const float* seed_point,
                   const uint8_t* mask, const float* uv, const uint32_t* mapping,
                   const uint32_t* count, uint32_t* link, void* stream);
/* slm_thin: Zhang-Suen thinning of a 0/1 image [nx][ny] (x-major; outside
 * the image counts as 0) in place on the device, the host step that thins
 * the channel mask between the mapping kernels (the reference does it with
 * scikit-image's skeletonize(medial_axis(...)), mapping.py:707-719).  Each
 * iteration is two sub-iterations; stops after an iteration that removes
 * nothing, or after max_iter.  scratch: nx*ny bytes; flag: 1 uint32 of
 * device scratch; *iterations (may be NULL) receives the iterations run. */
int slm_thin(uint8_t* image, uint8_t* scratch, uint32_t nx, uint32_t ny, uint32_t max_iter,
             uint32_t* flag, uint32_t* iterations, void* stream);
/* ---- host steps between the mapping kernels, on the device (map_device.cu);
 * each restates the host wrappers' NumPy expression element for element ---- */
/* pick_seeds (useful.py:519-538): seed_point [capacity] float2 receives, in
 * argwhere (index) order, (x - pad, y - pad) of the pixels that are unmasked
 * (mask non-NULL) and have (map & flag) > 0 (map non-NULL; ~map when
 * invert_map); *n_picked = their number (SLM_ERR_CAPACITY if > capacity) */
size_t slm_pick_seeds_workspace(uint32_t n_pixels);
int slm_pick_seeds(const uint8_t* mask, const uint32_t* map, uint32_t flag, int invert_map,
                   uint32_t nx_padded, uint32_t ny_padded, uint32_t pad, float* seed_point,
                   uint32_t capacity, uint32_t* n_picked, void* workspace, size_t workspace_bytes,
                   void* stream);
/* map_channels (mapping.py:695-702): mapping = IS_CHANNEL where
 * slt >= thr and slt*2 >= slc (slt float32, slc float64, downstream) */
int slm_map_channels(const float* slt_down, const double* slc_down, float channel_threshold,
                     uint32_t n_pixels, uint32_t is_channel, uint32_t* mapping, void* stream);
/* flag updates: op 0 m[(m&a)==a] |= b; op 1 m[(m&a)!=0] ^= a;
 * op 2 m[select!=0] |= b; op 3 select = ((m&a)==a) | ((m&b)==b) */
int slm_flag_op(uint32_t* mapping, uint8_t* select, uint32_t n_pixels, int op, uint32_t a, uint32_t b,
                void* stream);
/* segment relabelling (segment.py:83-88): positive labels -> 1 + their rank
 * among the distinct positive labels; *n_labels = number of distinct ones */
size_t slm_relabel_workspace(uint32_t n_pixels);
int slm_relabel(uint32_t* label, uint32_t n_pixels, void* workspace, size_t workspace_bytes,
                uint32_t* n_labels, void* stream);
/* label[label < 0] = -(int64(label) + left_flank_addition) (mapping.py:772-773) */
int slm_signed_labels(uint32_t* label, uint32_t n_pixels, uint32_t left_flank_addition, void* stream);
/* hillslope_lengths (opencl/lengths.cl:37-116; lengths.py:33-92);
 * traj_length [n_seeds] float, written only where a channel is reached */
int slm_hillslope_lengths(const slm_params* p, uint32_t n_seeds, const float* seed_point,
                          const uint8_t* mask, const float* uv, const uint32_t* mapping,
                          const uint32_t* label, float* traj_length, void* stream);

/* ------------------------------------------------------------------------
 * Learned trajectory-length scheduler -- no counterpart in the reference.
 * A small BF16 CNN reads the 16x16x2 uv patch around each seed pixel and
 * predicts log(1 + RK steps) of its downstream and upstream trajectories;
 * slm_order_by_prediction turns one column of predictions into the
 * seed_order of slm_integrate_fields_scheduled (longest predicted first).
 * Ordering never changes the traced fields.
 *
 * Weights (fp32 arrays holding bfloat16-rounded values):
 *   w1 [32][32]  conv1 4x4/4, row f = 2*(4*di+dj)+c     b1 [32]
 *   w2 [128][64] conv2 2x2/2, row g = 32*(2*ei+ej)+o    b2 [64]
 *   w3 [256][2]  dense, row h = 64*u+o2                 b3 [2]
 * ---------------------------------------------------------------------- */
/* conv1 input rows: x1[(s*16 + t)*32 + f], the uv patch of seed index[s]
 * (index NULL: s), clamped to the padded grid, rounded to bfloat16 */
int slm_cnn_gather(const float* uv, uint32_t nx_padded, uint32_t ny_padded, uint32_t pad,
                   const float* seed_point, const uint32_t* index, uint32_t n, float* x1,
                   void* stream);
/* conv1 activations [n*16][32] -> conv2 input rows [n*4][128] (backward = 0),
 * or the gradient the other way (backward = 1) */
int slm_cnn_rearrange(const float* src, uint32_t n, float* dst, int backward, void* stream);
/* C[M][N] = op(A) op(B) (+ bias[N], ReLU, pre-activation into Z, bf16 round
 * of the output), fp32; op(A) = A [M][K] or, trans_a, A^T with A [K][M];
 * op(B) = B [K][N] or, trans_b, B^T with B [N][K]; N <= 256.  The products
 * run on the tensor cores (tcgen05) with A and B rounded to bfloat16 and fp32
 * accumulation.  split_k > 0 instead adds the product into C over split_k
 * K-slices (bias, Z, relu and round_out are then ignored): each slice's tile
 * goes to partial [split_k][M][N] (device workspace) and the slices are
 * added into C in slice order, so the result does not depend on the order
 * the blocks run in.  status: a device word; bit 0 is set if a tensor-core
 * wait ran out (the launch then leaves C incomplete). */
int slm_gemm(int trans_a, int trans_b, int M, int N, int K, const float* A, const float* B,
             float* C, float* Z, const float* bias, int relu, int round_out, int split_k,
             float* partial, uint32_t* status, void* stream);
/* dz[i] = z[i] > 0 ? da[i] : 0 */
int slm_relu_backward(const float* da, const float* z, uint64_t n, float* dz, void* stream);
/* db[c] += sum_r dz[r][c] */
int slm_bias_grad(const float* dz, uint64_t rows, int cols, float* db, void* stream);
/* dy = 2 w (y - t) * inv_n, *loss += sum w (y - t)^2 * inv_n (w NULL: 1) */
int slm_mse(const float* y, const float* t, const float* w, uint64_t n_el, float inv_n, float* dy,
            float* loss, void* stream);
/* one Adam step (bias corrections for step >= 1) on fp32 master weights w;
 * wq receives the bfloat16-rounded weights (round_w = 1) or a copy */
int slm_adam(float* w, float* wq, const float* g, float* m, float* v, uint64_t n, float lr,
             float b1, float b2, float eps, int step, int round_w, void* stream);
/* fused inference on the tensor cores: out [n][2] predictions for seeds
 * seed_point [n] (float2 pixel coordinates, unpadded).  index (NULL: none)
 * is the order the seeds are visited in (e.g. a spatial order, so that
 * neighbouring patches share cache lines); out stays indexed by seed. */
int slm_cnn_infer(const float* uv, uint32_t nx_padded, uint32_t ny_padded, uint32_t pad,
                  const float* seed_point, const uint32_t* index, uint32_t n,
                  const float* w1, const float* b1,
                  const float* w2, const float* b2, const float* w3, const float* b3,
                  float* out, void* stream);
/* order [n]: seed indices by column col of pred [n][stride], longest predicted
 * first, in n_bins equal bins over [lo, hi] (bins: n_bins uint32 scratch) */
int slm_order_by_prediction(const float* pred, uint32_t stride, uint32_t col, uint32_t n,
                            float lo, float hi, uint32_t n_bins, uint32_t* bins,
                            uint32_t* order, void* stream);
/* Spatial seed order (no counterpart in the reference, which shuffles the
 * seeds): order [n] lists the seeds by block_px x block_px pixel block of an
 * nx x ny (unpadded) grid, blocks x-major, so the trajectories traced at the
 * same time share uv / mask / slc / slt cache lines.  With pred (NULL: none),
 * the seeds whose pred[i*stride+col] >= threshold come first, each class in
 * spatial order.  bins: scratch of slm_order_spatial_bins(...) uint32. */
uint32_t slm_order_spatial_bins(uint32_t nx, uint32_t ny, uint32_t block_px, int with_prediction);
int slm_order_spatial(const float* seed_point, uint32_t n, uint32_t nx, uint32_t ny,
                      uint32_t block_px, const float* pred, uint32_t stride, uint32_t col,
                      float threshold, uint32_t* bins, uint32_t n_bins_capacity, uint32_t* order,
                      void* stream);

/* slm_create_seeds -- HOST code (all pointers are host memory): the field
 * seed list of create_seeds (python/streamlines/useful.py:470-517):
 * argwhere(~mask) - pad as float32 (x, y) rows, in the row order NumPy's
 * global legacy generator gives them after np.random.seed(rng_seed);
 * np.random.shuffle(...) when do_shuffle.  mask: [nx_padded][ny_padded]
 * uint8 (nonzero = masked).  *n_seeds receives the number of unmasked
 * pixels; with seed_point NULL nothing else happens (size query), else
 * seed_point [capacity][2] receives the rows (SLM_ERR_CAPACITY when too
 * small).  generator_state (NULL: not wanted) [625]: the MT19937 key and
 * position after the shuffle, for numpy.random.set_state. */
int slm_create_seeds(const uint8_t* mask, uint32_t nx_padded, uint32_t ny_padded, uint32_t pad, int do_shuffle,
                     uint32_t rng_seed, float* seed_point, uint64_t capacity, uint64_t* n_seeds,
                     uint32_t* generator_state);

/* slm_create_seeds_device -- the seed list of slm_create_seeds (the same
 * rows in the same order, and the same generator state), built in DEVICE
 * memory: argwhere by the order-preserving compaction of slm_pick_seeds; the
 * swap partners drawn on the host with the same generator, by a thread of
 * its own; the Fisher-Yates swaps applied on the device in reservation
 * rounds (a swap runs once it is the earliest pending swap on both of its
 * rows), chunk by chunk (4 M swaps, in sequential order) as their partners
 * are drawn, which replaces the host's random-access pass over the rows.  Replaces create_seeds
 * (python/streamlines/useful.py:470-517) for callers that trace on the GPU.
 *   mask        DEVICE [nx_padded][ny_padded] uint8 (nonzero = masked)
 *   seed_point  DEVICE [capacity][2] float32, 8-byte aligned
 *   n_seeds     host: the number of unmasked pixels (also on SLM_ERR_CAPACITY)
 *   generator_state  host [625] or NULL, as slm_create_seeds
 *   workspace   DEVICE, 256-byte aligned, slm_create_seeds_device_workspace
 *               (nx_padded * ny_padded) bytes
 * Synchronises the stream (it reads back the row count and, per round, the
 * number of swaps still pending). */
size_t slm_create_seeds_device_workspace(uint64_t n_pixels);
int slm_create_seeds_device(const uint8_t* mask, uint32_t nx_padded, uint32_t ny_padded, uint32_t pad,
                            int do_shuffle, uint32_t rng_seed, float* seed_point, uint64_t capacity,
                            uint64_t* n_seeds, uint32_t* generator_state, void* workspace,
                            size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------- preprocess
 * The conditioned gradient vector field of a DTM region of interest
 * (Preprocess.conditioned_gradient_vector_field + mask_nan_uv,
 * python/streamlines/preprocess.py:531-621; find_blockages :647-699,
 * find_and_fix_loops :302-349, fix_blockages :351-387), replacing the
 * reference's NumPy / scipy generic_filter / numba host code. */
#define SLM_F32 0
#define SLM_F64 1
typedef struct slm_preprocess_params {
    double pixel_size;           /* geodata.pixel_size (the gradient divides by its float32 value) */
    double vecsum_threshold;     /* preprocess parameters (json/defaults.json: 0.95, -0.5, 0.0) */
    double divergence_threshold;
    double curl_threshold;
    uint32_t pad_width;          /* geodata.pad_width */
    uint32_t do_normalize_speed; /* nonzero: renormalise after the fixes, else scale by the raw speed */
} slm_preprocess_params;
/* roi [nx][ny] (x-major, as geodata.roi_array; float32 or float64 by
 * roi_dtype; NaN = no data), nx, ny >= 2.  Outputs (device; every one but
 * uv may be NULL), padded = [nx + 2 pad][ny + 2 pad]:
 *   uv                padded float2, edge-padded, NaN vectors zeroed (uv_array)
 *   slope             padded float32 degrees (slope_array)
 *   uv_mask           padded uint8, 1 where uv was NaN (the 'uv' active mask)
 *   mask              padded uint8: the pad frame, NaN ROI pixels and uv_mask
 *                     (the 'dtm' mask with h_min 'none', or'd with 'uv')
 *   blockages, blocked_neighbors  [nx][ny] uint8 flow codes (find_blockages)
 *   loop_cells        [nx][ny] uint8, 1 at cell (x, y) (pixels x..x+1,
 *                     y..y+1) detected as a loop; the last row and column
 *                     are 0 (the reference's cells there read beyond the
 *                     grid and cannot change the field)
 *   gradx, grady      [nx][ny] float32 topographic gradient (roi_grad*_array)
 *   n_loop_cells      1 uint32: looped cells (the reference's n_loops is 4x) */
int slm_preprocess(const void* roi, int roi_dtype, uint32_t nx, uint32_t ny, const slm_preprocess_params* prm,
                   float* uv, float* slope, uint8_t* uv_mask, uint8_t* mask, uint8_t* blockages,
                   uint8_t* blocked_neighbors, uint8_t* loop_cells, float* gradx, float* grady,
                   uint32_t* n_loop_cells, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SLM_B200_H */
