/*
 * spk_b200.h - C ABI of the B200 spectral placement path.
 *
 * Plain pointers and sizes only.  Every entry point is noexcept, returns an
 * int status (0 = ok) and reports failures as values; spk_status_code() maps
 * a status to the reference's static string code (ADR 0015 convention,
 * reference engine/pack_compute/include/spectrapack/compute/correlation.hpp:52-56).
 * Buffers passed in are borrowed for the call; outputs go to caller buffers;
 * device memory is owned by the context.  One host thread drives a context at
 * a time (the reference's "one coordinator serialises calls" rule,
 * correlation.hpp:78-79).
 *
 * Storage order everywhere is X-fastest: cell (x, y, z) of a field with shape
 * (sx, sy, sz) lives at x + sx * (y + sy * z)  (correlation.hpp:20-21).
 */
#ifndef SPK_B200_H
#define SPK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct spk_context spk_context;

/* Arithmetic used by the FFT correlation.  SPK_FP16: FP32 transforms with the
 * joint spectrum stored in FP16 (power-of-two scaled) before the product;
 * the integer residual, mass and probe checks decide whether a result is
 * admissible (CORRELATION_NUMERIC otherwise; proximity tolerance 2^-8 of
 * the output scale). */
enum { SPK_FP32 = 0, SPK_FP64 = 1, SPK_FP16 = 2 };

/* Which translations spk_correlate_binary_mask marks: SPK_MASK_ZERO, those
 * with a zero overlap count (gap_fill.cpp:404-420, free translations);
 * SPK_MASK_NONZERO, those with a non-zero count (gap_fill.cpp:443-446,
 * blocked offsets; slab_lattice.cpp:675-691, no-fit maps). */
enum { SPK_MASK_ZERO = 0, SPK_MASK_NONZERO = 1 };

/* Reference: compute::CorrelationSpec, correlation.hpp:22-27. */
typedef struct spk_correlation_spec {
    uint32_t environment_shape[3];
    uint32_t kernel_shape[3];
    int64_t environment_first[3];
    int64_t kernel_first[3];
} spk_correlation_spec;

/* Reference: compute::CorrelationLimits, correlation.hpp:29-36 (device bytes). */
typedef struct spk_correlation_limits {
    uint64_t max_working_bytes;
    uint64_t reserved_bytes;
    uint64_t max_padded_cells;
    uint64_t max_direct_terms;
} spk_correlation_limits;

/* Reference: CorrelationResult metadata + NumericReport + CorrelationStats,
 * correlation.hpp:38-72.  `padded_shape` is the FFT grid actually used. */
typedef struct spk_correlation_result {
    int64_t translation_first[3];
    uint32_t shape[3];
    double max_integer_residual;
    double mass_residual;
    double max_probe_error;
    uint64_t padded_cells;
    uint64_t working_bytes_peak;
    uint64_t direct_terms;
    uint32_t padded_shape[3];
} spk_correlation_result;

/* Reference: CorrelationEstimate, correlation.hpp:100-104. */
typedef struct spk_correlation_estimate {
    uint32_t padded_shape[3];
    uint64_t padded_cells;
    uint64_t working_bytes;
} spk_correlation_estimate;

/* Reference: runtime::OperationControl stop token and deadline
 * (engine/common/include/spectrapack/runtime/operation_control.hpp:18-45).
 * A nonzero *stop_word means user stop; deadline_ns is CLOCK_MONOTONIC
 * nanoseconds, 0 for none.  Both are polled between device phases. */
typedef struct spk_control {
    const volatile uint32_t* stop_word;
    int64_t deadline_ns;
} spk_control;

/* ---- context ---------------------------------------------------------- */

/* Opens a context on `device` with a device-memory cap (0 = no cap).  It
 * holds what the reference's FftExecution holds (make_fft_execution,
 * correlation.hpp:80-98): execution resources reused across calls, which one
 * coordinator serialises (correlation.hpp:78-79). */
int spk_context_create(int device, uint64_t max_device_bytes, spk_context** out);
void spk_context_destroy(spk_context* context);
/* Static string for a status (e.g. "CORRELATION_NUMERIC"); never NULL.  The
 * reference's static code strings (correlation.hpp:52-56, ADR 0015). */
const char* spk_status_code(int status);
/* The failure message of the last correlation call on `context` (static
 * text, "" after a success), worded as the reference words the same failure
 * site: CorrelationFailure::message, correlation.cpp:255-590.  Sites with no
 * counterpart there (device FFT length, CUDA errors) carry the library's own
 * text.  Never NULL. */
const char* spk_context_message(const spk_context* context);
/* Measurement only, no counterpart in the reference: the number of kernels
 * this library launched on the context (all entry points). */
uint64_t spk_context_launches(const spk_context* context);
/* The CUDA stream (cudaStream_t) every launch of this context is queued on,
 * so a caller can record timing events on it. */
void* spk_context_stream(const spk_context* context);
/* Per-pass device timing of the page pipeline (CUDA events around each pass
 * launch when enabled): fills up to `capacity` entries of {launches, total_ms}
 * for passes 0 spectrum-A, 1 inverse-y, 2 inverse-x+epilogue, 3 merge+exact,
 * 4 the pipelined stage (pass A of one batch of orientations with B1 and B2
 * of the two batches before it, in one launch; only under
 * SPK_PAGE_SCHEDULE=staged). */
int spk_context_set_profiling(spk_context* context, int enabled);
int spk_context_pass_times(const spk_context* context, uint64_t* launches, double* total_ms, uint32_t capacity);
/* Algorithmic HBM bytes of the profiled launches of each pass (pass 0: the
 * spectrum read once per launch, each orientation's kernel planes read and
 * legal-z planes written), for achieved-bandwidth figures. */
int spk_context_pass_bytes(const spk_context* context, double* bytes, uint32_t capacity);

/* ---- full-range correlation drop-in ----------------------------------- */

/* Replaces compute::estimate_correlation_cpu (correlation.hpp:100-106,
 * correlation.cpp:596-641) for the GPU path: FFT grid and device bytes. */
int spk_estimate_correlation(const spk_correlation_spec* spec, uint32_t precision,
                             spk_correlation_estimate* out);

/* Replaces compute::correlate_binary_cpu (correlation.hpp:108-111,
 * correlation.cpp:238-592,643-648).  Output: (E+K-1) per axis doubles,
 * X-fastest, rounded to integers, with the reference's residual (<0.25),
 * range, mass and 8-probe direct checks.  Host pointers. */
int spk_correlate_binary(spk_context* context, const spk_correlation_spec* spec,
                         const uint8_t* environment, const uint8_t* kernel,
                         const spk_correlation_limits* limits, const spk_control* control,
                         uint32_t precision, double* out_values, uint64_t out_capacity,
                         spk_correlation_result* result);

/* The binary correlation thresholded on the device, for the solver's mask
 * callers: gap_fill.cpp:392 (free translations over the legal box, read back
 * at :404-420), gap_fill.cpp:432 (blocked offsets, :443-446) and
 * slab_lattice.cpp:675 (no-fit map).  Each of them calls
 * compute::correlate_binary_cpu and rounds the values on the host.  This
 * runs the same correlation with the same checks and status codes as
 * spk_correlate_binary.  Instead of the (E+K-1)^3 doubles it writes one byte
 * per translation of the caller's box: box_first is the absolute translation
 * of mask[0], box_shape its extent, X fastest.  mask[t] is 1 when t lies in
 * the correlation range and its rounded count is zero (SPK_MASK_ZERO) or
 * non-zero (SPK_MASK_NONZERO); otherwise it is 0.  result is filled as by
 * spk_correlate_binary, and mask_capacity must hold the box.  Host pointers;
 * on a non-zero status the mask's contents are unspecified. */
int spk_correlate_binary_mask(spk_context* context, const spk_correlation_spec* spec,
                              const uint8_t* environment, const uint8_t* kernel,
                              const spk_correlation_limits* limits, const spk_control* control,
                              uint32_t precision, const int64_t box_first[3], const uint32_t box_shape[3],
                              uint32_t select, uint8_t* mask, uint64_t mask_capacity,
                              spk_correlation_result* result);

/* Replaces compute::correlate_proximity_cpu (correlation.hpp:113-117,
 * correlation.cpp:650-655): f64 environment in [0,1], binary kernel. */
int spk_correlate_proximity(spk_context* context, const spk_correlation_spec* spec,
                            const double* environment, const uint8_t* kernel,
                            const spk_correlation_limits* limits, const spk_control* control,
                            uint32_t precision, double* out_values, uint64_t out_capacity,
                            spk_correlation_result* result);

/* ---- fields ------------------------------------------------------------ */

/* Replaces solver::detail::build_proximity
 * (engine/pack_solver/src/field_proximity.hpp:32-132): exact squared EDT to
 * the nearest occupied cell, then exp(-sqrt(d2)/2), 0 where no cell is
 * occupied.  Host pointers; returns kProximityShape (21) for shapes the
 * reference rejects (field_proximity.hpp:13-27). */
int spk_build_proximity(spk_context* context, const uint32_t shape[3], const uint8_t* occupied,
                        double* values);

/* Largest field spk_build_proximity_static accepts: 64 cells per axis. */
#define SPK_STATIC_PROXIMITY_MAX_AXIS 64u
#define SPK_STATIC_PROXIMITY_MAX_CELLS (64u * 64u * 64u)

/* No counterpart in the reference: an allocation-free spk_build_proximity
 * for callers that cannot allocate device memory - for example a host engine
 * whose device memory is owned by its own pool allocator, or a steady-state
 * loop that must not allocate (an allocation can block on the device and can
 * fail).  It takes no context and calls no cudaMalloc, cudaFree or other
 * allocating routine: the scratch (squared distances, line scratch and the
 * exp(-sqrt(d2)/2) table, about 5.3 MB) is one static device array that
 * every GPU which loads this library holds until the process exits.
 * `occupied` (u8) and `values` (f64) are device pointers the caller owns;
 * `stream` is a cudaStream_t (NULL = default stream) on the current device.
 * Fields with more than SPK_STATIC_PROXIMITY_MAX_AXIS (64) cells on any axis
 * are rejected with SPK_SCRATCH_LIMIT (status 25).  The first call on a device looks up the array's address
 * and uploads the table (synchronising `stream`); make that first call before
 * any stream capture.  All calls share the array: calls that overlap on the
 * GPU (concurrent streams) race, so serialise them.  The looked-up address is
 * kept per device index for the life of the process and does not survive a
 * reset of the device's context (cudaDeviceReset): do not call this again
 * after one. */
int spk_build_proximity_static(void* stream, const uint32_t shape[3], const uint8_t* occupied, double* values);

/* ---- spectral pages ---------------------------------------------------- */

/* Reference: SpectralPipelineResult::RankedCandidate,
 * engine/pack_solver/src/spectral_pipeline.hpp:26-32. */
typedef struct spk_candidate {
    int64_t translation[3];
    double score;
    int32_t direct_zero_overlap;
    int32_t reserved;
    uint64_t orientation_index;
    double binary_overlap;
} spk_candidate;

/* Reference: CandidatePageQuery, spectral_pipeline.hpp:45-51.  mode 0 is
 * CandidatePageMode::ordinary (candidates with a zero rounded overlap,
 * recounted exactly); mode 1 is CandidatePageMode::low_overlap (every legal
 * translation, ranked by (binary_overlap, score, orientation, z, y, x), not
 * recounted: direct_zero_overlap is 0), spectral_pipeline.cpp:1758-1824. */
typedef struct spk_page_query {
    uint64_t orientation_index;
    int32_t has_cursor;
    int32_t mode;
    spk_candidate exclusive_cursor;
} spk_page_query;

/* The environment window over which a layout is correlated
 * (spectral_pipeline.cpp:107-140 window(), lattice, container z range). */
typedef struct spk_page_scene {
    int64_t environment_first[3];
    uint32_t environment_shape[3];
    double lattice_origin_mm[3];
    double lattice_pitch_mm;
    double container_min_z_mm;
    double container_height_mm;
} spk_page_scene;

/* One oriented object field (voxelize_object window) and the oriented
 * bounds' max z (physical_bounds.cpp:347) used by the score's top term. */
typedef struct spk_page_kernel {
    int64_t first[3];
    uint32_t shape[3];
    double object_max_z_mm;
} spk_page_kernel;

typedef struct spk_page_report {
    double max_integer_residual;   /* largest |b - round(b)| over legal cells (FP32) */
    double max_score_error;        /* largest |approximate - exact| score seen */
    uint64_t rescored;             /* candidates rescored exactly */
    int32_t certified;
    int32_t threshold_pass;        /* an uncertified first pass was widened */
} spk_page_report;

/* One page of build_spectral_pipeline (spectral_pipeline.cpp:914-1876, page
 * scan :1706-1824 and recount :1825-1857) for the layout whose blocked
 * occupancy is `occupancy` (u8 over the scene window) and the oriented kernel
 * `kernel_cells`.  Scores use the exact, correctly rounded proximity sum;
 * page entries are ordered by (score, orientation, z, y, x).  Host pointers;
 * `page` holds up to 32 entries. */
int spk_spectral_page(spk_context* context, const spk_page_scene* scene, const uint8_t* occupancy,
                      const spk_page_kernel* kernel, const uint8_t* kernel_cells,
                      const spk_page_query* query, spk_candidate* page, uint32_t* count,
                      spk_page_report* report);

/* ---- geometry and conservative fields ---------------------------------- */

/* An accepted solid's local mesh (reference AcceptedSolid::mesh(),
 * engine/pack_geometry/include/spectrapack/geometry/import.hpp:184-219). */
typedef struct spk_mesh {
    const double* vertices;     /* vertex_count x 3 */
    uint64_t vertex_count;
    const uint32_t* triangles;  /* triangle_count x 3, outward winding */
    uint64_t triangle_count;
} spk_mesh;

/* Replaces geometry::voxelize_object (conservative_fields.hpp:106-112,
 * conservative_fields.cpp:919-1003): the object at lattice.origin with
 * rotation q (canonical XYZW), trimmed window, cells in {0,1}.  `first` and
 * `shape` receive the window; `cells` needs shape[0]*shape[1]*shape[2]. */
int spk_voxelize_object(spk_context* context, const spk_mesh* object, const double origin_mm[3], double pitch_mm,
                        const double q_xyzw[4], int64_t first[3], uint32_t shape[3], uint8_t* cells,
                        uint64_t capacity);

/* Replaces geometry::voxelize_container (conservative_fields.hpp:119-125,
 * conservative_fields.cpp:1124-1282) over a caller window: an analytic box
 * (box_mm non-NULL, per-cell inset test) or a closed container mesh (interior
 * is free, the rest blocked, dilated by the wall clearance).  1 = blocked. */
int spk_voxelize_container(spk_context* context, const double box_mm[3], const spk_mesh* container,
                           const double origin_mm[3], double pitch_mm, const int64_t first[3],
                           const uint32_t shape[3], double wall_clearance_mm, uint8_t* cells);

/* Replaces geometry::voxelize_placed (conservative_fields.hpp:113-118,
 * conservative_fields.cpp:1005-1122): one placed copy's pair-clearance
 * blocker over a caller window (support-cropped raster, then dilation). */
int spk_voxelize_placed(spk_context* context, const spk_mesh* object, const double origin_mm[3], double pitch_mm,
                        const int64_t first[3], const uint32_t shape[3], const double translation_mm[3],
                        const double q_xyzw[4], double pair_clearance_mm, uint8_t* cells);

/* Replaces geometry::oriented_bounds (physical_bounds.cpp:347): min xyz then
 * max xyz of the rotated mesh.  Host only. */
int spk_oriented_bounds(const spk_mesh* object, const double q_xyzw[4], double bounds_mm[6]);

/* ---- validator broad phase ------------------------------------------------
 * Replaces the posed-bounds part of geometry::validate's pair loop
 * (engine/pack_geometry/src/validation.cpp:404-418, which calls
 * validation_kernel::bounds_pair_certificate -> separated_conservative_bounds,
 * validation_kernel.cpp:1245-1261) for every pair of copies at once.
 *
 * spk_posed_bounds: validation_kernel::posed_bounds (validation_kernel.cpp:
 * 1000-1088) of `count` poses of `object` (translation in mm, XYZW
 * quaternion): conservative min/max corners, count x 3 each; finite[i] = 0
 * where the reference returns no bounds (invalid pose or interval overflow;
 * the validator then rejects the layout as indeterminate).  Host code.
 *
 * spk_broad_phase: the pairs (first, second), second < first, that the
 * outward-AABB test does not certify disjoint, in the validator's visiting
 * order (first ascending, then second), skipping pairs whose copies are both
 * proven (validate_incremental's `proven`, may be null).  They are written
 * to pairs (2 x uint32 each) up to `capacity`; *unresolved receives their
 * number.  The validator's remaining certificates and exact classification
 * run only for these pairs.  SPK_SCRATCH_LIMIT (25) when *unresolved exceeds
 * capacity; SPK_INVALID_ARGUMENT for a clearance that is negative or not
 * finite (the reference then certifies nothing and reports
 * KERNEL_CLEARANCE_INVALID) or more than 2^20 copies.  Device kernels; the
 * call returns after the pairs are on the host. */
int spk_posed_bounds(const spk_mesh* object, const double* translations_mm, const double* q_xyzw, uint64_t count,
                     double* bounds_min, double* bounds_max, uint8_t* finite);
int spk_broad_phase(spk_context* context, const double* bounds_min, const double* bounds_max, const uint8_t* finite,
                    const uint8_t* proven, uint64_t copies, double clearance_mm, uint32_t* pairs, uint64_t capacity,
                    uint64_t* unresolved);

/* ---- STL export of a placement sequence -----------------------------------
 * Replaces write_stl_stage (engine/pack_io/src/result_export.cpp:1034-1123):
 * the binary STL of `copies` copies of `object`, copy c posed by
 * translation_mm[3c..3c+2] and the XYZW quaternion q_xyzw[4c..4c+3]
 * (RigidTransform::make / apply, rigid_transform.cpp:11-42), in copy order,
 * each copy's triangles in mesh order: an 80-byte zero header, the uint32
 * triangle count, then 50-byte records (float32 unit normal from the float32
 * points, the three float32 points, a zero attribute).  *size receives the
 * file size, 84 + 50 x triangles; `out` must hold it (SPK_SCRATCH_LIMIT
 * otherwise).  SPK_INVALID_ARGUMENT with the reference's message for a pose
 * without a rigid transform, a coordinate that is not a finite float32, or
 * more than 2^32 - 1 triangles.  The records are computed on the device;
 * the call returns after they are in `out`. */
int spk_export_stl(spk_context* context, const spk_mesh* object, const double* translations_mm,
                   const double* q_xyzw, uint64_t copies, uint8_t* out, uint64_t capacity, uint64_t* size);

/* Environment window of a container's bounds (spectral_pipeline.cpp:107-140). */
int spk_environment_window(const double bounds_mm[6], const double origin_mm[3], double pitch_mm,
                           int64_t first[3], uint32_t shape[3]);

/* Orientation catalogs (orientation_cube.hpp:10-80, orientations.cpp:104-172):
 * the 24 cube rotations in the reference order, or a custom list made
 * canonical (unit, w > 0 sign rule) and de-duplicated. */
int spk_cube_catalog(double out_xyzw[96]);
int spk_custom_catalog(const double* in_xyzw, uint64_t count, double* out_xyzw, uint64_t* out_count);

/* ---- placement session ---------------------------------------------------
 * A device-resident SpectralWorkspace (spectral_pipeline.hpp:67-92): the
 * container blocker, per-copy counts (BlockedField), occupancy, exact
 * proximity, the environment spectrum and every catalog orientation's kernel
 * stay in HBM across placement steps.  One session per context. */
typedef struct spk_session_desc {
    spk_mesh object;
    int32_t container_is_box;
    int32_t reserved;
    double box_mm[3];
    spk_mesh container;
    double pair_clearance_mm;
    double wall_clearance_mm;
    double lattice_origin_mm[3];
    double lattice_pitch_mm;
    const double* orientations_xyzw;
    uint64_t orientation_count;
} spk_session_desc;

typedef struct spk_session_info {
    int64_t environment_first[3];
    uint32_t environment_shape[3];
    uint32_t fft_shape[3];
    uint64_t copies;
    uint64_t orientations;
    double container_min_z_mm;
    double container_height_mm;
} spk_session_info;

int spk_session_open(spk_context* context, const spk_session_desc* desc, spk_session_info* info);
int spk_session_close(spk_context* context);
int spk_session_info_get(spk_context* context, spk_session_info* info);
/* Stamps a copy at lattice translation t with catalog orientation o
 * (BlockedField::add, conservative_fields.hpp:134-138,
 * conservative_fields.cpp:1695-1808, of voxelize_placed at pose
 * origin + pitch * t). */
int spk_session_place(spk_context* context, uint64_t orientation, const int64_t translation[3]);
/* Unstamps the most recent copy (BlockedField::remove,
 * conservative_fields.hpp:140-143, conservative_fields.cpp:1810-1885). */
int spk_session_remove_last(spk_context* context);
/* Pages for n queries over the current layout, as build_spectral_pipeline's
 * page scan and recount (spectral_pipeline.cpp:1706-1857) make them; pages
 * holds n x 32 entries. */
int spk_session_pages(spk_context* context, uint64_t n, const spk_page_query* queries, spk_candidate* pages,
                      uint32_t* counts, spk_page_report* reports);
/* Greedy fill (spectral.cpp:1460-1591 page merge, direct-zero recount gate,
 * then the session's validator when one is set): up to max_steps copies are
 * placed. */
int spk_session_greedy(spk_context* context, uint64_t max_steps, uint64_t* placed, uint64_t* orientations,
                       int64_t* translations, double* scores);

/* The caller's native validation of a chosen pose, the reference's try_pose
 * -> geometry::validate_incremental gate (spectral.cpp:1289-1430, called at
 * :1571-1591).  The greedy loops (spk_session_greedy,
 * spk_session_greedy_proposed, spk_jobs_greedy) call it for each candidate
 * with a zero exact overlap, in rank order, before placing it: pose_mm is
 * origin + pitch * translation, exactly as the reference forms the
 * CopyPose; quaternion_xyzw is the catalog entry.  Return
 * SPK_POSE_ACCEPTED to place the copy, SPK_POSE_REJECTED to leave the layout
 * unchanged and go on to the next candidate (the reference counts an
 * invalid candidate and continues), anything else to stop the fill with
 * SPECTRAL_VALIDATION_ABORTED.  Called on the thread that drives the
 * context. */
enum { SPK_POSE_ACCEPTED = 0, SPK_POSE_REJECTED = 1 };
typedef int (*spk_validate_fn)(void* user, uint64_t orientation, const int64_t translation[3],
                               const double pose_mm[3], const double quaternion_xyzw[4]);
/* Sets (or, with NULL, clears) the session's validator. */
int spk_session_set_validator(spk_context* context, spk_validate_fn validator, void* user);
/* Poses the validator has seen and rejected since the session opened. */
int spk_session_validation_counts(spk_context* context, uint64_t* validated, uint64_t* rejected);
/* Measurement only, no counterpart in the reference.  Work counters of the
 * session's page pipeline since open or the last reset:
 * out[0] first-pass pages, [1] threshold passes, [2] exactly rescored
 * candidates, [3] pages certified by the first pass. */
int spk_session_stats(spk_context* context, uint64_t out[4], int reset);
/* The session's fields, which the reference keeps as host CellFields
 * (conservative_fields.hpp:71-126).  Readback: kind 0 container blocker,
 * 1 occupancy, 2 kernel of
 * `orientation` (window in first/shape), 3 proximity (f64). */
int spk_session_field(spk_context* context, int kind, uint64_t orientation, int64_t first[3], uint32_t shape[3],
                      void* out, uint64_t capacity_bytes);

/* ---- learned orientation proposal ------------------------------------------
 * No counterpart in the reference: a small 3D CNN that ranks the catalog's
 * orientations for the current layout so a placement step pages only the k
 * best (the exhaustive step remains the fallback).  Input per sample: 2 x 32^3
 * channels-last floats ([z][y][x][c]): c = 0 the layout's occupancy fraction
 * pooled over the environment window (cells outside count as occupied),
 * c = 1 the oriented item's cells pooled to 32^3 (corner aligned).  Network:
 * conv3d 3^3 pad 1 + ReLU: 2->16 s1, 16->32 s2, 32->64 s2, 64->64 s2; mean
 * over the 4^3 voxels; linear 64->1.  BF16 tensor-core arithmetic with FP32
 * accumulation; FP32 master parameters in the flat order: per conv layer
 * weights [cout][27][cin] (tap = (kz*3+ky)*3+kx, input = out*stride+k-1) and
 * bias [cout], then head weights [64] and bias [1].  Loss: mean squared error
 * of the prediction against the label. */
typedef struct spk_proposal spk_proposal;

typedef struct spk_proposal_dataset {
    const float* crops;           /* crop_count x 32^3 occupancy channels */
    uint64_t crop_count;
    const float* items;           /* item_count x 32^3 item channels */
    uint64_t item_count;
    const uint32_t* sample_crop;  /* per sample: crop index */
    const uint32_t* sample_item;  /* per sample: item index */
    const float* sample_label;    /* per sample: target */
    uint64_t sample_count;
} spk_proposal_dataset;

/* The expiry path of the library's bounded device waits (the tcgen05
 * convolutions' mbarrier waits), on its own: one CTA waits `spins` polls
 * (1 .. 2^22) on an mbarrier that nothing arrives at.  Returns
 * SPK_DEVICE_WAIT_LIMIT, the status those kernels report when a wait runs
 * out; the context stays usable.  For tests of the error path. */
int spk_check_bounded_wait(spk_context* context, uint32_t spins);

uint64_t spk_proposal_parameter_count(void);
/* He-initialised parameters from `seed`. */
int spk_proposal_create(spk_context* context, uint64_t seed, spk_proposal** out);
void spk_proposal_destroy(spk_proposal* proposal);
int spk_proposal_get_parameters(spk_context* context, spk_proposal* proposal, float* out);
/* Replaces the parameters and resets the optimiser state. */
int spk_proposal_set_parameters(spk_context* context, spk_proposal* proposal, const float* in);
/* Predictions for `batch` host samples (batch x 32^3 x 2 floats). */
int spk_proposal_forward(spk_context* context, spk_proposal* proposal, uint64_t batch, const float* inputs,
                         float* predictions);
/* Loss and the gradient of every parameter (flat order) for one batch. */
int spk_proposal_gradients(spk_context* context, spk_proposal* proposal, uint64_t batch, const float* inputs,
                           const float* labels, float* loss, float* gradients);
/* `steps` Adam steps (beta 0.9/0.999, eps 1e-8) on batches drawn from the
 * dataset with a splitmix64 stream seeded by `seed`; losses[steps] optional. */
int spk_proposal_train(spk_context* context, spk_proposal* proposal, const spk_proposal_dataset* data, uint32_t batch,
                       uint32_t steps, float learning_rate, uint64_t seed, float* losses);

/* Proposal inputs of the open session: the current layout's occupancy
 * channel (32^3 floats) and every orientation's item channel
 * (orientations x 32^3 floats); either pointer may be NULL. */
int spk_session_features(spk_context* context, float* crop, float* items);
/* The k orientations the network ranks best for the current layout, and
 * optionally every orientation's prediction. */
int spk_session_propose(spk_context* context, spk_proposal* proposal, uint32_t k, uint64_t* orientations,
                        float* predictions);
/* Greedy fill that pages only the k proposed orientations per step; a step
 * where none of them admits a copy runs the exhaustive step (counted in
 * *fallbacks). */
int spk_session_greedy_proposed(spk_context* context, spk_proposal* proposal, uint32_t k, uint64_t max_steps,
                                uint64_t* placed, uint64_t* orientations, int64_t* translations, double* scores,
                                uint64_t* fallbacks);
/* The proposed greedy with a margin: each step pages the k_min orientations
 * the network ranks best and every further one whose prediction lies within
 * `margin` of the k_min-th, at most k_max; the exhaustive fallback as in
 * spk_session_greedy_proposed.  *paged receives the orientations paged over
 * all steps (their mean is placed / paged).  No counterpart in the reference. */
int spk_session_greedy_proposed_margin(spk_context* context, spk_proposal* proposal, uint32_t k_min, uint32_t k_max,
                                       float margin, uint64_t max_steps, uint64_t* placed, uint64_t* orientations,
                                       int64_t* translations, double* scores, uint64_t* fallbacks, uint64_t* paged);

/* No counterpart in the reference.  The proposed greedy with widening: when
 * fewer than min_feasible of the k proposed orientations admit any copy, the
 * step pages the next k in the network's order, and so on, before choosing
 * (counted in *widenings, one per block added).  min_feasible = 0 is
 * spk_session_greedy_proposed. */
int spk_session_greedy_proposed_adaptive(spk_context* context, spk_proposal* proposal, uint32_t k,
                                         uint32_t min_feasible, uint64_t max_steps, uint64_t* placed,
                                         uint64_t* orientations, int64_t* translations, double* scores,
                                         uint64_t* fallbacks, uint64_t* widenings);

/* ---- independent jobs -------------------------------------------------------
 * No counterpart in the reference: several packing jobs (each a context with
 * an open session, of any grid size and catalog) filled concurrently.  Each
 * job runs on its own host thread and its own context's stream, so the jobs'
 * kernels share the GPU; results equal running each job alone. */
typedef struct spk_job {
    spk_context* context;    /* with an open session; one job per context */
    spk_proposal* proposal;  /* NULL: exhaustive greedy; else proposed greedy (one job per proposal) */
    uint32_t k;              /* proposed orientations per step */
    uint32_t reserved;
    uint64_t max_steps;
    uint64_t* orientations;  /* max_steps entries, or NULL */
    int64_t* translations;   /* 3 x max_steps entries, or NULL */
    double* scores;          /* max_steps entries, or NULL */
    uint64_t placed;         /* out: copies placed */
    uint64_t fallbacks;      /* out: exhaustive fallback steps (proposed greedy) */
    int32_t status;          /* out: the job's status */
    int32_t reserved2;
} spk_job;

/* Runs every job to completion (or max_steps); returns SPK_INVALID_ARGUMENT
 * when two jobs share a context or a proposal, else OK with per-job status. */
int spk_jobs_greedy(spk_job* jobs, uint64_t count);

#ifdef __cplusplus
}
#endif

#endif /* SPK_B200_H */
