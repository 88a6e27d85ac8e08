/*
 * hpgb.h -- C ABI of libhpgb.so, the sm_100a (B200) gridding / degridding
 * device for HPG (hannajonathan/hpg v2.0.1).
 *
 * The reference selects its device implementation through the abstract class
 * hpg::runtime::State (src/hpg_runtime.hpp:80-207); StateT<Device::Cuda>
 * (src/hpg_runtime.hpp:721-1750) is its Kokkos/CUDA implementation.  Every
 * entry point below replaces one State virtual (or one StateT constructor),
 * named in its comment, so that a host-side State subclass can forward each
 * virtual to exactly one call here.  The C++ API in hpg_b200/cpp does that.
 *
 * Conventions
 *  - Every function returns an int status: HPGB_SUCCESS (0) or 1 + the value
 *    of the matching hpg::ErrorType (src/hpg_error.hpp:26-38).  Failures that
 *    have no ErrorType (CUDA or cuFFT errors, bad arguments) return
 *    HPGB_ERROR_OTHER.  hpgb_last_error_message() describes the last failure
 *    on the calling thread.  No C++ exception crosses this interface.
 *  - Work is asynchronous on the gridder's CUDA stream, as in the reference
 *    (one stream per task, src/hpg_runtime.hpp:1496-1588); hpgb_fence() waits
 *    for it.  Functions that hand data to the host (hpgb_copy_*) fence first.
 *  - Grid and model values are complex<double> in the device layout of the
 *    reference's CUDA device, LayoutLeft [x, y, mrow, cube] (x fastest;
 *    src/hpg_impl.hpp:190-219).  Weights are double, [mrow, cube] LayoutLeft.
 *  - Visibilities are arrays of hpgb_visdataN, byte-for-byte the layout of
 *    hpg::VisData<N> (src/hpg.hpp:236-311).
 */
#ifndef HPGB_H
#define HPGB_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HPGB_API __attribute__((visibility("default")))
#else
#define HPGB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define HPGB_ABI_VERSION 1

/* status codes: 1 + hpg::ErrorType (src/hpg_error.hpp:26-38) */
enum hpgb_status {
  HPGB_SUCCESS = 0,
  HPGB_ERROR_DISABLED_DEVICE = 1,
  HPGB_ERROR_DISABLED_HOST_DEVICE = 2,
  HPGB_ERROR_OUT_OF_BOUNDS_CF_INDEX = 3,
  HPGB_ERROR_INVALID_NUMBER_MUELLER_INDEX_ROWS = 4,
  HPGB_ERROR_INVALID_NUMBER_POLARIZATIONS = 5,
  HPGB_ERROR_INVALID_CF_LAYOUT = 6,
  HPGB_ERROR_INVALID_MODEL_GRID_SIZE = 7,
  HPGB_ERROR_EXCESSIVE_NUMBER_VISIBILITIES = 8,
  HPGB_ERROR_UPDATE_WEIGHTS_WITHOUT_GRIDDING = 9,
  HPGB_ERROR_CF_SUPPORT_EXCEEDS_GRID = 10,
  HPGB_ERROR_OTHER = 11
};

/* grid_visibilities flags: the four booleans of State::grid_visibilities
 * (src/hpg_runtime.hpp:147-154) */
enum hpgb_grid_flags {
  HPGB_UPDATE_GRID_WEIGHTS = 1u,
  HPGB_DO_DEGRID = 2u,
  HPGB_RETURN_VISIBILITIES = 4u,
  HPGB_DO_GRID = 8u
};

/* hpg::Layout (src/hpg.hpp:611-614) */
enum hpgb_layout { HPGB_LAYOUT_RIGHT = 0, HPGB_LAYOUT_LEFT = 1 };

/* hpg::FFTSign (src/hpg.hpp:965-968) */
enum hpgb_fft_sign { HPGB_FFT_POSITIVE = 0, HPGB_FFT_NEGATIVE = 1 };

/* hpg::ShiftDirection (src/hpg.hpp:989-992) */
enum hpgb_shift_direction { HPGB_SHIFT_FORWARD = 0, HPGB_SHIFT_BACKWARD = 1 };

/* Arithmetic form of the gridding kernels.
 *  FP64:  the reference's arithmetic (FP32 CF x visibility products, FP64
 *         sums, FP64 grid accumulation, FP64 degridding).
 *  MIXED: FP32 products and FP32 shared-memory tiles, merged into the FP64
 *         grid by compensated (two-sum) flushes; coordinates, phases and
 *         weight sums stay FP64. */
enum hpgb_precision { HPGB_PRECISION_FP64 = 0, HPGB_PRECISION_MIXED = 1 };

/* Kernel family used by hpgb_grid_visibilities.
 *  AUTO:   the tiled kernel when the CF fits its shared-memory ring, else
 *          the per-visibility kernels.
 *  DIRECT: per-visibility kernels with global FP64 atomics (the reference's
 *          launch structure; FP64 form only).
 *  TILED:  the tiled kernel, or an error when it cannot take the batch. */
enum hpgb_kernel_kind {
  HPGB_KERNEL_AUTO = 0,
  HPGB_KERNEL_DIRECT = 1,
  HPGB_KERNEL_TILED = 2
};

/* Layout of CF values handed to hpgb_set_cf (one buffer per CF group).
 *  LOGICAL: complex<float> indexed like CFArray::operator()(x, y, mueller,
 *           cube) (src/hpg.hpp:677-684), rightmost index fastest:
 *           ((x*ext[1] + y)*ext[2] + mueller)*ext[3] + cube.
 *  CUDA_V0: the reference CUDA device layout "0-Cuda", LayoutLeft
 *           [x_major, y_major, mueller, cube, x_minor, y_minor]
 *           (src/hpg_impl.hpp:238-281).
 *  HOST_V0: the reference host device layout "0-Serial"/"0-OpenMP", strided
 *           with axis order mueller, y_major, x_major, cube, x_minor, y_minor
 *           (src/hpg_impl.hpp:229-235). */
enum hpgb_cf_layout {
  HPGB_CF_LAYOUT_LOGICAL = 0,
  HPGB_CF_LAYOUT_CUDA_V0 = 1,
  HPGB_CF_LAYOUT_HOST_V0 = 2
};

/* hpg::VisData<N> (src/hpg.hpp:236-311), same member order and padding */
#define HPGB_VISDATA_FIELDS(N)                                              \
  float visibilities[N][2]; /* complex<float> values, by polarization */    \
  float weights[N];                                                         \
  double frequency;                                                         \
  double phase;                                                             \
  double uvw[3];                                                            \
  unsigned grid_cube;                                                       \
  unsigned cf_index[2]; /* (cube, group) */                                 \
  double cf_phase_gradient[2];

typedef struct hpgb_visdata1 { HPGB_VISDATA_FIELDS(1) } hpgb_visdata1;
typedef struct hpgb_visdata2 { HPGB_VISDATA_FIELDS(2) } hpgb_visdata2;
typedef struct hpgb_visdata3 { HPGB_VISDATA_FIELDS(3) } hpgb_visdata3;
typedef struct hpgb_visdata4 { HPGB_VISDATA_FIELDS(4) } hpgb_visdata4;

/* per-visibility coordinates reported by hpgb_debug_coords: the values
 * computed by compute_vis_coord() and the Vis constructor
 * (src/hpg_core.hpp:422-446, :513-550) */
typedef struct hpgb_vis_coords {
  int32_t grid_coord[2];  /* left edge of the CF support on the grid */
  int32_t cf_major[2];
  int32_t cf_minor[2];
  int32_t fine_offset[2];
  int32_t cf_size[2];     /* support (taps) */
  int32_t pos_w;          /* uvw[2] > 0 */
  int32_t in_grid;        /* all_within_grid() (src/hpg_core.hpp:1070-1080) */
  /* Mueller routing of this visibility, [grid row][visibility pol], -1
   * inactive: the CF Mueller plane its gridding products use
   * ((pos_w ? mueller : conjugate)[r][v], src/hpg_core.hpp:808-817) and the
   * plane its degridding products use ((pos_w ? conjugate : mueller)[r][v],
   * :598-600) */
  int32_t grid_mueller[4][4];
  int32_t degrid_mueller[4][4];
} hpgb_vis_coords;

typedef struct hpgb_gridder hpgb_gridder;

/* ABI version of the loaded library (HPGB_ABI_VERSION). */
HPGB_API int hpgb_abi_version(void);

/* Message for the last failure on this thread ("" if none). */
HPGB_API const char* hpgb_last_error_message(void);

/* Number of usable CUDA devices (hpg::devices(), src/hpg.hpp:133-135). */
HPGB_API int hpgb_device_count(int* count);

/* StateT<Cuda> constructor (src/hpg_runtime.hpp:757-781) behind
 * GridderState::create (src/hpg.cc:226-264).  mueller_indexes and
 * conjugate_mueller_indexes are row-major [grid_size[2]][num_polarizations],
 * -1 marking an unused element; rows beyond grid_size[2] and columns beyond
 * num_polarizations are inactive.  The reference's init_cf_shape argument
 * maps to a following hpgb_allocate_cf_region call.  DisabledDevice when
 * device_id names no usable device (device_id < 0 selects device 0). */
HPGB_API int hpgb_create(int device_id, unsigned max_added_tasks,
                size_t max_visibility_batch_size, const unsigned grid_size[4],
                const double grid_scale[2], unsigned num_polarizations,
                const int* mueller_indexes,
                const int* conjugate_mueller_indexes,
                hpgb_gridder** gridder);

/* StateT copy constructor (src/hpg_runtime.hpp:783-799): fences the source
 * and deep-copies grid, weights, model and CF. */
HPGB_API int hpgb_clone(const hpgb_gridder* src, hpgb_gridder** gridder);

/* ~StateT (src/hpg_runtime.hpp:827-842): fences, then frees everything. */
HPGB_API int hpgb_destroy(hpgb_gridder* gridder);

/* Select the arithmetic form (enum hpgb_precision) of later gridding calls. */
HPGB_API int hpgb_set_precision(hpgb_gridder* gridder, int precision);

/* Select the kernel family (enum hpgb_kernel_kind) of later gridding calls;
 * no counterpart in the reference. */
HPGB_API int hpgb_set_gridding_kernel(hpgb_gridder* gridder, int kind);

/* The CUDA stream (cudaStream_t) all work of this gridder is issued on. */
HPGB_API int hpgb_get_stream(const hpgb_gridder* gridder, void** stream);

/* State::convolution_function_region_size (src/hpg_runtime.hpp:131-133):
 * device bytes the CF region needs for a CF of this shape. */
HPGB_API int hpgb_cf_region_size(const hpgb_gridder* gridder, unsigned oversampling,
                        unsigned num_groups, const unsigned* extents,
                        size_t* bytes);

/* State::allocate_convolution_function_region (src/hpg_runtime.hpp:135-136). */
HPGB_API int hpgb_allocate_cf_region(hpgb_gridder* gridder, unsigned oversampling,
                            unsigned num_groups, const unsigned* extents);

/* State::set_convolution_function (src/hpg_runtime.hpp:138-139, impl
 * :890-915).  extents: [num_groups][4] (x, y, mueller, cube) in oversampled
 * units; values[g]: complex<float> buffer of group g in the given
 * hpgb_cf_layout, in host memory (values_on_device 0) or device memory.
 * Returns CFSupportExceedsGrid as the reference does. */
HPGB_API int hpgb_set_cf(hpgb_gridder* gridder, unsigned oversampling,
                unsigned num_groups, const unsigned* extents,
                const void* const* values, int layout, int values_on_device);

/* State::set_model (src/hpg_runtime.hpp:141-142, impl :917-963).
 * values: complex<double> of extents[4] in hpgb_layout order. */
HPGB_API int hpgb_set_model(hpgb_gridder* gridder, const void* values,
                   const unsigned extents[4], int layout, int values_on_device);

/* State::grid_visibilities (src/hpg_runtime.hpp:144-151, impl :965-1188).
 * visibilities: num_visibilities hpgb_visdataN records with N =
 * num_polarizations, in host memory (vis_on_device 0) or device memory;
 * host records are copied asynchronously (from pinned memory the copy may
 * still run after the call returns), so they must stay unchanged until the
 * next hpgb_fence().  A host batch's copy runs on a stream of its own, into
 * one of two staging buffers taken in turn, so that it overlaps the work of
 * the previous call.
 * flags: hpgb_grid_flags.  When HPGB_RETURN_VISIBILITIES is set, the
 * predicted or residual records are written to returned (host or device
 * memory, same kind as the input; may equal visibilities) and are valid after
 * the next hpgb_fence().  Validation order of the reference
 * (src/hpg_runtime.hpp:1816-1828): ExcessiveNumberVisibilities,
 * InvalidNumberPolarizations, UpdateWeightsWithoutGridding. */
HPGB_API int hpgb_grid_visibilities(hpgb_gridder* gridder, const void* visibilities,
                           size_t num_visibilities, unsigned num_polarizations,
                           unsigned flags, int vis_on_device, void* returned);

/* Allocation-free degridding/gridding of device-resident visibilities.
 * No counterpart in the reference's State: it serves callers that must not
 * allocate device memory while they grid (cudaMalloc/cudaFree can
 * synchronize the device, and fail in a process whose memory is already
 * handed to its own pool).  It runs the direct kernels of
 * hpgb_grid_visibilities (those of HPGB_KERNEL_DIRECT, FP64 arithmetic, for
 * either precision setting) on the caller's records in place, with the one
 * per-call scratch array, the gridding value of each visibility
 * polarization, in a fixed device array of HPGB_NOALLOC_MAX_VALUES
 * complex<float> values (8 MiB) compiled into the library.
 *
 * visibilities: num_visibilities hpgb_visdataN records in DEVICE memory.
 * With HPGB_DO_DEGRID their vis values are overwritten in place (predicted
 * values, residuals with HPGB_DO_GRID) and are valid after hpgb_fence();
 * HPGB_RETURN_VISIBILITIES is not needed.  Validation as
 * hpgb_grid_visibilities, then: gridding a batch of more than
 * HPGB_NOALLOC_MAX_VALUES / num_polarizations visibilities returns
 * ExcessiveNumberVisibilities and launches nothing.
 * The scratch array needs no initial value (every entry read is written
 * earlier in the same call).  There is one per device, shared by all
 * gridders: calls that may run at the same time on one device (streams with
 * no ordering between them) race on it; calls on one gridder are ordered by
 * its stream.  The first call on a device looks up the array's address
 * (cudaGetSymbolAddress); make that first call before any stream capture
 * starts on the device. */
#define HPGB_NOALLOC_MAX_VALUES 1048576u
HPGB_API int hpgb_grid_visibilities_noalloc(hpgb_gridder* gridder,
                                            void* visibilities,
                                            size_t num_visibilities,
                                            unsigned num_polarizations,
                                            unsigned flags);

/* Differentiable imaging: the degridding and gridding maps as FP64 linear
 * operators and their adjoints (no counterpart in the reference's State;
 * the maps are those of src/hpg_core.hpp:580-682 and :791-886).
 * visibilities: num_visibilities hpgb_visdataN records in device memory;
 * only their geometry is read (uvw, freq, phase, weights, grid_cube,
 * cf_index, cf_phase_gradient), never their vis values.  Grid-shaped
 * arrays are complex<double> in the gridder's device grid layout
 * [cube][mrow][y][x] (as hpgb_grid_device_ptr); per-visibility arrays are
 * complex<double> [num_visibilities][num_polarizations].  All arrays are in
 * device memory; the work is queued on the gridder's stream (hpgb_fence
 * waits for it).  Visibilities outside the grid contribute nothing.
 *
 * hpgb_degrid_linear:  values = D model, the degridding prediction
 *   conj(phasor) / normaliser * sum cf * screen* * model, in FP64 without
 *   rounding to complex<float> (overwrites values).
 * hpgb_degrid_adjoint: model_cotangent += D^H values_cotangent.
 * hpgb_grid_linear:    grid += G values, gridding of phasor * weight * values
 *   with FP64 products.
 * hpgb_grid_adjoint:   values_cotangent = G^H grid_cotangent (overwrites). */
HPGB_API int hpgb_degrid_linear(hpgb_gridder* gridder, const void* visibilities,
                                size_t num_visibilities,
                                unsigned num_polarizations, const void* model,
                                void* values);
HPGB_API int hpgb_degrid_adjoint(hpgb_gridder* gridder,
                                 const void* visibilities,
                                 size_t num_visibilities,
                                 unsigned num_polarizations,
                                 const void* values_cotangent,
                                 void* model_cotangent);
HPGB_API int hpgb_grid_linear(hpgb_gridder* gridder, const void* visibilities,
                              size_t num_visibilities,
                              unsigned num_polarizations, const void* values,
                              void* grid);
HPGB_API int hpgb_grid_adjoint(hpgb_gridder* gridder, const void* visibilities,
                               size_t num_visibilities,
                               unsigned num_polarizations,
                               const void* grid_cotangent,
                               void* values_cotangent);

/* State::fence (src/hpg_runtime.hpp:153-154). */
HPGB_API int hpgb_fence(const hpgb_gridder* gridder);

/* State::grid_weights (:156-157): copy weights to host dst in layout. */
HPGB_API int hpgb_copy_weights(const hpgb_gridder* gridder, double* dst, int layout);

/* State::grid_values (:165-166): copy the grid to host dst in layout. */
HPGB_API int hpgb_copy_grid(const hpgb_gridder* gridder, void* dst, int layout);

/* State::model_values (:174-175): copy the model to host dst in layout;
 * zeros when no model is set (UnallocatedModelValueArray). */
HPGB_API int hpgb_copy_model(const hpgb_gridder* gridder, void* dst, int layout);

/* State::grid_weights_ptr/_span, grid_values_ptr/_span,
 * model_values_ptr/_span (:159-183): device pointers and element counts,
 * without a fence.  The model pointer is NULL when no model is set. */
HPGB_API int hpgb_weights_device_ptr(const hpgb_gridder* gridder, void** ptr,
                            size_t* span);
HPGB_API int hpgb_grid_device_ptr(const hpgb_gridder* gridder, void** ptr,
                         size_t* span);
HPGB_API int hpgb_model_device_ptr(const hpgb_gridder* gridder, void** ptr,
                          size_t* span);

/* State::reset_grid / reset_model (:171, :186). */
HPGB_API int hpgb_reset_grid(hpgb_gridder* gridder);
HPGB_API int hpgb_reset_model(hpgb_gridder* gridder);

/* State::normalize_by_weights (:189, impl :1293-1310). */
HPGB_API int hpgb_normalize_by_weights(hpgb_gridder* gridder, double wfactor);

/* State::apply_grid_fft / apply_model_fft (:192-196, impl :1312-1426). */
HPGB_API int hpgb_apply_grid_fft(hpgb_gridder* gridder, double norm, int sign,
                        int in_place);
HPGB_API int hpgb_apply_model_fft(hpgb_gridder* gridder, double norm, int sign,
                         int in_place);

/* The imaging tail in one call: the effect of hpgb_normalize_by_weights
 * (wfactor), hpgb_apply_grid_fft(norm, sign, in place) and
 * hpgb_shift_grid(direction) in that order, done as the FFT and one pass
 * over the grid (the per-plane normalisation commutes with the FFT and is
 * applied with 1/norm in the shift's pass); equal to the three calls to
 * FP64 rounding.  No counterpart in the reference. */
HPGB_API int hpgb_image_grid(hpgb_gridder* gridder, double wfactor, double norm,
                             int sign, int direction);

/* State::shift_grid / shift_model (:198-202, impl :1428-1456). */
HPGB_API int hpgb_shift_grid(hpgb_gridder* gridder, int direction);
HPGB_API int hpgb_shift_model(hpgb_gridder* gridder, int direction);

/* Number of CUDA kernels this gridder has launched since it was created
 * (instrumentation for benchmarks; no counterpart in the reference). */
HPGB_API int hpgb_kernel_launches(const hpgb_gridder* gridder,
                                  uint64_t* count);

/* Tiled-kernel plan overrides, no counterpart in the reference (tuning):
 * ring_parts = number of the largest per-row CF parts the shared-memory
 * ring holds (0 or 2..16; the tile side shrinks to make room), chunk_vis =
 * visibilities per tile pass between flushes of the shared-memory grid tile;
 * 0 keeps the plan's own choice.  The plan's own ring holds four or five
 * parts, or two or three for CF slices too wide for four (supports up to 64
 * with one or two Mueller planes per grid row).  A plan that does not fit
 * makes the tiled kernel unusable for the batch (HPGB_KERNEL_AUTO then uses
 * the direct kernels; hpgb_last_gridding_kernel tells which ran). */
HPGB_API int hpgb_set_tiled_plan(hpgb_gridder* gridder, int ring_parts,
                                 int chunk_vis);

/* The tiled kernel's whole plan, no counterpart in the reference (tuning).
 * Every field 0 means "the plan's own choice":
 *  ring_parts     2..16: CF ring depth, in largest per-row CF parts;
 *  chunk_vis      1..2^20: visibilities per tile pass (between flushes of
 *                 the shared-memory grid tile to the grid);
 *  tile_side      even, at most 128: side R of the shared-memory uv tile in
 *                 cells (the largest that fits the ring's leftover shared
 *                 memory when 0); a side the ring leaves no room for makes
 *                 the plan not fit; the CF ring takes every whole KB the
 *                 tiles leave (at least ring_parts parts), so a smaller
 *                 side deepens the ring;
 *  compensated    mixed form only: 1: plain FP32 grid tiles; 2: FP32
 *                 high/low tile pairs updated by two-sum, so that the tile
 *                 adds no accumulation error however long the pass (the
 *                 pairs take twice the tile memory: smaller tiles).
 * hpgb_set_tiled_plan(g, r, c) sets the first two fields and clears the
 * others. */
typedef struct hpgb_tiled_plan {
  int ring_parts;
  int chunk_vis;
  int tile_side;
  int compensated;
} hpgb_tiled_plan;
enum hpgb_plan_choice { HPGB_PLAN_AUTO = 0 };
enum hpgb_compensation { HPGB_COMPENSATED_OFF = 1, HPGB_COMPENSATED_ON = 2 };
HPGB_API int hpgb_set_tiled_plan_ex(hpgb_gridder* gridder,
                                    const hpgb_tiled_plan* plan);
HPGB_API int hpgb_get_tiled_plan(const hpgb_gridder* gridder,
                                 hpgb_tiled_plan* plan);

/* State::grid_visibilities for the batches of many gridders in ONE launch
 * of the tiled kernel, no counterpart in the reference (which launches per
 * gridder).  Gridder j takes visibilities[j] (num_visibilities[j] records;
 * host or device memory as vis_on_device says), exactly as
 * hpgb_grid_visibilities(gridders[j], ..., flags, ...) would, and with
 * HPGB_RETURN_VISIBILITIES writes its returned records to returned[j]
 * (valid after hpgb_fence(gridders[0])).  Up to 96 distinct gridders on one
 * device that share the number of polarizations, grid rows, Mueller tables,
 * precision and compensation setting, and -- when degridding -- whether a
 * model is set; grid sizes, CFs and batch sizes may all differ.  Every
 * gridder's batch is sorted into uv tiles with the tile side its own CF
 * allows, and the tile passes of all of them form one work list of one
 * persistent launch.  The work runs on gridders[0]'s stream, ordered after
 * the work already queued on the others' streams and before work queued on
 * them later (outside a stream capture; inside one, the caller orders the
 * other gridders' work).  Errors: those of hpgb_grid_visibilities, checked
 * per gridder, and HPGB_ERROR_OTHER when the gridders differ in a shared
 * property or the tiled kernel cannot take their CFs. */
HPGB_API int hpgb_grid_visibilities_batch(
    hpgb_gridder* const* gridders, size_t num_gridders,
    const void* const* visibilities, const size_t* num_visibilities,
    unsigned num_polarizations, unsigned flags, int vis_on_device,
    void* const* returned);

/* Bound of every device-side wait of the tiled kernel, in seconds (0.5 by
 * default; 1e-4..60), no counterpart in the reference.  A wait that runs out
 * ends the launch early with an error status: the next hpgb_fence returns
 * HPGB_ERROR_OTHER ("a device-side wait gave up"), the batch's results are
 * incomplete, and the gridder stays usable. */
HPGB_API int hpgb_set_wait_limit(hpgb_gridder* gridder, double seconds);

/* Test hook, no counterpart in the reference: in the next tiled launches,
 * the CTA of grid row 0 that takes the visibility at this position of the
 * tile-sorted batch (of the first gridder, in a batched launch) never
 * issues its bulk copies (-1: none), so that the waits for them run out and
 * the kernel takes its timeout path.  For tests of that path only. */
HPGB_API int hpgb_debug_withhold_copy(hpgb_gridder* gridder,
                                      long long visibility);

/* Which kernel gridded/degridded the gridder's last non-empty batch:
 * HPGB_KERNEL_TILED or HPGB_KERNEL_DIRECT (HPGB_KERNEL_AUTO before the first
 * batch).  No counterpart in the reference: it makes the tiled kernel's
 * fallback to the per-visibility kernels visible to the caller. */
HPGB_API int hpgb_last_gridding_kernel(const hpgb_gridder* gridder,
                                       int* kind);

/* Autotuner of the tiled kernel, no counterpart in the reference: runs the
 * batch (as hpgb_grid_visibilities would with these flags) three times per
 * candidate plan -- CF ring depths 2..8, then uv tile sides 0, 4, 8, 12 and
 * 16 cells below the largest that fits at the fastest depth and at one part
 * less (the ring takes the bytes a smaller side frees), then tile-pass
 * lengths -- ranks the candidates by their median CUDA-event time (a launch that
 * reported a device wait timeout does not count), restores the grid and
 * weights on every exit path, and keeps the fastest plan for the gridder's
 * later calls (readable with hpgb_get_tiled_plan), returning its ring depth
 * and pass length.  The mixed form's compensation setting is kept.  Results
 * are cached in the process per workload (grid shape, polarizations,
 * Mueller tables, CF group shapes, precision, compensation, flags, model,
 * log2 of the batch size): a later call with the same workload applies the
 * cached plan at once.  Synchronous; costs about sixty runs of the batch
 * the first time: tune on a representative batch once, then grid. */
HPGB_API int hpgb_autotune_tiled(hpgb_gridder* gridder, const void* visibilities,
                                 size_t num_visibilities,
                                 unsigned num_polarizations, unsigned flags,
                                 int vis_on_device, int* ring_parts,
                                 int* chunk_vis);

/* CUDA-graph capture of a gridder's work, no counterpart in the reference
 * (the reference launches every kernel of a batch from the host each time).
 * hpgb_begin_capture fences the gridder and starts capturing its stream;
 * the calls that follow are recorded instead of run, up to
 * hpgb_end_capture, which returns an instantiated graph; hpgb_graph_launch
 * replays it on the gridder's stream (asynchronously, like the calls it
 * holds).  Capture only calls whose inputs stay where they are between
 * replays: device-resident visibilities (vis_on_device 1) or pinned host
 * buffers, the same batch size as an uncaptured call made before the
 * capture (so that no buffer grows), and no call that waits for the device
 * (hpgb_fence, copies of the grid, weights or model to the host).  A graph
 * must not outlive its gridder; destroy it with hpgb_graph_destroy. */
typedef struct hpgb_graph hpgb_graph;
HPGB_API int hpgb_begin_capture(hpgb_gridder* gridder);
HPGB_API int hpgb_end_capture(hpgb_gridder* gridder, hpgb_graph** graph);
HPGB_API int hpgb_graph_launch(hpgb_gridder* gridder, const hpgb_graph* graph);
HPGB_API int hpgb_graph_destroy(hpgb_graph* graph);

/* Benchmark instrumentation, no counterpart in the reference: while
 * enabled, CUDA events are recorded on the gridder's stream around every
 * launch of the tiled gridding kernel.  hpgb_tiled_kernel_time waits for the
 * stream, returns the summed device time (ms) and the number of launches
 * recorded since the last query, and forgets them. */
HPGB_API int hpgb_profile_tiled_kernel(hpgb_gridder* gridder, int enable);
HPGB_API int hpgb_tiled_kernel_time(hpgb_gridder* gridder, double* total_ms,
                                    uint64_t* count);

/* Debug: coordinates the device computes for each visibility (host input,
 * host output), for bit-exact comparison with the reference's
 * compute_vis_coord().  No counterpart in the reference's State. */
HPGB_API int hpgb_debug_coords(hpgb_gridder* gridder, const void* visibilities,
                      size_t num_visibilities, unsigned num_polarizations,
                      hpgb_vis_coords* out);

#ifdef __cplusplus
}
#endif

#endif /* HPGB_H */
