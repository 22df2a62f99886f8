/* isaac_b200.h -- C ABI of the B200-native ISAAC in-situ rendering hot path.
 *
 * One context renders one local volume (plus optional particle sources) into
 * an RGBA8 framebuffer on one GPU.  All device work is enqueued on the
 * caller's CUDA stream (passed as `void*` = cudaStream_t, NULL = legacy
 * default stream) and is asynchronous unless an entry point says otherwise.
 * Every entry point returns an isaacb_status; a failing call leaves a message
 * in isaacb_last_error().  No call aborts, traps or exits.
 *
 * The reference is a header-only C++ template library; its per-frame entry
 * is IsaacVisualization::doVisualization (lib/isaac.hpp:1298-2104) with the
 * draw callback drawCallBack (lib/isaac.hpp:2140-2543).  Each function below
 * names the reference interface it replaces.
 *
 * Source indices are "combined" indices as in the reference
 * (lib/isaac.hpp:720-731): volume sources first, then particle sources.
 * Field sources (advected vector fields, lib/isaac/isaac_common_kernel.hpp:500-550)
 * are not part of this library.
 */
#ifndef ISAAC_B200_H
#define ISAAC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ISAACB_MAX_SOURCES 16 /* ISAAC_MAX_SOURCES, lib/isaac/isaac_defines.hpp:36-38 */
#define ISAACB_MAX_FUNCTORS 3 /* ISAAC_MAX_FUNCTORS, lib/isaac/isaac_defines.hpp:27-29 */
#define ISAACB_MAX_CLIPPING 16 /* ISAAC_MAX_CLIPPING, lib/isaac/isaac_defines.hpp:44-46 */

typedef enum isaacb_status
{
    ISAACB_OK = 0,
    ISAACB_INVALID_ARG = 1,
    ISAACB_PARSE_ERROR = 2, /* functor chain had an error code; the parsed prefix is applied */
    ISAACB_CUDA_ERROR = 3,
    ISAACB_TIMEOUT = 4,
    ISAACB_OOM = 5,
    ISAACB_NOT_READY = 6 /* a required input (source pointer, camera) was never set */
} isaacb_status;

typedef enum isaacb_dtype
{
    ISAACB_F32 = 0,
    ISAACB_BF16 = 1,
    ISAACB_F16 = 2
} isaacb_dtype;

typedef enum isaacb_renderer
{
    /* pre-classified RGBA8 volume + iso textures, the reference default
     * (ISAAC_RENDERER_OPTIMIZED, lib/ISAACConfig.cmake:50-53) */
    ISAACB_RENDERER_COMBINED = 0,
    /* per-source sampling, functor chain and transfer function at every sample
     * (ISAAC_RENDERER_LEGACY, lib/isaac/isaac_volume_kernel.hpp:91-632) */
    ISAACB_RENDERER_PER_SOURCE = 1
} isaacb_renderer;

/* Geometry and source layout.  Mirrors the IsaacVisualization constructor
 * arguments (lib/isaac.hpp:565-583) minus the alpaka/stream/server arguments. */
typedef struct isaacb_desc
{
    uint32_t framebuffer[2]; /* width, height */
    uint32_t global_size[3];
    uint32_t local_size[3];
    uint32_t local_particle_size[3];
    int32_t position[3];
    float scale[3];
    uint32_t transfer_size; /* T_transferSize, 1024 in the reference example */
    uint32_t n_volume_sources;
    uint32_t n_particle_sources;
    uint32_t feature_dim[ISAACB_MAX_SOURCES]; /* 1..4 */
    uint32_t persistent[ISAACB_MAX_SOURCES]; /* T_Source::persistent */
    uint32_t guard_size[ISAACB_MAX_SOURCES]; /* T_Source::guardSize; must be 0 */
} isaacb_desc;

typedef struct isaacb_ctx isaacb_ctx;

/* Constructor + init (lib/isaac.hpp:565-945): allocates textures, transfer
 * tables and G-buffer; sets the reference defaults (step 0.5, weight 2,
 * chain "idem", hue-ramp transfer functions, dither mode 1, render mode 0,
 * AO off with weight 0.5, nearest filtering). */
isaacb_status isaacb_create(const isaacb_desc* desc, isaacb_ctx** out);
/* Destructor (lib/isaac.hpp ~IsaacVisualization). */
isaacb_status isaacb_destroy(isaacb_ctx* ctx);
/* Last error message of this context (or of the last failed create if ctx is NULL). */
const char* isaacb_last_error(const isaacb_ctx* ctx);

/* Volume source memory: `dev` points to (local+2*guard)^3 voxels, x fastest,
 * feature_dim floats per voxel -- what the reference reads through
 * T_Source::operator[] (example/example.cpp:66-71).  The pointer is borrowed. */
isaacb_status isaacb_set_source(isaacb_ctx* ctx, uint32_t src, const float* dev);

/* Particle source as a cell list -- what the reference reads through
 * T_ParticleSource::getIterator(cell) (example/example.cpp:148-228):
 * cell_offsets[ncells+1] (cell = x + y*PX + z*PX*PY), positions relative to the
 * cell in [0,1)^3 (3 floats), feature_dim attribute floats, per-particle radius
 * (or NULL to use const_radius).  All device pointers, borrowed. */
isaacb_status isaacb_set_particles(
    isaacb_ctx* ctx,
    uint32_t src,
    const uint32_t* cell_offsets,
    const float* positions,
    const float* attributes,
    const float* radii,
    float const_radius);

/* Functor chain (lib/isaac.hpp:1079-1241): same grammar ("op(p0,..)|op|op"),
 * pool order idem, add, mul, length, pow, sum, and error codes
 * (1 too many functors, -1 missing ')', 2 more than 4 parameters,
 * -2 bad number or unknown functor).  As in the reference the parsed prefix
 * is applied even when error_code != 0; the call then returns PARSE_ERROR. */
isaacb_status isaacb_set_functions(isaacb_ctx* ctx, uint32_t src, const char* chain, int32_t* error_code);
/* Pure host parser of one chain string (no context, no GPU). */
isaacb_status isaacb_parse_chain(
    const char* chain,
    int32_t bytecode[ISAACB_MAX_FUNCTORS],
    float params[4 * ISAACB_MAX_FUNCTORS],
    int32_t* error_code);

/* Transfer function control points (lib/isaac.hpp:1591-1612) and table
 * rebuild (updateTransfer, lib/isaac.hpp:1244-1266).  keys ascending or not;
 * a repeated key keeps its first value. */
isaacb_status isaacb_set_transfer(
    isaacb_ctx* ctx,
    uint32_t src,
    uint32_t n_points,
    const uint32_t* keys,
    const float* rgba);
/* Host copy of a source's transfer table (transfer_size x float4). */
isaacb_status isaacb_get_transfer(isaacb_ctx* ctx, uint32_t src, float* lut_rgba);

/* Steering setters: "weight" (lib/isaac.hpp:1700-1706), "iso threshold"
 * (:1684-1690), "step" (:1626-1635, raised to 0.01), "interpolation"
 * (:1613-1618), "render optimization" (:1619-1625), "ao" (:1768-1778),
 * "render mode" (:1780-1786), "dither mode" (:1788-1795; 0 round, 1 ordered 4^3, 2 / 3 / >= 4 blue noise 4^3 / 8^3 / 16^3). */
isaacb_status isaacb_set_weight(isaacb_ctx* ctx, uint32_t src, float weight);
isaacb_status isaacb_set_iso_threshold(isaacb_ctx* ctx, uint32_t src, float iso);
isaacb_status isaacb_set_step(isaacb_ctx* ctx, float step);
isaacb_status isaacb_set_interpolation(isaacb_ctx* ctx, int32_t enabled);
isaacb_status isaacb_set_renderer(isaacb_ctx* ctx, int32_t renderer);
isaacb_status isaacb_set_ao(isaacb_ctx* ctx, int32_t enabled, float weight, int32_t filter);
/* SSAO tap pattern (no reference counterpart; the reference always tests the 7x7
 * grid of taps 10 px apart, lib/isaac/isaac_ssao_kernel.hpp:38-184).  samples = 0
 * restores that grid.  1..32 samples on a golden-angle spiral filling a disc of
 * `radius` pixels (1..127), rounded to whole pixels; a tap occludes when its depth
 * is below the pixel's, and ao = clamp(occluded / (samples * 42/48), 0, 1), the
 * grid's normalisation per tap.  isaacb_get_ao_pattern returns the count and the
 * (x, y) offsets (2 * samples ints). */
isaacb_status isaacb_set_ao_pattern(isaacb_ctx* ctx, uint32_t samples, float radius);
isaacb_status isaacb_get_ao_pattern(isaacb_ctx* ctx, uint32_t* samples, int32_t* offsets);
isaacb_status isaacb_set_render_mode(isaacb_ctx* ctx, int32_t mode);
isaacb_status isaacb_set_dither_mode(isaacb_ctx* ctx, int32_t mode);
/* Storage type of the per-source renderer's bricks (no reference counterpart;
 * FP32 is the reference behaviour). */
isaacb_status isaacb_set_storage(isaacb_ctx* ctx, uint32_t src, int32_t dtype);
/* Slot order inside the combined texture's bricks (no reference counterpart; it
 * changes speed only, never a texel or a pixel).  -1 (default): chosen by each merge
 * from its camera for textures larger than 4x the L2 cache, x fastest otherwise;
 * 0: x fastest; 1: y fastest.  Takes effect at the next update. */
isaacb_status isaacb_set_slot_order(isaacb_ctx* ctx, int32_t order);
/* Background colour as handed to the draw callback (lib/isaac.hpp:2245-2249
 * swizzles it to (a,b,g,r) with alpha 0 for the G-buffer clear). */
isaacb_status isaacb_set_background(isaacb_ctx* ctx, const float rgba[4]);

/* Clipping planes: addClipping / editClipping / removeClipping
 * (lib/isaac.hpp:956-1015).  INVALID_ARG where the reference returns false. */
isaacb_status isaacb_add_clipping(isaacb_ctx* ctx, const float position[3], const float normal[3]);
isaacb_status isaacb_edit_clipping(isaacb_ctx* ctx, uint32_t nr, const float position[3], const float normal[3]);
isaacb_status isaacb_remove_clipping(isaacb_ctx* ctx, uint32_t nr);

/* Camera: projection and modelview matrices, column major (the doubles IceT
 * passes to drawCallBack, lib/isaac.hpp:2140-2178).  The inverse of P*MV is
 * formed in FP32 exactly as the reference does. */
isaacb_status isaacb_set_camera(isaacb_ctx* ctx, const double projection[16], const double modelview[16]);

/* Buffer update of doVisualization (lib/isaac.hpp:1805-1947): per-source
 * textures of non-persistent sources and the merge into the combined RGBA8
 * volume and iso textures.  Asynchronous on `stream`. */
isaacb_status isaacb_update(isaacb_ctx* ctx, void* stream);

/* drawCallBack (lib/isaac.hpp:2140-2543): clear, particles, iso, SSAO,
 * shading, volume.  The frame stays in the context's device framebuffer;
 * if rgba_dev is not NULL it is also copied there.  Asynchronous. */
isaacb_status isaacb_render(isaacb_ctx* ctx, void* stream, uint8_t* rgba_dev);

/* One whole doVisualization frame with a host result: update, render and the
 * device-to-host framebuffer copy (lib/isaac.hpp:2532-2542) into rgba_host
 * (W*H*4 bytes, row 0 = bottom).  Synchronous on `stream`. */
isaacb_status isaacb_frame(isaacb_ctx* ctx, void* stream, uint8_t* rgba_host);

/* Device pointer of the context's RGBA8 framebuffer. */
isaacb_status isaacb_framebuffer(isaacb_ctx* ctx, uint8_t** rgba_dev);

/* Min/max of every source after its functor chain ("minmax" request,
 * lib/isaac.hpp:1951-2006 with MinMaxKernel/MinMaxParticleKernel,
 * lib/isaac/isaac_min_max_kernel.hpp:22-97).  Results are bit-identical to
 * the reference's column scan.  mn/mx are host arrays of n_sources floats.
 * Synchronous on `stream`. */
isaacb_status isaacb_minmax(isaacb_ctx* ctx, void* stream, float* mn, float* mx);

/* Diagnostics used by the parity tests.  Synchronous on `stream`. */
/* G-buffer readback: depth (W*H), normal (W*H*3), ao (W*H); any may be NULL. */
isaacb_status isaacb_get_gbuffer(isaacb_ctx* ctx, void* stream, float* depth, float* normal, float* ao);
/* Combined textures in reference layout (local size, x fastest, RGBA8); either may be NULL. */
isaacb_status isaacb_get_combined(isaacb_ctx* ctx, void* stream, uint8_t* volume, uint8_t* iso);
/* Enable per-frame counting of executed ray-march iterations (the reference's
 * loop trips, including those empty-space skipping jumps over). */
isaacb_status isaacb_set_counting(isaacb_ctx* ctx, int32_t enabled);
/* Counters of the last rendered frame.  Synchronous on `stream`. */
isaacb_status isaacb_get_counters(isaacb_ctx* ctx, void* stream, uint64_t* volume_samples, uint64_t* iso_samples);
/* Per-kernel timing with CUDA events recorded on the launch stream around
 * every kernel of isaacb_update / isaacb_render (off by default).
 * isaacb_get_timing returns, for the last update+render, the milliseconds of
 * ISAACB_TIMING_SLOTS phases in this order: merge (or per-source bricks),
 * clear+particles, iso, ssao, shade+volume; a phase that did not run is 0.
 * Synchronous on `stream`. */
#define ISAACB_TIMING_SLOTS 5
isaacb_status isaacb_set_timing(isaacb_ctx* ctx, int32_t enabled);
isaacb_status isaacb_get_timing(isaacb_ctx* ctx, void* stream, float ms[ISAACB_TIMING_SLOTS]);

/* Min/max of one volume source after a functor chain, allocating nothing.
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc -- e.g. a simulation that reserves nearly all device memory for
 * its own heap, or a loop that must not take cudaMalloc's implicit device
 * synchronisation.  It needs no context.  `src` is the source (size[0]*size[1]*size[2]
 * voxels, x fastest, feature_dim floats each), bytecode/params come from
 * isaacb_parse_chain, `result` is 2 device floats (min, max), bit-identical to
 * isaacb_minmax.  Scratch is one static device array of 2 MiB per GPU: sources
 * with more than 262144 (x,y) columns or more than 2^20 z planes are rejected
 * (INVALID_ARG).  Every call looks the array's address up in the current
 * context (nothing is cached across device resets); the first call in a
 * context should precede any stream capture.  Calls that overlap on the GPU
 * race on the shared array.
 * Asynchronous on `stream`; errors via isaacb_last_error(NULL). */
isaacb_status isaacb_minmax_noalloc(
    const float* src,
    const uint32_t size[3],
    uint32_t feature_dim,
    const int32_t bytecode[ISAACB_MAX_FUNCTORS],
    const float params[4 * ISAACB_MAX_FUNCTORS],
    float* result,
    void* stream);

/* ---- Batched views (no counterpart in the reference, which draws one view per
 * doVisualization).  A batch renders many views of one or more contexts -- e.g.
 * the timesteps of a simulation, each its own context -- in ONE persistent
 * launch whose CTAs take 256-pixel tiles from a work queue.  Views draw the
 * combined volume exactly as isaacb_render does for a context without particle
 * sources, iso thresholds or SSAO (those contexts are rejected). */
typedef struct isaacb_view
{
    uint32_t ctx_index; /* index into the batch's context array */
    uint32_t width, height;
    uint32_t reserved;
    double projection[16]; /* column major, as isaacb_set_camera */
    double modelview[16];
    uint8_t* rgba_dev; /* width*height*4 bytes of device memory */
} isaacb_view;

typedef struct isaacb_batch_config
{
    uint32_t tile_w, tile_h; /* tile_w*tile_h == 256, tile_w % 8 == 0, tile_h % 4 == 0 */
    uint32_t blocks_per_sm; /* 0 = as many as fit */
    int32_t skip_empty; /* 1 check per-brick emptiness, 0 never, -1 when the context's last merge found empty bricks (default) */
} isaacb_batch_config;

typedef struct isaacb_batch isaacb_batch;

isaacb_status isaacb_batch_create(
    isaacb_ctx* const* ctxs,
    uint32_t n_ctx,
    const isaacb_view* views,
    uint32_t n_views,
    isaacb_batch** out);
isaacb_status isaacb_batch_destroy(isaacb_batch* batch);
isaacb_status isaacb_batch_set_config(isaacb_batch* batch, const isaacb_batch_config* cfg);
isaacb_status isaacb_batch_get_config(const isaacb_batch* batch, isaacb_batch_config* cfg);
/* New camera of one view; takes effect at the next render or graph launch. */
isaacb_status isaacb_batch_set_camera(isaacb_batch* batch, uint32_t view, const double projection[16], const double modelview[16]);
/* One batch frame on `stream`: with `update`, the merge of every context first
 * (isaacb_update), then the persistent launch over all views.  Asynchronous. */
isaacb_status isaacb_batch_render(isaacb_batch* batch, void* stream, int32_t update);
/* Capture the same work (merges when `update`, queue reset, persistent launch)
 * into a CUDA graph; isaacb_batch_launch_graph replays it.  `stream` must not be
 * the legacy default stream.  Cameras, transfer tables and shading settings
 * are read at every launch; when a context's merge inputs (functors, weights,
 * storage, source memory) changed since the capture, the next launch
 * recaptures. */
isaacb_status isaacb_batch_capture(isaacb_batch* batch, void* stream, int32_t update);
isaacb_status isaacb_batch_launch_graph(isaacb_batch* batch, void* stream);
/* Time every tile shape x occupancy x skipping candidate on the current views
 * (CUDA events, a few launches each), keep the fastest, return it and its time.
 * Synchronous on `stream`. */
isaacb_status isaacb_batch_autotune(isaacb_batch* batch, void* stream, isaacb_batch_config* best, float* best_ms);
/* Ray-march loop trips of the last batch render (counting costs one atomic per warp). */
isaacb_status isaacb_batch_set_counting(isaacb_batch* batch, int32_t enabled);
isaacb_status isaacb_batch_get_samples(isaacb_batch* batch, void* stream, uint64_t* samples);
/* Kernels the last isaacb_batch_render or isaacb_batch_capture enqueued (a graph
 * launch replays the captured ones). */
isaacb_status isaacb_batch_get_launch_count(isaacb_batch* batch, uint32_t* launches);

/* ---- Tensor-core convolution (no counterpart in the reference): the
 * building block of the learned frame reconstructor, exposed for testing.
 * Tensors are NHWC bf16 in device memory, channel counts multiples of 8.
 *
 * isaacb_conv_forward computes y[p][co] = sum_{tap,ci} x[in(p,tap)][ci] * w[co][tap*c_in+ci]
 * over the out_h x out_w grid, with in(p,tap) = p*stride - pad + tap per axis
 * (zero outside the in_h x in_w input), or, with `transposed`,
 * in(p,tap) = (p + pad - tap) / stride where that divides exactly (the
 * input-gradient form).  `w` is bf16 [roundup(c_out,16)][roundup(ksize^2*c_in,64)],
 * zero padded.  Epilogue, in order: + bias[co] (optional), ReLU (`relu`),
 * * (mask > 0) with `mask` NHWC like y (optional), + the existing output
 * (`accumulate`); stored as bf16 `y`, or FP32 `y_f32` when that is set.
 *
 * isaacb_conv_wgrad adds sum_p x[in(p,tap)][ci] * dy[p][co] into the FP32
 * matrix dw[(tap*c_in+ci)][roundup(c_out,16)] (forward gather form).
 *
 * `error_flag` (optional, device int) is set when a bounded wait inside the
 * kernel gave up.  Asynchronous on `stream`; errors via isaacb_last_error(NULL).
 *
 * `wait_check_us` (forward only; 0 for normal use) checks the failure path: the
 * kernel, before any copy or MMA, waits that many microseconds on an mbarrier
 * that nothing arrives at, sets error_flag, releases its TMEM and returns
 * without writing the output. */
typedef struct isaacb_conv_args
{
    const void* x;
    const void* w;
    const float* bias;
    void* y;
    float* y_f32;
    const void* mask;
    const void* dy;
    float* dw;
    int32_t* error_flag;
    uint32_t batch, in_h, in_w, c_in;
    uint32_t out_h, out_w, c_out;
    uint32_t ksize, stride, pad;
    int32_t transposed, relu, accumulate;
    uint32_t wait_check_us;
} isaacb_conv_args;

isaacb_status isaacb_conv_forward(const isaacb_conv_args* args, void* stream);
/* Input staging of the row-tile convolutions (stride 1, or stride 2 forward): 1 (the
 * default) loads each run of the input rows with one tiled TMA copy where the input
 * allows it (16-byte aligned, an even width for stride 2), 0 gathers it with cp.async
 * in four producer warps.  The results are identical; process-wide setting. */
isaacb_status isaacb_conv_set_producer(int32_t tma);
isaacb_status isaacb_conv_wgrad(const isaacb_conv_args* args, void* stream);

/* ---- Learned frame reconstructor (no counterpart in the reference).  A
 * 4-level convolutional U-Net (32/64/96/128 channels, 216,464 parameters, bf16
 * weights, FP32 accumulation on the tensor cores) rebuilds a full-size RGBA8
 * frame from a half-size render: frame = bilinear x2 of the half-size frame
 * + the network's residual.  Frames are RGBA8 rows, row 0 = bottom, in device
 * memory.  Training and inference run on the GPU in the library's own
 * forward and backward kernels. */
typedef struct isaacb_recon isaacb_recon;

uint32_t isaacb_recon_param_count(void);
/* Buffers for up to `max_batch` half-size inputs of max_h x max_w; weights
 * He-initialised from `seed`. */
isaacb_status isaacb_recon_create(uint32_t max_batch, uint32_t max_h, uint32_t max_w, uint64_t seed, isaacb_recon** out);
isaacb_status isaacb_recon_destroy(isaacb_recon* recon);
/* FP32 parameters, per layer the weights [c_out][ky][kx][c_in] then the bias. */
isaacb_status isaacb_recon_get_params(isaacb_recon* recon, float* host);
isaacb_status isaacb_recon_set_params(isaacb_recon* recon, const float* host);
/* One optimiser step on `batch` pairs: half-size frames low[index[b]]
 * (h x w) against full-size targets high[index[b]] (2h x 2w); index may be
 * NULL for 0..batch-1.  The mean squared error (RGBA in [0,1]) is written to
 * loss_dev when it is set.  With grads_host set, the step computes the
 * gradient, copies it there (layout of the parameters) and does NOT update. */
isaacb_status isaacb_recon_train_step(
    isaacb_recon* recon,
    const uint8_t* low,
    const uint8_t* high,
    const int32_t* index,
    uint32_t batch,
    uint32_t h,
    uint32_t w,
    float learning_rate,
    float* loss_dev,
    float* grads_host,
    void* stream);
/* One full-size frame (2h x 2w) from one half-size frame (h x w). */
isaacb_status isaacb_recon_infer(isaacb_recon* recon, const uint8_t* low, uint32_t h, uint32_t w, uint8_t* out, void* stream);
/* Reads and clears the flag the kernels raise when a bounded wait gave up. */
isaacb_status isaacb_recon_error(isaacb_recon* recon, int32_t* flag);
/* Checks the failure path: the first convolution of the next inference or
 * training step runs the wait check of isaacb_conv_args.wait_check_us with this
 * budget (microseconds, > 0), so that step raises the flag isaacb_recon_error
 * reads and its output is not meaningful; later calls run normally. */
isaacb_status isaacb_recon_arm_wait_check(isaacb_recon* recon, uint32_t budget_us);
/* The method without the network: bilinear x2 alone (2h x 2w RGBA8). */
isaacb_status isaacb_upsample_bilinear2(const uint8_t* low, uint32_t h, uint32_t w, uint8_t* out, void* stream);
/* Adds the sum of squared byte differences of two RGBA8 images to *sum_dev. */
isaacb_status isaacb_image_sq_error(const uint8_t* a, const uint8_t* b, uint64_t bytes, unsigned long long* sum_dev, void* stream);

/* ---- Field sources and advection (lib/isaac.hpp:292-370, 499-562, 1819-1850;
 * lib/isaac/isaac_common_kernel.hpp:334-430, 500-550, 618-686).  The reference
 * keeps vector fields in a separate source list, merged after the volume sources;
 * here they are the LAST volume sources (feature_dim 3), flagged with
 * isaacb_set_field_source.  Each update then swaps the field's two advection
 * textures, counts the step, advects the texture along the field (noise blended in
 * by the seeding period / duration) and the merge multiplies the field source's
 * alpha by the advection texture / 255.  The reference leaves the advection
 * textures uninitialised; here they start at zero.  Combined renderer only. */
isaacb_status isaacb_set_field_source(isaacb_ctx* ctx, uint32_t source, int32_t enabled);
/* "advection step" (factor of the 3-cell maximum step), "advection weight"
 * (history weight), "advection seeding period", "advection seeding duration",
 * "seed points" (isaac.hpp:1636-1662); defaults 1, 0.95, 1, 1, 1000. */
isaacb_status isaacb_set_advection(
    isaacb_ctx* ctx,
    float step_factor,
    float history_weight,
    int32_t seeding_period,
    int32_t seeding_duration,
    int32_t seed_points);
/* Read back the current advection texture of a field source (local size, x fastest)
 * and the noise texture (floats); synchronous on `stream`. */
isaacb_status isaacb_get_advection(isaacb_ctx* ctx, void* stream, uint32_t source, uint8_t* host);
isaacb_status isaacb_get_noise(isaacb_ctx* ctx, void* stream, float* host);

/* ---- Advection borders between ranks (the reference's guard exchange,
 * lib/isaac.hpp:1856-1913, and its advection textures' guard band,
 * lib/isaac.hpp:206-214).  Each field source's advection texture carries a guard
 * band of ceil((ISAAC_MAX_ADVECTION_STEP_SIZE + 1) / scale) voxels per axis
 * (isaacb_advection_guard); the advection step samples it, so a neighbour's
 * border values reach across the boundary.  A multi-rank caller runs, per frame:
 * isaacb_advect; per field source and per neighbour direction, isaacb_pack_guard
 * into a device buffer, the exchange with that neighbour, isaacb_unpack_guard
 * from the received buffer; then isaacb_update, which merges without advecting
 * again.  Directions are the reference's neighbour indices 1-26 (base-3 digits
 * x, y, z; digit 2 = -1; lib/isaac/isaac_types.hpp:133-161); a slab is
 * (|d| ? guard : local) voxels per axis, x fastest.  Pack and unpack follow the
 * reference's SyncToOwnGuard / SyncFromNeighbourGuard index arithmetic
 * (lib/isaac/isaac_common_kernel.hpp:454-498), including its placement of the
 * positive-side slabs one voxel lower.  Asynchronous on `stream`. */
isaacb_status isaacb_advect(isaacb_ctx* ctx, void* stream);
isaacb_status isaacb_advection_guard(const isaacb_ctx* ctx, uint32_t guard[3]);
isaacb_status isaacb_pack_guard(isaacb_ctx* ctx, uint32_t src, uint32_t direction, uint8_t* slab, void* stream);
isaacb_status isaacb_unpack_guard(isaacb_ctx* ctx, uint32_t src, uint32_t direction, const uint8_t* slab, void* stream);
/* the "advection border" key switched off: both advection textures of every field
 * source are cleared (lib/isaac.hpp:1668-1683) */
isaacb_status isaacb_clear_advection(isaacb_ctx* ctx, void* stream);

/* ---- Stereo compositing (lib/isaac/isaac_compositors.hpp:37-116, done on the GPU).
 * mode 0: out = left (width x height); mode 1: left and right side by side
 * (2*width x height); mode 2: per pixel (left & left_filter) | (right & right_filter)
 * on the 32-bit RGBA8 word (bytes R, G, B, A from the low end).  Device frames,
 * asynchronous on `stream`. */
isaacb_status isaacb_composite(
    int32_t mode,
    const uint8_t* left,
    const uint8_t* right,
    uint32_t width,
    uint32_t height,
    uint32_t left_filter,
    uint32_t right_filter,
    uint8_t* out,
    void* stream);

/* ---- Frame output (IsaacCommunicator::serverSendFrame and setJpegQuality,
 * lib/isaac/isaac_communicator.hpp:207-290).  An encoder turns a device RGBA8
 * frame (row 0 = bottom, sent first as the reference does) into the payload
 * message {"payload": "data:image/jpeg;base64,<text>"} (raw frames:
 * "data:image/raw-rgba;base64,"), or into the JPEG bytes alone.  The JPEG is
 * baseline, 2x2-subsampled chroma, standard Huffman tables, alpha dropped (the
 * reference's libjpeg settings); base64 as boost's base64_from_binary: ceil(8n/6)
 * characters, no '=' padding.  The returned pointers are pinned memory owned by
 * the encoder, valid until its next encode call; the calls synchronize `stream`. */
typedef struct isaacb_encoder isaacb_encoder;
isaacb_status isaacb_encoder_create(isaacb_encoder** out);
isaacb_status isaacb_encoder_destroy(isaacb_encoder* encoder);
/* quality > 100 is clamped to 100 (setJpegQuality); the default is 90 */
isaacb_status isaacb_encoder_set_quality(isaacb_encoder* encoder, uint32_t quality);
isaacb_status isaacb_encoder_get_quality(const isaacb_encoder* encoder, uint32_t* quality);
isaacb_status isaacb_encode_jpeg(
    isaacb_encoder* encoder,
    const uint8_t* rgba,
    uint32_t width,
    uint32_t height,
    void* stream,
    const uint8_t** jpeg,
    size_t* length);
/* jpeg = 0 sends the raw RGBA bytes (the reference built with ISAAC_JPEG off);
 * *length excludes the terminating NUL */
isaacb_status isaacb_encode_frame(
    isaacb_encoder* encoder,
    const uint8_t* rgba,
    uint32_t width,
    uint32_t height,
    int32_t jpeg,
    void* stream,
    const char** message,
    size_t* length);
/* base64 of n device bytes into ceil(8n/6) device characters (no terminator), asynchronous */
isaacb_status isaacb_base64(const uint8_t* in, size_t n, char* out, void* stream);

/* Sort-last compositing of several ranks' frames (IceT's ordered BLEND composite,
 * lib/isaac.hpp:820-826 and 2015-2055).  `images` are `count` (1-64) device RGBA8
 * buffers of `pixels` pixels each (whole frames, or the same stripe of every
 * frame); `order` lists the image indices front to back, as the reference's
 * icetCompositeOrder array does.  Each channel is folded front to back with the
 * premultiplied "under" operator in 8-bit integers,
 * acc += src * (255 - acc.alpha) / 255; `background` (4 bytes RGBA, host) goes under
 * the result when not null.  Asynchronous on `stream`. */
isaacb_status isaacb_blend_ordered(
    const uint8_t* const* images,
    uint32_t count,
    const int32_t* order,
    uint32_t pixels,
    const uint8_t* background,
    uint8_t* out,
    void* stream);

/* Number of kernels the last isaacb_update / isaacb_render enqueued. */
isaacb_status isaacb_get_launch_count(isaacb_ctx* ctx, uint32_t* update_launches, uint32_t* render_launches);

#ifdef __cplusplus
}
#endif

#endif /* ISAAC_B200_H */
