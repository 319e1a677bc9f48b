/*
 * vsfeel_bm3d.h -- C ABI of the B200-native BM3Dv2 basic estimate.
 *
 * The entry points mirror the VapourSynth filter that the reference
 * registers as core.vsfeel.BM3Dv2 (src/bm3d.cpp:1558-1574):
 *
 *   vsfeel_bm3d_create      <- BM3DCreate      src/bm3d.cpp:1043-1552
 *   vsfeel_bm3d_frame_range <- BM3DGetFrame, arInitial         :704-712
 *   vsfeel_bm3d_get_frame   <- BM3DGetFrame, arAllFramesReady  :713-1025
 *   vsfeel_bm3d_free        <- BM3DFree                        :1030-1037
 *
 * plus clip-level entry points (host or device buffers) that a batch caller
 * or the torch extension uses instead of per-frame callbacks.
 *
 * Conventions: pure C, no exceptions cross the boundary. Every function
 * returns 0 on success or a negative VSFEEL_E_* code; the message (prefixed
 * "BM3D: " like the reference's errors) is available from
 * vsfeel_bm3d_last_error() on the calling thread. A context is internally
 * synchronised: calls from several threads are serialised (get_frame calls
 * only while they enqueue their work). Strides are in
 * bytes for host buffers and in elements (floats) for device buffers.
 */
#ifndef VSFEEL_BM3D_H
#define VSFEEL_BM3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VSFEEL_BM3D_ABI_VERSION 3

#if defined(__GNUC__)
#define VSFEEL_API __attribute__((visibility("default")))
#else
#define VSFEEL_API
#endif

enum {
    VSFEEL_OK = 0,
    VSFEEL_E_ARG = -1,      /* invalid argument (message names it)          */
    VSFEEL_E_FORMAT = -2,   /* unsupported clip format                      */
    VSFEEL_E_CUDA = -3,     /* CUDA runtime error                           */
    VSFEEL_E_MEMORY = -4,   /* device or pinned allocation failed           */
    VSFEEL_E_TIMEOUT = -5,  /* a bounded wait on the GPU expired            */
    VSFEEL_E_FETCH = -6,    /* the frame callback returned no frame         */
    VSFEEL_E_UNSUPPORTED = -7
};

/* Clip format, mirroring the VSVideoFormat fields the reference checks
 * (src/bm3d.cpp:1085-1088, 1257-1275). */
enum { VSFEEL_CF_GRAY = 1, VSFEEL_CF_YUV = 3 };
enum { VSFEEL_ST_INTEGER = 0, VSFEEL_ST_FLOAT = 1 };

typedef struct vsfeel_bm3d_video_info {
    int width, height, num_frames;
    int color_family;     /* VSFEEL_CF_GRAY or VSFEEL_CF_YUV             */
    int sample_type;      /* VSFEEL_ST_FLOAT                              */
    int bits_per_sample;  /* 32                                           */
    int sub_sampling_w, sub_sampling_h;
} vsfeel_bm3d_video_info;

/* The BM3Dv2 argument map (registration string at src/bm3d.cpp:1562-1571).
 * An array argument with count 0 is absent and takes the reference default;
 * a missing element copies the previous one (src/bm3d.cpp:1090-1167).
 * Only element [0] of each array is used, as in the reference, except by
 * vsfeel_bm3d_create_plane for planes 1 and 2. */
typedef struct vsfeel_bm3d_args {
    float sigma[3];      int sigma_count;       /* default 3.0  */
    int block_step[3];   int block_step_count;  /* default 8    */
    int bm_range[3];     int bm_range_count;    /* default 9    */
    int radius;          int radius_set;        /* default 0    */
    int ps_num[3];       int ps_num_count;      /* default 2    */
    int ps_range[3];     int ps_range_count;    /* default 4    */
    int num_streams;     int num_streams_set;   /* default 4    */
    int extractor_exp;   int extractor_exp_set; /* default 0    */
    int has_ref;         /* a "ref" clip was given (final Wiener pass)     */
    const vsfeel_bm3d_video_info* ref_info;  /* its format, when has_ref */
} vsfeel_bm3d_args;

typedef struct vsfeel_bm3d vsfeel_bm3d;

/* Fills args with "all arguments absent". */
VSFEEL_API void vsfeel_bm3d_args_init(vsfeel_bm3d_args* args);

/* BM3DCreate: validates the arguments exactly as the reference does and
 * binds a CUDA device context (device ordinal `device`, normally 0). */
VSFEEL_API int vsfeel_bm3d_create(const vsfeel_bm3d_args* args, const vsfeel_bm3d_video_info* vi,
                       int device, vsfeel_bm3d** out);

/* Per-plane denoising, an extension past the reference: the reference parses
 * sigma, block_step, bm_range, ps_num and ps_range per plane but applies
 * element [0] to luma and passes chroma through (src/bm3d.cpp:1090-1167,
 * 1265-1272). vsfeel_bm3d_create_plane binds a context to plane `plane`
 * (0 = luma; 1, 2 = the chroma planes of a YUV clip, of size
 * (width >> sub_sampling_w) x (height >> sub_sampling_h)) with element
 * [plane] of every array, filled by the reference's rule. Every other entry
 * point then works on that plane: the fetch callbacks and the host or device
 * buffers hold plane `plane` of each frame. In the final pass, ref supplies
 * the same plane. vsfeel_bm3d_create is vsfeel_bm3d_create_plane(.., 0, ..).
 * Planes narrower or shorter than 8 are rejected. */
VSFEEL_API int vsfeel_bm3d_create_plane(const vsfeel_bm3d_args* args, const vsfeel_bm3d_video_info* vi,
                             int plane, int device, vsfeel_bm3d** out);

/* The effective parameters (vsfeel_bm3d_info, device_bytes 0) that
 * vsfeel_bm3d_create_plane would use for `plane`, after the same validation;
 * no device is touched. */
struct vsfeel_bm3d_info;
VSFEEL_API int vsfeel_bm3d_plane_params(const vsfeel_bm3d_args* args, const vsfeel_bm3d_video_info* vi,
                             int plane, struct vsfeel_bm3d_info* info);

/* BM3DFree. Accepts NULL. */
VSFEEL_API void vsfeel_bm3d_free(vsfeel_bm3d* ctx);

/* arInitial: the source frames output n needs, [*first, *last]
 * (n - 2r .. n + 2r clamped to the clip). */
VSFEEL_API int vsfeel_bm3d_frame_range(const vsfeel_bm3d* ctx, int n, int* first, int* last);

/* Frame source for vsfeel_bm3d_get_frame: returns the luma plane of frame
 * n with its row stride in bytes, or NULL on failure; the pointer stays
 * valid until release(user, n) is called. */
typedef const float* (*vsfeel_fetch_fn)(void* user, int n, ptrdiff_t* stride_bytes);
typedef void (*vsfeel_release_fn)(void* user, int n);

/* arAllFramesReady: denoises output frame n into dst (luma plane). Frames
 * are fetched through the callbacks only when not already resident (the
 * frames of frame_range(n) only), and computed stacks are cached, so
 * requests in or near order compute each stack once. Calls from several
 * threads may overlap: a call holds the context while it enqueues its work
 * and waits for its own output without it. A frame is released once the
 * library no longer reads it; if a bounded wait for its upload runs out
 * (VSFEEL_E_TIMEOUT) the frame is not released, since the copy may still
 * read it, and stays the caller's to release after vsfeel_bm3d_free. */
VSFEEL_API int vsfeel_bm3d_get_frame(vsfeel_bm3d* ctx, int n, vsfeel_fetch_fn fetch,
                          vsfeel_release_fn release, void* user, float* dst,
                          ptrdiff_t dst_stride_bytes);

/* The final (Wiener) pass, for a context created with a "ref" clip (the
 * basic estimate): block matching runs on ref, ref's groups give the Wiener
 * coefficients, and src is the clip denoised (src/bm3d.comp:73-81,
 * 401-443). The plain entry points reject such a context and the *_ref ones
 * reject the others. For get_frame_ref, fetch(user, clip, n, stride) returns
 * frame n of the source (clip 0) or of ref (clip 1), and release(user, clip,
 * n) hands it back. */
typedef const float* (*vsfeel_fetch2_fn)(void* user, int clip, int n, ptrdiff_t* stride_bytes);
typedef void (*vsfeel_release2_fn)(void* user, int clip, int n);

VSFEEL_API int vsfeel_bm3d_get_frame_ref(vsfeel_bm3d* ctx, int n, vsfeel_fetch2_fn fetch,
                                         vsfeel_release2_fn release, void* user, float* dst,
                                         ptrdiff_t dst_stride_bytes);

/* Whole clip from host memory: src holds all num_frames luma planes
 * (frame f at src + f*frame_stride_bytes, rows row_stride_bytes apart);
 * writes output frames first .. first+count-1 to dst (same layout, frame 0
 * of dst = output `first`). Pinned host buffers give the fastest copies.
 * A VSFEEL_E_TIMEOUT return leaves copies from src and into dst queued or
 * running: both buffers stay in use until a later call on the same context
 * returns VSFEEL_OK (it runs after all earlier work) or vsfeel_bm3d_free
 * returns, and must not be freed or reused before then. */
VSFEEL_API int vsfeel_bm3d_process_host(vsfeel_bm3d* ctx, const float* src, ptrdiff_t src_frame_stride_bytes,
                             ptrdiff_t src_row_stride_bytes, float* dst,
                             ptrdiff_t dst_frame_stride_bytes, ptrdiff_t dst_row_stride_bytes,
                             int first, int count);

/* process_host for the final pass: ref holds the basic estimate's luma
 * planes in the same form as src. */
VSFEEL_API int vsfeel_bm3d_process_host_ref(vsfeel_bm3d* ctx, const float* src,
                                            ptrdiff_t src_frame_stride_bytes,
                                            ptrdiff_t src_row_stride_bytes, const float* ref,
                                            ptrdiff_t ref_frame_stride_bytes,
                                            ptrdiff_t ref_row_stride_bytes, float* dst,
                                            ptrdiff_t dst_frame_stride_bytes,
                                            ptrdiff_t dst_row_stride_bytes, int first, int count);

/* Whole clip already in device memory (strides in floats), enqueued on
 * `stream` (a cudaStream_t, used as given: NULL is the default stream).
 * Returns after the work is enqueued; synchronise the stream before reading
 * dst, and keep src and dst alive until then. */
VSFEEL_API int vsfeel_bm3d_process_device(vsfeel_bm3d* ctx, const float* src, int64_t src_frame_stride,
                               int64_t src_row_stride, float* dst, int64_t dst_frame_stride,
                               int64_t dst_row_stride, int first, int count, void* stream);

/* process_device for the final pass: ref's rows must have src's stride. */
VSFEEL_API int vsfeel_bm3d_process_device_ref(vsfeel_bm3d* ctx, const float* src,
                                              int64_t src_frame_stride, int64_t src_row_stride,
                                              const float* ref, int64_t ref_frame_stride,
                                              int64_t ref_row_stride, float* dst,
                                              int64_t dst_frame_stride, int64_t dst_row_stride,
                                              int first, int count, void* stream);

/* Effective parameters after defaults and scaling (for callers and tests). */
typedef struct vsfeel_bm3d_info {
    int width, height, num_frames, radius, block_step, bm_range, ps_num, ps_range, num_streams;
    float sigma;      /* user sigma[0]                                    */
    float threshold;  /* SIGMA_Y: sigma * 0x3f021bb6, or * 0x3e40c0c1 in the
                         final pass (src/bm3d.cpp:1103-1113)              */
    float extractor;  /* 2^extractor_exp, or 0 (src/bm3d.cpp:1188-1190)   */
    int blocks_x, blocks_y;
    int64_t device_bytes;  /* device memory held by the context           */
    int match_tile_shape;  /* VSFEEL_TILE_* the matcher's table launches use
                              (the autotuner's choice once it has run, the
                              largest shape that fits before), or -1: the
                              direct-read matcher                         */
    int match_lanes;       /* lanes per block of the sliding matcher, 8 or 16 */
    int autotuned;         /* 1 once the plain path's autotuner has timed the
                              shapes (0 while untuned, with VSFEEL_AUTOTUNE=0,
                              radius >= 3 or the final pass)                */
} vsfeel_bm3d_info;

VSFEEL_API int vsfeel_bm3d_get_info(const vsfeel_bm3d* ctx, vsfeel_bm3d_info* info);

/* Match table of stack m (testing and the adjoint): table receives
 * blocks_x*blocks_y*8 entries of (x, y, z) int32 triples, blocks in raster
 * order, computed from the device frames given as in process_device. */
VSFEEL_API int vsfeel_bm3d_match_table_device(vsfeel_bm3d* ctx, const float* src, int64_t src_frame_stride,
                                   int64_t src_row_stride, int m, int32_t* table_host);

/* Kernel launches issued by this context since creation (all kernels). */
VSFEEL_API int64_t vsfeel_bm3d_launch_count(const vsfeel_bm3d* ctx);

/* Per-kernel GPU timing with CUDA events on the launch stream (the
 * reference's BM3D_GPUTRACE, src/bm3d.cpp:978-994). enable != 0 starts (and
 * resets) the trace, 0 stops it. */
enum { VSFEEL_KERNEL_MATCH = 0, VSFEEL_KERNEL_FILTER = 1, VSFEEL_KERNEL_NORMALIZE = 2,
       VSFEEL_KERNEL_ADJOINT = 3, VSFEEL_KERNEL_KINDS = 4 };
VSFEEL_API int vsfeel_bm3d_trace(vsfeel_bm3d* ctx, int enable);

/* Waits for the traced work, then returns per kernel kind the summed device
 * milliseconds and the number of traced launches. */
VSFEEL_API int vsfeel_bm3d_trace_read(vsfeel_bm3d* ctx, double ms[VSFEEL_KERNEL_KINDS],
                                      int64_t launches[VSFEEL_KERNEL_KINDS]);

/* ---- Differentiable form (no counterpart in the reference) --------------
 *
 * The forward pass of a whole clip that also records what its adjoint needs,
 * and the adjoint: dLoss/dInput from dLoss/dOutput with the match table, the
 * threshold keep masks and the aggregation weights frozen at the forward
 * pass. With those frozen the denoiser is linear in its input, and the
 * adjoint applies the transpose of that linear map (the 3D spectra are
 * recomputed from the saved match table, not stored). The extractor's
 * rounding of the scattered values (extractor_exp != 0) is taken as the
 * identity. Both calls cover the whole clip (outputs 0 .. num_frames-1) with
 * device buffers (strides in floats) and only enqueue work on `stream`.
 *
 * The saved state is one caller-owned device buffer of `bytes`, 256-byte
 * aligned: for each stack m a record at m * stack_bytes holding
 *   match_xy_offset: [num_blocks][8] uint32, x | y << 16 of each match
 *   match_z_offset:  [num_blocks] uint32, 4 bits per match: its slice z
 *   mask_offset:     [num_blocks][8] uint64; word h, bit 8*g + v is set
 *                    when the 3D coefficient of group frequency g, vertical
 *                    frequency v and horizontal frequency h was kept
 * then, at den_offset, the frozen denominators: float planes of output n at
 * n * den_frame_stride floats, rows den_row_stride floats apart. Blocks are
 * in raster order of the block grid. */
typedef struct vsfeel_bm3d_saved_info {
    int64_t bytes, stack_bytes;
    int64_t match_xy_offset, match_z_offset, mask_offset;
    int64_t den_offset, den_row_stride, den_frame_stride;
    int64_t num_blocks;
} vsfeel_bm3d_saved_info;

VSFEEL_API int vsfeel_bm3d_saved_layout(const vsfeel_bm3d* ctx, vsfeel_bm3d_saved_info* out);

/* Denoises every frame of the clip like process_device and writes the saved
 * state into `saved` (vsfeel_bm3d_saved_layout().bytes). */
VSFEEL_API int vsfeel_bm3d_forward_saved(vsfeel_bm3d* ctx, const float* src, int64_t src_frame_stride,
                                         int64_t src_row_stride, float* dst,
                                         int64_t dst_frame_stride, int64_t dst_row_stride,
                                         void* saved, void* stream);

/* Writes dLoss/dInput into grad_in (overwritten) from dLoss/dOutput and the
 * saved state of a forward_saved call of the same context. The context keeps
 * a scratch ring of (stacks per adjoint launch + 2 * radius) frame planes for
 * the scaled output gradient (dLoss/dOutput over the frozen denominator),
 * allocated on the first call and freed with the context. */
VSFEEL_API int vsfeel_bm3d_backward(vsfeel_bm3d* ctx, const void* saved, const float* grad_out,
                                    int64_t go_frame_stride, int64_t go_row_stride, float* grad_in,
                                    int64_t gi_frame_stride, int64_t gi_row_stride, void* stream);

/* ---- Batched form (no counterpart in the reference) -----------------------
 *
 * Many clips of uneven sizes and settings denoised together; this replaces
 * the reference's num_streams concurrency. Clips are grouped into shape
 * classes (equal radius, block_step, bm_range, ps_num and ps_range). Per
 * class, the clips are cut into chunks of whole clips (at least ~16 waves
 * of tiles); per chunk one persistent launch works through a device queue
 * of (stack, tile) items of its clips, matching each tile, one launch
 * filters every block of its stacks and one normalises its output frames.
 * The class's work is captured once in a CUDA graph; a run replays the
 * classes' graphs one after another on the caller's stream. With
 * VSFEEL_BATCH_AUTOTUNE, vsfeel_bm3d_batch_create times every tile shape
 * that fits a class (its reference blocks per CTA and the shape of the
 * search region it stages) with 8 and with 16 lanes per reference block
 * (threads per group) on one of its stacks, and keeps the fastest pair;
 * otherwise the largest fitting shape with 8 lanes is used. A class that no shape fits (radius >= 3,
 * or windows too large) runs the direct-read kernels stack by stack inside
 * its graph.
 *
 * Buffers are bound at creation: every vsfeel_bm3d_batch_run replays the
 * graphs on the same src/dst buffers (device memory, strides in floats), so
 * new input goes into the same src buffers. Each clip is a GRAYS 32-bit
 * float clip; its outputs are all its frames. */
typedef struct vsfeel_bm3d_batch_clip {
    vsfeel_bm3d_args args;          /* per clip; "ref" is not supported   */
    int width, height, num_frames;
    const float* src;
    int64_t src_frame_stride, src_row_stride;
    float* dst;
    int64_t dst_frame_stride, dst_row_stride;
} vsfeel_bm3d_batch_clip;

typedef struct vsfeel_bm3d_batch vsfeel_bm3d_batch;

enum { VSFEEL_BATCH_AUTOTUNE = 1 };
/* flags: use tile shape s for every class it fits (tests and tuning runs) */
#define VSFEEL_BATCH_FORCE_SHAPE(s) ((((s) + 1) & 15) << 4)
/* flags: use 8 or 16 lanes per reference block in every tiled class */
#define VSFEEL_BATCH_FORCE_LANES(l) (((l) == 16 ? 2 : 1) << 8)

/* Tile shapes of the tiled matcher, in reference blocks (x by y). */
enum { VSFEEL_TILE_8X4 = 0, VSFEEL_TILE_16X2 = 1, VSFEEL_TILE_4X8 = 2, VSFEEL_TILE_8X2 = 3,
       VSFEEL_TILE_4X4 = 4, VSFEEL_TILE_SHAPES = 5 };

typedef struct vsfeel_bm3d_batch_class_info {
    int radius, block_step, bm_range, ps_num, ps_range;
    int clips, stacks;
    int64_t tiles;          /* work-queue items per run                      */
    int tile_shape;         /* VSFEEL_TILE_*, or -1: direct-read kernels     */
    double tuned_ms[VSFEEL_TILE_SHAPES]; /* autotuner's time per shape, 8 lanes, or 0 */
    int lanes;              /* lanes per reference block of the tiled matcher */
    double tuned_ms_16[VSFEEL_TILE_SHAPES]; /* the same with 16 lanes, or 0 */
} vsfeel_bm3d_batch_class_info;

VSFEEL_API int vsfeel_bm3d_batch_create(const vsfeel_bm3d_batch_clip* clips, int nclips, int device,
                                        int flags, vsfeel_bm3d_batch** out);

/* Enqueues one denoising of every clip, ordered after the work already on
 * `stream` (used as given); the call returns once the work is enqueued and
 * later work on `stream` waits for it. */
VSFEEL_API int vsfeel_bm3d_batch_run(vsfeel_bm3d_batch* batch, void* stream);

/* Waits (bounded) for the batch's enqueued work and reports an internal
 * error the kernels flagged. */
VSFEEL_API int vsfeel_bm3d_batch_finish(vsfeel_bm3d_batch* batch);

VSFEEL_API int vsfeel_bm3d_batch_classes(const vsfeel_bm3d_batch* batch, int* nclasses,
                                         int64_t* device_bytes);
VSFEEL_API int vsfeel_bm3d_batch_class(const vsfeel_bm3d_batch* batch, int index,
                                       vsfeel_bm3d_batch_class_info* info);

/* Frees the batch (waits, bounded, for its work first). Accepts NULL. */
VSFEEL_API void vsfeel_bm3d_batch_free(vsfeel_bm3d_batch* batch);

/* Allocation-free form of vsfeel_bm3d_process_device; it has no counterpart
 * in the reference. It is for callers that cannot let this library allocate
 * device memory: processes that reserve the GPU's memory in their own fixed
 * pools up front, and real-time pipelines that must not pay the implicit
 * device synchronisation of cudaMalloc/cudaFree. It takes the arguments and
 * clip format directly (no context), reads src and writes dst as
 * process_device does, and keeps every intermediate in one static device
 * array of vsfeel_bm3d_noalloc_scratch_bytes() (32 MiB), held by every GPU
 * that loads the library until exit; clips whose match table and
 * accumulator planes need more are rejected with an error. The array's
 * device address belongs to a CUDA context: the first call in each context
 * (the current one; a host's own driver-API context and a primary context
 * re-created after cudaDeviceReset each count as new) resolves and caches
 * it, so make that first call before any stream capture. The call only
 * enqueues work on `stream` (used as given) and never waits. All calls share
 * the array: calls that overlap on the GPU race and must be serialised by
 * the caller. */
VSFEEL_API int vsfeel_bm3d_process_device_noalloc(const vsfeel_bm3d_args* args,
                                                  const vsfeel_bm3d_video_info* vi,
                                                  const float* src, int64_t src_frame_stride,
                                                  int64_t src_row_stride, float* dst,
                                                  int64_t dst_frame_stride,
                                                  int64_t dst_row_stride, int first, int count,
                                                  void* stream);

/* Size of the allocation-free entry point's static scratch array, bytes. */
VSFEEL_API int64_t vsfeel_bm3d_noalloc_scratch_bytes(void);

/* The calling thread's last error message ("" when none). */
VSFEEL_API const char* vsfeel_bm3d_last_error(void);

/* ABI version of the loaded library (VSFEEL_BM3D_ABI_VERSION). */
VSFEEL_API int vsfeel_bm3d_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* VSFEEL_BM3D_H */
