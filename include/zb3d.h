/*
 * zb3d — B200-native BM3D / BM3Dv2 / VAggregate behind a plain C ABI.
 *
 * Drop-in replacement for the BM3D path of the vszipcu VapourSynth plugin.
 * Each entry point states the reference interface it replaces (paths inside the
 * vszipcu project).  No CUDA or torch types cross this boundary: frames are
 * plain float pointers with byte strides, device buffers are pointers, streams
 * are opaque `void *` (a cudaStream_t, or NULL for the default stream).
 *
 * Threading: a filter may be called from several threads at once (VapourSynth's
 * fmParallel): up to `num_streams` frames are in flight, each on its own pair of
 * CUDA streams; further callers wait for a free slot.
 */
#ifndef ZB3D_H
#define ZB3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* "argument not given" for the optional int arguments of zb3d_args. */
#define ZB3D_UNSET (-2147483647 - 1)

/* VapourSynth colour families (cfGray, cfRGB, cfYUV) and sample types. */
enum { ZB3D_GRAY = 1, ZB3D_RGB = 2, ZB3D_YUV = 3 };
enum { ZB3D_INTEGER = 0, ZB3D_FLOAT = 1 };

/* The part of VSVideoInfo / VSVideoFormat the filters read
 * (vszipcu src/bm3d.zig:990-1011, 1090-1092). */
typedef struct zb3d_video_info {
    int color_family;
    int sample_type;
    int bits_per_sample;
    int subsampling_w, subsampling_h;
    int num_planes;
    int width, height;
    int num_frames;
} zb3d_video_info;

/* The BM3D / BM3Dv2 argument map (vszipcu src/plugin.zig:84-90, defaults in
 * src/bm3d.zig:1013-1081).  Per-plane arrays hold n_* elements (0 = not given);
 * a missing element i falls back to element i-1, as the reference does.
 * Optional ints use ZB3D_UNSET for "not given".  Strings are case-insensitive. */
typedef struct zb3d_args {
    const zb3d_video_info *ref;            /* "ref" clip, or NULL */
    const float *sigma;            int n_sigma;
    const int *block_step;         int n_block_step;
    const int *bm_range;           int n_bm_range;
    int radius;
    const int *ps_num;             int n_ps_num;
    const int *ps_range;           int n_ps_range;
    int chroma;
    int device_id;
    int num_streams;
    int extractor_exp;
    const char *const *bm_error_s;      int n_bm_error_s;
    const char *const *transform_2d_s;  int n_transform_2d_s;
    const char *const *transform_1d_s;  int n_transform_1d_s;
    int zero_init;
    int fast_fused;
    /* Not in the reference.  Block-matching form for ssd: 0 = the FP32 scan of
     * every candidate; 1 = tensor-core distance bound plus exact FP32 re-rank of
     * the candidates under it, where the tile geometry allows it (block_step 4
     * with bm_range <= 13, for example); not given = the autotuner picks per plane
     * (zb3d_entry_tuning).  Every form gives the same lists. */
    int match_form;
    /* Not in the reference.  A learned pilot network (zb3d_pilot_load) that makes
     * BM3Dv2's step-1 estimate: the filter then runs both steps in one call, the pilot
     * (or, for a plane entry whose sigma the pilot's gate refuses, the plain step 1: hard
     * threshold with the step-1 sigma factor) into the reference slot, then step 2
     * (Wiener) matching on it, and returns step 2.  This is the two-pass
     * BM3Dv2(clip, ref=BM3Dv2(clip)) of the reference (src/bm3d.zig:995-1011) with
     * step 1 replaced.  BM3Dv2 only, no "ref" clip, radius 0, the pilot on device_id;
     * the filter does not own the pilot, which must outlive it.  NULL = off. */
    const struct zb3d_pilot *pilot;
    /* Not in the reference.  The collaborative filter's 2D transforms: 0 (not given) = the
     * FP32 SIMT transforms, bit for bit the reference's; 1 = the precision form, the 2D DCT
     * of every group's patches on the tensor cores in TF32 with the hi/lo split (FP32-level
     * error, not bitwise: a coefficient within rounding of the hard threshold may go either
     * way).  DCT in both dimensions only. */
    int filter_form;
} zb3d_args;

/* Fills `a` with "nothing given" (all defaults). */
void zb3d_args_init(zb3d_args *a);

/* One frame: up to three float planes, strides in bytes. */
typedef struct zb3d_frame {
    const float *ptr[3];
    ptrdiff_t stride[3];
} zb3d_frame;

typedef struct zb3d_frame_out {
    float *ptr[3];
    ptrdiff_t stride[3];
} zb3d_frame_out;

typedef struct zb3d_filter zb3d_filter;

/*
 * Creates a BM3D (v2 = 0) or BM3Dv2 (v2 = 1) filter for `clip`.
 * Replaces: vszipcu src/bm3d.zig:965 `create` / :1432 `createV2` (validation and
 * error strings :990-1256).  Returns NULL and writes the reference's error text
 * ("BM3D: ...") into err on failure.  BM3Dv2 with every plane's sigma below
 * FLT_EPSILON returns a pass-through filter (src/bm3d.zig:1449-1456).
 */
zb3d_filter *zb3d_create(const zb3d_video_info *clip, const zb3d_args *args, int v2, char *err, size_t errlen);

/* Output clip info: BM3D with radius > 0 emits the stacked accumulator clip of
 * height h*2*(2r+1) (src/bm3d.zig:1224-1231). */
void zb3d_output_info(const zb3d_filter *f, zb3d_video_info *out);

/* Source frames [*first, *last] that frame n needs from clip (and from ref),
 * the request pattern of src/bm3d.zig:643-650. */
void zb3d_frame_range(const zb3d_filter *f, int n, int *first, int *last);

/* Frame properties of the stacked output (BM3D_V_radius, BM3D_V_process), src/bm3d.zig:716-720. */
void zb3d_output_props(const zb3d_filter *f, int *radius, int process[3]);

/*
 * Produces frame n into dst.  clip_frames / ref_frames hold the frames
 * [first, last] of zb3d_frame_range (ref_frames NULL when there is no ref).
 * Replaces: vszipcu src/bm3d.zig:635 `getFrame` (process :274, processFused :481,
 * download :427).  Planes whose sigma is below FLT_EPSILON are not written
 * (the caller copies them, as newVideoFrame2 does), except that the stacked
 * output zeroes them when zero_init is set (src/bm3d.zig:708-715).
 * Returns 0, or -1 with "BM3D: process frame failed." style text in err.
 */
int zb3d_get_frame(zb3d_filter *f, int n, const zb3d_frame *clip_frames, const zb3d_frame *ref_frames,
                   zb3d_frame_out *dst, char *err, size_t errlen);

/* Releases the filter and its device memory (src/bm3d.zig:739 `free`). */
void zb3d_free(zb3d_filter *f);

/* ---- device-resident path (inputs already in HBM) ----------------------- */

/* One plane entry of a filter: a processed plane, or Y+U+V when chroma. */
typedef struct zb3d_entry_layout {
    int nplanes;              /* 1, or 3 for CBM3D */
    int plane[3];             /* clip plane index of each entry plane */
    int width, height, pitch; /* pitch in floats */
    int tw;                   /* temporal window 2r+1 of one frame's window */
    int nclips;               /* 2 when a ref clip drives matching */
    size_t src_offset, src_elems;  /* [clips][planes][tw][height][pitch] floats */
    size_t dst_offset, dst_elems;  /* [planes][height][pitch] (stacked: [planes][tw][2][height][pitch]) */
} zb3d_entry_layout;

int zb3d_num_entries(const zb3d_filter *f);
int zb3d_entry_layout_get(const zb3d_filter *f, int e, zb3d_entry_layout *out);
size_t zb3d_src_elems(const zb3d_filter *f);
size_t zb3d_dst_elems(const zb3d_filter *f);

/*
 * Runs one frame window entirely on the device: d_src holds zb3d_src_elems floats
 * in the entry layout, d_dst receives zb3d_dst_elems floats (the denoised planes,
 * or the stacked accumulators of BM3D radius > 0).  Enqueued on `stream`; uses
 * the filter's slot 0 workspace, so concurrent calls on one filter must not overlap.
 * Replaces the device half of src/bm3d.zig:375-401.
 */
int zb3d_process_device(zb3d_filter *f, const float *d_src, float *d_dst, void *stream, char *err, size_t errlen);

/*
 * One entry of one window on the device, with caller-placed buffers: d_src is the
 * entry's [clips][planes][tw][height][pitch] block, d_dst its
 * [planes][height][pitch] output (stacked [planes][tw][2][height][pitch] when
 * radius > 0).  Lets a two-pass pipeline write the basic estimate straight into
 * the ref slot of the second pass.  Same slot-0 workspace rule as above.
 */
int zb3d_process_entry_device(zb3d_filter *f, int e, const float *d_src, float *d_dst, void *stream, char *err,
                              size_t errlen);

/*
 * Launch timing: with `on`, every block-matching launch of this filter is
 * bracketed by CUDA events on its stream; zb3d_profile_collect waits for them
 * and returns the summed milliseconds and launch count since the last collect.
 */
void zb3d_profile_enable(zb3d_filter *f, int on);
int zb3d_profile_collect(zb3d_filter *f, double *match_ms, int *match_launches, double *filter_ms,
                         int *filter_launches);

/*
 * Block matching only, for entry e of one window already on the device: writes
 * the 8-entry match list of every reference block to d_list
 * (int32 pairs [nby][nbx][8][2]: x, then y | z << 24, in list order; z is the
 * window frame).  Blocks sit at x = min(bs*kx, w-8), y = min(bs*ky, h-8).
 * Replaces the matching half of vszipcu src/bm3d.cu:571-788 (its index8_x/y/z).
 */
int zb3d_match_device(zb3d_filter *f, int e, const float *d_src, int32_t *d_list, void *stream, char *err,
                      size_t errlen);

/*
 * The matching configuration the autotuner chose for entry e at creation: form
 * (0 FP32 scan, 1 tensor-core) and block rows per CTA of the tiled FP32 kernels.
 * The choice is timed once per GPU and plane geometry and cached in
 * $ZB3D_TUNE_CACHE (default ~/.cache/zb3d/tune-v2.txt); ZB3D_AUTOTUNE=0 skips the
 * timing.  It replaces the reference's per-configuration module cache
 * (src/bm3d.zig:57-70, 780-835).  Returns 0, or -1 for no such entry.
 */
int zb3d_entry_tuning(const zb3d_filter *f, int e, int *form, int *rows);

/*
 * Counters of the tensor-core matching form, summed over every call since the
 * last reset: out[0] tiles, out[1] reference blocks, out[2] candidates given the
 * exact re-rank, out[3] blocks handed to the FP32 scan.  Waits for slot 0's stream.
 */
int zb3d_match_stats(zb3d_filter *f, unsigned long long out[4], int reset);

/*
 * Diagnostic of the tensor-core form on one device plane (ssd, radius 0): writes
 * the match lists like zb3d_match_device, and the pass-1 distance matrix of
 * tile (0, 0) to d_dist: [128][zb3d_tc_probe_cols(...)] floats, row m = block
 * (m mod 8, m / 8) of the tile, column = flat candidate index of the tile's
 * union; only the rows and columns the kernel reads are written.  d_prof (may be
 * NULL): 16 counters per tile, zeroed by the caller: clock64 at the start, after
 * the region load, the FP16 copies, the candidate tables, operand A, the MMA
 * stream with the region reload, the exact errors and at the end (0-7), then the
 * unsuccessful mbarrier polls of the block, builder and issuer warps (8-10).
 * Returns 0, 1 when the geometry is outside the tensor-core form, -1 on error.
 */
int zb3d_tc_probe_cols(int width, int height, int block_step, int bm_range);
int zb3d_tc_probe(const float *d_plane, int width, int height, int pitch, int block_step, int bm_range,
                  int32_t *d_list, float *d_dist, unsigned long long *d_prof, unsigned long long stats[4], char *err,
                  size_t errlen);

/*
 * Temporal aggregation on the device over float accumulator stacks (the
 * stacked BM3D output): dst = sum_t num[t] / sum_t den[t] in ascending t, IEEE
 * division.  stacks[t] points to the stacked entry buffer of frame clamp(n-r+t),
 * z[t] is the slot aggZ(t, n, nframes, r).  Replaces src/bm3d_vagg.cu:18-48.
 */
int zb3d_vaggregate_device(const float *const *stacks, const int *z, int tw, int width, int height, int pitch,
                           int nplanes, unsigned proc_mask, float *d_dst, void *stream);

/*
 * One BM3D pass (radius 0, ssd matching, dct transforms) over one float plane that
 * is already in device memory, without allocating any device memory: the scratch
 * it needs lives in a fixed 24 MiB array inside the library.  No counterpart in
 * the reference.  It is for callers that cannot call cudaMalloc while they run: a
 * host that fixes each plugin's device-memory budget at load time, or one that
 * cannot afford cudaMalloc's implicit device-wide synchronisation mid-frame.
 *   d_src   [1 or 2][height][pitch] floats: the noisy plane; with final = 1, the
 *           basic estimate (matched on, Wiener reference) followed by the noisy plane
 *   d_dst   [height][pitch] denoised output
 *   sigma   8-bit-scale sigma as in zb3d_args (scaled internally like BM3D)
 * A sigma below FLT_EPSILON leaves the plane unprocessed, as BM3D does: the noisy
 * plane is copied to d_dst.
 * Limits: height*pitch <= 1048576 and at most 131072 reference blocks; larger
 * planes are rejected with an error.  The first call on a device looks up the
 * array's device address (make that first call before any stream capture); the
 * address is kept for the life of the process, so a device that was reset
 * (cudaDeviceReset) must not be given to this entry point again.
 * Every call reuses the same array, so calls that overlap on the GPU race.
 * Returns 0, or -1 with the reason in err.
 */
int zb3d_bm3d_plane_noalloc(const float *d_src, float *d_dst, int width, int height, int pitch, int final_,
                            float sigma, int block_step, int bm_range, int extractor_exp, void *stream, char *err,
                            size_t errlen);

/* ---- VAggregate -------------------------------------------------------- */

typedef struct zb3d_vagg zb3d_vagg;

/* Replaces: vszipcu src/bm3d.zig:1372 `createVAggregate` (errors :1391-1417). */
zb3d_vagg *zb3d_vaggregate_create(const zb3d_video_info *clip, const zb3d_video_info *src, const int *planes,
                                  int n_planes, char *err, size_t errlen);
void zb3d_vaggregate_output_info(const zb3d_vagg *v, zb3d_video_info *out);
/* Stacked frames [*first, *last] of `clip` that output frame n needs (src/bm3d.zig:1327-1331). */
void zb3d_vaggregate_frame_range(const zb3d_vagg *v, int n, int *first, int *last);
/* stacks = the stacked frames [first, last]; planes not listed are left to the caller.
 * Replaces src/bm3d.zig:1319 `aggGetFrame` / :1284 `aggPlane`. */
int zb3d_vaggregate_get_frame(zb3d_vagg *v, int n, const zb3d_frame *stacks, zb3d_frame_out *dst, char *err,
                              size_t errlen);
void zb3d_vaggregate_free(zb3d_vagg *v);

/* aggZ of src/bm3d.zig:46-48: the slot of stacked frame clamp(n-r+i) that belongs to frame n. */
int zb3d_agg_z(int i, int n, int nframes, int radius);

/*
 * Page-locked host memory for frames, from a pool of reused blocks (not in the
 * reference, whose frames come from VapourSynth).  zb3d_get_frame copies frames
 * that live in page-locked memory (this allocator, cudaHostAlloc or
 * cudaHostRegister) straight to and from the device, without the staging copy
 * that pageable frames take.  Returns NULL when the allocation fails.
 */
void *zb3d_host_alloc(size_t bytes);
void zb3d_host_free(void *p);

/* ---- batches (not in the reference) ---------------------------------------------
 *
 * One window (the zb3d_process_device layout: d_src, d_dst of that filter) of each job,
 * all on the filters' device, in one call: the plane entries of every job that use SSD
 * matching at block_step 4 or 8 (FP32 scan), radius 0 and the DCT in both dimensions are
 * matched and filtered by one persistent launch per filter step over a work list (match
 * tiles of every entry, then filter chunks, each chunk waiting, bounded, for its entry's
 * matching), then finished; any other entry runs on its own as in zb3d_process_device.
 * The call returns when the outputs are written (it synchronises `stream`).  Returns 0,
 * or -1 with the reason in err; a chunk that gave up waiting (about half a second)
 * reports "gave up waiting ... status 1" and leaves that batch's outputs incomplete, the
 * device stays usable.  Calls on one device are serialised; a filter in a batch must not
 * be used by another call at the same time.
 * Replaces: the per-frame launch sequence of vszipcu src/bm3d.zig:375-401 for many
 * windows at once. */
typedef struct zb3d_batch_job {
    zb3d_filter *filter;
    const float *d_src;
    float *d_dst;
} zb3d_batch_job;
int zb3d_process_batch(const zb3d_batch_job *jobs, int njobs, void *stream, char *err, size_t errlen);
/* The same with the wait bound in polls (about 0.1 us each; 0 = the default, 2^22) and a
 * testing switch that makes the first entry's filter chunks wait for one match tile more
 * than exists, so that their waits run out. */
int zb3d_process_batch_ex(const zb3d_batch_job *jobs, int njobs, void *stream, unsigned wait_polls,
                          int unsatisfiable, char *err, size_t errlen);

/* The same batch captured once into a CUDA graph (work-list launches, finishes, the
 * entries outside the work list and the status read-back), with scratch of its own:
 * zb3d_batch_launch replays it on `stream` asynchronously, for the same jobs and buffers.
 * Launches of one batch must not overlap on the GPU; different batches may.  After the
 * caller has synchronised the stream, zb3d_batch_status returns 0, or -1 with the reason
 * when a filter chunk of the last launch gave up waiting.  Creation holds one slot of each
 * filter whose entries run outside the work list until zb3d_batch_free (waiting for a free
 * one), so such a filter needs a slot per live batch that uses it beside its own callers'.
 * NULL with the reason in err on failure. */
typedef struct zb3d_batch zb3d_batch;
zb3d_batch *zb3d_batch_create(const zb3d_batch_job *jobs, int njobs, char *err, size_t errlen);
int zb3d_batch_launch(zb3d_batch *b, void *stream, char *err, size_t errlen);
int zb3d_batch_status(zb3d_batch *b, char *err, size_t errlen);
void zb3d_batch_free(zb3d_batch *b);

/* ---- learned pilot (not in the reference) -------------------------------------
 *
 * Kernels of the residual conv net that can replace the BM3D step-1 estimate as
 * step 2's reference (zb3d/pilot.py trains and runs it).  BF16 tensors (void *),
 * NHWC with channel counts 16, 32 or 48; weights [cout][3][3][cin]; FP32 accumulation.
 * All calls are asynchronous on `stream` and return 0, or -1 on a launch error.
 */
/* y = conv3x3(x) + bias (may be NULL), ReLU if relu, zeroed where mask (NHWC, cout
 * channels, may be NULL) is <= 0; y (may be NULL) BF16 NHWC; y0 (may be NULL) the
 * FP32 channel 0 plus resid (may be NULL).  (cin, cout) in {(16,48), (48,48), (48,16), (16,32),
 * (32,32), (32,16), (16,16)}.  mma.sync BF16 tiles of 8 x 16 pixels; the training passes use it. */
int zb3d_pilot_conv3x3(const void *x, int n, int h, int w, int cin, const void *wgt, const float *bias, int cout,
                       int relu, const void *mask, void *y, float *y0, const float *resid, void *stream);
/* The same forward convolution (no mask) on the tensor cores, for inference: tcgen05.mma
 * with the accumulator in tensor memory, input rows staged by TMA, persistent CTAs down
 * 128-pixel column strips.  x and y use the channel-blocked layout [n][C/8][h][w][8]
 * (BF16); same shapes; x, wgt and y 16-byte aligned.  The images of y0 and resid are
 * y0_stride and resid_stride floats apart (0: h * w).  status (device int, may be NULL)
 * becomes non-zero if a pipeline wait timed out. */
int zb3d_pilot_conv3x3_tc(const void *x, int n, int h, int w, int cin, const void *wgt, const float *bias, int cout,
                          int relu, void *y, float *y0, const float *resid, long long y0_stride,
                          long long resid_stride, int *status, void *stream);
/* Grid of zb3d_pilot_conv3x3_tc for the whole process: at most ctas CTAs per SM (1..4; 4
 * by default, i.e. the layer's own count: 4 up to 32 channels, 2 with 48).  The default
 * fills each SM and is fastest alone; 1 leaves room for kernels of other streams.
 * Returns 0, or -1 for an unsupported value. */
int zb3d_pilot_tc_ctas_per_sm(int ctas);
/* Precision form of the patch transform (no counterpart in the reference, whose 2D
 * transform is FP32 SIMT code, src/bm3d.cu:32-110 and :392-413): the 2D DCT of npatches
 * row-major 8x8 FP32 patches (d_x, d_y: [npatches][64] in device memory, d_y 16-byte
 * aligned) on the tcgen05 tensor cores in TF32 with FP32 accumulation.  split = 1 adds
 * the hi/lo products that win the accuracy back (Xl.Kh + Xh.Kl + Xh.Kh), split = 0 is
 * one TF32 product.  The first call on a device copies the transform matrix to it
 * (synchronous).  *d_status (device) becomes 1 if a wait for the products timed out and
 * they then landed, 2 if they had not landed even after a second wait: the device is then
 * unhealthy (tensor memory was released under a running MMA) and the call must not be
 * retried.  Returns 0, 1 for bad arguments, 2 for a CUDA error. */
int zb3d_dct2d_tf32(const float *d_x, float *d_y, long long npatches, int split, int *d_status, void *stream);
/* The network input of zb3d_pilot_pack_input in the channel-blocked layout ([n][2][h][w][8]);
 * the noisy images are noisy_stride floats apart (0: h * w). */
int zb3d_pilot_pack_input_blocked(const float *noisy, long long noisy_stride, const float *sigma, int n, int h,
                                  int w, float level_scale, void *x0, void *stream);
/* dw += dL/dw, db += dL/db of one layer from its input x and its pre-activation gradient dy. */
int zb3d_pilot_conv3x3_wgrad(const void *x, const void *dy, int n, int h, int w, int cin, int cout, float *dw,
                             float *db, void *stream);
/* network input: channel 0 = noisy, 1 = sigma[image] / 255 * level_scale, others 0 (16 channels). */
int zb3d_pilot_pack_input(const float *noisy, const float *sigma, int n, int h, int w, float level_scale, void *x0,
                          void *stream);
/* dy (16 channels) = scale * dMSE/dy in channel 0; loss_partials[k] (may be NULL; ceil(count / 256)
 * floats) = the FP32 sum of squared errors of elements [256 k, 256 k + 256), for the host to add up. */
int zb3d_pilot_mse_grad(const float *y, const float *t, long long count, float scale, void *dy,
                        float *loss_partials, void *stream);
/* Adam step (step >= 1) on FP32 weights w with loss-scaled gradient g / gscale; keep (may be NULL)
 * pins entries to 0 where keep == 0; w16 (may be NULL) receives the BF16 copy. */
int zb3d_pilot_adam(float *w, float *m, float *v, const float *g, long long count, float lr, float b1, float b2,
                    float eps, int step, float gscale, const float *keep, void *w16, void *stream);
/* wt[ci][8 - tap][co] = w[co][tap][ci]: weights of the backward pass to a layer's input. */
int zb3d_pilot_flip_weights(const void *w, int cin, int cout, void *wt, void *stream);
int zb3d_pilot_to_bf16(const float *a, long long count, void *b, void *stream);

/* ---- the pilot network as one object (not in the reference) ----------------------
 *
 * Weights file "ZB3DPLT1": header (architecture, noise-level input scale, the gate
 * table), FP32 weights and biases of each layer, CRC-32 of the whole; written by
 * zb3d.pilot.save_weights.  The gate table lists, per calibrated noise level (8-bit
 * scale) and plane size, the mean two-pass PSNR difference (pilot minus plain step 1)
 * measured on held-out synthetic planes of that size; the pilot is accepted for a plane
 * when the level of the nearest calibrated size (by area) nearest to its sigma has a
 * difference >= -tol (tol = 0.05 dB in the shipped files). */
typedef struct zb3d_pilot zb3d_pilot;
/* Loads a weights file (or the same bytes from memory) onto device_id.  Returns NULL
 * and writes a reason into err when the file is missing, damaged (checksum), of another
 * version or architecture, or the device has no room. */
zb3d_pilot *zb3d_pilot_load(const char *path, int device_id, char *err, size_t errlen);
zb3d_pilot *zb3d_pilot_from_memory(const void *data, size_t bytes, int device_id, char *err, size_t errlen);
void zb3d_pilot_free(zb3d_pilot *p);
/* Hidden channels, layer count and gate levels of the network. */
void zb3d_pilot_describe(const zb3d_pilot *p, int *width, int *layers, int *gate_levels);
/* Gate level i: its noise level, plane size and measured two-pass difference in dB.
 * 0, or -1 out of range. */
int zb3d_pilot_gate_level(const zb3d_pilot *p, int i, float *sigma, int *width, int *height, float *delta_db);
/* 1 if the gate accepts the pilot for a width x height plane at this noise level (8-bit
 * scale), else 0. */
int zb3d_pilot_accepts(const zb3d_pilot *p, float sigma, int width, int height);
/* Device workspace zb3d_pilot_run needs for a width x height plane (bytes). */
size_t zb3d_pilot_workspace_bytes(const zb3d_pilot *p, int width, int height);
/* The pilot estimate of one FP32 plane: d_out = d_noisy + net(d_noisy, sigma), rows
 * pitch / out_pitch floats apart (0: width).  d_workspace: zb3d_pilot_workspace_bytes,
 * 256-byte aligned, not shared with a concurrent call.  d_status (device int, may be
 * NULL) becomes non-zero if a convolution pipeline wait timed out.  Asynchronous on
 * stream (a cudaStream_t or NULL); call with the pilot's device current.  Returns 0, or -1
 * for bad arguments or a launch error. */
int zb3d_pilot_run(const zb3d_pilot *p, const float *d_noisy, int width, int height, int pitch, float sigma,
                   float *d_out, int out_pitch, void *d_workspace, int *d_status, void *stream);

/* Library version string. */
const char *zb3d_version(void);

#ifdef __cplusplus
}
#endif

#endif /* ZB3D_H */
