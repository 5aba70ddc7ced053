/*
 * av1pf.h — C ABI of the B200 (sm_100a) AV1 frame post-filter chain.
 *
 * The chain is the one the reference decoder runs after tile decoding
 * (rivet-av1 src/decoder/mod.rs:747-759 `decode_frame_wrapup`, and the output
 * process at :846-917): deblocking loop filter (7.14) -> CDEF (7.15) ->
 * super-resolution (7.16) -> loop restoration (7.17) -> reference frame, then
 * on output crop + film grain (7.18.3) + packing into the `Frame` layout.
 *
 * Every entry point is `extern "C"`, takes plain structs and pointers, and
 * returns an `int` status (AV1PF_OK or an AV1PF_ERR_* code); nothing throws
 * or aborts across the boundary. Sample planes and per-4x4 maps passed to the
 * device entry points are DEVICE pointers; the `_host` entry points take host
 * pointers and do the copies themselves. Streams are `cudaStream_t` passed as
 * `void*` (NULL = the legacy default stream), so this header needs no CUDA
 * include.
 *
 * A context is used from one host thread at a time; the serving API
 * (av1pf_serve_*) is internally synchronised.
 */
#ifndef AV1PF_H
#define AV1PF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes. The reference's post-filters are infallible (they panic on  */
/* out-of-bounds through SharedPlane's asserts, postfilter.rs:41,48,57); its */
/* decode-level errors are Error::{Bitstream, Unsupported, InvalidInput}     */
/* (lib.rs:60-73). These codes map onto those, plus device-side conditions.  */
/* ------------------------------------------------------------------------ */
enum {
  AV1PF_OK = 0,
  AV1PF_ERR_INVALID_INPUT = 1, /* bad descriptor, size or parameter       */
  AV1PF_ERR_UNSUPPORTED = 2,   /* valid AV1 but outside this build        */
  AV1PF_ERR_OOM = 3,           /* device allocation failed                */
  AV1PF_ERR_ADMISSION = 4,     /* refused: would exceed the HBM cap       */
  AV1PF_ERR_TIMEOUT = 5,       /* a bounded wait ran out                  */
  AV1PF_ERR_CUDA = 6,          /* a CUDA runtime call failed              */
  AV1PF_ERR_NOT_FOUND = 7      /* unknown ticket / stream                 */
};

/* Restoration types (consts.rs:284-286). */
enum { AV1PF_RESTORE_NONE = 0, AV1PF_RESTORE_WIENER = 1, AV1PF_RESTORE_SGRPROJ = 2 };

#define AV1PF_MAX_PLANES 3

/* One plane of samples. `data` points at sample (0,0); samples are uint8_t
 * when the frame's sample_bytes is 1 (8-bit only) and uint16_t when it is 2.
 * The reference keeps every plane as u16 with stride = allocated width
 * (src/decoder/state.rs:9-42); rows are `stride` samples apart here too. */
typedef struct av1pf_plane {
  void* data;
  int64_t stride; /* row pitch in samples */
  int32_t width;  /* allocated (readable) width in samples  */
  int32_t height; /* allocated rows */
} av1pf_plane;

/* Frame geometry and format: FrameCtx fields bit_depth, ssx, ssy, num_planes,
 * mi_rows, mi_cols (decoder/mod.rs:44-52) plus the header's frame_width,
 * frame_height, upscaled_width (header.rs:117-121) and the sequence's
 * matrix_coefficients (read by film grain, grain.rs:287). */
typedef struct av1pf_frame_info {
  int32_t bit_depth;      /* 8, 10 or 12 */
  int32_t sample_bytes;   /* 1 (bit_depth 8 only) or 2 */
  int32_t subsampling_x;  /* 0/1 */
  int32_t subsampling_y;  /* 0/1 */
  int32_t num_planes;     /* 1 (monochrome) or 3 */
  int32_t frame_width;    /* coded width (after superres downscaling) */
  int32_t frame_height;
  int32_t upscaled_width; /* == frame_width without superres */
  int32_t mi_rows;        /* 2*((frame_height+7)>>3), header.rs:728-731 */
  int32_t mi_cols;        /* 2*((frame_width+7)>>3) */
  int32_t matrix_coefficients;
} av1pf_frame_info;

/* Mode info of one 4x4 luma block: the fields of the reference's `Mi`
 * (decoder/state.rs:55-75) that the loop filter reads (postfilter.rs:133-138,
 * 215-224) and CDEF's skip test (postfilter.rs:306-307). 8 bytes. */
typedef struct av1pf_mi {
  uint8_t mi_size;      /* BLOCK_4X4 (0) .. BLOCK_64X16 (21) */
  uint8_t y_mode;       /* YMode: intra 0..12, inter NEARESTMV (14) .. */
  int8_t ref_frame0;    /* RefFrame[0]: 0 = INTRA_FRAME, 1..7 inter */
  uint8_t skip_segment; /* bit 7: skip; bits 0..2: segment_id */
  int8_t delta_lf[4];   /* DeltaLF[0..3] */
} av1pf_mi;

#define AV1PF_MI_SKIP 0x80u

/* One loop-restoration unit (LrType, LrWiener, LrSgrSet, LrSgrXqd of
 * decoder/mod.rs:31-41), 12 bytes. */
typedef struct av1pf_lr_unit {
  uint8_t type;       /* AV1PF_RESTORE_* */
  uint8_t sgr_set;    /* 0..15 */
  int8_t sgr_xqd[2];
  int8_t wiener[2][3]; /* [0] vertical, [1] horizontal coefficients */
  uint8_t _pad[2];
} av1pf_lr_unit;

/* Per-4x4 and per-unit maps the chain reads (device pointers for the device
 * entry points). Layouts follow the reference's FrameCtx arrays
 * (decoder/mod.rs:547-611): `mi` is row-major with row stride `mi_stride`
 * (the reference uses mi_cols + 32); lf_tx_size[p] is indexed
 * (row >> ssy) * mi_stride + (col >> ssx) in every plane
 * (postfilter.rs:135); cdef_idx is one int8 per 64x64, index
 * (r >> 4) * cdef_stride + (c >> 4), -1 = CDEF off for that 64x64
 * (postfilter.rs:285); lr_units[p] holds unit_rows x unit_cols units. */
typedef struct av1pf_maps {
  const av1pf_mi* mi;
  int32_t mi_stride;
  int32_t cdef_stride;
  const uint8_t* lf_tx_size[AV1PF_MAX_PLANES];
  const int8_t* cdef_idx;
  const av1pf_lr_unit* lr_units[AV1PF_MAX_PLANES];
} av1pf_maps;

/* Film grain parameters (FilmGrainParams, header.rs:14-45). `apply` is
 * film_grain_params_present && apply_grain (decoder/mod.rs:865). */
typedef struct av1pf_film_grain {
  int32_t apply;
  int32_t grain_seed;
  int32_t num_y_points;
  int32_t point_y_value[16];
  int32_t point_y_scaling[16];
  int32_t chroma_scaling_from_luma;
  int32_t num_cb_points;
  int32_t point_cb_value[16];
  int32_t point_cb_scaling[16];
  int32_t num_cr_points;
  int32_t point_cr_value[16];
  int32_t point_cr_scaling[16];
  int32_t grain_scaling_minus_8;
  int32_t ar_coeff_lag;
  int32_t ar_coeffs_y_plus_128[24];
  int32_t ar_coeffs_cb_plus_128[25];
  int32_t ar_coeffs_cr_plus_128[25];
  int32_t ar_coeff_shift_minus_6;
  int32_t grain_scale_shift;
  int32_t cb_mult, cb_luma_mult, cb_offset;
  int32_t cr_mult, cr_luma_mult, cr_offset;
  int32_t overlap_flag;
  int32_t clip_to_restricted_range;
} av1pf_film_grain;

/* The frame header's filter fields (FrameHeader, header.rs:89-177) that the
 * chain reads, plus the derived enables. */
typedef struct av1pf_params {
  /* loop filter (7.14): postfilter.rs:67-264 */
  int32_t loop_filter_level[4];
  int32_t loop_filter_sharpness;
  int32_t loop_filter_delta_enabled;
  int32_t loop_filter_ref_deltas[8];
  int32_t loop_filter_mode_deltas[2];
  int32_t delta_lf_multi;
  int32_t segmentation_enabled;
  uint8_t feature_enabled[8][8];
  int32_t feature_data[8][8];
  /* CDEF (7.15): postfilter.rs:273-342. cdef_enabled is
   * !coded_lossless && !allow_intrabc && enable_cdef (postfilter.rs:276). */
  int32_t cdef_enabled;
  int32_t cdef_damping; /* 3..6 */
  int32_t cdef_bits;
  int32_t cdef_y_pri_strength[8];
  int32_t cdef_y_sec_strength[8];
  int32_t cdef_uv_pri_strength[8];
  int32_t cdef_uv_sec_strength[8];
  /* super-resolution (7.16): postfilter.rs:521-566 */
  int32_t use_superres;
  /* loop restoration (7.17): postfilter.rs:608-1004 */
  int32_t uses_lr;
  int32_t frame_restoration_type[3];
  int32_t loop_restoration_size[3];
  int32_t lr_unit_rows[3];
  int32_t lr_unit_cols[3];
  /* film grain (7.18.3): grain.rs */
  av1pf_film_grain film_grain;
} av1pf_params;

/* ------------------------------------------------------------------------ */
/* Context                                                                   */
/* ------------------------------------------------------------------------ */
typedef struct av1pf_ctx av1pf_ctx;

/* Creates a context on CUDA device `device`. `hbm_cap_bytes` bounds the
 * device memory the context's scratch, batches and served streams may hold
 * (0 = no cap). Replaces the reference's Decoder::new (decoder/mod.rs:273). */
int av1pf_ctx_create(int device, uint64_t hbm_cap_bytes, av1pf_ctx** out);
int av1pf_ctx_destroy(av1pf_ctx* ctx);

/* Mirrors Decoder::set_threads (decoder/mod.rs:323-329): the reference's
 * worker-thread count for the post-filter bands. On the device the bands all
 * run at once; here `n` is the number of frames av1pf_chain_host_many keeps
 * in flight, each in a device frame slot of its own (its upload, chain and
 * download overlap those of the other slots' frames): 0 = the default of 3,
 * values above 8 mean 8. Each slot holds one frame's input planes, maps,
 * reference frame and packed frame, allocated on first use. */
int av1pf_set_threads(av1pf_ctx* ctx, int n);

/* Bytes of device memory the context currently holds. */
int av1pf_ctx_memory(const av1pf_ctx* ctx, uint64_t* bytes);

/* Validates a frame descriptor, params and plane geometry without touching
 * the device (the reference's setup_frame limits, decoder/mod.rs:501-589). */
int av1pf_validate(const av1pf_frame_info* info, const av1pf_params* params,
                   const av1pf_plane* planes);

/* ------------------------------------------------------------------------ */
/* Per-stage device entry points (device pointers, stream-ordered).          */
/* ------------------------------------------------------------------------ */

/* Loop filter (7.14), in place on `planes`, both passes, every plane whose
 * level is set. Replaces loop_filter_threads (postfilter.rs:67-104). */
int av1pf_loop_filter(av1pf_ctx* ctx, const av1pf_frame_info* info,
                      const av1pf_params* params, const av1pf_maps* maps,
                      av1pf_plane* planes, void* stream);

/* CDEF (7.15) from `cur` into `out` (every sample of the MI area written:
 * filtered, or copied where CDEF is off). Replaces cdef (postfilter.rs:273),
 * which returns a filtered clone of `cur`. */
int av1pf_cdef(av1pf_ctx* ctx, const av1pf_frame_info* info,
               const av1pf_params* params, const av1pf_maps* maps,
               const av1pf_plane* cur, av1pf_plane* out, void* stream);

/* Super-resolution upscaling (7.16) of `in` (coded width) into `out`
 * (upscaled width), rows 0..round2(frame_height, ssy). Replaces upscale
 * (postfilter.rs:521-566). Requires params->use_superres. */
int av1pf_superres(av1pf_ctx* ctx, const av1pf_frame_info* info,
                   const av1pf_params* params, const av1pf_plane* in,
                   av1pf_plane* out, void* stream);

/* Loop restoration (7.17) of the upscaled CDEF frame `cdef` into `out`, with
 * the stripe-boundary rows taken from the upscaled pre-CDEF frame `cur`
 * (LrCtx::sample, postfilter.rs:581-597). `out` receives the whole visible
 * area (restored units, copies elsewhere). Replaces loop_restoration
 * (postfilter.rs:608-636). */
int av1pf_loop_restoration(av1pf_ctx* ctx, const av1pf_frame_info* info,
                           const av1pf_params* params, const av1pf_maps* maps,
                           const av1pf_plane* cur, const av1pf_plane* cdef,
                           av1pf_plane* out, void* stream);

/* Output process (7.18): crops the reference frame `ref` to
 * upscaled_width x frame_height, applies film grain when
 * params->film_grain.apply, and packs the planes into `frame_out` in the
 * reference's Frame layout (frame.rs:135-192, decoder/mod.rs:893-915): Y then
 * U then V, each plane row-major with stride = plane width, u8 samples at
 * 8-bit and little-endian u16 above. Replaces grain::apply (grain.rs:24) plus
 * the packing loop of Decoder::output. */
int av1pf_output(av1pf_ctx* ctx, const av1pf_frame_info* info,
                 const av1pf_params* params, const av1pf_plane* ref,
                 uint8_t* frame_out, void* stream);

/* Bytes av1pf_output writes for `info`. */
size_t av1pf_frame_bytes(const av1pf_frame_info* info);

/* The MD5 a conformance vector's .md5 file holds for a decoded frame
 * (tests/common/mod.rs:101-119 `frame_md5`): MD5 (RFC 1321) of the packed
 * frame as av1pf_output writes it (HOST memory, av1pf_frame_bytes bytes),
 * followed for a monochrome frame by two neutral chroma planes
 * (ceil(w/2) x ceil(h/2) samples of 1 << (bit_depth - 1), as a 4:2:0 file
 * carries it). Writes 32 lowercase hex digits and a NUL. Runs on the host:
 * MD5 is one serial chain of 64-byte blocks. */
int av1pf_frame_md5(const av1pf_frame_info* info, const uint8_t* frame,
                    char md5_hex[33]);
/* MD5 (RFC 1321) of n host bytes, as 32 hex digits and a NUL. */
int av1pf_md5(const uint8_t* data, size_t n, char md5_hex[33]);

/* av1pf_output for callers that cannot allocate device memory — a decoder
 * embedded in a host whose device memory belongs to another allocator, or a
 * real-time output path that cannot take an allocation's latency or an
 * out-of-memory failure mid-stream. No counterpart in the reference (its
 * output process allocates freely on the host).
 *
 * It takes no context and allocates nothing: its scratch (descriptor, work
 * list, film-grain templates and block offsets) is one fixed device array of
 * about 260 KB inside libav1pf, which every GPU that loads the library holds
 * until the process exits. Limit: with film grain on, frames up to
 * ceil(upscaled_width/32) * ceil(frame_height/32) <= 65536 (e.g. 8192x8192);
 * larger frames are refused with AV1PF_ERR_UNSUPPORTED. Runs on the current
 * device. The first call in a device's context does a one-time set-up there
 * (looks up the array's device address, uploads the grain RNG tables); make
 * that first call before any stream capture. After a cudaDeviceReset the
 * device's next context gets the same set-up on its first call. Every call
 * shares the one array, and each
 * call rewrites all of it that it reads, so nothing depends on earlier
 * contents; calls that overlap on the GPU (different streams, or several
 * host threads at once) race on it — issue them on one stream. */
int av1pf_output_noalloc(const av1pf_frame_info* info, const av1pf_params* params,
                         const av1pf_plane* ref, uint8_t* frame_out, void* stream);

/* ------------------------------------------------------------------------ */
/* Whole chain                                                               */
/* ------------------------------------------------------------------------ */

/* decode_frame_wrapup's filter chain (decoder/mod.rs:748-759) plus the
 * output process: reads the pre-filter planes `in` (left unchanged), writes
 * the LR frame (the reference frame, RefData.frame) into `ref_out` over the
 * visible area, and — when `frame_out` is not NULL — the packed output frame
 * as av1pf_output does. Scratch comes from the context. The kernels are
 * queued on `stream`; the call returns once the frame's descriptors are on
 * the device. The context keeps two descriptor buffers in turn, so the call
 * may first wait on the host for the chain it queued two calls earlier:
 * a caller runs at most about two calls ahead of the GPU per context. */
int av1pf_chain(av1pf_ctx* ctx, const av1pf_frame_info* info,
                const av1pf_params* params, const av1pf_maps* maps,
                const av1pf_plane* in, av1pf_plane* ref_out,
                uint8_t* frame_out, void* stream);

/* av1pf_chain from HOST memory: uploads the planes and maps, runs the chain,
 * downloads the reference frame (when ref_out is not NULL) and the packed
 * frame (when frame_out is not NULL), and returns when they are on the host.
 * The host-side drop-in for decode_frame_wrapup + output. Host planes use
 * their own strides; ref_out planes must be at least visible-area sized. */
int av1pf_chain_host(av1pf_ctx* ctx, const av1pf_frame_info* info,
                     const av1pf_params* params, const av1pf_maps* maps,
                     const av1pf_plane* in, av1pf_plane* ref_out,
                     uint8_t* frame_out);

/* One frame of av1pf_chain_host_many: the arguments of av1pf_chain_host. */
typedef struct av1pf_host_job {
  const av1pf_frame_info* info;
  const av1pf_params* params;
  const av1pf_maps* maps;
  const av1pf_plane* in;
  av1pf_plane* ref_out;  /* NULL: no reference-frame download */
  uint8_t* frame_out;    /* NULL: no packed-frame download */
} av1pf_host_job;

/* n av1pf_chain_host calls in one, for a decoder that holds several decoded
 * frames (a sequence's frames, or several streams'): the frames' uploads,
 * filter chains and downloads overlap on separate streams, over device frame
 * slots used in turn (3, or as av1pf_set_threads sets), so the copies in both directions and the
 * kernels run at the same time. Returns when every job's outputs are on the
 * host; the results equal n av1pf_chain_host calls. Every job is validated
 * before anything is queued. Host buffers should be pinned (page-locked),
 * or the copies do not overlap. */
int av1pf_chain_host_many(av1pf_ctx* ctx, int n, const av1pf_host_job* jobs);

/* ------------------------------------------------------------------------ */
/* Reference frames on the device: the reference frame update process (7.20, */
/* decoder/mod.rs:797-806) over frames the chain leaves on the device. Each  */
/* of the 8 slots holds a frame (RefData.frame, state.rs:79-101: the LR      */
/* frame) by reference count, several slots sharing one, as the reference's  */
/* Arc<RefData> does; a GPU decoder upstream reads a slot's planes for inter */
/* prediction without a copy.                                                */
/* ------------------------------------------------------------------------ */
typedef struct av1pf_refs av1pf_refs;

/* What a slot holds. */
typedef struct av1pf_ref_frame {
  int32_t valid;              /* 0: the slot is empty (the rest is zero) */
  av1pf_frame_info info;      /* the frame's geometry */
  uint32_t order_hint;        /* as given to av1pf_refs_chain */
  uint64_t frame_id;          /* 1, 2, ...: the av1pf_refs_chain call that made it */
  av1pf_plane planes[AV1PF_MAX_PLANES]; /* device: the LR frame over the visible area */
} av1pf_ref_frame;

/* An empty table (no device memory until the first frame). The table uses
 * the context's device, scratch and HBM cap. */
int av1pf_refs_create(av1pf_ctx* ctx, av1pf_refs** out);
/* Synchronises the device, then frees the table's frames. */
int av1pf_refs_destroy(av1pf_refs* refs);

/* decode_frame_wrapup (decoder/mod.rs:747-806) for a frame kept on the
 * device: av1pf_chain with its reference frame written into a frame of the
 * table, then the reference frame update process: every slot i whose bit i
 * of refresh_frame_flags is set now holds that frame. A frame no slot holds
 * any longer returns to the table's pool, and a later call writes into it in
 * stream order: use one stream per table (or order the streams that read
 * slot planes before the next call). frame_out as for av1pf_chain (may be
 * NULL). */
int av1pf_refs_chain(av1pf_refs* refs, const av1pf_frame_info* info,
                     const av1pf_params* params, const av1pf_maps* maps,
                     const av1pf_plane* in, uint32_t refresh_frame_flags,
                     uint32_t order_hint, uint8_t* frame_out, void* stream);

/* The frame slot `slot` (0..7) holds. Its planes stay valid until calls have
 * replaced it in every slot that holds it. */
int av1pf_refs_get(const av1pf_refs* refs, int slot, av1pf_ref_frame* out);

/* show_existing_frame (decoder/mod.rs:819-842): the output process on the
 * frame in `slot` with the film grain of `params` into `frame_out` (device),
 * then the update with refresh_frame_flags (a shown key frame passes all
 * slots; otherwise 0). AV1PF_ERR_INVALID_INPUT for an empty slot. */
int av1pf_refs_show(av1pf_refs* refs, int slot, const av1pf_params* params,
                    uint32_t refresh_frame_flags, uint8_t* frame_out, void* stream);

/* Device bytes the table's frames hold, and how many frames it has made. */
int av1pf_refs_memory(const av1pf_refs* refs, uint64_t* bytes, int32_t* frames);

/* ------------------------------------------------------------------------ */
/* Batched path: many frames of mixed shape / bit depth / subsampling, one   */
/* persistent launch per stage, replayed from a captured CUDA graph.         */
/* ------------------------------------------------------------------------ */
typedef struct av1pf_job {
  const av1pf_frame_info* info;
  const av1pf_params* params;
  const av1pf_maps* maps;   /* device */
  const av1pf_plane* in;    /* device, num_planes entries */
  av1pf_plane* ref_out;     /* device, num_planes entries */
  uint8_t* frame_out;       /* device, or NULL */
} av1pf_job;

typedef struct av1pf_batch av1pf_batch;

/* Plans a batch: validates the jobs, allocates per-frame scratch, builds the
 * per-stage work lists and captures the stage launches into a CUDA graph.
 * `flags`: AV1PF_BATCH_NO_GRAPH launches the stages directly. */
#define AV1PF_BATCH_NO_GRAPH 1u
/* AV1PF_BATCH_AUTOTUNE: first run av1pf_autotune on the jobs' shapes that
 * the context has not measured, then time each kernel variant applied to the
 * whole batch (and the per-shape choices) on the batch itself and plan the
 * fastest. The jobs' outputs are overwritten while timing. */
#define AV1PF_BATCH_AUTOTUNE 2u
/* Frame groups: (n << AV1PF_BATCH_GROUPS_SHIFT), n in 1..15, splits the
 * frames into n groups of about equal samples whose stage chains run as
 * parallel branches of the graph, so stages of different groups overlap on
 * the device. 0 (the default): 2 groups from 8 frames up, else 1. With
 * AV1PF_BATCH_AUTOTUNE the tuned count replaces it. */
#define AV1PF_BATCH_GROUPS_SHIFT 8
int av1pf_batch_create(av1pf_ctx* ctx, const av1pf_job* jobs, int n_jobs,
                       uint32_t flags, av1pf_batch** out);
/* Runs the planned batch on `stream` (graph launch). */
int av1pf_batch_run(av1pf_batch* batch, void* stream);
int av1pf_batch_destroy(av1pf_batch* batch);

/* ------------------------------------------------------------------------ */
/* Kernel variants and the autotuner. No counterpart in the reference, whose  */
/* filters each have one code path; the variants compute the same samples.    */
/* ------------------------------------------------------------------------ */
typedef struct av1pf_tuning {
  /* How the loop filter runs in chain calls. -1: per frame shape, the mode
   * av1pf_autotune measured fastest (mode 3 while a shape is unmeasured).
   * 0: one kernel decides every 4x4 edge into a compact list per direction,
   *    then one kernel per direction filters the listed edges in place;
   * 1: vertical edges filtered per 64x64 tile in shared memory (the tile
   *    staged with 16 columns of halo), horizontal edges from a list;
   * 2: as 1, with the horizontal edges filtered inside the CDEF kernel on
   *    its staged superblock window (frames with CDEF enabled; others use
   *    mode 1);
   * 3: one kernel per 64x64 tile stages the tile and 8 samples of halo on
   *    every side once, filters the vertical edges (halo rows included) and
   *    then the horizontal edges in shared memory, and writes the tile. */
  int32_t lf_mode;
  /* 0: per frame shape, as measured (64 while unmeasured); 32 or 64: the
   *    width of the loop-restoration rectangles one CTA restores. */
  int32_t lr_rect_cols;
} av1pf_tuning;

/* Sets / reads the context's variant choices (chain, chain_host, batches
 * created afterwards, and servers created from the context). */
int av1pf_set_tuning(av1pf_ctx* ctx, const av1pf_tuning* tuning);
int av1pf_get_tuning(av1pf_ctx* ctx, av1pf_tuning* tuning);

/* Times every variant on the first job of each frame shape (frame and
 * upscaled width, height, bit depth, subsampling, planes) among `jobs`, as
 * a one-frame batch replayed `reps` times, and records the fastest per
 * shape in the context. The jobs' outputs are overwritten. Shapes already
 * recorded are measured again. *n_shapes (may be NULL) = shapes measured. */
int av1pf_autotune(av1pf_ctx* ctx, const av1pf_job* jobs, int n_jobs, int32_t reps, int32_t* n_shapes);

/* The recorded choice for the shape of `info` (lf_mode 0-3 and
 * lr_rect_cols) and its measured device time per frame in ms;
 * AV1PF_ERR_NOT_FOUND when the shape has not been measured. */
int av1pf_tuned_choice(av1pf_ctx* ctx, const av1pf_frame_info* info, av1pf_tuning* choice, float* ms);

/* ------------------------------------------------------------------------ */
/* Serving: continuous batching of post-filter jobs from many streams.       */
/* ------------------------------------------------------------------------ */
typedef struct av1pf_server av1pf_server;

typedef struct av1pf_serve_config {
  uint64_t hbm_cap_bytes;  /* admission cap on resident stream + batch memory */
  int32_t max_batch_frames; /* most frames one tick takes (0 = 64) */
  int32_t inflight_batches; /* batches on the device at once (0 = 2) */
  int32_t tick_us;          /* longest wait for more work before a tick */
  int32_t slots_per_stream; /* frames of one stream resident at once (0 = 2);
                               more slots let one batch take more of a
                               stream's queued frames */
} av1pf_serve_config;

/* A submitted frame. With device == 0, `maps` and `in` are host pointers,
 * copied at submit time, and av1pf_serve_poll returns the packed frame. With
 * device != 0 they are device pointers (a decoder that produced the planes
 * on the GPU), which must stay valid until the frame completes; the server
 * reads them in place and writes the reference frame to `ref_out` and the
 * packed frame to `frame_out` (device pointers; either may be NULL). */
typedef struct av1pf_request {
  const av1pf_frame_info* info;
  const av1pf_params* params;
  const av1pf_maps* maps;
  const av1pf_plane* in;
  int32_t device;
  av1pf_plane* ref_out;    /* device requests only */
  uint8_t* frame_out;      /* device requests only */
} av1pf_request;

typedef struct av1pf_serve_stats {
  uint64_t submitted, completed, refused, batches;
  double p50_ms, p99_ms, mean_batch_frames;
  uint64_t resident_bytes;
} av1pf_serve_stats;

int av1pf_serve_open(av1pf_ctx* ctx, const av1pf_serve_config* cfg,
                     av1pf_server** out);
/* Registers a stream: its device planes and maps stay resident until
 * av1pf_serve_close_stream. Admission is by free HBM under the cap. */
int av1pf_serve_open_stream(av1pf_server* s, const av1pf_frame_info* info,
                            int32_t* stream_id);
/* Waits for the stream's queued and running frames, then frees its slots.
 * Results of host requests not polled yet go with them: polling such a
 * ticket afterwards returns AV1PF_ERR_NOT_FOUND. */
int av1pf_serve_close_stream(av1pf_server* s, int32_t stream_id);
/* Queues one frame of `stream_id`; returns a ticket. Never blocks on the GPU. */
int av1pf_serve_submit(av1pf_server* s, int32_t stream_id,
                       const av1pf_request* req, uint64_t* ticket);
/* Queues n frames (frame k of stream stream_ids[k]) under one lock, in
 * order, so one tick can batch them together; tickets[k] receives frame k's
 * ticket. All or nothing: if one request is refused, none is queued. A
 * group of host requests is copied into staging by up to 8 threads. */
int av1pf_serve_submit_many(av1pf_server* s, int32_t n, const int32_t* stream_ids,
                            const av1pf_request* reqs, uint64_t* tickets);
/* Waits up to `wait_ms` for `ticket`; on completion copies the packed output
 * frame to `frame_out` (av1pf_frame_bytes bytes; may be NULL) and returns the
 * submit->completion latency. AV1PF_ERR_TIMEOUT if not done in time. */
int av1pf_serve_poll(av1pf_server* s, uint64_t ticket, int32_t wait_ms,
                     uint8_t* frame_out, double* latency_ms);
int av1pf_serve_stats_get(av1pf_server* s, av1pf_serve_stats* out);
int av1pf_serve_close(av1pf_server* s);

/* ------------------------------------------------------------------------ */
/* Encoder filter searches: the encoder's choice of loop-filter levels and   */
/* CDEF strengths, every candidate filtered and scored on the device.        */
/* ------------------------------------------------------------------------ */

/* Candidate (primary, secondary) strength pairs of the CDEF search
 * (encoder/cdef.rs:60-80): luma primaries {0,1,2,4,6,9,12} (thorough:
 * {0,1,2,3,4,5,6,8,10,12,15}) x coded secondaries {0,1,2,3}; chroma
 * primaries {0,1,2,4,7} (thorough: {0,1,2,3,4,6,8,11}) x {0,1,2}; pairs
 * ordered primary-major. */
#define AV1PF_CDEF_SEARCH_NY 28
#define AV1PF_CDEF_SEARCH_NUV 15
#define AV1PF_CDEF_SEARCH_NY_THOROUGH 44
#define AV1PF_CDEF_SEARCH_NUV_THOROUGH 24

/* CdefParams (encoder/cdef.rs:18-29): 1 << bits index entries; secondary
 * strengths as coded (3 means 4, 6.10.14). */
typedef struct av1pf_cdef_search_result {
  int32_t damping_minus_3;
  int32_t bits;
  int32_t y_pri[8], y_sec[8];
  int32_t uv_pri[8], uv_sec[8];
} av1pf_cdef_search_result;

/* cdef::search (encoder/cdef.rs:52-251). `cur` holds the deblocked frame and
 * `src` the source planes (device planes in the frame's sample format, at
 * least mi_cols*4 x mi_rows*4 luma samples readable in `cur`, the frame area
 * in `src`); `maps` (device) gives the mode info (skip flags) and the
 * first pass's cdef_idx table, whose entries >= 0 mark the 64x64 blocks that
 * code an index. Every candidate strength pair filters every 8x8 block CDEF
 * would filter, with the decoder's direction search and filter, and its
 * squared error against the source inside the frame is summed per 64x64
 * block, luma and chroma apart; then up to eight (luma, chroma) pairs are
 * chosen greedily to minimise the error plus lambda * bits per block, and
 * each block takes its best.
 * Writes the result to `result` (host) and the table to `cdef_idx_out`
 * (host, cdef_stride * ceil(mi_rows/16) entries: the input table with each
 * coding block's chosen index). `block_sse` (host, may be NULL) receives the
 * per-block errors: ceil(mi_rows/16) * ceil(mi_cols/16) blocks in raster
 * order, each NY luma then NUV chroma u64 sums (zero for blocks that code no
 * index). Returns once the outputs are on the host. */
int av1pf_cdef_search(av1pf_ctx* ctx, const av1pf_frame_info* info,
                      const av1pf_maps* maps, const av1pf_plane* cur,
                      const av1pf_plane* src, int32_t base_q_idx,
                      double lambda, int32_t thorough,
                      av1pf_cdef_search_result* result, int8_t* cdef_idx_out,
                      uint64_t* block_sse, void* stream);

/* One frame of av1pf_cdef_search_many: the arguments of av1pf_cdef_search. */
typedef struct av1pf_cdef_search_job {
  const av1pf_frame_info* info;
  const av1pf_maps* maps;    /* device */
  const av1pf_plane* cur;    /* device */
  const av1pf_plane* src;    /* device */
  int32_t base_q_idx;
  double lambda;
  av1pf_cdef_search_result* result; /* host */
  int8_t* cdef_idx_out;      /* host, or NULL */
  uint64_t* block_sse;       /* host, or NULL */
} av1pf_cdef_search_job;

/* av1pf_cdef_search for n frames (shapes may differ) in one call: one launch
 * scores every frame's blocks and each greedy step advances every frame, so
 * small frames share the device and the per-call costs (an encoder's
 * lookahead or the rungs of a resolution ladder). Each result equals that of
 * av1pf_cdef_search on its frame. n <= 4096. */
int av1pf_cdef_search_many(av1pf_ctx* ctx, int n, const av1pf_cdef_search_job* jobs,
                           int32_t thorough, void* stream);

/* One frame of av1pf_lf_search_many: the arguments of av1pf_lf_search, the
 * chosen levels written into it. */
typedef struct av1pf_lf_search_job {
  const av1pf_frame_info* info;
  const av1pf_params* params;
  const av1pf_maps* maps;    /* device */
  const av1pf_plane* cur;    /* device */
  const av1pf_plane* src;    /* device */
  int32_t levels_out[4];     /* written */
  uint64_t* sse_out;         /* host 6 x 3, or NULL */
} av1pf_lf_search_job;

/* av1pf_lf_search for n frames in one call: every frame's filtered scales
 * run as one batch and every error in one launch. Each frame's result
 * equals that of av1pf_lf_search on it. n <= 1024. */
int av1pf_lf_search_many(av1pf_ctx* ctx, int n, av1pf_lf_search_job* jobs, void* stream);

/* Effort of the loop-restoration search (encoder/lr.rs:47-58): fast fits
 * on every other row and column and tries 2 self-guided parameter sets,
 * normal 6, thorough all 16. */
enum { AV1PF_LR_FAST = 0, AV1PF_LR_NORMAL = 1, AV1PF_LR_THOROUGH = 2 };

/* lr::search (encoder/lr.rs:64-210): each restoration unit's filter — none,
 * a Wiener filter fitted to the source by least squares, or a self-guided
 * filter with fitted projection weights for each parameter set tried — the
 * cheapest of error + lambda * (1, 40 or 28 for a luma or chroma Wiener
 * filter, 20), measured with the decoder's own restoration over the samples
 * it reads; and each plane's frame restoration type (0 none, 1 Wiener,
 * 2 self-guided, 3 switchable). `params` gives the unit grid
 * (loop_restoration_size, lr_unit_rows, lr_unit_cols; the restoration
 * types are ignored); `cur` (deblocked frame, read at stripe boundaries),
 * `cdef` (CDEF output) and `src` are device planes covering the visible
 * frame. Writes units_out[p] (host, lr_unit_rows[p] * lr_unit_cols[p]
 * entries, NULL to skip a plane) and frame_type_out. Any finite lambda.
 * Returns once the outputs are on the host. */
int av1pf_lr_search(av1pf_ctx* ctx, const av1pf_frame_info* info,
                    const av1pf_params* params, const av1pf_plane* cur,
                    const av1pf_plane* cdef, const av1pf_plane* src,
                    double lambda, int32_t effort,
                    av1pf_lr_unit* const units_out[3],
                    int32_t frame_type_out[3], void* stream);

/* One frame of av1pf_lr_search_many: the arguments of av1pf_lr_search, with
 * its outputs inside. */
typedef struct av1pf_lr_search_job {
  const av1pf_frame_info* info;
  const av1pf_params* params;
  const av1pf_plane* cur;   /* device */
  const av1pf_plane* cdef;  /* device */
  const av1pf_plane* src;   /* device */
  double lambda;
  av1pf_lr_unit* units_out[3];  /* host, or NULL per plane */
  int32_t frame_type_out[3];    /* written */
} av1pf_lr_search_job;

/* av1pf_lr_search for n frames (shapes may differ, one effort) in one call:
 * every frame's units run in the same launches. Each frame's result equals
 * that of av1pf_lr_search on it. n <= 4096. */
int av1pf_lr_search_many(av1pf_ctx* ctx, int n, av1pf_lr_search_job* jobs,
                         int32_t effort, void* stream);

/* search_lf (encoder/mod.rs:1457-1506): the loop-filter levels with the
 * least error. `params` carries the starting levels (loop_filter_level) and
 * the other loop-filter fields the filter reads; `cur` (device, left
 * unchanged) is the unfiltered reconstruction and `src` the source planes.
 * The six scales {0, 0.5, 0.75, 1, 1.25, 1.5} of the starting levels are
 * filtered as one batch, and each plane's squared error against the source
 * inside the frame picks that plane's level. Writes the chosen levels to
 * `levels_out` (host) and, when `sse_out` is not NULL, the 6 x 3 errors
 * (scale-major; zero for absent planes). Returns once they are on the host. */
int av1pf_lf_search(av1pf_ctx* ctx, const av1pf_frame_info* info,
                    const av1pf_params* params, const av1pf_maps* maps,
                    const av1pf_plane* cur, const av1pf_plane* src,
                    int32_t levels_out[4], uint64_t* sse_out, void* stream);

/* ------------------------------------------------------------------------ */
/* DSP entry points: the reference's src/dsp post-filter kernels over many   */
/* independent inputs at once (device pointers), for conformance tests.     */
/* ------------------------------------------------------------------------ */

/* dsp::lf::Params (lf.rs:14-21). */
typedef struct av1pf_lf_edge_params {
  int32_t limit, blimit, thresh;
  int32_t filter_size; /* 4, 6, 8 or 16 */
  int32_t chroma;
  int32_t bit_depth;
} av1pf_lf_edge_params;

/* dsp::lf::filter (lf.rs:25) on `n` edges: edges[e*56 + k*4 + lane] is
 * sample k (q0 at 7) of lane `lane`, filtered in place. */
int av1pf_dsp_lf_filter(av1pf_ctx* ctx, int32_t* edges,
                        const av1pf_lf_edge_params* params, int n, void* stream);

/* dsp::cdef::Taps (cdef.rs:13-25); offsets are in a 12-wide window. */
typedef struct av1pf_cdef_taps {
  int32_t pri_str, sec_str, pri_adj, sec_adj;
  int32_t pri_taps[2], sec_taps[2];
  int32_t pri_off[2];
  int32_t sec_off[2][2];
  int32_t w, h; /* block: 8x8, 4x4, 4x8 or 8x4 */
} av1pf_cdef_taps;

/* dsp::cdef::filter (cdef.rs:29) on `n` windows: win[e*144 ..] is a 12x12
 * window (INT32_MIN = unavailable), result res[e*64 ..] with row stride w. */
int av1pf_dsp_cdef_filter(av1pf_ctx* ctx, const int32_t* win,
                          const av1pf_cdef_taps* taps, uint16_t* res, int n,
                          void* stream);

/* Per-stage device timing of the per-frame entry points (diagnostics). When
 * on, every av1pf_chain / per-stage call records CUDA events on its stream
 * between stages. */
int av1pf_set_profiling(av1pf_ctx* ctx, int on);
/* Sums, in milliseconds, of the stage times of every profiled call since the
 * last read: [0] loop filter, [1] CDEF, [2] superres, [3] loop restoration,
 * [4] output (film grain + packing); *calls = number of calls summed. Waits
 * for those calls to finish, then resets the sums. */
int av1pf_stage_times(av1pf_ctx* ctx, float ms[5], uint32_t* calls);

/* Last CUDA error string seen by this thread (diagnostics). */
const char* av1pf_last_error(void);

/* Count of device kernel launches this library has issued in this process
 * (every stage launch, graph launches counted by the kernels they hold). */
uint64_t av1pf_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* AV1PF_H */
