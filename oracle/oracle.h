/*
 * oracle.h — CPU restatement of the reference's AV1 post-filter chain.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA path and
 * the timed CPU baseline ("port"); the product (libav1pf) never links, loads
 * or calls it. It restates rivet-av1's src/decoder/postfilter.rs,
 * src/dsp/lf.rs, src/dsp/cdef.rs, src/decoder/grain.rs and the chain/output
 * of src/decoder/mod.rs:747-917, function by function, in 16-bit samples as
 * the reference keeps them.
 *
 * Parity status: pinned by the reference's own known-answer tests for the
 * path (the loop-filter lane kernel against the one-sample process of 7.14.6,
 * lf.rs:213-353, and the CDEF block filter cases of cdef.rs:244-312), both
 * restated here with the reference's xorshift seeds. At the frame boundary
 * (whole planes in, planes out) parity with the reference's own binary is
 * UNPINNED: the reference is Rust, no Rust toolchain exists here, and the
 * reference ships no pre/post-filter plane dumps.
 */
#ifndef AV1PF_ORACLE_H
#define AV1PF_ORACLE_H

#include "av1pf.h"

#ifdef __cplusplus
extern "C" {
#endif

/* All planes/maps are HOST pointers. `threads` follows set_threads: 0 = all
 * hardware threads, 1 = serial. Return AV1PF_OK or AV1PF_ERR_INVALID_INPUT. */

/* loop_filter_threads (postfilter.rs:67), in place. */
int oracle_loop_filter(const av1pf_frame_info* info, const av1pf_params* p,
                       const av1pf_maps* maps, av1pf_plane* planes, int threads);
/* cdef (postfilter.rs:273): out = clone of cur, filtered. */
int oracle_cdef(const av1pf_frame_info* info, const av1pf_params* p,
                const av1pf_maps* maps, const av1pf_plane* cur, av1pf_plane* out,
                int threads);
/* upscale (postfilter.rs:521). */
int oracle_superres(const av1pf_frame_info* info, const av1pf_params* p,
                    const av1pf_plane* in, av1pf_plane* out);
/* loop_restoration (postfilter.rs:608): out = clone of cdef, restored. */
int oracle_loop_restoration(const av1pf_frame_info* info, const av1pf_params* p,
                            const av1pf_maps* maps, const av1pf_plane* cur,
                            const av1pf_plane* cdef, av1pf_plane* out, int threads);
/* Decoder::output (decoder/mod.rs:846-917): crop, grain, pack. */
int oracle_output(const av1pf_frame_info* info, const av1pf_params* p,
                  const av1pf_plane* ref, uint8_t* frame_out);
/* decode_frame_wrapup's chain (decoder/mod.rs:748-759) + output. `ref_out`
 * receives the LR frame's visible area; frame_out may be NULL. */
int oracle_chain(const av1pf_frame_info* info, const av1pf_params* p,
                 const av1pf_maps* maps, const av1pf_plane* in,
                 av1pf_plane* ref_out, uint8_t* frame_out, int threads);

/* dsp::lf::filter_lanes (lf.rs:58-211) on n edges (56 ints each, in place). */
void oracle_lf_filter_lanes(int32_t* edges, const av1pf_lf_edge_params* p, int n);
/* The one-sample process of 7.14.6 (lf.rs:218-306), lane by lane. */
void oracle_lf_reference(int32_t* edges, const av1pf_lf_edge_params* p, int n);
/* The random edges of lanes_match_the_process (lf.rs:309-353): `cases` edges
 * from the reference's xorshift seed, written to edges/params. */
void oracle_lf_kat_cases(uint64_t seed, int cases, int32_t* edges,
                         av1pf_lf_edge_params* params);
/* dsp::cdef::filter_scalar (cdef.rs:54-90) on n windows. */
void oracle_cdef_filter(const int32_t* win, const av1pf_cdef_taps* taps,
                        uint16_t* res, int n);
/* The random windows of simd_matches_scalar (cdef.rs:250-311): `cases`
 * windows x 3 block shapes -> 3*cases entries. */
void oracle_cdef_kat_cases(uint64_t seed, int cases, int32_t* win,
                           av1pf_cdef_taps* taps);

/* cdef::search (encoder/cdef.rs:52-251): outputs as av1pf_cdef_search
 * (host pointers; block_sse and cdef_idx_out may be NULL). */
int oracle_cdef_search(const av1pf_frame_info* info, const av1pf_maps* maps,
                       const av1pf_plane* cur, const av1pf_plane* src,
                       int32_t base_q_idx, double lambda, int32_t thorough,
                       av1pf_cdef_search_result* result, int8_t* cdef_idx_out,
                       uint64_t* block_sse, int threads);
/* search_lf (encoder/mod.rs:1457-1506): outputs as av1pf_lf_search. */
int oracle_lf_search(const av1pf_frame_info* info, const av1pf_params* p,
                     const av1pf_maps* maps, const av1pf_plane* cur,
                     const av1pf_plane* src, int32_t levels_out[4],
                     uint64_t* sse_out, int threads);
/* lr::search (encoder/lr.rs:64-210): outputs as av1pf_lr_search (host
 * pointers; units_out[p] may be NULL). */
int oracle_lr_search(const av1pf_frame_info* info, const av1pf_params* p,
                     const av1pf_plane* cur, const av1pf_plane* cdef,
                     const av1pf_plane* src, double lambda, int32_t effort,
                     av1pf_lr_unit* const units_out[3], int32_t frame_type_out[3],
                     int threads);

#ifdef __cplusplus
}
#endif
#endif
