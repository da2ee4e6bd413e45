/*
 * ironav_inter.h — C ABI of the P-picture inter-analysis stage of IronAV's software H.264 encoder
 * (crate ironav-codec, module h264::enc), re-implemented for NVIDIA B200 (sm_100a).
 *
 * The stage covers:
 *   - the half-sample planes of each reference picture      (HalfPel::new, enc/subpel.rs:42-115)
 *   - the P_Skip vector and its SAD                          (code_mb, enc/frame.rs:722-729; skip_mv 597-603)
 *   - the inter partition decision with motion search       (best_inter, enc/frame.rs:839-938;
 *                                                             motion_search 949-1019)
 * and, around it, the steps either side that keep a P picture on the device: the coding of inter
 * macroblocks once decided (code_inter, enc/frame.rs:1202-1305), the whole CAVLC macroblock decision
 * with intra prediction (decide mode: code_mb, enc/frame.rs:715-790), B-picture searches, the deblocking
 * filter and the scene-cut measure. Entropy coding and the CABAC rate-distortion decision (decide_rd,
 * enc/frame.rs:1462-1513) stay with the caller.
 *
 * Two libraries implement this header:
 *   libironav_inter_cuda.so  the product: CUDA kernels for sm_100a (ironav_b200/).
 *   libironav_inter_cpu.so   the CPU restatement used as the parity checker (oracle/).
 * A caller switches between them by linking the other library; every entry point, argument and
 * status code means the same in both.
 *
 * Conventions
 *   - Plain C types, caller-owned host buffers unless a name ends in _device (device pointers,
 *     work queued on the context's stream, no host synchronisation).
 *   - Vectors are in quarter luma samples, (x, y), int16, exactly as the encoder keeps them.
 *   - Macroblocks are numbered in raster order, mb_w * mb_h of them, mb_w = ceil(width / 16).
 *   - Every entry point returns an ironav_status; none throws, none aborts.
 *   - A context is not thread-safe; many contexts may live in one process.
 */
#ifndef IRONAV_INTER_H
#define IRONAV_INTER_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: 1 + the index of ironav_core::ErrorCode (crates/ironav-core/src/error.rs:9-27), so a
 * Rust binding maps them back with ErrorCode::ALL[status - 1]. IRONAV_TIMEOUT has no counterpart
 * there (the reference never waits on another device); a binding maps it to ErrorCode::Internal. */
typedef enum ironav_status {
    IRONAV_OK = 0,
    IRONAV_INVALID_INPUT = 2,         /* ErrorCode::InvalidInput: a frame or state that does not fit the context */
    IRONAV_INVALID_ARGUMENT = 3,      /* ErrorCode::InvalidArgument: bad sizes, null pointers, out-of-range params */
    IRONAV_HARDWARE_UNAVAILABLE = 8,  /* ErrorCode::HardwareUnavailable: no CUDA device / kernels not loadable */
    IRONAV_INTERNAL = 13,             /* ErrorCode::Internal: a CUDA call failed */
    IRONAV_TIMEOUT = 100              /* a bounded device-side wait gave up (wavefront dependency never published) */
} ironav_status;

/* What later macroblocks need to know about a decided one: the list-0 subset of MbState
 * (enc/frame.rs:246-272) that the vector predictors read (nb_motion, enc/frame.rs:522-538), and, for
 * the newest reference picture, what col_mv (enc/frame.rs:944-947) reads of MbInfo (h264/mb.rs:34-64). */
typedef struct ironav_mbstate {
    uint8_t inter;        /* Kind::Inter (P_L0_*, P_8x8 and P_Skip); 0 for intra or not coded */
    int8_t refs[4];       /* refs[0]: ref_idx_l0 per 8x8 block, -1 for none */
    uint8_t pad[3];
    int16_t mvs[16][2];   /* list-0 vector per 4x4 block, raster order */
} ironav_mbstate;         /* 72 bytes */

/* The stage's answer for one macroblock. */
typedef struct ironav_mbresult {
    int16_t skip_mv[2];   /* P_Skip vector (8.4.1.1), skip_mv enc/frame.rs:597-603 */
    int32_t skip_sad;     /* SAD of the 16x16 P_Skip prediction against the source, enc/frame.rs:725-729 */
    uint8_t part;         /* best_inter: 0 16x16, 1 16x8, 2 8x16, 3 8x8 (PARTS, enc/frame.rs:182) */
    uint8_t refs[4];      /* best_inter: reference index of each partition / 8x8 block */
    uint8_t sub[4];       /* best_inter: sub_mb_type of each 8x8 block of P_8x8 (SUB, enc/frame.rs:204) */
    uint8_t flags;        /* IRONAV_RESULT_* below */
    uint8_t pad[2];
    int32_t cost;         /* best_inter: SATD + lambda * (mv, mb_type, ref bits) of the winner */
    int16_t mvs[16][2];   /* best_inter: vector of each partition in coding order (rects, enc/frame.rs:208-213) */
    int32_t cost16;       /* the 16x16 candidate's cost for the winning reference */
    uint32_t sad_px;      /* samples compared by integer SAD evaluations in the reference's order (work count) */
    uint32_t satd_px;     /* samples compared by sub-sample SATD evaluations (work count) */
    uint32_t pad2;
} ironav_mbresult;        /* 104 bytes */

#define IRONAV_RESULT_INTER 1u   /* best_inter was evaluated (fields part..cost16 are valid) */
#define IRONAV_RESULT_SKIP  2u   /* auto policy only: the macroblock was decided as P_Skip */

/* ---- host helpers (f64 arithmetic that the reference does on the host) -------------------------- */

/* lambda(qp') = max(1, round(2^((qp' - 12) / 6))), enc/frame.rs:164-166. */
int ironav_lambda(int qp_prime);
/* Smallest integer T with (sad < T) <=> (sad as f64 < 256 * 0.625 * 2^(qp'/6)), the P_Skip test of
 * enc/frame.rs:730,742 rewritten on integers. */
int ironav_skip_threshold(int qp_prime);
/* Bits of se(v) / ue(v) Exp-Golomb codes, enc/bitw.rs:81-89. */
int ironav_se_bits(int v);
int ironav_ue_bits(unsigned v);
/* Version string of the implementation ("cuda-sm_100a ..." or "cpu-oracle ..."). */
const char* ironav_version(void);

/* ---- context -------------------------------------------------------------------------------------- */

typedef struct ironav_ctx ironav_ctx;

/* One stream: width x height luma of bd = 8 or 10 bits (the encoder's Yuv420p and Yuv420p10 formats,
 * enc/mod.rs:140-143; even sizes, mb_w and mb_h <= 1024 like H264Encoder::new, enc/mod.rs:143-152), up to max_refs reference pictures (1..16, with_refs enc/mod.rs:265-268), and
 * nslices slice bands. band_rows holds nslices + 1 macroblock-row boundaries, or is NULL for the
 * encoder's own split, band i = [i*mb_h/n, (i+1)*mb_h/n) (enc/mod.rs:603). Neighbours in an earlier
 * band are unavailable to the vector predictors (nb_state, enc/frame.rs:509-515). */
int ironav_ctx_create(ironav_ctx** out, int width, int height, int bd, int max_refs, int nslices,
                      const int* band_rows);
int ironav_ctx_destroy(ironav_ctx* ctx);
/* Geometry: mb_w, mb_h, and the padded plane size sw x sh of each half-sample plane
 * (sw = 16*mb_w + 96, sh = 16*mb_h + 96, PAD = 48 on each side, enc/subpel.rs:7). */
int ironav_ctx_dims(const ironav_ctx* ctx, int* mb_w, int* mb_h, int* sw, int* sh);
/* Makes the context queue its device work on this cudaStream_t (NULL: the legacy default stream). */
int ironav_ctx_set_stream(ironav_ctx* ctx, void* cuda_stream);

/* Sample buffers. Every luma buffer the entry points below take or fill holds samples of the context's
 * depth: uint8_t when bd = 8, uint16_t (host byte order, values below 2^bd) when bd = 10, as the
 * reference's Source keeps them (enc/mod.rs:486-526). Strides count samples, not bytes. */

/* The picture to analyse: width x height luma, rows `stride` samples apart, padded to whole macroblocks
 * by repeating its right and bottom edges (H264Encoder::source, enc/mod.rs:481-529). */
int ironav_set_source(ironav_ctx* ctx, const void* y, int stride);

/* Adds the newest reference picture (a decoded/reconstructed luma plane) and builds its half-sample
 * planes (HalfPel::new, enc/subpel.rs:42-115; the reference list, enc/mod.rs:551-559,660-666). w x h is
 * either the picture size (edges repeated to whole macroblocks) or the macroblock-aligned size
 * 16*mb_w x 16*mb_h (a reconstruction, used as is). col holds the picture's own macroblock decisions
 * (mb_w*mb_h), read for the co-located candidate (col_mv, enc/frame.rs:944-947), or NULL when the
 * picture was intra coded. The oldest reference is dropped once max_refs are held. */
int ironav_push_reference(ironav_ctx* ctx, const void* y, int stride, int w, int h,
                          const ironav_mbstate* col);
/* Forgets every reference (an IDR picture, enc/mod.rs:541-545). */
int ironav_clear_references(ironav_ctx* ctx);
/* Copies reference `idx` (0 = newest) planes G, b, h, j to out (4 * sw * sh samples), for checks. */
int ironav_get_planes(ironav_ctx* ctx, int idx, void* out);

/* Parameters of the P picture to analyse (FrameCoder::new / with_sub8x8 / with_fast,
 * enc/frame.rs:381-440): qp_prime = QP'Y; lambda and skip_thresh from the helpers above (the host
 * works them out in f64 like the reference); nrefs_active = list-0 length (enc/mod.rs:559);
 * fast = H264Encoder::realtime's shorter search; sub8 = sub-partitions of P_8x8 searched. */
int ironav_begin_p_picture(ironav_ctx* ctx, int qp_prime, int lambda, int skip_thresh, int nrefs_active,
                           int fast, int sub8);

/* Replay mode: final_states holds every macroblock's final decision (mb_w*mb_h), as the caller's
 * mode decision made it; each macroblock is analysed against its neighbours' final states, so all
 * macroblocks are independent. out receives mb_w*mb_h results, with P_Skip and best_inter for every
 * macroblock. */
int ironav_analyse_picture_replay(ironav_ctx* ctx, const ironav_mbstate* final_states,
                                  ironav_mbresult* out);

/* Auto mode: the stage decides every macroblock itself with the analysis policy (P_Skip when
 * skip_sad < skip_thresh, else the best_inter result) and the macroblocks follow their left, top and
 * top-right neighbours' decisions in a wavefront within each slice band. out_states receives the
 * decisions (usable as the next picture's col and as replay input). */
int ironav_analyse_picture_auto(ironav_ctx* ctx, ironav_mbstate* out_states, ironav_mbresult* out);

/* ---- device-resident forms (pointers in device memory; asynchronous on the context's stream) ------ */

int ironav_set_source_device(ironav_ctx* ctx, const void* d_y, int stride);
int ironav_push_reference_device(ironav_ctx* ctx, const void* d_y, int stride, int w, int h,
                                 const ironav_mbstate* d_col);
int ironav_analyse_picture_replay_device(ironav_ctx* ctx, const ironav_mbstate* d_final_states,
                                         ironav_mbresult* d_out);
int ironav_analyse_picture_auto_device(ironav_ctx* ctx, ironav_mbstate* d_out_states,
                                       ironav_mbresult* d_out);
/* Waits for the context's queued work; returns a pending device error (IRONAV_TIMEOUT for a wavefront
 * wait that gave up). */
int ironav_ctx_sync(ironav_ctx* ctx);

/* ---- scene-cut measure ------------------------------------------------------------------------------ */

/* How well cur_y is predicted from prev_y against from itself (change_threads, codec/change.rs:56-90), on
 * the low-resolution luma the encoder takes of its padded source (H264Encoder::low_res, enc/mod.rs:689-693;
 * LowRes::new, codec/change.rs:16-24): out[0] = inter, out[1] = intra totals. The encoder starts an IDR
 * picture when (double)inter > 0.8 * (double)intra (SCENE_CUT, enc/mod.rs:707-711); the comparison stays
 * with the caller, in f64 like the reference. Both pictures are width x height, rows `stride` apart. */
int ironav_scene_change(ironav_ctx* ctx, const void* prev_y, const void* cur_y, int stride, int64_t* out);
/* The same on device pointers (returns when the totals are in out, a host array). */
int ironav_scene_change_device(ironav_ctx* ctx, const void* d_prev, const void* d_cur, int stride, int64_t* out);

/* ---- B pictures ------------------------------------------------------------------------------------- */

/* The searches of a B macroblock (decide_b, enc/frame.rs:1518-1572; best_b_parts 1626-1687; spatial direct
 * direct_mvs 1715-1747), in replay mode: every macroblock against its neighbours' final decisions. The
 * rate-distortion choice among B_Skip / B_Direct_16x16, the 16x16 and smaller partitionings and intra
 * stays with the caller, which codes the residuals (decide_b's rd_cost).
 *
 * A B macroblock's final decision as its neighbours' predictors see it (MbState with both lists,
 * enc/frame.rs:246-272): per list the reference index of each 8x8 block (-1: the list is not used there)
 * and the vector of each 4x4 block. */
typedef struct ironav_mbstate_b {
    uint8_t inter;
    int8_t refs[2][4];
    uint8_t pad[3];
    int16_t mvs[2][16][2];
} ironav_mbstate_b;                /* 140 bytes */

typedef struct ironav_bresult {
    int16_t direct_mv[2][16][2];   /* spatial direct vectors per list and 4x4 block */
    uint8_t direct_use[2];         /* the lists the direct prediction uses */
    uint8_t dir16;                 /* the best 16x16: 1 list 0, 2 list 1, 3 both averaged */
    uint8_t has_parts;             /* best_b_parts found a partitioning cheaper than the best 16x16 */
    uint8_t part;                  /* its partitioning: 1 16x8, 2 8x16, 3 8x8 */
    uint8_t bdir[4];               /* per partition: 0 direct (8x8 only), bit 0 list 0, bit 1 list 1 */
    uint8_t pad[3];
    int16_t mv16[2][2];            /* the 16x16 vector of each list */
    int32_t cost16[2];             /* per list: SATD + lambda (the vector's bits + 3) */
    int32_t cost_bi;               /* both lists averaged: SATD + lambda (both vectors' bits + 5) */
    int16_t pmv[2][4][2];          /* per list and partition, the partitioning's vectors */
    uint32_t sad_px, satd_px;      /* samples compared by SAD and by SATD, in the reference's order */
} ironav_bresult;                  /* 200 bytes */

/* Parameters of the B picture to analyse (FrameCoder for a B picture, enc/frame.rs:381-440): qp_prime and
 * lambda as for P pictures (the B picture's own QP'); ref_l0 / ref_l1: which held references (0 = newest)
 * are list 0 and list 1 (the encoder's refp and refp1, one picture each); col: the list-1 picture's own
 * decisions (mb_w*mb_h; its list-0 motion feeds spatial direct and the co-located candidate), or NULL
 * when it was intra coded; tb, td: the picture's distance from the list-0 picture and the distance between
 * the two (FrameCoder::dist), both nonzero; fast: H264Encoder::realtime's shorter search. col is copied
 * before the call returns; the _device form keeps the device pointer d_col, which must stay valid until
 * the pictures analysed with these parameters are done. */
int ironav_begin_b_picture(ironav_ctx* ctx, int qp_prime, int lambda, int ref_l0, int ref_l1, const ironav_mbstate* col,
                           int tb, int td, int fast);
int ironav_begin_b_picture_device(ironav_ctx* ctx, int qp_prime, int lambda, int ref_l0, int ref_l1,
                                  const ironav_mbstate* d_col, int tb, int td, int fast);
/* final_states: every macroblock's final decision (mb_w*mb_h); out: mb_w*mb_h results. */
int ironav_analyse_b_replay(ironav_ctx* ctx, const ironav_mbstate_b* final_states, ironav_bresult* out);
int ironav_analyse_b_replay_device(ironav_ctx* ctx, const ironav_mbstate_b* d_final_states, ironav_bresult* d_out);

/* ---- inter residual coding and reconstruction --------------------------------------------------------- */

/* The coding of inter macroblocks once their decisions are made (code_inter / code_inter_residual /
 * code_luma8 / code_chroma, enc/frame.rs:1202-1305, 1856-1915): the luma and chroma prediction, the
 * transform, quantisation and decimation of the residual, and the reconstruction. Every inter macroblock
 * is independent of its neighbours here, so a whole picture is coded at once; intra macroblocks (coded in
 * order against their neighbours' reconstruction) and the entropy coding stay with the caller.
 *
 * Chroma is 4:2:0. The source's chroma (width/2 x height/2, padded to 8*mb_w x 8*mb_h by repeating its
 * edges like the luma) and each reference picture's chroma (its reconstruction, 8*mb_w x 8*mb_h, or the
 * picture size to be padded) come in through: */
int ironav_set_source_chroma(ironav_ctx* ctx, const void* cb, const void* cr, int stride);
/* attaches chroma to reference 0 (the newest, as pushed with ironav_push_reference) */
int ironav_push_reference_chroma(ironav_ctx* ctx, const void* cb, const void* cr, int stride, int w, int h);

/* One macroblock's inter coding decision (code_inter's arguments). */
typedef struct ironav_interdec {
    uint8_t mode;          /* 0: not an inter macroblock (left alone); 1: P_Skip (the prediction is the
                              reconstruction, no residual); 2: coded with its residual */
    uint8_t part;          /* 0 16x16, 1 16x8, 2 8x16, 3 8x8 */
    uint8_t sub[4];        /* sub_mb_type per 8x8 block (part 3) */
    uint8_t refs[4];       /* reference index per partition (per 8x8 block for part 3) */
    uint8_t t8;            /* the 8x8 transform is tried (kept only when some luma is coded) */
    uint8_t pad[3];
    int16_t mvs[16][2];    /* one vector per partition, in coding order (rects(part, sub)) */
} ironav_interdec;         /* 78 bytes */

/* The coded residual of an inter macroblock (MbCode's levels; enc/frame.rs:1217-1305, 1856-1915). */
typedef struct ironav_intercode {
    int16_t luma[16][16];  /* 4x4 transform: the levels of each 4x4 block (raster order), zigzag order */
    int16_t luma8[4][64];  /* 8x8 transform (t8x8): the levels of each 8x8 block, 8x8 zigzag order */
    int16_t cdc[2][4];     /* chroma DC levels of Cb and Cr */
    int16_t cac[2][4][16]; /* chroma AC levels per 4x4 block, zigzag order (position 0 unused) */
    uint8_t nnz[16];       /* non-zero levels per 4x4 luma block (for the 8x8 transform: its 8x8 block's) */
    uint8_t cnnz[2][4];    /* non-zero AC levels per chroma 4x4 block */
    uint8_t cbp;           /* coded_block_pattern: luma in bits 0-3, chroma (0, 1 DC, 2 AC) in bits 4-5 */
    uint8_t t8x8;          /* the 8x8 transform is used */
    uint8_t pad[2];
} ironav_intercode;        /* 1324 bytes */

/* Codes the inter macroblocks of the current picture (the source set with ironav_set_source and
 * ironav_set_source_chroma) at QP_Y qp: decs and codes hold mb_w*mb_h entries; the reconstruction
 * planes (luma 16*mb_w x 16*mb_h, rows y_stride samples apart; chroma 8*mb_w x 8*mb_h, rows c_stride
 * apart) receive the inter macroblocks and keep every other macroblock as they were; the codes of a
 * macroblock that is not inter are zero. References are those held (0 = newest), each with its chroma. */
int ironav_code_inter_picture(ironav_ctx* ctx, int qp, const ironav_interdec* decs, ironav_intercode* codes, void* rec_y,
                              int y_stride, void* rec_cb, void* rec_cr, int c_stride);
/* The same on device pointers, queued on the context's stream; the reconstruction planes as for
 * ironav_deblock_picture_device (16-byte aligned, aligned row strides), d_decs 2-byte and d_codes 4-byte
 * aligned. */
int ironav_code_inter_picture_device(ironav_ctx* ctx, int qp, const ironav_interdec* d_decs, ironav_intercode* d_codes,
                                     void* d_rec_y, int y_stride, void* d_rec_cb, void* d_rec_cr, int c_stride);

/* ---- the P macroblock decision (decide mode) -------------------------------------------------------- */

/* The whole of code_mb for a P picture coded with CAVLC (enc/frame.rs:715-790): P_Skip when the skip
 * vector leaves nothing to code (the fast test on luma and chroma SADs, then code_inter's cbp == 0), else
 * the best Intra16x16 mode (best_i16, 812-835), the best inter partitioning (best_inter), Intra4x4 coded
 * block by block when intra is competitive (code_i4, 1050-1138), and the cheapest of them coded: inter
 * (code_inter), Intra4x4 or Intra16x16 (code_i16, 1140-1200) with intra chroma (code_intra_chroma,
 * 1807-1854). Macroblocks are decided in each slice band's raster order on the device (a wavefront: a
 * macroblock waits for its left and top-right neighbours), each against the final decisions and the
 * unfiltered reconstruction of those before it, as FrameCoder::encode does (452-487); the host is left
 * the entropy coding. The picture parameters are those of ironav_begin_p_picture (QP', lambda, the P_Skip
 * threshold, active references, fast, sub8x8); the source and every active reference need their chroma.
 * The code of one macroblock (MbCode, 275-300): */
typedef struct ironav_mbcode {
    ironav_intercode res;  /* levels: luma (4x4 blocks; Intra16x16: AC, scan position 0 unused), luma8 and
                              t8x8 (the 8x8 transform: Intra8x8, and inter macroblocks under CABAC with
                              transform8; CAVLC codes none), cdc, cac, nnz, cnnz, cbp (luma bits 0-3,
                              chroma 4-5) */
    int16_t dc[16];        /* Intra16x16 luma DC levels, zigzag order */
    int16_t mvs[16][2];    /* inter: a vector per partition in coding order (rects(part, sub)); P_Skip and
                              16x16: the vector in all 16 */
    int16_t mvds[16][2];   /* inter, not skipped: each vector less its predictor (part_mvps) */
    uint8_t modes[16];     /* Intra4x4 prediction modes, raster 4x4 order (Intra8x8: each 8x8 block's mode in
                              its four 4x4 blocks; 2 elsewhere) */
    uint8_t kind;          /* the reference's Kind: 1 Intra4x4, 2 Intra8x8 (CABAC with the 8x8 transform),
                              3 Intra16x16, 5 inter */
    uint8_t skip;          /* P_Skip */
    uint8_t i16_mode;      /* Intra16x16 prediction mode */
    uint8_t chroma_mode;   /* intra chroma prediction mode */
    uint8_t part;          /* inter partitioning */
    uint8_t sub[4];        /* sub_mb_type per 8x8 block (part 3) */
    uint8_t refs[4];       /* reference index per 8x8 block (per partition for 16x8 / 8x16) */
    uint8_t pad[3];
} ironav_mbcode;           /* 1516 bytes */

/* Decides and codes every macroblock of the current P picture: states receives each macroblock's
 * MbState (the ironav_mbstate a later picture reads as co-located; intra: inter 0, refs -1), codes the
 * codes, and the reconstruction planes (luma 16*mb_w x 16*mb_h, rows y_stride samples apart; chroma
 * 8*mb_w x 8*mb_h, rows c_stride apart) every macroblock's reconstruction before deblocking. */
int ironav_decide_p_picture(ironav_ctx* ctx, ironav_mbstate* states, ironav_mbcode* codes, void* rec_y, int y_stride, void* rec_cb,
                            void* rec_cr, int c_stride);
/* The same on device pointers, queued on the context's stream (planes as for
 * ironav_deblock_picture_device; states and codes 4-byte aligned). */
int ironav_decide_p_picture_device(ironav_ctx* ctx, ironav_mbstate* d_states, ironav_mbcode* d_codes, void* d_rec_y, int y_stride,
                                   void* d_rec_cb, void* d_rec_cr, int c_stride);

/* ---- High profile: CABAC with rate-distortion decisions ------------------------------------------- */

/* The entropy coding that decide mode and the slice writer follow (H264Encoder's cabac and transform8,
 * enc/mod.rs:136-283: the default encoder and low_latency code CABAC with the 8x8 transform,
 * constrained_baseline codes CAVLC). cabac = 0: CAVLC, a new context's setting; 1: CABAC. transform8
 * (CABAC only, else ignored) = transform_8x8_mode_flag. Under CABAC the decisions are FrameCoder's
 * decide_rd (enc/frame.rs:1462-1513): after code_mb's P_Skip tests (715-751), P_Skip, best_inter's
 * partitioning (4x4 transform, and with transform8 the 8x8 transform when no 8x8 block is split),
 * Intra16x16 in its best mode, Intra4x4 and (transform8) Intra8x8 (code_i8, 1307-1388), each with intra
 * chroma, are coded and the one of least SSD + lambda2 * bits is kept, lambda2 = 1.6 * 2^((QP'Y - 12) / 3)
 * and the bits those of CABAC (CabacCost, enc/cabac.rs:150-192) from the slice's contexts after the
 * macroblocks before it. Each slice band is then one chain in raster order: a macroblock's cost depends on
 * every earlier one's bins. The slices are written by ironav_write_slices with the same contexts. */
int ironav_set_entropy(ironav_ctx* ctx, int cabac, int transform8);

/* ---- intra (IDR) pictures in decide mode ------------------------------------------------------------ */

/* Parameters of an IDR picture (FrameCoder::new without a reference, enc/frame.rs:381-412; the encoder
 * codes IDR pictures at its QP - 3, QP_OFFSET enc/mod.rs:33): qp_prime = QP'Y, lambda from ironav_lambda,
 * fast = H264Encoder::realtime (flat macroblocks left to Intra16x16, enc/frame.rs:762-765). Replaces the
 * P picture's parameters until the next ironav_begin_p_picture. */
int ironav_begin_i_picture(ironav_ctx* ctx, int qp_prime, int lambda, int fast);
/* code_mb for every macroblock of the IDR picture (enc/frame.rs:752-790 with no reference: best_i16,
 * the Intra4x4 trial, code_i16 or the trial's blocks, code_intra_chroma), in each slice band's raster
 * order, each against the reconstruction of those before it; outputs as ironav_decide_p_picture's
 * (every state intra: inter 0, refs -1). Needs the source's luma and chroma; no reference is read. */
int ironav_decide_i_picture(ironav_ctx* ctx, ironav_mbstate* states, ironav_mbcode* codes, void* rec_y, int y_stride, void* rec_cb,
                            void* rec_cr, int c_stride);
int ironav_decide_i_picture_device(ironav_ctx* ctx, ironav_mbstate* d_states, ironav_mbcode* d_codes, void* d_rec_y, int y_stride,
                                   void* d_rec_cb, void* d_rec_cr, int c_stride);
/* ironav_set_source_chroma and ironav_push_reference_chroma on device pointers (queued on the context's
 * stream; the source's chroma is width/2 x height/2 samples, rows `stride` apart). */
int ironav_set_source_chroma_device(ironav_ctx* ctx, const void* d_cb, const void* d_cr, int stride);
int ironav_push_reference_chroma_device(ironav_ctx* ctx, const void* d_cb, const void* d_cr, int stride, int w, int h);

/* ---- the bitstream (Annex B) ------------------------------------------------------------------------ */

/* What the sequence and picture parameter sets say (H264Encoder::sps / pps, enc/mod.rs:296-400, without B
 * pictures: Constrained Baseline (CAVLC at 8 bits), Main (CABAC without the 8x8 transform), High (CABAC
 * with it) or High 10 (10 bits); picture order type 2, one slice group, no weighted prediction,
 * deblocking not signalled). */
typedef struct ironav_stream_params {
    int32_t width, height;       /* the picture size; the SPS crops the macroblock-aligned size to it */
    int32_t bd;                  /* 8 or 10 */
    int32_t fps_num, fps_den;    /* frame rate: the level (Table A-1, enc/mod.rs:154-157) and the VUI timing;
                                    0, 0: 25 fps for the level, no timing */
    int32_t refs;                /* max_num_ref_frames: reference pictures the stream keeps (1..16) */
    int32_t cabac;               /* entropy_coding_mode_flag (0 CAVLC, 1 CABAC) */
    int32_t transform8;          /* transform_8x8_mode_flag (with CABAC only) */
} ironav_stream_params;

/* The SPS and PPS NAL units (Annex B: 4-byte start codes, emulation prevention, put_nal enc/bitw.rs:91-103)
 * that the encoder puts ahead of every IDR picture (enc/mod.rs:636-640). Writes *len bytes to out;
 * IRONAV_INVALID_ARGUMENT when cap is too small (*len then says how many are needed). */
int ironav_write_parameter_sets(const ironav_stream_params* p, uint8_t* out, size_t cap, size_t* len);

/* The slice NAL units of the current picture (one per slice band, enc/mod.rs:641-643), from its codes
 * (ironav_decide_i_picture / ironav_decide_p_picture outputs, mb_w*mb_h): the slice header (enc/mod.rs:566-600),
 * each macroblock's CAVLC syntax (write_mb, enc/frame.rs:1922-2016: mb_skip_run, mb_type, prediction modes,
 * sub_mb_type, ref_idx, mvd, coded_block_pattern, mb_qp_delta, residual blocks by enc/cavlc.rs:47-122) and
 * the slice's trailing bits (enc/frame.rs:480-486); under CABAC (ironav_set_entropy) cabac_init_idc 0 in
 * the header, cabac_alignment_one_bit, and each macroblock's bins (write_mb_cabac / mb_bins,
 * enc/frame.rs:2020-2279, residual blocks by enc/cabac.rs:194-250) arithmetic coded (CabacWriter,
 * enc/cabac.rs:42-147) with end_of_slice_flag after each. idr: the picture is the IDR picture (slice type I, NAL
 * type 5, idr_pic_id) set up by ironav_begin_i_picture, else a P picture set up by ironav_begin_p_picture
 * (its active references give num_ref_idx_active and ref_idx's range); frame_num and idr_pic_id as the
 * encoder counts them (enc/mod.rs:541-545,667-668). Writes *len bytes of Annex B to out; IRONAV_INVALID_ARGUMENT
 * when cap is too small (*len then says how many are needed). */
int ironav_write_slices(ironav_ctx* ctx, int idr, int frame_num, int idr_pic_id, const ironav_mbcode* codes, uint8_t* out,
                        size_t cap, size_t* len);
/* The same from codes in device memory (4-byte aligned); out is a host buffer. Returns when the bytes
 * are in out. */
int ironav_write_slices_device(ironav_ctx* ctx, int idr, int frame_num, int idr_pic_id, const ironav_mbcode* d_codes,
                               uint8_t* out, size_t cap, size_t* len);

/* ---- deblocking of the reconstruction ------------------------------------------------------------ */

/* The in-loop deblocking filter (h264/deblock.rs:410-720, ITU-T H.264 8.7) of a reconstructed picture,
 * frame coded (not MBAFF) and 4:2:0 as the encoder codes it (enc/mod.rs:633,650-655), before the
 * picture becomes a reference (ironav_push_reference). The result is the reference's deblock_picture
 * (raster order), which deblock_picture_par reproduces with a macroblock-row wavefront; so does this.
 *
 * One macroblock as the filter sees it: the MbInfo fields deblock.rs reads (h264/mb.rs:34-68). */
typedef struct ironav_dbk_mb {
    uint16_t slice;         /* 1-based slice id (an index into the slice table + 1); 0: not coded, left alone */
    uint8_t inter;          /* 1: Kind::Inter (P or B, skipped or not); 0: an intra kind */
    int8_t qp;              /* QP_Y */
    uint8_t t8x8;           /* 8x8 transform: only the even luma edges are filtered */
    uint8_t keep;           /* I_PCM or lossless: its samples are put back after each filtered line */
    uint8_t pad[2];
    uint8_t nnz[16];        /* non-zero coefficient counts of the 16 luma 4x4 blocks, raster order */
    int8_t ref_idx[2][4];   /* per list and 8x8 block; -1 when the list is not used */
    int32_t ref_id[2][4];   /* identity of the picture behind ref_idx; -1 when not used */
    int16_t mv[2][16][2];   /* per list and 4x4 block, quarter samples */
} ironav_dbk_mb;            /* 192 bytes */

/* A slice's filter parameters (SliceParams, h264/mb.rs:115-120). */
typedef struct ironav_dbk_slice {
    int32_t disable_deblocking;   /* 0: filter; 1: leave the slice alone; 2: not across its edges */
    int32_t alpha_offset;         /* FilterOffsetA */
    int32_t beta_offset;          /* FilterOffsetB */
    int32_t chroma_qp_offset[2];  /* Cb, Cr */
} ironav_dbk_slice;

/* The filter's record of every macroblock decide mode coded, as finish_mb makes MbInfo
 * (enc/frame.rs:2323-2339): the slice id (band + 1, enc/mod.rs:608), inter or not, QP_Y of the picture's
 * parameters, t8x8 and the luma coefficient counts of its code, and for an inter macroblock list 0's
 * reference index per 8x8 block with its identity (1 + index) and the vectors of its state. codes and
 * states are one picture's ironav_decide_p_picture outputs; mbs receives mb_w*mb_h records. */
int ironav_decide_dbk_records(ironav_ctx* ctx, const ironav_mbcode* codes, const ironav_mbstate* states, ironav_dbk_mb* mbs);
/* The same on device pointers (4-byte aligned), queued on the context's stream. */
int ironav_decide_dbk_records_device(ironav_ctx* ctx, const ironav_mbcode* d_codes, const ironav_mbstate* d_states, ironav_dbk_mb* d_mbs);

/* Filters a picture of the context's size and sample depth in place: luma 16*mb_w x 16*mb_h samples,
 * rows y_stride samples apart; Cb and Cr 8*mb_w x 8*mb_h, rows c_stride apart (the layout of
 * Picture::planes). mbs: mb_w*mb_h records; slices: nslices entries, the slice ids of mbs index them.
 * A slice id above nslices gives IRONAV_INVALID_INPUT (the picture is then left partly filtered). */
int ironav_deblock_picture(ironav_ctx* ctx, void* y, int y_stride, void* cb, void* cr, int c_stride,
                           const ironav_dbk_mb* mbs, const ironav_dbk_slice* slices, int nslices);
/* The same on device pointers (planes and mbs), queued on the context's stream; slices is a host array,
 * copied before the call returns. ironav_ctx_sync reports a slice id out of range. The planes must start
 * on 16-byte boundaries, luma rows a multiple of 16 bytes apart and chroma rows a multiple of 8 samples
 * apart (IRONAV_INVALID_ARGUMENT otherwise; the host form has no such rule). */
int ironav_deblock_picture_device(ironav_ctx* ctx, void* d_y, int y_stride, void* d_cb, void* d_cr, int c_stride,
                                  const ironav_dbk_mb* d_mbs, const ironav_dbk_slice* slices, int nslices);

/* ---- in-loop mode ---------------------------------------------------------------------------------- */

/* The encoder's own loop (FrameCoder::encode, enc/frame.rs:467-478): the caller makes each macroblock's
 * final decision itself (code_mb's rate-distortion choice, enc/frame.rs:752-790) and commits it
 * (finish_mb, enc/frame.rs:2281-2339); the device analyses every macroblock as soon as the decisions of
 * its left and top-right neighbours are committed, and publishes its result. Results and decisions
 * travel through host memory mapped into the device.
 *
 * The caller must read results and commit decisions in the order it names here, which is also the
 * order the device takes macroblocks in, so that no macroblock it waits for sits behind one that waits
 * for it:
 *   IRONAV_INLOOP_RASTER  one caller thread, picture raster order (slice band after slice band);
 *   IRONAV_INLOOP_BANDS   one caller thread per slice band, raster order within the band.
 * Every device wait is bounded in time (ironav_inloop_set_wait, 10 s by default); a wait that runs out
 * ends the picture with IRONAV_TIMEOUT from ironav_inloop_end.
 *
 * While a picture is open its kernel stays resident waiting for the caller's commits, so a CUDA call that
 * synchronises the whole device — cudaFree, cudaDeviceSynchronize, destroying any context
 * (ironav_ctx_destroy frees device memory) — waits for the picture to end. Make no such call from a thread
 * whose commits the picture still needs (it would stall until the wait bound) before ironav_inloop_end. */
#define IRONAV_INLOOP_RASTER 0
#define IRONAV_INLOOP_BANDS 1
int ironav_inloop_begin(ironav_ctx* ctx, int order);
/* Waits (at most timeout_ms) for macroblock mb's result and copies it to out. */
int ironav_inloop_result(ironav_ctx* ctx, int mb, ironav_mbresult* out, int timeout_ms);
/* Commits macroblock mb's final decision. */
int ironav_inloop_commit(ironav_ctx* ctx, int mb, const ironav_mbstate* final_state);
/* Ends the picture: waits for the device, reports IRONAV_TIMEOUT if any wait gave up. */
int ironav_inloop_end(ironav_ctx* ctx);
int ironav_inloop_set_wait(ironav_ctx* ctx, int wait_ms);

/* ---- batched form ---------------------------------------------------------------------------------- */

/* Many streams analysed together: each stream is a context (its own size, slice bands, references and
 * picture parameters); a frame step copies every stream's new picture, builds every stream's new
 * reference planes and then analyses every stream's macroblock wavefronts in auto mode in one
 * persistent launch. All contexts of a batch must have the same sample depth (bd 8 or 10: every sample
 * buffer below then holds uint8_t or uint16_t samples) and use the same CUDA stream (ironav_ctx_set_stream);
 * the work is queued there, so a frame step can be captured in a CUDA graph. */
typedef struct ironav_batch ironav_batch;
int ironav_batch_create(ironav_batch** out, ironav_ctx* const* ctxs, int n);
int ironav_batch_destroy(ironav_batch* batch);
/* One frame step. Arrays of n device pointers (host arrays): d_src[i], the new picture of stream i
 * (width x height samples, rows width apart); d_ref[i], the reference it predicts from (same layout; pushed as
 * the stream's newest reference); d_col[i], that reference's own decisions (NULL entry or NULL array:
 * none); d_states[i] / d_results[i], where stream i's decisions and results go (mb_w*mb_h each). Each
 * stream's picture parameters are those of its last ironav_begin_p_picture. Asynchronous. */
int ironav_batch_step(ironav_batch* batch, const void* const* d_src, const void* const* d_ref,
                      const ironav_mbstate* const* d_col, ironav_mbstate* const* d_states,
                      ironav_mbresult* const* d_results);
/* Waits for the batch's queued work; IRONAV_TIMEOUT if a wavefront wait gave up. */
int ironav_batch_sync(ironav_batch* batch);
/* Decide mode for the current P picture of every stream in one persistent launch (the streams' wavefronts
 * merged as in ironav_batch_step): each context prepared as for ironav_decide_p_picture_device (source,
 * chroma, references with chroma, picture parameters); arrays of n device pointers and strides, stream
 * i's outputs as that call's. Under CABAC (every context of the batch with the same ironav_set_entropy
 * setting, else IRONAV_INVALID_ARGUMENT) every stream's slice bands are chains of the rate-distortion
 * decision, the longest on three warps each and the rest on one, in two launches side by side.
 * Asynchronous; ironav_batch_sync waits. */
int ironav_batch_decide(ironav_batch* batch, ironav_mbstate* const* d_states, ironav_mbcode* const* d_codes, void* const* d_rec_y,
                        const int* y_strides, void* const* d_rec_cb, void* const* d_rec_cr, const int* c_strides);
/* The deblocking filter of every stream's reconstructed picture, two launches in all (the streams' edge
 * passes together, then their macroblock rows interleaved): arrays of n device pointers and strides, and
 * per stream its records (d_mbs[i], 4-byte aligned) and slice table (slices[i], nslices[i]: host
 * arrays), each as ironav_deblock_picture_device takes them. Asynchronous; ironav_batch_sync waits
 * (IRONAV_INVALID_INPUT: a record names a slice beyond its stream's table). */
int ironav_batch_deblock(ironav_batch* batch, void* const* d_y, const int* y_strides, void* const* d_cb, void* const* d_cr,
                         const int* c_strides, const ironav_dbk_mb* const* d_mbs, const ironav_dbk_slice* const* slices,
                         const int* nslices);

/* The batched step's tuning: no counterpart in the reference (its analysis runs on host threads with
 * nothing to tune). The knobs are the analysis launch's CTAs per SM (4, 5 or 6; its register cap becomes
 * 128, 96 or 80 a thread: more warps in flight against more spills), the half-sample planes' tile rows
 * (16 or 8) and the ticket order of the merged wavefronts (0: ties between streams by stream index; 1: by
 * stream size, largest first). k2_group picks the analysis' form: 0, one macroblock a warp; 8, one macroblock
 * per 8-lane group, four a warp, so that the search's control runs once for four macroblocks (k2_ctas_per_sm
 * is then 4). The default is 4, 16, 0, 0. Every setting gives the same results; only the time changes. */
typedef struct ironav_batch_tuning {
    int32_t k2_ctas_per_sm;
    int32_t k1_tile_rows;
    int32_t order;
    int32_t k2_group;
    float ms;                    /* ironav_batch_autotune: the setting's median step time (milliseconds) */
} ironav_batch_tuning;
int ironav_batch_set_tuning(ironav_batch* batch, const ironav_batch_tuning* t);
int ironav_batch_get_tuning(const ironav_batch* batch, ironav_batch_tuning* t);
/* Times every setting ((3 + 1) x 2 x 2: the warp form at 4, 5 and 6 CTAs an SM and the group form) on `reps` batched steps of these inputs (arguments as ironav_batch_step's;
 * CUDA events on the batch's stream, after a warm-up step each), keeps the fastest by median and returns it
 * in best (and, when all is not NULL, up to cap settings with their times, *n_all of them). Each context's
 * reference ring is put back before every step, so the batch ends exactly as after one ironav_batch_step
 * with these inputs: call it in place of a step. Synchronous. */
int ironav_batch_autotune(ironav_batch* batch, const void* const* d_src, const void* const* d_ref,
                          const ironav_mbstate* const* d_col, ironav_mbstate* const* d_states,
                          ironav_mbresult* const* d_results, int reps, ironav_batch_tuning* best,
                          ironav_batch_tuning* all, int cap, int* n_all);

/* ---- the learned proposer (form 4): its network's kernels ------------------------------------------- */

/* The proposer is a small network (4 conv3x3 layers of 32 channels with ReLU, then a linear head) that, from a
 * macroblock's 16x16 luma tiled 3x3 and the co-located 48x48 reference window, proposes 4 candidate vectors
 * and 5 partition logits; the exact integer cost then judges the candidates. It has no counterpart in the
 * reference: these are its building blocks, which the Python driver (ironav_b200/proposer.py) strings into
 * training steps and proposals. Tensors are "chunk-major padded": each sample a 50 x 50 raster (its 48 x 48
 * interior and a ring of zeros), C channels as C / 8 planes of 16-byte pixels, element (c, q, e) at
 * ((c * Q) + q) * 8 + e with Q = samples * 2500; BF16 values, 16-byte aligned. Weights of a layer are
 * [9 taps][32 out][cin in] (tap = 3 * dy + dx). Every call queues its work on `stream` (a cudaStream_t) and
 * returns; a device wait that gave up sets bit 0 of *d_err (a word in device memory the caller clears and
 * reads). All pointers are device pointers. */
typedef struct ironav_prop_sample {
    const uint8_t* cur;           /* the current picture's luma (8-bit) */
    const uint8_t* ref;           /* the reference picture's luma */
    int32_t w, h, stride;         /* picture size and the current picture's row stride (samples) */
    int32_t mbx, mby;             /* the macroblock */
    int32_t ref_stride;           /* the reference's row stride (0: stride) */
} ironav_prop_sample;             /* 40 bytes */

/* One conv3x3 layer on the tensor cores (tcgen05, BF16 operands, FP32 accumulation in tensor memory):
 * y = act(conv(x, w) + bias) with act ReLU when relu, then times (mask > 0) when d_mask is not NULL; cin is 16
 * or 32, 32 output channels, y's ring zero. d_bias may be NULL. */
int ironav_prop_conv3x3(const void* d_x, int cin, long long samples, const void* d_w, const float* d_bias, int relu, const void* d_mask,
                        void* d_y, unsigned* d_err, void* stream);
/* The weight and bias gradients of a conv3x3 layer on the tensor cores: d_dw[t][o][i] += sum_q dz[q][o] x[q +
 * shift_t][i], d_db[o] += sum_q dz[q][o] (FP32, accumulated; d_db may be NULL). */
int ironav_prop_wgrad3x3(const void* d_x, int cin, const void* d_dz, long long samples, float* d_dw, float* d_db, unsigned* d_err,
                         void* stream);
/* The network's input (two planes: channel 0 the macroblock tiled, channel 1 the reference window, both / 255)
 * for n samples. */
int ironav_prop_prep(const ironav_prop_sample* d_samples, int n, void* d_x, void* stream);
/* The head: d_out[s][j] = d_hb[j] + sum_f d_hw[j][f] feat(s, f), 13 outputs (4 vectors (x, y) in units of 32
 * luma samples, then 5 logits), features f = ((iy * 48 + ix) * 32 + c) of layer 4's output. */
int ironav_prop_head_fwd(const void* d_feat, int n, const float* d_hw, const float* d_hb, float* d_out, void* stream);
/* The head's weights packed for ironav_prop_head_fwd_packed: d_hwt[f][16] = d_hw[j][f] (j < 13; zero after),
 * 73,728 x 16 floats, 16-byte aligned. */
int ironav_prop_head_pack(const float* d_hw, float* d_hwt, void* stream);
/* The head as ironav_prop_head_fwd, from the packed weights: one thread per sample over slices of the pixels,
 * the slices' sums added atomically into d_out (so the order of the additions, and the last bits of the
 * outputs, vary from run to run). */
int ironav_prop_head_fwd_packed(const void* d_feat, int n, const float* d_hwt, const float* d_hb, float* d_out, void* stream);
/* The loss (winner-takes-all L1 on the vectors against d_target_mv (quarter samples), cross-entropy on the
 * logits against d_target_part (0 P_Skip, 1 16x16, 2 16x8, 3 8x16, 4 8x8)) and its gradient d_dout (mean over
 * the n samples); d_sums[0..2] += the vector loss, the partition loss and the partition hits. */
int ironav_prop_loss(const float* d_out, const int16_t* d_target_mv, const uint8_t* d_target_part, int n, float* d_dout, float* d_sums,
                     void* stream);
/* The head's backward pass: d_ghw, d_ghb += its gradients; d_dz = the gradient into layer 4's output through
 * its ReLU (4 planes). */
int ironav_prop_head_bwd(const void* d_feat, int n, const float* d_dout, const float* d_hw, float* d_ghw, float* d_ghb, void* d_dz,
                         void* stream);
/* Adam on n parameters (bias-corrected at `step` >= 1); the gradients are cleared. */
int ironav_prop_adam(float* d_p, float* d_g, float* d_m, float* d_v, long long n, float lr, float beta1, float beta2, int step, float eps,
                     void* stream);
/* A layer's BF16 weights for its forward convolution (d_wf, [9][32][cin]) and, when d_wt is not NULL (cin 32),
 * for its data gradient: transposed and mirrored, d_wt[t][i][o] = w[8 - t][o][i]. */
int ironav_prop_weights(const float* d_w, int cin, void* d_wf, void* d_wt, void* stream);
/* The judge's inputs from the head's outputs of n macroblocks (in raster order): d_cands[s][k] = the k-th vector
 * in quarter samples (rounded, clamped to +-2048 x +-512), d_cls[s] = the partition class of largest logit when
 * its softmax probability is at least min_conf, else 5 (unsure: the plain search). */
int ironav_prop_propose(const float* d_out, int n, float min_conf, int16_t* d_cands, uint8_t* d_cls, void* stream);

/* Replay mode's kernel (all give the same results): 0, one macroblock per 8-lane group (four a warp: the
 * search's control runs once for four macroblocks; the default at 8 bits); 1, one macroblock per warp (the
 * default at 10 bits, where a row of samples is twice the words and 32 lanes share them better; the form auto,
 * in-loop and decide modes use); 2, one macroblock per 16-lane group; 3, per 4-lane group. The oracle accepts
 * and ignores it. */
int ironav_set_replay_form(ironav_ctx* ctx, int form);

/* The learned form's judge (no counterpart in the reference: the north star's form 4). With proposals set, the
 * context's analyses (auto, replay, in-loop and decide modes) judge the newest reference's 16x16 partitioning
 * from them instead of searching: the exact integer cost (SAD + lambda * the vector's bits) of every integer
 * vector within +-2 samples of each of the 4 proposals, then the plain search's sub-sample refinement; the
 * plain search (best_inter) takes over when the proposed partitioning class is not P_Skip or 16x16, or when
 * the best proposal costs more than the predictor's start plus `margin`. d_cands: per macroblock 4 vectors
 * (x, y) in quarter samples (int16, mb_w*mb_h*8); d_cls: per macroblock the class (0 P_Skip, 1 16x16, 2 16x8,
 * 3 8x16, 4 8x8, 5 unsure); d_stats: 3 counters the analyses add to (judged from the proposals, fallbacks on the class,
 * fallbacks on the cost). Device pointers, read when the analyses run; d_cands NULL: the plain search again.
 * The oracle implements the same judge on host pointers. */
int ironav_set_learned(ironav_ctx* ctx, const int16_t* d_cands, const uint8_t* d_cls, int margin, unsigned* d_stats);

/* ---- analysis without allocation ------------------------------------------------------------------ */

/* No counterpart in the reference: an entry point for callers that cannot allocate device memory (a
 * host callback or real-time thread with a fixed memory budget, a custom allocator that owns all device
 * memory, a plugin host that only hands out its own buffers), which therefore cannot create an
 * ironav_ctx. It runs the auto-mode analysis of one P picture against one reference picture, with every
 * input and output in the caller's device memory, and allocates nothing (no cudaMalloc, no library
 * allocation): its scratch (progress flags, counters, slice bands, co-located vectors) is one fixed
 * array of 446,720 bytes (436 KiB) in the library's device memory, which every GPU that loads the
 * library keeps until the process exits.
 *   d_src      the source, padded to whole macroblocks (16*mb_w x 16*mb_h, edges repeated as
 *              ironav_set_source does), 16-byte aligned, rows src_stride bytes apart (a multiple of 16)
 *   d_ref      the reference luma, ref_w x ref_h = width x height or 16*mb_w x 16*mb_h, rows ref_stride apart
 *   d_col      the reference picture's own decisions (mb_w*mb_h) or NULL when it was intra coded
 *   d_planes   out: its half-sample planes G, b, h, j (4 * sw * sh bytes, 4-byte aligned)
 *   d_states   out: the decisions (mb_w*mb_h); d_results: out, the results (mb_w*mb_h)
 *   stream     cudaStream_t for the work (NULL: the legacy default stream)
 * At most IRONAV_NOALLOC_MAX_MBS macroblocks (larger pictures: IRONAV_INVALID_ARGUMENT). The call
 * returns when the work is done (IRONAV_TIMEOUT if a wavefront wait gave up). Every call uses the same
 * scratch array and clears what must start at zero; calls that overlap on the GPU (other streams or
 * host threads) race on it, so make them one after another. The first call on a device looks up the
 * array's address with that device current: make it before any stream capture (a lookup that fails is
 * tried again by the next call; a device reset, cudaDeviceReset, is not supported). qp_prime is only
 * checked (0..63): the analysis reads lambda and skip_thresh, which must come from ironav_lambda and
 * ironav_skip_threshold for that QP'. */
#define IRONAV_NOALLOC_MAX_MBS 36864
int ironav_analyse_auto_noalloc(const uint8_t* d_src, int src_stride, const uint8_t* d_ref, int ref_stride,
                                int ref_w, int ref_h, const ironav_mbstate* d_col, int width, int height,
                                int nslices, int qp_prime, int lambda, int skip_thresh, int fast, int sub8,
                                uint8_t* d_planes, ironav_mbstate* d_states, ironav_mbresult* d_results,
                                void* stream);

#ifdef __cplusplus
}
#endif

#endif /* IRONAV_INTER_H */
