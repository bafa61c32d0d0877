/*
 * v3dm.h -- C ABI of the B200-native SIFT descriptor matching library (libv3dm.so).
 *
 * Drop-in boundary for ETH-V3D's CUDA matching path.  The reference exposes it as the C++
 * structs V3D_CUDA::SIFT_Matching and V3D_CUDA::VocabularyTreeTraversal<BF, Depth>
 * (V3D/CUDA/v3d_cudamatching.h:15-105); each entry point below names the member it
 * replaces.  compat/CUDA/v3d_cudamatching.h (in the package directory) re-creates that
 * C++ surface on top of these functions.
 *
 * Conventions (differences from the reference are deliberate and listed):
 *   - every call returns a status code (V3DM_OK == 0); nothing prints or exits.  The
 *     reference prints and calls exit() on CUDA errors (v3d_cudamatching.cu:12-27);
 *   - a handle owns one CUDA stream and all its device buffers; calls on one handle are
 *     serialised by the caller (the reference is single-threaded too);
 *   - descriptors are 128 bytes (uint8) or 128 floats each, descriptor-contiguous, the
 *     layout of SIFT_Feature::descriptor (V3D/Base/v3d_feature.h:17);
 *   - scores of uint8 descriptors u, v are S * 2^-18 with S = sum u_i v_i: the exact FP32
 *     score the reference computes for descriptors u/512, v/512;
 *   - match pairs are (left index, right index) int32 pairs in ascending left order, the
 *     order of the reference's mutual filter (v3d_cudamatching.cu:546-551);
 *   - feature counts are taken as given (no rounding to multiples of 32); the compat
 *     header applies the reference's rounding and clamping.
 */
#ifndef V3DM_H
#define V3DM_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define V3DM_API __attribute__((visibility("default")))
#else
#define V3DM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
#define V3DM_OK 0
#define V3DM_ERR_ARG 1             /* null pointer, negative size, bad enum            */
#define V3DM_ERR_CUDA 2            /* a CUDA runtime or driver call failed             */
#define V3DM_ERR_NOT_ALLOCATED 3   /* call before allocate / set_nodes                 */
#define V3DM_ERR_SIZE 4            /* count above the allocated maximum or 131072      */
#define V3DM_ERR_CAPACITY 5        /* output buffer smaller than the result; the first
                                      'cap' entries are written, *nOut holds the total */
#define V3DM_ERR_NOT_U8 6          /* float descriptor not of the form u/512, u in 0..255 */
#define V3DM_ERR_UNSUPPORTED 7     /* parameter combination outside the exact domain   */
#define V3DM_ERR_TIMEOUT 8         /* a bounded device-side wait gave up               */
#define V3DM_ERR_NO_DEVICE 9       /* no sm_100 device (the library has no CPU path)   */
#define V3DM_ERR_CANDIDATES 10     /* a device-only call overflowed the candidate list; the
                                      list has been grown, repeat the call             */
#define V3DM_ERR_IO 11             /* a feature file cannot be opened, is not a feature
                                      archive, is malformed or shorter than its count  */

V3DM_API const char* v3dm_status_string(int status);
/* Detail of the last V3DM_ERR_CUDA raised by a matcher call on this thread (the CUDA error
 * and the call that returned it); empty when none. */
V3DM_API const char* v3dm_last_error(void);

/* Largest feature count per image side (17-bit index field of the device state). */
#define V3DM_MAX_FEATURES 131072
/* Largest number of compounding guided gates on one putative result. */
#define V3DM_MAX_GATES 8

/* ---- matcher (V3D_CUDA::SIFT_Matching) -------------------------------------------- */
typedef struct v3dm_matcher v3dm_matcher;

/* Kernel selection flags for v3dm_matcher_create. */
#define V3DM_KERNEL_TCGEN05 0u /* tcgen05 integer MMA with fused selection (default) */
#define V3DM_KERNEL_SIMT 1u    /* dp4a SIMT kernel with the same fused selection     */

/* Creates a matcher on CUDA device 'device'.  Replaces the constructor
 * SIFT_Matching::SIFT_Matching (v3d_cudamatching.h:17-21). */
V3DM_API int v3dm_matcher_create(v3dm_matcher** out, int device, unsigned kernel);
V3DM_API int v3dm_matcher_destroy(v3dm_matcher* h);

/* SIFT_Matching::allocate(nMaxLeft, nMaxRight, useGuidedMatching)
 * (v3d_cudamatching.h:33, v3d_cudamatching.cu:439-474).  Sizes are used as given. */
V3DM_API int v3dm_allocate(v3dm_matcher* h, int nMaxLeft, int nMaxRight, int useGuided);
/* SIFT_Matching::deallocate (v3d_cudamatching.h:39, .cu:476-488). */
V3DM_API int v3dm_deallocate(v3dm_matcher* h);

/* SIFT_Matching::setLeftFeatures / setRightFeatures (v3d_cudamatching.h:41-42,
 * .cu:490-520): float descriptors (see below for values that are not u/512). */
V3DM_API int v3dm_set_left_f32(v3dm_matcher* h, int n, const float* desc);
V3DM_API int v3dm_set_right_f32(v3dm_matcher* h, int n, const float* desc);
/* Float descriptors that are not of the form u/512 are scored, on a tcgen05 handle, with a
 * BF16 hi/lo split (x = hi + lo, score = hi.hi + lo.hi + hi.lo, FP32 accumulation on the
 * tensor cores) in place of the reference's FP32 cublasSgemm (.cu:529-530); decisions, ratio
 * test and mutual filter are the reference's on those scores.  The SIMT handle returns
 * V3DM_ERR_NOT_U8 for them.  u/512 descriptors use the exact integer path.  The _bf16x3
 * variants take the BF16 hi/lo path for any float descriptors (u/512 ones included, for which
 * it is exact).  Non-finite values: V3DM_ERR_ARG. */
V3DM_API int v3dm_set_left_f32_bf16x3(v3dm_matcher* h, int n, const float* desc);
V3DM_API int v3dm_set_right_f32_bf16x3(v3dm_matcher* h, int n, const float* desc);
/* setLeftFeatures / setRightFeatures (.cu:490-520) with the float descriptors already in
 * device memory (for instance a loader's float descriptors, V3DM_LOAD_KEEP_F32 below); the
 * same rules as v3dm_set_left_f32: u/512 values take the exact integer path, other finite
 * values the BF16 hi/lo path on a tcgen05 handle. */
V3DM_API int v3dm_set_left_f32_device(v3dm_matcher* h, int n, const float* d_desc);
V3DM_API int v3dm_set_right_f32_device(v3dm_matcher* h, int n, const float* d_desc);
/* Diagnostic: the BF16 hi/lo scores of the current descriptors, nLeft x nRight floats (row =
 * left), at most 2^26 of them. */
V3DM_API int v3dm_scores_f32(v3dm_matcher* h, float* scores);
/* Float candidate threshold of the BF16 hi/lo path: second values below it never change a
 * decision of findPutativeMatches(minScore, minRatio). */
V3DM_API int v3dm_float_threshold(float minScore, float minRatio, float* T);
/* Native uint8 descriptors (u = 512 * the reference's float value). */
V3DM_API int v3dm_set_left_u8(v3dm_matcher* h, int n, const uint8_t* desc);
V3DM_API int v3dm_set_right_u8(v3dm_matcher* h, int n, const uint8_t* desc);
/* The same with descriptors already in device memory (for instance a loader's, below). */
V3DM_API int v3dm_set_left_u8_device(v3dm_matcher* h, int n, const uint8_t* d_desc);
V3DM_API int v3dm_set_right_u8_device(v3dm_matcher* h, int n, const uint8_t* d_desc);

/* SIFT_Matching::findPutativeMatches(matches, minScore, minRatio)
 * (v3d_cudamatching.h:45-46, .cu:522-552).  minRatio < 0 disables the ratio test.
 * pairs: 2*cap int32 (left, right); *nOut = number of pairs.  Clears the guided gates. */
V3DM_API int v3dm_putative(v3dm_matcher* h, float minScore, float minRatio, int32_t* pairs, int cap, int* nOut);

/* SIFT_Matching::runGuidedMatching(F, thr, leftPos, rightPos, matches, minScore, minRatio)
 * (v3d_cudamatching.h:48-52, .cu:554-623).  F: row-major 3x3 double with q^T F p = 0 for
 * left p, right q.  Positions: interleaved (x, y) floats, one pair per current feature.
 * Like the reference, the gate compounds with the gates of earlier guided calls since the
 * last putative call. */
V3DM_API int v3dm_guided_F(v3dm_matcher* h, const double* F, float thr, const float* leftPos, const float* rightPos,
                  float minScore, float minRatio, int32_t* pairs, int cap, int* nOut);
/* SIFT_Matching::runGuidedHomographyMatching (v3d_cudamatching.h:54-58, .cu:625-694). */
V3DM_API int v3dm_guided_H(v3dm_matcher* h, const double* H, float thr, const float* leftPos, const float* rightPos,
                  float minScore, float minRatio, int32_t* pairs, int cap, int* nOut);

/* Device-resident variants (no host copies, no synchronisation): the result is written to
 * device memory on the handle's stream.  d_pairs holds 2*min(nLeft, nRight) int32 (8-byte
 * aligned), d_count one int32, positions 2 floats per feature (8-byte aligned); misaligned
 * buffers give V3DM_ERR_ARG.  Used to time the kernels with inputs resident in HBM. */
V3DM_API int v3dm_putative_device(v3dm_matcher* h, float minScore, float minRatio, int32_t* d_pairs, int32_t* d_count);
V3DM_API int v3dm_guided_F_device(v3dm_matcher* h, const double* F, float thr, const float* d_leftPos,
                         const float* d_rightPos, float minScore, float minRatio, int32_t* d_pairs,
                         int32_t* d_count);
/* Waits for the handle's stream and returns the status of the last device-only call. */
V3DM_API int v3dm_matcher_wait(v3dm_matcher* h);
/* The handle's CUDA stream (a cudaStream_t). */
V3DM_API int v3dm_matcher_stream(v3dm_matcher* h, void** stream);
/* CUDA-event timing of the fused matching kernel: enable (clears the record), then read
 * the summed duration in milliseconds and the number of timed launches since. */
V3DM_API int v3dm_matcher_profile(v3dm_matcher* h, int enable);
V3DM_API int v3dm_matcher_profile_read(v3dm_matcher* h, double* msTotal, int* launches);
/* The same per pass of the tcgen05 path: pass 0 = lefts x rights (the full contraction),
 * pass 1 = chosen rights x lefts.  Reading pass 1 clears the record. */
V3DM_API int v3dm_matcher_profile_read_pass(v3dm_matcher* h, int pass, double* msTotal, int* launches);
/* Tile configurations of the fused kernel (shape of the left group x right tile and the
 * pipeline depths).  v3dm_matcher_autotune times every configuration on the current
 * features (putative matching, 'reps' timed runs each), keeps the fastest and returns it;
 * it is the tuner the batched and single-pair paths use to pick their tile shape. */
V3DM_API int v3dm_matcher_num_configs(v3dm_matcher* h, int* n);
V3DM_API int v3dm_matcher_get_config(v3dm_matcher* h, int* cfg, int* rowsPerGroup, int* colsPerTile);
V3DM_API int v3dm_matcher_set_config(v3dm_matcher* h, int cfg);
V3DM_API int v3dm_matcher_autotune(v3dm_matcher* h, float minScore, float minRatio, int reps, int* best,
                                   double* msBest);
/* Number of kernels the last matching call launched. */
V3DM_API int v3dm_matcher_last_launches(v3dm_matcher* h, int* n);
/* Test of the failure path (no counterpart in the reference, which exits on any CUDA error,
 * v3d_cudamatching.cu:12-27).  Every device wait of the tcgen05 side pass is bounded; when one
 * runs out, the CTA raises an abort flag, its roles stop, wait (bounded) for their own copies and
 * MMAs in flight, free TMEM and return, and the call reports V3DM_ERR_TIMEOUT; the handle stays
 * usable.  This hook makes that happen on purpose: pass A's bounded waits give up after
 * waitCycles SM cycles, and with skipLoad = k > 0 the producer of CTA 0 does not issue its k-th B
 * tile load, so the MMA issuer's wait for that tile runs out.  waitCycles = skipLoad = 0 (the
 * default) turns it off. */
V3DM_API int v3dm_matcher_test_wait_fault(v3dm_matcher* h, long long waitCycles, int skipLoad);

/* Candidate threshold of the fused selection: every score S >= T is examined exactly and
 * no score below T can change a decision.  Exposed for tests.  Host-only, no device. */
V3DM_API int v3dm_candidate_threshold(float minScore, float minRatio, int gated, int32_t* T);

/* ---- putative matching without device allocation --------------------------------- */
/* No counterpart in the reference: an addition for callers that cannot allocate device
 * memory while they match (a host application that owns all GPU memory and gives plug-ins
 * a fixed budget, a frame loop where cudaMalloc/cudaFree would synchronise the device, a
 * service that must not hit out-of-memory halfway through a job).
 *
 * Same result as v3dm_putative (findPutativeMatches, v3d_cudamatching.cu:522-552) for uint8
 * descriptors already in device memory, computed by the dp4a kernels.  All working memory is
 * one fixed array inside the library's device image, held by every GPU that loads the
 * library until the process exits; nothing is allocated per call.
 *   d_left / d_right: nLeft / nRight x 128 uint8 in device memory of 'device';
 *   d_pairs: room for 2 * min(nLeft, nRight) int32 (left, right pairs, ascending left);
 *   d_count: one int32, the number of pairs, or -1 if a call exceeded the candidate limit;
 *   stream: cudaStream_t the work is queued on (asynchronous; nothing is copied to the host).
 * Limits: nLeft, nRight <= V3DM_NOALLOC_MAX_FEATURES (else V3DM_ERR_SIZE) and at most
 * V3DM_NOALLOC_MAX_CANDIDATES scores at or above the candidate threshold per call.
 * All calls share the one array: calls that overlap on the GPU race, so serialise them.
 * The first call on a device looks up the array's address (cudaGetSymbolAddress with that
 * device current); make it before any stream capture begins.  Descriptors 4-byte aligned,
 * d_pairs 8-byte aligned (else V3DM_ERR_ARG). */
#define V3DM_NOALLOC_MAX_FEATURES 8192
#define V3DM_NOALLOC_MAX_CANDIDATES 524288
V3DM_API int v3dm_putative_u8_noalloc(int device, const uint8_t* d_left, int nLeft, const uint8_t* d_right, int nRight,
                                      float minScore, float minRatio, int32_t* d_pairs, int32_t* d_count,
                                      void* stream);

/* ---- batched matching of many image pairs ------------------------------------------ */
/* Replaces the apps' loop over image pairs (V3D/Apps/SfM/match_sequence.cpp:165-234 and
 * match_using_voctree.cpp:290-336: setLeftFeatures once per left image, then
 * setRightFeatures + findPutativeMatches per right image).  Each pair's result equals that
 * findPutativeMatches call (v3d_cudamatching.cu:522-552) on the two images' descriptors as
 * given (no rounding to multiples of 32); all pairs run in two persistent launches. */
typedef struct v3dm_batch v3dm_batch;

V3DM_API int v3dm_batch_create(v3dm_batch** out, int device);
V3DM_API int v3dm_batch_destroy(v3dm_batch* b);
/* nImages images with counts[i] uint8 descriptors each, concatenated (image 0 first,
 * 128 bytes per descriptor).  Host memory, or device memory (16-byte aligned) for the
 * _device variant.  New image counts invalidate the pair table (set it again); the same
 * counts keep it, so a new image set of the same sizes only uploads descriptors. */
V3DM_API int v3dm_batch_set_images_u8(v3dm_batch* b, int nImages, const int32_t* counts, const uint8_t* desc);
V3DM_API int v3dm_batch_set_images_u8_device(v3dm_batch* b, int nImages, const int32_t* counts,
                                             const uint8_t* d_desc);
/* The same for float descriptors (128 floats each; the reference's float setLeftFeatures /
 * setRightFeatures, v3d_cudamatching.cu:490-520).  When every value is of the form u/512 the
 * integer layout is used; otherwise every image is held in the BF16 hi/lo layouts of the
 * single-pair float matcher and each pair's result equals SIFTMatching's float
 * findPutativeMatches on the two images, and each pair's v3dm_batch_match_guided result equals
 * that putative call followed by one runGuidedMatching / runGuidedHomographyMatching with the
 * pair's gate.  Proposal calls need the integer layout (V3DM_ERR_UNSUPPORTED on float images).
 * Non-finite values: V3DM_ERR_ARG.  *isFloat reports which layout the last upload chose. */
V3DM_API int v3dm_batch_set_images_f32(v3dm_batch* b, int nImages, const int32_t* counts, const float* desc);
V3DM_API int v3dm_batch_set_images_f32_device(v3dm_batch* b, int nImages, const int32_t* counts,
                                              const float* d_desc);
V3DM_API int v3dm_batch_float_mode(v3dm_batch* b, int* isFloat);
/* nPairs (left image, right image) int32 pairs; nPairs == -1 (pairs NULL) means every
 * (i, j) with i < j, left = i, in row-major order. */
V3DM_API int v3dm_batch_set_pairs(v3dm_batch* b, int nPairs, const int32_t* pairs);
/* findPutativeMatches(minScore, minRatio) of every pair.  Output: *nOut (pair, left, right)
 * int32 triples, grouped by pair (pairs ordered by left image, then by table index),
 * ascending left within a pair; the first 'cap' are written (V3DM_ERR_CAPACITY if more). */
V3DM_API int v3dm_batch_match(v3dm_batch* b, float minScore, float minRatio, int32_t* triples, long long cap,
                              long long* nOut);
/* Positions (x, y) of every image's descriptors, two floats each, concatenated in the order of
 * the descriptors given to v3dm_batch_set_images_*; host or device memory (the _device name is
 * an alias).  The guided call needs them; new images drop them. */
V3DM_API int v3dm_batch_set_positions(v3dm_batch* b, const float* positions);
V3DM_API int v3dm_batch_set_positions_device(v3dm_batch* b, const float* d_positions);
/* runGuidedMatching (type 1: M = the pair's fundamental matrix, epipolar gate,
 * v3d_cudamatching.cu:554-623) or runGuidedHomographyMatching (type 2: M = H, transfer-distance
 * gate, .cu:625-694) of every pair of the table, each after its findPutativeMatches: the apps'
 * per-pair sequence putative -> RANSAC -> guided (match_sequence.cpp:306-324) for a whole batch.
 * M: 9 doubles per pair (row-major), thr: one distance threshold per pair, both in the caller's
 * pair order.  Each pair's scores are masked by its own gate only (one guided call after a
 * putative call).  Output and errors as v3dm_batch_match; V3DM_ERR_NOT_ALLOCATED without
 * images, pairs or positions. */
V3DM_API int v3dm_batch_match_guided(v3dm_batch* b, int type, const double* M, const float* thr, float minScore,
                                     float minRatio, int32_t* triples, long long cap, long long* nOut);
/* Device-resident variant: enqueues the call on the batch's stream (replayed as a CUDA graph
 * while images, pairs, parameters and configuration stay the same) and copies the triple
 * count to d_count (device int32, may be NULL).  v3dm_batch_wait checks the call; it returns
 * V3DM_ERR_CANDIDATES when an internal list overflowed (it has been grown: repeat the call).
 * The triples stay in the batch's buffer (v3dm_batch_result_device) until the next call. */
V3DM_API int v3dm_batch_match_device(v3dm_batch* b, float minScore, float minRatio, int32_t* d_count);
V3DM_API int v3dm_batch_wait(v3dm_batch* b);
V3DM_API int v3dm_batch_result_device(v3dm_batch* b, const int32_t** d_triples);
V3DM_API int v3dm_batch_stream(v3dm_batch* b, void** stream);
/* CUDA-graph replay on (default) or off. */
V3DM_API int v3dm_batch_use_graph(v3dm_batch* b, int enable);
/* Tile configuration (as v3dm_matcher_set_config) and row schedule: 0 = rows interleaved over
 * the persistent CTAs (neighbouring CTAs share the right image in L2), 1 = contiguous row
 * ranges per CTA, 2 = chunks of 32 consecutive rows interleaved over the CTAs (consecutive rows
 * that share their left block keep it on chip; meant for the proposal matcher's short rows).
 * The autotune below tries schedules 0 and 1 of the exhaustive matcher. */
V3DM_API int v3dm_batch_set_config(v3dm_batch* b, int cfg, int schedule);
V3DM_API int v3dm_batch_get_config(v3dm_batch* b, int* cfg, int* schedule);
/* Times every (configuration, schedule) on the current batch (reps calls each) and keeps the
 * fastest; ms[2 * cfg + schedule] receives the averages (ms may be NULL). */
V3DM_API int v3dm_batch_autotune(v3dm_batch* b, float minScore, float minRatio, int reps, int* bestCfg,
                                 int* bestSchedule, float* ms);
/* CUDA-event timing of the two side-pass launches (pass 0 = lefts x rights of every pair,
 * pass 1 = chosen rights x lefts); calls run without the graph while it is on. */
V3DM_API int v3dm_batch_profile(v3dm_batch* b, int enable);
V3DM_API int v3dm_batch_profile_read(v3dm_batch* b, int pass, double* msTotal, int* launches);
V3DM_API int v3dm_batch_last_launches(v3dm_batch* b, int* n);
/* Algorithmic work of the current pair table: sum over pairs of 2 * 128 * nLeft * nRight
 * int8 operations, and the number of pairs. */
V3DM_API int v3dm_batch_work(v3dm_batch* b, long long* int8Ops, long long* nPairs);

/* Candidate-proposal matching of every pair (no counterpart in the reference; see the learned
 * projection below): left l and right r are candidates when one of l's 'probesLeft' best cells
 * of the projection is one of r's 'probesRight' best cells; decisions, ratio test and mutual
 * filter are the reference's (.cu:133-210, :546-551) applied to the candidate scores, which
 * are exact uint8 scores.  Same output as v3dm_batch_match.  A true match is found when its
 * two descriptors share a probed cell; recall against v3dm_batch_match is what the projection
 * is trained for. */
typedef struct v3dm_projection v3dm_projection;
V3DM_API int v3dm_batch_match_proposal(v3dm_batch* b, v3dm_projection* proj, int probesLeft, int probesRight,
                                       float minScore, float minRatio, int32_t* triples, long long cap,
                                       long long* nOut);
V3DM_API int v3dm_batch_match_proposal_device(v3dm_batch* b, v3dm_projection* proj, int probesLeft,
                                              int probesRight, float minScore, float minRatio, int32_t* d_count);
/* (left, right) scores pass A of the last proposal call computed (a pair that shares several
 * probed cells is scored once per shared cell), and the exhaustive count sum(nL * nR). */
V3DM_API int v3dm_batch_proposal_scored(v3dm_batch* b, long long* scored, long long* exhaustive);

/* ---- learned candidate proposal ----------------------------------------------------- */
/* No counterpart in the reference: a learned projection f(x) = W2 relu(W1 x + b1) + b2
 * (128 -> 64 -> 32, x = u / 512, BF16 weights, FP32 accumulation, FP32 master copies) trained
 * on the GPU with a symmetric InfoNCE loss on matched descriptor pairs, and C cells (unit
 * centroids) in its output space.  The proposal matcher (v3dm_batch_match_proposal) scores a
 * left descriptor exactly, in uint8, against the right descriptors that share a cell with it:
 * one of the left's probesLeft best cells among the right's probesRight best cells;
 * exhaustive matching stays the reference result.
 * Parameter layout (V3DM_PROJ_PARAMS floats): W1[64][128], b1[64], W2[32][64], b2[32]. */
#define V3DM_PROJ_PARAMS 10336
#define V3DM_PROJ_MAX_CELLS 256
#define V3DM_PROJ_MAX_PROBES 8
#define V3DM_PROJ_MAX_BATCH 4096

/* Creates the network with seeded He-uniform weights and zero biases. */
V3DM_API int v3dm_projection_create(v3dm_projection** out, int device, unsigned long long seed);
V3DM_API int v3dm_projection_destroy(v3dm_projection* p);
V3DM_API int v3dm_projection_get_params(v3dm_projection* p, float* params);
/* Sets the FP32 master parameters (and their BF16 copies); resets the optimiser state. */
V3DM_API int v3dm_projection_set_params(v3dm_projection* p, const float* params);
/* Loss and gradient (V3DM_PROJ_PARAMS floats, grad may be NULL) of a batch of B matched pairs
 * (anchors[k], positives[k]), uint8 descriptors in host memory, temperature T; no update. */
V3DM_API int v3dm_projection_loss_grad(v3dm_projection* p, const uint8_t* anchors, const uint8_t* positives, int B,
                                       float temperature, float* loss, float* grad);
/* One Adam step (beta 0.9 / 0.999) on a batch in device memory; *loss (host, may be NULL)
 * receives the batch loss before the step. */
V3DM_API int v3dm_projection_train_step(v3dm_projection* p, const uint8_t* d_anchors, const uint8_t* d_positives,
                                        int B, float temperature, float lr, float* loss);
/* Unit-length 32-d outputs of n descriptors (host memory). */
V3DM_API int v3dm_projection_embed(v3dm_projection* p, const uint8_t* desc, int n, float* z);
/* The C cells (C x 32 floats, unit vectors). */
V3DM_API int v3dm_projection_set_cells(v3dm_projection* p, int nCells, const float* centroids);
/* The 'probes' best cells of n descriptors, best first (n x probes bytes, host memory). */
V3DM_API int v3dm_projection_assign(v3dm_projection* p, const uint8_t* desc, int n, int probes, uint8_t* cells);

/* ---- vocabulary tree (V3D_CUDA::VocabularyTreeTraversal<BF, Depth>) --------------- */
typedef struct v3dm_voctree v3dm_voctree;

#define V3DM_LEAF_GLOBAL 0 /* node index of the leaf, as _cuda_traverseTree (.cu:791)        */
#define V3DM_LEAF_LOCAL 1  /* leaf index within the last level, as VocabularyTree (v3d_voctree.h:78) */

/* Constructor of VocabularyTreeTraversal<BF, Depth> (v3d_cudamatching.h:71, .cu:797-801);
 * the shape is a runtime parameter here. */
V3DM_API int v3dm_voctree_create(v3dm_voctree** out, int device, int branchFactor, int depth);
V3DM_API int v3dm_voctree_destroy(v3dm_voctree* t);
/* getNodeCount / getLeaveCount (v3d_cudamatching.h:80-99). */
V3DM_API int v3dm_voctree_counts(int branchFactor, int depth, int64_t* nodeCount, int64_t* leafCount);
/* allocate(nMaxFeatures) / deallocate (v3d_cudamatching.h:73-74, .cu:803-829). */
V3DM_API int v3dm_voctree_allocate(v3dm_voctree* t, int nMax);
/* setNodes(nodes) (v3d_cudamatching.h:76, .cu:831-843) and VocabularyTree::loadTreeFromFile's
 * node array (v3d_voctree.h:38-52): nodeCount x 128 descriptors in breadth-first order without
 * the root.  Float nodes may hold any finite values (the apps' trees are k-means centres of
 * unit-L2 descriptors); u8 nodes are u/512 values. */
V3DM_API int v3dm_voctree_set_nodes_f32(v3dm_voctree* t, const float* nodes);
V3DM_API int v3dm_voctree_set_nodes_u8(v3dm_voctree* t, const uint8_t* nodes);
/* traverseTree(n, features, leaveIds) (v3d_cudamatching.h:78, .cu:845-863) and
 * VocabularyTree::getVisualWord (v3d_voctree.h:56-79, with V3DM_LEAF_LOCAL).  The ids are those
 * of the reference's CPU descent, VocabularyTree::findBestNodeIndex (v3d_voctree.h:82-99): each
 * dot product is the sequential FP32 sum over i = 0..127 of the rounded products key[i] *
 * node[i], and the first child whose score is strictly above the running maximum (initially
 * -1e30f) wins.  For u/512 data every such sum is exact, and the integer descent is used.
 * (The reference's GPU kernel, .cu:705-792, sums in a different order with fast-math and can
 * differ from its CPU tree at near ties of float data; the CPU order is the one the apps use.)
 * V3DM_ERR_ARG when the tree holds values that make a descent leave the node array. */
V3DM_API int v3dm_voctree_quantize_f32(v3dm_voctree* t, int n, const float* keys, int32_t* ids, int idMode);
V3DM_API int v3dm_voctree_quantize_u8(v3dm_voctree* t, int n, const uint8_t* keys, int32_t* ids, int idMode);
/* Device-resident variants: keys and ids in device memory, asynchronous on the tree's stream;
 * keys 16-byte aligned and ids 4-byte aligned (else V3DM_ERR_ARG).  The u8 variant needs a u/512
 * tree (else V3DM_ERR_NOT_U8). */
V3DM_API int v3dm_voctree_quantize_u8_device(v3dm_voctree* t, int n, const uint8_t* d_keys, int32_t* d_ids, int idMode);
V3DM_API int v3dm_voctree_quantize_f32_device(v3dm_voctree* t, int n, const float* d_keys, int32_t* d_ids,
                                              int idMode);
/* Diagnostic: key-levels, since the tree was created, whose float scores were too close to
 * decide from the fast pass and were replayed in the reference's sequential order. */
V3DM_API int v3dm_voctree_replays(v3dm_voctree* t, long long* n);
V3DM_API int v3dm_voctree_stream(v3dm_voctree* t, void** stream);
/* Kernels launched by the last quantization call (the float conversion of float keys excluded). */
V3DM_API int v3dm_voctree_last_launches(v3dm_voctree* t, int* n);

/* ---- feature files ------------------------------------------------------------------ */
/* serializeDataFromFile(path, SerializableVector<SIFT_Feature>&) (v3d_serialization.h:983-1017;
 * SIFT_Feature fields v3d_feature.h:12-47).  Binary archive: "V3DBIN", uint32 count, then per
 * feature int32 id, position[2], direction[2], scale, magnitude, descriptor[128].  Text archive
 * (writeBinary = false): "V3DTXT" and the same fields as whitespace-separated tokens with the
 * tags and brackets of TextOStreamArchive (:177-265), parsed as the stream extraction parses them
 * (:267-338); a value it cannot read ("nan", "inf", an overflow), a wrong tag or bracket gives
 * V3DM_ERR_IO, where the reference throws.  For a text archive with every array NULL only the
 * head is read.
 * *n = number of features.  With every array NULL only *n is set; otherwise cap must be >= *n
 * (else V3DM_ERR_CAPACITY).  NULL arrays are skipped.  positions / directions: 2n floats,
 * descriptors: 128n floats.  An unknown tag, a missing or a short file gives V3DM_ERR_IO. */
V3DM_API int v3dm_features_read(const char* path, int cap, int32_t* n, int32_t* ids, float* positions,
                                float* directions, float* scales, float* magnitudes, float* descriptors);
/* u8 re-quantisation on the device: out = round(512 * x) (half to even) clamped to 0..255,
 * NaN -> 0; the identity for descriptors of the form u/512.  nValues a multiple of 4; d_values
 * 16-byte and d_out 4-byte aligned (else V3DM_ERR_ARG).  No counterpart in the reference (its
 * matcher takes the floats). */
V3DM_API int v3dm_quantize_u8_device(const float* d_values, long long nValues, uint8_t* d_out, void* stream);

/* Loader: the apps read one feature file per image and copy each pair's descriptors to the
 * matcher (match_sequence.cpp:124-146, 183-186, 214-231).  A loader reads many files at once
 * (host threads, one file each at a time), keeps the positions on the host, and copies all
 * descriptors to the device in one transfer from pinned memory.  No counterpart in the
 * reference.
 * The extractors store unit-L2 floats (SIFT_Feature::normalizeDescriptor, v3d_feature.h:19-39,
 * called by Apps/SfM/extract_sift_*.cpp), which are not of the form u/512 in general; the
 * reference's matcher scores them in FP32.  So:
 *   - by default the descriptors become u8 only when every value is exactly u/512 (u = 0..255);
 *     otherwise the load returns V3DM_ERR_NOT_U8 (nothing is rounded silently);
 *   - V3DM_LOAD_KEEP_F32 keeps the float descriptors on the device (v3dm_loader_descriptors_
 *     f32_device) for v3dm_set_left_f32_device / v3dm_set_right_f32_device, which score
 *     non-u/512 values with the BF16 hi/lo path; the load then succeeds whatever the values,
 *     and u8 descriptors exist only when they are all u/512;
 *   - V3DM_LOAD_LOSSY_U8 re-quantises any values to u = round(512 x) clamped to 0..255 (lossy
 *     for unit-L2 floats: scores and pairs can differ from the reference's). */
typedef struct v3dm_loader v3dm_loader;
#define V3DM_LOAD_ROUND32 1  /* keep a multiple of 32 features per file, as the apps' '& 0xffe0' */
#define V3DM_LOAD_KEEP_F32 2 /* keep the float descriptors on the device                      */
#define V3DM_LOAD_LOSSY_U8 4 /* round any values to u8 (lossy unless they are u/512)           */
V3DM_API int v3dm_loader_create(int device, v3dm_loader** out);
V3DM_API int v3dm_loader_destroy(v3dm_loader* ld);
/* Reads nFiles files; counts[i] = features kept from file i (its first ones: at most
 * maxPerImage when > 0, a multiple of 32 with V3DM_LOAD_ROUND32).  Returns when the device
 * descriptors are ready; they stay until the next load. */
V3DM_API int v3dm_loader_load(v3dm_loader* ld, int nFiles, const char* const* paths, int maxPerImage, int flags,
                              int32_t* counts);
/* Positions of the kept features (2 floats each), files in order. */
V3DM_API int v3dm_loader_positions(v3dm_loader* ld, float* positions);
/* Device u8 descriptors of the kept features (128 bytes each), files in order, and their count.
 * V3DM_ERR_NOT_U8 when the last load kept floats that are not all u/512 (and was not lossy). */
V3DM_API int v3dm_loader_descriptors_device(v3dm_loader* ld, const uint8_t** d_desc, long long* total);
/* Device float descriptors of the kept features (128 floats each), files in order, as read from
 * the files; only after a load with V3DM_LOAD_KEEP_F32 (else V3DM_ERR_NOT_ALLOCATED). */
V3DM_API int v3dm_loader_descriptors_f32_device(v3dm_loader* ld, const float** d_desc, long long* total);
/* *exact = 1 when every descriptor value of the last load was exactly u/512, u in 0..255. */
V3DM_API int v3dm_loader_exact_u8(v3dm_loader* ld, int* exact);

/* ---- retrieval scoring (V3D::LeafDocuments, v3d_voctree.h:105-289) ------------------- */
/* The image loop of match_using_voctree.cpp:176-222 over visual words: image i is scored
 * against every earlier image with computeBinomialScores(pMatch, words of i, scores,
 * nBest) (v3d_voctree.h:233-278) and then inserted (insertDocument, :143-163).  All images are
 * scored in one call; results are bit-identical to that loop (scores as floats, ties of equal
 * scores by image index).  Scores are finite while every image's p = nFeatures / nLeaves
 * satisfies p + pMatch < 1 and no two empty images meet; outside that domain the reference
 * computes infinities or NaN (its std::sort order is then unspecified: NaN scores rank last
 * here, by image index). */
typedef struct v3dm_retrieval v3dm_retrieval;
#define V3DM_RETRIEVAL_MAX_IMAGES 32768
#define V3DM_RETRIEVAL_MAX_BEST 1024
V3DM_API int v3dm_retrieval_create(v3dm_retrieval** out, int device);
V3DM_API int v3dm_retrieval_destroy(v3dm_retrieval* r);
/* words: the leaf-local visual words (VocabularyTree::getVisualWord, v3d_voctree.h:56-58; the
 * V3DM_LEAF_LOCAL ids of v3dm_voctree_quantize_*) of every image, images concatenated, image i
 * at words[offsets[i] .. offsets[i + 1]) (host offsets, nImages + 1 entries, offsets[0] = 0).
 * nLeaves = the tree's leaf count.  Outputs nImages x nBest: row i holds the min(nBest, i) best
 * earlier images of image i, best first, and their scores, then -1 / 0.  A word outside
 * 0..nLeaves-1 gives V3DM_ERR_ARG (it is skipped). */
V3DM_API int v3dm_retrieval_binomial(v3dm_retrieval* r, int nLeaves, int nImages, const int32_t* offsets,
                                     const int32_t* words, double pMatch, int nBest, int32_t* bestDocs,
                                     float* bestScores);
/* Device-resident variant: words and outputs in device memory, enqueued on the retrieval's
 * stream; v3dm_retrieval_wait returns the call's status (V3DM_ERR_ARG for a word out of range). */
V3DM_API int v3dm_retrieval_binomial_device(v3dm_retrieval* r, int nLeaves, int nImages, const int32_t* offsets,
                                            const int32_t* d_words, double pMatch, int nBest, int32_t* d_bestDocs,
                                            float* d_bestScores);
V3DM_API int v3dm_retrieval_wait(v3dm_retrieval* r);
V3DM_API int v3dm_retrieval_stream(v3dm_retrieval* r, void** stream);
/* CUDA-event timing of the two kernels of each call (kernel 0 = the inverted-file bitmap with
 * its clearing, 1 = counting, scores and selection); read returns the milliseconds and
 * launches since the last read of that kernel. */
V3DM_API int v3dm_retrieval_profile(v3dm_retrieval* r, int enable);
V3DM_API int v3dm_retrieval_profile_read(v3dm_retrieval* r, int kernel, double* msTotal, int* launches);
/* The app's putativePairwiseMatches (match_using_voctree.cpp:196-216) from the bestDocs table
 * (host): (view1, view2) int32 pairs, view1 = the retrieved earlier image, view2 = the query,
 * ordered by view1 then view2 -- the pair table v3dm_batch_set_pairs takes.  *nPairs = the
 * count; with pairs NULL only the count; else the first 'cap' (V3DM_ERR_CAPACITY if more).
 * Host code, no device. */
V3DM_API int v3dm_retrieval_pairs(int nImages, int nBest, const int32_t* bestDocs, long long cap, int32_t* pairs,
                                  long long* nPairs);

/* ---- robust relative orientation (computeRobustOrientationMLE) ------------------------ */
/* The apps' RANSAC for the essential matrix between putative and guided matching
 * (V3D/Apps/SfM/reconstruction_common.cpp:139-340, called at match_sequence.cpp:260-268), for
 * many pairs in one call.  Per pair: samples of 5 correspondences in loop order; for each, the
 * essential matrices of the five-point problem (computeEssentialsFromFiveCorrs,
 * v3d_poseutilities.cpp:1016-1060; Nister's method, restated); each is scored with
 * sum_i min(sampson_i, thr^2) over the pair's correspondences (sampsonEpipolarError of
 * F = K2^-T E K1^-1, reconstruction_common.h:589-607) and kept when its cost is strictly below
 * the best so far and its pose is consistent on the sample (relativePoseFromEssential,
 * v3d_poseutilities.cpp:1264-1294); each kept one lowers the sample budget to
 * ransacNSamples(5, outlier fraction, 1 - 1e-9) (reconstruction_common.h:627-635), and the loop
 * stops once more than 'budget' samples have been drawn.  mode.iterativeRefinement is not run
 * (RobustOrientationMode() default).
 * Inputs: offsets[nPairs + 1] (host) delimit each pair's correspondences in corrs: 4 floats each
 * (left x, left y, right x, right y, pixels, as PointCorrespondence positions); K: 18 doubles per
 * pair (K1 then K2, row-major).  samples: nPairs x nDraw x 5 int32 indices into the pair's
 * correspondences, in the loop's order (at most nSamples + 1 are used), or NULL to draw them on
 * the device from 'seed' (a counter-based hash; not the reference's rand() sequence --
 * v3dm_ransac_shuffle_samples gives that one).
 * Outputs: models, 31 doubles per pair: essential 9, fundamental 9, rotation 9, translation 3
 * (row-major), error (= best cost / N; -1 when the pair has fewer than 5 correspondences or no
 * sample gave a consistent pose, with everything else 0); nInliers per pair (-1 then);
 * inlierFlags (may be NULL): 1 byte per correspondence, sampson < thr^2 under the chosen F.
 * The scores are evaluated in double in the reference's operation order; the five-point solutions
 * agree with the reference's to about 1e-12 (same count), so choices can differ only between
 * candidates whose costs tie to within that. */
typedef struct v3dm_ransac v3dm_ransac;
#define V3DM_RANSAC_MAX_DRAW 65536
#define V3DM_RANSAC_MAX_SAMPLES 4194304 /* nPairs x nDraw */
#define V3DM_RANSAC_MAX_PAIRS 32768     /* pairs per call (the buffers of one round of 128 samples) */
V3DM_API int v3dm_ransac_create(v3dm_ransac** out, int device);
V3DM_API int v3dm_ransac_destroy(v3dm_ransac* r);
V3DM_API int v3dm_ransac_essential(v3dm_ransac* r, int nPairs, const int32_t* offsets, const float* corrs,
                                   const double* K, double inlierThreshold, int nSamples, int nDraw,
                                   const int32_t* samples, uint64_t seed, double* models, int32_t* nInliers,
                                   uint8_t* inlierFlags);
/* Device-resident variant: corrs (16-byte aligned), samples and the outputs in device memory
 * (offsets and K on the host); enqueued on the RANSAC handle's stream, v3dm_ransac_wait
 * synchronises.  A device sample with an index outside its pair's correspondences yields no
 * candidate.  nInliers is -1 for pairs without a model. */
V3DM_API int v3dm_ransac_essential_device(v3dm_ransac* r, int nPairs, const int32_t* offsets, const float* d_corrs,
                                          const double* K, double inlierThreshold, int nSamples, int nDraw,
                                          const int32_t* d_samples, uint64_t seed, double* d_models,
                                          int32_t* d_nInliers, uint8_t* d_inlierFlags);
V3DM_API int v3dm_ransac_wait(v3dm_ransac* r);
/* RobustOrientationMode::iterativeRefinement (reconstruction_common.h:631-640; the apps switch it
 * on, match_sequence.cpp:267): each accepted candidate's pose is refined by refineRelativePose
 * (v3d_poseutilities.cpp:1063-1101) on its inliers, the loop keeps min(cost, refined cost) and the
 * refined model, and the refined inlier count sets the sample budget
 * (reconstruction_common.cpp:255-314).  Off by default, as in the reference.  The refinement's
 * sums over the inliers run in parallel, so the refined pose agrees with the reference's to
 * rounding, not bit for bit. */
V3DM_API int v3dm_ransac_set_refinement(v3dm_ransac* r, int enable);
/* The sample sequence computeRobustOrientationMLE draws for a pair of N correspondences after
 * srand(seed): getShuffleCount(N, nSamples, 5) shuffles of 0..N-1 (random_shuffle over the C
 * library's rand()), each cut into consecutive 5-tuples while j < N - 5; at most cap tuples are
 * written (5 int32 each), *nDraw = the count written (at most nSamples + 1 are ever used).  Host
 * code; it reseeds the C library's generator with srand(seed). */
V3DM_API int v3dm_ransac_shuffle_samples(int N, int nSamples, unsigned seed, int cap, int32_t* samples, int* nDraw);
/* The five-point solutions of n samples on the device (diagnostic): pts holds, per sample,
 * x1[5] y1[5] x2[5] y2[5] (normalised coordinates, q^T E p = 0); Es receives up to 10 row-major
 * essential matrices per sample (90 doubles), counts the number of each. */
V3DM_API int v3dm_essential_five_point(v3dm_ransac* r, int n, const double* pts, double* Es, int32_t* counts);
V3DM_API int v3dm_ransac_stream(v3dm_ransac* r, void** stream);
V3DM_API int v3dm_ransac_last_launches(v3dm_ransac* r, int* n);
/* CUDA-event timing of kernel 0 (five-point solutions of every sample) and kernel 1 (the costs of
 * every candidate); read returns the milliseconds and launches since the last read. */
/* Work of the last call: candidates scored (five-point solutions of all samples) and Sampson
 * evaluations (sum over candidates of their pair's correspondence count). */
V3DM_API int v3dm_ransac_candidates(v3dm_ransac* r, long long* nCandidates, long long* nEvaluations);
V3DM_API int v3dm_ransac_profile(v3dm_ransac* r, int enable);
V3DM_API int v3dm_ransac_profile_read(v3dm_ransac* r, int kernel, double* msTotal, int* launches);

#ifdef __cplusplus
}
#endif

#endif /* V3DM_H */
