/*
 * v3dm_oracle.c -- CPU restatement of ETH-V3D's CUDA SIFT matching path and of its
 * vocabulary-tree quantizer.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker and the timed CPU
 * baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it; the library under eth-v3d-lgpl_b200/ never links, calls or falls back to it.
 *
 * What it restates (file:line in the reference project):
 *   score matrix        V3D/CUDA/v3d_cudamatching.cu:529-530   cublasSgemm('T','N',nL,nR,128,...)
 *   column rule         V3D/CUDA/v3d_cudamatching.cu:133-162   per LEFT l: scan r ascending
 *   row rule            V3D/CUDA/v3d_cudamatching.cu:164-210   per RIGHT r: scan l ascending
 *   no-ratio rules      V3D/CUDA/v3d_cudamatching.cu:33-85     (selected when minRatio < 0, .cu:535-539)
 *   epipolar gate       V3D/CUDA/v3d_cudamatching.cu:277-311   with the double->float cast of F at .cu:591-595
 *   homography gate     V3D/CUDA/v3d_cudamatching.cu:313-343   with the cast at .cu:662-666
 *   mutual filter       V3D/CUDA/v3d_cudamatching.cu:546-551   (repeated at :616-621 and :687-692)
 *   voctree descent     V3D/CUDA/v3d_cudamatching.cu:705-792   (global node id of the leaf)
 *                       V3D/Base/v3d_voctree.h:63-99           (CPU version, leaf-local id)
 *   retrieval scores    V3D/Base/v3d_voctree.h:143-278         LeafDocuments insertDocument /
 *                       getDocumentHistogram / computeBinomialScores, in the image loop of
 *                       V3D/Apps/SfM/match_using_voctree.cpp:176-222
 *
 * Domain and pinned arithmetic.
 *   Descriptors are uint8 values u fed to the reference as floats u/512.  Every FP32 product
 *   (u/512)(v/512) = uv*2^-18 is exact and every partial sum is an integer multiple of 2^-18
 *   below 255*255*128*2^-18 < 2^23 * 2^-18, so cublasSgemm's FP32 result is exactly
 *   S*2^-18 with S = sum_i u_i v_i, whatever the summation order or FMA use.  The oracle
 *   therefore computes S in integers and forms the score (float)S * 2^-18.
 *   The reference was built with --use_fast_math (V3D/CMakeLists.txt:146); the oracle fixes
 *   IEEE round-to-nearest semantics with no FMA contraction (built with -ffp-contract=off):
 *     bestDist = 2 - 2*s1                                   (float)
 *     nextDist = (float) max(0.001, (double)(2 - 2*s2))     (the reference's mixed max)
 *     ratio    = bestDist / nextDist                         (IEEE float division)
 *   Gate expressions are evaluated left to right in float, one rounding per operation.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_NONE (-1e30f)   /* initial maxVal / nextVal of the reference kernels (.cu:138-139) */
#define ORC_MASKED (-1e20f) /* value written by the gates (.cu:308, :340) */

typedef struct {
    float best;
    int arg;
    float next;
} orc_top2;

static inline void top2_init(orc_top2* t) {
    t->best = ORC_NONE;
    t->arg = -1;
    t->next = ORC_NONE;
}

/* One step of the scan in .cu:145-147 (and :192-194):
 *   argMax  = (val > maxVal) ? idx : argMax;
 *   nextVal = (val > maxVal) ? maxVal : max(val, nextVal);
 *   maxVal  = max(maxVal, val);                                                         */
static inline void top2_push(orc_top2* t, float val, int idx) {
    int gt = val > t->best;
    t->arg = gt ? idx : t->arg;
    t->next = gt ? t->best : fmaxf(val, t->next);
    t->best = fmaxf(t->best, val);
}

/* Result of scanning block A and then block B (A holds the lower indices).  Equal to
 * pushing A's values and then B's values one by one: the best is the first index of the
 * maximum, and next is the second largest value of the multiset union.                 */
static inline orc_top2 top2_concat(orc_top2 a, orc_top2 b) {
    orc_top2 r;
    if (b.best > a.best) {
        r.best = b.best;
        r.arg = b.arg;
        r.next = fmaxf(a.best, b.next);
    } else {
        r.best = a.best;
        r.arg = a.arg;
        r.next = fmaxf(a.next, b.best);
    }
    return r;
}

/* Decision of one scan, .cu:147-161 (ratio) and .cu:48 (no ratio).  USE_ARCCOS_RATIO is
 * off in the reference (.cu:150), so the ratio lives in 2-2s (squared L2) space.         */
static inline int top2_decide(orc_top2 t, float minScore, float minRatio) {
    if (minRatio < 0.0f) return (t.best > minScore) ? t.arg : -1;
    float nextDist = (float)fmax(0.001, (double)(2.0f - 2.0f * t.next));
    float bestDist = 2.0f - 2.0f * t.best;
    float ratio = bestDist / nextDist;
    return (t.best > minScore && ratio < minRatio) ? t.arg : -1;
}

/* ----------------------------------------------------------------------------------- */
/* Gates.  Each gate is {type, m[9] (row-major double 3x3), thr}; type 1 = epipolar       */
/* (F, .cu:277-311), type 2 = homography (H, .cu:313-343).  The reference mutates the   */
/* score matrix in place, so gates of consecutive guided calls compound: an element is   */
/* masked (-1e20f) when any gate rejects it.                                             */

typedef struct {
    int type;
    double m[9];
    float thr;
} orc_gate;

typedef struct {
    /* per left: epipolar Fp (3) or homography Hp dehomogenised (2) */
    float* lv;
    /* per right: epipolar (q.x, q.y, Ftq.x, Ftq.y) or homography (q.x, q.y) */
    float* rv;
    float sqrThr;
    int type;
} orc_gate_pre;

static void gate_precompute(const orc_gate* g, int nL, int nR, const float* lpos, const float* rpos,
                            orc_gate_pre* out) {
    /* .cu:591-595: float3 F1 = (F[0][0], F[0][1], F[0][2]) etc., each a double->float cast */
    float m[9];
    for (int i = 0; i < 9; ++i) m[i] = (float)g->m[i];
    out->type = g->type;
    out->sqrThr = g->thr * g->thr; /* .cu:591 float const sqrThreshold = thr*thr */
    out->lv = (float*)malloc(sizeof(float) * 3 * (size_t)(nL > 0 ? nL : 1));
    out->rv = (float*)malloc(sizeof(float) * 4 * (size_t)(nR > 0 ? nR : 1));
    for (int l = 0; l < nL; ++l) {
        float px = lpos[2 * l], py = lpos[2 * l + 1];
        float x = m[0] * px + m[1] * py + m[2]; /* .cu:289-291 / :325-327 */
        float y = m[3] * px + m[4] * py + m[5];
        float z = m[6] * px + m[7] * py + m[8];
        if (g->type == 2) { /* .cu:329-330 Hp.x /= Hp.z; Hp.y /= Hp.z */
            x /= z;
            y /= z;
        }
        out->lv[3 * l] = x;
        out->lv[3 * l + 1] = y;
        out->lv[3 * l + 2] = z;
    }
    for (int r = 0; r < nR; ++r) {
        float qx = rpos[2 * r], qy = rpos[2 * r + 1];
        out->rv[4 * r] = qx;
        out->rv[4 * r + 1] = qy;
        if (g->type == 1) { /* .cu:298-299 Ftq.x, Ftq.y (Ftq.z, .cu:300, is unused) */
            out->rv[4 * r + 2] = m[0] * qx + m[3] * qy + m[6];
            out->rv[4 * r + 3] = m[1] * qx + m[4] * qy + m[7];
        } else {
            out->rv[4 * r + 2] = 0.f;
            out->rv[4 * r + 3] = 0.f;
        }
    }
}

static inline int gate_rejects(const orc_gate_pre* g, int l, int r) {
    const float* p = g->lv + 3 * l;
    const float* q = g->rv + 4 * r;
    if (g->type == 1) {
        /* .cu:302-308 */
        float num = q[0] * p[0] + q[1] * p[1] + p[2];
        num *= num;
        float denom = p[0] * p[0] + p[1] * p[1] + q[2] * q[2] + q[3] * q[3];
        float sampsonDist = num / denom;
        return sampsonDist > g->sqrThr;
    } else {
        /* .cu:337-340 */
        float dx = p[0] - q[0], dy = p[1] - q[1];
        float sqrDist = dx * dx + dy * dy;
        return sqrDist > g->sqrThr;
    }
}

/* ----------------------------------------------------------------------------------- */

static inline int dot_u8(const uint8_t* a, const uint8_t* b) {
    int s = 0;
    for (int i = 0; i < 128; ++i) s += (int)a[i] * (int)b[i];
    return s;
}

/* Full matching call: findPutativeMatches (.cu:522-552) when nGates == 0, runGuidedMatching
 * (.cu:554-623) / runGuidedHomographyMatching (.cu:625-694) otherwise.
 *   L: nL x 128 uint8 (descriptor-contiguous), R: nR x 128 uint8.
 *   lpos / rpos: interleaved (x, y) floats, the layout of V3D::Vector2f arrays.
 *   colMaxOut (nL) / rowMaxOut (nR): optional, the two direction results.
 *   pairsOut: capacity min(nL, nR) pairs (left, right), ascending left.
 * Returns the number of pairs, or -1 on bad arguments.                                   */
int orc_match_u8(int nL, int nR, const uint8_t* L, const uint8_t* R, float minScore, float minRatio,
                 int nGates, const orc_gate* gates, const float* lpos, const float* rpos, int* colMaxOut,
                 int* rowMaxOut, int* pairsOut, int nThreads) {
    if (nL < 0 || nR < 0 || (nGates > 0 && (!lpos || !rpos))) return -1;
    if (nL == 0 || nR == 0) return 0;
#ifdef _OPENMP
    if (nThreads <= 0) nThreads = omp_get_max_threads();
#else
    nThreads = 1;
#endif
    orc_gate_pre* pre = NULL;
    if (nGates > 0) {
        pre = (orc_gate_pre*)calloc((size_t)nGates, sizeof(orc_gate_pre));
        for (int g = 0; g < nGates; ++g) gate_precompute(&gates[g], nL, nR, lpos, rpos, &pre[g]);
    }
    int* colMax = (int*)malloc(sizeof(int) * (size_t)nL);
    int* rowMax = (int*)malloc(sizeof(int) * (size_t)nR);
    /* Per-thread column (per-left) states over a contiguous range of r; merged in thread
     * order afterwards so the result equals the sequential scan of .cu:142-148.         */
    orc_top2* colPart = (orc_top2*)malloc(sizeof(orc_top2) * (size_t)nL * (size_t)nThreads);
    float* rowBuf = (float*)malloc(sizeof(float) * (size_t)nL * (size_t)nThreads);

#pragma omp parallel num_threads(nThreads)
    {
        int tid = 0, nt = 1;
#ifdef _OPENMP
        tid = omp_get_thread_num();
        nt = omp_get_num_threads();
#endif
        orc_top2* cp = colPart + (size_t)tid * nL;
        float* sc = rowBuf + (size_t)tid * nL;
        for (int l = 0; l < nL; ++l) top2_init(&cp[l]);
        int r0 = (int)((long long)nR * tid / nt), r1 = (int)((long long)nR * (tid + 1) / nt);
        for (int r = r0; r < r1; ++r) {
            const uint8_t* rr = R + (size_t)r * 128;
            for (int l = 0; l < nL; ++l) sc[l] = (float)dot_u8(L + (size_t)l * 128, rr) * 0x1p-18f;
            for (int g = 0; g < nGates; ++g)
                for (int l = 0; l < nL; ++l)
                    if (gate_rejects(&pre[g], l, r)) sc[l] = ORC_MASKED;
            orc_top2 rt;
            top2_init(&rt);
            for (int l = 0; l < nL; ++l) {
                top2_push(&rt, sc[l], l);
                top2_push(&cp[l], sc[l], r);
            }
            rowMax[r] = top2_decide(rt, minScore, minRatio);
        }
    }
    for (int l = 0; l < nL; ++l) {
        orc_top2 acc = colPart[l];
        for (int t = 1; t < nThreads; ++t) acc = top2_concat(acc, colPart[(size_t)t * nL + l]);
        colMax[l] = top2_decide(acc, minScore, minRatio);
    }
    /* mutual filter, .cu:546-551 */
    int n = 0;
    for (int k = 0; k < nL; ++k) {
        int l = colMax[k];
        if (l >= 0 && rowMax[l] == k) {
            if (pairsOut) {
                pairsOut[2 * n] = k;
                pairsOut[2 * n + 1] = l;
            }
            ++n;
        }
    }
    if (colMaxOut) memcpy(colMaxOut, colMax, sizeof(int) * (size_t)nL);
    if (rowMaxOut) memcpy(rowMaxOut, rowMax, sizeof(int) * (size_t)nR);
    for (int g = 0; g < nGates; ++g) {
        free(pre[g].lv);
        free(pre[g].rv);
    }
    free(pre);
    free(colMax);
    free(rowMax);
    free(colPart);
    free(rowBuf);
    return n;
}

/* A findPutativeMatches call followed by guided calls on the same features, from ONE score
 * computation, as the reference does: the putative call writes the score matrix
 * (.cu:529-530) and each later runGuidedMatching / runGuidedHomographyMatching masks that
 * stored matrix in place and re-runs the maxima (.cu:554-623, :625-694), so gates compound.
 * Call c (0 <= c < nCalls) sees gates[0 .. gatesUpTo[c]-1]; gatesUpTo[0] is normally 0 (the
 * putative call).  pairsOut holds nCalls blocks of min(nL, nR) pairs; nOut[c] gets call c's
 * pair count.  Results equal nCalls separate orc_match_u8 calls.  Returns 0, or -1 on bad
 * arguments.                                                                             */
int orc_match_u8_calls(int nL, int nR, const uint8_t* L, const uint8_t* R, float minScore, float minRatio,
                       int nCalls, const int* gatesUpTo, const orc_gate* gates, const float* lpos,
                       const float* rpos, int* pairsOut, int* nOut, int nThreads) {
    if (nL < 0 || nR < 0 || nCalls < 1 || !gatesUpTo || !nOut) return -1;
    int nGates = 0;
    for (int c = 0; c < nCalls; ++c) {
        if (gatesUpTo[c] < 0 || (c > 0 && gatesUpTo[c] < gatesUpTo[c - 1])) return -1;
        nGates = gatesUpTo[c];
    }
    if (nGates > 0 && (!lpos || !rpos || !gates)) return -1;
    for (int c = 0; c < nCalls; ++c) nOut[c] = 0;
    if (nL == 0 || nR == 0) return 0;
#ifdef _OPENMP
    if (nThreads <= 0) nThreads = omp_get_max_threads();
#else
    nThreads = 1;
#endif
    orc_gate_pre* pre = NULL;
    if (nGates > 0) {
        pre = (orc_gate_pre*)calloc((size_t)nGates, sizeof(orc_gate_pre));
        for (int g = 0; g < nGates; ++g) gate_precompute(&gates[g], nL, nR, lpos, rpos, &pre[g]);
    }
    const size_t cap = (size_t)(nL < nR ? nL : nR);
    int* rowMax = (int*)malloc(sizeof(int) * (size_t)nR * (size_t)nCalls);
    orc_top2* colPart = (orc_top2*)malloc(sizeof(orc_top2) * (size_t)nL * (size_t)nThreads * (size_t)nCalls);
    float* rowBuf = (float*)malloc(sizeof(float) * (size_t)nL * (size_t)nThreads * 2);

#pragma omp parallel num_threads(nThreads)
    {
        int tid = 0, nt = 1;
#ifdef _OPENMP
        tid = omp_get_thread_num();
        nt = omp_get_num_threads();
#endif
        float* sc = rowBuf + (size_t)tid * nL * 2;
        float* masked = sc + nL;
        for (int c = 0; c < nCalls; ++c) {
            orc_top2* cp = colPart + ((size_t)c * nThreads + tid) * nL;
            for (int l = 0; l < nL; ++l) top2_init(&cp[l]);
        }
        int r0 = (int)((long long)nR * tid / nt), r1 = (int)((long long)nR * (tid + 1) / nt);
        for (int r = r0; r < r1; ++r) {
            const uint8_t* rr = R + (size_t)r * 128;
            for (int l = 0; l < nL; ++l) sc[l] = (float)dot_u8(L + (size_t)l * 128, rr) * 0x1p-18f;
            memcpy(masked, sc, sizeof(float) * (size_t)nL);
            int applied = 0;
            for (int c = 0; c < nCalls; ++c) {
                for (; applied < gatesUpTo[c]; ++applied)
                    for (int l = 0; l < nL; ++l)
                        if (gate_rejects(&pre[applied], l, r)) masked[l] = ORC_MASKED;
                orc_top2* cp = colPart + ((size_t)c * nThreads + tid) * nL;
                orc_top2 rt;
                top2_init(&rt);
                for (int l = 0; l < nL; ++l) {
                    top2_push(&rt, masked[l], l);
                    top2_push(&cp[l], masked[l], r);
                }
                rowMax[(size_t)c * nR + r] = top2_decide(rt, minScore, minRatio);
            }
        }
    }
    for (int c = 0; c < nCalls; ++c) {
        const int* rm = rowMax + (size_t)c * nR;
        int* out = pairsOut ? pairsOut + 2 * cap * (size_t)c : NULL;
        int n = 0;
        for (int k = 0; k < nL; ++k) {
            orc_top2 acc = colPart[((size_t)c * nThreads) * nL + k];
            for (int t = 1; t < nThreads; ++t) acc = top2_concat(acc, colPart[((size_t)c * nThreads + t) * nL + k]);
            int l = top2_decide(acc, minScore, minRatio);
            if (l >= 0 && rm[l] == k) { /* mutual filter, .cu:546-551 */
                if (out) {
                    out[2 * n] = k;
                    out[2 * n + 1] = l;
                }
                ++n;
            }
        }
        nOut[c] = n;
    }
    for (int g = 0; g < nGates; ++g) {
        free(pre[g].lv);
        free(pre[g].rv);
    }
    free(pre);
    free(rowMax);
    free(colPart);
    free(rowBuf);
    return 0;
}

/* The reference's size handling in front of every call (.cu:444-460 allocate, .cu:493-519
 * setLeft/RightFeatures): round down to a multiple of 32, then clamp to nMax.             */
int orc_ref_feature_count(int n, int nMaxRounded) {
    if (n % 32 != 0) n = n - (n & 31);
    return n < nMaxRounded ? n : nMaxRounded;
}

/* ----------------------------------------------------------------------------------- */
/* Vocabulary tree.  Nodes in breadth-first order without the root: level-1 nodes 0..BF-1,
 * children of node i at (i+1)*BF + k (.cu:784-785, v3d_voctree.h:74-75).  Each level takes
 * the child with the largest dot product, first child on ties (strict '>', .cu:781,
 * v3d_voctree.h:93).  Dot products are sequential FP32 sums as in v3d_voctree.h:91; for
 * uint8-valued data every sum is an exact integer below 2^24, so the GPU's reduction order
 * (.cu:770-779) gives the same value.  globalIds != 0 returns the node index of the leaf as
 * _cuda_traverseTree does (.cu:791); otherwise the leaf-local index of
 * VocabularyTree::findBestLeafIndex (v3d_voctree.h:78).                                  */
int orc_voctree_quantize_f32(int bf, int depth, const float* nodes, int n, const float* keys, int* out,
                             int globalIds, int nThreads) {
    if (bf < 1 || depth < 1 || n < 0) return -1;
    long long levelStartLast = 0, len = 1;
    for (int d = 0; d < depth - 1; ++d) {
        len *= bf;
        levelStartLast += len;
    }
#ifdef _OPENMP
    if (nThreads <= 0) nThreads = omp_get_max_threads();
#endif
#pragma omp parallel for schedule(static) num_threads(nThreads > 0 ? nThreads : 1)
    for (int j = 0; j < n; ++j) {
        const float* key = keys + (size_t)j * 128;
        long long leafId = 0, nextLeafId = 0;
        for (int d = 0; d < depth; ++d) {
            const float* base = nodes + (size_t)nextLeafId * 128;
            int bestNode = -1;
            float maxScore = -1e30f;
            for (int k = 0; k < bf; ++k) {
                const float* cur = base + (size_t)k * 128;
                float score = 0.f;
                for (int i = 0; i < 128; ++i) score += key[i] * cur[i];
                if (score > maxScore) {
                    bestNode = k;
                    maxScore = score;
                }
            }
            leafId = nextLeafId + bestNode;
            nextLeafId = (leafId + 1) * bf;
        }
        out[j] = (int)(globalIds ? leafId : leafId - levelStartLast);
    }
    return 0;
}

/* uint8 variant: identical result to the float variant on u-valued floats (exact sums). */
int orc_voctree_quantize_u8(int bf, int depth, const uint8_t* nodes, int n, const uint8_t* keys, int* out,
                            int globalIds, int nThreads) {
    if (bf < 1 || depth < 1 || n < 0) return -1;
    long long levelStartLast = 0, len = 1;
    for (int d = 0; d < depth - 1; ++d) {
        len *= bf;
        levelStartLast += len;
    }
#ifdef _OPENMP
    if (nThreads <= 0) nThreads = omp_get_max_threads();
#endif
#pragma omp parallel for schedule(static) num_threads(nThreads > 0 ? nThreads : 1)
    for (int j = 0; j < n; ++j) {
        const uint8_t* key = keys + (size_t)j * 128;
        long long leafId = 0, nextLeafId = 0;
        for (int d = 0; d < depth; ++d) {
            const uint8_t* base = nodes + (size_t)nextLeafId * 128;
            int bestNode = -1;
            int maxScore = -1;
            for (int k = 0; k < bf; ++k) {
                int score = dot_u8(key, base + (size_t)k * 128);
                if (score > maxScore) {
                    bestNode = k;
                    maxScore = score;
                }
            }
            leafId = nextLeafId + bestNode;
            nextLeafId = (leafId + 1) * bf;
        }
        out[j] = (int)(globalIds ? leafId : leafId - levelStartLast);
    }
    return 0;
}

/* Exact score matrix for small cases (tests): S[r*nL + l] = sum_i L[l][i] R[r][i], the
 * integer behind the reference's row-major Scores[r*nL + l] (.cu:36-41).                 */
void orc_scores_u8(int nL, int nR, const uint8_t* L, const uint8_t* R, int32_t* S) {
    for (int r = 0; r < nR; ++r)
        for (int l = 0; l < nL; ++l) S[(size_t)r * nL + l] = dot_u8(L + (size_t)l * 128, R + (size_t)r * 128);
}

/* ----------------------------------------------------------------------------------- */
/* Retrieval scoring.  Image i queries the inverted files of images 0..i-1 and is then   */
/* inserted (match_using_voctree.cpp:187-220).  getDocumentHistogram (v3d_voctree.h:     */
/* 165-177) adds 1 to document d for every query feature whose leaf lists d, and a leaf  */
/* lists a document once (insertDocument, :143-163, stores a word histogram).  The score */
/* of d is computeBinomialScores' expression (:250-270) in double with the C library's   */
/* log, stored as float, and std::sort / partial_sort order the (score, d) pairs         */
/* (:273-276).  Since every inverted file lists documents in insertion order, the files  */
/* of all images are built first and query i reads the part below i, so queries run in   */
/* parallel.  NaN scores (both images empty) rank after every number, by index here; the */
/* reference's sort order is unspecified for them.                                      */
typedef struct {
    float score;
    int doc;
} orc_doc_score;

static int orc_doc_score_cmp(const void* pa, const void* pb) {
    const orc_doc_score* a = (const orc_doc_score*)pa;
    const orc_doc_score* b = (const orc_doc_score*)pb;
    const int an = isnan(a->score), bn = isnan(b->score);
    if (an != bn) return an ? 1 : -1;
    if (!an) {
        if (a->score < b->score) return -1;
        if (b->score < a->score) return 1;
    }
    return (a->doc > b->doc) - (a->doc < b->doc);
}

int orc_retrieval_binomial(int nLeaves, int nImages, const int* offsets, const int* words, double pMatch,
                           int nBest, int* bestDocs, float* bestScores, int threads) {
    if (nLeaves < 1 || nImages < 0 || nBest < 1) return -1;
    for (int j = 0; j < (nImages > 0 ? offsets[nImages] : 0); ++j)
        if (words[j] < 0 || words[j] >= nLeaves) return -1;
    /* inverted files: per leaf the images that have it, ascending, each once */
    int* fileStart = (int*)calloc((size_t)nLeaves + 1, sizeof(int));
    int* last = (int*)malloc((size_t)nLeaves * sizeof(int));
    for (int w = 0; w < nLeaves; ++w) last[w] = -1;
    for (int d = 0; d < nImages; ++d)
        for (int j = offsets[d]; j < offsets[d + 1]; ++j)
            if (last[words[j]] != d) {
                last[words[j]] = d;
                ++fileStart[words[j] + 1];
            }
    for (int w = 0; w < nLeaves; ++w) fileStart[w + 1] += fileStart[w];
    int* files = (int*)malloc((size_t)(fileStart[nLeaves] > 0 ? fileStart[nLeaves] : 1) * sizeof(int));
    int* fill = (int*)malloc((size_t)nLeaves * sizeof(int));
    memcpy(fill, fileStart, (size_t)nLeaves * sizeof(int));
    for (int w = 0; w < nLeaves; ++w) last[w] = -1;
    for (int d = 0; d < nImages; ++d)
        for (int j = offsets[d]; j < offsets[d + 1]; ++j)
            if (last[words[j]] != d) {
                last[words[j]] = d;
                files[fill[words[j]]++] = d;
            }
    free(fill);
    free(last);
    const double normalizer = 1.0 / nLeaves;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
#pragma omp parallel
    {
        int* hist = (int*)malloc((size_t)(nImages > 0 ? nImages : 1) * sizeof(int));
        orc_doc_score* sc = (orc_doc_score*)malloc((size_t)(nImages > 0 ? nImages : 1) * sizeof(orc_doc_score));
#pragma omp for schedule(dynamic, 4)
        for (int i = 0; i < nImages; ++i) {
            memset(hist, 0, (size_t)i * sizeof(int));
            for (int j = offsets[i]; j < offsets[i + 1]; ++j) {
                const int w = words[j];
                for (int p = fileStart[w]; p < fileStart[w + 1] && files[p] < i; ++p) hist[files[p]] += 1;
            }
            const int nq = offsets[i + 1] - offsets[i];
            for (int d = 0; d < i; ++d) {
                const int nd = offsets[d + 1] - offsets[d];
                const double k = hist[d];
                const double n = nd < nq ? nd : nq;
                const double pRandom = (nd > nq ? nd : nq) * normalizer;
                const double logP0 = log(pRandom);
                const double log1P0 = log(1.0 - pRandom);
                const double pMatching = pRandom + pMatch < 1.0 ? pRandom + pMatch : 1.0;
                const double logP1 = log(pMatching);
                const double log1P1 = log(1.0 - pMatching);
                const double z0 = k * logP0 + (n - k) * log1P0;
                const double z1 = k * logP1 + (n - k) * log1P1;
                sc[d].score = (float)(z0 - z1);
                sc[d].doc = d;
            }
            qsort(sc, (size_t)i, sizeof(orc_doc_score), orc_doc_score_cmp);
            for (int j = 0; j < nBest; ++j) {
                bestDocs[(size_t)i * nBest + j] = j < i ? sc[j].doc : -1;
                bestScores[(size_t)i * nBest + j] = j < i ? sc[j].score : 0.0f;
            }
        }
        free(sc);
        free(hist);
    }
    free(files);
    free(fileStart);
    return 0;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
