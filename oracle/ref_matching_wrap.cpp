/*
 * ref_matching_wrap.cpp -- extern "C" entry point around the reference's own
 * V3D_CUDA::SIFT_Matching (V3D/CUDA/v3d_cudamatching.h:15-67), compiled from the
 * reference's sources by oracle/Makefile into oracle/_ref/libv3dref_cuda.so.
 *
 * TEST INFRASTRUCTURE ONLY: the reference's GPU matcher, run on a B200, pins the CPU
 * oracle.  It follows the app call sequence of V3D/Apps/SfM/match_sequence.cpp:111-139,
 * :188, :231, :234, :324 (cublasInit, allocate, setLeft/RightFeatures, findPutativeMatches,
 * then runGuidedMatching / runGuidedHomographyMatching once per gate, in order).
 * The reduction path (enableReductionPath) is never enabled: its kernels read shared
 * memory past their arrays (v3d_cudamatching.cu:108-121, :246-250).
 * The reference exits the process on any CUDA error (v3d_cudamatching.cu:12-27), so
 * callers run this in a child process.
 */
#include <cublas.h>
#include <vector>
#include "CUDA/v3d_cudamatching.h"

extern "C" int v3dref_match(int nMaxL, int nMaxR, int nL, int nR, const float* L, const float* R, float minScore,
                            float minRatio, int nGates, const int* gateTypes, const double* gateMats,
                            const float* gateThr, const float* lpos, const float* rpos, int* pairs,
                            int* nPutative) {
    // The reference kernels index whole 32-thread blocks; only multiples of 32 are safe.
    if (nL < 32 || nR < 32 || (nL % 32) || (nR % 32) || nL > nMaxL || nR > nMaxR) return -1;
    static bool inited = false;
    if (!inited) {
        cublasInit();
        inited = true;
    }
    V3D_CUDA::SIFT_Matching m;
    m.enableRoundingWarning(false);
    m.enableReductionPath(false);
    m.allocate(nMaxL, nMaxR, nGates > 0);
    m.setLeftFeatures(nL, L);
    m.setRightFeatures(nR, R);
    std::vector<std::pair<int, int> > matches;
    m.findPutativeMatches(matches, minScore, minRatio);
    if (nPutative) *nPutative = (int)matches.size();
    const V3D::Vector2f* lp = reinterpret_cast<const V3D::Vector2f*>(lpos);
    const V3D::Vector2f* rp = reinterpret_cast<const V3D::Vector2f*>(rpos);
    for (int g = 0; g < nGates; ++g) {
        V3D::Matrix3x3d M;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) M[i][j] = gateMats[9 * g + 3 * i + j];
        if (gateTypes[g] == 1)
            m.runGuidedMatching(M, gateThr[g], lp, rp, matches, minScore, minRatio);
        else
            m.runGuidedHomographyMatching(M, gateThr[g], lp, rp, matches, minScore, minRatio);
    }
    m.deallocate();
    for (size_t k = 0; k < matches.size(); ++k) {
        pairs[2 * k] = matches[k].first;
        pairs[2 * k + 1] = matches[k].second;
    }
    return (int)matches.size();
}

/*
 * Timing of the reference matcher in the apps' loop (V3D/Apps/SfM/match_sequence.cpp:165-234:
 * one allocate, then per pair setLeftFeatures, setRightFeatures, findPutativeMatches and,
 * for guided matching, runGuidedMatching with the pair's F).  Feature counts are rounded
 * down to multiples of 32 and clamped to nMax, as the apps do ('& 0xffe0') before the call.
 * Images: desc holds the images' descriptors concatenated (u/512 floats), image i at rows
 * offsets[i] .. offsets[i+1]-1; pos the matching keypoint positions (x, y) when guided.
 * pairs: nPairs (left image, right image); F: 9 doubles per pair (row-major) when guided.
 * The loop runs `reps` times; seconds[k] is the wall time of repetition k (the reference's
 * copies are blocking, so a call has finished when it returns).  *nMatches is the total of
 * the last repetition's pairs (putative, plus guided when guided).
 */
#include <chrono>

extern "C" int v3dref_time_pairs(int nMax, int nImages, const int* offsets, const float* desc, const float* pos,
                                 int nPairs, const int* pairs, int guided, const double* F, float thr,
                                 float minScore, float minRatio, int reps, double* seconds, long long* nMatches) {
    if (nMax < 32 || nImages < 1 || nPairs < 0 || reps < 1) return -1;
    static bool inited = false;
    if (!inited) {
        cublasInit();
        inited = true;
    }
    V3D_CUDA::SIFT_Matching m;
    m.enableRoundingWarning(false);
    m.enableReductionPath(false);
    m.allocate(nMax, guided != 0);
    std::vector<std::pair<int, int> > matches;
    long long total = 0;
    for (int rep = 0; rep < reps; ++rep) {
        total = 0;
        auto t0 = std::chrono::steady_clock::now();
        for (int p = 0; p < nPairs; ++p) {
            const int i = pairs[2 * p], j = pairs[2 * p + 1];
            int nL = (offsets[i + 1] - offsets[i]) & ~31, nR = (offsets[j + 1] - offsets[j]) & ~31;
            if (nL > nMax) nL = nMax;
            if (nR > nMax) nR = nMax;
            if (nL < 32 || nR < 32) continue;
            m.setLeftFeatures(nL, desc + (size_t)offsets[i] * 128);
            m.setRightFeatures(nR, desc + (size_t)offsets[j] * 128);
            m.findPutativeMatches(matches, minScore, minRatio);
            total += (long long)matches.size();
            if (guided) {
                V3D::Matrix3x3d M;
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) M[a][b] = F[9 * p + 3 * a + b];
                m.runGuidedMatching(M, thr, reinterpret_cast<const V3D::Vector2f*>(pos + 2 * (size_t)offsets[i]),
                                    reinterpret_cast<const V3D::Vector2f*>(pos + 2 * (size_t)offsets[j]), matches,
                                    minScore, minRatio);
                total += (long long)matches.size();
            }
        }
        seconds[rep] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    m.deallocate();
    if (nMatches) *nMatches = total;
    return 0;
}
