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
