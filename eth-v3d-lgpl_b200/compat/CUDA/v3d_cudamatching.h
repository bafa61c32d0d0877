// -*- C++ -*-
// compat/CUDA/v3d_cudamatching.h -- the V3D_CUDA matching classes on top of libv3dm.so.
//
// Same struct names, member functions, arguments and defaults as the reference header
// V3D/CUDA/v3d_cudamatching.h:15-105, so that the SfM apps (V3D/Apps/SfM/match_sequence.cpp,
// match_using_voctree.cpp) compile unchanged when this directory comes first on their include
// path and they link libv3dm.so.  Behaviour kept from the reference (v3d_cudamatching.cu):
//   - allocate() and set*Features() round counts down to a multiple of 32 (warning on stderr
//     when enableRoundingWarning is on) and clamp them to the allocated maximum (.cu:444-519);
//   - findPutativeMatches() clears 'matches' and fills (left, right) pairs in ascending left
//     order (.cu:522-552); minRatio < 0 disables the ratio test (.cu:535);
//   - runGuided*Matching() applies its gate on top of the gates of earlier guided calls since
//     the last findPutativeMatches(), as the reference's in-place masking does (.cu:597, :668);
//   - any error prints a message and exits (CUDA_SAFE_CALL, .cu:12-27) -- or throws
//     std::runtime_error when V3DM_COMPAT_THROW is defined before this header.
// Differences: enableReductionPath() is accepted and has no effect (the reference's reduction
// kernels read past their shared arrays and race, .cu:87-130, :212-273; the non-reduction
// semantics are used); float descriptors of the form u/512 are scored exactly on the integer
// path, any other finite floats (the extractors' unit-L2 descriptors) with a BF16 hi/lo split
// (score error <= 2e-5 of FP64, then the reference's decision rules; the reference scores them
// with FP32 cuBLAS); VocabularyTreeTraversal returns the ids of the reference's CPU tree
// (v3d_voctree.h:82-99: sequential FP32 dot products) for any float tree and features.  The guided
// calls take the reference's V3D::Matrix3x3d / V3D::Vector2f (any type indexable as F[i][j] and
// p[k]).
#ifndef V3D_CUDA_MATCHING_H
#define V3D_CUDA_MATCHING_H

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "v3dm.h"

namespace V3D_CUDA {

namespace detail {

inline void check(int status, const char* what) {
  if (status == V3DM_OK) return;
  std::string msg = std::string("V3D_CUDA ") + what + ": " + v3dm_status_string(status);
  if (status == V3DM_ERR_CUDA) msg += std::string(" [") + v3dm_last_error() + "]";
#ifdef V3DM_COMPAT_THROW
  throw std::runtime_error(msg);
#else
  std::fprintf(stderr, "%s\n", msg.c_str());
  std::exit(EXIT_FAILURE);
#endif
}

// Round down to a multiple of 32 as the reference does, with its warning text.
inline int round32(int n, bool warn, const char* who, const char* what) {
  if (n % 32 != 0) {
    if (warn) {
      std::cerr << who << " warning: " << what << " should be a multiple of 32" << std::endl;
      std::cerr << "Rounding " << what << " down." << std::endl;
    }
    n = n - (n & 31);
  }
  return n;
}

}  // namespace detail

struct SIFT_Matching {
  SIFT_Matching()
      : _warnOnRounding(true),
        _useReductionPath(false),
        _useGuidedMatching(false),
        _nMaxLeftFeatures(0),
        _nMaxRightFeatures(0),
        _nLeftFeatures(0),
        _nRightFeatures(0),
        _h(nullptr) {
    detail::check(v3dm_matcher_create(&_h, 0, V3DM_KERNEL_TCGEN05), "SIFT_Matching()");
  }

  ~SIFT_Matching() {
    if (_h) v3dm_matcher_destroy(_h);
  }

  SIFT_Matching(const SIFT_Matching&) = delete;
  SIFT_Matching& operator=(const SIFT_Matching&) = delete;

  void enableRoundingWarning(bool flag = true) { _warnOnRounding = flag; }

  // Accepted for source compatibility; the non-reduction semantics are always used.
  void enableReductionPath(bool flag = true) { _useReductionPath = flag; }

  void allocate(int nMaxLeftFeatures, int nMaxRightFeatures, bool useGuidedMatching = false) {
    _useGuidedMatching = useGuidedMatching;
    nMaxLeftFeatures = detail::round32(nMaxLeftFeatures, _warnOnRounding, "SIFT_Matching::allocate()", "nMaxLeftFeatures");
    nMaxRightFeatures =
        detail::round32(nMaxRightFeatures, _warnOnRounding, "SIFT_Matching::allocate()", "nMaxRightFeatures");
    _nMaxLeftFeatures = nMaxLeftFeatures;
    _nMaxRightFeatures = nMaxRightFeatures;
    detail::check(v3dm_allocate(_h, nMaxLeftFeatures, nMaxRightFeatures, useGuidedMatching ? 1 : 0), "allocate");
  }

  void allocate(int nMaxFeatures, bool useGuidedMatching = false) {
    this->allocate(nMaxFeatures, nMaxFeatures, useGuidedMatching);
  }

  void deallocate() { detail::check(v3dm_deallocate(_h), "deallocate"); }

  void setLeftFeatures(int nFeatures, float const* descriptors) {
    nFeatures = detail::round32(nFeatures, _warnOnRounding, "SIFT_Matching::setLeftFeatures()", "nFeatures");
    _nLeftFeatures = std::min(nFeatures, _nMaxLeftFeatures);
    detail::check(v3dm_set_left_f32(_h, _nLeftFeatures, descriptors), "setLeftFeatures");
  }

  void setRightFeatures(int nFeatures, float const* descriptors) {
    nFeatures = detail::round32(nFeatures, _warnOnRounding, "SIFT_Matching::setRightFeatures()", "nFeatures");
    _nRightFeatures = std::min(nFeatures, _nMaxRightFeatures);
    detail::check(v3dm_set_right_f32(_h, _nRightFeatures, descriptors), "setRightFeatures");
  }

  // Ratio test is disabled if minRatio < 0.
  void findPutativeMatches(std::vector<std::pair<int, int> >& matches, float const minScore = 0.9f,
                           float const minRatio = 0.8f) {
    const int cap = std::min(_nLeftFeatures, _nRightFeatures);
    std::vector<int32_t> buf(2 * (size_t)std::max(cap, 1));
    int n = 0;
    detail::check(v3dm_putative(_h, minScore, minRatio, buf.data(), cap, &n), "findPutativeMatches");
    fill(matches, buf, n);
  }

  template <class Mat, class Vec2>
  void runGuidedMatching(Mat const& F, float const distanceThreshold, Vec2 const* leftPositions,
                         Vec2 const* rightPositions, std::vector<std::pair<int, int> >& matches,
                         float const minScore = 0.9f, float const minRatio = 0.8f) {
    guided(1, F, distanceThreshold, leftPositions, rightPositions, matches, minScore, minRatio);
  }

  template <class Mat, class Vec2>
  void runGuidedHomographyMatching(Mat const& H, float const distanceThreshold, Vec2 const* leftPositions,
                                   Vec2 const* rightPositions, std::vector<std::pair<int, int> >& matches,
                                   float const minScore = 0.9f, float const minRatio = 0.8f) {
    guided(2, H, distanceThreshold, leftPositions, rightPositions, matches, minScore, minRatio);
  }

 protected:
  static void fill(std::vector<std::pair<int, int> >& matches, const std::vector<int32_t>& buf, int n) {
    matches.clear();
    matches.reserve((size_t)n);
    for (int k = 0; k < n; ++k) matches.push_back(std::make_pair(buf[2 * k], buf[2 * k + 1]));
  }

  template <class Mat, class Vec2>
  void guided(int type, Mat const& M, float thr, Vec2 const* lp, Vec2 const* rp,
              std::vector<std::pair<int, int> >& matches, float minScore, float minRatio) {
    double m[9];
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) m[3 * i + j] = M[i][j];
    // Interleaved (x, y) floats, the memory layout of a V3D::Vector2f array.
    std::vector<float> l(2 * (size_t)std::max(_nLeftFeatures, 1)), r(2 * (size_t)std::max(_nRightFeatures, 1));
    for (int k = 0; k < _nLeftFeatures; ++k) {
      l[2 * k] = lp[k][0];
      l[2 * k + 1] = lp[k][1];
    }
    for (int k = 0; k < _nRightFeatures; ++k) {
      r[2 * k] = rp[k][0];
      r[2 * k + 1] = rp[k][1];
    }
    const int cap = std::min(_nLeftFeatures, _nRightFeatures);
    std::vector<int32_t> buf(2 * (size_t)std::max(cap, 1));
    int n = 0;
    const int st = type == 1 ? v3dm_guided_F(_h, m, thr, l.data(), r.data(), minScore, minRatio, buf.data(), cap, &n)
                             : v3dm_guided_H(_h, m, thr, l.data(), r.data(), minScore, minRatio, buf.data(), cap, &n);
    detail::check(st, type == 1 ? "runGuidedMatching" : "runGuidedHomographyMatching");
    fill(matches, buf, n);
  }

  bool _warnOnRounding;
  bool _useReductionPath;
  bool _useGuidedMatching;
  int _nMaxLeftFeatures, _nMaxRightFeatures, _nLeftFeatures, _nRightFeatures;
  v3dm_matcher* _h;
};  // end struct SIFT_Matching

template <int BranchFactor, int Depth>
struct VocabularyTreeTraversal {
  VocabularyTreeTraversal() : _nMaxFeatures(0), _h(nullptr) {
    detail::check(v3dm_voctree_create(&_h, 0, BranchFactor, Depth), "VocabularyTreeTraversal()");
  }

  ~VocabularyTreeTraversal() {
    if (_h) v3dm_voctree_destroy(_h);
  }

  VocabularyTreeTraversal(const VocabularyTreeTraversal&) = delete;
  VocabularyTreeTraversal& operator=(const VocabularyTreeTraversal&) = delete;

  void allocate(int nMaxFeatures) {
    if (nMaxFeatures % 32 != 0) {
      std::cerr << "VocabularyTreeTraversal::allocate() warning: nMaxFeatures should be a multiple of 32" << std::endl;
      std::cerr << "Rounding nFeatures down." << std::endl;
      nMaxFeatures = nMaxFeatures - (nMaxFeatures & 31);
    }
    _nMaxFeatures = nMaxFeatures;
    detail::check(v3dm_voctree_allocate(_h, nMaxFeatures), "allocate");
  }

  void deallocate() {}

  // Nodes in breadth-first order without the root (getNodeCount() x 128 floats).
  void setNodes(float const* nodes) { detail::check(v3dm_voctree_set_nodes_f32(_h, nodes), "setNodes"); }

  // Writes the node index of each feature's leaf, as the reference's traverseTree (.cu:791).
  void traverseTree(int nFeatures, float const* features, int* leaveIds) {
    if (nFeatures > _nMaxFeatures) {
      std::cerr << "VocabularyTreeTraversal::traverseTree() warning: nFeatures is larger than nMaxFeatures."
                << std::endl;
      std::cerr << "Reducing nFeatures." << std::endl;
      nFeatures = _nMaxFeatures;
    }
    detail::check(v3dm_voctree_quantize_f32(_h, nFeatures, features, reinterpret_cast<int32_t*>(leaveIds),
                                            V3DM_LEAF_GLOBAL),
                  "traverseTree");
  }

  static inline int getNodeCount() {
    int res = 0, len = 1;
    for (int d = 0; d < Depth; ++d) {
      len *= BranchFactor;
      res += len;
    }
    return res;
  }

  static inline int getLeaveCount() {
    int res = 1;
    for (int d = 0; d < Depth; ++d) res *= BranchFactor;
    return res;
  }

 protected:
  int _nMaxFeatures;
  v3dm_voctree* _h;
};  // end struct VocabularyTreeTraversal

}  // end namespace V3D_CUDA

#endif
