// -*- C++ -*-
// compat/V3DM/v3dm_sfm_stages.h -- SfM-app stages around the matcher, batched on libv3dm.so, with
// the apps' own containers:
//   - findPutativeMatchesBatch() / runGuidedMatchingBatch(): match_sequence's per-pair loop
//     (V3D/Apps/SfM/match_sequence.cpp:165-234: setLeftFeatures, then setRightFeatures and
//     findPutativeMatches for every right view; runGuidedMatching after RANSAC, :306-324) for a
//     whole list of view pairs in one batched call, each pair's matches as that loop gets them;
//   - retrieveSequence(): the voctree app's retrieval loop (V3D/Apps/SfM/match_using_voctree.cpp:
//     176-222: LeafDocuments::computeBinomialScores, then insertDocument, for every image) in one
//     call, filling the same per-image score lists (nBestDocuments entries, best first) and the same
//     putativePairwiseMatches map (view1 -> set of view2);
//   - computeRobustOrientationBatch(): computeRobustOrientationMLE
//     (V3D/Apps/SfM/reconstruction_common.cpp:139-340, RobustOrientationMode() default, i.e. without
//     the iterative refinement) for many pairs at once; pair p draws its samples as that function
//     does after srand(seed + p).
// The result and matrix types are templates: any type with the members of
// RobustOrientationResult (essential, fundamental, rotation [i][j], translation [k], inliers,
// error) and correspondences with left.pos[k] / right.pos[k] work, the reference's included.
// Errors print and exit like the matcher header, or throw std::runtime_error with
// V3DM_COMPAT_THROW.
#ifndef V3DM_SFM_STAGES_H
#define V3DM_SFM_STAGES_H

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "v3dm.h"

namespace V3D_B200 {

namespace detail {

inline void check(int status, const char* what) {
  if (status == V3DM_OK) return;
  std::string msg = std::string("V3D_B200 ") + what + ": " + v3dm_status_string(status);
  if (status == V3DM_ERR_CUDA) msg += std::string(" [") + v3dm_last_error() + "]";
#ifdef V3DM_COMPAT_THROW
  throw std::runtime_error(msg);
#else
  std::fprintf(stderr, "%s\n", msg.c_str());
  std::exit(EXIT_FAILURE);
#endif
}

// Concatenated float descriptors of the views, each view cut to the count the apps pass to
// setLeftFeatures / setRightFeatures: min(nMaxFeatures, size & 0xffe0) (match_sequence.cpp:183,
// :215), its first descriptors in order.
template <typename Views>
inline void viewDescriptors(Views const& views, int nMaxFeatures, std::vector<int32_t>& counts,
                            std::vector<float>& desc) {
  const int n = (int)views.size();
  counts.assign(n, 0);
  size_t total = 0;
  for (int v = 0; v < n; ++v) {
    counts[v] = std::min(nMaxFeatures, int(views[v].size() & 0xffe0));
    if (counts[v] < 0) counts[v] = 0;
    total += (size_t)counts[v];
  }
  desc.resize(total * 128);
  size_t at = 0;
  for (int v = 0; v < n; ++v)
    for (int k = 0; k < counts[v]; ++k, ++at)
      for (int i = 0; i < 128; ++i) desc[at * 128 + i] = views[v][k].descriptor[i];
}

// Runs one batched call (putative, or guided with M/thr) and splits the (pair, left, right)
// triples into one (left, right) list per pair, ascending left.
inline void batchMatches(v3dm_batch* b, std::vector<std::pair<int, int> > const& pairs, const double* M,
                         const float* thr, float minScore, float minRatio,
                         std::vector<std::vector<std::pair<int, int> > >& matches, const char* who) {
  std::vector<int32_t> tab(2 * pairs.size());
  for (size_t p = 0; p < pairs.size(); ++p) {
    tab[2 * p] = pairs[p].first;
    tab[2 * p + 1] = pairs[p].second;
  }
  check(v3dm_batch_set_pairs(b, (int)pairs.size(), tab.data()), who);
  long long cap = 1 << 20, n = 0;
  std::vector<int32_t> t;
  for (int attempt = 0; attempt < 2; ++attempt) {
    t.resize((size_t)3 * (size_t)(cap > 0 ? cap : 1));
    const int st = M ? v3dm_batch_match_guided(b, 1, M, thr, minScore, minRatio, t.data(), cap, &n)
                     : v3dm_batch_match(b, minScore, minRatio, t.data(), cap, &n);
    if (st == V3DM_ERR_CAPACITY && attempt == 0) {
      cap = n;
      continue;
    }
    check(st, who);
    break;
  }
  matches.assign(pairs.size(), std::vector<std::pair<int, int> >());
  for (long long k = 0; k < n; ++k) matches[t[3 * k]].push_back(std::make_pair(t[3 * k + 1], t[3 * k + 2]));
}

}  // namespace detail

// views[v]: view v's features (any container of elements with descriptor[128] floats, e.g.
// SerializableVector<SIFT_Feature>); pairs[p] = (view1, view2), view1 the left.  matches[p]
// receives what findPutativeMatches(matches, minScore, minRatio) returns for that pair in the
// app's loop, with each view cut to min(nMaxFeatures, size & 0xffe0) features.  Descriptors that
// are not u/512 take the BF16 hi/lo path of the float matcher, as setLeftFeatures(float*) does.
template <typename Views>
inline void findPutativeMatchesBatch(Views const& views, int nMaxFeatures,
                                     std::vector<std::pair<int, int> > const& pairs, float minScore, float minRatio,
                                     std::vector<std::vector<std::pair<int, int> > >& matches, int device = 0) {
  const char* who = "findPutativeMatchesBatch()";
  std::vector<int32_t> counts;
  std::vector<float> desc;
  detail::viewDescriptors(views, nMaxFeatures, counts, desc);
  v3dm_batch* b = nullptr;
  detail::check(v3dm_batch_create(&b, device), who);
  const int st = v3dm_batch_set_images_f32(b, (int)counts.size(), counts.data(), desc.data());
  if (st != V3DM_OK) {
    v3dm_batch_destroy(b);
    detail::check(st, who);
  }
  detail::batchMatches(b, pairs, nullptr, nullptr, minScore, minRatio, matches, who);
  v3dm_batch_destroy(b);
}

// The same pairs after RANSAC: matches[p] receives runGuidedMatching(F[p], thr[p], leftPos,
// rightPos, matches, minScore, minRatio) of pair p after its findPutativeMatches, the positions
// being the features' position[0], position[1].  F[p] indexable as F[i][j] (e.g. Matrix3x3d).
template <typename Views, typename Mat3>
inline void runGuidedMatchingBatch(Views const& views, int nMaxFeatures, std::vector<std::pair<int, int> > const& pairs,
                                   std::vector<Mat3> const& F, std::vector<float> const& thr, float minScore,
                                   float minRatio, std::vector<std::vector<std::pair<int, int> > >& matches,
                                   int device = 0) {
  const char* who = "runGuidedMatchingBatch()";
  if (F.size() != pairs.size() || thr.size() != pairs.size()) detail::check(V3DM_ERR_ARG, who);
  std::vector<int32_t> counts;
  std::vector<float> desc;
  detail::viewDescriptors(views, nMaxFeatures, counts, desc);
  std::vector<float> pos;
  for (size_t v = 0; v < views.size(); ++v)
    for (int k = 0; k < counts[v]; ++k) {
      pos.push_back(views[v][k].position[0]);
      pos.push_back(views[v][k].position[1]);
    }
  std::vector<double> M(9 * pairs.size());
  for (size_t p = 0; p < pairs.size(); ++p)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) M[9 * p + 3 * i + j] = F[p][i][j];
  v3dm_batch* b = nullptr;
  detail::check(v3dm_batch_create(&b, device), who);
  int st = v3dm_batch_set_images_f32(b, (int)counts.size(), counts.data(), desc.data());
  if (st == V3DM_OK) st = v3dm_batch_set_positions(b, pos.empty() ? nullptr : pos.data());
  if (st != V3DM_OK) {
    v3dm_batch_destroy(b);
    detail::check(st, who);
  }
  detail::batchMatches(b, pairs, M.data(), thr.data(), minScore, minRatio, matches, who);
  v3dm_batch_destroy(b);
}

// visualWords[i]: the leaf-local words of image i (VocabularyTree::getVisualWord, or
// v3dm_voctree_quantize_* with V3DM_LEAF_LOCAL); nLeaves = the tree's visualWordCount().
// scores[i] = the first min(nBestDocuments, i) entries of the app's 'scores' for image i.
inline void retrieveSequence(int nLeaves, std::vector<std::vector<int> > const& visualWords, double pMatch,
                             int nBestDocuments, std::vector<std::vector<std::pair<float, int> > >& scores,
                             std::map<int, std::set<int> >& putativePairwiseMatches, int device = 0) {
  const int n = (int)visualWords.size();
  scores.assign(n, std::vector<std::pair<float, int> >());
  putativePairwiseMatches.clear();
  if (n == 0 || nBestDocuments < 1) return;
  std::vector<int32_t> offsets(n + 1, 0), words;
  for (int i = 0; i < n; ++i) {
    offsets[i + 1] = offsets[i] + (int32_t)visualWords[i].size();
    words.insert(words.end(), visualWords[i].begin(), visualWords[i].end());
  }
  std::vector<int32_t> docs((size_t)n * nBestDocuments);
  std::vector<float> sc((size_t)n * nBestDocuments);
  v3dm_retrieval* r = nullptr;
  detail::check(v3dm_retrieval_create(&r, device), "retrieveSequence()");
  const int st = v3dm_retrieval_binomial(r, nLeaves, n, offsets.data(), words.data(), pMatch, nBestDocuments,
                                         docs.data(), sc.data());
  v3dm_retrieval_destroy(r);
  detail::check(st, "retrieveSequence()");
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < nBestDocuments; ++j) {
      const int d = docs[(size_t)i * nBestDocuments + j];
      if (d < 0) break;
      scores[i].push_back(std::make_pair(sc[(size_t)i * nBestDocuments + j], d));
      putativePairwiseMatches[d].insert(i);
    }
}

// corrs[p]: the putative correspondences of pair p; K1[p], K2[p]: its calibrations (indexable as
// K[i][j]).  res[p] receives the result; pairs with fewer than 6 correspondences (for which the
// reference draws no sample; it throws below 5) or without a consistent sample get error -1 and no
// inliers.  iterativeRefinement is RobustOrientationMode::iterativeRefinement (the apps set it).
template <typename Corr, typename Mat3, typename Result>
inline void computeRobustOrientationBatch(std::vector<std::vector<Corr> > const& corrs, std::vector<Mat3> const& K1,
                                          std::vector<Mat3> const& K2, double inlierThreshold, int nSamples,
                                          std::vector<Result>& res, unsigned seed, int device = 0,
                                          bool iterativeRefinement = false) {
  const int nPairs = (int)corrs.size();
  res.assign(nPairs, Result());
  if (nPairs == 0) return;
  if ((int)K1.size() != nPairs || (int)K2.size() != nPairs)
    detail::check(V3DM_ERR_ARG, "computeRobustOrientationBatch(): one K1 and one K2 per pair");
  const int nDraw = nSamples + 1;
  // the reference's draws per pair; pairs for which it draws nothing (fewer than 6
  // correspondences) stay out of the batch and get no model
  std::vector<int> batch;  // pair of each batch entry
  std::vector<int32_t> samplesAll;
  for (int p = 0; p < nPairs; ++p) {
    std::vector<int32_t> s((size_t)nDraw * 5);
    int nd = 0;
    detail::check(v3dm_ransac_shuffle_samples((int)corrs[p].size(), nSamples, seed + (unsigned)p, nDraw, s.data(),
                                              &nd),
                  "computeRobustOrientationBatch()");
    if (nd == 0) continue;
    // a shorter sequence is padded with its last sample: a repeated sample's candidates never
    // beat the best so far, so the result is that of the sequence itself
    for (int k = nd; k < nDraw; ++k)
      for (int j = 0; j < 5; ++j) s[(size_t)5 * k + j] = s[(size_t)5 * (nd - 1) + j];
    batch.push_back(p);
    samplesAll.insert(samplesAll.end(), s.begin(), s.end());
  }
  for (int p = 0; p < nPairs; ++p) {
    res[p].error = -1.0;
    res[p].inliers.clear();
  }
  const int nb = (int)batch.size();
  if (nb == 0) return;
  std::vector<int32_t> offsets(nb + 1, 0);
  for (int q = 0; q < nb; ++q) offsets[q + 1] = offsets[q] + (int32_t)corrs[batch[q]].size();
  std::vector<float> c((size_t)offsets[nb] * 4);
  std::vector<double> K((size_t)nb * 18);
  for (int q = 0; q < nb; ++q) {
    const int p = batch[q];
    for (size_t i = 0; i < corrs[p].size(); ++i) {
      float* o = c.data() + 4 * ((size_t)offsets[q] + i);
      o[0] = corrs[p][i].left.pos[0];
      o[1] = corrs[p][i].left.pos[1];
      o[2] = corrs[p][i].right.pos[0];
      o[3] = corrs[p][i].right.pos[1];
    }
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        K[(size_t)q * 18 + 3 * a + b] = K1[p][a][b];
        K[(size_t)q * 18 + 9 + 3 * a + b] = K2[p][a][b];
      }
  }
  std::vector<double> models((size_t)nb * 31);
  std::vector<int32_t> nIn(nb);
  std::vector<uint8_t> flags((size_t)offsets[nb] + 1);
  v3dm_ransac* r = nullptr;
  detail::check(v3dm_ransac_create(&r, device), "computeRobustOrientationBatch()");
  int st = v3dm_ransac_set_refinement(r, iterativeRefinement ? 1 : 0);
  if (st == V3DM_OK)
    st = v3dm_ransac_essential(r, nb, offsets.data(), c.data(), K.data(), inlierThreshold, nSamples, nDraw,
                                       samplesAll.data(), 0, models.data(), nIn.data(), flags.data());
  v3dm_ransac_destroy(r);
  detail::check(st, "computeRobustOrientationBatch()");
  for (int q = 0; q < nb; ++q) {
    const int p = batch[q];
    const double* m = models.data() + (size_t)q * 31;
    if (m[30] < 0.0) continue;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        res[p].essential[a][b] = m[3 * a + b];
        res[p].fundamental[a][b] = m[9 + 3 * a + b];
        res[p].rotation[a][b] = m[18 + 3 * a + b];
      }
    for (int k = 0; k < 3; ++k) res[p].translation[k] = m[27 + k];
    res[p].error = m[30];
    for (int i = 0; i < (int)corrs[p].size(); ++i)
      if (flags[(size_t)offsets[q] + i]) res[p].inliers.push_back(i);
  }
}

}  // namespace V3D_B200

#endif  // V3DM_SFM_STAGES_H
