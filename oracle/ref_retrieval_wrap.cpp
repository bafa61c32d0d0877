// C entry point over the reference's own vocabulary-tree retrieval scoring: the image loop of
// match_using_voctree.cpp:176-222 (query the inverted files with computeBinomialScores, keep the
// nBestDocuments best earlier images, then insertDocument) on V3D::LeafDocuments
// (V3D/Base/v3d_voctree.h:105-289).  TEST INFRASTRUCTURE ONLY: the parity pin and the timed CPU
// baseline of the retrieval workload.  Built into oracle/_ref from the sources where they lie.
#include <algorithm>
#include <chrono>
#include <utility>
#include <vector>

#include "Base/v3d_voctree.h"

extern "C" {

// words: the leaf-local visual words of every image, images concatenated (offsets[nImages + 1]).
// For image i, bestDocs[i * nBest + j] / bestScores[...] receive the j-th best earlier image and
// its score (fewer than nBest when i < nBest; the rest is set to -1 / 0).  Returns 0.
int ref_retrieval(int nLeaves, int nImages, const int* offsets, const int* words, double pMatch, int nBest,
                  int* bestDocs, float* bestScores) {
  V3D::LeafDocuments inv(nLeaves);
  for (int i = 0; i < nImages; ++i) {
    std::vector<int> vw(words + offsets[i], words + offsets[i + 1]);
    std::vector<std::pair<float, int> > scores;
    inv.computeBinomialScores(pMatch, vw, scores, nBest);
    for (int j = 0; j < nBest; ++j) {
      const bool have = j < (int)scores.size();
      bestDocs[(size_t)i * nBest + j] = have ? scores[j].second : -1;
      bestScores[(size_t)i * nBest + j] = have ? scores[j].first : 0.0f;
    }
    inv.insertDocument(vw);
  }
  return 0;
}

// The same loop with the queries of a sample of the images timed: every image is inserted; image
// i is queried when i % stride == phase.  *queryS = the time of those queries, *insertS = the
// time of all insertions, *nQueries = their count; *checksum = the sum of the best documents'
// ids of the queried images.  Returns 0.
int ref_retrieval_sampled(int nLeaves, int nImages, const int* offsets, const int* words, double pMatch, int nBest,
                          int stride, int phase, double* queryS, double* insertS, int* nQueries, long long* checksum) {
  typedef std::chrono::steady_clock clk;
  V3D::LeafDocuments inv(nLeaves);
  double tq = 0.0, ti = 0.0;
  int nq = 0;
  long long sum = 0;
  for (int i = 0; i < nImages; ++i) {
    std::vector<int> vw(words + offsets[i], words + offsets[i + 1]);
    if (i % stride == phase) {
      std::vector<std::pair<float, int> > scores;
      const clk::time_point t0 = clk::now();
      inv.computeBinomialScores(pMatch, vw, scores, nBest);
      tq += std::chrono::duration<double>(clk::now() - t0).count();
      ++nq;
      for (int j = 0; j < std::min(nBest, (int)scores.size()); ++j) sum += scores[j].second;
    }
    const clk::time_point t1 = clk::now();
    inv.insertDocument(vw);
    ti += std::chrono::duration<double>(clk::now() - t1).count();
  }
  *queryS = tq;
  *insertS = ti;
  *nQueries = nq;
  *checksum = sum;
  return 0;
}

}  // extern "C"
