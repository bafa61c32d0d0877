// Application-side use of the compat header: the calls V3D/Apps/SfM/match_sequence.cpp makes on
// V3D_CUDA::SIFT_Matching and the ones match_using_voctree.cpp makes on VocabularyTreeTraversal,
// with small stand-ins for V3D::Matrix3x3d and V3D::Vector2f (anything indexable as M[i][j], p[k]).
//
//   compat_main match <in> <out>    in:  int32 nL, nR; float minScore, minRatio, thr; double F[9];
//                                        float L[nL*128], R[nR*128], lpos[nL*2], rpos[nR*2]
//                                   out: int32 nPutative, pairs..., int32 nGuided, pairs...
//   compat_main voctree <in> <out>  in:  int32 n; float nodes[1110*128]; float keys[n*128]
//                                   out: int32 ids[n]   (VocabularyTreeTraversal<10, 3>)
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#define V3DM_COMPAT_THROW
#include "CUDA/v3d_cudamatching.h"

namespace {

struct Matrix3x3d {
  double m[3][3];
  const double* operator[](int i) const { return m[i]; }
};

struct Vector2f {
  float v[2];
  float operator[](int k) const { return v[k]; }
};

template <class T>
void read_into(FILE* f, T* dst, size_t n) {
  if (n && std::fread(dst, sizeof(T), n, f) != n) {
    std::fprintf(stderr, "short read\n");
    std::exit(3);
  }
}

void write_pairs(FILE* f, const std::vector<std::pair<int, int> >& m) {
  const int n = (int)m.size();
  std::fwrite(&n, sizeof(int), 1, f);
  for (const auto& p : m) {
    std::fwrite(&p.first, sizeof(int), 1, f);
    std::fwrite(&p.second, sizeof(int), 1, f);
  }
}

int run_match(FILE* in, FILE* out) {
  int nL = 0, nR = 0;
  float minScore = 0, minRatio = 0, thr = 0;
  Matrix3x3d F;
  read_into(in, &nL, 1);
  read_into(in, &nR, 1);
  read_into(in, &minScore, 1);
  read_into(in, &minRatio, 1);
  read_into(in, &thr, 1);
  read_into(in, &F.m[0][0], 9);
  std::vector<float> L((size_t)nL * 128), R((size_t)nR * 128);
  std::vector<Vector2f> lp((size_t)nL), rp((size_t)nR);
  read_into(in, L.data(), L.size());
  read_into(in, R.data(), R.size());
  read_into(in, &lp[0].v[0], 2 * lp.size());
  read_into(in, &rp[0].v[0], 2 * rp.size());

  V3D_CUDA::SIFT_Matching matcher;
  matcher.enableRoundingWarning(false);
  matcher.allocate(nL > nR ? nL : nR, true);
  matcher.setLeftFeatures(nL, L.data());
  matcher.setRightFeatures(nR, R.data());
  std::vector<std::pair<int, int> > matches;
  matcher.findPutativeMatches(matches, minScore, minRatio);
  write_pairs(out, matches);
  matcher.runGuidedMatching(F, thr, lp.data(), rp.data(), matches, minScore, minRatio);
  write_pairs(out, matches);
  matcher.deallocate();
  return 0;
}

int run_voctree(FILE* in, FILE* out) {
  typedef V3D_CUDA::VocabularyTreeTraversal<10, 3> Tree;
  int n = 0;
  read_into(in, &n, 1);
  std::vector<float> nodes((size_t)Tree::getNodeCount() * 128), keys((size_t)n * 128);
  read_into(in, nodes.data(), nodes.size());
  read_into(in, keys.data(), keys.size());
  Tree tree;
  tree.allocate(n);
  tree.setNodes(nodes.data());
  std::vector<int> ids((size_t)n, -1);
  tree.traverseTree(n, keys.data(), ids.data());
  tree.deallocate();
  std::fwrite(ids.data(), sizeof(int), ids.size(), out);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: %s match|voctree <in> <out>\n", argv[0]);
    return 2;
  }
  FILE* in = std::fopen(argv[2], "rb");
  FILE* out = std::fopen(argv[3], "wb");
  if (!in || !out) return 2;
  int rc = 2;
  try {
    if (!std::strcmp(argv[1], "match")) rc = run_match(in, out);
    else if (!std::strcmp(argv[1], "voctree")) rc = run_voctree(in, out);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "%s\n", e.what());
    rc = 1;
  }
  std::fclose(in);
  std::fclose(out);
  return rc;
}
