// Builds against compat/V3DM/v3dm_sfm_stages.h with stand-ins for the apps' types (the same member
// names as V3D's PointCorrespondence, Matrix3x3d, RobustOrientationResult and SIFT_Feature) and runs
// one stage on a tiny input.  Without a GPU it must fail loudly (exit 1 with the header's message).
// Mode 'm' / 'g' with an input and an output file: the batched putative / guided matching stage on
// the views and pairs of the input, its per-pair matches written to the output.
#include <cstdint>
#include <cstdio>
#include <vector>

#include "V3DM/v3dm_sfm_stages.h"

struct Vec2 {
  float v[2];
  float& operator[](int k) { return v[k]; }
  float operator[](int k) const { return v[k]; }
};
struct Measurement {
  Vec2 pos;
};
struct Corr {
  Measurement left, right;
};
struct Mat3 {
  double m[3][3];
  double* operator[](int i) { return m[i]; }
  const double* operator[](int i) const { return m[i]; }
};
struct Vec3 {
  double v[3];
  double& operator[](int k) { return v[k]; }
};
struct Result {
  Mat3 essential, fundamental, rotation;
  Vec3 translation;
  std::vector<int> inliers;
  double error;
};

struct Feature {
  Vec2 position;
  float descriptor[128];
};

// Input: int32 nViews, nPairs, nMaxFeatures; float minScore, minRatio; per view int32 n then n
// features (2 floats position, 128 floats descriptor); per pair int32 view1, view2, 9 doubles F,
// float thr.  Output: per pair int32 count then count (left, right) int32 pairs.
static int run_matching(bool guided, const char* in, const char* out) {
  FILE* f = std::fopen(in, "rb");
  if (!f) return 2;
  int32_t head[3];
  float params[2];
  if (std::fread(head, 4, 3, f) != 3 || std::fread(params, 4, 2, f) != 2) return 2;
  std::vector<std::vector<Feature> > views(head[0]);
  for (auto& v : views) {
    int32_t n = 0;
    if (std::fread(&n, 4, 1, f) != 1) return 2;
    v.resize(n);
    for (auto& x : v)
      if (std::fread(x.position.v, 4, 2, f) != 2 || std::fread(x.descriptor, 4, 128, f) != 128) return 2;
  }
  std::vector<std::pair<int, int> > pairs(head[1]);
  std::vector<Mat3> F(head[1]);
  std::vector<float> thr(head[1]);
  for (int p = 0; p < head[1]; ++p) {
    int32_t vv[2];
    if (std::fread(vv, 4, 2, f) != 2 || std::fread(F[p].m, 8, 9, f) != 9 || std::fread(&thr[p], 4, 1, f) != 1)
      return 2;
    pairs[p] = std::make_pair(vv[0], vv[1]);
  }
  std::fclose(f);
  std::vector<std::vector<std::pair<int, int> > > matches;
  if (guided)
    V3D_B200::runGuidedMatchingBatch(views, head[2], pairs, F, thr, params[0], params[1], matches);
  else
    V3D_B200::findPutativeMatchesBatch(views, head[2], pairs, params[0], params[1], matches);
  FILE* o = std::fopen(out, "wb");
  if (!o) return 2;
  for (auto const& m : matches) {
    const int32_t n = (int32_t)m.size();
    std::fwrite(&n, 4, 1, o);
    for (auto const& pr : m) {
      const int32_t lr[2] = {pr.first, pr.second};
      std::fwrite(lr, 4, 2, o);
    }
  }
  std::fclose(o);
  return 0;
}

int main(int argc, char** argv) {
  if (argc > 3 && (argv[1][0] == 'm' || argv[1][0] == 'g')) return run_matching(argv[1][0] == 'g', argv[2], argv[3]);
  const bool ransacFirst = argc > 1 && argv[1][0] == 'r';
  std::vector<std::vector<Corr> > corrs(2, std::vector<Corr>(40));
  for (int p = 0; p < 2; ++p)
    for (int i = 0; i < 40; ++i) {
      corrs[p][i].left.pos[0] = 10.0f * i;
      corrs[p][i].left.pos[1] = 7.0f * i;
      corrs[p][i].right.pos[0] = 10.0f * i + 3.0f;
      corrs[p][i].right.pos[1] = 7.0f * i;
    }
  Mat3 K = {{{1000, 0, 500}, {0, 1000, 400}, {0, 0, 1}}};
  std::vector<Mat3> K1(2, K), K2(2, K);
  std::vector<Result> res;
  std::vector<std::vector<int> > words(3, std::vector<int>(5, 1));
  std::vector<std::vector<std::pair<float, int> > > scores;
  std::map<int, std::set<int> > pairs;
  if (ransacFirst) {
    V3D_B200::computeRobustOrientationBatch(corrs, K1, K2, 2.0, 100, res, 7u);
  } else {
    V3D_B200::retrieveSequence(100, words, 0.1, 2, scores, pairs);
  }
  std::printf("ran\n");
  return 0;
}
