// Builds against compat/V3DM/v3dm_sfm_stages.h with stand-ins for the apps' types (the same member
// names as V3D's PointCorrespondence, Matrix3x3d and RobustOrientationResult) and runs both stages
// on a tiny input.  Without a GPU it must fail loudly (exit 1 with the header's message).
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

int main(int argc, char** argv) {
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
