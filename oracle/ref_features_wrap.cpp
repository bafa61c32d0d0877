// C entry points over the reference's own feature-file serializer (serializeDataToFile /
// serializeDataFromFile of SerializableVector<SIFT_Feature>, V3D/Base/v3d_serialization.h:956-1017,
// V3D/Base/v3d_feature.h:12-49).  TEST INFRASTRUCTURE ONLY: it writes the fixtures the parser
// of the library is checked against, reads files back the reference's way, and is the timed
// CPU baseline of the ingestion workload.  Built into oracle/_ref from the sources where they lie.
#include <cstring>
#include <exception>
#include <vector>

#include "Base/v3d_feature.h"
#include "Base/v3d_serialization.h"

using V3D::SerializableVector;
using V3D::SIFT_Feature;

extern "C" {

// Writes n features, a binary archive when binary != 0, else a text archive.  Returns 0, or -1
// on an exception.
int ref_features_write_as(const char* path, int binary, int n, const int* ids, const float* pos, const float* dir,
                          const float* scale, const float* mag, const float* desc) {
  try {
    SerializableVector<SIFT_Feature> v(n);
    for (int i = 0; i < n; ++i) {
      SIFT_Feature& f = v[i];
      f.id = ids[i];
      f.position[0] = pos[2 * i];
      f.position[1] = pos[2 * i + 1];
      f.direction[0] = dir[2 * i];
      f.direction[1] = dir[2 * i + 1];
      f.scale = scale[i];
      f.magnitude = mag[i];
      std::memcpy(f.descriptor, desc + (size_t)i * 128, 128 * sizeof(float));
    }
    V3D::serializeDataToFile(path, v, binary != 0);
    return 0;
  } catch (...) {
    return -1;
  }
}

// Writes n features (binary archive).
int ref_features_write(const char* path, int n, const int* ids, const float* pos, const float* dir,
                       const float* scale, const float* mag, const float* desc) {
  return ref_features_write_as(path, 1, n, ids, pos, dir, scale, mag, desc);
}

// Reads a feature file the reference's way.  With cap < count only *n is set.  Returns 0, or
// -1 on an exception (unknown magic tag and the like).
int ref_features_read(const char* path, int cap, int* n, int* ids, float* pos, float* dir, float* scale, float* mag,
                      float* desc) {
  try {
    SerializableVector<SIFT_Feature> v;
    V3D::serializeDataFromFile(path, v);
    *n = (int)v.size();
    if (cap < (int)v.size()) return 0;
    for (size_t i = 0; i < v.size(); ++i) {
      const SIFT_Feature& f = v[i];
      ids[i] = f.id;
      pos[2 * i] = f.position[0];
      pos[2 * i + 1] = f.position[1];
      dir[2 * i] = f.direction[0];
      dir[2 * i + 1] = f.direction[1];
      scale[i] = f.scale;
      mag[i] = f.magnitude;
      std::memcpy(desc + i * 128, f.descriptor, 128 * sizeof(float));
    }
    return 0;
  } catch (...) {
    return -1;
  }
}

}  // extern "C"
