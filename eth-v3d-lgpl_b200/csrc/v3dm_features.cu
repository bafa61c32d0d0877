// v3dm_features.cu -- ingestion of the reference's feature files (".features").
//
// The SfM apps load one binary archive per image with serializeDataFromFile(name,
// SerializableVector<SIFT_Feature>&) (V3D/Base/v3d_serialization.h:983-1017; the loader is
// match_sequence.cpp:124-146), then copy each feature's 128 floats into a per-pair array for
// setLeftFeatures / setRightFeatures (match_sequence.cpp:183-186, 214-231).  The archive is
//   "V3DBIN" (6 bytes), uint32 count (little endian, put_uint32, v3d_serialization.h:418-426),
//   then per feature: int32 id (little endian), position[2], direction[2], scale, magnitude and
//   descriptor[128] as raw 4-byte floats (put_blob, :428-432; field order v3d_feature.h:38-47),
// 540 bytes per feature.  Here:
//   - v3dm_features_read parses one file into caller arrays (the reference's deserializer);
//   - a loader reads many files at once (one host thread per file at a time), keeps the
//     positions on the host and copies all descriptors to the device in one transfer from
//     pinned memory.  There they become u8 (u = 512 x) for the u8 matchers
//     (v3dm_batch_set_images_u8_device, v3dm_set_left_u8_device) when every value is exactly
//     u/512; the extractors' unit-L2 floats (normalizeDescriptor, v3d_feature.h:19-39) are not,
//     so those are kept as floats (V3DM_LOAD_KEEP_F32) for the float matcher
//     (v3dm_set_left_f32_device: BF16 hi/lo scores), refused (V3DM_ERR_NOT_U8), or rounded
//     only when the caller asks for it (V3DM_LOAD_LOSSY_U8).
// The text archive ("V3DTXT", serializeDataToFile(..., writeBinary = false), :956-977) is read
// too: "V3DTXT", then whitespace-separated tokens written by TextOStreamArchive (:177-265): the
// count, "{", per feature the tag "SIFT_Feature", "{", the 135 values and "}", and a closing "}".
// Values are parsed as TextIStreamArchive's `is >> value` parses them (:267-338: decimal digits,
// sign, point and exponent only, strtof rounding for floats); a value it could not read (a
// "nan" or "inf" the writer printed, an overflow, a stray character) or a wrong tag or bracket
// gives V3DM_ERR_IO, where the reference throws.
#include <algorithm>
#include <atomic>
#include <cctype>
#include <cstdio>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <thread>
#include <vector>

#include "v3dm_device.cuh"

namespace v3dm {

namespace {

constexpr int kTagLen = 6;
constexpr size_t kHeaderBytes = kTagLen + 4;
constexpr size_t kFeatureBytes = 4 + 6 * 4 + 128 * 4;

uint32_t le32(const unsigned char* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

// Floats are written in the host's byte order by the reference (put_blob); the archives this
// reads come from little-endian hosts, as this one is.
bool host_little_endian() {
  const uint32_t one = 1;
  unsigned char b;
  std::memcpy(&b, &one, 1);
  return b == 1;
}

struct FileReader {
  FILE* f = nullptr;
  bool text = false;        // a V3DTXT archive: the rest of the file is in txt
  std::vector<char> txt;    // text after the tag, NUL-terminated
  size_t at = 0;            // next unread character of txt
  ~FileReader() {
    if (f) std::fclose(f);
  }
  // The next whitespace-delimited token of a text archive, or nullptr at its end.  The token is
  // NUL-terminated in place.
  char* token() {
    char* p = txt.data();
    const size_t n = txt.size() - 1;
    while (at < n && std::isspace((unsigned char)p[at])) ++at;
    if (at >= n) return nullptr;
    char* t = p + at;
    while (at < n && !std::isspace((unsigned char)p[at])) ++at;
    p[at] = '\0';
    if (at < n) ++at;
    return t;
  }
};

// A token of a number as the stream extraction accepts it: digits, signs, point and exponent.
bool number_chars(const char* t, bool allowFloat) {
  if (!*t) return false;
  for (const char* c = t; *c; ++c) {
    const bool ok = (*c >= '0' && *c <= '9') || *c == '+' || *c == '-' ||
                    (allowFloat && (*c == '.' || *c == 'e' || *c == 'E'));
    if (!ok) return false;
  }
  return true;
}

bool parse_float(const char* t, float* v) {
  if (!t || !number_chars(t, true)) return false;
  char* end = nullptr;
  const float x = std::strtof(t, &end);
  if (end == t || *end != '\0' || std::isinf(x)) return false;  // an overflow fails the extraction
  *v = x;
  return true;
}

bool parse_long(const char* t, long long lo, long long hi, long long* v) {
  if (!t || !number_chars(t, false)) return false;
  char* end = nullptr;
  errno = 0;
  const long long x = std::strtoll(t, &end, 10);
  if (end == t || *end != '\0' || errno == ERANGE || x < lo || x > hi) return false;
  *v = x;
  return true;
}

bool is_tag(const char* t, const char* want) { return t && std::strcmp(t, want) == 0; }

// Opens a feature file and checks its header; *count is the number of features it holds.
int open_features(const char* path, FileReader& r, uint32_t* count) {
  r.f = std::fopen(path, "rb");
  if (!r.f) return V3DM_ERR_IO;
  unsigned char head[kHeaderBytes];
  if (std::fread(head, 1, kTagLen, r.f) != (size_t)kTagLen) return V3DM_ERR_IO;
  if (std::memcmp(head, "V3DTXT", kTagLen) == 0) {
    r.text = true;
    if (std::fseek(r.f, 0, SEEK_END) != 0) return V3DM_ERR_IO;
    const long long size = std::ftell(r.f);
    if (size < kTagLen || std::fseek(r.f, (long)kTagLen, SEEK_SET) != 0) return V3DM_ERR_IO;
    r.txt.assign((size_t)(size - kTagLen) + 1, '\0');
    if (std::fread(r.txt.data(), 1, (size_t)(size - kTagLen), r.f) != (size_t)(size - kTagLen)) return V3DM_ERR_IO;
    long long c = 0;
    // an unsigned int, then the vector's opening bracket (serializeVector, :852-859)
    if (!parse_long(r.token(), 0, 0xffffffffLL, &c) || !is_tag(r.token(), "{")) return V3DM_ERR_IO;
    *count = (uint32_t)c;
    return V3DM_OK;
  }
  if (std::memcmp(head, "V3DBIN", kTagLen) != 0) return V3DM_ERR_IO;
  if (std::fread(head + kTagLen, 1, 4, r.f) != 4) return V3DM_ERR_IO;
  *count = le32(head + kTagLen);
  // the file must hold all of its features
  if (std::fseek(r.f, 0, SEEK_END) != 0) return V3DM_ERR_IO;
  const long long size = std::ftell(r.f);
  if (size < 0 || (unsigned long long)size < kHeaderBytes + (unsigned long long)*count * kFeatureBytes)
    return V3DM_ERR_IO;
  if (std::fseek(r.f, (long)kHeaderBytes, SEEK_SET) != 0) return V3DM_ERR_IO;
  return V3DM_OK;
}

// Decodes the first n features of a text archive opened by open_features.  With n equal to the
// file's count (whole) the closing bracket must follow, as the reference's reader requires.
int decode_text(FileReader& r, long long n, bool whole, int32_t* ids, float* pos, float* dir, float* scale,
                float* mag, float* desc) {
  for (long long i = 0; i < n; ++i) {
    if (!is_tag(r.token(), "SIFT_Feature") || !is_tag(r.token(), "{")) return V3DM_ERR_IO;
    long long id = 0;
    if (!parse_long(r.token(), -2147483648LL, 2147483647LL, &id)) return V3DM_ERR_IO;
    float v[134];
    for (int k = 0; k < 134; ++k)
      if (!parse_float(r.token(), &v[k])) return V3DM_ERR_IO;
    if (!is_tag(r.token(), "}")) return V3DM_ERR_IO;
    if (ids) ids[i] = (int32_t)id;
    if (pos) {
      pos[2 * i] = v[0];
      pos[2 * i + 1] = v[1];
    }
    if (dir) {
      dir[2 * i] = v[2];
      dir[2 * i + 1] = v[3];
    }
    if (scale) scale[i] = v[4];
    if (mag) mag[i] = v[5];
    if (desc) std::memcpy(desc + i * 128, v + 6, 128 * sizeof(float));
  }
  if (whole && !is_tag(r.token(), "}")) return V3DM_ERR_IO;
  return V3DM_OK;
}

// Decodes the first n features of an open file (positioned after the header).  Null outputs
// are skipped.  Binary archives are read in blocks of kBlock features.
int decode_features(FileReader& r, long long n, bool whole, int32_t* ids, float* pos, float* dir, float* scale,
                    float* mag, float* desc) {
  if (r.text) return decode_text(r, n, whole, ids, pos, dir, scale, mag, desc);
  FILE* f = r.f;
  constexpr int kBlock = 2048;
  std::vector<unsigned char> buf((size_t)kBlock * kFeatureBytes);
  for (long long i0 = 0; i0 < n; i0 += kBlock) {
    const int m = (int)std::min<long long>(kBlock, n - i0);
    if (std::fread(buf.data(), kFeatureBytes, (size_t)m, f) != (size_t)m) return V3DM_ERR_IO;
    for (int k = 0; k < m; ++k) {
      const unsigned char* p = buf.data() + (size_t)k * kFeatureBytes;
      const long long i = i0 + k;
      if (ids) ids[i] = (int32_t)le32(p);
      float six[6];
      std::memcpy(six, p + 4, sizeof(six));
      if (pos) {
        pos[2 * i] = six[0];
        pos[2 * i + 1] = six[1];
      }
      if (dir) {
        dir[2 * i] = six[2];
        dir[2 * i + 1] = six[3];
      }
      if (scale) scale[i] = six[4];
      if (mag) mag[i] = six[5];
      if (desc) std::memcpy(desc + i * 128, p + 28, 128 * sizeof(float));
    }
  }
  return V3DM_OK;
}

// u8 re-quantisation: u = round(512 x) (half to even), clamped to 0..255; NaN gives 0.  For
// descriptors of the form u/512 it returns u.  Four values per thread.  When inexact is not
// null, it is set to 1 if any value is not exactly u/512 with u in 0..255 (one atomic per
// warp that saw such a value).
__global__ void k_quantize_u8(const float4* __restrict__ x, long long n4, uchar4* __restrict__ out,
                              int* __restrict__ inexact) {
  bool bad = false;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const float4 v = x[i];
    auto q = [&bad](float a) -> unsigned char {
      if (!(a == a)) {
        bad = true;
        return 0;
      }
      const float t = a * 512.0f;  // exact: a power-of-two scale
      const float r = rintf(t);
      const float c = fminf(fmaxf(r, 0.0f), 255.0f);
      bad |= c != t;
      return (unsigned char)c;
    };
    out[i] = make_uchar4(q(v.x), q(v.y), q(v.z), q(v.w));
  }
  if (inexact && __any_sync(__activemask(), bad) && (threadIdx.x & 31) == (__ffs(__activemask()) - 1))
    atomicOr(inexact, 1);
}

}  // namespace

cudaError_t launch_quantize_u8(const float* d_x, long long nValues, uint8_t* d_out, cudaStream_t s,
                               int* d_inexact) {
  if (nValues <= 0) return cudaSuccess;
  if (nValues % 4 != 0) return cudaErrorInvalidValue;
  const long long n4 = nValues / 4;
  const long long blocks = std::min<long long>((n4 + 255) / 256, 148LL * 16);
  k_quantize_u8<<<(unsigned)blocks, 256, 0, s>>>(reinterpret_cast<const float4*>(d_x), n4,
                                                  reinterpret_cast<uchar4*>(d_out), d_inexact);
  return cudaGetLastError();
}

}  // namespace v3dm

using namespace v3dm;

struct v3dm_loader {
  int device = 0;
  cudaStream_t stream = nullptr;
  float* hStage = nullptr;  // pinned: descriptors of the last load, image-concatenated
  long long stageCap = 0;   // floats
  float* dStage = nullptr;
  long long dStageCap = 0;
  uint8_t* dDesc = nullptr;
  long long descCap = 0;    // bytes
  std::vector<float> positions;
  long long total = 0;      // features kept by the last load
  int* dInexact = nullptr;  // device flag: a value of the last load was not u/512
  int* hInexact = nullptr;  // pinned copy
  bool keptF32 = false;     // dStage holds the last load's floats for the caller
  bool u8Valid = false;     // dDesc holds the last load's descriptors as u8 (exact or lossy by request)
  bool exact = false;       // every value of the last load was u/512, u in 0..255
};

namespace {

struct LoaderDeviceGuard {
  int prev = -1;
  explicit LoaderDeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
  }
  ~LoaderDeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

#define V3DM_LTRY(expr)                                           \
  do {                                                            \
    cudaError_t e_ = (expr);                                      \
    if (e_ != cudaSuccess) {                                      \
      record_cuda_error(e_, __FILE__, __LINE__, #expr);           \
      return V3DM_ERR_CUDA;                                       \
    }                                                             \
  } while (0)

}  // namespace

extern "C" {

int v3dm_features_read(const char* path, int cap, int32_t* n, int32_t* ids, float* positions, float* directions,
                       float* scales, float* magnitudes, float* descriptors) {
  if (!path || !n || cap < 0) return V3DM_ERR_ARG;
  if (!host_little_endian()) return V3DM_ERR_UNSUPPORTED;
  FileReader r;
  uint32_t count = 0;
  const int st = open_features(path, r, &count);
  if (st != V3DM_OK) return st;
  if (count > 0x7fffffffu) return V3DM_ERR_SIZE;
  *n = (int32_t)count;
  const bool any = ids || positions || directions || scales || magnitudes || descriptors;
  if (!any) return V3DM_OK;
  if ((long long)count > cap) return V3DM_ERR_CAPACITY;
  return decode_features(r, count, true, ids, positions, directions, scales, magnitudes, descriptors);
}

int v3dm_quantize_u8_device(const float* d_values, long long nValues, uint8_t* d_out, void* stream) {
  if (nValues < 0 || (nValues > 0 && (!d_values || !d_out))) return V3DM_ERR_ARG;
  if (!dev_aligned(d_values, 16) || !dev_aligned(d_out, 4)) return V3DM_ERR_ARG;  // float4 in, uchar4 out
  if (nValues % 4 != 0) return V3DM_ERR_ARG;
  V3DM_LTRY(launch_quantize_u8(d_values, nValues, d_out, static_cast<cudaStream_t>(stream)));
  return V3DM_OK;
}

int v3dm_loader_create(int device, v3dm_loader** out) {
  if (!out) return V3DM_ERR_ARG;
  *out = nullptr;
  int nDev = 0;
  if (cudaGetDeviceCount(&nDev) != cudaSuccess || device < 0 || device >= nDev) return V3DM_ERR_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess || prop.major != 10) return V3DM_ERR_NO_DEVICE;
  v3dm_loader* ld = new (std::nothrow) v3dm_loader();
  if (!ld) return V3DM_ERR_ARG;
  ld->device = device;
  LoaderDeviceGuard g(device);
  if (cudaStreamCreateWithFlags(&ld->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(reinterpret_cast<void**>(&ld->dInexact), sizeof(int)) != cudaSuccess ||
      cudaMallocHost(reinterpret_cast<void**>(&ld->hInexact), sizeof(int)) != cudaSuccess) {
    if (ld->dInexact) cudaFree(ld->dInexact);
    if (ld->stream) cudaStreamDestroy(ld->stream);
    delete ld;
    return V3DM_ERR_CUDA;
  }
  *out = ld;
  return V3DM_OK;
}

int v3dm_loader_destroy(v3dm_loader* ld) {
  if (!ld) return V3DM_OK;
  LoaderDeviceGuard g(ld->device);
  if (ld->stream) cudaStreamSynchronize(ld->stream);
  if (ld->hStage) cudaFreeHost(ld->hStage);
  if (ld->dStage) cudaFree(ld->dStage);
  if (ld->dDesc) cudaFree(ld->dDesc);
  if (ld->dInexact) cudaFree(ld->dInexact);
  if (ld->hInexact) cudaFreeHost(ld->hInexact);
  if (ld->stream) cudaStreamDestroy(ld->stream);
  delete ld;
  return V3DM_OK;
}

int v3dm_loader_load(v3dm_loader* ld, int nFiles, const char* const* paths, int maxPerImage, int flags,
                     int32_t* counts) {
  if (!ld || nFiles < 0 || (nFiles > 0 && (!paths || !counts))) return V3DM_ERR_ARG;
  if ((flags & ~(V3DM_LOAD_ROUND32 | V3DM_LOAD_KEEP_F32 | V3DM_LOAD_LOSSY_U8)) != 0) return V3DM_ERR_ARG;
  if (!host_little_endian()) return V3DM_ERR_UNSUPPORTED;
  LoaderDeviceGuard g(ld->device);
  // headers: how many features each file holds and how many are kept
  std::vector<long long> kept(nFiles), off(nFiles + 1, 0);
  for (int i = 0; i < nFiles; ++i) {
    if (!paths[i]) return V3DM_ERR_ARG;
    FileReader r;
    uint32_t c = 0;
    const int st = open_features(paths[i], r, &c);
    if (st != V3DM_OK) return st;
    long long k = c;
    if (flags & V3DM_LOAD_ROUND32) k &= ~31LL;  // the apps' "& 0xffe0" (match_sequence.cpp:183)
    if (maxPerImage > 0) k = std::min<long long>(k, maxPerImage);
    if (k > 0x7fffffffLL) return V3DM_ERR_SIZE;
    kept[i] = k;
    off[i + 1] = off[i] + k;
  }
  const long long total = off[nFiles];
  const long long nValues = total * 128;
  // buffers (kept between loads, grown when needed)
  V3DM_LTRY(cudaStreamSynchronize(ld->stream));  // the previous load's copies have finished
  if (nValues > ld->stageCap) {
    if (ld->hStage) cudaFreeHost(ld->hStage);
    ld->hStage = nullptr;
    ld->stageCap = 0;
    V3DM_LTRY(cudaMallocHost(reinterpret_cast<void**>(&ld->hStage), (size_t)nValues * sizeof(float)));
    ld->stageCap = nValues;
  }
  if (nValues > ld->dStageCap) {
    if (ld->dStage) cudaFree(ld->dStage);
    ld->dStage = nullptr;
    ld->dStageCap = 0;
    V3DM_LTRY(cudaMalloc(reinterpret_cast<void**>(&ld->dStage), (size_t)nValues * sizeof(float)));
    ld->dStageCap = nValues;
  }
  if (nValues > ld->descCap) {
    if (ld->dDesc) cudaFree(ld->dDesc);
    ld->dDesc = nullptr;
    ld->descCap = 0;
    V3DM_LTRY(cudaMalloc(reinterpret_cast<void**>(&ld->dDesc), (size_t)nValues));
    ld->descCap = nValues;
  }
  ld->positions.assign((size_t)total * 2, 0.0f);
  ld->total = 0;
  ld->keptF32 = ld->u8Valid = ld->exact = false;
  // decode: files are handed out to the host threads one at a time
  std::atomic<int> next(0), err(V3DM_OK);
  auto work = [&]() {
    for (int i = next++; i < nFiles; i = next++) {
      FileReader r;
      uint32_t c = 0;
      int st = open_features(paths[i], r, &c);
      if (st == V3DM_OK && (long long)c < kept[i]) st = V3DM_ERR_IO;  // the file changed since its header was read
      if (st == V3DM_OK)
        st = decode_features(r, kept[i], kept[i] == (long long)c, nullptr, ld->positions.data() + 2 * off[i],
                             nullptr, nullptr, nullptr, ld->hStage + off[i] * 128);
      if (st != V3DM_OK) {
        int expect = V3DM_OK;
        err.compare_exchange_strong(expect, st);
      }
    }
  };
  const int nThreads = std::max(1, std::min<int>(nFiles, (int)std::max(1u, std::thread::hardware_concurrency())));
  std::vector<std::thread> pool;
  for (int t = 1; t < nThreads; ++t) pool.emplace_back(work);
  work();
  for (auto& t : pool) t.join();
  if (err.load() != V3DM_OK) return err.load();
  // one copy to the device, u8 conversion there with a flag for values that are not u/512
  *ld->hInexact = 0;
  V3DM_LTRY(cudaMemsetAsync(ld->dInexact, 0, sizeof(int), ld->stream));
  if (nValues > 0) {
    V3DM_LTRY(cudaMemcpyAsync(ld->dStage, ld->hStage, (size_t)nValues * sizeof(float), cudaMemcpyHostToDevice,
                              ld->stream));
    V3DM_LTRY(launch_quantize_u8(ld->dStage, nValues, ld->dDesc, ld->stream, ld->dInexact));
    V3DM_LTRY(cudaMemcpyAsync(ld->hInexact, ld->dInexact, sizeof(int), cudaMemcpyDeviceToHost, ld->stream));
  }
  V3DM_LTRY(cudaStreamSynchronize(ld->stream));
  for (int i = 0; i < nFiles; ++i) counts[i] = (int32_t)kept[i];
  ld->total = total;
  ld->exact = *ld->hInexact == 0;
  ld->keptF32 = (flags & V3DM_LOAD_KEEP_F32) != 0;
  ld->u8Valid = ld->exact || (flags & V3DM_LOAD_LOSSY_U8) != 0;
  // floats that are not u/512 with neither floats kept nor rounding asked for: refuse
  if (!ld->u8Valid && !ld->keptF32) return V3DM_ERR_NOT_U8;
  return V3DM_OK;
}

int v3dm_loader_positions(v3dm_loader* ld, float* positions) {
  if (!ld || (ld->total > 0 && !positions)) return V3DM_ERR_ARG;
  if (ld->total > 0) std::memcpy(positions, ld->positions.data(), (size_t)ld->total * 2 * sizeof(float));
  return V3DM_OK;
}

int v3dm_loader_descriptors_device(v3dm_loader* ld, const uint8_t** d_desc, long long* total) {
  if (!ld || !d_desc || !total) return V3DM_ERR_ARG;
  *d_desc = nullptr;
  *total = ld->total;
  if (ld->total > 0 && !ld->u8Valid) return V3DM_ERR_NOT_U8;
  *d_desc = ld->dDesc;
  return V3DM_OK;
}

int v3dm_loader_descriptors_f32_device(v3dm_loader* ld, const float** d_desc, long long* total) {
  if (!ld || !d_desc || !total) return V3DM_ERR_ARG;
  *d_desc = nullptr;
  *total = ld->total;
  if (!ld->keptF32) return V3DM_ERR_NOT_ALLOCATED;
  *d_desc = ld->dStage;
  return V3DM_OK;
}

int v3dm_loader_exact_u8(v3dm_loader* ld, int* exact) {
  if (!ld || !exact) return V3DM_ERR_ARG;
  *exact = ld->exact ? 1 : 0;
  return V3DM_OK;
}

}  // extern "C"
