// v3dm_internal.h -- host-side structures shared by the library's translation units.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "v3dm.h"
#include "v3dm_common.cuh"

namespace v3dm {

// Launches kernel k with programmatic stream serialization (see pdl_wait in v3dm_device.cuh).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
}

// Device error flags (bitwise OR into MatchArgs::err).
constexpr int kErrWaitTimeout = 1;  // a bounded mbarrier wait in the tcgen05 kernel gave up
constexpr int kErrNotU8 = 2;        // a float descriptor was not u/512-valued
constexpr int kErrTmem = 4;         // TMEM allocation returned an unexpected address
constexpr int kErrBadTree = 8;      // a vocabulary-tree descent would have left the node array

// Layout of the small info block every matching call writes (int32 words).
constexpr int kInfoPairs = 0;     // number of mutual pairs
constexpr int kInfoErr = 1;       // device error flags
constexpr int kInfoMaxSeg = 2;    // largest candidate count of one list segment
constexpr int kInfoWords = 4;

struct MatchArgs {
  int nL, nR;
  int32_t T;                       // candidate threshold
  unsigned long long* lBest;       // per left: best key over rights
  unsigned int* lSec;              // per left: second value + 1
  unsigned long long* rBest;       // per right: best key over lefts
  unsigned int* rSec;              // per right: second value + 1
  unsigned long long* cand;        // candidate list, nSeg segments of segCap entries
  int* segCount;                   // per segment: number of candidates found
  long long segCap;
  int nSeg;
  int* err;
  int nGates;
  GateParams gates[V3DM_MAX_GATES];
  const GateParams* gatesDev;      // device copy of gates[] (kernels index it at run time)
};

// Kernel launchers (v3dm_match.cu, v3dm_match_tc.cu).
cudaError_t launch_match_simt(const uint8_t* dL, const uint8_t* dR, const MatchArgs& a, cudaStream_t s);
cudaError_t launch_seconds(const MatchArgs& a, cudaStream_t s);
cudaError_t launch_finalize(const MatchArgs& a, float minScore, float minRatio, int32_t* dScratch, int32_t* dPairs,
                            int32_t* dInfo, cudaStream_t s);
cudaError_t launch_gate_precompute(int type, const double* m, const float* dLPos, int nL, const float* dRPos,
                                   int nR, float4* lv, float4* rv, cudaStream_t s);
cudaError_t launch_f32_to_u8(const float* src, uint8_t* dst, int n, int* err, cudaStream_t s);

// ---- tcgen05 path (v3dm_match_tc.cu, v3dm_pair.cu) ------------------------------------
// One row of a batched side pass: one A group (up to rowsPerGroup descriptors of one image,
// or of one list of chosen descriptors) against every tile of one B image.
struct BatchRow {
  int aRow;          // first row of the group in the A tensor
  int validRows;     // descriptors in the group; rows past it are padding
  int bRow0;         // first row of the B image in the B tensor
  int nB;            // descriptors of the B image
  int nTiles;        // ceil(nB / colsPerTile)
  int pad;
  long long state0;  // state index of the group's first descriptor
};

// Gates of a batched guided call (v3dm_batch.cu): one gate per pair, evaluated on the fly from
// the positions.  gm: per pair (caller's order) the 3x3 matrix as floats, then thr^2.
constexpr int kBGateFloats = 10;
struct BatchGateArgs {
  int on;                        // 0: no batched gates
  int type;                      // 1 epipolar (F), 2 homography (H)
  const float* gm;
  const int2* pairLR;            // per pair (caller's order): left image, right image
  const float2* pos;             // positions of all images' descriptors, concatenated
  const long long* posOff;       // per image: its first descriptor in pos
  const long long* stateA0;      // per pair in batch order: its first pass-A state
  const int* origOf;             // per pair in batch order: its index in the caller's order
  int nPairs;
  const int* chosenPair;         // per pass-B state: its pair (caller's order) and right
  const int* chosenRight;
};

// One side pass scores the nA descriptors of side A against the nB descriptors of side B
// (single pair), or walks a table of BatchRows (batched pass).
struct SideArgs {
  const int* nAptr;              // device count of A rows (null: use nA)
  int nA;                        // A rows (upper bound when nAptr is set)
  int nB;                        // B rows
  int32_t Smin;                  // smallest score that can pass the min-score test
  int32_t Tsec;                  // second scores below this decide like none (0: keep every bound)
  const int* amap;               // single pair: A row -> index on its side (null: identity);
                                 // batched pass: absolute A row -> index within its image
                                 // (null: the row's place in its group)
  int aIsLeft;                   // 1: A = lefts, B = rights; 0: A = rights, B = lefts
  unsigned long long* best;      // per A index: best key over B (atomicMax)
  unsigned int* sec;             // per A index: second score + 1 (exact, or a bound with gates)
  uint4* records;                // per-warp segments of chunk records (kRecordQuads uint4 each)
  int* segCount;                 // per segment: records written
  long long segCap;              // records per segment
  int nSeg;
  int* err;
  int nGates;
  const GateParams* gatesDev;    // device array of the call's gates
  // batched pass only
  const BatchRow* rows;          // row table
  const int* nRowsPtr;           // device row count (null: use nRows)
  int nRows;
  int schedule;                  // 0: rows interleaved over the CTAs, 1: contiguous row ranges,
                                 // 2: chunks of consecutive rows interleaved over the CTAs
  // gathered A (launch_side_gather): A row e of the row table is descriptor aSrcRow[e] of aSrc
  const uint8_t* aSrc;
  const int* aSrcRow;
  // batched float pass (launch_side_f_batch): decisions written per state, the float rules
  int32_t* decision;
  float minScore, minRatio;
  BatchGateArgs bg;              // batched float pass of a guided call: each pair's gate (on = 0: none)
  // failure-path test hooks (zero in production): the bounded waits give up after waitLimit
  // cycles (0: the default), and CTA 0's producer does not issue its skipLoad-th B tile load
  // (0: none), so that the consumer's bounded wait for it runs out
  long long waitLimit;
  int skipLoad;
};
// Chunk record: {A index (state), first B column, B count, first B row of the tile's image
// block} then the chunk's 32 scores.
constexpr int kRecordQuads = 9;

struct TcPlan;
struct TcMaps {
  CUtensorMap a, b;
  int cfg;
};
cudaError_t tc_plan_create(TcPlan** p, int device);
void tc_plan_destroy(TcPlan* p);
int tc_num_configs();
int tc_get_config(TcPlan* p);
cudaError_t tc_set_config(TcPlan* p, int cfg);
void tc_config_shape(int cfg, int* rowsPerGroup, int* colsPerTile);
// Number of list segments a side pass uses (one per epilogue warp of a full grid).
int tc_segments(TcPlan* p);
// Tensor maps of a side pass for the plan's current configuration.
cudaError_t tc_side_maps(TcPlan* p, TcMaps* m, const uint8_t* dA, int rowsA, const uint8_t* dB, int rowsB);
cudaError_t launch_side(TcPlan* p, const TcMaps& m, const SideArgs& a, cudaStream_t st);
// Batched side pass over a.rows (a.nRows, or *a.nRowsPtr rows): one persistent launch.
cudaError_t launch_side_batch(TcPlan* p, const TcMaps& m, const SideArgs& a, cudaStream_t st);
// Sets the batched kernel's launch attributes for configuration cfg (before a stream capture).
cudaError_t tc_prepare_batch(TcPlan* p, int cfg);
// Batched pass whose A blocks are gathered row by row (SideArgs::aSrc / aSrcRow) instead of
// loaded as tiles; B through the tensor map of tc_gather_map.  Its left groups have
// tc_gather_rows() rows.
int tc_gather_rows();
int tc_gather_cols();
cudaError_t tc_gather_map(CUtensorMap* m, const uint8_t* dB, int rowsB);
cudaError_t launch_side_gather(TcPlan* p, const CUtensorMap& mB, const SideArgs& a, cudaStream_t st);

// Tensor-core voctree phase (v3dm_voctree_tc.cu): every work item (bucket b, first position,
// count) descends `levels` (1 or 2) levels below its bucket node (bucketBase + b; the root when
// bucketBase < 0) for the keys perm[first .. first + count) (positions themselves when perm is
// null).  final: out[key] = the node reached (minus leafBase with V3DM_LEAF_LOCAL); else
// next[key] = node - nextBase and hist[node - nextBase] counts it (bins buckets).
struct VtcArgs {
  const uint8_t* nodes;
  int bf, levels;
  long long bucketBase;
  const int4* items;
  const int* nItems;
  int singleN;                   // > 0: one bucket of singleN keys (items and nItems unused)
  const int32_t* perm;
  const uint8_t* keys;
  int final;
  int32_t* out;
  int idMode;
  long long leafBase;
  int32_t* next;
  long long nextBase;
  int* hist;
  int bins;
  int* err;
};
bool vtc_supported(int bf);
// Rows of the tree read by the phases: a tensor map over the node rows with boxes of kVtcBoxRows;
// the keys of a phase with singleN > 0: a map over the key rows with boxes of kVtcKeyBox rows.
constexpr int kVtcBoxRows = 16;
constexpr int kVtcKeyBox = 128;
cudaError_t launch_vtc(const VtcArgs& a, const CUtensorMap& nodeMap, const CUtensorMap& keyMap, int grid,
                       cudaStream_t st);
// 2-D map over rows x 128 bytes with a box of boxRows rows and the 128-byte swizzle (v3dm_match_tc.cu).
cudaError_t tc_rows_map(CUtensorMap* m, const uint8_t* base, int rows, int boxRows);


// Decision and bookkeeping kernels around the side passes (v3dm_pair.cu).
struct PostArgs {
  int nRows;                     // rows of the pass (A side); with rowsPtr the device count
  const int* rowsPtr;
  const int* amap;               // row -> index (null: identity)
  unsigned long long* best;
  unsigned int* sec;
  const uint4* records;          // chunk records of the side pass
  const int* bmap;               // absolute B row -> index within its image (null: the column)
  int* segCount;                 // read, then cleared (kept when keepSegments is set)
  long long segCap;
  int nSeg;
  int keepSegments;              // the records stay valid for a later call (pass-A cache)
  const unsigned int* secBound;  // optional second bound per index, read-only (pass-A cache)
  int nB;
  int aIsLeft;
  int32_t Smin;
  int nGates;
  const GateParams* gatesDev;
  BatchGateArgs bg;              // batched guided call: per-pair gates instead of gatesDev
  float minScore, minRatio;
  int gated;
  int32_t* decision;             // per index: accepted partner or -1
  int* flagged;                  // indices whose decision needs an exact re-score
  int* flaggedCount;
  int* err;
  // Optional (pass A of one pair): every accepted partner is also 'chosen' right here -- flagged,
  // listed once, and its descriptor row gathered for pass B (planar BF16 rows when choosePlanes
  // is 6, else 128-byte rows).
  int* chooseFlag;
  int* chooseList;
  int* chooseCount;
  const uint8_t* chooseSrc;
  uint8_t* chooseDst;
  int chooseCapSrc, chooseCapDst;
  int choosePlanes;
};
cudaError_t launch_post(const PostArgs& a, cudaStream_t s);
// u8 re-quantisation of nValues floats (a multiple of 4), v3dm_features.cu.
cudaError_t launch_quantize_u8(const float* d_x, long long nValues, uint8_t* d_out, cudaStream_t s,
                               int* d_inexact = nullptr);

// ---- float descriptors: BF16 hi/lo scores (v3dm_match_f.cu) ------------------------------
// Operand layouts: 6 planes of rowsCap x 128 bytes (64 BF16 values of a K slice per row).
constexpr int kFloatRowBytes = 768;
int f_segments(int numSMs);
cudaError_t f_maps(CUtensorMap* mA, const void* dA, int rowsA, CUtensorMap* mB, const void* dB, int rowsB);
cudaError_t launch_side_f(const CUtensorMap& mA, const CUtensorMap& mB, const SideArgs& a, float Tf, float* dump,
                          int numSMs, cudaStream_t st);
// Batched float side pass over a.rows (a.nRows, or *a.nRowsPtr rows), rows interleaved over the
// persistent CTAs; A groups of f_group_rows() rows, B tiles of f_tile_cols() columns.  Writes
// the decision of every state of the rows to a.decision (the float rules with a.minScore,
// a.minRatio and the candidate threshold Tf); no chunk records.  With a.rows null: one pair,
// a.nA A rows against a.nB B rows, decisions indexed by A row.
cudaError_t launch_side_f_batch(const CUtensorMap& mA, const CUtensorMap& mB, const SideArgs& a, float Tf,
                                int numSMs, cudaStream_t st);
int f_group_rows();
int f_tile_cols();
cudaError_t launch_post_f(const PostArgs& a, float Tf, cudaStream_t s);
cudaError_t launch_hilo(const float* f, const uint8_t* u, int n, int rowsCap, void* la, void* lb, int* err,
                        cudaStream_t s);
// The same layouts for the n concatenated descriptors of nImages images: image i (first
// descriptor srcOff[i], ascending) goes to rows rowOff[i] onwards of the rowsCap-row planes.
cudaError_t launch_hilo_images(const float* f, long long n, const long long* srcOff, const int* rowOff, int nImages,
                               int rowsCap, void* la, void* lb, int* err, cudaStream_t s);
float host_float_threshold(float minScore, float minRatio);
// Exact re-score of the flagged descriptors of side A against side B.
struct RescoreArgs {
  const uint8_t* descA;          // side A descriptors by index
  const uint8_t* descB;
  int nB;
  int aIsLeft;
  int nGates;
  const GateParams* gatesDev;
  float minScore, minRatio;
  int32_t T;                     // candidate threshold: scores below it cannot change a decision
  const int* flagged;
  const int* flaggedCount;
  unsigned long long* best;
  unsigned int* sec;
  int32_t* decision;
};
cudaError_t launch_rescore(const RescoreArgs& a, int grid, cudaStream_t s);
// Rights accepted by some left: de-duplicated list, their descriptors gathered into dRc.
cudaError_t launch_choose(const int32_t* leftDec, int nL, int* chosenFlag, int* chosenList, int* chosenCount,
                          const uint8_t* dR, uint8_t* dRc, cudaStream_t s);
// The same for rows of 'planes' 128-byte blocks (block p of row r at (p * cap + r) * 128).
cudaError_t launch_choose_planes(const int32_t* leftDec, int nL, int* chosenFlag, int* chosenList, int* chosenCount,
                                 const uint8_t* src, uint8_t* dst, int planes, int capSrc, int capDst,
                                 cudaStream_t s);
// Mutual filter and ordered compaction (blockCount: nL/2048 + 1 ints of scratch); clears chosenFlag.
// The pair count goes to info[kInfoPairs] and, when countOut is set, to *countOut.
cudaError_t launch_mutual(const int32_t* leftDec, int nL, const int32_t* rightDec, int* chosenFlag, int* blockCount,
                          int2* pairs, int32_t* info, int32_t* countOut, cudaStream_t s);

// Candidate threshold (v3dm_api.cu).
int host_candidate_threshold(float minScore, float minRatio, bool gated, int32_t* T);
// Learned projection (v3dm_proposal.cu): the 'probes' best cells of n descriptors (n x probes
// bytes) on stream s, the number of cells, and the projection's stream.
cudaError_t proj_assign(const v3dm_projection* p, const uint8_t* dDesc, long long n, int probes, uint8_t* dCells,
                        cudaStream_t s);
int proj_cells(const v3dm_projection* p);
cudaStream_t proj_stream(const v3dm_projection* p);

// Whether a caller's device buffer meets the alignment its kernels access it with (a power of two).
inline bool dev_aligned(const void* p, uintptr_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }

// Records the detail v3dm_last_error() reports for this thread (v3dm_api.cu).
void record_cuda_error(cudaError_t e, const char* file, int line, const char* what);
// Smallest integer score S whose float score S * 2^-18 passes 's > minScore' (v3dm_api.cu).
int32_t host_smallest_passing_score(float minScore);

}  // namespace v3dm
