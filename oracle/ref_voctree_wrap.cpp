/*
 * ref_voctree_wrap.cpp -- extern "C" entry point around the reference's own CPU quantizer
 * V3D::VocabularyTree<Depth, BranchFactor, 128>::getVisualWord (V3D/Base/v3d_voctree.h:19-103),
 * compiled from the reference headers by oracle/Makefile into oracle/_ref/libv3dref_voctree.so.
 *
 * TEST INFRASTRUCTURE ONLY: it pins the oracle's voctree descent and gives golden leaf ids.
 * The tree shape is a template argument in the reference, so a fixed set of shapes is
 * instantiated here.  Returns the leaf-local id (v3d_voctree.h:78).
 */
#include <algorithm>
#include "Base/v3d_voctree.h"

namespace {
template <int D, int BF>
struct Loaded : public V3D::VocabularyTree<D, BF, 128> {
    void set(const float* nodes) { std::copy(nodes, nodes + this->_tree.size(), this->_tree.begin()); }
};

template <int D, int BF>
int run(const float* nodes, int n, const float* keys, int* out) {
    Loaded<D, BF>* t = new Loaded<D, BF>();
    t->set(nodes);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n; ++j) out[j] = t->getVisualWord(keys + (size_t)j * 128);
    delete t;
    return 0;
}
}  // namespace

extern "C" int v3dref_voctree_quantize(int bf, int depth, const float* nodes, int n, const float* keys, int* out) {
#define V3DREF_SHAPE(B, D) \
    if (bf == B && depth == D) return run<D, B>(nodes, n, keys, out);
    V3DREF_SHAPE(2, 1)
    V3DREF_SHAPE(3, 2)
    V3DREF_SHAPE(4, 3)
    V3DREF_SHAPE(5, 4)
    V3DREF_SHAPE(10, 2)
    V3DREF_SHAPE(10, 3)
    V3DREF_SHAPE(10, 4)
    V3DREF_SHAPE(10, 5)
    V3DREF_SHAPE(10, 6)
    V3DREF_SHAPE(50, 3)
    V3DREF_SHAPE(300, 2)
#undef V3DREF_SHAPE
    return -1;
}
