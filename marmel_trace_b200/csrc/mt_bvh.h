// mt_bvh.h - host BVH builder and device-layout flattening.
#pragma once

#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/mtgpu.h"

namespace mt {

// Binary node in the reference's layout and order (BvhNode, src/bvh.c:50-57).
struct HostNode {
    double mn[3], mx[3];
    int left, right, first, count;
};

struct HostBvh {
    std::vector<HostNode> nodes;   // preorder, node 0 = root
    std::vector<int> order;        // leaf-ordered prim indices (tree prims)
    std::vector<int> planes;       // plane prim indices, file order
    int depth = 0;                 // leaf depth, root = 1
};

// primitive_bounds (src/geometry.c:1503-1584) for the kinds on the GPU path.
void prim_bounds(const mt_prim &p, double mn[3], double mx[3]);

// bvh_build (src/bvh.c:364-422): binned SAH over 12 bins, leaf <= 4 prims,
// median fallback, planes in a side list. Deterministic and identical to the
// reference builder for the same primitive array.
int build_bvh(const mt_prim *prims, int n, HostBvh *out);

// The same build on the current CUDA device (mt_bvh_gpu.cu): the tree of
// build_bvh with the primitives of each node in another order (see there).
// Returns 0 or an MT_ERR_* code (message in *err); *ms: device build time.
int build_bvh_device(const mt_prim *prims, int n, HostBvh *out, std::string *err, float *ms);

// The tree `b` restricted to the primitives with keep[prim] != 0: each leaf
// keeps only those primitives, subtrees left empty are dropped, an inner node
// left with one child is replaced by that child, and every box is refit to
// the primitives left (prim_bounds, padded outward by a few parts per
// million so that no FP32 slab test can cull a kept primitive's hit). Planes
// are not carried over. `out->nodes` is empty when nothing is kept. Linear
// in the size of `b` (no new SAH build).
int prune_bvh(const HostBvh &b, const mt_prim *prims, const std::vector<char> &keep, HostBvh *out);

// Device-ready flattened tree (see mt_layout.h for the node record).
struct FlatBvh {
    std::vector<float> nodes;      // 16 floats per node (q0..q3; q3 holds ints)
    std::vector<int> ref_prim;     // leaf-ordered prim index
    int node_count = 0;
    int depth = 0;                 // depth of the flattened inner-node tree
};

// Flatten `b` into two-child nodes with FP32 boxes rounded outward. Leaves
// of more than 7 prims (the reference's coincident-centroid leaves) are split
// into small subtrees with the same box; nearest-hit results do not depend on
// the tree shape.
int flatten_bvh(const HostBvh &b, FlatBvh *out);

// Wide tree for the traversal kernels: every node holds up to W (4 or 8)
// children, made by collapsing the device binary tree `nodes2` (16 floats per
// node, its final child codes in the last 4) from the root down: a node's
// child slots start as the two binary children and the inner slot with the
// largest box surface area is replaced by its two children until W slots are
// filled or only leaves are left. Leaf codes are kept, so both trees share
// the leaves. Record (float words): lo_x, hi_x, lo_y, hi_y, lo_z, hi_z (W
// each), the W child codes, padding to 32 (W = 4) or 64 (W = 8) words. An
// unused slot has child code INT_MIN. *stack_bound is the most entries a
// walk can hold: the sum over a root-to-leaf path of (children - 1).
int collapse_bvh(const std::vector<float> &nodes2, int node_count, int W, std::vector<float> *out,
                 int *stack_bound);

}  // namespace mt
