// mt_bvh.cpp - host binned-SAH BVH builder (restating the reference builder)
// and flattening into the GPU node layout.
//
// The builder follows src/bvh.c:140-422 step for step (same bin count, cost,
// partition loops and preorder node numbering) so the tree equals the
// reference's node for node; the test suite checks that against the reference
// builder. Primitive bounds and centroids are computed once up front instead
// of on every visit, which changes the cost, not the values.
#include "mt_bvh.h"

#include <math.h>
#include <string.h>

#include <algorithm>

namespace mt {

namespace {

const int kLeafSize = 4;            // BVH_LEAF_SIZE, src/bvh.c:41
const int kBins = 12;               // BVH_NBINS, src/bvh.c:43
const double kBoundsEps = 1e-7;     // BVH_BOUNDS_EPS, src/bvh.c:45

inline double vmin(double a, double b) { return a < b ? a : b; }   // vec3_min, src/vec3.h:122-127
inline double vmax(double a, double b) { return a > b ? a : b; }   // vec3_max, src/vec3.h:129-134

double surface_area(const double *mn, const double *mx)
{
    double dx = mx[0] - mn[0];
    double dy = mx[1] - mn[1];
    double dz = mx[2] - mn[2];
    if (dx < 0.0) dx = 0.0;
    if (dy < 0.0) dy = 0.0;
    if (dz < 0.0) dz = 0.0;
    return 2.0 * (dx * dy + dy * dz + dz * dx);
}

struct Builder {
    const double *pmin;   // 3 per prim
    const double *pmax;
    const double *cen;    // centroid (pmin + pmax) * 0.5
    HostBvh *b;

    void range_info(int first, int count, double *mn, double *mx, double *cmn, double *cmx) const
    {
        for (int k = 0; k < 3; ++k) {
            mn[k] = 1e300;
            mx[k] = -1e300;
            cmn[k] = 1e300;
            cmx[k] = -1e300;
        }
        for (int i = 0; i < count; ++i) {
            int p = b->order[first + i];
            for (int k = 0; k < 3; ++k) {
                mn[k] = vmin(mn[k], pmin[3 * p + k]);
                mx[k] = vmax(mx[k], pmax[3 * p + k]);
                cmn[k] = vmin(cmn[k], cen[3 * p + k]);
                cmx[k] = vmax(cmx[k], cen[3 * p + k]);
            }
        }
        for (int k = 0; k < 3; ++k) {
            mn[k] = mn[k] - kBoundsEps;
            mx[k] = mx[k] + kBoundsEps;
        }
    }

    int make_leaf(const double *mn, const double *mx, int first, int count)
    {
        HostNode n;
        memcpy(n.mn, mn, sizeof n.mn);
        memcpy(n.mx, mx, sizeof n.mx);
        n.left = -1;
        n.right = -1;
        n.first = first;
        n.count = count;
        b->nodes.push_back(n);
        return (int)b->nodes.size() - 1;
    }

    int bin_of(int p, int axis, double cmin, double scale) const
    {
        double cv = cen[3 * p + axis];
        int bin = (int)((cv - cmin) * scale);
        if (bin < 0) bin = 0;
        if (bin >= kBins) bin = kBins - 1;
        return bin;
    }

    // bvh_build_node (src/bvh.c:180-362)
    int build(int first, int count, int depth)
    {
        if (depth > b->depth) b->depth = depth;
        double mn[3], mx[3], cmn[3], cmx[3];
        range_info(first, count, mn, mx, cmn, cmx);
        if (count <= kLeafSize) return make_leaf(mn, mx, first, count);

        double ex = cmx[0] - cmn[0], ey = cmx[1] - cmn[1], ez = cmx[2] - cmn[2];
        int axis = 0;
        double max_ext = ex;
        if (ey > max_ext) {
            max_ext = ey;
            axis = 1;
        }
        if (ez > max_ext) {
            max_ext = ez;
            axis = 2;
        }
        if (!(max_ext > 0.0)) return make_leaf(mn, mx, first, count);

        double cmin = cmn[axis];
        double cmax = cmx[axis];
        double scale = kBins / max_ext;

        double bmin[kBins][3], bmax[kBins][3];
        int bcount[kBins];
        for (int i = 0; i < kBins; ++i) {
            for (int k = 0; k < 3; ++k) {
                bmin[i][k] = 1e300;
                bmax[i][k] = -1e300;
            }
            bcount[i] = 0;
        }
        for (int i = 0; i < count; ++i) {
            int p = b->order[first + i];
            int bin = bin_of(p, axis, cmin, scale);
            bcount[bin]++;
            for (int k = 0; k < 3; ++k) {
                bmin[bin][k] = vmin(bmin[bin][k], pmin[3 * p + k]);
                bmax[bin][k] = vmax(bmax[bin][k], pmax[3 * p + k]);
            }
        }

        double rmin[kBins][3], rmax[kBins][3];
        int rcount[kBins];
        double acc_min[3] = {1e300, 1e300, 1e300}, acc_max[3] = {-1e300, -1e300, -1e300};
        int acc_n = 0;
        for (int i = kBins - 1; i >= 0; --i) {
            if (bcount[i] > 0) {
                for (int k = 0; k < 3; ++k) {
                    acc_min[k] = vmin(acc_min[k], bmin[i][k]);
                    acc_max[k] = vmax(acc_max[k], bmax[i][k]);
                }
                acc_n += bcount[i];
            }
            memcpy(rmin[i], acc_min, sizeof acc_min);
            memcpy(rmax[i], acc_max, sizeof acc_max);
            rcount[i] = acc_n;
        }

        double lmin[3] = {1e300, 1e300, 1e300}, lmax[3] = {-1e300, -1e300, -1e300};
        int lacc_n = 0;
        double best_cost = 1e300;
        int best_split = -1;
        for (int i = 0; i < kBins - 1; ++i) {
            if (bcount[i] > 0) {
                for (int k = 0; k < 3; ++k) {
                    lmin[k] = vmin(lmin[k], bmin[i][k]);
                    lmax[k] = vmax(lmax[k], bmax[i][k]);
                }
                lacc_n += bcount[i];
            }
            int rn = rcount[i + 1];
            if (lacc_n == 0 || rn == 0) continue;
            double la = surface_area(lmin, lmax);
            double ra = surface_area(rmin[i + 1], rmax[i + 1]);
            double cost = la * (double)lacc_n + ra * (double)rn;
            if (cost < best_cost) {
                best_cost = cost;
                best_split = i;
            }
        }

        double leaf_cost = surface_area(mn, mx) * (double)count;
        int use_split = -1;
        int median_mid = -1;
        if (best_split >= 0 && best_cost < leaf_cost) use_split = best_split;

        int *order = b->order.data();
        if (use_split < 0) {
            double mid = 0.5 * (cmin + cmax);
            int i = first, j = first + count - 1;
            while (i <= j) {
                double cv = cen[3 * order[i] + axis];
                if (cv < mid) {
                    ++i;
                } else {
                    std::swap(order[i], order[j]);
                    --j;
                }
            }
            median_mid = i;
            if (median_mid <= first || median_mid >= first + count) median_mid = first + count / 2;
        }

        int mid_index;
        if (use_split >= 0) {
            int i = first, j = first + count - 1;
            while (i <= j) {
                if (bin_of(order[i], axis, cmin, scale) <= best_split) {
                    ++i;
                } else {
                    std::swap(order[i], order[j]);
                    --j;
                }
            }
            mid_index = i;
            if (mid_index == first || mid_index == first + count) mid_index = first + count / 2;
        } else {
            mid_index = median_mid;
            if (mid_index == first || mid_index == first + count) mid_index = first + count / 2;
        }

        int left_count = mid_index - first;
        int right_count = count - left_count;
        if (left_count <= 0 || right_count <= 0) return make_leaf(mn, mx, first, count);

        HostNode inner;
        memcpy(inner.mn, mn, sizeof mn);
        memcpy(inner.mx, mx, sizeof mx);
        inner.left = inner.right = -1;
        inner.first = 0;
        inner.count = 0;
        b->nodes.push_back(inner);
        int this_idx = (int)b->nodes.size() - 1;
        int l = build(first, left_count, depth + 1);
        int r = build(mid_index, right_count, depth + 1);
        b->nodes[this_idx].left = l;
        b->nodes[this_idx].right = r;
        return this_idx;
    }
};

// Round a double box outward to float.
float round_down(double v)
{
    float f = (float)v;
    if ((double)f > v) f = nextafterf(f, -INFINITY);
    return f;
}
float round_up(double v)
{
    float f = (float)v;
    if ((double)f < v) f = nextafterf(f, INFINITY);
    return f;
}

struct Flattener {
    const HostBvh &b;
    FlatBvh *out;
    int max_depth = 0;

    int alloc_node()
    {
        out->nodes.resize(out->nodes.size() + 16, 0.0f);
        return out->node_count++;
    }

    void set_child(int node, int side, const double *mn, const double *mx, int code, int count)
    {
        float *q = &out->nodes[16 * (size_t)node];
        float lo[3] = {round_down(mn[0]), round_down(mn[1]), round_down(mn[2])};
        float hi[3] = {round_up(mx[0]), round_up(mx[1]), round_up(mx[2])};
        if (side == 0) {
            q[0] = lo[0]; q[1] = hi[0]; q[2] = lo[1]; q[3] = hi[1];
            q[8] = lo[2]; q[9] = hi[2];
        } else {
            q[4] = lo[0]; q[5] = hi[0]; q[6] = lo[1]; q[7] = hi[1];
            q[10] = lo[2]; q[11] = hi[2];
        }
        int ci[2] = {code, count};
        memcpy(&q[12 + side], &ci[0], 4);
        memcpy(&q[14 + side], &ci[1], 4);
    }

    // Child code for a leaf range; ranges of more than 7 prims become a
    // balanced subtree of nodes that all carry the leaf's box.
    int leaf_code(const double *mn, const double *mx, int first, int count, int depth)
    {
        if (count <= 7) {
            if (depth > max_depth) max_depth = depth;
            // ~((first << 4) | (tri_only << 3) | count); the triangle-only
            // flag is set at upload time, when primitive kinds are known.
            return ~((first << 4) | count);
        }
        int node = alloc_node();
        if (depth + 1 > max_depth) max_depth = depth + 1;
        int half = count / 2;
        int cl = leaf_code(mn, mx, first, half, depth + 1);
        int cr = leaf_code(mn, mx, first + half, count - half, depth + 1);
        set_child(node, 0, mn, mx, cl, 0);
        set_child(node, 1, mn, mx, cr, 0);
        return node;
    }

    int child_code(int ref_node, int depth)
    {
        const HostNode &n = b.nodes[ref_node];
        if (n.count > 0) return leaf_code(n.mn, n.mx, n.first, n.count, depth);
        return inner(ref_node, depth);
    }

    int inner(int ref_node, int depth)
    {
        const HostNode &n = b.nodes[ref_node];
        int node = alloc_node();
        if (depth > max_depth) max_depth = depth;
        int cl = child_code(n.left, depth + 1);
        int cr = child_code(n.right, depth + 1);
        const HostNode &L = b.nodes[n.left];
        const HostNode &R = b.nodes[n.right];
        set_child(node, 0, L.mn, L.mx, cl, 0);
        set_child(node, 1, R.mn, R.mx, cr, 0);
        return node;
    }
};

}  // namespace

void prim_bounds(const mt_prim &p, double mn[3], double mx[3])
{
    switch (p.kind) {
    case MT_PRIM_SPHERE:
        for (int k = 0; k < 3; ++k) {
            mn[k] = p.v[k] - p.v[3];
            mx[k] = p.v[k] + p.v[3];
        }
        break;
    case MT_PRIM_PLANE:
        for (int k = 0; k < 3; ++k) {
            mn[k] = -1e4;
            mx[k] = 1e4;
        }
        break;
    case MT_PRIM_BOX:
        for (int k = 0; k < 3; ++k) {
            double h = fabs(p.v[3 + k]);
            mn[k] = p.v[k] - h;
            mx[k] = p.v[k] + h;
        }
        break;
    case MT_PRIM_TRIANGLE:
        for (int k = 0; k < 3; ++k) {
            mn[k] = vmin(p.v[k], vmin(p.v[3 + k], p.v[6 + k]));
            mx[k] = vmax(p.v[k], vmax(p.v[3 + k], p.v[6 + k]));
        }
        break;
    case MT_PRIM_CYLINDER: {
        double rmax = (p.v[6] > p.v[7]) ? p.v[6] : p.v[7];
        if (rmax < 0.0) rmax = 0.0;
        for (int k = 0; k < 3; ++k) {
            mn[k] = vmin(p.v[k], p.v[3 + k]) - rmax;
            mx[k] = vmax(p.v[k], p.v[3 + k]) + rmax;
        }
        break;
    }
    default:
        for (int k = 0; k < 3; ++k) mn[k] = mx[k] = 0.0;
        break;
    }
}

namespace {

struct Pruner {
    const HostBvh &b;
    const mt_prim *prims;
    const std::vector<char> &keep;
    std::vector<HostNode> post;  // kept nodes, children before parents
    std::vector<int> order;

    static void pad(HostNode &n)
    {
        for (int k = 0; k < 3; ++k) {
            const double m = fabs(n.mn[k]) > fabs(n.mx[k]) ? fabs(n.mn[k]) : fabs(n.mx[k]);
            const double e = 4e-6 * (m + (n.mx[k] - n.mn[k])) + 1e-12;
            n.mn[k] -= e;
            n.mx[k] += e;
        }
    }

    // index in `post` of the pruned subtree of b.nodes[i], -1 when empty
    int run(int i)
    {
        const HostNode &n = b.nodes[i];
        HostNode o;
        for (int k = 0; k < 3; ++k) {
            o.mn[k] = 1e300;
            o.mx[k] = -1e300;
        }
        o.left = o.right = -1;
        o.first = o.count = 0;
        if (n.count > 0) {
            o.first = (int)order.size();
            for (int j = 0; j < n.count; ++j) {
                const int pi = b.order[n.first + j];
                if (!keep[pi]) continue;
                order.push_back(pi);
                double mn[3], mx[3];
                prim_bounds(prims[pi], mn, mx);
                for (int k = 0; k < 3; ++k) {
                    o.mn[k] = vmin(o.mn[k], mn[k]);
                    o.mx[k] = vmax(o.mx[k], mx[k]);
                }
            }
            o.count = (int)order.size() - o.first;
            if (!o.count) return -1;
            pad(o);
            post.push_back(o);
            return (int)post.size() - 1;
        }
        const int l = run(n.left), r = run(n.right);
        if (l < 0) return r;
        if (r < 0) return l;
        for (int k = 0; k < 3; ++k) {
            o.mn[k] = vmin(post[l].mn[k], post[r].mn[k]);
            o.mx[k] = vmax(post[l].mx[k], post[r].mx[k]);
        }
        o.left = l;
        o.right = r;
        post.push_back(o);
        return (int)post.size() - 1;
    }

    // copy the kept subtree at post[p] into out->nodes in preorder
    int emit(int p, int depth, HostBvh *out)
    {
        const int idx = (int)out->nodes.size();
        out->nodes.push_back(post[p]);
        if (post[p].count > 0) {
            if (depth > out->depth) out->depth = depth;
            return idx;
        }
        const int l = emit(post[p].left, depth + 1, out);
        const int r = emit(post[p].right, depth + 1, out);
        out->nodes[idx].left = l;
        out->nodes[idx].right = r;
        return idx;
    }
};

}  // namespace

int prune_bvh(const HostBvh &b, const mt_prim *prims, const std::vector<char> &keep, HostBvh *out)
{
    out->nodes.clear();
    out->order.clear();
    out->planes.clear();
    out->depth = 0;
    if (b.nodes.empty()) return 0;
    Pruner pr{b, prims, keep, {}, {}};
    const int root = pr.run(0);
    if (root < 0) return 0;
    out->order = std::move(pr.order);
    out->nodes.reserve(pr.post.size());
    pr.emit(root, 1, out);
    return 0;
}

int build_bvh(const mt_prim *prims, int n, HostBvh *out)
{
    out->nodes.clear();
    out->order.clear();
    out->planes.clear();
    out->depth = 0;
    if (n <= 0) return 0;
    std::vector<double> pmin(3 * (size_t)n), pmax(3 * (size_t)n), cen(3 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        if (prims[i].kind == MT_PRIM_PLANE) {
            out->planes.push_back(i);
            continue;
        }
        out->order.push_back(i);
        prim_bounds(prims[i], &pmin[3 * (size_t)i], &pmax[3 * (size_t)i]);
        for (int k = 0; k < 3; ++k) cen[3 * (size_t)i + k] = (pmin[3 * (size_t)i + k] + pmax[3 * (size_t)i + k]) * 0.5;
    }
    if (!out->order.empty()) {
        Builder bld{pmin.data(), pmax.data(), cen.data(), out};
        out->nodes.reserve(2 * out->order.size() / 3 + 16);
        bld.build(0, (int)out->order.size(), 1);
    }
    return 0;
}

int flatten_bvh(const HostBvh &b, FlatBvh *out)
{
    out->nodes.clear();
    out->ref_prim = b.order;
    out->node_count = 0;
    out->depth = 0;
    if (b.nodes.empty()) return 0;
    Flattener f{b, out};
    const HostNode &root = b.nodes[0];
    if (root.count > 0) {
        // A single-leaf tree: node 0 holds the leaf on the left and an empty
        // leaf (count 0) on the right.
        int node = f.alloc_node();
        int cl = f.leaf_code(root.mn, root.mx, root.first, root.count, 1);
        f.set_child(node, 0, root.mn, root.mx, cl, 0);
        f.set_child(node, 1, root.mn, root.mx, ~0, 0);
        f.max_depth = std::max(f.max_depth, 1);
    } else {
        f.inner(0, 1);
    }
    out->depth = f.max_depth;
    return 0;
}

namespace {

struct Slot {
    float mn[3], mx[3];
    int code;
};

struct Collapser {
    const std::vector<float> &n2;
    int W;
    std::vector<float> *out;
    int words;

    // child `side` (0 left, 1 right) of binary node `i`
    Slot child(int i, int side) const
    {
        const float *q = n2.data() + 16 * (size_t)i;
        Slot s;
        if (side == 0) {
            s.mn[0] = q[0], s.mx[0] = q[1], s.mn[1] = q[2], s.mx[1] = q[3], s.mn[2] = q[8], s.mx[2] = q[9];
        } else {
            s.mn[0] = q[4], s.mx[0] = q[5], s.mn[1] = q[6], s.mx[1] = q[7], s.mn[2] = q[10], s.mx[2] = q[11];
        }
        memcpy(&s.code, q + 12 + side, sizeof(int));
        return s;
    }
    static double area(const Slot &s)
    {
        double dx = (double)s.mx[0] - s.mn[0], dy = (double)s.mx[1] - s.mn[1], dz = (double)s.mx[2] - s.mn[2];
        return 2.0 * (dx * dy + dy * dz + dz * dx);
    }
    static bool empty_leaf(int code) { return code < 0 && ((~code) & 7) == 0; }

    // Emit the wide node for binary node i; returns its index and the stack
    // bound of its subtree.
    int emit(int i, int *bound)
    {
        std::vector<Slot> slots = {child(i, 0), child(i, 1)};
        while ((int)slots.size() < W) {
            int best = -1;
            double ba = -1.0;
            for (int k = 0; k < (int)slots.size(); ++k)
                if (slots[k].code >= 0 && area(slots[k]) > ba) {
                    ba = area(slots[k]);
                    best = k;
                }
            if (best < 0) break;
            int inner = slots[best].code;
            slots[best] = child(inner, 0);
            slots.insert(slots.begin() + best + 1, child(inner, 1));
        }
        std::vector<Slot> used;
        for (const Slot &s : slots)
            if (!empty_leaf(s.code)) used.push_back(s);
        const int idx = (int)(out->size() / (size_t)words);
        out->resize(out->size() + (size_t)words, 0.0f);
        int sub = 0;
        std::vector<int> codes(W, (int)0x80000000);
        for (int k = 0; k < (int)used.size(); ++k) {
            int code = used[k].code;
            if (code >= 0) {
                int b = 0;
                code = emit(code, &b);
                sub = std::max(sub, b);
            }
            codes[k] = code;
        }
        float *rec = out->data() + (size_t)idx * words;
        for (int k = 0; k < W; ++k) {
            bool on = k < (int)used.size();
            for (int a = 0; a < 3; ++a) {
                rec[(2 * a) * W + k] = on ? used[k].mn[a] : 0.0f;
                rec[(2 * a + 1) * W + k] = on ? used[k].mx[a] : 0.0f;
            }
            memcpy(rec + 6 * W + k, &codes[k], sizeof(int));
        }
        *bound = std::max(0, (int)used.size() - 1) + sub;
        return idx;
    }
};

}  // namespace

int collapse_bvh(const std::vector<float> &nodes2, int node_count, int W, std::vector<float> *out, int *stack_bound)
{
    out->clear();
    *stack_bound = 0;
    if (W != 4 && W != 8) return -1;
    if (node_count <= 0) return 0;
    Collapser c{nodes2, W, out, W == 4 ? 32 : 64};
    c.emit(0, stack_bound);
    return 0;
}

}  // namespace mt
