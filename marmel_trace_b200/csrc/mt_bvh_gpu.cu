// mt_bvh_gpu.cu - the reference's binned-SAH BVH builder (src/bvh.c:180-422)
// run breadth-first on the device.
//
// Every split decision of the reference builder is a function of the SET of
// primitives in the node: the node and centroid bounds, the 12 bins' counts
// and bounds along the axis of largest centroid extent, the SAH sweep, and
// the median test (centroid < midpoint). Only the order of primitives inside
// a node depends on its in-place two-pointer partition. This builder
// evaluates the same decisions with the same double arithmetic, level by
// level for all nodes of a level at once, and partitions each node stably
// (an exclusive scan of the "goes left" flags). The tree is therefore the
// reference's tree -- same nodes, bounds, leaves and left/right order, node
// numbering in preorder -- with the primitives of each node in a different
// order. The one exception is the median fallback's positional split, which
// the reference takes only when the midpoint rounds onto the smallest
// centroid (centroids one ulp apart): it splits the current order at count/2,
// and the current order differs.
//
// Per level: (1) node bounds and centroid bounds by atomic min / max on an
// order-preserving integer image of the doubles, reduced within a warp first;
// (2) per node: bounds +- BVH_BOUNDS_EPS, leaf test, split axis; (3) bin
// counts and bounds by atomics; (4) per node: the SAH sweep, or the median;
// (5) goes-left flags and a device-wide exclusive scan; (6) per node: child
// allocation; (7) the stable scatter into the next level's order.
#include <cub/cub.cuh>

#include <string>
#include <vector>

#include "mt_bvh.h"

namespace mt {

namespace {

constexpr int kLeafSizeG = 4;         // BVH_LEAF_SIZE, src/bvh.c:41
constexpr int kBinsG = 12;            // BVH_NBINS, src/bvh.c:43
constexpr double kBoundsEpsG = 1e-7;  // BVH_BOUNDS_EPS, src/bvh.c:45
constexpr int kModeLeaf = -1, kModeMedian = 100, kModePositional = 200;

// order-preserving image of a double in uint64 (atomicMin / atomicMax)
__device__ __forceinline__ unsigned long long ord(double d)
{
    unsigned long long b = (unsigned long long)__double_as_longlong(d);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double unord(unsigned long long u)
{
    unsigned long long b = (u >> 63) ? (u & 0x7fffffffffffffffull) : ~u;
    return __longlong_as_double((long long)b);
}

__device__ __forceinline__ double surface_area_d(const double *mn, const double *mx)
{
    double dx = mx[0] - mn[0];
    double dy = mx[1] - mn[1];
    double dz = mx[2] - mn[2];
    if (dx < 0.0) dx = 0.0;
    if (dy < 0.0) dy = 0.0;
    if (dz < 0.0) dz = 0.0;
    return 2.0 * (dx * dy + dy * dz + dz * dx);
}

struct Tasks {
    int *first, *count, *node, *depth, *mode, *axis, *nleft, *child;  // child: left task id (right = +1)
    double *cmin, *scale, *mid;
    unsigned long long *acc;   // 12 per task: mn, mx, cmn, cmx (xyz each)
    int *bcount;               // 12 per task
    unsigned long long *bacc;  // 72 per task: per bin mn xyz, mx xyz
};

struct Nodes {
    double *mn, *mx;  // 3 each
    int *left, *right, *first, *count, *depth;
};

__global__ void k_init_tasks(Tasks T, int n)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    for (int k = 0; k < 12; ++k) T.acc[12 * (size_t)t + k] = ((k / 3) % 2 == 0) ? ord(1e300) : ord(-1e300);
    for (int b = 0; b < kBinsG; ++b) {
        T.bcount[kBinsG * (size_t)t + b] = 0;
        for (int k = 0; k < 6; ++k) T.bacc[72 * (size_t)t + 6 * b + k] = k < 3 ? ord(1e300) : ord(-1e300);
    }
}

// (1) node bounds and centroid bounds
__global__ void k_node_bounds(int m, const int *pos_task, const int *order, const double *pmin, const double *pmax,
                              const double *cen, Tasks T)
{
    const int stride = gridDim.x * blockDim.x;
    const int m_round = (m + stride - 1) / stride * stride;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m_round; i += stride) {
        const int t = i < m ? pos_task[i] : -1;
        unsigned long long v[12];
        if (t >= 0) {
            const int p = order[i];
            for (int k = 0; k < 3; ++k) {
                v[k] = ord(pmin[3 * (size_t)p + k]);
                v[3 + k] = ord(pmax[3 * (size_t)p + k]);
                v[6 + k] = ord(cen[3 * (size_t)p + k]);
                v[9 + k] = ord(cen[3 * (size_t)p + k]);
            }
        }
        const int t0 = __shfl_sync(0xffffffffu, t, 0);
        if (__all_sync(0xffffffffu, t == t0)) {
            if (t0 < 0) continue;
            for (int k = 0; k < 12; ++k) {
                const bool is_min = (k / 3) % 2 == 0;
                for (int o = 16; o > 0; o >>= 1) {
                    unsigned long long w = __shfl_xor_sync(0xffffffffu, v[k], o);
                    v[k] = is_min ? (w < v[k] ? w : v[k]) : (w > v[k] ? w : v[k]);
                }
            }
            if ((threadIdx.x & 31) == 0)
                for (int k = 0; k < 12; ++k) {
                    if ((k / 3) % 2 == 0) atomicMin(&T.acc[12 * (size_t)t0 + k], v[k]);
                    else atomicMax(&T.acc[12 * (size_t)t0 + k], v[k]);
                }
        } else if (t >= 0) {
            for (int k = 0; k < 12; ++k) {
                if ((k / 3) % 2 == 0) atomicMin(&T.acc[12 * (size_t)t + k], v[k]);
                else atomicMax(&T.acc[12 * (size_t)t + k], v[k]);
            }
        }
    }
}

// (2) bounds, leaf test, split axis (bvh_build_node, src/bvh.c:180-215)
__global__ void k_node_setup(int n_tasks, Tasks T, Nodes N)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tasks) return;
    const unsigned long long *a = T.acc + 12 * (size_t)t;
    double mn[3], mx[3], cmn[3], cmx[3];
    for (int k = 0; k < 3; ++k) {
        mn[k] = unord(a[k]) - kBoundsEpsG;
        mx[k] = unord(a[3 + k]) + kBoundsEpsG;
        cmn[k] = unord(a[6 + k]);
        cmx[k] = unord(a[9 + k]);
    }
    const int nd = T.node[t];
    for (int k = 0; k < 3; ++k) {
        N.mn[3 * (size_t)nd + k] = mn[k];
        N.mx[3 * (size_t)nd + k] = mx[k];
    }
    N.depth[nd] = T.depth[t];
    N.left[nd] = -1;
    N.right[nd] = -1;
    N.first[nd] = 0;
    N.count[nd] = 0;
    const int count = T.count[t];
    int mode = 0;
    if (count <= kLeafSizeG) {
        mode = kModeLeaf;
    } else {
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
        if (!(max_ext > 0.0)) {
            mode = kModeLeaf;
        } else {
            T.axis[t] = axis;
            T.cmin[t] = cmn[axis];
            T.scale[t] = kBinsG / max_ext;
            T.mid[t] = 0.5 * (cmn[axis] + cmx[axis]);
        }
    }
    if (mode == kModeLeaf) {
        N.first[nd] = T.first[t];
        N.count[nd] = count;
    }
    T.mode[t] = mode;
}

__device__ __forceinline__ int bin_of_d(double cv, double cmin, double scale)
{
    int bin = (int)((cv - cmin) * scale);
    if (bin < 0) bin = 0;
    if (bin >= kBinsG) bin = kBinsG - 1;
    return bin;
}

// (3) bins
__global__ void k_bins(int m, const int *pos_task, const int *order, const double *pmin, const double *pmax,
                       const double *cen, Tasks T)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const int t = pos_task[i];
        if (t < 0 || T.mode[t] == kModeLeaf) continue;
        const int p = order[i];
        const int axis = T.axis[t];
        const int bin = bin_of_d(cen[3 * (size_t)p + axis], T.cmin[t], T.scale[t]);
        atomicAdd(&T.bcount[kBinsG * (size_t)t + bin], 1);
        unsigned long long *b = T.bacc + 72 * (size_t)t + 6 * bin;
        for (int k = 0; k < 3; ++k) {
            atomicMin(&b[k], ord(pmin[3 * (size_t)p + k]));
            atomicMax(&b[3 + k], ord(pmax[3 * (size_t)p + k]));
        }
    }
}

// (4) the SAH sweep (src/bvh.c:230-282); no cheaper split: median
__global__ void k_sah(int n_tasks, Tasks T, Nodes N)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tasks || T.mode[t] == kModeLeaf) return;
    const int *bc = T.bcount + kBinsG * (size_t)t;
    const unsigned long long *ba = T.bacc + 72 * (size_t)t;
    double rmin[kBinsG][3], rmax[kBinsG][3];
    int rcount[kBinsG];
    double acc_min[3] = {1e300, 1e300, 1e300}, acc_max[3] = {-1e300, -1e300, -1e300};
    int acc_n = 0;
    for (int i = kBinsG - 1; i >= 0; --i) {
        if (bc[i] > 0) {
            for (int k = 0; k < 3; ++k) {
                double lo = unord(ba[6 * i + k]), hi = unord(ba[6 * i + 3 + k]);
                acc_min[k] = acc_min[k] < lo ? acc_min[k] : lo;
                acc_max[k] = acc_max[k] > hi ? acc_max[k] : hi;
            }
            acc_n += bc[i];
        }
        for (int k = 0; k < 3; ++k) {
            rmin[i][k] = acc_min[k];
            rmax[i][k] = acc_max[k];
        }
        rcount[i] = acc_n;
    }
    double lmin[3] = {1e300, 1e300, 1e300}, lmax[3] = {-1e300, -1e300, -1e300};
    int lacc_n = 0;
    double best_cost = 1e300;
    int best_split = -1;
    for (int i = 0; i < kBinsG - 1; ++i) {
        if (bc[i] > 0) {
            for (int k = 0; k < 3; ++k) {
                double lo = unord(ba[6 * i + k]), hi = unord(ba[6 * i + 3 + k]);
                lmin[k] = lmin[k] < lo ? lmin[k] : lo;
                lmax[k] = lmax[k] > hi ? lmax[k] : hi;
            }
            lacc_n += bc[i];
        }
        const int rn = rcount[i + 1];
        if (lacc_n == 0 || rn == 0) continue;
        const double la = surface_area_d(lmin, lmax);
        const double ra = surface_area_d(rmin[i + 1], rmax[i + 1]);
        const double cost = la * (double)lacc_n + ra * (double)rn;
        if (cost < best_cost) {
            best_cost = cost;
            best_split = i;
        }
    }
    const int nd = T.node[t];
    const double leaf_cost = surface_area_d(N.mn + 3 * (size_t)nd, N.mx + 3 * (size_t)nd) * (double)T.count[t];
    T.mode[t] = (best_split >= 0 && best_cost < leaf_cost) ? best_split : kModeMedian;
}

// (5) goes-left flags
__global__ void k_flags(int m, const int *pos_task, const int *order, const double *cen, Tasks T, int *flags)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= m; i += gridDim.x * blockDim.x) {
        int f = 0;
        if (i < m) {
            const int t = pos_task[i];
            if (t >= 0) {
                const int mode = T.mode[t];
                if (mode != kModeLeaf) {
                    const double cv = cen[3 * (size_t)order[i] + T.axis[t]];
                    f = mode == kModeMedian ? (cv < T.mid[t]) : (bin_of_d(cv, T.cmin[t], T.scale[t]) <= mode);
                }
            }
        }
        flags[i] = f;
    }
}

// (6) child nodes and tasks of the next level
__global__ void k_children(int n_tasks, Tasks T, Tasks Tn, Nodes N, const int *scan, int *next_tasks,
                           int *node_counter)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_tasks || T.mode[t] == kModeLeaf) return;
    const int first = T.first[t], count = T.count[t];
    int nleft = scan[first + count] - scan[first];
    if (nleft <= 0 || nleft >= count) {
        // src/bvh.c:306-308: a one-sided median split falls back to count / 2
        nleft = count / 2;
        T.mode[t] = kModePositional;
    }
    T.nleft[t] = nleft;
    const int c = atomicAdd(next_tasks, 2);
    const int nd = atomicAdd(node_counter, 2);
    T.child[t] = c;
    const int me = T.node[t];
    N.left[me] = nd;
    N.right[me] = nd + 1;
    Tn.first[c] = first;
    Tn.count[c] = nleft;
    Tn.node[c] = nd;
    Tn.depth[c] = T.depth[t] + 1;
    Tn.first[c + 1] = first + nleft;
    Tn.count[c + 1] = count - nleft;
    Tn.node[c + 1] = nd + 1;
    Tn.depth[c + 1] = T.depth[t] + 1;
}

// (7) stable scatter into the next level's order
__global__ void k_scatter(int m, const int *pos_task, const int *order, const int *flags, const int *scan, Tasks T,
                          int *order_next, int *pos_next)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const int t = pos_task[i];
        if (t < 0 || T.mode[t] == kModeLeaf) {
            order_next[i] = order[i];
            pos_next[i] = -1;
            continue;
        }
        const int first = T.first[t];
        const int nleft = T.nleft[t];
        const int rank = i - first;
        int lrank;
        bool left;
        if (T.mode[t] == kModePositional) {
            left = rank < nleft;
            lrank = left ? rank : nleft;
        } else {
            left = flags[i] != 0;
            lrank = scan[i] - scan[first];
        }
        const int np = left ? first + lrank : first + nleft + (rank - lrank);
        order_next[np] = order[i];
        pos_next[np] = T.child[t] + (left ? 0 : 1);
    }
}

template <typename T> struct DBuf {
    T *p = nullptr;
    size_t n = 0;
    ~DBuf()
    {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t count)
    {
        if (count <= n) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, (count ? count : 1) * sizeof(T));
        if (e == cudaSuccess) n = count;
        return e;
    }
};

struct TaskBufs {
    DBuf<int> first, count, node, depth, mode, axis, nleft, child;
    DBuf<double> cmin, scale, mid;
    DBuf<unsigned long long> acc, bacc;
    DBuf<int> bcount;
    cudaError_t alloc(size_t n)
    {
        cudaError_t e = cudaSuccess;
        DBuf<int> *ints[] = {&first, &count, &node, &depth, &mode, &axis, &nleft, &child, &bcount};
        for (DBuf<int> *b : ints)
            if (e == cudaSuccess) e = b->alloc(b == &bcount ? n * kBinsG : n);
        DBuf<double> *ds[] = {&cmin, &scale, &mid};
        for (DBuf<double> *b : ds)
            if (e == cudaSuccess) e = b->alloc(n);
        if (e == cudaSuccess) e = acc.alloc(n * 12);
        if (e == cudaSuccess) e = bacc.alloc(n * 72);
        return e;
    }
    Tasks view()
    {
        return Tasks{first.p, count.p, node.p, depth.p, mode.p, axis.p, nleft.p, child.p,
                     cmin.p,  scale.p, mid.p,  acc.p,   bcount.p, bacc.p};
    }
};

int grid_of(long long n, int block)
{
    long long g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > 148 * 32) g = 148 * 32;
    return (int)g;
}

}  // namespace

#define GB_CK(call)                                                                   \
    do {                                                                              \
        cudaError_t e_ = (call);                                                      \
        if (e_ != cudaSuccess) {                                                      \
            if (err) *err = std::string(#call) + ": " + cudaGetErrorString(e_);       \
            return e_ == cudaErrorMemoryAllocation ? MT_ERR_OOM : MT_ERR_LAUNCH;      \
        }                                                                             \
    } while (0)

int build_bvh_device(const mt_prim *prims, int n, HostBvh *out, std::string *err, float *ms)
{
    out->nodes.clear();
    out->order.clear();
    out->planes.clear();
    out->depth = 0;
    if (ms) *ms = 0.f;
    if (n <= 0) return 0;
    // primitive bounds and centroids on the host (primitive_bounds restated,
    // O(n)); the tree build itself runs on the device
    std::vector<int> tree_prims;
    std::vector<double> pmin, pmax, cen;
    tree_prims.reserve(n);
    for (int i = 0; i < n; ++i) {
        if (prims[i].kind == MT_PRIM_PLANE) {
            out->planes.push_back(i);
            continue;
        }
        double mn[3], mx[3];
        prim_bounds(prims[i], mn, mx);
        tree_prims.push_back(i);
        for (int k = 0; k < 3; ++k) {
            pmin.push_back(mn[k]);
            pmax.push_back(mx[k]);
            cen.push_back((mn[k] + mx[k]) * 0.5);
        }
    }
    const int m = (int)tree_prims.size();
    if (m == 0) return 0;

    cudaEvent_t e0 = nullptr, e1 = nullptr;
    GB_CK(cudaEventCreate(&e0));
    GB_CK(cudaEventCreate(&e1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard()
        {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } evg{e0, e1};

    DBuf<double> d_pmin, d_pmax, d_cen;
    DBuf<int> order[2], pos[2], flags, scan, counters;
    GB_CK(d_pmin.alloc(3 * (size_t)m));
    GB_CK(d_pmax.alloc(3 * (size_t)m));
    GB_CK(d_cen.alloc(3 * (size_t)m));
    for (int k = 0; k < 2; ++k) {
        GB_CK(order[k].alloc(m));
        GB_CK(pos[k].alloc(m));
    }
    GB_CK(flags.alloc(m + 1));
    GB_CK(scan.alloc(m + 1));
    GB_CK(counters.alloc(2));  // next-level task count, node count
    const size_t max_nodes = 2 * (size_t)m;
    DBuf<double> nmn, nmx;
    DBuf<int> nleft_, nright, nfirst, ncount, ndepth;
    GB_CK(nmn.alloc(3 * max_nodes));
    GB_CK(nmx.alloc(3 * max_nodes));
    GB_CK(nleft_.alloc(max_nodes));
    GB_CK(nright.alloc(max_nodes));
    GB_CK(nfirst.alloc(max_nodes));
    GB_CK(ncount.alloc(max_nodes));
    GB_CK(ndepth.alloc(max_nodes));
    Nodes N{nmn.p, nmx.p, nleft_.p, nright.p, nfirst.p, ncount.p, ndepth.p};
    size_t scan_bytes = 0;
    GB_CK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, flags.p, scan.p, m + 1));
    DBuf<unsigned char> scan_tmp;
    GB_CK(scan_tmp.alloc(scan_bytes));

    GB_CK(cudaMemcpy(d_pmin.p, pmin.data(), pmin.size() * sizeof(double), cudaMemcpyHostToDevice));
    GB_CK(cudaMemcpy(d_pmax.p, pmax.data(), pmax.size() * sizeof(double), cudaMemcpyHostToDevice));
    GB_CK(cudaMemcpy(d_cen.p, cen.data(), cen.size() * sizeof(double), cudaMemcpyHostToDevice));
    {
        std::vector<int> iota(m), zeros(m, 0);
        for (int i = 0; i < m; ++i) iota[i] = i;
        GB_CK(cudaMemcpy(order[0].p, iota.data(), m * sizeof(int), cudaMemcpyHostToDevice));
        GB_CK(cudaMemcpy(pos[0].p, zeros.data(), m * sizeof(int), cudaMemcpyHostToDevice));
    }
    TaskBufs tb[2];
    GB_CK(tb[0].alloc(1));
    {
        int root[4] = {0, m, 0, 1};  // first, count, node, depth
        GB_CK(cudaMemcpy(tb[0].first.p, &root[0], sizeof(int), cudaMemcpyHostToDevice));
        GB_CK(cudaMemcpy(tb[0].count.p, &root[1], sizeof(int), cudaMemcpyHostToDevice));
        GB_CK(cudaMemcpy(tb[0].node.p, &root[2], sizeof(int), cudaMemcpyHostToDevice));
        GB_CK(cudaMemcpy(tb[0].depth.p, &root[3], sizeof(int), cudaMemcpyHostToDevice));
    }
    int node_count = 1;
    GB_CK(cudaMemcpy(counters.p + 1, &node_count, sizeof(int), cudaMemcpyHostToDevice));
    GB_CK(cudaEventRecord(e0, 0));
    int n_tasks = 1, cur = 0;
    const int B = 256;
    const int G = grid_of(m, B);
    for (int level = 0; n_tasks > 0; ++level) {
        if (level > 4096) {
            if (err) *err = "device BVH build did not terminate";
            return MT_ERR_WATCHDOG;
        }
        TaskBufs &T = tb[cur];
        TaskBufs &Tn = tb[cur ^ 1];
        GB_CK(Tn.alloc(2 * (size_t)n_tasks));
        Tasks tv = T.view(), tnv = Tn.view();
        const int Gt = grid_of(n_tasks, B);
        k_init_tasks<<<(n_tasks + B - 1) / B, B>>>(tv, n_tasks);
        k_node_bounds<<<G, B>>>(m, pos[0].p, order[0].p, d_pmin.p, d_pmax.p, d_cen.p, tv);
        k_node_setup<<<(n_tasks + B - 1) / B, B>>>(n_tasks, tv, N);
        k_bins<<<G, B>>>(m, pos[0].p, order[0].p, d_pmin.p, d_pmax.p, d_cen.p, tv);
        k_sah<<<(n_tasks + 63) / 64, 64>>>(n_tasks, tv, N);
        k_flags<<<grid_of(m + 1, B), B>>>(m, pos[0].p, order[0].p, d_cen.p, tv, flags.p);
        GB_CK(cub::DeviceScan::ExclusiveSum(scan_tmp.p, scan_bytes, flags.p, scan.p, m + 1));
        GB_CK(cudaMemset(counters.p, 0, sizeof(int)));
        k_children<<<(n_tasks + B - 1) / B, B>>>(n_tasks, tv, tnv, N, scan.p, counters.p, counters.p + 1);
        k_scatter<<<G, B>>>(m, pos[0].p, order[0].p, flags.p, scan.p, tv, order[1].p, pos[1].p);
        (void)Gt;
        GB_CK(cudaGetLastError());
        std::swap(order[0].p, order[1].p);
        std::swap(pos[0].p, pos[1].p);
        GB_CK(cudaMemcpy(&n_tasks, counters.p, sizeof(int), cudaMemcpyDeviceToHost));
        cur ^= 1;
    }
    GB_CK(cudaEventRecord(e1, 0));
    GB_CK(cudaMemcpy(&node_count, counters.p + 1, sizeof(int), cudaMemcpyDeviceToHost));
    if (ms) GB_CK(cudaEventElapsedTime(ms, e0, e1));

    // download and renumber in preorder (the reference's node order)
    std::vector<double> hmn(3 * (size_t)node_count), hmx(3 * (size_t)node_count);
    std::vector<int> hl(node_count), hr(node_count), hf(node_count), hc(node_count), hd(node_count), hord(m);
    GB_CK(cudaMemcpy(hmn.data(), nmn.p, hmn.size() * sizeof(double), cudaMemcpyDeviceToHost));
    GB_CK(cudaMemcpy(hmx.data(), nmx.p, hmx.size() * sizeof(double), cudaMemcpyDeviceToHost));
    GB_CK(cudaMemcpy(hl.data(), nleft_.p, node_count * sizeof(int), cudaMemcpyDeviceToHost));
    GB_CK(cudaMemcpy(hr.data(), nright.p, node_count * sizeof(int), cudaMemcpyDeviceToHost));
    GB_CK(cudaMemcpy(hf.data(), nfirst.p, node_count * sizeof(int), cudaMemcpyDeviceToHost));
    GB_CK(cudaMemcpy(hc.data(), ncount.p, node_count * sizeof(int), cudaMemcpyDeviceToHost));
    GB_CK(cudaMemcpy(hd.data(), ndepth.p, node_count * sizeof(int), cudaMemcpyDeviceToHost));
    GB_CK(cudaMemcpy(hord.data(), order[0].p, m * sizeof(int), cudaMemcpyDeviceToHost));

    out->order.resize(m);
    for (int i = 0; i < m; ++i) out->order[i] = tree_prims[hord[i]];
    out->nodes.reserve(node_count);
    std::vector<int> stack = {0};
    std::vector<int> new_index(node_count, -1);
    // preorder: a node, then its left subtree, then its right subtree
    while (!stack.empty()) {
        const int d = stack.back();
        stack.pop_back();
        new_index[d] = (int)out->nodes.size();
        HostNode h;
        for (int k = 0; k < 3; ++k) {
            h.mn[k] = hmn[3 * (size_t)d + k];
            h.mx[k] = hmx[3 * (size_t)d + k];
        }
        h.left = hl[d];
        h.right = hr[d];
        h.first = hf[d];
        h.count = hc[d];
        out->nodes.push_back(h);
        if (hd[d] > out->depth) out->depth = hd[d];
        if (hl[d] >= 0) {
            stack.push_back(hr[d]);
            stack.push_back(hl[d]);
        }
    }
    for (HostNode &h : out->nodes)
        if (h.left >= 0) {
            h.left = new_index[h.left];
            h.right = new_index[h.right];
        }
    return 0;
}

}  // namespace mt
