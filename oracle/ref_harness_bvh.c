/*
 * ref_harness_bvh.c - oracle harness: the reference BVH.
 *
 * TEST INFRASTRUCTURE ONLY (see ref_harness.h). Includes src/bvh.c to reach
 * the opaque `struct Bvh` (src/bvh.c:66-76) so the tests can compare the
 * GPU library's host builder with the reference builder node by node, and
 * count node-pair / primitive tests of the reference traversal for the
 * algorithmic-bytes accounting of the roofline.
 */
#include "bvh.c"

#include "ref_harness.h"

/* Export nodes ({min xyz, max xyz} + {left, right, first, count}), the
 * permutation `order` and the plane list. Any array may be NULL. */
int mtref_bvh_export(void *hp, double *bounds6, int *links4, int *order, int *node_count,
                     int *order_count, int *planes, int *plane_count, int *depth)
{
    const Bvh *b = ((MtRefHandle *)hp)->scene.bvh;
    if (!b) return 1;
    if (node_count) *node_count = b->node_count;
    if (order_count) *order_count = b->order_count;
    if (plane_count) *plane_count = b->plane_count;
    if (depth) *depth = b->depth;
    for (int i = 0; i < b->node_count; ++i) {
        const BvhNode *n = &b->nodes[i];
        if (bounds6) {
            bounds6[6 * i + 0] = n->bounds_min.x;
            bounds6[6 * i + 1] = n->bounds_min.y;
            bounds6[6 * i + 2] = n->bounds_min.z;
            bounds6[6 * i + 3] = n->bounds_max.x;
            bounds6[6 * i + 4] = n->bounds_max.y;
            bounds6[6 * i + 5] = n->bounds_max.z;
        }
        if (links4) {
            links4[4 * i + 0] = n->left;
            links4[4 * i + 1] = n->right;
            links4[4 * i + 2] = n->first;
            links4[4 * i + 3] = n->count;
        }
    }
    if (order)
        for (int i = 0; i < b->order_count; ++i) order[i] = b->order[i];
    if (planes)
        for (int i = 0; i < b->plane_count; ++i) planes[i] = b->planes[i];
    return 0;
}

/*
 * Counting copy of the bvh_intersect traversal (src/bvh.c:557-712): same
 * stack discipline, cull rule and child order, with counters for inner
 * nodes whose two children were slab-tested and for primitive tests (plane
 * list included). Used only to state algorithmic bytes per ray.
 */
int mtref_bvh_count(void *hp, int n, const double *o, const double *d, double tmin,
                    double tmax, long long *node_pairs, long long *prim_tests,
                    long long *leaf_visits)
{
    const Scene *s = &((MtRefHandle *)hp)->scene;
    const Bvh *b = s->bvh;
    const Geometry *g = &s->geo;
    long long np = 0, pt = 0, lv = 0;
    if (!b) return 1;
    for (int k = 0; k < n; ++k) {
        Ray r;
        r.origin = vec3(o[3 * k], o[3 * k + 1], o[3 * k + 2]);
        r.dir = vec3(d[3 * k], d[3 * k + 1], d[3 * k + 2]);
        Vec3 inv = vec3(1.0 / r.dir.x, 1.0 / r.dir.y, 1.0 / r.dir.z);
        int found = 0;
        double closest = tmax;
        Hit best;
        for (int i = 0; i < b->plane_count; ++i) {
            int pi = b->planes[i];
            Hit h;
            h.prim_index = pi;
            ++pt;
            if (primitive_intersect(&g->prims[pi], r, tmin, closest, &h)) {
                if (!found || h.t < best.t || (h.t == best.t && h.prim_index < best.prim_index)) {
                    best = h;
                    closest = h.t;
                    found = 1;
                }
            }
        }
        if (b->node_count > 0) {
            BvhStackEntry stack[512];
            int sp = 0;
            BvhRaySimd rs;
            bvh_ray_simd_init(&rs, r.origin, inv);
            double t_root;
            if (bvh_slab(b->nodes[0].bounds_min, b->nodes[0].bounds_max, r.origin, inv, tmin,
                         closest, &t_root)) {
                stack[sp].idx = 0;
                stack[sp].t = t_root;
                ++sp;
            }
            while (sp > 0) {
                BvhStackEntry e = stack[--sp];
                if (found && e.t > closest) continue;
                const BvhNode *node = &b->nodes[e.idx];
                if (node->count > 0) {
                    ++lv;
                    for (int i = 0; i < node->count; ++i) {
                        int pi = b->order[node->first + i];
                        Hit h;
                        h.prim_index = pi;
                        ++pt;
                        if (primitive_intersect_norm(&g->prims[pi], r, tmin, closest, &h)) {
                            if (!found || h.t < best.t ||
                                (h.t == best.t && h.prim_index < best.prim_index)) {
                                best = h;
                                closest = h.t;
                                found = 1;
                            }
                        }
                    }
                } else {
                    double tl = 0.0, tr = 0.0;
                    int hl = 0, hr = 0;
                    ++np;
                    bvh_slab_2way(&b->nodes[node->left], &b->nodes[node->right], &rs, tmin,
                                  closest, &tl, &tr, &hl, &hr);
                    if (sp + 2 > 512) return 2;
                    if (hl && hr) {
                        if (tl <= tr) {
                            stack[sp].idx = node->right; stack[sp].t = tr; ++sp;
                            stack[sp].idx = node->left; stack[sp].t = tl; ++sp;
                        } else {
                            stack[sp].idx = node->left; stack[sp].t = tl; ++sp;
                            stack[sp].idx = node->right; stack[sp].t = tr; ++sp;
                        }
                    } else if (hl) {
                        stack[sp].idx = node->left; stack[sp].t = tl; ++sp;
                    } else if (hr) {
                        stack[sp].idx = node->right; stack[sp].t = tr; ++sp;
                    }
                }
            }
        }
    }
    *node_pairs = np;
    *prim_tests = pt;
    if (leaf_visits) *leaf_visits = lv;
    return 0;
}

/*
 * Canonical traversal work on the reference's tree for a batch of queries
 * with per-query bounds, on `threads` threads: the nearest-hit walk of
 * bvh_intersect (src/bvh.c:557-712) or the any-hit walk of bvh_occluded
 * (src/bvh.c:714-813, without its last-occluder shortcut), both restated
 * with counters. out[0] = inner nodes whose two child boxes were tested,
 * out[1] = triangle tests, out[2] = other primitive tests (planes included).
 * Used only for the algorithmic-bytes accounting of the roofline.
 */
#include <pthread.h>

typedef struct {
    const Scene *s;
    int any, n;
    const double *o, *d, *tmin, *tmax;
    long long out[3];
    int next;
    pthread_mutex_t lock;
} CountJob;

static void count_prim(const Primitive *p, long long *c)
{
    if (p->kind == PRIM_TRIANGLE)
        ++c[1];
    else
        ++c[2];
}

static void count_one(const Scene *s, int any, Ray r, double tmin, double tmax, long long *c)
{
    const Bvh *b = s->bvh;
    const Geometry *g = &s->geo;
    double len_sq = vec3_length_sq(r.dir);
    if (len_sq > 0.0 && fabs(len_sq - 1.0) > 1e-12) r.dir = vec3_normalize(r.dir);
    Vec3 inv = vec3(1.0 / r.dir.x, 1.0 / r.dir.y, 1.0 / r.dir.z);
    int found = 0;
    double closest = tmax;
    Hit best;
    best.t = 0.0;
    best.prim_index = -1;
    for (int i = 0; i < b->plane_count; ++i) {
        int pi = b->planes[i];
        count_prim(&g->prims[pi], c);
        if (any) {
            if (primitive_occluded(&g->prims[pi], r, tmin, tmax)) return;
        } else {
            Hit h;
            h.prim_index = pi;
            if (primitive_intersect(&g->prims[pi], r, tmin, closest, &h) &&
                (!found || h.t < best.t || (h.t == best.t && h.prim_index < best.prim_index))) {
                best = h;
                closest = h.t;
                found = 1;
            }
        }
    }
    if (b->node_count <= 0) return;
    struct { int idx; double t; } stack[512];
    int sp = 0;
    BvhRaySimd rs;
    bvh_ray_simd_init(&rs, r.origin, inv);
    double t_root;
    if (bvh_slab(b->nodes[0].bounds_min, b->nodes[0].bounds_max, r.origin, inv, tmin, closest, &t_root)) {
        stack[sp].idx = 0;
        stack[sp].t = t_root;
        ++sp;
    }
    while (sp > 0) {
        --sp;
        if (!any && found && stack[sp].t > closest) continue;
        const BvhNode *node = &b->nodes[stack[sp].idx];
        if (node->count > 0) {
            for (int i = 0; i < node->count; ++i) {
                int pi = b->order[node->first + i];
                count_prim(&g->prims[pi], c);
                if (any) {
                    if (primitive_occluded_norm(&g->prims[pi], r, tmin, tmax)) return;
                } else {
                    Hit h;
                    h.prim_index = pi;
                    if (primitive_intersect_norm(&g->prims[pi], r, tmin, closest, &h) &&
                        (!found || h.t < best.t || (h.t == best.t && h.prim_index < best.prim_index))) {
                        best = h;
                        closest = h.t;
                        found = 1;
                    }
                }
            }
        } else {
            double tl = 0.0, tr = 0.0;
            int hl = 0, hr = 0;
            ++c[0];
            bvh_slab_2way(&b->nodes[node->left], &b->nodes[node->right], &rs, tmin, closest, &tl, &tr, &hl,
                          &hr);
            if (sp + 2 > 512) return;
            if (hl && hr) {
                int first = tl <= tr ? node->right : node->left, second = tl <= tr ? node->left : node->right;
                double tf = tl <= tr ? tr : tl, ts = tl <= tr ? tl : tr;
                stack[sp].idx = first; stack[sp].t = tf; ++sp;
                stack[sp].idx = second; stack[sp].t = ts; ++sp;
            } else if (hl) {
                stack[sp].idx = node->left; stack[sp].t = tl; ++sp;
            } else if (hr) {
                stack[sp].idx = node->right; stack[sp].t = tr; ++sp;
            }
        }
    }
}

static void *count_worker(void *arg)
{
    CountJob *J = (CountJob *)arg;
    long long c[3] = {0, 0, 0};
    const int chunk = 1024;
    for (;;) {
        int i0;
        pthread_mutex_lock(&J->lock);
        i0 = J->next;
        J->next += chunk;
        pthread_mutex_unlock(&J->lock);
        if (i0 >= J->n) break;
        int i1 = i0 + chunk < J->n ? i0 + chunk : J->n;
        for (int i = i0; i < i1; ++i) {
            Ray r;
            r.origin = vec3(J->o[3 * i], J->o[3 * i + 1], J->o[3 * i + 2]);
            r.dir = vec3(J->d[3 * i], J->d[3 * i + 1], J->d[3 * i + 2]);
            count_one(J->s, J->any, r, J->tmin[i], J->tmax[i], c);
        }
    }
    pthread_mutex_lock(&J->lock);
    for (int k = 0; k < 3; ++k) J->out[k] += c[k];
    pthread_mutex_unlock(&J->lock);
    return NULL;
}

int mtref_bvh_count_batch(void *hp, int any, int n, const double *o, const double *d, const double *tmin,
                          const double *tmax, long long *out3, int threads)
{
    CountJob J;
    pthread_t tids[256];
    int nt = threads > 0 ? threads : 1;
    if (nt > 256) nt = 256;
    J.s = &((MtRefHandle *)hp)->scene;
    if (!J.s->bvh) return 1;
    J.any = any;
    J.n = n;
    J.o = o; J.d = d; J.tmin = tmin; J.tmax = tmax;
    J.out[0] = J.out[1] = J.out[2] = 0;
    J.next = 0;
    pthread_mutex_init(&J.lock, NULL);
    for (int i = 0; i < nt; ++i) pthread_create(&tids[i], NULL, count_worker, &J);
    for (int i = 0; i < nt; ++i) pthread_join(tids[i], NULL);
    pthread_mutex_destroy(&J.lock);
    for (int k = 0; k < 3; ++k) out3[k] = J.out[k];
    return 0;
}
