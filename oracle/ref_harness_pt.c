/*
 * ref_harness_pt.c - oracle harness: the reference path tracer.
 *
 * TEST INFRASTRUCTURE ONLY (see ref_harness.h). Includes src/pathtrace.c to
 * reach its file-static PRNG (pt_hash3 / pt_rand01, src/pathtrace.c:92-117).
 * mtref_pathtrace_linear restates pt_render_pixel (src/pathtrace.c:1047-1096)
 * without the final quantisation, so tests can compare linear means.
 */
#include "pathtrace.c"

#include "ref_harness.h"

#include <pthread.h>
#include <stdlib.h>

unsigned mtref_pt_hash3(unsigned a, unsigned b, unsigned c) { return pt_hash3(a, b, c); }
double mtref_pt_rand01(unsigned a, unsigned b, unsigned c) { return pt_rand01(a, b, c); }
unsigned char mtref_pt_to_byte(double v) { return pathtrace_to_byte(v); }

/* The reference entry point (src/pathtrace.c:1256), threaded by RAYTRACER_THREADS. */
int mtref_pathtrace_render(void *hp, int w, int h, int spp, int depth, unsigned char *rgb)
{
    MtRefHandle *H = (MtRefHandle *)hp;
    return pathtrace_render(&H->scene, &H->cam, w, h, spp, depth, rgb);
}

/* Primary ray of sample s at pixel (x, y), src/pathtrace.c:1057-1082. */
static Ray mtref_pt_primary(const MtRefHandle *H, int w, int h, int x, int y, int s)
{
    const Scene *scene = &H->scene;
    const Camera *cam = &H->cam;
    double jx = pt_rand01((unsigned)x, (unsigned)y, (unsigned)(s * 2 + 0));
    double jy = pt_rand01((unsigned)x, (unsigned)y, (unsigned)(s * 2 + 1));
    double lr1 = pt_rand01((unsigned)x, (unsigned)y, (unsigned)(s * 2 + 100));
    double lr2 = pt_rand01((unsigned)x, (unsigned)y, (unsigned)(s * 2 + 101));
    double uu = ((double)x + jx) / (double)w;
    double vv = 1.0 - ((double)y + jy) / (double)h;
    Ray ray = camera_ray_dof(cam, uu, vv, lr1, lr2);
    if (cam->dome_radius > 1e-4 && scene->water_material >= 0) {
        Vec3 p_dome = vec3_add(ray.origin, vec3_scale(ray.dir, cam->dome_radius));
        double wh = scene_water_height(scene, p_dome.x, p_dome.z);
        if (p_dome.y < wh) ray.origin = vec3_sub(p_dome, vec3(0.0, 1e-3, 0.0));
    }
    return ray;
}

/* Rays for every (x, y, s) in ((y*w + x)*spp + s) order, 6 doubles each. */
int mtref_pt_primary_rays(void *hp, int w, int h, int spp, double *out)
{
    MtRefHandle *H = (MtRefHandle *)hp;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x)
            for (int s = 0; s < spp; ++s) {
                Ray r = mtref_pt_primary(H, w, h, x, y, s);
                double *o = out + 6 * (((size_t)y * (size_t)w + (size_t)x) * (size_t)spp + (size_t)s);
                o[0] = r.origin.x; o[1] = r.origin.y; o[2] = r.origin.z;
                o[3] = r.dir.x; o[4] = r.dir.y; o[5] = r.dir.z;
            }
    return 0;
}

/* Batched pathtrace_radiance (src/pathtrace.c:800). */
int mtref_pathtrace_radiance(void *hp, int n, const double *o, const double *d, int depth,
                             const unsigned *seeds, double *out)
{
    MtRefHandle *H = (MtRefHandle *)hp;
    for (int i = 0; i < n; ++i) {
        Ray r;
        r.origin = vec3(o[3 * i], o[3 * i + 1], o[3 * i + 2]);
        r.dir = vec3(d[3 * i], d[3 * i + 1], d[3 * i + 2]);
        Vec3 L = pathtrace_radiance(&H->scene, r, depth, seeds[i]);
        out[3 * i] = L.x;
        out[3 * i + 1] = L.y;
        out[3 * i + 2] = L.z;
    }
    return 0;
}

typedef struct {
    MtRefHandle *H;
    int w, h, spp, s0, depth;
    double *out;
    int next_row;
    pthread_mutex_t lock;
} PtJob;

static void *mtref_pt_worker(void *arg)
{
    PtJob *J = (PtJob *)arg;
    for (;;) {
        int y;
        pthread_mutex_lock(&J->lock);
        y = J->next_row++;
        pthread_mutex_unlock(&J->lock);
        if (y >= J->h) break;
        for (int x = 0; x < J->w; ++x) {
            Vec3 acc = vec3(0.0, 0.0, 0.0);
            for (int s = J->s0; s < J->s0 + J->spp; ++s) {
                Ray ray = mtref_pt_primary(J->H, J->w, J->h, x, y, s);
                unsigned seed_key = pt_hash3((unsigned)x, (unsigned)y, (unsigned)s);
                acc = vec3_add(acc, pathtrace_radiance(&J->H->scene, ray, J->depth, seed_key));
            }
            /* SUM over the window; the caller scales by 1/spp. */
            double *p = J->out + 3 * ((size_t)y * (size_t)J->w + (size_t)x);
            p[0] = acc.x;
            p[1] = acc.y;
            p[2] = acc.z;
        }
    }
    return NULL;
}

/*
 * Per-pixel SUM of the linear radiance of samples [s0, s0+spp), summed in
 * sample order as pt_render_pixel does (src/pathtrace.c:1053-1088).
 * `threads` <= 0 means one thread.
 */
int mtref_pathtrace_linear(void *hp, int w, int h, int s0, int spp, int depth, double *out,
                           int threads)
{
    PtJob J;
    pthread_t tids[256];
    int nt = threads > 0 ? threads : 1;
    if (nt > 256) nt = 256;
    J.H = (MtRefHandle *)hp;
    J.w = w; J.h = h; J.spp = spp; J.s0 = s0; J.depth = depth;
    J.out = out;
    J.next_row = 0;
    pthread_mutex_init(&J.lock, NULL);
    for (int i = 0; i < nt; ++i) pthread_create(&tids[i], NULL, mtref_pt_worker, &J);
    for (int i = 0; i < nt; ++i) pthread_join(tids[i], NULL);
    pthread_mutex_destroy(&J.lock);
    return 0;
}

/*
 * Batched traversal queries with per-query bounds, on `threads` threads, for
 * checking logged device queries one by one:
 *   kind 0: scene_intersect over [tmin[i], tmax[i]] (src/scene.c:767-775):
 *           result = prim_index (-1: miss), t_out = hit distance;
 *   kind 1: pt_occluded_segment over [tmin[i], tmax[i]] (src/pathtrace.c:504-532),
 *           the path tracer's shadow query: result = 1 when blocked.
 */
typedef struct {
    MtRefHandle *H;
    int kind, n;
    const double *o, *d, *tmin, *tmax;
    int *result;
    double *t_out;
    int next;
    pthread_mutex_t lock;
} QueryJob;

static void *mtref_query_worker(void *arg)
{
    QueryJob *J = (QueryJob *)arg;
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
            if (J->kind == 0) {
                Hit h;
                if (scene_intersect(&J->H->scene, r, J->tmin[i], J->tmax[i], &h)) {
                    J->result[i] = h.prim_index;
                    if (J->t_out) J->t_out[i] = h.t;
                } else {
                    J->result[i] = -1;
                    if (J->t_out) J->t_out[i] = 0.0;
                }
            } else {
                Vec3 att;
                J->result[i] = pt_occluded_segment(&J->H->scene, r, J->tmin[i], J->tmax[i], &att);
            }
        }
    }
    return NULL;
}

int mtref_queries(void *hp, int kind, int n, const double *o, const double *d, const double *tmin,
                  const double *tmax, int *result, double *t_out, int threads)
{
    QueryJob J;
    pthread_t tids[256];
    int nt = threads > 0 ? threads : 1;
    if (nt > 256) nt = 256;
    if (kind != 0 && kind != 1) return 1;
    J.H = (MtRefHandle *)hp;
    J.kind = kind;
    J.n = n;
    J.o = o; J.d = d; J.tmin = tmin; J.tmax = tmax;
    J.result = result;
    J.t_out = t_out;
    J.next = 0;
    pthread_mutex_init(&J.lock, NULL);
    for (int i = 0; i < nt; ++i) pthread_create(&tids[i], NULL, mtref_query_worker, &J);
    for (int i = 0; i < nt; ++i) pthread_join(tids[i], NULL);
    pthread_mutex_destroy(&J.lock);
    return 0;
}
