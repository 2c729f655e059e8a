/*
 * ref_harness_render.c - oracle harness: the reference Whitted renderer.
 *
 * TEST INFRASTRUCTURE ONLY (see ref_harness.h). Includes src/render.c to reach
 * the file-static trace() / sample_offset() / render_hash3() / to_byte()
 * (src/render.c:371-396,842-907). mtref_whitted_linear restates
 * render_region's per-pixel loop (src/render.c:924-970) without quantisation.
 */
#include "render.c"

#include "ref_harness.h"

#include <pthread.h>

unsigned mtref_render_hash3(unsigned a, unsigned b, unsigned c) { return render_hash3(a, b, c); }
unsigned char mtref_to_byte(double c) { return to_byte(c); }

/* render_image (src/render.c:1522): the fixed-spp Whitted entry point. */
int mtref_render_image(void *hp, int w, int h, int spp, int depth, unsigned char *rgb)
{
    MtRefHandle *H = (MtRefHandle *)hp;
    return render_image(&H->scene, &H->cam, w, h, spp, depth, rgb);
}

/* render_image_ex (src/render.c:1627). */
int mtref_render_image_ex(void *hp, int w, int h, int spp, int depth, int adaptive,
                          int adaptive_max, double tau, unsigned char *rgb)
{
    MtRefHandle *H = (MtRefHandle *)hp;
    RenderParams p;
    p.samples_per_pixel = spp;
    p.max_depth = depth;
    p.adaptive = adaptive;
    p.adaptive_max_spp = adaptive_max;
    p.adaptive_tau = tau;
    return render_image_ex(&H->scene, &H->cam, w, h, &p, rgb);
}

double mtref_render_last_seconds(void) { return render_last_seconds(); }

/* Primary ray of Whitted sample s at (x, y), src/render.c:935-949. */
static Ray mtref_wh_primary(const MtRefHandle *H, int w, int h, int spp, int x, int y, int s)
{
    double du, dv;
    sample_offset(spp, s, (unsigned)x, (unsigned)y, &du, &dv);
    double uu = ((double)x + du) / (double)w;
    double vv = 1.0 - ((double)y + dv) / (double)h;
    double lr1 = render_rand01((unsigned)x, (unsigned)y, (unsigned)(s * 2 + 2));
    double lr2 = render_rand01((unsigned)x, (unsigned)y, (unsigned)(s * 2 + 3));
    return camera_ray_dof(&H->cam, uu, vv, lr1, lr2);
}

int mtref_wh_primary_rays(void *hp, int w, int h, int spp, double *out)
{
    MtRefHandle *H = (MtRefHandle *)hp;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x)
            for (int s = 0; s < spp; ++s) {
                Ray r = mtref_wh_primary(H, w, h, spp, x, y, s);
                double *o = out + 6 * (((size_t)y * (size_t)w + (size_t)x) * (size_t)spp + (size_t)s);
                o[0] = r.origin.x; o[1] = r.origin.y; o[2] = r.origin.z;
                o[3] = r.dir.x; o[4] = r.dir.y; o[5] = r.dir.z;
            }
    return 0;
}

/* Batched Whitted trace() (src/render.c:842) at depth 0 with time 0. */
int mtref_whitted_trace(void *hp, int n, const double *o, const double *d, int depth,
                        const unsigned *seeds, double *out)
{
    MtRefHandle *H = (MtRefHandle *)hp;
    for (int i = 0; i < n; ++i) {
        Ray r;
        r.origin = vec3(o[3 * i], o[3 * i + 1], o[3 * i + 2]);
        r.dir = vec3(d[3 * i], d[3 * i + 1], d[3 * i + 2]);
        Vec3 c = trace(&H->scene, r, 0, depth, 0.0, seeds[i]);
        out[3 * i] = c.x;
        out[3 * i + 1] = c.y;
        out[3 * i + 2] = c.z;
    }
    return 0;
}

typedef struct {
    MtRefHandle *H;
    int w, h, spp, depth;
    double *out;
    int next_row;
    pthread_mutex_t lock;
} WhJob;

static void *mtref_wh_worker(void *arg)
{
    WhJob *J = (WhJob *)arg;
    for (;;) {
        int y;
        pthread_mutex_lock(&J->lock);
        y = J->next_row++;
        pthread_mutex_unlock(&J->lock);
        if (y >= J->h) break;
        for (int x = 0; x < J->w; ++x) {
            Vec3 acc = vec3(0.0, 0.0, 0.0);
            for (int s = 0; s < J->spp; ++s) {
                Ray ray = mtref_wh_primary(J->H, J->w, J->h, J->spp, x, y, s);
                unsigned seed_key = render_hash3((unsigned)x, (unsigned)y, (unsigned)s);
                acc = vec3_add(acc, trace(&J->H->scene, ray, 0, J->depth, 0.0, seed_key));
            }
            acc = vec3_scale(acc, 1.0 / (double)J->spp);
            double *p = J->out + 3 * ((size_t)y * (size_t)J->w + (size_t)x);
            p[0] = acc.x;
            p[1] = acc.y;
            p[2] = acc.z;
        }
    }
    return NULL;
}

/* Per-pixel MEAN linear Whitted colour (before to_byte). */
int mtref_whitted_linear(void *hp, int w, int h, int spp, int depth, double *out, int threads)
{
    WhJob J;
    pthread_t tids[256];
    int nt = threads > 0 ? threads : 1;
    if (nt > 256) nt = 256;
    J.H = (MtRefHandle *)hp;
    J.w = w; J.h = h; J.spp = spp; J.depth = depth;
    J.out = out;
    J.next_row = 0;
    pthread_mutex_init(&J.lock, NULL);
    for (int i = 0; i < nt; ++i) pthread_create(&tids[i], NULL, mtref_wh_worker, &J);
    for (int i = 0; i < nt; ++i) pthread_join(tids[i], NULL);
    pthread_mutex_destroy(&J.lock);
    return 0;
}
