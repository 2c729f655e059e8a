// mt_noalloc.cu - a path-tracing entry point that allocates no memory.
//
// Who needs it: callers that cannot call cudaMalloc / cudaFree while they
// render. One example is a host application that hands the whole device
// memory budget to its own pool allocator up front, so a library allocation
// would fail or would break the pool's accounting. Another is a render loop
// that must not pay the implicit device-wide synchronisation cudaMalloc and
// cudaFree perform. mt_render_accumulate_device_noalloc serves them. It runs
// the same wavefront stage kernels as mt_render_accumulate_device, but its
// queues and path state live in one fixed array owned by this file instead
// of in buffers allocated on demand.
//
// The array (kScratchBytes, 12 MiB) is a file-scope __device__ variable. A
// GPU holds it from the moment this file's device code is loaded on it until
// the process exits. CUDA loads modules lazily by default (CUDA 12.2 and
// later), so that moment is the first call of this entry point on the device
// (its cudaGetSymbolAddress), not the library's load; with
// CUDA_MODULE_LOADING=EAGER it is the process's first CUDA call. A caller
// whose pool later takes the whole device budget must therefore make one
// call on each device (a warm-up) before the pool reserves its memory, or
// run with CUDA_MODULE_LOADING=EAGER. If the array cannot be loaded, the
// call returns MT_ERR_OOM with error text. The array bounds one call to
// kMaxPixels pixels (one sample of every pixel per batch); larger images are
// rejected with MT_ERR_INVALID.
//
// Host code cannot use the array's name as a device address (on the host it
// names a host-side stand-in). The first call on each device therefore looks
// up the array's device address with cudaGetSymbolAddress while that device
// is current, and caches it. Make that first call on a device before
// capturing any stream.
//
// The call's parameter block (camera, window, output) is written into the
// array by a one-thread kernel that receives it by value, so no host buffer
// has to outlive the call.
//
// Renders through this entry point are not counted by mt_set_counting /
// mt_get_stats.
//
// All calls share the one array and it keeps the last call's contents. Every
// value a call reads is written earlier by the same call: the queue counters
// are zeroed at the start of each batch, and path state, NEE slots and the
// pixel accumulator are initialised before they are read. Calls that overlap
// on the GPU (two streams, or two host threads at once) race on the array;
// serialise them.
#include <mutex>

#include "mt_wavefront_host.cuh"

void mt_set_last_error_text(const char *msg);

namespace {

constexpr int kMaxPixels = 16384;
constexpr size_t kScratchBytes = size_t(12) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mutex;
unsigned char *g_scratch_ptr[kMaxDevices] = {nullptr};
int g_grid[kMaxDevices] = {0};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Store the call's parameter block (passed by value in the launch) into the
// scratch array.
__global__ void k_noalloc_params(const mt::WfParams<float> p, mt::WfParams<float> *dst) { *dst = p; }

int fail_text(int code, const char *msg)
{
    mt_set_last_error_text(msg);
    return code;
}

// Carve the wavefront buffers for `n_paths` paths / `wh` pixels out of the
// scratch array; returns the bytes used.
size_t carve(unsigned char *base, size_t n_paths, size_t wh, int light_count, mt::WavefrontState *st)
{
    using namespace mt;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char *p = base + off;
        off += align256(bytes);
        return (void *)p;
    };
    st->paths = take(n_paths * sizeof(WfPath<float>));
    st->rays[0] = take(n_paths * sizeof(WfRay<float>));
    st->rays[1] = take(n_paths * sizeof(WfRay<float>));
    st->hits = take(n_paths * sizeof(WfHit<float>));
    st->nee = take(n_paths * kNeeSlots * 3 * sizeof(float));
    st->shadow = take(n_paths * (size_t)(light_count + 1) * sizeof(WfShadow<float>));
    st->sample_buf = take(n_paths * 3 * sizeof(float));
    st->acc = take(wh * 3 * sizeof(float));
    st->params = take(sizeof(WfParams<float>));
    st->counters = (WfCounters *)take(sizeof(WfCounters));
    return off;
}

}  // namespace

// The scene's FP32 device arrays (mt_api.cu).
const mt::DevScene<float> *mt_scene_dev_f32(const mt_scene *scene);
int mt_scene_precision(const mt_scene *scene);
int mt_scene_device(const mt_scene *scene);

extern "C" int mt_render_accumulate_device_noalloc(mt_scene *scene, const mt_camera *cam, int width, int height,
                                                   int spp_begin, int spp_end, int max_depth, float *accum_dev,
                                                   int accumulate, void *stream)
{
    using namespace mt;
    if (!scene || !cam || !accum_dev) return MT_ERR_NULL;
    if (width <= 0 || height <= 0) return MT_ERR_DIMS;
    if (spp_end - spp_begin < 1 || spp_begin < 0 || max_depth < 0) return MT_ERR_COUNTS;
    if ((long long)width * height > kMaxPixels) {
        mt_set_last_error_text("mt_render_accumulate_device_noalloc: width * height exceeds the fixed scratch "
                               "array's limit of 16384 pixels");
        return MT_ERR_INVALID;
    }
    if (mt_scene_precision(scene) != MT_PRECISION_FP32) {
        mt_set_last_error_text("mt_render_accumulate_device_noalloc: FP32 scenes only");
        return MT_ERR_UNSUPPORTED;
    }
    const int dev = mt_scene_device(scene);
    if (dev < 0 || dev >= kMaxDevices)
        return fail_text(MT_ERR_INVALID, "mt_render_accumulate_device_noalloc: device index out of range");
    if (cudaSetDevice(dev) != cudaSuccess)
        return fail_text(MT_ERR_NO_DEVICE, "mt_render_accumulate_device_noalloc: cudaSetDevice failed");

    const DevScene<float> &S = *mt_scene_dev_f32(scene);
    {
        // Once per device, with that device current: the device address of
        // the scratch array, and the persistent grid of the stage kernels.
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
                cudaGetLastError();  // clear the (non-sticky) error of the failed lookup
                return fail_text(MT_ERR_OOM, "mt_render_accumulate_device_noalloc: could not load the 12 MiB "
                                             "scratch array on this device (device memory exhausted?)");
            }
            int sms = 0, per_sm = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wf_extend<float, 2>, 128,
                                                          (size_t)(S.stack_depth > 0 ? S.stack_depth : 1) * 128 * 4);
            g_grid[dev] = sms * (per_sm > 0 ? per_sm : 1);
            g_scratch_ptr[dev] = (unsigned char *)p;
        }
    }

    const int wh = width * height;
    WavefrontState st;  // a view of the scratch array: nothing here is allocated
    if (carve(g_scratch_ptr[dev], (size_t)wh, (size_t)wh, S.light_count, &st) > kScratchBytes)
        return fail_text(MT_ERR_INVALID, "mt_render_accumulate_device_noalloc: the buffers of this image do not "
                                         "fit the scratch array");
    st.grid = g_grid[dev];

    WfParams<float> hp;
    memset(&hp, 0, sizeof hp);
    for (int k = 0; k < 3; ++k) {
        hp.cam.position[k] = (float)cam->position[k];
        hp.cam.lower_left[k] = (float)cam->lower_left[k];
        hp.cam.horizontal[k] = (float)cam->horizontal[k];
        hp.cam.vertical[k] = (float)cam->vertical[k];
    }
    hp.cam.aperture = (float)cam->aperture;
    hp.cam.focus_distance = (float)cam->focus_distance;
    hp.cam.dome_radius = (float)cam->dome_radius;
    hp.cam.anamorphic_squeeze = (float)cam->anamorphic_squeeze;
    hp.out = accum_dev;
    hp.w = width;
    hp.h = height;
    hp.wh = wh;
    hp.s0 = spp_begin;
    hp.spp_window = spp_end - spp_begin;
    hp.out_kind = accumulate ? OUT_ADD_F32 : OUT_SUM_F32;
    cudaStream_t s = (cudaStream_t)stream;
    k_noalloc_params<<<1, 1, 0, s>>>(hp, (WfParams<float> *)st.params);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::string msg = std::string("mt_render_accumulate_device_noalloc: parameter kernel: ") + cudaGetErrorString(e);
        return fail_text(MT_ERR_LAUNCH, msg.c_str());
    }
    // One sample of every pixel per batch: n_paths == pixels.
    int rc = wf_enqueue<float>(&st, S, width, height, 1, spp_end - spp_begin, max_depth, s, false, 128);
    if (rc) {
        std::string msg = std::string("mt_render_accumulate_device_noalloc: ") + wavefront_last_error();
        return fail_text(rc, msg.c_str());
    }
    return 0;
}
