// mt_batch.cu - many images of uneven size, spp, depth and scene in one
// CUDA-graph launch (FP32 wavefront integrator).
//
// A batch context owns `lanes` sets of wavefront queues. The items are
// spread over the lanes longest-first by estimated cost (pixels x samples x
// bounces); each lane renders its items one after the other, and the lanes
// run concurrently. The whole schedule -- every item's sample window, batch
// by batch, bounce by bounce -- is captured once into one graph: a fork from
// the launching stream into one capture stream per lane and a join back. The
// stage kernels of different lanes then share the GPU: while one lane's
// queues drain at the deep bounces (few paths left), another lane's
// full-size stages fill the SMs. A graph is re-captured only when the item
// list changes shape (scenes, sizes, windows, depths, lane buffers).
//
// Per-item completion times come from event-record nodes inside the graph,
// measured from the graph's first node.
#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "mt_wavefront_host.cuh"

const mt::DevScene<float> *mt_scene_dev_f32(const mt_scene *scene);
int mt_scene_precision(const mt_scene *scene);
int mt_scene_device(const mt_scene *scene);
void mt_set_last_error_text(const char *msg);

struct mt_batch {
    int lanes = 1;
    int device = 0;
    long long capacity = 0;                 // path slots per lane
    std::vector<mt::WavefrontState *> st;   // queues of each lane
    std::vector<cudaStream_t> streams;      // capture streams of the lanes
    std::vector<cudaEvent_t> ev_join;
    cudaStream_t cap = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_start = nullptr, ev_end = nullptr;
    std::vector<cudaEvent_t> ev_item;
    cudaGraphExec_t exec = nullptr;
    std::string key;
    void *params = nullptr;    // device WfParams<float> per item
    void *h_params = nullptr;  // pinned staging of the same
    int params_cap = 0;
    int grid = 0;
};

namespace {

// Lanes sort a bounce's hits by material and place above this many paths,
// the library's default sort threshold.
constexpr int kBatchSortThreshold = 1 << 18;

int bfail(int code, const std::string &msg)
{
    mt_set_last_error_text(msg.c_str());
    return code;
}

#define BCK(call, what)                                                                                         \
    do {                                                                                                        \
        cudaError_t e_ = (call);                                                                                \
        if (e_ != cudaSuccess)                                                                                  \
            return bfail(e_ == cudaErrorMemoryAllocation ? MT_ERR_OOM : MT_ERR_LAUNCH,                           \
                         std::string(what) + ": " + cudaGetErrorString(e_));                                    \
    } while (0)

void fill_params(const mt_batch_item &it, mt::WfParams<float> *hp)
{
    memset(hp, 0, sizeof *hp);
    const mt_camera *c = it.cam;
    for (int k = 0; k < 3; ++k) {
        hp->cam.position[k] = (float)c->position[k];
        hp->cam.lower_left[k] = (float)c->lower_left[k];
        hp->cam.horizontal[k] = (float)c->horizontal[k];
        hp->cam.vertical[k] = (float)c->vertical[k];
    }
    hp->cam.aperture = (float)c->aperture;
    hp->cam.focus_distance = (float)c->focus_distance;
    hp->cam.dome_radius = (float)c->dome_radius;
    hp->cam.anamorphic_squeeze = (float)c->anamorphic_squeeze;
    hp->out = it.out_dev;
    hp->w = it.width;
    hp->h = it.height;
    hp->wh = it.width * it.height;
    hp->s0 = it.s0;
    hp->spp_window = it.spp;
    hp->out_kind = mt::OUT_MEAN_F32;
}

}  // namespace

extern "C" {

int mt_batch_create(int32_t lanes, int32_t queue_capacity, int32_t device, mt_batch **out)
{
    if (!out) return MT_ERR_NULL;
    *out = nullptr;
    if (lanes < 1 || lanes > 64) return bfail(MT_ERR_INVALID, "mt_batch_create: lanes must be in [1, 64]");
    if (queue_capacity < 0) return bfail(MT_ERR_INVALID, "mt_batch_create: negative queue capacity");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return bfail(MT_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return bfail(MT_ERR_INVALID, "mt_batch_create: device out of range");
    BCK(cudaSetDevice(device), "cudaSetDevice");
    mt_batch *b = new mt_batch();
    b->lanes = lanes;
    b->device = device;
    b->capacity = queue_capacity > 0 ? queue_capacity : (2ll << 20);
    auto bail = [&](int rc) {
        mt_batch_release(b);
        return rc;
    };
    b->st.assign(lanes, nullptr);
    b->streams.assign(lanes, nullptr);
    b->ev_join.assign(lanes, nullptr);
    for (int l = 0; l < lanes; ++l) {
        b->st[l] = new mt::WavefrontState();
        if (cudaStreamCreateWithFlags(&b->streams[l], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->ev_join[l], cudaEventDisableTiming) != cudaSuccess)
            return bail(bfail(MT_ERR_LAUNCH, "mt_batch_create: stream / event"));
    }
    if (cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&b->ev_start) != cudaSuccess || cudaEventCreate(&b->ev_end) != cudaSuccess)
        return bail(bfail(MT_ERR_LAUNCH, "mt_batch_create: stream / event"));
    *out = b;
    return MT_OK;
}

void mt_batch_release(mt_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    for (mt::WavefrontState *s : b->st)
        if (s) mt::wavefront_destroy(s);
    for (cudaStream_t s : b->streams)
        if (s) cudaStreamDestroy(s);
    for (cudaEvent_t e : b->ev_join)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : b->ev_item)
        if (e) cudaEventDestroy(e);
    if (b->cap) cudaStreamDestroy(b->cap);
    if (b->ev_fork) cudaEventDestroy(b->ev_fork);
    if (b->ev_start) cudaEventDestroy(b->ev_start);
    if (b->ev_end) cudaEventDestroy(b->ev_end);
    if (b->params) cudaFree(b->params);
    if (b->h_params) cudaFreeHost(b->h_params);
    delete b;
}

int mt_batch_render(mt_batch *b, int32_t n, const mt_batch_item *items, void *stream, float *item_ms,
                    float *total_ms)
{
    using namespace mt;
    if (!b || (n > 0 && !items)) return MT_ERR_NULL;
    if (n < 0) return bfail(MT_ERR_COUNTS, "mt_batch_render: negative item count");
    if (n == 0) return MT_OK;
    for (int i = 0; i < n; ++i) {
        const mt_batch_item &it = items[i];
        if (!it.scene || !it.cam || !it.out_dev) return bfail(MT_ERR_NULL, "mt_batch_render: NULL in item");
        if (it.width <= 0 || it.height <= 0 || (long long)it.width * it.height > (1ll << 28))
            return bfail(MT_ERR_DIMS, "mt_batch_render: bad image size");
        if (it.spp < 1 || it.s0 < 0 || it.depth < 0) return bfail(MT_ERR_COUNTS, "mt_batch_render: bad window");
        if (mt_scene_precision(it.scene) != MT_PRECISION_FP32)
            return bfail(MT_ERR_UNSUPPORTED, "mt_batch_render: FP32 scenes only");
        if (mt_scene_device(it.scene) != b->device)
            return bfail(MT_ERR_INVALID, "mt_batch_render: scene on another device");
    }
    BCK(cudaSetDevice(b->device), "cudaSetDevice");

    // ---- lanes: longest estimated item first onto the least-loaded lane ----
    std::vector<double> cost(n);
    for (int i = 0; i < n; ++i)
        cost[i] = (double)items[i].width * items[i].height * items[i].spp * (items[i].depth + 1);
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return cost[a] > cost[c]; });
    std::vector<double> load(b->lanes, 0.0);
    std::vector<std::vector<int>> lane_items(b->lanes);
    for (int i : order) {
        int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[l] += cost[i];
        lane_items[l].push_back(i);
    }
    // ---- queues of each lane: its largest batch ----
    std::vector<int> bspp(n), nbat(n);
    for (int l = 0; l < b->lanes; ++l) {
        size_t paths = 0, pixels = 0;
        for (int i : lane_items[l]) {
            const int wh = items[i].width * items[i].height;
            wf_batch_split(wh, items[i].spp, b->capacity, &bspp[i], &nbat[i]);
            paths = std::max(paths, (size_t)wh * bspp[i]);
            pixels = std::max(pixels, (size_t)wh);
        }
        if (!paths) continue;
        int rc = wf_reserve<float>(b->st[l], paths, pixels, kMaxLights);
        int buckets = 1;
        for (int i : lane_items[l])
            buckets = std::max(buckets, sort_buckets(mt_scene_dev_f32(items[i].scene)->material_count + 1));
        if (!rc) rc = wf_reserve_sort<float>(b->st[l], buckets);
        if (rc) return bfail(rc, std::string("mt_batch_render: ") + wavefront_last_error());
        bool pass = false;
        for (int i : lane_items[l]) pass = pass || mt_scene_dev_f32(items[i].scene)->has_passthrough;
        if (pass) wf_reserve_links<float>(b->st[l]);
    }
    if (!b->grid) {
        int sms = 0, per_sm = 0;
        const DevScene<float> &S0 = *mt_scene_dev_f32(items[0].scene);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wf_extend<float, 2>, 128,
                                                      (size_t)(S0.stack_depth > 0 ? S0.stack_depth : 1) * 128 * 4);
        b->grid = sms * (per_sm > 0 ? per_sm : 1);
    }
    for (int l = 0; l < b->lanes; ++l) {
        b->st[l]->grid = b->grid;
        b->st[l]->occ_cache_on = true;  // reset before each item: a lane renders several scenes
        b->st[l]->pass_cache_on = false;
    }
    // ---- parameter blocks ----
    if (n > b->params_cap) {
        if (b->params) cudaFree(b->params);
        if (b->h_params) cudaFreeHost(b->h_params);
        b->params = b->h_params = nullptr;
        b->params_cap = 0;
        BCK(cudaMalloc(&b->params, (size_t)n * sizeof(WfParams<float>)), "cudaMalloc(params)");
        BCK(cudaMallocHost(&b->h_params, (size_t)n * sizeof(WfParams<float>)), "cudaMallocHost(params)");
        b->params_cap = n;
    }
    while ((int)b->ev_item.size() < n) {
        cudaEvent_t e;
        BCK(cudaEventCreate(&e), "cudaEventCreate");
        b->ev_item.push_back(e);
    }
    // ---- graph: captured once per item-list shape ----
    std::string key = std::to_string(n) + ":" + std::to_string((uintptr_t)b->params);
    for (int l = 0; l < b->lanes; ++l)
        key += ":" + std::to_string((uintptr_t)b->st[l]->paths) + "/" + std::to_string((uintptr_t)b->st[l]->link[0]);
    for (int i = 0; i < n; ++i) {
        const DevScene<float> &S = *mt_scene_dev_f32(items[i].scene);
        char buf[160];
        snprintf(buf, sizeof buf, "|%p:%d:%d:%d:%d:%d", (const void *)S.nodes, S.version, items[i].width,
                 items[i].height, items[i].spp, items[i].depth);
        key += buf;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (!b->exec || b->key != key) {
        if (b->exec) cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
        b->key.clear();
        BCK(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "begin capture");
        int erc = 0;
        cudaError_t ce = cudaEventRecordWithFlags(b->ev_start, b->cap, cudaEventRecordExternal);
        if (ce == cudaSuccess) ce = cudaEventRecord(b->ev_fork, b->cap);
        for (int l = 0; l < b->lanes && ce == cudaSuccess && !erc; ++l) {
            ce = cudaStreamWaitEvent(b->streams[l], b->ev_fork, 0);
            for (int i : lane_items[l]) {
                if (ce != cudaSuccess || erc) break;
                DevScene<float> S = *mt_scene_dev_f32(items[i].scene);
                S.counters = nullptr;
                const WfParams<float> *P = (const WfParams<float> *)b->params + i;
                // the occluder cache holds BVH leaves of one scene
                ce = cudaMemsetAsync(b->st[l]->occ_cache, 0xFF, occ_cache_ints(b->st[l]->acc_pixels) * sizeof(int),
                                     b->streams[l]);
                if (ce != cudaSuccess) break;
                erc = wf_enqueue<float>(b->st[l], S, items[i].width, items[i].height, bspp[i], nbat[i],
                                        items[i].depth, b->streams[l], false, 128, false, false, P, kBatchSortThreshold);
                if (!erc) ce = cudaEventRecordWithFlags(b->ev_item[i], b->streams[l], cudaEventRecordExternal);
            }
            if (ce == cudaSuccess && !erc) ce = cudaEventRecord(b->ev_join[l], b->streams[l]);
            if (ce == cudaSuccess && !erc) ce = cudaStreamWaitEvent(b->cap, b->ev_join[l], 0);
        }
        if (ce == cudaSuccess && !erc) ce = cudaEventRecordWithFlags(b->ev_end, b->cap, cudaEventRecordExternal);
        cudaGraph_t graph = nullptr;
        cudaError_t ee = cudaStreamEndCapture(b->cap, &graph);
        if (erc || ce != cudaSuccess || ee != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            if (erc) return bfail(erc, std::string("mt_batch_render: ") + wavefront_last_error());
            return bfail(MT_ERR_LAUNCH, std::string("mt_batch_render: capture: ") +
                                            cudaGetErrorString(ce != cudaSuccess ? ce : ee));
        }
        cudaError_t ie = cudaGraphInstantiate(&b->exec, graph, 0);
        cudaGraphDestroy(graph);
        BCK(ie, "graph instantiate");
        b->key = key;
    }
    // ---- launch: parameter blocks, then the graph ----
    BCK(cudaStreamSynchronize(s), "cudaStreamSynchronize");  // the pinned staging may be in use
    WfParams<float> *hp = (WfParams<float> *)b->h_params;
    for (int i = 0; i < n; ++i) fill_params(items[i], hp + i);
    BCK(cudaMemcpyAsync(b->params, b->h_params, (size_t)n * sizeof(WfParams<float>), cudaMemcpyHostToDevice, s),
        "params copy");
    BCK(cudaGraphLaunch(b->exec, s), "graph launch");
    if (item_ms || total_ms) {
        BCK(cudaStreamSynchronize(s), "batch");
        for (int i = 0; item_ms && i < n; ++i) BCK(cudaEventElapsedTime(&item_ms[i], b->ev_start, b->ev_item[i]), "t");
        if (total_ms) BCK(cudaEventElapsedTime(total_ms, b->ev_start, b->ev_end), "t");
    }
    return MT_OK;
}

}  // extern "C"
