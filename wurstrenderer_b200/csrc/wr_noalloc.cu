// wr_render_device_noalloc: the wavefront render with all of its scratch memory
// in one fixed, statically allocated device array, so that the call itself
// allocates nothing.
//
// Who needs it: host applications that run under a fixed device-memory budget
// or must not allocate once they are running -- for example an engine that has
// handed the rest of the GPU to its own caching allocator, or a latency-bound
// service that cannot afford the implicit device synchronisation that
// cudaMalloc/cudaFree may perform while other streams are busy. wr_render_device
// allocates its wavefront buffers on first use (and again when the film size or
// queue capacity changes); this variant never does.
//
// Limits and rules:
//   * scratch: kScratchBytes = 10 MiB in a file-scope __device__ array; every
//     GPU that loads this library holds it until the process exits;
//   * film at most kMaxPixels = 65,536 pixels (e.g. 256 x 256); larger cameras
//     are rejected with WR_ERR_INVALID_ARGUMENT;
//   * the wavefront holds kCapacity = 32,768 paths (desc->queue_capacity,
//     use_graph and profile are ignored; kernels are launched one by one);
//   * the integrator is chosen as wr_render_device chooses it (desc->integrator,
//     else the render entry's "integrator"); the learned proposal needs its own
//     network buffers, so desc->guiding != 0 is rejected with WR_ERR_UNSUPPORTED;
//   * all calls share the one array: the film, counters and sample cursor are
//     cleared at the start of every call, and two calls whose work overlaps on
//     the GPU (for example from two threads with two scene handles on one
//     device) race on it -- serialise them;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (with that device current); make that first call
//     before any stream capture is started.

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/wurst_b200.h"
#include "wr_host.h"
#include "wr_kernels.h"

namespace wr_internal {
struct SceneView {
    wrd::DevScene dev;
    cudaStream_t stream;
    int device;
    uint32_t *pinned;
    cudaEvent_t ev0, ev1;
    const wr::Scene *host;
    wr_render_stats *stats;
};
bool scene_view(wr_scene *s, SceneView *v);
wrd::DevCamera camera_constants(const wr::Camera &c);
void set_last_error(const std::string &m);
int resolve_request(const wr::Scene &h, const wr_render_desc &desc, int *spp, int *nverts, int *integrator);
}  // namespace wr_internal

namespace {

constexpr size_t kScratchBytes = size_t(10) << 20;
constexpr uint32_t kCapacity = 32768;
constexpr size_t kMaxPixels = 65536;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_setup_mutex;
unsigned char *g_scratch_ptr[kMaxDevices] = {};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// carves the wavefront and film out of the scratch array; returns the bytes used
size_t carve(unsigned char *base, size_t npix, wrk::WaveBuffers &b) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char *p = base + off;
        off = align256(off + bytes);
        return p;
    };
    for (int p = 0; p < 2; ++p) {
        b.o[p] = reinterpret_cast<float4 *>(take(size_t(kCapacity) * 16));
        b.d[p] = reinterpret_cast<float4 *>(take(size_t(kCapacity) * 16));
        b.thr[p] = reinterpret_cast<float4 *>(take(size_t(kCapacity) * 16));
        b.meta[p] = reinterpret_cast<uint32_t *>(take(size_t(kCapacity) * 4));
    }
    b.hit = reinterpret_cast<float4 *>(take(size_t(kCapacity) * 16));
    b.sh_o = reinterpret_cast<float4 *>(take(size_t(kCapacity) * 2 * 16));
    b.sh_d = reinterpret_cast<float4 *>(take(size_t(kCapacity) * 2 * 16));
    b.sh_c = reinterpret_cast<float4 *>(take(size_t(kCapacity) * 2 * 16));
    b.ctr = reinterpret_cast<uint32_t *>(take(wrd::CTR_COUNT * 4));
    b.sample_next = reinterpret_cast<unsigned long long *>(take(8));
    b.film = reinterpret_cast<double *>(take(npix * 6 * 8));
    b.capacity = kCapacity;
    b.shadow_capacity = 2 * kCapacity;
    return off;
}

int fail(int code, const std::string &m) {
    wr_internal::set_last_error(m);
    return code;
}

// makes the scene's device current for the call and gives the caller's device back on every return
struct DeviceGuard {
    int prev = -1;
    cudaError_t enter(int device) {
        cudaError_t e = cudaGetDevice(&prev);
        if (e != cudaSuccess) {
            prev = -1;
            return e;
        }
        if (prev == device) {
            prev = -1;   // nothing to restore
            return cudaSuccess;
        }
        e = cudaSetDevice(device);
        if (e != cudaSuccess) prev = -1;
        return e;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

#define NA_CUDA(call)                                                                         \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(WR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

}  // namespace

extern "C" int wr_render_device_noalloc(wr_scene *scene, const wr_render_desc *desc_in, double *out_rgb_device) {
    wr_internal::SceneView v;
    if (!wr_internal::scene_view(scene, &v) || !out_rgb_device) return fail(WR_ERR_INVALID_ARGUMENT, "null argument");
    const wr::Scene &h = *v.host;
    wr_render_desc desc{};
    if (desc_in) desc = *desc_in;
    if (desc.guiding != 0)
        return fail(WR_ERR_UNSUPPORTED, "wr_render_device_noalloc: the learned proposal (guiding) needs network "
                                        "buffers of its own; use wr_render_device");
    if (desc.max_iterations < 0) return fail(WR_ERR_INVALID_ARGUMENT, "max_iterations must be >= 0");
    int spp = 0, nverts = 0, integrator = 0;
    // camera, render entry, spp, vertices and integrator exactly as wr_render_device resolves them
    const int rc = wr_internal::resolve_request(h, desc, &spp, &nverts, &integrator);
    if (rc != WR_OK) return rc;
    if (spp <= 0) return fail(WR_ERR_INVALID_ARGUMENT, "num_spp must be positive");
    const size_t npix = size_t(h.camera.width) * size_t(h.camera.height);
    if (npix > kMaxPixels)
        return fail(WR_ERR_INVALID_ARGUMENT, "wr_render_device_noalloc: film of " + std::to_string(npix) +
                                                 " pixels exceeds the fixed scratch limit of " + std::to_string(kMaxPixels) +
                                                 " pixels (use wr_render_device)");
    if (v.device < 0 || v.device >= kMaxDevices) return fail(WR_ERR_UNSUPPORTED, "device index out of range");

    DeviceGuard guard;
    NA_CUDA(guard.enter(v.device));
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_scratch_ptr[v.device]) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
            if (e != cudaSuccess)
                return fail(WR_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
            g_scratch_ptr[v.device] = static_cast<unsigned char *>(p);
        }
        base = g_scratch_ptr[v.device];
    }
    wrk::WaveBuffers b{};
    const size_t used = carve(base, npix, b);
    if (used > kScratchBytes) return fail(WR_ERR_INVALID_ARGUMENT, "film does not fit the fixed scratch array");

    int sms = 148;
    NA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, v.device));
    wrk::RenderLaunch r{};
    r.jobs = nullptr;
    r.num_jobs = 1;
    r.job0 = wrd::DevJob{};
    r.job0.cam = wr_internal::camera_constants(h.camera);
    r.job0.spp = spp;
    // a BSDF-only path of one vertex traces nothing (as wr_render_device)
    r.job0.nverts = (integrator == wrd::INTEGRATOR_PRIMITIVE && nverts <= 1) ? 1 : nverts;
    r.job0.npix = uint32_t(npix);
    r.job0.pix_offset = 0;
    r.job0.sample_begin = 0;
    r.job0.seed = desc.seed;
    r.job0.integrator = integrator;
    // the same shade kernel as wr_render_device picks for a one-job NEE render, so that both entry
    // points compute the same image
    r.nee_only = integrator == wrd::INTEGRATOR_NEE ? 1 : 0;
    r.total_pix = uint32_t(npix);
    r.total_samples = (unsigned long long)npix * unsigned(spp);
    const unsigned long long waves = (r.total_samples + kCapacity - 1) / kCapacity;
    r.iter_limit = uint32_t(std::min<unsigned long long>((waves + 2) * (unsigned long long)(std::max(nverts, 0) + 2) + 64,
                                                         0xffffffffull));
    if (desc.max_iterations > 0) r.iter_limit = std::min(r.iter_limit, uint32_t(desc.max_iterations));
    r.trace_block = (desc.trace_block == 64 || desc.trace_block == 256) ? desc.trace_block : 128;
    r.grid_trace = desc.grid_trace > 0 ? desc.grid_trace
                                       : sms * std::max(1, wrk::occupancy_blocks(0, r.trace_block, v.dev.patches != nullptr, v.dev.wnodes != nullptr));
    r.grid_shade = desc.grid_shade > 0 ? desc.grid_shade : sms * (wrk::occupancy_blocks(1) > 0 ? wrk::occupancy_blocks(1) : 1);
    if (desc.fetch_threshold < 0 || desc.fetch_threshold > 32)
        return fail(WR_ERR_INVALID_ARGUMENT, "fetch_threshold must be 0..32");
    r.fetch_min = desc.fetch_threshold > 0 ? desc.fetch_threshold : 20;
    r.has_cond = 0;
    r.prof = nullptr;

    cudaStream_t st = v.stream;
    NA_CUDA(cudaMemsetAsync(b.film, 0, npix * 6 * 8, st));
    NA_CUDA(cudaMemsetAsync(b.ctr, 0, wrd::CTR_COUNT * 4, st));
    NA_CUDA(cudaMemsetAsync(b.sample_next, 0, 8, st));
    NA_CUDA(cudaEventRecord(v.ev0, st));
    const bool trace = nverts > 1;
    unsigned long long launches = 0;
    if (trace) {
        wrk::launch_prime(v.dev, b, r, st);
        NA_CUDA(cudaGetLastError());
        launches += 3;
        bool done = false;
        while (!done) {
            wrk::launch_iteration(v.dev, b, r, 0, st);
            wrk::launch_iteration(v.dev, b, r, 1, st);
            NA_CUDA(cudaGetLastError());
            launches += 10;
            NA_CUDA(cudaMemcpyAsync(v.pinned, b.ctr, wrd::CTR_COUNT * 4, cudaMemcpyDeviceToHost, st));
            NA_CUDA(cudaStreamSynchronize(st));
            done = v.pinned[wrd::CTR_DONE] != 0;
        }
        if (v.pinned[wrd::CTR_TIMEOUT]) return fail(WR_ERR_TIMEOUT, "wavefront did not drain within the iteration bound");
        if (v.pinned[wrd::CTR_OVERFLOW]) return fail(WR_ERR_CUDA, "shadow queue overflow");
    }
    wrk::launch_resolve(b.film, out_rgb_device, r, st);
    NA_CUDA(cudaGetLastError());
    launches += 1;
    NA_CUDA(cudaEventRecord(v.ev1, st));
    NA_CUDA(cudaStreamSynchronize(st));
    float ms = 0.f;
    NA_CUDA(cudaEventElapsedTime(&ms, v.ev0, v.ev1));
    wr_render_stats &stats = *v.stats;
    stats = wr_render_stats{};
    stats.render_ms = ms;
    stats.paths = r.total_samples;
    stats.iterations = trace ? v.pinned[wrd::CTR_ITER] : 0;   // bounce iterations + 1, as wr_render_device
    stats.max_shadow_queue = trace ? v.pinned[wrd::CTR_SHADOW_MAX] : 0;
    stats.queue_capacity = kCapacity;
    stats.grid_trace = r.grid_trace;
    stats.grid_shade = r.grid_shade;
    stats.trace_block = r.trace_block;
    stats.kernel_launches = launches;
    return WR_OK;
}
