// dc_runtime.cu — device contexts, cached buffers and textures, profiler.
#include <atomic>
#include <algorithm>
#include <condition_variable>
#include <thread>
#include <cstdlib>
#include <cuda.h>

#include "dc_runtime.cuh"
#include "dc_common.cuh"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>

#include "../../include/dosecuda.h"

namespace dc {

static thread_local std::string g_last_error;

void set_last_error(const std::string &msg) { g_last_error = msg; }
const char *last_error_cstr() { return g_last_error.c_str(); }

void throw_cuda(cudaError_t e, const char *what) {
    // The reference reports "CUDA error: <cudaGetErrorString>" (dosemodule.cu:195).
    std::string m = cudaGetErrorString(e);
    m += " (";
    m += what;
    m += ")";
    throw Error(DC_ERR_CUDA, m);
}

void check_launch(const char *kernel) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw_cuda(e, kernel);
}

// ---------------------------------------------------------------------------
// Allocation-failure injection for failure tests: with DC_INJECT_ALLOC_FAIL=N
// in the environment, the N-th device / pinned / array allocation of the
// process fails (before the CUDA call) as an out-of-memory would.
void check_injected_alloc(const char *what) {
    static const long long fail_at = [] {
        const char *e = std::getenv("DC_INJECT_ALLOC_FAIL");
        return e ? std::atoll(e) : 0LL;
    }();
    static std::atomic<long long> count{0};
    if (fail_at <= 0) return;
    const long long k = ++count;
    if (k == fail_at)
        throw Error(DC_ERR_CUDA, std::string("out of memory (injected failure of allocation ") + std::to_string(k) +
                                     ", " + what + ")");
}

namespace {
using PointerAttrFn = CUresult (*)(void *, CUpointer_attribute, CUdeviceptr);

PointerAttrFn pointer_attr_fn() {
    static PointerAttrFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuPointerGetAttribute", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            (void)cudaGetLastError();
            return (PointerAttrFn) nullptr;
        }
        return reinterpret_cast<PointerAttrFn>(p);
    }();
    return fn;
}
}  // namespace

void *mapped_host_range(const void *host, size_t bytes) {
    if (host == nullptr || bytes == 0) return nullptr;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, host) != cudaSuccess) {
        (void)cudaGetLastError();
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || a.devicePointer == nullptr) return nullptr;
    PointerAttrFn fn = pointer_attr_fn();
    if (fn == nullptr) return nullptr;
    CUdeviceptr start = 0;
    size_t size = 0;
    const CUdeviceptr d = reinterpret_cast<CUdeviceptr>(a.devicePointer);
    if (fn(&start, CU_POINTER_ATTRIBUTE_RANGE_START_ADDR, d) != CUDA_SUCCESS ||
        fn(&size, CU_POINTER_ATTRIBUTE_RANGE_SIZE, d) != CUDA_SUCCESS || size == 0)
        return nullptr;
    if (d < start || bytes > size || d - start > size - bytes) return nullptr;
    return a.devicePointer;
}

void *DeviceBuffer::ensure(size_t n) {
    if (n <= bytes && ptr) return ptr;
    release();
    check_injected_alloc("device buffer");
    size_t want = n < 256 ? 256 : n;
    void *p = nullptr;
    DC_CUDA(cudaMalloc(&p, want));
    ptr = p;
    bytes = want;
    return ptr;
}

void DeviceBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

void *PinnedBuffer::ensure(size_t n) {
    if (n <= bytes && ptr) return ptr;
    release();
    check_injected_alloc("pinned host buffer");
    size_t want = n < 4096 ? 4096 : n;
    void *p = nullptr;
    DC_CUDA(cudaMallocHost(&p, want));
    ptr = p;
    bytes = want;
    return ptr;
}

void PinnedBuffer::release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
}

// ---------------------------------------------------------------------------
void VolumeArray::ensure(int nx_, int ny_, int nz_, bool want_surface, int channels_) {
    if (arr && nx_ == nx && ny_ == ny && nz_ == nz && channels_ == channels && (surface || !want_surface)) return;
    release();
    check_injected_alloc("texture array");
    cudaChannelFormatDesc ch = channels_ == 2 ? cudaCreateChannelDesc<float2>() : cudaCreateChannelDesc<float>();
    channels = channels_;
    cudaExtent ext = make_cudaExtent((size_t)nx_, (size_t)ny_, (size_t)nz_);
    unsigned flags = want_surface ? cudaArraySurfaceLoadStore : cudaArrayDefault;
    DC_CUDA(cudaMalloc3DArray(&arr, &ch, ext, flags));
    nx = nx_;
    ny = ny_;
    nz = nz_;
    surface = want_surface;
    if (want_surface) {
        cudaResourceDesc rd{};
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = arr;
        DC_CUDA(cudaCreateSurfaceObject(&surf, &rd));
    }
}

cudaTextureObject_t VolumeArray::texture(float border0, float border1) {
    const std::pair<float, float> key(border0, border1);
    auto it = tex.find(key);
    if (it != tex.end()) return it->second;
    // Same sampler state as the reference (TextureClasses.cu:5-38): border
    // addressing on all axes, hardware linear filtering, unnormalised
    // coordinates, element-type reads.
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = arr;
    cudaTextureDesc td{};
    td.addressMode[0] = cudaAddressModeBorder;
    td.addressMode[1] = cudaAddressModeBorder;
    td.addressMode[2] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.borderColor[0] = border0;
    td.borderColor[1] = border1;
    td.normalizedCoords = 0;
    cudaTextureObject_t t = 0;
    DC_CUDA(cudaCreateTextureObject(&t, &rd, &td, nullptr));
    tex[key] = t;
    return t;
}

void VolumeArray::release() {
    for (auto &kv : tex) cudaDestroyTextureObject(kv.second);
    tex.clear();
    if (surf) cudaDestroySurfaceObject(surf);
    surf = 0;
    if (arr) cudaFreeArray(arr);
    arr = nullptr;
    nx = ny = nz = 0;
    surface = false;
}

// ---------------------------------------------------------------------------
DeviceContext::DeviceContext(int dev) : device(dev) {
    // DC_PHOTON_DEPTH=march|lattice sets the photon depth mode new contexts
    // start with (dc_photon_set_depth_mode changes it afterwards)
    if (const char *e = std::getenv("DC_PHOTON_DEPTH")) {
        if (std::strcmp(e, "lattice") == 0) photon_depth_mode = 1;
        if (std::strcmp(e, "march") == 0) photon_depth_mode = 0;
    }
    DC_CUDA(cudaSetDevice(dev));
    DC_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    DC_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    DC_CUDA(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
    DC_CUDA(cudaEventCreateWithFlags(&join_ev, cudaEventDisableTiming));
    DC_CUDA(cudaEventCreateWithFlags(&side_idle, cudaEventDisableTiming));
    for (auto &e : pin_ev) DC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto &e : stage_ev) DC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    DC_CUDA(cudaEventCreateWithFlags(&last_use, cudaEventDisableTiming));
}

bool DeviceContext::capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    DC_CUDA(cudaStreamIsCapturing(s, &st));
    return st != cudaStreamCaptureStatusNone;
}

void DeviceContext::begin_call(cudaStream_t s) {
    head_forked = false;  // a fork left by a call that failed midway is never joined
    if (!capturing(s)) {
        DC_CUDA(cudaStreamWaitEvent(s, last_use, 0));
        // work a call that failed midway left on the side stream is ordered
        // before this call's use of the shared scratch
        DC_CUDA(cudaEventRecord(side_idle, side));
        DC_CUDA(cudaStreamWaitEvent(s, side_idle, 0));
    }
}

void DeviceContext::end_call(cudaStream_t s) {
    if (!capturing(s)) DC_CUDA(cudaEventRecord(last_use, s));
}

DeviceContext::~DeviceContext() { release_all(); }

void DeviceContext::release_all() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    if (side) cudaStreamSynchronize(side);
    head_forked = false;
    wet_raw.release();
    vol_a.release();
    vol_b.release();
    vol_c.release();
    electron.release();
    active.release();
    xlat.release();
    xstat.release();
    head.release();
    small.release();
    lut.release();
    tables.release();
    density.release();
    terma.release();
    for (auto &b : pin_ring) b.release();
    for (auto &p : pending) {
        event_pool.push_back(p.a);
        event_pool.push_back(p.b);
    }
    pending.clear();
    for (auto e : event_pool) cudaEventDestroy(e);
    event_pool.clear();
    for (auto &e : pin_ev) {
        if (e) cudaEventDestroy(e);
        e = nullptr;
    }
    for (auto &b : stage) b.release();
    for (auto &e : stage_ev) {
        if (e) cudaEventDestroy(e);
        e = nullptr;
    }
    if (last_use) cudaEventDestroy(last_use);
    last_use = nullptr;
    for (cudaEvent_t *e : {&fork_ev, &join_ev, &side_idle}) {
        if (*e) cudaEventDestroy(*e);
        *e = nullptr;
    }
    if (side) cudaStreamDestroy(side);
    side = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
}

cudaEvent_t DeviceContext::take_event() {
    if (!event_pool.empty()) {
        cudaEvent_t e = event_pool.back();
        event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    DC_CUDA(cudaEventCreate(&e));
    return e;
}

void DeviceContext::prof_begin(const char *name, cudaStream_t s, cudaEvent_t *a, cudaEvent_t *b) {
    *a = take_event();
    *b = take_event();
    pending.push_back({name, *a, *b});
    DC_CUDA(cudaEventRecord(*a, s));
}

void DeviceContext::prof_end(cudaEvent_t b, cudaStream_t s) { cudaEventRecord(b, s); }

void DeviceContext::prof_collect() {
    DC_CUDA(cudaSetDevice(device));
    for (auto &p : pending) {
        DC_CUDA(cudaEventSynchronize(p.b));
        float ms = 0.f;
        DC_CUDA(cudaEventElapsedTime(&ms, p.a, p.b));
        auto &e = profile[p.name];
        e.launches += 1;
        e.total_ms += ms;
        event_pool.push_back(p.a);
        event_pool.push_back(p.b);
    }
    pending.clear();
}

// ---------------------------------------------------------------------------
static std::mutex g_ctx_mu;
static std::map<int, std::unique_ptr<DeviceContext>> g_ctx;

DeviceContext &context(int device) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) throw_cuda(e, "cudaGetDeviceCount");
    if (device < 0 || device >= count) {
        throw Error(DC_ERR_CUDA, std::string(cudaGetErrorString(cudaErrorInvalidDevice)) +
                                     " (gpu_id " + std::to_string(device) + " of " +
                                     std::to_string(count) + " devices)");
    }
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    auto it = g_ctx.find(device);
    if (it == g_ctx.end()) {
        it = g_ctx.emplace(device, std::unique_ptr<DeviceContext>(new DeviceContext(device))).first;
    }
    DC_CUDA(cudaSetDevice(device));
    return *it->second;
}

void release_context(int device) {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    auto it = g_ctx.find(device);
    if (it != g_ctx.end()) {
        std::lock_guard<std::mutex> lk2(it->second->mu);
        it->second->release_all();
        g_ctx.erase(it);
    }
}

// ---------------------------------------------------------------------------
// Host geometry (reference CudaBeam ctor, CudaClasses.cu:17-51; IMRTBeam ctor
// IMRTClasses.cu:30-39; gantry offset and isocentre shift dosemodule.cu:148-164).
Frame make_frame(const float iso[3], const float origin[3], double gantry_deg, double couch_deg,
                 double collimator_deg, float src_dist) {
    Frame f;
    f.isox = iso[0] - origin[0];
    f.isoy = iso[1] - origin[1];
    f.isoz = iso[2] - origin[2];
    const float gantry = fmodf((float)(gantry_deg + 180.0f), 360.0f);
    const float couch = (float)couch_deg;
    const float coll = (float)collimator_deg;
    const float ga = gantry * CUDART_PI_F / 180.0f;
    const float ta = couch * CUDART_PI_F / 180.0f;
    const float ca = coll * CUDART_PI_F / 180.0f;
    f.sga = sinf(ga);
    f.cga = cosf(ga);
    f.sta = sinf(ta);
    f.cta = cosf(ta);
    f.sca = sinf(ca);
    f.cca = cosf(ca);
    const float xg = -src_dist * f.sga;
    const float yg = src_dist * f.cga;
    f.srcx = xg * f.cta;
    f.srcy = yg;
    f.srcz = -xg * f.sta;
    return f;
}

Grid make_grid(int nz, int ny, int nx, const float spacing[3]) {
    Grid g;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.sx = spacing[0];
    g.sy = spacing[1];
    g.sz = spacing[2];
    g.inv_sx = 1.0f / g.sx;
    g.inv_sy = 1.0f / g.sy;
    g.inv_sz = 1.0f / g.sz;
    return g;
}

// ---------------------------------------------------------------------------
// Parallel host copies for pageable uploads: a few persistent worker threads
// (kept for the life of the process; they sleep between copies).
namespace {

class HostCopyPool {
   public:
    HostCopyPool() {
        const unsigned hw = std::thread::hardware_concurrency();
        n_ = std::max(1u, std::min(8u, hw / 2));
        for (unsigned t = 1; t < n_; ++t) std::thread([this, t] { worker(t); }).detach();
    }
    // dst[0, n) = src[0, n), split over the workers and the calling thread.
    void copy(void *dst, const void *src, size_t n) {
        constexpr size_t kMinPart = 256 << 10;
        unsigned parts = (unsigned)std::min<size_t>(n_, std::max<size_t>(1, n / kMinPart));
        if (parts <= 1) {
            std::memcpy(dst, src, n);
            return;
        }
        std::lock_guard<std::mutex> one_at_a_time(call_mu_);  // callers on other devices wait here
        std::unique_lock<std::mutex> lk(mu_);
        dst_ = static_cast<char *>(dst);
        src_ = static_cast<const char *>(src);
        bytes_ = n;
        parts_ = parts;
        pending_ = parts - 1;
        ++gen_;
        lk.unlock();
        cv_.notify_all();
        run_part(0);
        lk.lock();
        done_.wait(lk, [this] { return pending_ == 0; });
    }

   private:
    void run_part(unsigned t) const {
        const size_t chunk = (bytes_ + parts_ - 1) / parts_;
        const size_t b = std::min(bytes_, (size_t)t * chunk), e = std::min(bytes_, b + chunk);
        if (e > b) std::memcpy(dst_ + b, src_ + b, e - b);
    }
    void worker(unsigned t) {
        unsigned long long seen = 0;
        std::unique_lock<std::mutex> lk(mu_);
        while (true) {
            cv_.wait(lk, [&] { return gen_ != seen; });
            seen = gen_;
            if (t >= parts_) continue;
            lk.unlock();
            run_part(t);
            lk.lock();
            if (--pending_ == 0) done_.notify_one();
        }
    }
    unsigned n_ = 1;
    std::mutex call_mu_, mu_;
    std::condition_variable cv_, done_;
    unsigned long long gen_ = 0;
    char *dst_ = nullptr;
    const char *src_ = nullptr;
    size_t bytes_ = 0;
    unsigned parts_ = 0, pending_ = 0;
};

HostCopyPool &host_copy_pool() {
    static HostCopyPool *pool = new HostCopyPool();  // never destroyed: its threads run until exit
    return *pool;
}

bool page_locked(const void *p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

void upload_host_volume(DeviceContext &ctx, const float *src, int nz, int ny, int nx, VolumeArray *arr, float *lin,
                        cudaStream_t s, const std::function<void(int)> &on_slab) {
    const size_t plane = (size_t)nx * ny * sizeof(float);
    auto enqueue = [&](const float *from, int z0, int nzc) {
        if (arr) {
            cudaMemcpy3DParms p{};
            p.srcPtr = make_cudaPitchedPtr((void *)from, (size_t)nx * sizeof(float), (size_t)nx, (size_t)ny);
            p.dstArray = arr->arr;
            p.dstPos = make_cudaPos(0, 0, (size_t)z0);
            p.extent = make_cudaExtent((size_t)nx, (size_t)ny, (size_t)nzc);
            p.kind = cudaMemcpyHostToDevice;
            DC_CUDA(cudaMemcpy3DAsync(&p, s));
        } else {
            DC_CUDA(cudaMemcpyAsync(reinterpret_cast<char *>(lin) + (size_t)z0 * plane, from, (size_t)nzc * plane,
                                    cudaMemcpyHostToDevice, s));
        }
    };
    constexpr size_t kSlab = 1u << 20;  // bytes per pinned slab (at least one plane)
    const int zc = (int)std::max<size_t>(1, kSlab / plane);
    if (page_locked(src)) {
        if (!on_slab) {
            enqueue(src, 0, nz);
            return;
        }
        for (int z0 = 0; z0 < nz; z0 += zc) {
            const int n = std::min(zc, nz - z0);
            enqueue(src + (size_t)z0 * nx * ny, z0, n);
            on_slab(z0 + n);
        }
        return;
    }
    int slot = 0;
    for (int z0 = 0; z0 < nz; z0 += zc, slot = (slot + 1) % DeviceContext::kStageSlots) {
        const int n = std::min(zc, nz - z0);
        // the DMA that last read this slab must be done before it is refilled
        DC_CUDA(cudaEventSynchronize(ctx.stage_ev[slot]));
        char *pin = static_cast<char *>(ctx.stage[slot].ensure((size_t)zc * plane));
        host_copy_pool().copy(pin, reinterpret_cast<const char *>(src) + (size_t)z0 * plane, (size_t)n * plane);
        enqueue(reinterpret_cast<const float *>(pin), z0, n);
        DC_CUDA(cudaEventRecord(ctx.stage_ev[slot], s));
        if (on_slab) on_slab(z0 + n);
    }
}

}  // namespace dc
