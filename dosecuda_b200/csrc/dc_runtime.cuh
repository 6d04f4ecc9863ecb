// dc_runtime.cuh — per-device runtime of the DoseCUDA B200 engines.
//
// The reference allocates, uploads and frees everything on every call
// (MemoryClasses.h:85-137, TextureClasses.cu:44-59).  Here each device gets
// one long-lived context holding:
//  * a non-blocking stream for the synchronous host entry points;
//  * grow-only device buffers (WET, dose, TERMA, spot/layer tables, LUTs);
//  * grow-only 3D cudaArrays with texture objects (hardware trilinear
//    filtering, border addressing) and, for the TERMA volume, a surface
//    object so that the TERMA kernel writes the array directly;
//  * a small kernel profiler (CUDA events per launch, opt-in).
// Calls on one device are serialised by the context mutex.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "../../include/dosecuda.h"

#include <functional>
#include <map>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

namespace dc {

// Error carrying the C-ABI status code.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] void throw_cuda(cudaError_t e, const char *what);

inline void cuda_check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw_cuda(e, what);
}
#define DC_CUDA(call) ::dc::cuda_check((call), #call)

void set_last_error(const std::string &msg);

// Runs fn and maps what it throws onto the C-ABI status codes (the message
// goes to dc_last_error): Error -> its code, std::bad_alloc ->
// DC_ERR_MEMORY, anything else -> DC_ERR_CUDA.
template <class F>
int guarded(F &&fn) {
    try {
        fn();
        set_last_error("");
        return DC_OK;
    } catch (const Error &e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc &) {
        set_last_error("Not enough host memory");
        return DC_ERR_MEMORY;
    } catch (const std::exception &e) {
        set_last_error(e.what());
        return DC_ERR_CUDA;
    }
}

// Grow-only device allocation.
struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    void *ensure(size_t n);
    void release();
    template <class T>
    T *as() const { return static_cast<T *>(ptr); }
};

// Grow-only pinned host allocation.
struct PinnedBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    void *ensure(size_t n);
    void release();
};

// A 3D float cudaArray (1 or 2 channels) with linear-filter texture objects
// for a set of border values, and optionally a surface object.
struct VolumeArray {
    cudaArray_t arr = nullptr;
    int nx = 0, ny = 0, nz = 0;
    int channels = 1;
    bool surface = false;
    cudaSurfaceObject_t surf = 0;
    std::map<std::pair<float, float>, cudaTextureObject_t> tex;  // border values -> texture

    // (Re)allocate for the given extent; keeps the array when it matches.
    void ensure(int nx_, int ny_, int nz_, bool want_surface, int channels_ = 1);
    cudaTextureObject_t texture(float border0, float border1 = 0.0f);
    void release();
};

struct ProfileEntry {
    int launches = 0;
    double total_ms = 0.0;
};

class DeviceContext {
   public:
    explicit DeviceContext(int device);
    ~DeviceContext();

    int device;
    std::mutex mu;
    cudaStream_t stream = nullptr;  // for the host (synchronous) entry points
    // Side stream for work that runs beside a call's own stream: forked after
    // fork_ev (recorded on the call's stream), joined through join_ev.
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr, side_idle = nullptr;
    bool head_forked = false;  // photon head factors enqueued on `side`, not yet joined

    DeviceBuffer wet_raw;     // unsmoothed WET (cm)
    DeviceBuffer vol_a;       // generic volume scratch (input staging)
    DeviceBuffer vol_b;       // generic volume scratch (output)
    DeviceBuffer vol_c;       // generic volume scratch (second output)
    DeviceBuffer electron;    // electron contamination term
    DeviceBuffer active;      // CCCS active-voxel list (count in the first 256 B)
    DeviceBuffer small;       // per-call small device tables (cone directions)
    DeviceBuffer lut;         // proton LUT rows uploaded by the host entry point
    DeviceBuffer tables;      // proton layer + spot tables
    DeviceBuffer xlat;        // photon ray-lattice integrals G[node][ray] (dc_xray.cu)
    DeviceBuffer xstat;       // voxels the last photon depth pass marched exactly
    DeviceBuffer head;        // photon head factors (tp, ts, oaf, soft) per voxel, float4
    VolumeArray density;      // density / RLSP texture
    VolumeArray terma;        // TERMA texture (surface-writable)
    // Photon radiological depth: 0 = the reference's per-voxel 1 mm march,
    // 1 = the beam's-eye-view ray lattice (dc_xray.cu).  Set by
    // dc_photon_set_depth_mode; read when a photon call is enqueued.
    int photon_depth_mode = 1;
    // Ring of pinned staging slots for per-call tables: the host reuses a slot
    // only after the copy out of it (event) has completed.
    static constexpr int kPinSlots = 4;
    PinnedBuffer pin_ring[kPinSlots];
    cudaEvent_t pin_ev[kPinSlots] = {};
    int pin_next = 0;
    // Ring of pinned slabs for uploading pageable host volumes
    // (upload_host_volume): a slab is rewritten only after the copy out of it
    // (event) has completed.
    static constexpr int kStageSlots = 3;
    PinnedBuffer stage[kStageSlots];
    cudaEvent_t stage_ev[kStageSlots] = {};
    cudaEvent_t last_use = nullptr;  // recorded after the last enqueued call

    // Orders a call on stream s after every earlier call on this device
    // (the cached scratch buffers are shared), and marks its end.  While s is
    // being captured into a CUDA graph the graph's own edges order the work,
    // so neither the wait nor the record is issued (nor profiler events).
    void begin_call(cudaStream_t s);
    void end_call(cudaStream_t s);
    static bool capturing(cudaStream_t s);

    // Profiler.
    bool profiling = false;
    struct Pending {
        std::string name;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> event_pool;
    std::map<std::string, ProfileEntry> profile;
    void prof_begin(const char *name, cudaStream_t s, cudaEvent_t *a, cudaEvent_t *b);
    void prof_end(cudaEvent_t b, cudaStream_t s);
    void prof_collect();  // synchronises the device
    void release_all();

   private:
    cudaEvent_t take_event();
};

// Returns the context for `device` (created on first use) with the device
// made current.  Throws Error(DC_ERR_CUDA) for an invalid ordinal, as the
// reference's cudaSetDevice failure surfaces as a CUDA error.
DeviceContext &context(int device);
void release_context(int device);

// RAII bracket for a profiled kernel launch on stream s: an NVTX range (the
// host-side enqueue, visible to any NVTX-aware tracer) and, when the
// profiler is enabled, CUDA events around the kernel.
struct KernelTimer {
    DeviceContext &ctx;
    cudaStream_t s;
    cudaEvent_t a = nullptr, b = nullptr;
    KernelTimer(DeviceContext &c, const char *name, cudaStream_t st) : ctx(c), s(st) {
        nvtxRangePushA(name);
        if (ctx.profiling && !DeviceContext::capturing(s)) ctx.prof_begin(name, s, &a, &b);
    }
    ~KernelTimer() {
        if (b) ctx.prof_end(b, s);
        nvtxRangePop();
    }
};

// Throws the injected out-of-memory when DC_INJECT_ALLOC_FAIL selects this
// allocation (see dc_runtime.cu).
void check_injected_alloc(const char *what);

// Device address through which kernels on the current device may store into
// the caller's host buffer [host, host + bytes) directly, or nullptr: the
// buffer must be page-locked host memory mapped into the device's address
// space (cudaHostAlloc / cudaHostRegister, e.g. torch's pinned allocator),
// and the whole range must lie inside the one allocation.  Results written
// this way cross the bus while the kernel runs instead of in a copy after it.
void *mapped_host_range(const void *host, size_t bytes);

// Host volume (nz, ny, nx floats) -> the cudaArray `arr` or, when `arr` is
// null, the linear device buffer `lin`, enqueued on s.  A page-locked source
// is copied directly.  A pageable one is pipelined through the context's
// pinned slabs: host threads copy slab c into a pinned buffer while the DMA
// of slab c-1 runs, instead of the driver staging the whole volume serially.
// With `on_slab`, the copy goes in slabs either way and on_slab(z) is called
// after each slab's copy is enqueued, z = the planes enqueued so far, so that
// the caller can enqueue work on those planes behind it.
void upload_host_volume(DeviceContext &ctx, const float *src, int nz, int ny, int nx, VolumeArray *arr, float *lin,
                        cudaStream_t s, const std::function<void(int)> &on_slab = nullptr);

// Throws Error(DC_ERR_CUDA) if the last launch failed.
void check_launch(const char *kernel);

}  // namespace dc
