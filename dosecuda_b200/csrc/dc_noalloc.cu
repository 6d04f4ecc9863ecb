// dc_noalloc.cu — proton WET ray trace that allocates nothing.
//
// For callers that cannot let a library call cudaMalloc: host applications
// (treatment-planning systems, optimisers) that own every device allocation
// and hand the library pre-allocated buffers; callers working inside a fixed
// device-memory budget, where an allocation the library makes on its own could
// fail mid-run; and latency-sensitive loops where the implicit device-wide
// synchronisation of cudaMalloc/cudaFree would stall the caller's other
// streams.  dc_proton_raytrace_noalloc does the same work as
// dc_proton_raytrace_dev — the 1 mm ray march to the source followed by the
// beam's-eye-view smoothing — but:
//  * its only scratch, the unsmoothed WET volume, is the file-scope device
//    array g_noalloc_wet below (kNoAllocMaxVoxels floats = 16 MiB).  CUDA
//    commits it on a device when the library's device code is loaded there,
//    which with lazy module loading (the CUDA 12 default) is the first call of
//    this entry point on that device; from then on the device holds it until
//    the process exits.  That first call can therefore fail with an
//    out-of-memory status on a full device, and should come before any stream
//    capture;
//  * it samples the caller's linear RLSP buffer with its own trilinear
//    interpolation (border value 0, interpolation weights rounded to 1/256
//    as the texture unit does) instead of building a cudaArray and a
//    texture object, so its WET can differ from the texture path by
//    rounding of the weights (a few 1e-4 cm);
//  * it creates no stream, event or context state: the kernels go on the
//    caller's stream, and the caller's current device is restored on return.
// The host code never dereferences g_noalloc_wet (in host code the name is
// only a stand-in, not a device address): the first call in each CUDA context
// looks up the array's device address with cudaGetSymbolAddress, with that
// device current, and every call passes that pointer to the kernels.  The
// lookup is keyed by the context's unique id, so a device reset
// (cudaDeviceReset, which replaces the context and may move the array) makes
// the next call look it up again.  The march writes every voxel of the
// scratch it uses before the smoothing reads it, so nothing needs clearing
// between calls.
#include <cmath>
#include <cuda.h>
#include <mutex>
#include <string>

#include "../../include/dosecuda.h"
#include "dc_common.cuh"
#include "dc_runtime.cuh"

namespace dc {

// Reference smoothing kernel (dc_wet.cu), reused unchanged.
__global__ void wet_smooth_kernel(Grid g, Frame f, const float *__restrict__ wet, float *__restrict__ wet_s);

constexpr long long kNoAllocMaxVoxels = 4LL << 20;  // 4,194,304 voxels

DC_BOUNDS_WORD

// Unsmoothed WET of the last call.  Every call overwrites the voxels it uses
// before reading them; calls that overlap on the GPU (two streams, two host
// threads) share this array and race.
static __device__ __align__(256) float g_noalloc_wet[kNoAllocMaxVoxels];

// Trilinear fetch from a linear (nz, ny, nx) volume at unnormalised texel
// coordinates, border value 0 — the filtering the texture unit applies
// (coordinate - 0.5, 8-bit fractional weights).
__device__ __forceinline__ float linear_fetch(const float *__restrict__ v, const Grid &g, float3 t) {
    const float x = t.x - 0.5f, y = t.y - 0.5f, z = t.z - 0.5f;
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const int i0 = (int)fx, j0 = (int)fy, k0 = (int)fz;
    const float a = rintf((x - fx) * 256.0f) * (1.0f / 256.0f);
    const float b = rintf((y - fy) * 256.0f) * (1.0f / 256.0f);
    const float c = rintf((z - fz) * 256.0f) * (1.0f / 256.0f);
    float r = 0.0f;
#pragma unroll
    for (int dk = 0; dk < 2; ++dk) {
        const int k = k0 + dk;
        const float wz = dk ? c : 1.0f - c;
#pragma unroll
        for (int dj = 0; dj < 2; ++dj) {
            const int j = j0 + dj;
            const float wyz = (dj ? b : 1.0f - b) * wz;
#pragma unroll
            for (int di = 0; di < 2; ++di) {
                const int i = i0 + di;
                const float w = (di ? a : 1.0f - a) * wyz;
                if ((unsigned)i < (unsigned)g.nx && (unsigned)j < (unsigned)g.ny && (unsigned)k < (unsigned)g.nz) {
                    const long long idx = (long long)i + (long long)g.nx * (j + (long long)g.ny * k);
                    if (DC_IN_BOUNDS(idx, g.n(), 1)) r = fmaf(w, __ldg(v + idx), r);
                }
            }
        }
    }
    return r;
}

// The ray march of wet_march_kernel with linear_fetch in place of tex3D.
__global__ void __launch_bounds__(128) wet_march_linear_kernel(Grid g, Frame f, const float *__restrict__ rho,
                                                               float *__restrict__ wet) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const float3 p = voxel_xyz(g, f, i, j, k);
    const float3 u = unit_to_source(f, p);
    float wet_sum = -0.05f;
    float t = 0.0f;
    while (true) {
        float3 q;
        q.x = fmaf(u.x, t, p.x);
        q.y = fmaf(u.y, t, p.y);
        q.z = fmaf(u.z, t, p.z);
        const float3 tc = tex_coord(g, f, q);
        if (!tex_inside(g, tc)) break;
        wet_sum = fmaf(fmaxf(linear_fetch(rho, g, tc), 0.0f), 0.1f, wet_sum);
        t += 1.0f;
    }
    const long long v = (long long)i + (long long)g.nx * (j + (long long)g.ny * k);
    if (DC_IN_BOUNDS(v, kNoAllocMaxVoxels, 2)) wet[v] = wet_sum;
}

DC_BOUNDS_TAKE(take_bounds_noalloc)

namespace {

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_symbol_mu;
struct SymbolCache {
    unsigned long long ctx_id = 0;  // unique id of the context the address belongs to (0: none)
    float *ptr = nullptr;
};
SymbolCache g_symbol[kNoAllocMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

template <class Fn>
Fn driver_entry(const char *name) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess) {
        (void)cudaGetLastError();
        return nullptr;
    }
    return reinterpret_cast<Fn>(p);
}

// Unique id of the calling thread's current CUDA context (made current by the
// runtime call before this one).  Ids are never reused within a process, so a
// context created after a device reset gets a new one.
unsigned long long current_context_id() {
    static const CtxGetCurrentFn get_current = driver_entry<CtxGetCurrentFn>("cuCtxGetCurrent");
    static const CtxGetIdFn get_id = driver_entry<CtxGetIdFn>("cuCtxGetId");
    if (!get_current || !get_id) throw Error(DC_ERR_CUDA, "cuCtxGetCurrent/cuCtxGetId unavailable in this driver");
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current(&c) != CUDA_SUCCESS || c == nullptr || get_id(c, &id) != CUDA_SUCCESS)
        throw Error(DC_ERR_CUDA, "no current CUDA context after cudaSetDevice");
    return id;
}

// Device address of g_noalloc_wet in the current context of device `dev`,
// looked up once per context.
float *scratch_for(int dev) {
    // cudaSetDevice (CUDA 12 and later) has made the device's primary context
    // current on this thread.
    const unsigned long long id = current_context_id();
    std::lock_guard<std::mutex> lk(g_symbol_mu);
    SymbolCache &c = g_symbol[dev];
    if (c.ptr == nullptr || c.ctx_id != id) {
        float *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_wet);
        if (e != cudaSuccess) throw_cuda(e, "cudaGetSymbolAddress(g_noalloc_wet)");
        c.ptr = p;
        c.ctx_id = id;
    }
    return c.ptr;
}

// Restores the calling thread's current device when the entry point returns.
struct CurrentDeviceGuard {
    int saved = -1;
    CurrentDeviceGuard() {
        if (cudaGetDevice(&saved) != cudaSuccess) {
            (void)cudaGetLastError();
            saved = -1;
        }
    }
    ~CurrentDeviceGuard() {
        if (saved >= 0) (void)cudaSetDevice(saved);
    }
};

int fail(int code, const std::string &msg) {
    set_last_error(msg);
    return code;
}

}  // namespace
}  // namespace dc

extern "C" int dc_proton_raytrace_noalloc(int gpu_id, const float *rlsp_dev, int nz, int ny, int nx,
                                          const float spacing[3], const float origin[3], const float iso[3],
                                          double gantry_deg, float couch_deg, float vsadx, float vsady,
                                          float *wet_out_dev, void *stream) {
    using namespace dc;
    if (!rlsp_dev || !wet_out_dev || !spacing || !origin || !iso)
        return fail(DC_ERR_VALUE, "dc_proton_raytrace_noalloc: NULL argument.");
    if (nz <= 0 || ny <= 0 || nx <= 0) return fail(DC_ERR_VALUE, "'voxel_data' must have positive dimensions.");
    const long long n = (long long)nz * ny * nx;
    if (n > kNoAllocMaxVoxels)
        return fail(DC_ERR_VALUE, "volume of " + std::to_string(n) + " voxels exceeds the no-allocation scratch limit "
                                  "of " + std::to_string(kNoAllocMaxVoxels) + " voxels.");
    for (int a = 0; a < 3; ++a)
        if (!(std::isfinite(spacing[a]) && spacing[a] > 0.0f) || !std::isfinite(origin[a]))
            return fail(DC_ERR_VALUE, "'spacing' must be positive and 'origin' finite.");
    if (!(std::isfinite(vsadx) && std::isfinite(vsady) && vsadx != 0.0f && vsady != 0.0f))
        return fail(DC_ERR_VALUE, "'VSADX' and 'VSADY' must be finite and non-zero.");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) return fail(DC_ERR_CUDA, cudaGetErrorString(e));
    if (gpu_id < 0 || gpu_id >= count || gpu_id >= kNoAllocMaxDevices)
        return fail(DC_ERR_CUDA, cudaGetErrorString(cudaErrorInvalidDevice));
    CurrentDeviceGuard keep_device;
    try {
        DC_CUDA(cudaSetDevice(gpu_id));
        float *scratch = scratch_for(gpu_id);
        const Grid g = make_grid(nz, ny, nx, spacing);
        const Frame f = make_frame(iso, origin, gantry_deg, couch_deg, 0.0, (vsadx + vsady) / 2.0f);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        const dim3 grid((unsigned)((nx + 31) / 32), (unsigned)((ny + 3) / 4), (unsigned)nz), block(32, 4, 1);
        wet_march_linear_kernel<<<grid, block, 0, s>>>(g, f, rlsp_dev, scratch);
        check_launch("wet_march_linear_kernel");
        wet_smooth_kernel<<<grid, block, 0, s>>>(g, f, scratch, wet_out_dev);
        check_launch("wet_smooth_kernel");
    } catch (const Error &err) {
        return fail(err.code, err.what());
    }
    return DC_OK;
}
