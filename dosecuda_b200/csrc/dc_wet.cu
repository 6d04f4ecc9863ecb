// dc_wet.cu — radiological depth: per-voxel ray march to the source and the
// proton beam's-eye-view smoothing.
//
// wet_march_kernel restates rayTraceKernel (CudaClasses.cu:180-228): from
// each voxel centre, 1 mm steps towards the source, hardware-trilinear
// density samples, WET(cm) = -0.05 + sum 0.1*max(rho,0) until the sample's
// texture coordinate leaves [0,n).  wet_smooth_kernel restates
// smoothRayKernel (IMPTClasses.cu:139-202): the mean of the voxel's WET and
// the nearest-voxel WET at radii 1,2,.. mm (r < min(10*WET, 10)) along six
// BEV directions.
//
// B200 mapping: one thread per voxel with a warp covering 32 consecutive x
// voxels (coalesced loads/stores; the 32 rays of a warp march side by side so
// their texture samples share cache lines), blocks of 32x4 voxels.  The march
// is bound by the texture unit's trilinear fetch rate, one fetch per 1 mm
// sample.  The smoothing's nearest-voxel lookups avoid the IEEE division and
// float-to-int conversion on the special-function unit wherever the result
// is provably the same (nearest_index), which leaves it bound by issue and
// gather latency.
#include "dc_common.cuh"
#include "dc_runtime.cuh"
#include "dc_kernels.cuh"

namespace dc {

DC_BOUNDS_WORD

__global__ void __launch_bounds__(128) wet_march_kernel(Grid g, Frame f, cudaTextureObject_t density,
                                                        float *__restrict__ wet) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;

    const float3 p = voxel_xyz(g, f, i, j, k);
    const float3 u = unit_to_source(f, p);

    float wet_sum = -0.05f;
    float t = 0.0f;
    // The samples inside the volume form a prefix of t = 0,1,2,... (each
    // coordinate is monotonic in t), so the loop stops at the first exit.
    while (true) {
        float3 q;
        q.x = fmaf(u.x, t, p.x);
        q.y = fmaf(u.y, t, p.y);
        q.z = fmaf(u.z, t, p.z);
        const float3 tc = tex_coord(g, f, q);
        if (!tex_inside(g, tc)) break;
        const float rho = tex3D<float>(density, tc.x, tc.y, tc.z);
        wet_sum = fmaf(fmaxf(rho, 0.0f), 0.1f, wet_sum);
        t += 1.0f;
    }
    const long long v = (long long)i + (long long)g.nx * (j + (long long)g.ny * k);
    if (DC_IN_BOUNDS(v, g.n(), 1)) wet[v] = wet_sum;
}

// Nearest voxel index (int)roundf(v / s) of the reference's smoothing
// (CudaClasses.cuh:112-116: IEEE division, then round half away from zero),
// without the division and the float-to-int conversion on the common path.
// With r = RN(1/s), qa = RN(v * r) differs from Q = RN(v / s) by less than
// |qa| * 2^-22 (two relative roundings of 2^-24 each on r and qa, one on Q).
// When no half-integer lies within |qa| * 2^-21 of qa, Q and qa round to the
// same integer, which the magic-number addition (1.5 * 2^23, exact for
// |qa| < 2^21) delivers as bits of a float.  Otherwise — and for inf/NaN —
// the reference's expression itself is evaluated, so the index is always
// exactly the reference's.
__device__ __forceinline__ int nearest_index(float v, float s, float r) {
    const float magic = 12582912.0f;  // 1.5 * 2^23
    const float qa = __fmul_rn(v, r);
    const float t = __fadd_rn(qa, magic);
    const float d = fabsf(__fsub_rn(qa, __fsub_rn(t, magic)));  // distance to the nearest integer
    const float aq = fabsf(qa);
    if (aq < 2097152.0f && __fsub_rn(0.5f, d) > __fmul_rn(aq, 4.76837158203125e-07f)) {  // 2^-21
        return __float_as_int(t) - 0x4B400000;
    }
    return (int)roundf(v / s);
}

__global__ void __launch_bounds__(128) wet_smooth_kernel(Grid g, Frame f, const float *__restrict__ wet,
                                                         float *__restrict__ wet_s) {
    // The six direction cosines/sines, evaluated once per block with the same
    // call the per-voxel loop used to make (identical values).
    __shared__ float s_dir[2][6];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (tid < 6) sincosf((float)tid * CUDART_PI_F / 3.0f, &s_dir[0][tid], &s_dir[1][tid]);
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;

    const long long v = (long long)i + (long long)g.nx * (j + (long long)g.ny * k);
    const float3 p = voxel_xyz(g, f, i, j, k);
    const float3 h = image_to_head<false>(f, p);
    const float c = DC_IN_BOUNDS(v, g.n(), 2) ? __ldg(wet + v) : 0.0f;
    const float rmax = c * 10.0f;
    const float rsx = 1.0f / g.sx, rsy = 1.0f / g.sy, rsz = 1.0f / g.sz;
    float sum = c;
    int n = 1;
    for (int d = 0; d < 6; ++d) {
        const float s = s_dir[0][d], co = s_dir[1][d];
        for (float dr = 1.0f; dr < rmax && dr < 10.0f; dr += 1.0f) {
            float3 hc = make_float3(h.x + dr * co, h.y + dr * s, h.z);
            const float3 q = head_to_image<false>(f, hc);
            // Nearest voxel (CudaClasses.cuh:112-116).
            const int qi = nearest_index(q.x + f.isox, g.sx, rsx);
            const int qj = nearest_index(q.y + f.isoy, g.sy, rsy);
            const int qk = nearest_index(q.z + f.isoz, g.sz, rsz);
            if ((unsigned)qi < (unsigned)g.nx && (unsigned)qj < (unsigned)g.ny &&
                (unsigned)qk < (unsigned)g.nz) {
                const long long u = (long long)qi + (long long)g.nx * (qj + (long long)g.ny * qk);
                sum += DC_IN_BOUNDS(u, g.n(), 3) ? __ldg(wet + u) : 0.0f;
                n += 1;
            }
        }
    }
    if (DC_IN_BOUNDS(v, g.n(), 2)) wet_s[v] = sum / (float)n;
}

static dim3 volume_grid(const Grid &g) {
    return dim3((unsigned)((g.nx + 31) / 32), (unsigned)((g.ny + 3) / 4), (unsigned)g.nz);
}

DC_BOUNDS_TAKE(take_bounds_wet)

void launch_wet_march(DeviceContext &ctx, const Grid &g, const Frame &f, cudaTextureObject_t density,
                      float *wet, cudaStream_t s) {
    KernelTimer kt(ctx, "wet_march", s);
    wet_march_kernel<<<volume_grid(g), dim3(32, 4, 1), 0, s>>>(g, f, density, wet);
    check_launch("wet_march_kernel");
}

void launch_wet_smooth(DeviceContext &ctx, const Grid &g, const Frame &f, const float *wet, float *wet_s,
                       cudaStream_t s) {
    KernelTimer kt(ctx, "wet_smooth", s);
    wet_smooth_kernel<<<volume_grid(g), dim3(32, 4, 1), 0, s>>>(g, f, wet, wet_s);
    check_launch("wet_smooth_kernel");
}

}  // namespace dc
