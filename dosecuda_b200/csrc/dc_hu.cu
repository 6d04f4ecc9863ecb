// dc_hu.cu — HU -> relative stopping power / relative density on the device.
//
// The reference converts on the host with np.interp over the machine's
// HU_RLSP.csv / HU_Density.csv tables and casts the float64 result to float32
// (plan_impt.py:112-122, plan_imrt.py:114-124).  This kernel restates the
// same piecewise-linear interpolation in float64 with every operation
// explicitly rounded (no fused multiply-add), so its float32 result is the
// host's bit for bit, and it can write straight into the ray tracer's texture
// array (surface store), which removes the host O(N) pass and the per-call
// upload of the converted volume.
#include "dc_kernels.cuh"
#include "dc_runtime.cuh"

namespace dc {

// np.interp for a strictly increasing table: x below the first point gives
// the first value, at or above the last point the last value, on a
// breakpoint that point's value, else the linear interpolation
// slope*(x - xp[j]) + fp[j] with slope = (fp[j+1]-fp[j])/(xp[j+1]-xp[j]).
__device__ __forceinline__ float hu_interp(const HuTable &t, float hu) {
    const double x = (double)hu;
    if (x != x) return __double2float_rn(x);  // NaN stays NaN
    const int n = t.n;
    if (x < t.hu[0]) return __double2float_rn(t.val[0]);
    if (x >= t.hu[n - 1]) return __double2float_rn(t.val[n - 1]);
    int lo = 0, hi = n - 1;  // largest j with hu[j] <= x, j < n-1
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (t.hu[mid] <= x) lo = mid;
        else hi = mid;
    }
    const int j = lo;
    if (t.hu[j] == x) return __double2float_rn(t.val[j]);
    const double slope = __ddiv_rn(__dsub_rn(t.val[j + 1], t.val[j]), __dsub_rn(t.hu[j + 1], t.hu[j]));
    return __double2float_rn(__dadd_rn(__dmul_rn(slope, __dsub_rn(x, t.hu[j])), t.val[j]));
}

__global__ void __launch_bounds__(128) hu_convert_kernel(const float *__restrict__ hu, int nx, int ny, int nz,
                                                         HuTable t, float *__restrict__ out,
                                                         cudaSurfaceObject_t surf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= nx || j >= ny || k >= nz) return;
    const long long v = (long long)i + (long long)nx * (j + (long long)ny * k);
    const float r = hu_interp(t, __ldg(hu + v));
    if (out) out[v] = r;
    if (surf) surf3Dwrite(r, surf, i * (int)sizeof(float), j, k);
}

void launch_hu_convert(const HuTable &t, const float *hu, int nx, int ny, int nz, float *out, cudaSurfaceObject_t surf,
                       cudaStream_t s) {
    const dim3 grid((unsigned)((nx + 31) / 32), (unsigned)((ny + 3) / 4), (unsigned)nz);
    hu_convert_kernel<<<grid, dim3(32, 4, 1), 0, s>>>(hu, nx, ny, nz, t, out, surf);
    check_launch("hu_convert_kernel");
}

}  // namespace dc
