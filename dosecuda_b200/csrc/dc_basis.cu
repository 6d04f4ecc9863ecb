// dc_basis.cu — a linear dose basis on the device: combination and adjoint.
//
// A photon beam's plan dose is linear in the weights of its control points
// (segments): D(w) = sum_b w_b OF_b D_b, with D_b the CCCS dose of control
// point b and OF_b its output factor (plan_imrt.py:140-156 accumulates
// exactly these terms with w = 1).  With the per-control-point doses kept on
// the device as a basis, the plan dose for any segment weights is one
// combination pass and the gradient of an objective f(D) with respect to the
// weights is the adjoint  df/dw_b = OF_b sum_v g_v D_b[v],  g = df/dD.
//
// basis_combine_kernel: one thread per voxel walks the basis in order with
//   acc = float32(double(acc) + double(D_b[v]) * coef_b),
// numpy's float32 += float32 * float64 of the reference's plan loop, so with
// coef = OF the result equals the control-point loop bit for bit.  Bound by
// HBM: n_basis * 4 B read + 4 B read/write per voxel.
//
// basis_adjoint_kernel: blocks tile (voxel chunk, basis); each thread sums
// g_v * D_b[v] in float64 over a strided voxel range, a warp and block
// reduction follows, and one float64 atomic per block adds into grad_b.
// Bound by HBM (the basis is read once; g stays in L2 across the bases).
#include <algorithm>

#include "../../include/dosecuda.h"
#include "dc_common.cuh"
#include "dc_runtime.cuh"

namespace dc {

DC_BOUNDS_WORD

namespace {

constexpr int kBasisThreads = 256;

void need(bool ok, const char *msg) {
    if (!ok) throw Error(DC_ERR_VALUE, msg);
}

cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

__global__ void __launch_bounds__(kBasisThreads) basis_combine_kernel(const float *__restrict__ basis, int n_basis,
                                                                      long long n, const double *__restrict__ coef,
                                                                      float *__restrict__ out) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x) {
        float acc = out[v];
        for (int b = 0; b < n_basis; ++b) {
            const long long u = (long long)b * n + v;
            acc = __double2float_rn(__dadd_rn((double)acc, __dmul_rn(DC_IN_BOUNDS(u, (long long)n_basis * n, 30)
                                                                          ? (double)__ldg(basis + u)
                                                                          : 0.0,
                                                                      __ldg(coef + b))));
        }
        out[v] = acc;
    }
}

__global__ void __launch_bounds__(kBasisThreads) basis_adjoint_kernel(const float *__restrict__ basis, long long n,
                                                                      const float *__restrict__ g,
                                                                      double *__restrict__ grad) {
    const int b = blockIdx.y;
    const float *d = basis + (long long)b * n;
    double s = 0.0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
        s = fma((double)__ldg(g + v), (double)__ldg(d + v), s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    __shared__ double s_part[kBasisThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_part[warp] = s;
    __syncthreads();
    if (warp == 0) {
        s = lane < kBasisThreads / 32 ? s_part[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0 && s != 0.0) atomicAdd(grad + b, s);
    }
}

void check_basis(const float *basis, int n_basis, long long n_vox) {
    need(basis != nullptr, "the basis must not be NULL.");
    need(n_basis >= 1 && n_basis <= 65535, "the basis must hold 1 to 65535 volumes.");
    need(n_vox >= 1, "the basis volumes must hold at least one voxel.");
}

}  // namespace

DC_BOUNDS_TAKE(take_bounds_basis)

}  // namespace dc

extern "C" {

int dc_basis_combine_dev(int gpu_id, const float *basis, int n_basis, long long n_vox, const double *coef_dev,
                         float *out_dev, void *stream) {
    using namespace dc;
    return guarded([&] {
        check_basis(basis, n_basis, n_vox);
        need(coef_dev != nullptr && out_dev != nullptr, "coefficients and output must not be NULL.");
        DeviceContext &ctx = context(gpu_id);
        cudaStream_t s = as_stream(stream);
        int sms = 0;
        DC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
        const long long blocks = std::min<long long>((n_vox + kBasisThreads - 1) / kBasisThreads, (long long)sms * 8);
        KernelTimer kt(ctx, "basis_combine", s);
        basis_combine_kernel<<<(unsigned)blocks, kBasisThreads, 0, s>>>(basis, n_basis, n_vox, coef_dev, out_dev);
        check_launch("basis_combine_kernel");
    });
}

int dc_basis_adjoint_dev(int gpu_id, const float *basis, int n_basis, long long n_vox, const float *grad_dose_dev,
                         double *grad_out_dev, void *stream) {
    using namespace dc;
    return guarded([&] {
        check_basis(basis, n_basis, n_vox);
        need(grad_dose_dev != nullptr && grad_out_dev != nullptr, "gradient buffers must not be NULL.");
        DeviceContext &ctx = context(gpu_id);
        cudaStream_t s = as_stream(stream);
        int sms = 0;
        DC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
        // enough (chunk, basis) blocks for a few waves; each chunk strides the volume
        const long long per_basis = std::max<long long>(
            1, std::min<long long>((n_vox + kBasisThreads - 1) / kBasisThreads, ((long long)sms * 8 + n_basis - 1) / n_basis));
        DC_CUDA(cudaMemsetAsync(grad_out_dev, 0, sizeof(double) * (size_t)n_basis, s));
        KernelTimer kt(ctx, "basis_adjoint", s);
        basis_adjoint_kernel<<<dim3((unsigned)per_basis, (unsigned)n_basis), kBasisThreads, 0, s>>>(basis, n_vox,
                                                                                                   grad_dose_dev,
                                                                                                   grad_out_dev);
        check_launch("basis_adjoint_kernel");
    });
}

}  // extern "C"
