// dc_fluence.cu — photon dose as a function of a beamlet fluence map, and
// its adjoint (the transpose of the collapsed-cone superposition).
//
// The reference's photon dose of one control point (IMRTClasses.cu:209-350)
// is linear in its TERMA and electron volumes: the CCCS sums, per voxel, 72
// cone directions of the backward recursions
//     Rp <- Rp e_m + T_m cp (1 - e_m),   Rs <- Rs (1 - b D_m) + T_m D_m cs,
// whose coefficients depend on the density samples only.  A fluence map F on
// a beam's-eye-view grid of beamlets (head frame, isocentre plane) scales
// both volumes voxel by voxel with its bilinear interpolation at the voxel's
// ray, m(v) = sum_q w_q(v) F_q, so the dose is linear in F:
//     D = s (K diag(m) T0 + diag(m) E0)   on the voxels with T0 > 0.01
// (the reference's TERMA mask, held fixed at the unmodulated TERMA).
//
//  * fluence_modulate_kernel writes m T0 into the CCCS's (TERMA, density)
//    array and m E0 into the electron term; the
//    unchanged CCCS kernel then gives D.  F = 1 gives T0 and E0 bit for bit.
//  * cccs_adjoint_kernel computes h = s K^T g: per voxel p with g(p) != 0
//    and per direction, the recursion's sensitivity to each sample's TERMA,
//    dD/dT_m = a cp (1 - e_m) prod_{nearer} e + b cs D_m prod_{nearer}(1 - b D),
//    evaluated from the voxel outwards, is scattered onto the sample's eight
//    texels with the texture unit's interpolation weights (float atomics).
//  * fluence_grad_kernel reduces T0 h + s E0 g over each beamlet's bilinear
//    footprint (per-block shared-memory sums, one float64 atomic per block and
//    beamlet).
#include <algorithm>
#include <cmath>

#include "dc_common.cuh"
#include "dc_kernels.cuh"
#include "dc_photon.cuh"
#include "dc_runtime.cuh"

namespace dc {

DC_BOUNDS_WORD

namespace {

constexpr int kMaxSmemBeamlets = 4096;  // float64 beamlet sums kept in shared memory per block

// Bilinear weights of the fluence map at the voxel's beam's-eye-view position
// (clamped to the map's edge, so that a constant map gives that constant).
__device__ __forceinline__ void fluence_taps(const FluenceMap &M, const Frame &f, float3 p, int idx[4], float w[4],
                                             float *wa_out = nullptr, float *wb_out = nullptr) {
    const float3 h = image_to_head<true>(f, p);
    const float den = M.sad - h.z;
    float ua = (h.x * M.sad / den - M.a0) * M.inv_pitch;
    float ub = (h.y * M.sad / den - M.b0) * M.inv_pitch;
    ua = fminf(fmaxf(ua, 0.0f), (float)(M.na - 1));  // NaN -> 0
    ub = fminf(fmaxf(ub, 0.0f), (float)(M.nb - 1));
    const int ia = min((int)ua, M.na - 2 < 0 ? 0 : M.na - 2), ib = min((int)ub, M.nb - 2 < 0 ? 0 : M.nb - 2);
    const float wa = M.na > 1 ? ua - (float)ia : 0.0f, wb = M.nb > 1 ? ub - (float)ib : 0.0f;
    const int ia1 = M.na > 1 ? ia + 1 : ia, ib1 = M.nb > 1 ? ib + 1 : ib;
    idx[0] = ib * M.na + ia;
    idx[1] = ib * M.na + ia1;
    idx[2] = ib1 * M.na + ia;
    idx[3] = ib1 * M.na + ia1;
    w[0] = (1.0f - wa) * (1.0f - wb);
    w[1] = wa * (1.0f - wb);
    w[2] = (1.0f - wa) * wb;
    w[3] = wa * wb;
    if (wa_out) *wa_out = wa;
    if (wb_out) *wb_out = wb;
}

}  // namespace

__global__ void __launch_bounds__(128) fluence_modulate_kernel(Grid g, Frame f, FluenceMap M,
                                                               const float *__restrict__ F,
                                                               const float *__restrict__ T0,
                                                               const float *__restrict__ E0,
                                                               cudaTextureObject_t dens_tex,
                                                               cudaSurfaceObject_t td_surf,
                                                               float *__restrict__ electron) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const long long v = (long long)i + (long long)g.nx * (j + (long long)g.ny * k);
    int idx[4];
    float w[4];
    float wa, wb;
    fluence_taps(M, f, voxel_xyz(g, f, i, j, k), idx, w, &wa, &wb);
    const int nmap = M.na * M.nb;
    (void)nmap;  // read by the bounds checks of debug builds
    float fv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) fv[q] = DC_IN_BOUNDS(idx[q], nmap, 50) ? __ldg(F + idx[q]) : 0.0f;
    // bilinear as nested linear interpolations, so that a constant map gives
    // exactly that constant (products of weights need not sum to 1 in float)
    const float m0 = fmaf(wa, fv[1] - fv[0], fv[0]), m1 = fmaf(wa, fv[3] - fv[2], fv[2]);
    const float m = fmaf(wb, m1 - m0, m0);
    const bool ok = DC_IN_BOUNDS(v, g.n(), 51);
    const float T = ok ? m * __ldg(T0 + v) : 0.0f;
    const float rho = tex3D<float>(dens_tex, (float)i + 0.5f, (float)j + 0.5f, (float)k + 0.5f);
    surf3Dwrite(make_float2(T, rho), td_surf, i * (int)sizeof(float2), j, k);
    if (ok) electron[v] = m * __ldg(E0 + v);
}

__global__ void __launch_bounds__(128) cccs_adjoint_kernel(Grid g, Frame f, CccsCones C, float sp_cm, float scale,
                                                           const float4 *__restrict__ dirs,
                                                           cudaTextureObject_t td_tex,
                                                           const int *__restrict__ active,
                                                           const unsigned *__restrict__ n_active,
                                                           const float *__restrict__ grad_dose, float *__restrict__ h) {
    __shared__ float4 s_dir[kMaxCones * 12];
    __shared__ float s_rl10[kMaxConeSteps];
    for (int q = threadIdx.x; q < C.n_cones * 12; q += blockDim.x) s_dir[q] = dirs[q];
    for (int q = threadIdx.x; q < C.total_steps; q += blockDim.x) s_rl10[q] = C.rl10[q];
    __syncthreads();
    const unsigned n = *n_active;
    const int plane = g.nx * g.ny;
    const long long nvox = g.n();
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int v = DC_IN_BOUNDS(t, nvox, 53) ? __ldg(active + t) : -1;
        if (!DC_IN_BOUNDS(v, nvox, 53)) continue;
        const float gp = scale * __ldg(grad_dose + v);
        if (gp == 0.0f) continue;
        const int k = v / plane;
        const int rem = v - k * plane;
        const int j = rem / g.nx;
        const int i = rem - j * g.nx;
        const float3 p = voxel_xyz(g, f, i, j, k);
        // kernelTilt, exactly as the forward (cccs_voxel)
        const float3 uvec = unit_to_source(f, p);
        const float3 axis0 = unit_to_source(f, make_float3(0.f, 0.f, 0.f));
        const float costh = axis0.x * uvec.x + axis0.y * uvec.y + axis0.z * uvec.z;
        const float3 ax = make_float3(axis0.y * uvec.z - axis0.z * uvec.y, axis0.z * uvec.x - axis0.x * uvec.z,
                                      axis0.x * uvec.y - axis0.y * uvec.x);
        const float inv1c = 1.0f / (1.0f + costh);
        for (int c = 0; c < C.n_cones; ++c) {
            const float Am = C.Am[c], am = C.am[c], Bm = C.Bm[c], bm = C.bm[c];
            const float nam_l2e = -am * kLog2e;
            const int s0 = C.step_off[c], ns = C.n_steps[c];
            for (int az = 0; az < 12; ++az) {
                const float4 dv = s_dir[c * 12 + az];
                const float sinth = dv.w;
                const float cp = sinth * (Am / (am * am));
                const float cs = sinth * (Bm / bm);
                float3 r;
                r.x = ax.y * dv.z - ax.z * dv.y;
                r.y = ax.z * dv.x - ax.x * dv.z;
                r.z = ax.x * dv.y - ax.y * dv.x;
                r.x += dv.x * costh;
                r.y += dv.y * costh;
                r.z += dv.z * costh;
                const float sc = (ax.x * dv.x + ax.y * dv.y + ax.z * dv.z) * inv1c;
                r.x += ax.x * sc;
                r.y += ax.y * sc;
                r.z += ax.z * sc;
                float Pe = 1.0f, Pb = 1.0f;  // products of the nearer samples' factors
                for (int s = ns - 1; s >= 0; --s) {
                    const float rl10 = s_rl10[s0 + s];
                    float3 q;
                    q.x = fmaf(r.x, rl10, p.x);
                    q.y = fmaf(r.y, rl10, p.y);
                    q.z = fmaf(r.z, rl10, p.z);
                    const float3 tc = tex_coord(g, f, q);
                    const float rho = tex3D<float2>(td_tex, tc.x, tc.y, tc.z).y;
                    const float Di = fmaxf(rho, kAirDensity) * sp_cm;
                    const float ex = fast_exp2(nam_l2e * Di);
                    const float wT = gp * (am * cp * (1.0f - ex) * Pe + bm * cs * Di * Pb);
                    Pe *= ex;
                    Pb *= 1.0f - bm * Di;
                    // scatter onto the sample's texels with the texture unit's weights
                    const float x = tc.x - 0.5f, y = tc.y - 0.5f, z = tc.z - 0.5f;
                    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
                    const float wa = rintf((x - fx) * 256.0f) * (1.0f / 256.0f);
                    const float wb = rintf((y - fy) * 256.0f) * (1.0f / 256.0f);
                    const float wc = rintf((z - fz) * 256.0f) * (1.0f / 256.0f);
                    const int i0 = (int)fx, j0 = (int)fy, k0 = (int)fz;
#pragma unroll
                    for (int dk = 0; dk < 2; ++dk) {
                        const int kk = k0 + dk;
                        if ((unsigned)kk >= (unsigned)g.nz) continue;
                        const float wzz = dk ? wc : 1.0f - wc;
#pragma unroll
                        for (int dj = 0; dj < 2; ++dj) {
                            const int jj = j0 + dj;
                            if ((unsigned)jj >= (unsigned)g.ny) continue;
                            const float wyz = (dj ? wb : 1.0f - wb) * wzz;
#pragma unroll
                            for (int di = 0; di < 2; ++di) {
                                const int ii = i0 + di;
                                if ((unsigned)ii >= (unsigned)g.nx) continue;
                                const float wt = (di ? wa : 1.0f - wa) * wyz;
                                if (wt == 0.0f) continue;
                                const long long u = (long long)ii + (long long)g.nx * (jj + (long long)g.ny * kk);
                                if (DC_IN_BOUNDS(u, nvox, 54)) atomicAdd(h + u, wT * wt);
                            }
                        }
                    }
                }
            }
        }
    }
}

__global__ void __launch_bounds__(128) fluence_grad_kernel(Grid g, Frame f, FluenceMap M, float scale,
                                                           const float *__restrict__ T0,
                                                           const float *__restrict__ E0,
                                                           const float *__restrict__ h,
                                                           const float *__restrict__ grad_dose,
                                                           double *__restrict__ grad_F) {
    extern __shared__ double s_acc[];
    const int nmap = M.na * M.nb;
    (void)nmap;  // read by the bounds checks of debug builds
    const bool in_smem = nmap <= kMaxSmemBeamlets;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    if (in_smem)
        for (int q = tid; q < nmap; q += blockDim.x * blockDim.y) s_acc[q] = 0.0;
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i < g.nx && j < g.ny) {
        const long long v = (long long)i + (long long)g.nx * (j + (long long)g.ny * k);
        if (DC_IN_BOUNDS(v, g.n(), 55)) {
            const float t0 = __ldg(T0 + v);
            // the electron term reaches the dose only where the CCCS mask lets
            // it (TERMA <= 0.01 writes 0, IMRTClasses.cu:270-273)
            const float val = t0 * __ldg(h + v) + (t0 <= 0.01f ? 0.0f : scale * __ldg(E0 + v) * __ldg(grad_dose + v));
            if (val != 0.0f) {
                int idx[4];
                float w[4];
                fluence_taps(M, f, voxel_xyz(g, f, i, j, k), idx, w);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (w[q] == 0.0f || !DC_IN_BOUNDS(idx[q], nmap, 56)) continue;
                    const double add = (double)w[q] * (double)val;
                    if (in_smem)
                        atomicAdd(s_acc + idx[q], add);
                    else
                        atomicAdd(grad_F + idx[q], add);
                }
            }
        }
    }
    __syncthreads();
    if (in_smem)
        for (int q = tid; q < nmap; q += blockDim.x * blockDim.y)
            if (s_acc[q] != 0.0) atomicAdd(grad_F + q, s_acc[q]);
}

DC_BOUNDS_TAKE(take_bounds_fluence)

static dim3 fl_grid(const Grid &g) {
    return dim3((unsigned)((g.nx + 31) / 32), (unsigned)((g.ny + 3) / 4), (unsigned)g.nz);
}

void enqueue_fluence_modulate(DeviceContext &ctx, const Grid &g, const Frame &f, const FluenceMap &M,
                              const float *F, const float *T0, const float *E0, const PhotonWork &w, cudaStream_t s) {
    KernelTimer kt(ctx, "fluence_modulate", s);
    fluence_modulate_kernel<<<fl_grid(g), dim3(32, 4, 1), 0, s>>>(g, f, M, F, T0, E0, w.dens_tex, w.td_surf,
                                                                  w.electron);
    check_launch("fluence_modulate_kernel");
}

void enqueue_fluence_adjoint(DeviceContext &ctx, const Grid &g, const Frame &f, const CccsCones &C,
                             const FluenceMap &M, float dose_scale, const float *T0, const float *E0,
                             const PhotonWork &w, const float *grad_dose, float *h, double *grad_F, cudaStream_t s) {
    DC_CUDA(cudaMemsetAsync(h, 0, (size_t)g.n() * sizeof(float), s));
    DC_CUDA(cudaMemsetAsync(grad_F, 0, (size_t)M.na * M.nb * sizeof(double), s));
    {
        KernelTimer kt(ctx, "cccs_adjoint", s);
        int sms = 0, per_sm = 0;
        DC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
        DC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cccs_adjoint_kernel, 128, 0));
        const long long want = (g.n() + 127) / 128;
        const unsigned blocks = (unsigned)std::max(1LL, std::min<long long>(want, (long long)sms * std::max(per_sm, 1)));
        cccs_adjoint_kernel<<<blocks, 128, 0, s>>>(g, f, C, g.sx / 10.0f, dose_scale, w.dirs, w.td_tex, w.active,
                                                   w.n_active, grad_dose, h);
        check_launch("cccs_adjoint_kernel");
    }
    {
        KernelTimer kt(ctx, "fluence_grad", s);
        const int nmap = M.na * M.nb;
    (void)nmap;  // read by the bounds checks of debug builds
        const size_t smem = nmap <= kMaxSmemBeamlets ? (size_t)nmap * sizeof(double) : 0;
        fluence_grad_kernel<<<fl_grid(g), dim3(32, 4, 1), smem, s>>>(g, f, M, dose_scale, T0, E0, h, grad_dose, grad_F);
        check_launch("fluence_grad_kernel");
    }
}

}  // namespace dc
