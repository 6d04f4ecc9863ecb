// dc_photon.cu — photon TERMA and collapsed-cone convolution/superposition.
//
// terma_kernel restates termaKernel (IMRTClasses.cu:209-250) with
// headTransmission (:120-150) and offAxisFactors (:152-171): per voxel, the
// primary and scatter source occlusion by every MLC leaf pair (a product of
// erf edges), the off-axis intensity/softening profile, the 12-bin spectrum
// attenuated along the radiological depth, and the electron contamination.
//
// cccs_kernel restates cccKernel (IMRTClasses.cu:252-350) with kernelTilt
// (:173-203): per voxel with TERMA > 0.01, for 6 zenith cones x 12 azimuths,
// a backward recursive march from ray_length (cm) down to 0 in steps of one
// voxel spacing, sampling TERMA and density (hardware trilinear), with the
// cone direction tilted so that its axis points at the source.
//
// B200 design points:
//  * TERMA and density are written as one float2 texel into the
//    surface-writable cudaArray that the CCCS kernel samples, so one filtered
//    fetch per cone sample serves both (the reference writes TERMA to linear
//    memory, copies it into a fresh array and samples two textures,
//    IMRTClasses.cu:398-399,423-424).
//  * Leaf pairs whose two edges lie on the same side of the voxel's
//    projection, both more than 3.92 * sqrt(2) source-sigmas from it, give
//    exactly erf = +-1 on both edges (kErfSaturated), i.e. no transmission;
//    they are skipped without evaluating erf, and with ascending leaf edges
//    the pairs that remain form one range found by binary search.  Within
//    it, erf values of equal arguments are reused: a pair's bottom edge is
//    the previous pair's top edge, and open fields repeat the leaf x
//    positions, so the scatter source (about 33 pairs in range) costs
//    about one erf per pair instead of four.
//  * The TERMA kernel applies the CCCS mask and lists the active voxels; the
//    CCCS is a persistent grid-stride loop over that list, so every lane of
//    every warp marches (masked voxels no longer idle lanes).
//  * The 72 image-space cone directions, the per-cone step tables (the float
//    sequence ray_length, ray_length - sp, ... >= 0 that sets each cone's
//    sample count) and the cone coefficients are computed once per call and
//    held in shared memory; per sample the kernel does 3 FMAs of position,
//    one float2 texture fetch, one SFU exponential and the two recursions.
//  * The TERMA kernel maps threads to 32x4 voxel tiles (coalesced stores).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/dosecuda.h"

#include "dc_common.cuh"
#include "dc_kernels.cuh"
#include "dc_photon.cuh"
#include "dc_runtime.cuh"

namespace dc {

DC_BOUNDS_WORD

// ---------------------------------------------------------------------------
// TERMA
// ---------------------------------------------------------------------------
// Scaled erf argument of a leaf edge at y (isocentre plane) seen from a
// voxel at lateral position py: ((y - py) * div + py) * kinv, as in
// headTransmission (IMRTClasses.cu:130-142), with the multiply-add fused.
// Written with explicit round-to-nearest intrinsics, which the compiler
// neither contracts nor reorders, so that every evaluation — the range
// search, the pair loop's test, and the erf arguments — is the same
// function of its inputs.
__device__ __forceinline__ float edge_pos(float y, float py, float div) {
    return __fmaf_rn(__fsub_rn(y, py), div, py);
}
__device__ __forceinline__ float edge_arg(float y, float py, float div, float kinv) {
    return __fmul_rn(edge_pos(y, py, div), kinv);
}

// Edge arguments larger in magnitude than this give erff = +-1 exactly, so a
// leaf pair whose two edges both lie beyond it on the same side transmits
// exactly 0 and can be skipped without changing the sum.  Checked over every
// float in [3, 4.5] by photon_erf_unsaturated (dc_photon_head_selftest): on
// sm_100a with CUDA 12.9 the largest unsaturated argument is 3.9140925f
// (erfc(3.914) = 3.1e-8, half an ulp of 1); 3.92 skips about 13 % more pairs
// than the 4.5 used before that check.
constexpr float kErfSaturated = 3.92f;

__device__ __forceinline__ float head_transmission(const PhotonParams &P, float3 p, float iso_to_source,
                                                   float source_sigma) {
    const float div = (iso_to_source - p.z) / (P.mlc_distance - p.z);
    const float kinv = 1.0f / (source_sigma * sqrtf(2.f));
    // |edge * kinv| > lim on both edges of the same side => erf terms cancel.
    const float lim = kErfSaturated;
    // With the pairs' y edges in ascending order (P.edges_sorted) and a
    // finite, positive scaling, a1 and a2 below are non-decreasing in q
    // (every operation is monotone), so the pairs the loop skips as
    // "a2 < -lim" form a prefix and those skipped as "a1 > lim" a suffix:
    // two binary searches over the same expression find the loop's range,
    // and the loop still applies its own test to each pair in it — the same
    // pairs in the same order as a scan of all pairs.
    int q0 = 0, q1 = P.n_pairs;
    bool searched = false;
    if (P.edges_sorted && div > 0.0f && div < INFINITY && kinv > 0.0f && kinv < INFINITY && fabsf(p.y) < INFINITY) {
        searched = true;
        int lo = 0, hi = P.n_pairs;
        while (lo < hi) {  // first pair with a2 >= -lim
            const int mid = (lo + hi) >> 1;
            if (edge_arg(P.mlc_yt[mid], p.y, div, kinv) < -lim) lo = mid + 1; else hi = mid;
        }
        q0 = lo;
        hi = P.n_pairs;
        while (lo < hi) {  // first pair with a1 > lim
            const int mid = (lo + hi) >> 1;
            if (edge_arg(P.mlc_yb[mid], p.y, div, kinv) > lim) hi = mid; else lo = mid + 1;
        }
        q1 = lo;
    }
    // erf of equal arguments is equal: adjacent pairs share a y edge (the
    // top of one is the bottom of the next) and open fields repeat the same
    // leaf x positions, so the last top-edge erf and the last x factor are
    // reused whenever their inputs are the same floats as before.
    float cached_y = NAN, cached_erf_y = 0.0f;
    float cached_xl = NAN, cached_xr = NAN, cached_ex = 0.0f;
    float trans = 0.0f;
    for (int q = q0; q < q1; ++q) {
        const float xl = P.mlc_xl[q], xr = P.mlc_xr[q];
        if (xl == xr) continue;  // closed pair: exposed source X is exactly 0
        const float yb = P.mlc_yb[q], yt = P.mlc_yt[q];
        const float a1 = edge_arg(yb, p.y, div, kinv);
        const float a2 = edge_arg(yt, p.y, div, kinv);
        // in a searched range a2 >= -lim (q >= q0) and a1 <= lim (q < q1), so
        // the test can only skip pairs of the unsorted scan
        if (!searched && ((a1 > lim && a2 > lim) || (a1 < -lim && a2 < -lim))) continue;
        if (!(xl == cached_xl && xr == cached_xr)) {
            cached_ex = 0.5f * (erff(edge_arg(xr, p.x, div, kinv)) - erff(edge_arg(xl, p.x, div, kinv)));
            cached_xl = xl;
            cached_xr = xr;
        }
        const float erf_b = (yb == cached_y) ? cached_erf_y : erff(a1);
        const float erf_t = erff(a2);
        cached_y = yt;
        cached_erf_y = erf_t;
        const float ey = 0.5f * (erf_t - erf_b);
        trans = __fmaf_rn(cached_ex, ey, trans);
    }
    return trans;
}

// Largest float x in [lo, hi] (lo > 0) with erff(x) != 1 or erff(-x) != -1,
// as float bits through atomicMax (positive floats order like their bits).
__global__ void erf_saturation_kernel(unsigned lo, unsigned hi, unsigned *__restrict__ largest) {
    const unsigned stride = gridDim.x * blockDim.x;
    for (unsigned b = lo + blockIdx.x * blockDim.x + threadIdx.x; b <= hi; b += stride) {
        const float x = __uint_as_float(b);
        if (erff(x) != 1.0f || erff(-x) != -1.0f) atomicMax(largest, b);
    }
}

float photon_erf_unsaturated(float lo, float hi) {
    if (!(lo > 0.0f && hi >= lo && hi < 1.0e30f)) throw Error(DC_ERR_VALUE, "need 0 < lo <= hi");
    unsigned *d = nullptr;
    DC_CUDA(cudaMalloc(&d, sizeof(unsigned)));
    unsigned bits = 0;
    try {
        DC_CUDA(cudaMemset(d, 0, sizeof(unsigned)));
        unsigned lo_b, hi_b;
        std::memcpy(&lo_b, &lo, sizeof(float));
        std::memcpy(&hi_b, &hi, sizeof(float));
        erf_saturation_kernel<<<1184, 256>>>(lo_b, hi_b, d);
        check_launch("erf_saturation_kernel");
        DC_CUDA(cudaMemcpy(&bits, d, sizeof(unsigned), cudaMemcpyDeviceToHost));
    } catch (...) {
        cudaFree(d);
        throw;
    }
    DC_CUDA(cudaFree(d));
    float x;
    std::memcpy(&x, &bits, sizeof(float));
    return x;
}

float photon_erf_skip_bound() { return kErfSaturated; }

// Head factors of each voxel, which do not depend on the density: the
// primary and scatter transmission through the collimator
// (headTransmission, IMRTClasses.cu:120-150) and the off-axis intensity and
// softening (offAxisFactors, IMRTClasses.cu:152-171), as (tp, ts, oaf, soft).
// Split from the TERMA kernel so that it can run on a side stream while the
// density is uploaded or the radiological depth is traced.
__global__ void __launch_bounds__(128) head_kernel(Grid g, Frame f, PhotonParams P, float4 *__restrict__ head) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const long long v = (long long)i + (long long)g.nx * (j + (long long)g.ny * k);

    const float3 p = voxel_xyz(g, f, i, j, k);
    const float3 h = image_to_head<true>(f, p);
    const float d_src = P.psd - h.z;
    const float r_cax = hypotf(h.x, h.y) * d_src / P.psd;
    float oaf, soft;
    {
        const int n = P.n_prof;
        const int q = lower_bound(P.prof_r, n, r_cax);
        if (q == n) {
            oaf = P.prof_i[q - 1];
            soft = P.prof_s[q - 1];
        } else if (q == 0) {
            oaf = P.prof_i[0];
            soft = P.prof_s[0];
        } else {
            const float m = (r_cax - P.prof_r[q - 1]) / (P.prof_r[q] - P.prof_r[q - 1]);
            oaf = fmaf(P.prof_i[q] - P.prof_i[q - 1], m, P.prof_i[q - 1]);
            soft = fmaf(P.prof_s[q] - P.prof_s[q - 1], m, P.prof_s[q - 1]);
        }
    }
    const float tp = head_transmission(P, h, P.psd, P.pss);
    const float ts = head_transmission(P, h, P.ssd, P.sss);
    if (DC_IN_BOUNDS(v, g.n(), 11)) head[v] = make_float4(tp, ts, oaf, soft);
}

// Writes (TERMA, density) of each voxel as one float2 texel of the CCCS
// volume; the density is the input texture read at the texel centre, where
// linear filtering returns the stored value unchanged.  It also applies the
// CCCS mask (dose 0 where TERMA <= 0.01, IMRTClasses.cu:270-273): masked
// voxels get their zero dose here, the others are appended to `active`
// (warp-aggregated), so the CCCS runs on full warps of active voxels only.
// dose (or null) receives the zero of masked voxels; terma_out (or null) a
// linear copy of the TERMA volume.  `head` holds head_kernel's factors.
__global__ void __launch_bounds__(128) terma_kernel(Grid g, Frame f, PhotonParams P, const float *__restrict__ wet,
                                                    const float4 *__restrict__ head,
                                                    cudaTextureObject_t dens_tex, cudaSurfaceObject_t td_surf,
                                                    float *__restrict__ electron,
                                                    float *__restrict__ dose, float *__restrict__ terma_out,
                                                    int *__restrict__ active, unsigned *__restrict__ n_active) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const long long v = (long long)i + (long long)g.nx * (j + (long long)g.ny * k);
    const bool v_ok = DC_IN_BOUNDS(v, g.n(), 10);

    const float3 p = voxel_xyz(g, f, i, j, k);
    const float3 h = image_to_head<true>(f, p);
    const float d_primary = P.psd - h.z;
    const float d_scatter = P.ssd - h.z;
    const float4 hf = v_ok ? __ldg(head + v) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float tp = hf.x, ts = hf.y, oaf = hf.z, soft = hf.w;
    const float w = __ldg(wet + v);
    const float ratio = fminf(1.00f, ts / tp);
    const float geo_p = sqr(P.psd / d_primary);
    const float geo_s = P.ssd / d_scatter;
    float terma = 0.f;
    for (int e = 0; e < P.n_spec; ++e) {
        const float att = expf(-P.spec_mu[e] * w * soft);
        terma += (1.0f - ratio) * (P.spec_pw[e] * att * geo_p) + ratio * P.spec_sw[e] * att * geo_s;
    }
    const float e_dmax = expf(-P.ea * P.efd);
    const float elec = fmaxf(0.0f, (expf(-P.ea * w) - e_dmax) / (1.0f - e_dmax));
    const float T = oaf * ((1.0f - P.ssw) * tp * terma + P.ssw * ts * terma);
    const float rho = tex3D<float>(dens_tex, (float)i + 0.5f, (float)j + 0.5f, (float)k + 0.5f);
    surf3Dwrite(make_float2(T, rho), td_surf, i * (int)sizeof(float2), j, k);
    if (v_ok) electron[v] = P.esw * (0.4f + (0.3f * ratio)) * elec * tp;
    if (terma_out && v_ok) terma_out[v] = T;

    const bool act = !(T <= 0.01f);
    if (!act && dose && v_ok) dose[v] = 0.0f;
    const unsigned live = __activemask();
    const unsigned bal = __ballot_sync(live, act);
    if (act) {
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(bal) - 1;
        unsigned base = 0;
        if (lane == leader) base = atomicAdd(n_active, (unsigned)__popc(bal));
        base = __shfl_sync(bal, base, leader);
        const long long slot = (long long)base + __popc(bal & ((1u << lane) - 1u));
        if (DC_IN_BOUNDS(slot, g.n(), 12)) active[slot] = (int)v;
    }
}

// ---------------------------------------------------------------------------
// Cone directions (voxel independent part): head-frame tangent of each of the
// 72 cone directions rotated into the image frame (IMRTClasses.cu:282-308).
// Computed on the device with the same math functions as the reference.
// ---------------------------------------------------------------------------
__global__ void cone_dirs_kernel(Frame f, CccsCones C, float4 *__restrict__ dirs) {
    const int d = threadIdx.x;
    if (d >= C.n_cones * 12) return;
    const int i = d / 12, jj = d % 12;
    float sj, cj;
    sincosf((float)jj * CUDART_PI_F / 6.0f, &sj, &cj);
    const float th = C.theta_deg[i] * CUDART_PI_F / 180.0f;
    const float sth = sinf(th), cth = cosf(th);
    const float3 th_head = make_float3(sth * cj, sth * sj, cth);
    const float3 t = head_to_image<true>(f, th_head);
    dirs[d] = make_float4(t.x, t.y, t.z, sth);
}

// ---------------------------------------------------------------------------
// CCCS
// ---------------------------------------------------------------------------
// td_tex: float2 (TERMA, density) texture, border (0, AIR_DENSITY) — one
// filtered fetch serves both of the reference's textures (the same
// coordinates and weights apply to both channels).
// Persistent grid-stride loop over the active voxels listed by the TERMA
// kernel (every lane of a warp does a full 72-direction march).
__device__ __forceinline__ float cccs_voxel(const Grid &g, const Frame &f, const CccsCones &C, float sp_cm,
                                            const float4 *s_dir, const float *s_rl10, cudaTextureObject_t td_tex,
                                            float3 p);

__global__ void __launch_bounds__(128) cccs_kernel(Grid g, Frame f, CccsCones C, float sp_cm, float dose_scale,
                                                   const float4 *__restrict__ dirs, cudaTextureObject_t td_tex,
                                                   const float *__restrict__ electron, const int *__restrict__ active,
                                                   const unsigned *__restrict__ n_active, float *__restrict__ dose) {
    __shared__ float4 s_dir[kMaxCones * 12];
    __shared__ float s_rl10[kMaxConeSteps];
    const int tid = threadIdx.x;
    for (int q = tid; q < C.n_cones * 12; q += blockDim.x) s_dir[q] = dirs[q];
    for (int q = tid; q < C.total_steps; q += blockDim.x) s_rl10[q] = C.rl10[q];
    __syncthreads();

    const unsigned n = *n_active;
    const int plane = g.nx * g.ny;
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int v = DC_IN_BOUNDS(t, g.n(), 13) ? __ldg(active + t) : -1;
        if (!DC_IN_BOUNDS(v, g.n(), 13)) continue;
        const int k = v / plane;
        const int rem = v - k * plane;
        const int j = rem / g.nx;
        const int i = rem - j * g.nx;
        const float3 p = voxel_xyz(g, f, i, j, k);
        float dose_value = cccs_voxel(g, f, C, sp_cm, s_dir, s_rl10, td_tex, p);
        dose_value += __ldg(electron + v);
        dose[v] = (!isnan(dose_value) && dose_value >= 0.0f) ? dose_scale * dose_value : 0.0f;  // v checked above
    }
}

// CCCS at an arbitrary list of voxels (the surrogate's probe): the same
// per-voxel sum as cccs_kernel, with the mask taken from the TERMA texel.
__global__ void __launch_bounds__(128) cccs_points_kernel(Grid g, Frame f, CccsCones C, float sp_cm, float dose_scale,
                                                          const float4 *__restrict__ dirs, cudaTextureObject_t td_tex,
                                                          const float *__restrict__ electron,
                                                          const int *__restrict__ voxels, int n,
                                                          float *__restrict__ out) {
    __shared__ float4 s_dir[kMaxCones * 12];
    __shared__ float s_rl10[kMaxConeSteps];
    const int tid = threadIdx.x;
    for (int q = tid; q < C.n_cones * 12; q += blockDim.x) s_dir[q] = dirs[q];
    for (int q = tid; q < C.total_steps; q += blockDim.x) s_rl10[q] = C.rl10[q];
    __syncthreads();
    const int plane = g.nx * g.ny;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int v = __ldg(voxels + t);
        if (v < 0 || (long long)v >= g.n()) {  // not a voxel of the grid
            out[t] = 0.0f;
            continue;
        }
        const int k = v / plane;
        const int rem = v - k * plane;
        const int j = rem / g.nx;
        const int i = rem - j * g.nx;
        const float T = tex3D<float2>(td_tex, (float)i + 0.5f, (float)j + 0.5f, (float)k + 0.5f).x;
        float r = 0.0f;
        if (!(T <= 0.01f)) {
            const float3 p = voxel_xyz(g, f, i, j, k);
            float dose_value = cccs_voxel(g, f, C, sp_cm, s_dir, s_rl10, td_tex, p);
            dose_value += __ldg(electron + v);
            r = (!isnan(dose_value) && dose_value >= 0.0f) ? dose_scale * dose_value : 0.0f;
        }
        out[t] = r;
    }
}

// Sum over the 6 zenith cones x 12 azimuths of the backward recursion
// (IMRTClasses.cu:289-339) for the voxel at image position p.
__device__ __forceinline__ float cccs_voxel(const Grid &g, const Frame &f, const CccsCones &C, float sp_cm,
                                            const float4 *s_dir, const float *s_rl10, cudaTextureObject_t td_tex,
                                            float3 p) {
    // kernelTilt (IMRTClasses.cu:173-203): rotate each direction by the
    // rotation taking the central axis (iso -> source) onto voxel -> source.
    const float3 uvec = unit_to_source(f, p);
    const float3 axis0 = unit_to_source(f, make_float3(0.f, 0.f, 0.f));
    const float costh = axis0.x * uvec.x + axis0.y * uvec.y + axis0.z * uvec.z;
    const float3 ax = make_float3(axis0.y * uvec.z - axis0.z * uvec.y, axis0.z * uvec.x - axis0.x * uvec.z,
                                  axis0.x * uvec.y - axis0.y * uvec.x);
    const float inv1c = 1.0f / (1.0f + costh);
    // A sample at distance 0 lies on the voxel centre whatever the direction
    // (fmaf(r, 0, p) == p), so every cone whose sample distances end exactly
    // at 0 fetches the same texel there: fetched once here and reused,
    // which gives the same value as the 72 separate fetches.
    const float3 tc0 = tex_coord(g, f, p);
    const float2 td0 = tex3D<float2>(td_tex, tc0.x, tc0.y, tc0.z);

    float dose_value = 0.0f;
    for (int c = 0; c < C.n_cones; ++c) {
        const float Am = C.Am[c], am = C.am[c], Bm = C.Bm[c], bm = C.bm[c];
        const float nam_l2e = -am * kLog2e;
        const int s0 = C.step_off[c], ns = C.n_steps[c];
        for (int az = 0; az < 12; ++az) {
            const float4 dv = s_dir[c * 12 + az];
            const float sinth = dv.w;
            const float cp = sinth * (Am / (am * am));
            const float cs = sinth * (Bm / bm);
            // Rodrigues: r = ax x v + v cos + ax (ax.v)/(1+cos)
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

            float Rp = 0.0f, Rs = 0.0f;
            for (int s = 0; s < ns; ++s) {
                const float rl10 = s_rl10[s0 + s];
                float3 q;
                q.x = fmaf(r.x, rl10, p.x);
                q.y = fmaf(r.y, rl10, p.y);
                q.z = fmaf(r.z, rl10, p.z);
                const float3 tc = tex_coord(g, f, q);
                const float2 td = rl10 == 0.0f ? td0 : tex3D<float2>(td_tex, tc.x, tc.y, tc.z);
                const float Ti = td.x;
                const float Di = fmaxf(td.y, kAirDensity) * sp_cm;
                const float ex = fast_exp2(nam_l2e * Di);
                Rp = Rp * ex + (Ti * cp * (1.0f - ex));
                Rs = Rs * (1.0f - (bm * Di)) + (Ti * Di * cs);
            }
            dose_value += am * Rp + bm * Rs;
        }
    }
    return dose_value;
}

// ---------------------------------------------------------------------------
// Host
// ---------------------------------------------------------------------------
static dim3 vol_grid(const Grid &g) {
    return dim3((unsigned)((g.nx + 31) / 32), (unsigned)((g.ny + 3) / 4), (unsigned)g.nz);
}

void build_photon_params(const dc_photon_model &m, const dc_control_point &cp, float spacing_cm,
                         PhotonParams &P, CccsCones &C) {
    auto need = [](bool ok, const std::string &msg) {
        if (!ok) throw Error(DC_ERR_VALUE, msg);
    };
    need(cp.n_mlc_pairs >= 0 && cp.n_mlc_pairs <= kMaxPairs,
         "'mlc' must have between 0 and " + std::to_string(kMaxPairs) + " leaf pairs.");
    need(m.n_profile_points >= 1 && m.n_profile_points <= kMaxProfile,
         "'profile_radius' must have between 1 and " + std::to_string(kMaxProfile) + " points.");
    need(m.n_spectral_energies >= 0 && m.n_spectral_energies <= kMaxSpectrum,
         "'spectrum_attenuation_coefficients' must have at most " + std::to_string(kMaxSpectrum) + " energies.");
    need(m.n_cones >= 1 && m.n_cones <= kMaxCones,
         "'kernel' must have between 1 and " + std::to_string(kMaxCones) + " cone rows.");
    need(spacing_cm > 0.0f, "'spacing' must be positive.");

    P.psd = m.primary_source_distance;
    P.ssd = m.scatter_source_distance;
    P.pss = m.primary_source_size;
    P.sss = m.scatter_source_size;
    P.mlc_distance = m.mlc_distance;
    P.ssw = m.scatter_source_weight;
    P.ea = m.electron_attenuation;
    P.esw = m.electron_source_weight;
    P.efd = m.electron_fitted_dmax;
    // headTransmission's leaf projection to the isocentre plane (IMRTClasses.cu:122,130-134).
    const float mlc_scale = (m.primary_source_distance - m.mlc_distance) / m.primary_source_distance;
    P.n_pairs = cp.n_mlc_pairs;
    for (int q = 0; q < cp.n_mlc_pairs; ++q) {
        P.mlc_yb[q] = (cp.mlc_y_offset[q] - 0.5f * cp.mlc_y_width[q]) * mlc_scale;
        P.mlc_yt[q] = (cp.mlc_y_offset[q] + 0.5f * cp.mlc_y_width[q]) * mlc_scale;
        P.mlc_xl[q] = cp.mlc_x1[q] * mlc_scale;
        P.mlc_xr[q] = cp.mlc_x2[q] * mlc_scale;
    }
    // Leaf-pair range search precondition (head_transmission): finite y
    // edges, bottom <= top within a pair, both ascending across pairs.
    P.edges_sorted = 1;
    for (int q = 0; q < P.n_pairs; ++q) {
        const bool ok = std::isfinite(P.mlc_yb[q]) && std::isfinite(P.mlc_yt[q]) && P.mlc_yb[q] <= P.mlc_yt[q] &&
                        (q == 0 || (P.mlc_yb[q - 1] <= P.mlc_yb[q] && P.mlc_yt[q - 1] <= P.mlc_yt[q]));
        if (!ok) P.edges_sorted = 0;
    }
    P.n_prof = m.n_profile_points;
    for (int q = 0; q < m.n_profile_points; ++q) {
        P.prof_r[q] = m.profile_radius[q];
        P.prof_i[q] = m.profile_intensities[q];
        P.prof_s[q] = m.profile_softening[q];
    }
    P.n_spec = m.n_spectral_energies;
    for (int q = 0; q < m.n_spectral_energies; ++q) {
        P.spec_mu[q] = m.spectrum_attenuation_coefficients[q];
        P.spec_pw[q] = m.spectrum_primary_weights[q];
        P.spec_sw[q] = m.spectrum_scatter_weights[q];
    }

    // Cones: sample positions ray_length, ray_length - sp, ... while >= 0,
    // accumulated in float exactly as the reference loop does
    // (IMRTClasses.cu:313-333), stored as ray_length*10 (mm).
    C.n_cones = m.n_cones;
    int off = 0;
    for (int c = 0; c < m.n_cones; ++c) {
        C.theta_deg[c] = m.kernel_theta_deg[c];
        C.Am[c] = m.kernel_Am[c];
        C.am[c] = m.kernel_am[c];
        C.Bm[c] = m.kernel_Bm[c];
        C.bm[c] = m.kernel_bm[c];
        C.step_off[c] = off;
        int n = 0;
        float rl = m.kernel_ray_length[c];
        while (rl >= 0.0f) {
            need(off + n < kMaxConeSteps, "CCCS kernel ray lengths need more than " +
                                              std::to_string(kMaxConeSteps) +
                                              " samples per direction set at this voxel spacing.");
            C.rl10[off + n] = rl * 10.0f;
            ++n;
            rl = rl - spacing_cm;
        }
        C.n_steps[c] = n;
        off += n;
    }
    C.total_steps = off;
}

static unsigned cccs_blocks(const DeviceContext &ctx, long long work) {
    // persistent grid: as many resident CTAs as fit on every SM
    int sms = 0, per_sm = 0;
    DC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
    DC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cccs_kernel, 128, 0));
    const long long want = (work + 127) / 128;
    return (unsigned)std::max(1LL, std::min<long long>(want, (long long)sms * std::max(per_sm, 1)));
}

DC_BOUNDS_TAKE(take_bounds_photon)

// WET (cm) below which the electron contamination term of terma_kernel is
// non-zero, plus a margin well above the lattice's interpolation error
// (0.03 cm): max(0, (e^{-ea w} - e^{-ea efd}) / (1 - e^{-ea efd})) vanishes
// for w >= efd when ea > 0 and efd > 0.  Without an electron term there is no
// bound (-inf); with parameters that keep it non-zero at every depth the
// lattice is not used at all (+inf).
static float electron_exact_wet(const PhotonParams &P) {
    if (P.esw == 0.0f) return -INFINITY;
    if (P.ea > 0.0f && P.efd > 0.0f && P.efd < 1.0e4f) return P.efd + 0.1f;
    return INFINITY;
}

void photon_head_fork(DeviceContext &ctx, const Grid &g, const Frame &f, const PhotonParams &P, cudaStream_t s) {
    float4 *head = static_cast<float4 *>(ctx.head.ensure((size_t)g.n() * sizeof(float4)));
    // With the kernel profiler on, the head factors run on s itself, so that
    // no kernel's timed interval includes another's share of the SMs.
    const cudaStream_t hs = ctx.profiling && !DeviceContext::capturing(s) ? s : ctx.side;
    DC_CUDA(cudaEventRecord(ctx.fork_ev, s));
    DC_CUDA(cudaStreamWaitEvent(hs, ctx.fork_ev, 0));
    {
        KernelTimer kt(ctx, "head", hs);
        head_kernel<<<vol_grid(g), dim3(32, 4, 1), 0, hs>>>(g, f, P, head);
        check_launch("head_kernel");
    }
    DC_CUDA(cudaEventRecord(ctx.join_ev, hs));
    ctx.head_forked = true;
}

void enqueue_terma(DeviceContext &ctx, const Grid &g, const Frame &f, const PhotonParams &P, const CccsCones &C,
                   const PhotonWork &w, float *dose_dev, float *terma_out, cudaStream_t s) {
    if (g.n() > 0x7fffffffLL) throw Error(DC_ERR_VALUE, "photon volumes are limited to 2^31 - 1 voxels.");
    // the head factors run beside the depth pass unless the caller forked them earlier
    if (!ctx.head_forked) photon_head_fork(ctx, g, f, P, s);
    if (w.depth_mode == 1 && w.xlat != nullptr)
        launch_xray_depth(ctx, g, f, w.dens_tex, w.wet, w.active, w.n_active, *w.xlat, w.depth_stats,
                          electron_exact_wet(P), s);  // the active list is free until the TERMA kernel fills it
    else {
        launch_wet_march(ctx, g, f, w.dens_tex, w.wet, s);
        if (w.depth_stats != nullptr) DC_CUDA(cudaMemsetAsync(w.depth_stats, 0xff, sizeof(unsigned), s));
    }
    DC_CUDA(cudaMemsetAsync(w.n_active, 0, sizeof(unsigned), s));
    DC_CUDA(cudaStreamWaitEvent(s, ctx.join_ev, 0));
    ctx.head_forked = false;
    {
        KernelTimer kt(ctx, "terma", s);
        terma_kernel<<<vol_grid(g), dim3(32, 4, 1), 0, s>>>(g, f, P, w.wet, ctx.head.as<const float4>(), w.dens_tex,
                                                            w.td_surf, w.electron, dose_dev, terma_out, w.active,
                                                            w.n_active);
        check_launch("terma_kernel");
    }
    cone_dirs_kernel<<<1, kMaxCones * 12, 0, s>>>(f, C, w.dirs);
    check_launch("cone_dirs_kernel");
}

void enqueue_cccs(DeviceContext &ctx, const Grid &g, const Frame &f, const CccsCones &C, const PhotonWork &w,
                  float dose_scale, float *dose_dev, cudaStream_t s) {
    KernelTimer kt(ctx, "cccs", s);
    cccs_kernel<<<cccs_blocks(ctx, g.n()), 128, 0, s>>>(g, f, C, g.sx / 10.0f, dose_scale, w.dirs, w.td_tex,
                                                        w.electron, w.active, w.n_active, dose_dev);
    check_launch("cccs_kernel");
}

void enqueue_cccs_points(DeviceContext &ctx, const Grid &g, const Frame &f, const CccsCones &C, const PhotonWork &w,
                         float dose_scale, const int *voxels, int n, float *out, cudaStream_t s) {
    if (n <= 0) return;
    KernelTimer kt(ctx, "cccs_points", s);
    cccs_points_kernel<<<cccs_blocks(ctx, n), 128, 0, s>>>(g, f, C, g.sx / 10.0f, dose_scale, w.dirs, w.td_tex,
                                                              w.electron, voxels, n, out);
    check_launch("cccs_points_kernel");
}

void run_photon_pipeline(DeviceContext &ctx, const Grid &g, const Frame &f, const PhotonParams &P,
                         const CccsCones &C, float dose_scale, float *dose_dev, cudaStream_t s) {
    const long long n = g.n();
    if (n > 0x7fffffffLL) throw Error(DC_ERR_VALUE, "photon volumes are limited to 2^31 - 1 voxels.");
    PhotonWork w;
    // The density volume is already in ctx.density; border AIR_DENSITY
    // (IMRTClasses.cu:394).
    w.dens_tex = ctx.density.texture(kAirDensity);
    // (TERMA, density) volume: TERMA border 0 (IMRTClasses.cu:399), density
    // border AIR_DENSITY (:394).
    ctx.terma.ensure(g.nx, g.ny, g.nz, true, 2);
    w.td_tex = ctx.terma.texture(0.0f, kAirDensity);
    w.td_surf = ctx.terma.surf;
    w.wet = static_cast<float *>(ctx.wet_raw.ensure((size_t)n * sizeof(float)));
    w.electron = static_cast<float *>(ctx.electron.ensure((size_t)n * sizeof(float)));
    w.dirs = static_cast<float4 *>(ctx.small.ensure(kMaxCones * 12 * sizeof(float4)));
    char *act = static_cast<char *>(ctx.active.ensure(256 + (size_t)n * sizeof(int)));
    w.n_active = reinterpret_cast<unsigned *>(act);
    w.active = reinterpret_cast<int *>(act + 256);
    w.xlat = &ctx.xlat;
    w.depth_mode = ctx.photon_depth_mode;
    w.depth_stats = static_cast<unsigned *>(ctx.xstat.ensure(sizeof(unsigned)));
    enqueue_terma(ctx, g, f, P, C, w, dose_dev, nullptr, s);
    enqueue_cccs(ctx, g, f, C, w, dose_scale, dose_dev, s);
}

}  // namespace dc

// ---------------------------------------------------------------------------
// Texture-unit calibration: the rate of trilinear float2 3D fetches in the
// CCCS kernel's access pattern (each thread marches a line of samples one
// voxel apart in a fixed direction; the 32 lanes of a warp start on adjacent
// voxels), with every fetch used, so that the CCCS's cone-sample rate can be
// read as a fraction of what the texture unit delivers on this GPU.
// ---------------------------------------------------------------------------
namespace dc {
namespace {
__global__ void __launch_bounds__(128) texture_rate_kernel(cudaTextureObject_t tex, int n, int steps,
                                                           float *__restrict__ sink) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const float x0 = (float)(t & 31) + 16.f, y0 = (float)((t >> 5) % 32) + 16.f, z0 = (float)((t >> 10) % 32) + 16.f;
    const int dir = blockIdx.x % 72;
    const float th = 0.4f + 0.03f * (float)dir, ph = 0.09f * (float)dir;
    const float dx = sinf(th) * cosf(ph), dy = sinf(th) * sinf(ph), dz = cosf(th);
    float acc = 0.f;
    for (int s = 0; s < steps; ++s) {
        const float u = (float)(s % 24);
        const float2 v = tex3D<float2>(tex, fmaf(dx, u, x0), fmaf(dy, u, y0), fmaf(dz, u, z0));
        acc = fmaf(v.x, v.y, acc);
    }
    if (acc == 12345.678f) sink[t] = acc;  // keeps the fetches live
}
}  // namespace
}  // namespace dc

extern "C" int dc_texture_fetch_rate(int gpu_id, double *fetches_per_s) {
    using namespace dc;
    return guarded([&] {
        if (fetches_per_s == nullptr) throw Error(DC_ERR_VALUE, "'fetches_per_s' must not be NULL.");
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        VolumeArray arr;
        constexpr int n = 64;
        arr.ensure(n, n, n, true, 2);
        cudaStream_t s = ctx.stream;
        {  // fill with (1, 1)
            std::vector<float2> host((size_t)n * n * n, make_float2(1.f, 1.f));
            cudaMemcpy3DParms p{};
            p.srcPtr = make_cudaPitchedPtr(host.data(), n * sizeof(float2), n, n);
            p.dstArray = arr.arr;
            p.extent = make_cudaExtent(n, n, n);
            p.kind = cudaMemcpyHostToDevice;
            DC_CUDA(cudaMemcpy3DAsync(&p, s));
            DC_CUDA(cudaStreamSynchronize(s));
        }
        const cudaTextureObject_t tex = arr.texture(0.0f, kAirDensity);
        int sms = 0, per_sm = 0;
        DC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
        DC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, texture_rate_kernel, 128, 0));
        const int blocks = sms * std::max(per_sm, 1);
        float *sink = static_cast<float *>(ctx.small.ensure((size_t)blocks * 128 * sizeof(float)));
        const int steps = 4096;
        texture_rate_kernel<<<blocks, 128, 0, s>>>(tex, n, 64, sink);
        check_launch("texture_rate_kernel");
        cudaEvent_t a, b;
        DC_CUDA(cudaEventCreate(&a));
        DC_CUDA(cudaEventCreate(&b));
        DC_CUDA(cudaEventRecord(a, s));
        texture_rate_kernel<<<blocks, 128, 0, s>>>(tex, n, steps, sink);
        DC_CUDA(cudaEventRecord(b, s));
        DC_CUDA(cudaEventSynchronize(b));
        float ms = 0.f;
        DC_CUDA(cudaEventElapsedTime(&ms, a, b));
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        check_launch("texture_rate_kernel");
        arr.release();
        *fetches_per_s = (double)blocks * 128.0 * steps / (ms * 1e-3);
    });
}
