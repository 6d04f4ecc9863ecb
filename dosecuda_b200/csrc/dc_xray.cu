// dc_xray.cu — photon radiological depth on a beam's-eye-view ray lattice.
//
// The reference computes every voxel's radiological depth with its own ray
// march (rayTraceKernel, CudaClasses.cu:180-228): 1 mm samples from the voxel
// centre towards the source, WET = -0.05 + 0.1 * sum max(rho, 0) over the K
// samples whose texture coordinate is inside the volume.  At 128^3 that is
// ~3.4e8 trilinear fetches, 36 % of a photon control point.  Neighbouring
// voxels' rays run side by side through the same density, so most of that
// work is repeated.  This file integrates the density once along a lattice of
// rays from the source and lets each voxel interpolate its own sum:
//
//  1. xray_lattice_kernel: rays from the source through a square grid of
//     pitch `pa` on the isocentre plane of the head frame (beam's eye view).
//     One warp per ray walks it in chunks of 32 nodes, 1 mm apart in distance
//     from the source (the same node distances on every ray); lane l fetches
//     node l of the chunk (hardware trilinear filter, 0 outside the volume's
//     texture box), a __shfl_up prefix scan turns the chunk into a running
//     integral G(R) (trapezoid rule), and the 32 warps of a block (32
//     neighbouring rays) store their chunk through shared memory transposed,
//     G[node][ray], so that both the stores here and the voxels' gathers
//     below are coalesced along the lattice rows.
//  2. xray_voxel_kernel: per voxel, K is the exact sample count of the
//     reference's loop (the analytic exit distance, then the reference's own
//     float exit test at the candidates); the voxel's samples k = 0..K-m-1
//     are replaced by the midpoint integral of the density over distances
//     [D-K+m+0.5, D+0.5] from the source, interpolated bilinearly at that
//     distance range from the four lattice rays around the voxel's ray; the
//     last m samples next to the volume's boundary, where the texture filter
//     blends in the border value and neighbouring rays leave the volume at
//     different distances, are fetched exactly.  Where the four rays' sums
//     differ by more than `tau` divided by the voxel's own density (capped at
//     water's; the CCCS weighs a voxel's TERMA by its density, so an air
//     voxel's WET matters little), and the second differences of the 4 x 4 rays around the cell
//     do not show the variation to be near-linear (a density edge running
//     along the beam, the volume's side faces), or the voxel falls outside
//     the lattice, the voxel joins a list instead.
//  3. xray_fallback_kernel: the reference's march, exactly, for the listed
//     voxels (a persistent grid over the device-side count).
//
// Error: the midpoint rule is exact for the texture's piecewise-linear
// density between kinks, and the interpolation error of a smooth field across
// one lattice cell is second order; where the four rays disagree by more than
// tau the exact march runs.  With tau = 0.3 mm of unit density the photon WET
// of a voxel in a field the lattice resolves stays within ~0.03 cm of the
// march, TERMA within ~0.15 % at 6 MV.  The spread does not bound every
// voxel: a ray grazing a voxelised surface (the stair-stepped boundary of a
// body in air) sees structure at the voxel scale, which a lattice of voxel
// pitch aliases, and a voxel's own ray can carry ~1 mm of unit density more
// than all four of its lattice rays (measured: TERMA 0.85 % off on 60 of
// 0.84 M voxels of such a phantom, the dose 0.05 % of its maximum).  The
// electron contamination term is far steeper in WET (its slope at the surface
// is ~1 per cm of WET: 0.03 cm would move a surface voxel's dose by ~3 % of
// the maximum), and it is non-zero only above its fitted depth efd, so a
// voxel whose interpolated WET is below efd + 0.1 cm is marched exactly
// (inline when its ray is short) wherever its four lattice rays disagree by
// more than tau_shallow = 0.01 mm of unit density (0.001 cm of WET); where
// they agree, in air or homogeneous tissue, the interpolation stands (air
// around a patient would otherwise send most of the volume to the march).
// The proton WET never uses this path: there the march is kept bit-exact.
#include <algorithm>
#include <cmath>

#include "dc_common.cuh"
#include "dc_kernels.cuh"
#include "dc_runtime.cuh"

namespace dc {

DC_BOUNDS_WORD

namespace {

constexpr int kRaysPerBlock = 32;  // rays of one lattice row per block, one warp each
constexpr int kMaxTail = 32;       // exact boundary samples before the whole march is taken instead
constexpr int kInlineMarch = 64;   // longest ray a shallow voxel marches inline instead of joining the list

__device__ __forceinline__ bool march_inside(const Grid &g, const Frame &f, float3 p, float3 u, float t) {
    float3 q;
    q.x = fmaf(u.x, t, p.x);
    q.y = fmaf(u.y, t, p.y);
    q.z = fmaf(u.z, t, p.z);
    return tex_inside(g, tex_coord(g, f, q));
}

__device__ __forceinline__ float march_sample(const Grid &g, const Frame &f, cudaTextureObject_t density, float3 p,
                                              float3 u, float t) {
    float3 q;
    q.x = fmaf(u.x, t, p.x);
    q.y = fmaf(u.y, t, p.y);
    q.z = fmaf(u.z, t, p.z);
    const float3 tc = tex_coord(g, f, q);
    return fmaxf(tex3D<float>(density, tc.x, tc.y, tc.z), 0.0f);
}

// The reference's march (rayTraceKernel) for one voxel, from sample `t0` on,
// added to `wet_sum` in the reference's order.
__device__ float march_from(const Grid &g, const Frame &f, cudaTextureObject_t density, float3 p, float3 u,
                            float t, float wet_sum) {
    while (true) {
        float3 q;
        q.x = fmaf(u.x, t, p.x);
        q.y = fmaf(u.y, t, p.y);
        q.z = fmaf(u.z, t, p.z);
        const float3 tc = tex_coord(g, f, q);
        if (!tex_inside(g, tc)) break;
        wet_sum = fmaf(fmaxf(tex3D<float>(density, tc.x, tc.y, tc.z), 0.0f), 0.1f, wet_sum);
        t += 1.0f;
    }
    return wet_sum;
}

// Exit of the ray from p along u out of the texture box: the distance t_exit,
// the exit face's |cos| to the ray and its voxel spacing.
struct RayExit {
    float t_exit, cos_face, sp_face;
};
__device__ __forceinline__ RayExit ray_exit(const Grid &g, const Frame &f, float3 p, float3 u) {
    RayExit e{3.0e38f, 1.0f, g.sx};
    const float lo[3] = {-0.5f * g.sx - f.isox, -0.5f * g.sy - f.isoy, -0.5f * g.sz - f.isoz};
    const float hi[3] = {((float)g.nx - 0.5f) * g.sx - f.isox, ((float)g.ny - 0.5f) * g.sy - f.isoy,
                         ((float)g.nz - 0.5f) * g.sz - f.isoz};
    const float pp[3] = {p.x, p.y, p.z}, uu[3] = {u.x, u.y, u.z}, ss[3] = {g.sx, g.sy, g.sz};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (uu[a] == 0.0f) continue;
        const float t = ((uu[a] > 0.0f ? hi[a] : lo[a]) - pp[a]) / uu[a];
        if (t < e.t_exit) {
            e.t_exit = t;
            e.cos_face = fabsf(uu[a]);
            e.sp_face = ss[a];
        }
    }
    return e;
}

// The reference loop's sample count K: the first t = 0, 1, 2, ... whose
// sample is outside the texture box.  Each texture coordinate is a monotone
// function of t (fma and the rounding are monotone), so the inside samples
// form a prefix, and K is the analytic exit distance corrected by the
// reference's own float test at the candidates.  Returns -1 when four steps
// either way do not settle it.
__device__ __forceinline__ int exact_sample_count(const Grid &g, const Frame &f, float3 p, float3 u, float t_exit) {
    int K = (int)fminf(floorf(t_exit), 1.0e6f) + 1;
    if (K < 1) K = 1;
    for (int it = 0; it < 4 && K > 1 && !march_inside(g, f, p, u, (float)(K - 1)); ++it) --K;
    for (int it = 0; it < 4 && march_inside(g, f, p, u, (float)K); ++it) ++K;
    if (!(march_inside(g, f, p, u, (float)(K - 1)) || K == 1) || march_inside(g, f, p, u, (float)K)) return -1;
    return K;
}

// The reference's march over its K inside samples, summed in its order, with
// the loop unrolled so that several texture fetches are in flight at once
// (the fetch addresses do not depend on the sum).  Equal to march_from from
// t = 0 bit for bit.
__device__ __forceinline__ float march_count(const Grid &g, const Frame &f, cudaTextureObject_t density, float3 p,
                                             float3 u, int K) {
    float wet_sum = -0.05f;
#pragma unroll 8
    for (int t = 0; t < K; ++t) wet_sum = fmaf(march_sample(g, f, density, p, u, (float)t), 0.1f, wet_sum);
    return wet_sum;
}

}  // namespace

__global__ void __launch_bounds__(1024) xray_lattice_kernel(Grid g, Frame f, XrayLattice L,
                                                            cudaTextureObject_t density, float *__restrict__ G) {
    __shared__ float tile[32][33];  // [node in chunk][ray in block], padded
    const int lane = threadIdx.x & 31;
    const int w = threadIdx.x >> 5;  // ray of this warp within the block
    const int ib = blockIdx.y;
    const int ia = blockIdx.x * kRaysPerBlock + w;
    const bool ray_ok = ia < L.na;
    // ray direction from the source through (a, b) on the isocentre plane
    const float a = L.a0 + (float)ia * L.pa, b = L.b0 + (float)ib * L.pa;
    float3 d;
    d.x = a * L.ex.x + b * L.ey.x - L.sad * L.ez.x;
    d.y = a * L.ex.y + b * L.ey.y - L.sad * L.ez.y;
    d.z = a * L.ex.z + b * L.ey.z - L.sad * L.ez.z;
    const float rn = rnorm3df(d.x, d.y, d.z);
    d.x *= rn;
    d.y *= rn;
    d.z *= rn;
    float carry = 0.0f;
    const long long row = (long long)L.na * L.nb;
    for (int c0 = 0; c0 < L.nm; c0 += 32) {
        const int m = c0 + lane;
        float rho = 0.0f;
        if (ray_ok && m < L.nm) {
            const float R = (float)(L.m0 + m);
            const float3 q = make_float3(fmaf(d.x, R, L.src.x), fmaf(d.y, R, L.src.y), fmaf(d.z, R, L.src.z));
            const float3 tc = tex_coord(g, f, q);
            if (tex_inside(g, tc)) rho = fmaxf(tex3D<float>(density, tc.x, tc.y, tc.z), 0.0f);
        }
        // inclusive prefix sum of the chunk
        float s = rho;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float v = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += v;
        }
        // trapezoid rule from node 0 (outside the volume, rho = 0):
        // G_m = sum_{j<=m} rho_j - rho_m / 2
        tile[lane][w] = carry + s - 0.5f * rho;
        carry += __shfl_sync(0xffffffffu, s, 31);
        __syncthreads();
        // warp w stores node c0 + w of the block's 32 rays (lane = ray)
        const int mo = c0 + w;
        const int iao = blockIdx.x * kRaysPerBlock + lane;
        if (mo < L.nm && iao < L.na) {
            const long long idx = (long long)mo * row + (long long)ib * L.na + iao;
            if (DC_IN_BOUNDS(idx, (long long)L.nm * row, 40)) G[idx] = tile[w][lane];
        }
        __syncthreads();
    }
}

__global__ void __launch_bounds__(128, 10) xray_voxel_kernel(Grid g, Frame f, XrayLattice L, cudaTextureObject_t density,
                                                         const float *__restrict__ G, float *__restrict__ wet,
                                                         int *__restrict__ list, unsigned *__restrict__ n_list) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= g.nx || j >= g.ny) return;
    const long long v = (long long)i + (long long)g.nx * (j + (long long)g.ny * k);
    const float3 p = voxel_xyz(g, f, i, j, k);
    const float3 u = unit_to_source(f, p);

    bool exact = false;
    float wet_sum = 0.0f;
    // --- exit distance along u from the texture box [lo, hi) per axis, the
    // exit face, and the exact sample count K of the reference's loop
    const RayExit ex = ray_exit(g, f, p, u);
    const float cos_face = ex.cos_face, sp_face = ex.sp_face;
    int K = exact_sample_count(g, f, p, u, ex.t_exit);
    if (K < 0) {
        exact = true;
        K = 1;
    }

    // --- exact boundary samples: the blend zone of the texture filter plus the
    // spread of exit distances between the voxel's ray and its lattice rays
    const float D = norm3df(L.src.x - p.x, L.src.y - p.y, L.src.z - p.z);
    const float sin_face = sqrtf(fmaxf(0.0f, 1.0f - cos_face * cos_face));
    const float lat = L.pa * 1.4143f * (D - (float)K) / L.sad;  // corner-ray offset at the exit
    const float tail_f = 0.5f * sp_face / fmaxf(cos_face, 1e-3f) + lat * sin_face / fmaxf(cos_face, 1e-3f) + 1.0f;
    int mt = (int)ceilf(fminf(tail_f, (float)(kMaxTail + 1)));
    if (mt > kMaxTail) exact = true;
    if (mt > K) mt = K;

    float S = 0.0f, spread = 0.0f;
    bool shallow_unsure = false;  // the lattice's sum is not known to 0.001 cm of WET
    if (!exact && K > mt) {
        const float3 h = image_to_head<true>(f, p);
        const float den = L.sad - h.z;
        const float fa = (h.x * L.sad / den - L.a0) * L.inv_pa;
        const float fb = (h.y * L.sad / den - L.b0) * L.inv_pa;
        const float xa = floorf(fa), xb = floorf(fb);
        const float x_hi = D + 0.5f - (float)L.m0;
        const float x_lo = D - (float)(K - mt) + 0.5f - (float)L.m0;
        const float n_hi = floorf(x_hi), n_lo = floorf(x_lo);
        // written so that a NaN anywhere fails the test
        const bool on_lattice = den > 0.0f && xa >= 0.0f && xb >= 0.0f && xa <= (float)(L.na - 2) &&
                                xb <= (float)(L.nb - 2) && n_lo >= 0.0f && n_hi <= (float)(L.nm - 2) && n_lo <= n_hi;
        if (!on_lattice) {
            exact = true;
        } else {
            const int ia = (int)xa, ib = (int)xb, mh = (int)n_hi, ml = (int)n_lo;
            const float wa = fa - xa, wb = fb - xb, fh = x_hi - n_hi, fl = x_lo - n_lo;
            const long long row = (long long)L.na * L.nb, total = row * L.nm;
            (void)total;  // read by the bounds checks of debug builds
            // the lattice ray (ra, rb)'s integral over the voxel's distance range
            auto cval = [&](int ra, int rb) -> float {
                const long long r = (long long)rb * L.na + ra;
                const long long h0 = (long long)mh * row + r, l0 = (long long)ml * row + r;
                float gh0 = 0.f, gh1 = 0.f, gl0 = 0.f, gl1 = 0.f;
                if (DC_IN_BOUNDS(h0 + row, total, 41) && DC_IN_BOUNDS(h0, total, 41)) {
                    gh0 = __ldg(G + h0);
                    gh1 = __ldg(G + h0 + row);
                }
                if (DC_IN_BOUNDS(l0 + row, total, 42) && DC_IN_BOUNDS(l0, total, 42)) {
                    gl0 = __ldg(G + l0);
                    gl1 = __ldg(G + l0 + row);
                }
                return fmaf(fh, gh1 - gh0, gh0) - fmaf(fl, gl1 - gl0, gl0);
            };
            float c[4];
            float cmin = 3.0e38f, cmax = -3.0e38f;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                c[q] = cval(ia + (q & 1), ib + (q >> 1));
                cmin = fminf(cmin, c[q]);
                cmax = fmaxf(cmax, c[q]);
            }
            spread = cmax - cmin;
            // Bilinear interpolation is exact for a field varying linearly
            // between the rays (a smooth gradient, e.g. behind a curved body
            // surface), so where the corners spread more than tau the error is
            // estimated from the second differences of the 4 x 4 rays around
            // the cell: |f - bilinear| <= (|f_aa| + |f_bb|) / 8 for a quadratic
            // field.  Computed on demand (+inf where the stencil leaves the
            // lattice).
            float est = -1.0f;
            auto estimate = [&]() -> float {
                if (est >= 0.0f) return est;
                if (!(xa >= 1.0f && xb >= 1.0f && xa <= (float)(L.na - 3) && xb <= (float)(L.nb - 3))) {
                    est = INFINITY;
                    return est;
                }
                float sv[4][4];
#pragma unroll
                for (int rb = 0; rb < 4; ++rb)
#pragma unroll
                    for (int ra = 0; ra < 4; ++ra) {
                        const bool corner = (rb == 1 || rb == 2) && (ra == 1 || ra == 2);
                        sv[rb][ra] = corner ? c[(rb - 1) * 2 + (ra - 1)] : cval(ia - 1 + ra, ib - 1 + rb);
                    }
                float curv = 0.0f;
#pragma unroll
                for (int rb = 1; rb <= 2; ++rb)
#pragma unroll
                    for (int ra = 1; ra <= 2; ++ra) {
                        const float d2a = sv[rb][ra - 1] - 2.0f * sv[rb][ra] + sv[rb][ra + 1];
                        const float d2b = sv[rb - 1][ra] - 2.0f * sv[rb][ra] + sv[rb + 1][ra];
                        curv = fmaxf(curv, fabsf(d2a) + fabsf(d2b));
                    }
                est = 0.125f * curv;
                return est;
            };
            // The CCCS weights the TERMA sampled at a point by the density
            // there (max(rho, 0.0012) x spacing), so a WET error enters the
            // dose in proportion to the voxel's own density: past tau the
            // tests are weighed by it, capped at water's (lung and air looser,
            // water and denser as tau), so the density is fetched only then.
            bool ok = spread <= L.tau;
            if (!ok) {
                const float rho_v = tex3D<float>(density, (float)i + 0.5f, (float)j + 0.5f, (float)k + 0.5f);
                const float wv = fmaxf(fminf(rho_v, 1.0f), L.rho_floor);
                ok = spread * wv <= L.tau || (spread * wv <= L.tau_big && estimate() * wv <= L.tau_curv);
            }
            if (!ok) {
                exact = true;
            } else {
                const float top = fmaf(wa, c[1] - c[0], c[0]);
                const float bot = fmaf(wa, c[3] - c[2], c[2]);
                S = fmaf(wb, bot - top, top);
                // a voxel in the electron term's range needs its sum to 0.001
                // cm; the second-difference estimate is not trusted that far
                // (it missed voxel-scale structure on a body in air)
                shallow_unsure = !(spread <= L.tau_shallow);
            }
        }
    } else if (!exact) {
        mt = K;  // short ray: every sample exactly
    }
    if (!exact) {
        if (mt == K) {
            wet_sum = march_count(g, f, density, p, u, K);  // the reference's own sum
        } else {
            float tail = 0.0f;
            for (int t = K - mt; t < K; ++t) tail += march_sample(g, f, density, p, u, (float)t);
            wet_sum = fmaf(S + tail, 0.1f, -0.05f);
            // Shallow voxels: the electron contamination term falls by ~1 % of
            // its value per 0.01 cm of WET there, far steeper than TERMA, so
            // where the four lattice rays disagree by more than tau_shallow
            // the depth is marched exactly (short rays inline, long ones join
            // the list).  Where they agree (air, homogeneous tissue) the
            // interpolation is kept.
            if (!(wet_sum >= L.wet_exact) && shallow_unsure) {
                if (K <= kInlineMarch)
                    wet_sum = march_count(g, f, density, p, u, K);
                else
                    exact = true;
            }
        }
    }
    // Voxels for the exact march go to the list in warp order (one atomic per
    // warp), so neighbouring rays stay together there and share texture lines.
    {
        const unsigned live = __activemask();
        const unsigned bal = __ballot_sync(live, exact);
        if (exact) {
            const int lane = (threadIdx.y * blockDim.x + threadIdx.x) & 31;
            const int leader = __ffs(bal) - 1;
            unsigned base = 0;
            if (lane == leader) base = atomicAdd(n_list, (unsigned)__popc(bal));
            base = __shfl_sync(bal, base, leader);
            const unsigned slot = base + __popc(bal & ((1u << lane) - 1u));
            if (DC_IN_BOUNDS(slot, g.n(), 43)) list[slot] = (int)v;
            return;
        }
    }
    if (DC_IN_BOUNDS(v, g.n(), 44)) wet[v] = wet_sum;
}

__global__ void __launch_bounds__(128) xray_fallback_kernel(Grid g, Frame f, cudaTextureObject_t density,
                                                            const int *__restrict__ list,
                                                            const unsigned *__restrict__ n_list,
                                                            float *__restrict__ wet) {
    const unsigned n = *n_list;
    const int plane = g.nx * g.ny;
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int v = DC_IN_BOUNDS(t, g.n(), 45) ? __ldg(list + t) : -1;
        if (!DC_IN_BOUNDS(v, g.n(), 45)) continue;
        const int k = v / plane;
        const int rem = v - k * plane;
        const int j = rem / g.nx;
        const int i = rem - j * g.nx;
        const float3 p = voxel_xyz(g, f, i, j, k);
        const float3 u = unit_to_source(f, p);
        const int K = exact_sample_count(g, f, p, u, ray_exit(g, f, p, u).t_exit);
        wet[v] = K >= 0 ? march_count(g, f, density, p, u, K) : march_from(g, f, density, p, u, 0.0f, -0.05f);
    }
}

DC_BOUNDS_TAKE(take_bounds_xray)

bool plan_xray_lattice(const Grid &g, const Frame &f, XrayLattice &L) {
    L = XrayLattice{};
    L.src = make_float3(f.srcx, f.srcy, f.srcz);
    const double sad = std::sqrt((double)f.srcx * f.srcx + (double)f.srcy * f.srcy + (double)f.srcz * f.srcz);
    if (!(sad > 0.0)) return false;
    L.sad = (float)sad;
    L.ex = head_to_image<true>(f, make_float3(1.f, 0.f, 0.f));
    L.ey = head_to_image<true>(f, make_float3(0.f, 1.f, 0.f));
    L.ez = head_to_image<true>(f, make_float3(0.f, 0.f, 1.f));
    // the lattice assumes the source on the head frame's +z axis at the source distance
    const float3 s_head = head_to_image<true>(f, make_float3(0.f, 0.f, (float)sad));
    if (std::fabs(s_head.x - f.srcx) + std::fabs(s_head.y - f.srcy) + std::fabs(s_head.z - f.srcz) > 1e-3 * sad)
        return false;
    // the texture box in image coordinates (relative to the isocentre)
    const double lo[3] = {-0.5 * g.sx - f.isox, -0.5 * g.sy - f.isoy, -0.5 * g.sz - f.isoz};
    const double hi[3] = {(g.nx - 0.5) * g.sx - f.isox, (g.ny - 0.5) * g.sy - f.isoy, (g.nz - 0.5) * g.sz - f.isoz};
    double amin = 1e300, amax = -1e300, bmin = 1e300, bmax = -1e300, rmax = 0.0;
    for (int c = 0; c < 8; ++c) {
        const float3 q = make_float3((float)((c & 1) ? hi[0] : lo[0]), (float)((c & 2) ? hi[1] : lo[1]),
                                     (float)((c & 4) ? hi[2] : lo[2]));
        const float3 h = image_to_head<true>(f, q);
        const double den = sad - h.z;
        if (den < 1.0) return false;  // the source sits inside or next to the volume
        amin = std::min(amin, h.x * sad / den);
        amax = std::max(amax, h.x * sad / den);
        bmin = std::min(bmin, h.y * sad / den);
        bmax = std::max(bmax, h.y * sad / den);
        const double dx = q.x - f.srcx, dy = q.y - f.srcy, dz = q.z - f.srcz;
        rmax = std::max(rmax, std::sqrt(dx * dx + dy * dy + dz * dz));
    }
    // nearest point of the box to the source
    double d2 = 0.0;
    const double s[3] = {f.srcx, f.srcy, f.srcz};
    for (int a = 0; a < 3; ++a) {
        const double e = s[a] < lo[a] ? lo[a] - s[a] : (s[a] > hi[a] ? s[a] - hi[a] : 0.0);
        d2 += e * e;
    }
    const double rmin = std::sqrt(d2);
    const double pa = std::min(g.sx, std::min(g.sy, g.sz));
    L.pa = (float)pa;
    L.inv_pa = (float)(1.0 / pa);
    L.a0 = (float)(amin - 2.0 * pa);
    L.b0 = (float)(bmin - 2.0 * pa);
    L.na = (int)std::ceil((amax - amin) / pa) + 5;
    L.nb = (int)std::ceil((bmax - bmin) / pa) + 5;
    L.m0 = (int)std::floor(rmin) - 2;
    L.nm = (int)std::ceil(rmax) - L.m0 + 3;
    L.tau = 0.3f;  // mm x unit density: 0.03 cm of WET
    const double bytes = (double)L.na * L.nb * L.nm * sizeof(float);
    if (L.na < 2 || L.nb < 2 || L.nm < 2 || L.nb > 65535 || bytes > 2.0e9) return false;
    return true;
}

void launch_xray_depth(DeviceContext &ctx, const Grid &g, const Frame &f, cudaTextureObject_t density, float *wet,
                       int *list, unsigned *n_list, DeviceBuffer &lattice, unsigned *stats, float wet_exact,
                       cudaStream_t s) {
    XrayLattice L;
    if (!(wet_exact < INFINITY) || !plan_xray_lattice(g, f, L)) {
        launch_wet_march(ctx, g, f, density, wet, s);
        if (stats != nullptr) DC_CUDA(cudaMemsetAsync(stats, 0xff, sizeof(unsigned), s));  // all voxels marched
        return;
    }
    L.wet_exact = wet_exact;
    L.rho_floor = 0.05f;    // smallest density the spread test weighs by
    L.tau_big = 3.0f;       // mm x density: largest spread accepted on a small second-difference estimate
    L.tau_curv = 0.1f;      // mm x density: largest second-difference error estimate accepted
    L.tau_shallow = 0.01f;  // mm x density: 0.001 cm of WET, ~0.2 % of the electron term at the surface
    float *G = static_cast<float *>(lattice.ensure((size_t)L.na * L.nb * L.nm * sizeof(float)));
    {
        KernelTimer kt(ctx, "xray_lattice", s);
        const dim3 grid((unsigned)((L.na + kRaysPerBlock - 1) / kRaysPerBlock), (unsigned)L.nb, 1);
        xray_lattice_kernel<<<grid, 32 * kRaysPerBlock, 0, s>>>(g, f, L, density, G);
        check_launch("xray_lattice_kernel");
    }
    DC_CUDA(cudaMemsetAsync(n_list, 0, sizeof(unsigned), s));
    {
        KernelTimer kt(ctx, "xray_voxel", s);
        const dim3 grid((unsigned)((g.nx + 31) / 32), (unsigned)((g.ny + 3) / 4), (unsigned)g.nz);
        xray_voxel_kernel<<<grid, dim3(32, 4, 1), 0, s>>>(g, f, L, density, G, wet, list, n_list);
        check_launch("xray_voxel_kernel");
    }
    {
        KernelTimer kt(ctx, "xray_fallback", s);
        int sms = 0, per_sm = 0;
        DC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
        DC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, xray_fallback_kernel, 128, 0));
        const long long want = (g.n() + 127) / 128;
        const unsigned blocks = (unsigned)std::max(1LL, std::min<long long>(want, (long long)sms * std::max(per_sm, 1)));
        xray_fallback_kernel<<<blocks, 128, 0, s>>>(g, f, density, list, n_list, wet);
        check_launch("xray_fallback_kernel");
    }
    if (stats != nullptr) DC_CUDA(cudaMemcpyAsync(stats, n_list, sizeof(unsigned), cudaMemcpyDeviceToDevice, s));
}

}  // namespace dc
