// dc_proton.cu — double-Gaussian proton pencil-beam dose.
//
// Restates pencilBeamKernel (IMPTClasses.cu:204-271) and its helpers
// (interpolateProtonLUT :69-92, sigmaAir :94-102, nuclearHalo :104-121,
// caxDistance :123-133).  For a voxel with smoothed WET w (mm) and an energy
// layer with range R80, skipped when w > 1.1*R80:
//   idd, sigma_mcs  = linear interpolation of the layer's LUT at depth w
//   sigma_air       = A d^2 + B d + C,  d = |voxel - source| - w + 0.7 R80
//   sigma_t         = sigma_air + sigma_mcs
//   sigma_h, w_h    = empirical nuclear halo (function of w, R80)
//   sigma_ht        = hypot(sigma_t, sigma_h)
//   D += sum_spots MU * [ (1-w_h) idd/(2 pi sigma_t^2)  exp(-r^2/2 sigma_t^2)
//                        +   w_h  idd/(2 pi sigma_ht^2) exp(-r^2/2 sigma_ht^2) ]
// with r^2 the squared distance from the voxel (BEV coordinates) to the
// spot's divergent axis.
//
// B200 mapping (instead of one thread per (voxel, layer) with a global
// atomicAdd per pair of the reference): a CTA owns a 16x8x4 tile of voxels,
// two voxels per thread, and walks all energy layers.  Per layer
// the CTA stages the layer's LUT rows and spot records in shared memory
// (broadcast reads in the spot loop); each thread keeps its voxels' dose in
// registers across layers and writes each voxel once — no atomics, so the
// result is deterministic.  The spot loop is two exponentials per
// (voxel, spot) pair on the special-function unit (ex2.approx with the
// log2(e) factor folded into the per-voxel Gaussian scales) plus ~12 FP32
// operations.  The FP32 part runs on the paired-lane f32x2 instructions of
// sm_100 (a thread's two voxels share one issue; same IEEE operations, same
// bits), which leaves the kernel bound by the SFU rate and instruction issue.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/dosecuda.h"
#include "dc_common.cuh"
#include "dc_kernels.cuh"
#include "dc_runtime.cuh"

namespace dc {

DC_BOUNDS_WORD

constexpr int kPbThreadsX = 32;
constexpr int kPbThreadsY = 8;
constexpr int kPbVoxY = 2;      // voxels per thread
constexpr int kPbSpotChunk = 512;
// Voxel tile of one CTA: the 32 lanes of a warp split kPbLanesX along x and
// kPbLanesZ along z, the warps (threadIdx.y) lie along y, and a thread's VY
// voxels step along z, so a tile is kPbLanesX x TY x (kPbLanesZ * VY) voxels
// (16 x 8 x 4 for the default shape).  A tile compact in all three axes has
// a smaller beam's-eye-view footprint whatever the beam direction, which
// keeps the per-CTA lateral cut-off tighter: a flat 32 x 16 x 1 tile reaches
// 64 mm across at 2 mm voxels and evaluates every spot within the cut-off of
// any of its voxels for all 512 of them.  Measured (96^3 beam; 4 plans of the
// batched workload): 32x16x1 0.195-0.205 ms / 18.0 ms, 8x8x8 0.181-0.186 /
// 17.0, 16x8x4 0.184 / 16.7, 4x8x16 0.188 / 19.1.
constexpr int kPbLanesX = 16;
constexpr int kPbLanesZ = kPbThreadsX / kPbLanesX;
static_assert(kPbLanesX * kPbLanesZ == kPbThreadsX, "lanes of a warp tile x and z");
template <int TY, int VY>
struct PbTileShape {
    static constexpr int x = kPbLanesX, y = TY, z = kPbLanesZ * VY;
};
// Tiles of a grid along each axis for the shape, and the voxel (i, j, k) of
// this thread's voxel v in tile (bx, by, bz) (possibly outside the grid).
template <int TY, int VY>
__host__ __device__ __forceinline__ int3 pb_tiles(const Grid &g) {
    using S = PbTileShape<TY, VY>;
    return make_int3((g.nx + S::x - 1) / S::x, (g.ny + S::y - 1) / S::y, (g.nz + S::z - 1) / S::z);
}
template <int TY, int VY>
__device__ __forceinline__ int3 pb_tile_voxel(int bx, int by, int bz, int v) {
    using S = PbTileShape<TY, VY>;
    return make_int3(bx * S::x + (int)(threadIdx.x % kPbLanesX), by * S::y + (int)threadIdx.y,
                     bz * S::z + (int)(threadIdx.x / kPbLanesX) + kPbLanesZ * v);
}
static_assert(2 * kPbThreadsX * kPbThreadsY == kPbSpotChunk, "two spots per thread per staging round");

void build_proton_tables(const float *spots, int n_spots, const float *dvp, int n_energies, int dvp_len,
                         float vsadx, float vsady, std::vector<LayerRec> &layers,
                         std::vector<SpotRec> &spot_recs) {
    if (n_spots <= 0) throw Error(DC_ERR_VALUE, "'spot_list' must hold at least one spot.");
    if (n_energies <= 0) throw Error(DC_ERR_VALUE, "'divergence_params' must hold at least one energy.");
    if (dvp_len < 5) throw Error(DC_ERR_VALUE, "'divergence_params' rows must hold energy, R80, A, B, C.");
    struct Tmp {
        int e;
        int order;
        float x, y, mu;
    };
    std::vector<Tmp> tmp((size_t)n_spots);
    for (int s = 0; s < n_spots; ++s) {
        const float *r = spots + 4 * (size_t)s;
        // static_cast<int> truncation of the energy column (dosemodule.cu:220).
        const float ef = r[3];
        if (!(ef > -1.0f) || !(ef < (float)n_energies)) {
            throw Error(DC_ERR_VALUE, "spot " + std::to_string(s) + ": energy id " + std::to_string(ef) +
                                          " outside the beam model's " + std::to_string(n_energies) +
                                          " energies.");
        }
        tmp[s] = {static_cast<int>(ef), s, r[0], r[1], r[2]};
    }
    // Sort by energy id (dosemodule.cu:224); stable, so the summation order is
    // reproducible.
    std::stable_sort(tmp.begin(), tmp.end(), [](const Tmp &a, const Tmp &b) { return a.e < b.e; });
    spot_recs.resize((size_t)n_spots);
    for (int s = 0; s < n_spots; ++s) {
        SpotRec &o = spot_recs[s];
        o.x = tmp[s].x;
        o.y = tmp[s].y;
        o.mu = tmp[s].mu;
        o.tx = tmp[s].x / vsadx;
        o.ty = tmp[s].y / vsady;
        o.inv_t2 = 1.0f / (o.tx * o.tx + o.ty * o.ty + 1.0f);
        o.orig = tmp[s].order;
        o.pad1 = 0.f;
    }
    layers.clear();
    int s = 0;
    while (s < n_spots) {
        int e = tmp[s].e;
        int t = s;
        while (t < n_spots && tmp[t].e == e) ++t;
        LayerRec L;
        L.spot_start = s;
        L.n_spots = t - s;
        L.energy_id = e;
        const float *row = dvp + (size_t)dvp_len * e;
        L.r80 = row[1];
        L.A = row[2];
        L.B = row[3];
        L.C = row[4];
        L.rcut = INFINITY;  // set on the device by layer_rcut_kernel
        layers.push_back(L);
        s = t;
    }
}

// Per (voxel, layer) Gaussian parameters.  Returns false if the layer does
// not reach the voxel (w > 1.1 R80).
struct PbVoxel {
    float pf, hf;      // primary / halo amplitude (idd/(2 pi sigma^2) weighted)
    float ps2, hs2;    // -0.5/sigma^2 * log2(e)
};

__device__ __forceinline__ bool pb_voxel_layer(const LayerRec &L, const float *s_depth, const float *s_sigma,
                                               const float *s_idd, int lut_len, float wet_mm,
                                               float dist_src, PbVoxel &o) {
    const float r80 = L.r80;
    if (wet_mm > 1.1f * r80) return false;
    // interpolateProtonLUT (IMPTClasses.cu:69-92)
    const int i = lower_bound(s_depth, lut_len, wet_mm);
    float idd, sig;
    if (i == lut_len) {
        idd = s_idd[i - 1];
        sig = s_sigma[i - 1];
    } else if (i == 0) {
        idd = s_idd[0];
        sig = s_sigma[0];
    } else {
        const float fac = (wet_mm - s_depth[i - 1]) / (s_depth[i] - s_depth[i - 1]);
        idd = fmaf(s_idd[i] - s_idd[i - 1], fac, s_idd[i - 1]);
        sig = fmaf(s_sigma[i] - s_sigma[i - 1], fac, s_sigma[i - 1]);
    }
    // sigmaAir (IMPTClasses.cu:94-102)
    const float d = dist_src - wet_mm + (0.7f * r80);
    const float sigma_t = fmaf(fmaf(L.A, d, L.B), d, L.C) + sig;
    // nuclearHalo (IMPTClasses.cu:104-121)
    const float w = clampf(wet_mm, 0.1f, r80 - 0.1f);
    const float hs_ = 2.85f + (0.0014f * r80 * logf(w + 3.0f)) + (0.06f * w) - (7.4e-5f * sqr(w)) -
                      ((0.22f * r80) / sqr(w - r80 - 5.0f));
    const float hw_ = 0.052f * logf(1.13f + (w / (11.2f - (0.023f * r80)))) +
                      (0.35f * ((0.0017f * sqr(r80)) - r80) / (sqr(r80 + 3.0f) - sqr(w))) -
                      (1.61e-9f * w * sqr(r80 + 3.0f));
    const float sigma_h = fmaxf(hs_, 0.0f);
    const float wh = clampf(hw_, 0.0f, 0.9f);
    const float sigma_ht = hypotf(sigma_t, sigma_h);
    o.pf = (1.0f - wh) * idd / (2.0f * CUDART_PI_F * sqr(sigma_t));
    o.hf = wh * idd / (2.0f * CUDART_PI_F * sqr(sigma_ht));
    o.ps2 = (sigma_t != 0.0f ? -0.5f / sqr(sigma_t) : -INFINITY) * kLog2e;
    o.hs2 = (sigma_ht != 0.0f ? -0.5f / sqr(sigma_ht) : -INFINITY) * kLog2e;
    return true;
}

// Squared distance from a voxel to one spot's divergent axis (caxDistance,
// IMPTClasses.cu:123-133), r^2 = |ray|^2 - (t.ray)^2 / |t|^2 with
// ray = (hx - sx, hy - sy, hz) and t = (tx, ty, -1), evaluated as
// |ray x t|^2 / |t|^2 (the same quantity by Lagrange's identity).  The
// reference's form subtracts two squares of ~|hz|^2 (4e4 mm^2 at 200 mm from
// the isocentre), so its float rounding moves r^2 by ~0.01 mm^2 and a far
// pair's Gaussian by ~1e-4; the cross product has no such cancellation and
// holds the FP64 value to a few ulps of r^2 itself.  With t_z = -1:
//   ray x t = (-(ry + hz ty), rx + hz tx, rx ty - ry tx).
__device__ __forceinline__ float pb_r2(float hx, float hy, float hz, float sx, float sy, float tx, float ty,
                                       float inv_t2) {
    const float rx = __fsub_rn(hx, sx), ry = __fsub_rn(hy, sy);
    const float cu = __fmaf_rn(hz, tx, rx), cw = __fmaf_rn(hz, ty, ry);
    const float cc = __fmaf_rn(rx, ty, __fmul_rn(ry, -tx));
    return __fmul_rn(__fmaf_rn(cu, cu, __fmaf_rn(cw, cw, __fmul_rn(cc, cc))), inv_t2);
}

// The same for two voxels (packed lanes) on the paired-lane FP32
// instructions of sm_100 (fma.rn.f32x2 and friends: one issue for both
// voxels).  Each lane performs exactly pb_r2's sequence (the negations are
// moved onto exactly negated operands: nsx = -sx, nsy = -sy, ntx = -tx), so
// the packed and the scalar forms agree bit for bit.
__device__ __forceinline__ float2 pb_r2_pair(float2 hx, float2 hy, float2 hz, float2 nsx, float2 nsy, float2 tx,
                                            float2 ty, float2 ntx, float2 inv_t2) {
    const float2 rx = __fadd2_rn(hx, nsx);
    const float2 ry = __fadd2_rn(hy, nsy);
    const float2 cu = __ffma2_rn(hz, tx, rx);
    const float2 cw = __ffma2_rn(hz, ty, ry);
    const float2 cc = __ffma2_rn(rx, ty, __fmul2_rn(ry, ntx));
    return __fmul2_rn(__ffma2_rn(cu, cu, __ffma2_rn(cw, cw, __fmul2_rn(cc, cc))), inv_t2);
}

__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 exp2_pair(float2 x) { return make_float2(fast_exp2(x.x), fast_exp2(x.y)); }

// Lateral cut-off per layer.  A spot's Gaussians are negligible beyond
// 6 sigma_ht (exp(-18) = 1.5e-8 of the halo peak); sigma_ht = hypot(sigma_t,
// sigma_h) is bounded over every voxel the layer can reach:
//  * |sigma_mcs| by the largest LUT sigma at depths up to 1.1 R80 (linear
//    interpolation stays between table entries);
//  * |sigma_air| by the quadratic's extremes over the range of
//    d = |voxel - source| - w + 0.7 R80 for voxels of the volume;
//  * sigma_h by sampling the halo formula over [0.1, R80 - 0.1] mm.
// One warp per layer: the lanes share the LUT scan and the halo-sigma
// samples, and the maxima are combined with shuffles.
__global__ void __launch_bounds__(32) layer_rcut_kernel(Grid g, Frame f, LayerRec *layers, int n_layers,
                                                        const float *lut_depths, const float *lut_sigmas,
                                                        int lut_len) {
    const int l = blockIdx.x;
    const int lane = threadIdx.x;
    if (l >= n_layers) return;
    LayerRec &L = layers[l];
    // source distance range over the volume's bounding box (image frame, relative to iso)
    const float lo[3] = {-f.isox - 0.5f * g.sx, -f.isoy - 0.5f * g.sy, -f.isoz - 0.5f * g.sz};
    const float hi[3] = {(g.nx - 0.5f) * g.sx - f.isox, (g.ny - 0.5f) * g.sy - f.isoy, (g.nz - 0.5f) * g.sz - f.isoz};
    const float src[3] = {f.srcx, f.srcy, f.srcz};
    float dmin2 = 0.f, dmax2 = 0.f;
    for (int a = 0; a < 3; ++a) {
        const float c = fminf(fmaxf(src[a], lo[a]), hi[a]);
        dmin2 += sqr(src[a] - c);
        dmax2 += fmaxf(sqr(src[a] - lo[a]), sqr(src[a] - hi[a]));
    }
    const float r80 = L.r80;
    const float wmax = 1.1f * r80;
    const float *D = lut_depths + (size_t)L.energy_id * lut_len;
    const float *S = lut_sigmas + (size_t)L.energy_id * lut_len;
    // |sigma| over the rows up to the first one deeper than wmax (that row
    // included: it brackets wmax from above)
    int q_end = lut_len;
    for (int q0 = 0; q0 < lut_len; q0 += 32) {
        const int q = q0 + lane;
        const bool deeper = q < lut_len && D[q] > wmax;
        const unsigned m = __ballot_sync(0xffffffffu, deeper);
        if (m) {
            q_end = q0 + __ffs(m);  // one past the first deeper row
            break;
        }
    }
    float smcs = 0.f;
    for (int q = lane; q < q_end; q += 32) smcs = fmaxf(smcs, fabsf(S[q]));
    // the halo sigma sampled over [0.1, R80 - 0.1] mm in 0.25 mm steps
    float sh = 0.f;
    const int n_w = r80 - 0.1f >= 0.1f ? (int)floorf((r80 - 0.2f) / 0.25f) + 1 : 0;
    for (int q = lane; q < n_w; q += 32) {
        const float w = 0.1f + 0.25f * (float)q;
        if (w > r80 - 0.1f) break;
        const float h = 2.85f + (0.0014f * r80 * logf(w + 3.0f)) + (0.06f * w) - (7.4e-5f * sqr(w)) -
                        ((0.22f * r80) / sqr(w - r80 - 5.0f));
        sh = fmaxf(sh, h);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        smcs = fmaxf(smcs, __shfl_xor_sync(0xffffffffu, smcs, o));
        sh = fmaxf(sh, __shfl_xor_sync(0xffffffffu, sh, o));
    }
    if (lane != 0) return;
    const float d0 = sqrtf(dmin2) - wmax + 0.7f * r80 - 1.0f;
    const float d1 = sqrtf(dmax2) + 0.5f + 0.7f * r80 + 1.0f;
    auto sair = [&](float d) { return fabsf(fmaf(fmaf(L.A, d, L.B), d, L.C)); };
    float sa = fmaxf(sair(d0), sair(d1));
    if (L.A != 0.0f) {
        const float dv = -L.B / (2.0f * L.A);
        if (dv > d0 && dv < d1) sa = fmaxf(sa, sair(dv));
    }
    const float sht = hypotf(sa + smcs, sh * 1.02f + 0.2f) * 1.01f + 0.5f;
    L.rcut = (sht == sht) ? 6.0f * sht : INFINITY;
}

void launch_layer_rcut(const Grid &g, const Frame &f, LayerRec *layers, int n_layers, const float *lut_depths,
                       const float *lut_sigmas, int lut_len, cudaStream_t s) {
    if (n_layers <= 0) return;
    layer_rcut_kernel<<<n_layers, 32, 0, s>>>(g, f, layers, n_layers, lut_depths, lut_sigmas, lut_len);
    check_launch("layer_rcut_kernel");
}

// The pencil-beam kernel family.  Every member walks the same tiles, layers
// and spots and evaluates the same per-pair influence
//   K_s(v) = pf exp2(ps2 r^2) + hf exp2(hs2 r^2)   (dose per MU),
// so the dose, its adjoint and the influence matrix agree to rounding.
//   kPbDose     dose(v)       = sum_s mu_s K_s(v)          (one write per voxel)
//   kPbAdjoint  grad_mu[s]   += sum_v g(v) K_s(v)          (warp reduction per spot,
//                                                           one FP64 atomic per CTA and spot)
//   kPbSpotMax  spot_max[s]   = max_v K_s(v)
//   kPbCount    counts[v]     = #{s : K_s(v) >= thr[s]}
//   kPbFill     CSR row v     = (s, K_s(v)) for K_s(v) >= thr[s], in spot-table order
//               (run by the kPbCount instantiation with x.row_ptr set: the
//               fill must take exactly the pairs the count took, so both
//               passes evaluate K_s(v) and the test with the same machine
//               code; separately compiled, the per-voxel parameters' plain
//               FP32 expressions may be contracted differently and a pair
//               at its threshold may flip between the passes)
//   list mode   the CTA's voxels are x.list[bx*(threads*VY) + v*threads + tid]
//               instead of an image tile (dose / adjoint of listed voxels)
template <int kMode, int TY, int VY, bool kList = false>
__device__ __forceinline__ void pb_tile(const Grid &g, const Frame &f, const ProtonTables &t,
                                        const float *__restrict__ wet_s, int bx, int by, int bz, float (&acc)[VY],
                                        const PbExtra &x) {
    extern __shared__ float4 smem4[];
    float4 *s_spot_a = smem4;                    // x, y, mu, orig (int bits)
    float4 *s_spot_b = smem4 + kPbSpotChunk;     // tx, ty, inv_t2, threshold
    float *s_acc = reinterpret_cast<float *>(smem4 + 2 * kPbSpotChunk);  // adjoint partial sums
    float *s_lut = s_acc + kPbSpotChunk;
    float *s_depth = s_lut;
    float *s_sigma = s_lut + t.lut_len;
    float *s_idd = s_lut + 2 * t.lut_len;

    constexpr int kThreads = kPbThreadsX * TY;
    constexpr int kSpt = kPbSpotChunk / kThreads;  // spots tested per thread per staging round
    static_assert(kSpt * kThreads == kPbSpotChunk, "staging round must cover the chunk");
    const int tid = threadIdx.y * kPbThreadsX + threadIdx.x;
    const int lane = threadIdx.x;
    const int nthreads = kThreads;
    __syncthreads();  // shared memory of a previous tile (persistent caller) no longer in use

    float hx[VY], hy[VY], hz[VY], wet_mm[VY], dsrc[VY];
    float gv[VY];
    long long vidx[VY];
    long long fill_off[VY], fill_end[VY];
    int cnt[VY];
    bool inside[VY];
#pragma unroll
    for (int v = 0; v < VY; ++v) {
        int ic, jc, kc;
        if constexpr (kList) {
            const int e = bx * (kThreads * VY) + v * kThreads + tid;
            const long long plane = (long long)g.nx * g.ny;
            long long vi = x.list[min(e, x.n_list - 1)];
            const bool valid = vi >= 0 && vi < plane * g.nz;  // out-of-grid entries give 0
            inside[v] = e < x.n_list && valid;
            vidx[v] = valid ? vi : 0;
            kc = (int)(vidx[v] / plane);
            const long long rem = vidx[v] - (long long)kc * plane;
            jc = (int)(rem / g.nx);
            ic = (int)(rem - (long long)jc * g.nx);
        } else {
            const int3 q = pb_tile_voxel<TY, VY>(bx, by, bz, v);
            inside[v] = q.x < g.nx && q.y < g.ny && q.z < g.nz;
            ic = min(q.x, g.nx - 1);
            jc = min(q.y, g.ny - 1);
            kc = min(q.z, g.nz - 1);
            vidx[v] = (long long)ic + (long long)g.nx * (jc + (long long)g.ny * kc);
        }
        cnt[v] = 0;
        const float3 p = voxel_xyz(g, f, ic, jc, kc);
        const float3 h = image_to_head<false>(f, p);
        hx[v] = h.x;
        hy[v] = h.y;
        hz[v] = h.z;
        dsrc[v] = distance_to_source(f, p);
        wet_mm[v] = (DC_IN_BOUNDS(vidx[v], g.n(), 21) ? __ldg(wet_s + vidx[v]) : 0.0f) * 10.0f;
        gv[v] = 0.0f;
        if (kMode == kPbAdjoint) {
            if constexpr (kList)
                gv[v] = inside[v] ? __ldg(x.grad_dose + bx * (kThreads * VY) + v * kThreads + tid) : 0.0f;
            else
                gv[v] = inside[v] ? __ldg(x.grad_dose + vidx[v]) : 0.0f;
        }
        fill_off[v] = fill_end[v] = 0;
        if (kMode == kPbCount && x.row_ptr != nullptr && inside[v]) {
            fill_off[v] = x.row_ptr[vidx[v]];
            fill_end[v] = min(x.row_ptr[vidx[v] + 1], x.cap);  // never past the counted row or the buffers
        }
    }

    // Beam's-eye-view bounding box of the CTA's voxels (for spot culling).
    __shared__ float s_red[TY][6];
    __shared__ float s_bb[6];
    __shared__ int s_wcnt[TY];
    __shared__ float s_sig[TY];
    {
        float b[6] = {INFINITY, -INFINITY, INFINITY, -INFINITY, INFINITY, -INFINITY};
#pragma unroll
        for (int v = 0; v < VY; ++v) {
            if (!inside[v]) continue;
            b[0] = fminf(b[0], hx[v]);
            b[1] = fmaxf(b[1], hx[v]);
            b[2] = fminf(b[2], hy[v]);
            b[3] = fmaxf(b[3], hy[v]);
            b[4] = fminf(b[4], hz[v]);
            b[5] = fmaxf(b[5], hz[v]);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int c = 0; c < 6; c += 2) {
                b[c] = fminf(b[c], __shfl_xor_sync(0xffffffffu, b[c], o));
                b[c + 1] = fmaxf(b[c + 1], __shfl_xor_sync(0xffffffffu, b[c + 1], o));
            }
        }
        if (lane == 0) {
#pragma unroll
            for (int c = 0; c < 6; ++c) s_red[threadIdx.y][c] = b[c];
        }
        __syncthreads();
        if (tid < 6) {
            float r = s_red[0][tid];
            for (int w = 1; w < TY; ++w) r = (tid & 1) ? fmaxf(r, s_red[w][tid]) : fminf(r, s_red[w][tid]);
            s_bb[tid] = r;
        }
        __syncthreads();
    }
    const float bx0 = s_bb[0], bx1 = s_bb[1], by0 = s_bb[2], by1 = s_bb[3], bz0 = s_bb[4], bz1 = s_bb[5];

    for (int l = 0; l < t.n_layers; ++l) {
        const LayerRec L = t.layers[l];
        // Cheap whole-CTA skips before any staging: no voxel within the
        // layer's range, or no spot of the layer within rcut of the CTA.
        {
            bool in_range = false;
#pragma unroll
            for (int v = 0; v < VY; ++v) in_range |= inside[v] && !(wet_mm[v] > 1.1f * L.r80);
            if (!__syncthreads_or(in_range)) continue;
            const float rc2 = L.rcut * L.rcut;
            int near = 0;
            for (int q = tid; q < L.n_spots; q += nthreads) {
                const float4 *sp = reinterpret_cast<const float4 *>(t.spots + L.spot_start + q);
                const float4 a = __ldg(sp), b = __ldg(sp + 1);
                const float ax0 = a.x - b.x * bz0, ax1 = a.x - b.x * bz1;
                const float ay0 = a.y - b.y * bz0, ay1 = a.y - b.y * bz1;
                const float dx = fmaxf(0.0f, fmaxf(fminf(ax0, ax1) - bx1, bx0 - fmaxf(ax0, ax1)));
                const float dy = fmaxf(0.0f, fmaxf(fminf(ay0, ay1) - by1, by0 - fmaxf(ay0, ay1)));
                near |= !((dx * dx + dy * dy) * b.z > rc2);
            }
            if (!__syncthreads_or(near)) continue;
        }
        __syncthreads();  // previous layer's shared data no longer in use
        const float *gd = t.lut_depths + (size_t)L.energy_id * t.lut_len;
        const float *gs = t.lut_sigmas + (size_t)L.energy_id * t.lut_len;
        const float *gi = t.lut_idds + (size_t)L.energy_id * t.lut_len;
        for (int q = tid; q < t.lut_len; q += nthreads) {
            s_depth[q] = __ldg(gd + q);
            s_sigma[q] = __ldg(gs + q);
            s_idd[q] = __ldg(gi + q);
        }
        __syncthreads();

        PbVoxel pv[VY];
        bool act[VY];
        bool any = false;
#pragma unroll
        for (int v = 0; v < VY; ++v) {
            act[v] = inside[v] && pb_voxel_layer(L, s_depth, s_sigma, s_idd, t.lut_len, wet_mm[v], dsrc[v], pv[v]);
            // adjoint: a voxel with zero gradient adds exactly zero to every
            // spot's sum, so it counts as inactive (an objective's gradient
            // vanishes outside its voxel sets)
            if (kMode == kPbAdjoint) act[v] = act[v] && gv[v] != 0.0f;
            if (!act[v]) {
                pv[v].pf = pv[v].hf = 0.f;
                pv[v].ps2 = pv[v].hs2 = 0.f;
            }
            any |= act[v];
        }
        const bool block_any = __syncthreads_or(any);
        if (!block_any) continue;

        // Lateral cut-off of this CTA for this layer: 6 x the widest halo
        // sigma of its active voxels (sigma_ht^2 = -log2(e) / (2 hs2)), never
        // wider than the layer's bound.  A spot whose axis stays farther than
        // that from the CTA's box lies beyond 6 sigma_ht of every voxel here,
        // where both Gaussians are below exp(-18) of their peaks.
        float rcut2;
        {
            float s2 = 0.0f;
#pragma unroll
            for (int v = 0; v < VY; ++v)
                if (act[v] && pv[v].hs2 < 0.0f) s2 = fmaxf(s2, -0.5f * kLog2e / pv[v].hs2);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s2 = fmaxf(s2, __shfl_xor_sync(0xffffffffu, s2, o));
            if (lane == 0) s_sig[threadIdx.y] = s2;
            __syncthreads();
            float m2 = s_sig[0];
#pragma unroll
            for (int w = 1; w < TY; ++w) m2 = fmaxf(m2, s_sig[w]);
            const float rc = 6.0f * (sqrtf(m2) * 1.01f + 0.1f);
            rcut2 = fminf(L.rcut * L.rcut, rc * rc);
        }
        for (int c0 = 0; c0 < L.n_spots; c0 += kPbSpotChunk) {
            const int craw = min(kPbSpotChunk, L.n_spots - c0);
            if (c0 > 0) __syncthreads();
            // Each thread tests two consecutive spots; the ones whose divergent
            // axis comes within rcut of the CTA's box are compacted in order.
            const float4 *gsp = reinterpret_cast<const float4 *>(t.spots + L.spot_start + c0);
            float4 a2[kSpt], b2[kSpt];
            bool keep[kSpt];
#pragma unroll
            for (int u = 0; u < kSpt; ++u) {
                const int q = kSpt * tid + u;
                keep[u] = false;
                if (q < craw) {
                    a2[u] = __ldg(gsp + 2 * q);
                    b2[u] = __ldg(gsp + 2 * q + 1);
                    // axis position at the box's height range: x(hz) = sx - tx * hz
                    const float ax0 = a2[u].x - b2[u].x * bz0, ax1 = a2[u].x - b2[u].x * bz1;
                    const float ay0 = a2[u].y - b2[u].y * bz0, ay1 = a2[u].y - b2[u].y * bz1;
                    const float dx = fmaxf(0.0f, fmaxf(fminf(ax0, ax1) - bx1, bx0 - fmaxf(ax0, ax1)));
                    const float dy = fmaxf(0.0f, fmaxf(fminf(ay0, ay1) - by1, by0 - fmaxf(ay0, ay1)));
                    // perpendicular distance >= lateral distance * cos(tilt), cos^2 = inv_t2
                    keep[u] = !((dx * dx + dy * dy) * b2[u].z > rcut2);
                }
            }
            int mine = 0;
#pragma unroll
            for (int u = 0; u < kSpt; ++u) mine += (int)keep[u];
            int incl = mine;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int n = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += n;
            }
            if (lane == 31) s_wcnt[threadIdx.y] = incl;
            __syncthreads();
            int base = 0, cn = 0;
#pragma unroll
            for (int w = 0; w < TY; ++w) {
                const int c = s_wcnt[w];
                base += (w < (int)threadIdx.y) ? c : 0;
                cn += c;
            }
            int pos = base + incl - mine;
#pragma unroll
            for (int u = 0; u < kSpt; ++u) {
                if (!keep[u]) continue;
                float4 a = a2[u], b = b2[u];
                const int orig = __float_as_int(a.w);
                if (x.mu) a.z = __ldg(x.mu + orig);
                if (kMode == kPbCount) b.w = __ldg(x.thr + orig);
                s_spot_a[pos] = a;
                s_spot_b[pos] = b;
                if (kMode == kPbAdjoint) s_acc[pos] = 0.0f;
                ++pos;
            }
            __syncthreads();
            if (cn == 0) continue;
            if constexpr (kMode == kPbDose && VY % 2 == 0) {
                if (!any) continue;
                // voxels (2p, 2p+1) of the thread share the paired lanes of p
                constexpr int VP = VY / 2;
                float2 hxp[VP], hyp[VP], hzp[VP], ps2p[VP], hs2p[VP], accp[VP], acch[VP];
#pragma unroll
                for (int p = 0; p < VP; ++p) {
                    hxp[p] = make_float2(hx[2 * p], hx[2 * p + 1]);
                    hyp[p] = make_float2(hy[2 * p], hy[2 * p + 1]);
                    hzp[p] = make_float2(hz[2 * p], hz[2 * p + 1]);
                    ps2p[p] = make_float2(pv[2 * p].ps2, pv[2 * p + 1].ps2);
                    hs2p[p] = make_float2(pv[2 * p].hs2, pv[2 * p + 1].hs2);
                    accp[p] = acch[p] = f2(0.f);
                }
#pragma unroll 4
                for (int q = 0; q < cn; ++q) {
                    const float4 a = s_spot_a[q];
                    const float4 b = s_spot_b[q];
                    const float2 nsx = f2(-a.x), nsy = f2(-a.y), tx = f2(b.x), ty = f2(b.y), ntx = f2(-b.x);
                    const float2 it2 = f2(b.z), mu = f2(a.z);
#pragma unroll
                    for (int p = 0; p < VP; ++p) {
                        const float2 r2 = pb_r2_pair(hxp[p], hyp[p], hzp[p], nsx, nsy, tx, ty, ntx, it2);
                        accp[p] = __ffma2_rn(mu, exp2_pair(__fmul2_rn(ps2p[p], r2)), accp[p]);
                        acch[p] = __ffma2_rn(mu, exp2_pair(__fmul2_rn(hs2p[p], r2)), acch[p]);
                    }
                }
#pragma unroll
                for (int p = 0; p < VP; ++p) {
                    if (act[2 * p]) acc[2 * p] += fmaf(pv[2 * p].pf, accp[p].x, pv[2 * p].hf * acch[p].x);
                    if (act[2 * p + 1]) acc[2 * p + 1] += fmaf(pv[2 * p + 1].pf, accp[p].y, pv[2 * p + 1].hf * acch[p].y);
                }
            } else if constexpr (kMode == kPbDose) {
                if (!any) continue;
                float accp[VY], acch[VY];
#pragma unroll
                for (int v = 0; v < VY; ++v) accp[v] = acch[v] = 0.f;
#pragma unroll 4
                for (int q = 0; q < cn; ++q) {
                    const float4 a = s_spot_a[q];
                    const float4 b = s_spot_b[q];
#pragma unroll
                    for (int v = 0; v < VY; ++v) {
                        const float r2 = pb_r2(hx[v], hy[v], hz[v], a.x, a.y, b.x, b.y, b.z);
                        accp[v] = fmaf(a.z, fast_exp2(pv[v].ps2 * r2), accp[v]);
                        acch[v] = fmaf(a.z, fast_exp2(pv[v].hs2 * r2), acch[v]);
                    }
                }
#pragma unroll
                for (int v = 0; v < VY; ++v) {
                    if (act[v]) acc[v] += fmaf(pv[v].pf, accp[v], pv[v].hf * acch[v]);
                }
            } else {
                // modes that need the per-pair influence K_s(v); a warp
                // without an active voxel contributes nothing and skips the
                // spots as a whole (its shuffles stay warp-uniform)
                const bool warp_any = __any_sync(0xffffffffu, any);
                for (int q = 0; q < (warp_any ? cn : 0); ++q) {
                    const float4 a = s_spot_a[q];
                    const float4 b = s_spot_b[q];
                    float kv[VY];
                    if constexpr (VY % 2 == 0) {
                        const float2 nsx = f2(-a.x), nsy = f2(-a.y), tx = f2(b.x), ty = f2(b.y), ntx = f2(-b.x);
                        const float2 it2 = f2(b.z);
#pragma unroll
                        for (int p = 0; p < VY / 2; ++p) {
                            const int v0 = 2 * p, v1 = 2 * p + 1;
                            const float2 r2 = pb_r2_pair(make_float2(hx[v0], hx[v1]), make_float2(hy[v0], hy[v1]),
                                                         make_float2(hz[v0], hz[v1]), nsx, nsy, tx, ty, ntx, it2);
                            const float2 ep = exp2_pair(__fmul2_rn(make_float2(pv[v0].ps2, pv[v1].ps2), r2));
                            const float2 eh = exp2_pair(__fmul2_rn(make_float2(pv[v0].hs2, pv[v1].hs2), r2));
                            const float2 k2 = __ffma2_rn(make_float2(pv[v0].pf, pv[v1].pf), ep,
                                                         __fmul2_rn(make_float2(pv[v0].hf, pv[v1].hf), eh));
                            kv[v0] = act[v0] ? k2.x : 0.0f;
                            kv[v1] = act[v1] ? k2.y : 0.0f;
                        }
                    } else {
#pragma unroll
                        for (int v = 0; v < VY; ++v) {
                            const float r2 = pb_r2(hx[v], hy[v], hz[v], a.x, a.y, b.x, b.y, b.z);
                            kv[v] = act[v] ? fmaf(pv[v].pf, fast_exp2(pv[v].ps2 * r2),
                                                  pv[v].hf * fast_exp2(pv[v].hs2 * r2))
                                           : 0.0f;
                        }
                    }
                    if (kMode == kPbAdjoint) {
                        float c = 0.0f;
#pragma unroll
                        for (int v = 0; v < VY; ++v) c = fmaf(gv[v], kv[v], c);
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
                        if (lane == 0 && c != 0.0f) atomicAdd(&s_acc[q], c);
                    } else if (kMode == kPbSpotMax) {
                        float m = 0.0f;
#pragma unroll
                        for (int v = 0; v < VY; ++v) m = fmaxf(m, kv[v]);
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
                        if (lane == 0 && m > 0.0f) atomicMax(x.spot_max + __float_as_int(a.w), __float_as_uint(m));
                    } else if (kMode == kPbCount) {
#pragma unroll
                        for (int v = 0; v < VY; ++v) {
                            const bool take = act[v] && kv[v] >= b.w && kv[v] > 0.0f;
                            if (x.row_ptr == nullptr) {
                                cnt[v] += take ? 1 : 0;
                            } else if (take && fill_off[v] < fill_end[v]) {
                                x.col[fill_off[v]] = __float_as_int(a.w);
                                x.val[fill_off[v]] = kv[v];
                                ++fill_off[v];
                            }
                        }
                    }
                }
                if (kMode == kPbAdjoint) {
                    __syncthreads();
                    for (int q = tid; q < cn; q += nthreads) {
                        const float c = s_acc[q];
                        if (c != 0.0f) atomicAdd(x.grad_mu + __float_as_int(s_spot_a[q].w), (double)c);
                    }
                }
            }
        }
    }

    if (kMode == kPbCount && x.row_ptr == nullptr) {
#pragma unroll
        for (int v = 0; v < VY; ++v)
            if (inside[v] && DC_IN_BOUNDS(vidx[v], g.n(), 24)) x.counts[vidx[v]] = cnt[v];
    }
}


// Minimum resident CTAs per SM the register allocation is held to: 4 CTAs
// of 256 threads (or 8 of 128; 64 registers) for the one-shot and the
// persistent batch kernels.  More resident warps hide the fixed-latency
// chains of the spot loop and the per-layer barriers; measured on the adjoint
// (0.492 -> 0.439 ms) and the batch (41.4 -> 35.2 ms for four plans at 3 CTAs
// of 256 threads, 16.7 -> 15.2 ms at 4 with the 16 x TY x 8 tiles) with the
// dose kernel unchanged, despite a few spilled words outside the spot loop.
constexpr int pb_min_ctas(int ty, int per_256) { return ty >= 8 ? per_256 : 2 * per_256; }

// One tile per CTA (grid = the tiles of the volume, pb_tiles).
template <int kMode, int TY, int VY>
__global__ void __launch_bounds__(kPbThreadsX *TY, pb_min_ctas(TY, 4))
    pb_kernel(Grid g, Frame f, ProtonTables t, const float *__restrict__ wet_s, float *__restrict__ dose, PbExtra x) {
    float acc[VY];
#pragma unroll
    for (int v = 0; v < VY; ++v) acc[v] = 0.0f;
    const int bz = (int)blockIdx.z + x.tile_z0;
    pb_tile<kMode, TY, VY>(g, f, t, wet_s, blockIdx.x, blockIdx.y, bz, acc, x);
    if (kMode == kPbDose) {
#pragma unroll
        for (int v = 0; v < VY; ++v) {
            const int3 q = pb_tile_voxel<TY, VY>(blockIdx.x, blockIdx.y, bz, v);
            const long long u = (long long)q.x + (long long)g.nx * (q.y + (long long)g.ny * q.z);
            if (q.x < g.nx && q.y < g.ny && q.z < g.nz && DC_IN_BOUNDS(u, g.n(), 20)) dose[u] = acc[v];
        }
    }
}

// Voxel-list kernel (dose / adjoint of listed voxels; one CTA per
// threads*VY consecutive list entries).  A sorted list keeps a CTA's voxels
// close together, so the per-CTA spot culling stays tight.
template <int kMode, int TY, int VY>
__global__ void __launch_bounds__(kPbThreadsX *TY, pb_min_ctas(TY, 4))
    pb_list_kernel(Grid g, Frame f, ProtonTables t, const float *__restrict__ wet_s, PbExtra x) {
    float acc[VY];
#pragma unroll
    for (int v = 0; v < VY; ++v) acc[v] = 0.0f;
    pb_tile<kMode, TY, VY, true>(g, f, t, wet_s, blockIdx.x, 0, 0, acc, x);
    if (kMode == kPbDose) {
        const int tid = threadIdx.y * kPbThreadsX + threadIdx.x;
#pragma unroll
        for (int v = 0; v < VY; ++v) {
            const int e = blockIdx.x * (kPbThreadsX * TY * VY) + v * (kPbThreadsX * TY) + tid;
            if (e < x.n_list && DC_IN_BOUNDS(e, x.n_list, 22)) x.list_out[e] = acc[v];
        }
    }
}

// Persistent batch kernel: CTAs take (plan, tile) work items from a device
// queue (most expensive plans first) and sum the dose of all the plan's beams
// for the tile in registers before one write per voxel.
//
// The plan and beam records are staged in shared memory and passed to pb_tile
// by reference: their fields are then read from shared memory where used
// instead of holding some twenty registers through the layer loop (the
// one-beam kernels read the same fields from the kernel parameters).
template <class T>
__device__ __forceinline__ void pb_stage_record(T *dst, const T *__restrict__ src, int tid, int nthreads) {
    static_assert(sizeof(T) % sizeof(int) == 0, "records are copied as words");
    const int *s = reinterpret_cast<const int *>(src);
    int *d = reinterpret_cast<int *>(dst);
    for (int q = tid; q < (int)(sizeof(T) / sizeof(int)); q += nthreads) d[q] = __ldg(s + q);
}

template <int TY, int VY>
__global__ void __launch_bounds__(kPbThreadsX *TY, pb_min_ctas(TY, 4))
    pb_batch_kernel(const PbBatchPlan *__restrict__ plans, const PbBatchBeam *__restrict__ beams,
                    const int2 *__restrict__ items, int n_items, unsigned *__restrict__ next) {
    __shared__ int s_item;
    __shared__ PbBatchPlan s_plan;
    __shared__ PbBatchBeam s_beam;
    const int tid = threadIdx.y * kPbThreadsX + threadIdx.x;
    while (true) {
        __syncthreads();  // the previous item's plan record no longer in use
        if (tid == 0) s_item = (int)atomicAdd(next, 1u);
        __syncthreads();
        const int it = s_item;
        if (it >= n_items) break;
        const int2 w = items[it];
        pb_stage_record(&s_plan, plans + w.x, tid, kPbThreadsX * TY);
        __syncthreads();
        const PbBatchPlan &P = s_plan;
        const int3 nt = pb_tiles<TY, VY>(P.g);
        const int bz = w.y / (nt.x * nt.y);
        const int rem = w.y - bz * nt.x * nt.y;
        const int by = rem / nt.x, bx = rem - by * nt.x;
        float acc[VY];
#pragma unroll
        for (int v = 0; v < VY; ++v) acc[v] = 0.0f;
        const int b1 = P.beam0 + P.n_beams;
        for (int b = P.beam0; b < b1; ++b) {
            __syncthreads();  // the previous beam's record no longer in use
            pb_stage_record(&s_beam, beams + b, tid, kPbThreadsX * TY);
            __syncthreads();
            PbExtra x;
            x.mu = s_beam.mu;
            pb_tile<kPbDose, TY, VY>(P.g, s_beam.f, s_beam.t, s_beam.wet, bx, by, bz, acc, x);
        }
#pragma unroll
        for (int v = 0; v < VY; ++v) {
            const int3 q = pb_tile_voxel<TY, VY>(bx, by, bz, v);
            const long long u = (long long)q.x + (long long)P.g.nx * (q.y + (long long)P.g.ny * q.z);
            if (q.x < P.g.nx && q.y < P.g.ny && q.z < P.g.nz && DC_IN_BOUNDS(u, P.g.n(), 23)) P.dose[u] = acc[v];
        }
    }
}

DC_BOUNDS_TAKE(take_bounds_proton)

static size_t pb_smem(int lut_len) {
    return 2 * kPbSpotChunk * sizeof(float4) + kPbSpotChunk * sizeof(float) + 3 * (size_t)lut_len * sizeof(float);
}

template <class K>
static void pb_attr(K kernel, size_t smem, int device, bool *done) {
    if (smem > 48 * 1024 && device < 64 && !done[device]) {
        DC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        done[device] = true;
    }
}

template <int kMode>
static void pb_launch(DeviceContext &ctx, const char *name, const Grid &g, const Frame &f, const ProtonTables &t,
                      const float *wet_s, float *dose, const PbExtra &x, cudaStream_t s) {
    const size_t smem = pb_smem(t.lut_len);
    static bool attr_set[64] = {false};
    pb_attr(pb_kernel<kMode, kPbThreadsY, kPbVoxY>, smem, ctx.device, attr_set);
    dim3 block(kPbThreadsX, kPbThreadsY, 1);
    const int3 nt = pb_tiles<kPbThreadsY, kPbVoxY>(g);
    // tiles x.tile_z0 .. tile_z1 - 1 along z (all of them by default)
    const int z1 = x.tile_z1 < 0 ? nt.z : std::min(x.tile_z1, nt.z);
    if (x.tile_z0 < 0 || x.tile_z0 >= z1) return;
    dim3 grid((unsigned)nt.x, (unsigned)nt.y, (unsigned)(z1 - x.tile_z0));
    KernelTimer kt(ctx, name, s);
    pb_kernel<kMode, kPbThreadsY, kPbVoxY><<<grid, block, smem, s>>>(g, f, t, wet_s, dose, x);
    check_launch(name);
}

void launch_pencil_beam(DeviceContext &ctx, const Grid &g, const Frame &f, const ProtonTables &t,
                        const float *wet_s, float *dose, cudaStream_t s, const float *mu_dev, int tile_z0,
                        int tile_z1) {
    PbExtra x;
    x.mu = mu_dev;
    x.tile_z0 = tile_z0;
    x.tile_z1 = tile_z1;
    pb_launch<kPbDose>(ctx, "pencil_beam", g, f, t, wet_s, dose, x, s);
}

int pencil_beam_tile_depth() { return PbTileShape<kPbThreadsY, kPbVoxY>::z; }

void launch_pencil_beam_mode(DeviceContext &ctx, int mode, const Grid &g, const Frame &f, const ProtonTables &t,
                             const float *wet_s, const PbExtra &x, cudaStream_t s) {
    switch (mode) {
        case kPbAdjoint: pb_launch<kPbAdjoint>(ctx, "pencil_beam_adjoint", g, f, t, wet_s, nullptr, x, s); break;
        case kPbSpotMax: pb_launch<kPbSpotMax>(ctx, "pencil_beam_spotmax", g, f, t, wet_s, nullptr, x, s); break;
        case kPbCount: pb_launch<kPbCount>(ctx, "pencil_beam_count", g, f, t, wet_s, nullptr, x, s); break;
        case kPbFill:
            if (x.row_ptr == nullptr) throw Error(DC_ERR_VALUE, "the fill pass needs the row starts");
            pb_launch<kPbCount>(ctx, "pencil_beam_fill", g, f, t, wet_s, nullptr, x, s);
            break;
        default: throw Error(DC_ERR_VALUE, "unknown pencil-beam mode");
    }
}

template <int kMode>
static void pb_list_launch(DeviceContext &ctx, const char *name, const Grid &g, const Frame &f,
                           const ProtonTables &t, const float *wet_s, const PbExtra &x, cudaStream_t s) {
    if (x.n_list <= 0) return;
    const size_t smem = pb_smem(t.lut_len);
    static bool attr_set[64] = {false};
    pb_attr(pb_list_kernel<kMode, kPbThreadsY, kPbVoxY>, smem, ctx.device, attr_set);
    const int per_cta = kPbThreadsX * kPbThreadsY * kPbVoxY;
    const unsigned blocks = (unsigned)((x.n_list + per_cta - 1) / per_cta);
    KernelTimer kt(ctx, name, s);
    pb_list_kernel<kMode, kPbThreadsY, kPbVoxY><<<blocks, dim3(kPbThreadsX, kPbThreadsY, 1), smem, s>>>(g, f, t,
                                                                                                     wet_s, x);
    check_launch(name);
}

void launch_pencil_beam_list(DeviceContext &ctx, int mode, const Grid &g, const Frame &f, const ProtonTables &t,
                             const float *wet_s, const PbExtra &x, cudaStream_t s) {
    switch (mode) {
        case kPbDose: pb_list_launch<kPbDose>(ctx, "pencil_beam_list", g, f, t, wet_s, x, s); break;
        case kPbAdjoint: pb_list_launch<kPbAdjoint>(ctx, "pencil_beam_list_adjoint", g, f, t, wet_s, x, s); break;
        default: throw Error(DC_ERR_VALUE, "voxel-list mode is for the dose and the adjoint");
    }
}

// Tile shapes of the batch kernel (threads along y, voxels per thread along y).
static const int kPbVariants[][2] = {{8, 2}, {4, 2}, {8, 1}, {4, 4}};
int pencil_beam_batch_variants() { return (int)(sizeof(kPbVariants) / sizeof(kPbVariants[0])); }
void pencil_beam_batch_tile(int variant, int *ty, int *vy) {
    *ty = kPbVariants[variant][0];
    *vy = kPbVariants[variant][1];
}
long long pencil_beam_batch_tiles(int variant, const Grid &g) {
    int3 n{};
    switch (variant) {
        case 0: n = pb_tiles<8, 2>(g); break;
        case 1: n = pb_tiles<4, 2>(g); break;
        case 2: n = pb_tiles<8, 1>(g); break;
        case 3: n = pb_tiles<4, 4>(g); break;
        default: throw Error(DC_ERR_VALUE, "unknown pencil-beam tile variant");
    }
    return (long long)n.x * n.y * n.z;
}

template <int TY, int VY>
static void pb_batch_launch(DeviceContext &ctx, const PbBatchPlan *plans, const PbBatchBeam *beams,
                            const int2 *items, int n_items, unsigned *next, int lut_len, cudaStream_t s) {
    const size_t smem = pb_smem(lut_len);
    static bool attr_set[64] = {false};
    pb_attr(pb_batch_kernel<TY, VY>, smem, ctx.device, attr_set);
    int sms = 0, per_sm = 0;
    DC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
    DC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pb_batch_kernel<TY, VY>, kPbThreadsX * TY, smem));
    const int blocks = std::max(1, std::min(n_items, sms * std::max(per_sm, 1)));
    DC_CUDA(cudaMemsetAsync(next, 0, sizeof(unsigned), s));
    KernelTimer kt(ctx, "pencil_beam_batch", s);
    pb_batch_kernel<TY, VY><<<blocks, dim3(kPbThreadsX, TY, 1), smem, s>>>(plans, beams, items, n_items, next);
    check_launch("pb_batch_kernel");
}

void launch_pencil_beam_batch(DeviceContext &ctx, int variant, const PbBatchPlan *plans, const PbBatchBeam *beams,
                              const int2 *items, int n_items, unsigned *next, int lut_len, cudaStream_t s) {
    switch (variant) {
        case 0: pb_batch_launch<8, 2>(ctx, plans, beams, items, n_items, next, lut_len, s); break;
        case 1: pb_batch_launch<4, 2>(ctx, plans, beams, items, n_items, next, lut_len, s); break;
        case 2: pb_batch_launch<8, 1>(ctx, plans, beams, items, n_items, next, lut_len, s); break;
        case 3: pb_batch_launch<4, 4>(ctx, plans, beams, items, n_items, next, lut_len, s); break;
        default: throw Error(DC_ERR_VALUE, "unknown pencil-beam tile variant");
    }
}

}  // namespace dc
