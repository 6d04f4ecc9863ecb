// dc_cccs_sweep.cu — collapsed-cone dose by cone-direction sweeps over line
// lattices (a selectable approximation of the reference's per-voxel march).
//
// The reference's CCCS (cccKernel, IMRTClasses.cu:252-350) marches, for each
// voxel and each of the 72 cone directions (kernel-tilted per voxel towards
// the source, :173-203), a window of n samples spaced one voxel apart and
// runs the truncated recursions
//     Rp <- Rp e_m + T_m cp (1 - e_m),   Rs <- Rs (1 - b D_m) + T_m D_m cs
// from the far sample to the voxel.  Along a line in direction t with nodes
// one voxel apart, the windows of neighbouring nodes overlap in n-1 samples,
// so one pass along the line serves every node:
//     R(k)   = x_k + e_k R(k+1)                  (the untruncated recursion)
//     Rw(k)  = R(k) - [prod_{i<n} e_{k+i}] R(k+n)  (its window of n samples)
// This file samples (TERMA, density) once per node of a lattice of parallel
// lines per direction, runs R(k) as a warp-level affine scan (one warp per
// line, 32 nodes per step, __shfl_up composition of x + e R), forms the
// windowed value with the window products from prefix sums of log factors,
// stores c(k) = a Rw_p(k) + b Rw_s(k) per node, and gathers c at every active
// voxel by trilinear interpolation of the lattice, summed over directions.
//
// What it gives up against the reference: (i) the per-voxel kernel tilt —
// every line of a direction has the central axis's orientation; (ii) the
// voxel's own sample positions — c is interpolated between lattice lines one
// voxel apart, which smooths the TERMA's steep field edges.  The lattice only
// covers the bounding box of the active voxels (TERMA > 0.01) widened by the
// longest window, so directions cost in proportion to the irradiated volume.
#include <algorithm>
#include <cmath>
#include <vector>

#include "dc_common.cuh"
#include "dc_kernels.cuh"
#include "dc_photon.cuh"
#include "dc_runtime.cuh"

namespace dc {

DC_BOUNDS_WORD

namespace {

struct SweepLattice {
    float3 e1, e2, e3;  // lateral axes and the line direction (image frame)
    float h, sp;        // lateral spacing and node spacing (mm)
    float u0, v0, k0;   // lattice origin in units of h, h, sp
    int nu, nv, nk;
};

struct SweepCone {
    float a, b, cp, cs;  // recursion constants of the direction's cone
    float r0;            // distance of the window's first sample from the voxel (mm)
    int n;               // window length (samples)
};

}  // namespace

// Bounding box of the active voxels (grid indices): min i,j,k, max i,j,k.
__global__ void active_bbox_kernel(Grid g, const int *__restrict__ active, const unsigned *__restrict__ n_active,
                                   int *__restrict__ box) {
    const unsigned n = *n_active;
    int lo[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, hi[3] = {-1, -1, -1};
    const int plane = g.nx * g.ny;
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int v = DC_IN_BOUNDS(t, g.n(), 60) ? __ldg(active + t) : -1;
        if (!DC_IN_BOUNDS(v, g.n(), 60)) continue;
        const int k = v / plane, rem = v - k * plane, j = rem / g.nx, i = rem - j * g.nx;
        lo[0] = min(lo[0], i), lo[1] = min(lo[1], j), lo[2] = min(lo[2], k);
        hi[0] = max(hi[0], i), hi[1] = max(hi[1], j), hi[2] = max(hi[2], k);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
        for (int a = 0; a < 3; ++a) {
            atomicMin(box + a, lo[a]);
            atomicMax(box + 3 + a, hi[a]);
        }
    }
}

// One warp per lattice line; lane l takes node k_top - l of each 32-node
// chunk, walking from the line's far (+t) end towards its near end.
__global__ void __launch_bounds__(256) sweep_line_kernel(Grid g, Frame f, SweepLattice S, SweepCone K,
                                                         cudaTextureObject_t td_tex, float sp_cm,
                                                         float *__restrict__ C) {
    const int lane = threadIdx.x & 31;
    const int line = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (line >= S.nu * S.nv) return;  // whole warps leave together
    const int u = line % S.nu, v = line / S.nu;
    const float pu = (S.u0 + (float)u) * S.h, pv = (S.v0 + (float)v) * S.h;
    const float3 base = make_float3(pu * S.e1.x + pv * S.e2.x, pu * S.e1.y + pv * S.e2.y, pu * S.e1.z + pv * S.e2.z);
    const float nal2e = -K.a * kLog2e;
    // carries from the chunk above: R values, and the running log sums
    float Rp_c = 0.0f, Rs_c = 0.0f, Qp_c = 0.0f, Qs_c = 0.0f;
    // the previous chunk's per-lane values (for windows reaching into it)
    float Rp_prev = 0.0f, Rs_prev = 0.0f, Qp_prev = 0.0f, Qs_prev = 0.0f;
    const long long lbase = (long long)line * S.nk;
    for (int top = S.nk - 1; top >= 0; top -= 32) {
        const int k = top - lane;
        float xp = 0.0f, xs = 0.0f, ep = 1.0f, es = 1.0f, lp = 0.0f, ls = 0.0f;
        if (k >= 0) {
            const float s = (S.k0 + (float)k) * S.sp;
            const float3 q = make_float3(fmaf(s, S.e3.x, base.x), fmaf(s, S.e3.y, base.y), fmaf(s, S.e3.z, base.z));
            const float3 tc = tex_coord(g, f, q);
            const float2 td = tex3D<float2>(td_tex, tc.x, tc.y, tc.z);
            const float D = fmaxf(td.y, kAirDensity) * sp_cm;
            ep = fast_exp2(nal2e * D);
            es = 1.0f - K.b * D;
            xp = td.x * K.cp * (1.0f - ep);
            xs = td.x * D * K.cs;
            lp = K.a * D;                      // -ln e_p
            ls = -__logf(fmaxf(es, 1e-30f));   // -ln e_s
        }
        // inclusive affine scan in lane order: R_l = A_l * carry + B_l
        float Ap = ep, Bp = xp, As = es, Bs = xs, Sp = lp, Ss = ls;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const float ap = __shfl_up_sync(0xffffffffu, Ap, o), bp = __shfl_up_sync(0xffffffffu, Bp, o);
            const float as = __shfl_up_sync(0xffffffffu, As, o), bs = __shfl_up_sync(0xffffffffu, Bs, o);
            const float sp_ = __shfl_up_sync(0xffffffffu, Sp, o), ss_ = __shfl_up_sync(0xffffffffu, Ss, o);
            if (lane >= o) {
                Bp = fmaf(Ap, bp, Bp);
                Ap *= ap;
                Bs = fmaf(As, bs, Bs);
                As *= as;
                Sp += sp_;
                Ss += ss_;
            }
        }
        const float Rp = fmaf(Ap, Rp_c, Bp), Rs = fmaf(As, Rs_c, Bs);
        const float Qp = Qp_c + Sp, Qs = Qs_c + Ss;  // log sums over nodes >= k (from the far end)
        // the node n further along the line: lane l - n of this chunk, or
        // lane l - n + 32 of the previous one (R and Q of that node)
        const int src = lane - K.n;
        const int sl = src >= 0 ? src : src + 32;
        const float Rp_n_cur = __shfl_sync(0xffffffffu, Rp, sl), Rs_n_cur = __shfl_sync(0xffffffffu, Rs, sl);
        const float Qp_n_cur = __shfl_sync(0xffffffffu, Qp, sl), Qs_n_cur = __shfl_sync(0xffffffffu, Qs, sl);
        const float Rp_n_prv = __shfl_sync(0xffffffffu, Rp_prev, sl), Rs_n_prv = __shfl_sync(0xffffffffu, Rs_prev, sl);
        const float Qp_n_prv = __shfl_sync(0xffffffffu, Qp_prev, sl), Qs_n_prv = __shfl_sync(0xffffffffu, Qs_prev, sl);
        const bool cur = src >= 0;
        const bool beyond = k + K.n > S.nk - 1;  // that node lies past the line's far end: R = 0, Q = 0
        const float Rp_n = beyond ? 0.0f : (cur ? Rp_n_cur : Rp_n_prv);
        const float Rs_n = beyond ? 0.0f : (cur ? Rs_n_cur : Rs_n_prv);
        const float Qp_n = beyond ? 0.0f : (cur ? Qp_n_cur : Qp_n_prv);
        const float Qs_n = beyond ? 0.0f : (cur ? Qs_n_cur : Qs_n_prv);
        const float Pp = fast_exp2(-(Qp - Qp_n) * kLog2e), Ps = fast_exp2(-(Qs - Qs_n) * kLog2e);
        const float c = K.a * (Rp - Pp * Rp_n) + K.b * (Rs - Ps * Rs_n);
        if (k >= 0) {
            const long long idx = lbase + k;
            if (DC_IN_BOUNDS(idx, (long long)S.nu * S.nv * S.nk, 61)) C[idx] = c;
        }
        Rp_c = __shfl_sync(0xffffffffu, Rp, 31);
        Rs_c = __shfl_sync(0xffffffffu, Rs, 31);
        Qp_c = __shfl_sync(0xffffffffu, Qp, 31);
        Qs_c = __shfl_sync(0xffffffffu, Qs, 31);
        Rp_prev = Rp, Rs_prev = Rs, Qp_prev = Qp, Qs_prev = Qs;
    }
}

// Adds c of one direction, interpolated at every active voxel's window start.
__global__ void __launch_bounds__(128) sweep_gather_kernel(Grid g, Frame f, SweepLattice S, float r0,
                                                           const float *__restrict__ C, const int *__restrict__ active,
                                                           const unsigned *__restrict__ n_active,
                                                           float *__restrict__ acc) {
    const unsigned n = *n_active;
    const int plane = g.nx * g.ny;
    const long long total = (long long)S.nu * S.nv * S.nk;
    (void)total;  // read by the bounds checks of debug builds
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int v = DC_IN_BOUNDS(t, g.n(), 62) ? __ldg(active + t) : -1;
        if (!DC_IN_BOUNDS(v, g.n(), 62)) continue;
        const int k = v / plane, rem = v - k * plane, j = rem / g.nx, i = rem - j * g.nx;
        float3 p = voxel_xyz(g, f, i, j, k);
        p.x = fmaf(r0, S.e3.x, p.x);
        p.y = fmaf(r0, S.e3.y, p.y);
        p.z = fmaf(r0, S.e3.z, p.z);
        const float fu = (p.x * S.e1.x + p.y * S.e1.y + p.z * S.e1.z) / S.h - S.u0;
        const float fv = (p.x * S.e2.x + p.y * S.e2.y + p.z * S.e2.z) / S.h - S.v0;
        const float fk = (p.x * S.e3.x + p.y * S.e3.y + p.z * S.e3.z) / S.sp - S.k0;
        const float xu = floorf(fu), xv = floorf(fv), xk = floorf(fk);
        if (!(xu >= 0.0f && xv >= 0.0f && xk >= 0.0f && xu <= (float)(S.nu - 2) && xv <= (float)(S.nv - 2) &&
              xk <= (float)(S.nk - 2)))
            continue;  // cannot happen for the lattice's own box; skipped rather than read out of range
        const int iu = (int)xu, iv = (int)xv, ik = (int)xk;
        const float wu = fu - xu, wv = fv - xv, wk = fk - xk;
        const long long b00 = ((long long)iv * S.nu + iu) * S.nk + ik;
        const long long du = S.nk, dv = (long long)S.nu * S.nk;
        if (!DC_IN_BOUNDS(b00 + dv + du + 1, total, 63)) continue;
        const float c000 = __ldg(C + b00), c001 = __ldg(C + b00 + 1);
        const float c100 = __ldg(C + b00 + du), c101 = __ldg(C + b00 + du + 1);
        const float c010 = __ldg(C + b00 + dv), c011 = __ldg(C + b00 + dv + 1);
        const float c110 = __ldg(C + b00 + dv + du), c111 = __ldg(C + b00 + dv + du + 1);
        const float a00 = fmaf(wk, c001 - c000, c000), a10 = fmaf(wk, c101 - c100, c100);
        const float a01 = fmaf(wk, c011 - c010, c010), a11 = fmaf(wk, c111 - c110, c110);
        const float b0 = fmaf(wu, a10 - a00, a00), b1 = fmaf(wu, a11 - a01, a01);
        acc[v] += fmaf(wv, b1 - b0, b0);
    }
}

__global__ void __launch_bounds__(128) sweep_finish_kernel(Grid g, float dose_scale, const float *__restrict__ acc,
                                                           const float *__restrict__ electron,
                                                           const int *__restrict__ active,
                                                           const unsigned *__restrict__ n_active,
                                                           float *__restrict__ dose) {
    const unsigned n = *n_active;
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int v = DC_IN_BOUNDS(t, g.n(), 64) ? __ldg(active + t) : -1;
        if (!DC_IN_BOUNDS(v, g.n(), 64)) continue;
        const float d = acc[v] + __ldg(electron + v);
        dose[v] = (!isnan(d) && d >= 0.0f) ? dose_scale * d : 0.0f;
    }
}

DC_BOUNDS_TAKE(take_bounds_sweep)

void enqueue_cccs_sweep(DeviceContext &ctx, const Grid &g, const Frame &f, const CccsCones &C, const PhotonWork &w,
                        float dose_scale, float *dose_dev, DeviceBuffer &lattice, DeviceBuffer &acc_buf,
                        DeviceBuffer &box_buf, cudaStream_t s) {
    int sms = 0;
    DC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
    const unsigned list_blocks = (unsigned)std::max<long long>(1, std::min<long long>((g.n() + 127) / 128, sms * 8LL));
    // 1. bounding box of the active voxels (one synchronous read of 6 ints)
    int *box = static_cast<int *>(box_buf.ensure(6 * sizeof(int)));
    const int init[6] = {0x7fffffff, 0x7fffffff, 0x7fffffff, -1, -1, -1};
    DC_CUDA(cudaMemcpyAsync(box, init, sizeof(init), cudaMemcpyHostToDevice, s));
    active_bbox_kernel<<<list_blocks, 128, 0, s>>>(g, w.active, w.n_active, box);
    check_launch("active_bbox_kernel");
    int hb[6];
    DC_CUDA(cudaMemcpyAsync(hb, box, sizeof(hb), cudaMemcpyDeviceToHost, s));
    DC_CUDA(cudaStreamSynchronize(s));
    float *acc = static_cast<float *>(acc_buf.ensure((size_t)g.n() * sizeof(float)));
    DC_CUDA(cudaMemsetAsync(acc, 0, (size_t)g.n() * sizeof(float), s));
    if (hb[3] < 0) {  // no active voxel: the dose is the TERMA kernel's zeros
        return;
    }
    // box corners in image coordinates, widened by the longest window
    float reach = 0.0f;
    for (int q = 0; q < C.total_steps; ++q) reach = std::max(reach, C.rl10[q]);
    reach += std::max(g.sx, std::max(g.sy, g.sz));
    const float lo[3] = {hb[0] * g.sx - f.isox, hb[1] * g.sy - f.isoy, hb[2] * g.sz - f.isoz};
    const float hi[3] = {hb[3] * g.sx - f.isox, hb[4] * g.sy - f.isoy, hb[5] * g.sz - f.isoz};
    // the image-frame (untilted) cone directions, as cone_dirs_kernel computes them
    std::vector<float4> dirs((size_t)C.n_cones * 12);
    DC_CUDA(cudaMemcpyAsync(dirs.data(), w.dirs, dirs.size() * sizeof(float4), cudaMemcpyDeviceToHost, s));
    DC_CUDA(cudaStreamSynchronize(s));
    const float sp_mm = g.sx;  // the CCCS step is the (isotropic) voxel spacing
    size_t cap = 0;
    KernelTimer kt(ctx, "cccs_sweep", s);
    for (int c = 0; c < C.n_cones; ++c) {
        SweepCone K{};
        K.a = C.am[c];
        K.b = C.bm[c];
        K.n = C.n_steps[c];
        K.r0 = C.rl10[C.step_off[c] + C.n_steps[c] - 1];
        for (int az = 0; az < 12; ++az) {
            const float4 dv = dirs[(size_t)c * 12 + az];
            K.cp = dv.w * (C.Am[c] / (C.am[c] * C.am[c]));
            K.cs = dv.w * (C.Bm[c] / C.bm[c]);
            SweepLattice S{};
            S.e3 = make_float3(dv.x, dv.y, dv.z);
            // lateral axes: e1 perpendicular to e3 and to the axis e3 leans on least
            const float ax = std::fabs(dv.x), ay = std::fabs(dv.y), az_ = std::fabs(dv.z);
            float3 ref = ax <= ay && ax <= az_ ? make_float3(1, 0, 0) : (ay <= az_ ? make_float3(0, 1, 0)
                                                                                 : make_float3(0, 0, 1));
            float3 e1 = make_float3(S.e3.y * ref.z - S.e3.z * ref.y, S.e3.z * ref.x - S.e3.x * ref.z,
                                    S.e3.x * ref.y - S.e3.y * ref.x);
            const float n1 = std::sqrt(e1.x * e1.x + e1.y * e1.y + e1.z * e1.z);
            e1 = make_float3(e1.x / n1, e1.y / n1, e1.z / n1);
            const float3 e2 = make_float3(S.e3.y * e1.z - S.e3.z * e1.y, S.e3.z * e1.x - S.e3.x * e1.z,
                                          S.e3.x * e1.y - S.e3.y * e1.x);
            S.e1 = e1;
            S.e2 = e2;
            S.h = sp_mm;
            S.sp = sp_mm;
            float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
            for (int q = 0; q < 8; ++q) {
                const float x = (q & 1) ? hi[0] + reach : lo[0] - reach;
                const float y = (q & 2) ? hi[1] + reach : lo[1] - reach;
                const float z = (q & 4) ? hi[2] + reach : lo[2] - reach;
                const float pr[3] = {x * e1.x + y * e1.y + z * e1.z, x * e2.x + y * e2.y + z * e2.z,
                                     x * S.e3.x + y * S.e3.y + z * S.e3.z};
                for (int a = 0; a < 3; ++a) mn[a] = std::min(mn[a], pr[a]), mx[a] = std::max(mx[a], pr[a]);
            }
            S.u0 = std::floor(mn[0] / S.h) - 1.0f;
            S.v0 = std::floor(mn[1] / S.h) - 1.0f;
            S.k0 = std::floor(mn[2] / S.sp) - 1.0f;
            S.nu = (int)std::ceil(mx[0] / S.h - S.u0) + 2;
            S.nv = (int)std::ceil(mx[1] / S.h - S.v0) + 2;
            S.nk = (int)std::ceil(mx[2] / S.sp - S.k0) + 2 + K.n;
            const size_t need_bytes = (size_t)S.nu * S.nv * S.nk * sizeof(float);
            if (need_bytes > cap) {
                // grows before any kernel of this call reads it; earlier launches
                // of this call have completed only in stream order, so wait
                DC_CUDA(cudaStreamSynchronize(s));
                lattice.ensure(need_bytes);
                cap = need_bytes;
            }
            float *Cl = lattice.as<float>();
            const long long lines = (long long)S.nu * S.nv;
            sweep_line_kernel<<<(unsigned)((lines + 7) / 8), 256, 0, s>>>(g, f, S, K, w.td_tex, g.sx / 10.0f, Cl);
            check_launch("sweep_line_kernel");
            sweep_gather_kernel<<<list_blocks, 128, 0, s>>>(g, f, S, K.r0, Cl, w.active, w.n_active, acc);
            check_launch("sweep_gather_kernel");
        }
    }
    sweep_finish_kernel<<<list_blocks, 128, 0, s>>>(g, dose_scale, acc, w.electron, w.active, w.n_active, dose_dev);
    check_launch("sweep_finish_kernel");
}

}  // namespace dc
