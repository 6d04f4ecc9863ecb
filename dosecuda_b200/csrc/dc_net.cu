// dc_net.cu — tensor-core kernels of the photon-dose surrogate network.
//
// Data layout: bf16 activations, channels-last (n, d, h, w, c).  A voxel's
// channels are 16-byte chunks of 8 channels; shared-memory tiles store chunk
// (voxel hv, chunk cc) at 16-byte slot hv*CC + (cc ^ swizzle(hv)), so that
// the 8 row addresses of one ldmatrix (8 consecutive voxels of a tap-shifted
// x-row) fall in 8 distinct bank groups.
//
// Convolutions are implicit GEMMs with mma.sync.m16n8k16 (bf16 in, fp32
// accumulate).  One m16 tile is 16 consecutive x of one output row; the K
// dimension runs over (tap, input-channel chunk) pairs; the B operand is read
// from a weight set pre-packed in mma fragment order (one 8-byte load per lane
// per n8 tile and k16 step, L1/L2 resident), so no weight staging is needed.
// Each CTA stages the input region its outputs need (the tile plus its halo)
// once with cp.async, zero-filling outside the volume (the convolution's zero
// padding), and then runs every tap from shared memory.
#include <algorithm>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <utility>

#include "../../include/dosecuda.h"
#include "dc_net.cuh"
#include "dc_runtime.cuh"

namespace dc {
namespace net {

namespace {

constexpr int kThreads = 128;

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void cp_async16(unsigned dst, const void *src, bool valid) {
    const int n = valid ? 16 : 0;  // src-size 0: the 16 bytes are zero-filled
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n));
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void ldsm_x4(unsigned addr, unsigned (&r)[4]) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

__device__ __forceinline__ void ldsm_x4_t(unsigned addr, unsigned (&r)[4]) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(addr));
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// 16-byte slot of chunk cc of tile voxel hv.  MODE kDown2 tiles are read with
// stride-2 x, so their swizzle keys on hv/2.
template <int CC, int MODE>
__device__ __forceinline__ int chunk_slot(int hv, int cc) {
    const int u = (MODE == kDown2) ? (hv >> 1) : hv;
    int sw;
    if (CC == 1)
        sw = 0;
    else if (CC == 2)
        sw = (u >> 2) & 1;
    else if (CC == 4)
        sw = (u >> 1) & 3;
    else
        sw = u & 7;
    return hv * CC + (cc ^ sw);
}

// Offset of tap t inside a tile of row length HX and HY rows per plane.
template <int MODE, int HX, int HY>
__device__ __forceinline__ int tap_offset(int t) {
    if (MODE == kConv3) {
        const int dz = t / 9, dy = (t / 3) % 3, dx = t % 3;
        return (dz * HY + dy) * HX + dx;
    }
    return ((t >> 2) * HY + ((t >> 1) & 1)) * HX + (t & 1);
}

template <int MODE, int TY, int TZ>
struct Halo {
    static constexpr int T = MODE == kConv3 ? 27 : 8;
    static constexpr int HX = MODE == kConv3 ? 18 : 32;
    static constexpr int HY = MODE == kConv3 ? TY + 2 : 2 * TY;
    static constexpr int HZ = MODE == kConv3 ? TZ + 2 : 2 * TZ;
    static constexpr int N = HX * HY * HZ;
    // halo voxel of output row r (= rz*TY + ry), x, for tap 0
    __device__ static int base(int r, int x) {
        const int ry = r % TY, rz = r / TY;
        if (MODE == kConv3) return (rz * HY + ry) * HX + x;
        return (2 * rz * HY + 2 * ry) * HX + 2 * x;
    }
};

// Stage a halo (or plain) tile of `CC` chunks per voxel into shared memory.
// (gz0, gy0, gx0): grid position of tile voxel 0; zero outside the grid.
template <int CC, int MODE, int HX, int HY, int HZ>
__device__ __forceinline__ void load_tile(uint4 *s, const bf16 *src, int ctot, int c0, int dd, int hh, int ww,
                                          int gz0, int gy0, int gx0, const bf16 *any_valid) {
    constexpr int N = HX * HY * HZ * CC;
    for (int q = threadIdx.x; q < N; q += kThreads) {
        const int cc = q % CC;
        const int hv = q / CC;
        const int hx = hv % HX;
        const int hy = (hv / HX) % HY;
        const int hz = hv / (HX * HY);
        const int gx = gx0 + hx, gy = gy0 + hy, gz = gz0 + hz;
        const bool ok = gx >= 0 && gx < ww && gy >= 0 && gy < hh && gz >= 0 && gz < dd;
        const bf16 *p = ok ? src + ((((size_t)gz * hh + gy) * ww + gx) * ctot + c0 + cc * 8) : any_valid;
        cp_async16(smem_u32(s + chunk_slot<CC, MODE>(hv, cc)), p, ok);
    }
}

// Stage the packed weight fragments of k16 steps [s0, s0+G) (of S) and
// n-tiles [j0, j0+NT) (of NTT) into dst, laid out [G][NT][32 lanes] uint2,
// with cp.async (256 contiguous bytes per (step, n-tile)).
template <int G, int NT>
__device__ __forceinline__ void stage_weights(uint2 *dst, const uint2 *wt, int s0, int S, int NTT, int j0) {
    constexpr int UNITS = G * NT * 16;
    for (int u = threadIdx.x; u < UNITS; u += kThreads) {
        const int q = u >> 4, part = u & 15;
        const int g = q / NT, j = q % NT;
        const int st = s0 + g;
        if (st < S)
            cp_async16(smem_u32(dst + (g * NT + j) * 32 + part * 2), wt + ((size_t)st * NTT + j0 + j) * 32 + part * 2,
                       true);
    }
}

// k16 steps staged per pipeline stage.
template <int S, int NT>
struct WeightStages {
    static constexpr int G0 = NT >= 8 ? 4 : 8;
    static constexpr int G = S < G0 ? S : G0;
    static constexpr int CHUNKS = (S + G - 1) / G;
    static constexpr int WORDS = G * NT * 32;  // uint2 per stage
};

// ---------------------------------------------------------------------------
// Gather convolution (3x3x3 s1 p1, or 2x2x2 s2): forward, and the
// backward-data pass of the 3x3x3 and of the transposed 2x2x2 convolution.
// ---------------------------------------------------------------------------
struct GatherArgs {
    const bf16 *x;
    const uint2 *wt;
    bf16 *y;
    double *stats;  // [n][cout][2] (sum, sum of squares) of the stored outputs, or null
    int id, ih, iw;
    int od, oh, ow;
    int tiles_x, tiles_y, tiles_z;
    int cout;  // total output channels; blockIdx.y selects a group of NT*8 of them
};

template <int MODE, int CC, int NT, int TY, int TZ>
__global__ void __launch_bounds__(kThreads) conv_gather_kernel(GatherArgs a) {
    using H = Halo<MODE, TY, TZ>;
    constexpr int WM = TY * TZ / 4;  // output rows (m16 tiles) per warp
    constexpr int KCH = H::T * CC;   // 8-channel chunks along K
    constexpr int S = (KCH + 1) / 2; // k16 steps
    constexpr int CG = NT * 8;  // output channels of this CTA
    static_assert(TY * TZ % 4 == 0, "4 warps share the rows of a tile");
    extern __shared__ uint4 smem[];
    __shared__ float s_stat[2 * CG];
    const int NTT = a.cout / 8;          // n-tiles of the whole layer
    const int j0 = blockIdx.y * NT;      // first n-tile of this CTA

    int b = blockIdx.x;
    const int tx = b % a.tiles_x;
    b /= a.tiles_x;
    const int ty = b % a.tiles_y;
    b /= a.tiles_y;
    const int tz = b % a.tiles_z;
    const int nb = b / a.tiles_z;
    const int ox0 = tx * 16, oy0 = ty * TY, oz0 = tz * TZ;
    const int tid = threadIdx.x;

    using WS = WeightStages<S, NT>;
    uint2 *sw = reinterpret_cast<uint2 *>(smem + H::N * CC);  // two weight stages after the tile
    {
        const bf16 *xs = a.x + (size_t)nb * a.id * a.ih * a.iw * (CC * 8);
        if (MODE == kConv3)
            load_tile<CC, MODE, H::HX, H::HY, H::HZ>(smem, xs, CC * 8, 0, a.id, a.ih, a.iw, oz0 - 1, oy0 - 1,
                                                     ox0 - 1, a.x);
        else
            load_tile<CC, MODE, H::HX, H::HY, H::HZ>(smem, xs, CC * 8, 0, a.id, a.ih, a.iw, 2 * oz0, 2 * oy0,
                                                     2 * ox0, a.x);
        stage_weights<WS::G, NT>(sw, a.wt, 0, S, NTT, j0);
        cp_async_commit();
    }
    if (a.stats)
        for (int q = tid; q < 2 * CG; q += kThreads) s_stat[q] = 0.f;

    const int warp = tid >> 5, lane = tid & 31;
    const int lrow = (lane & 7) + ((lane >> 3) & 1) * 8;  // ldmatrix row = output x in the tile
    const int khalf = lane >> 4;                          // which chunk of the k16 step
    int hv0[WM];
#pragma unroll
    for (int i = 0; i < WM; ++i) hv0[i] = H::base(warp * WM + i, lrow);

    float acc[WM][NT][4];
#pragma unroll
    for (int i = 0; i < WM; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

    const unsigned sbase = smem_u32(smem);
    // Weight pipeline: stage c+1 loads (cp.async) while stage c computes.
#pragma unroll 1
    for (int c = 0; c < WS::CHUNKS; ++c) {
        if (c + 1 < WS::CHUNKS) {
            stage_weights<WS::G, NT>(sw + ((c + 1) & 1) * WS::WORDS, a.wt, (c + 1) * WS::G, S, NTT, j0);
            cp_async_commit();
            cp_async_wait_group<1>();
        } else {
            cp_async_wait_group<0>();
        }
        __syncthreads();
        const uint2 *wb = sw + (c & 1) * WS::WORDS + lane;
#pragma unroll 1
        for (int g = 0; g < WS::G; ++g) {
            const int s = c * WS::G + g;
            if (s >= S) break;
            uint2 bfr[NT];
#pragma unroll
            for (int j = 0; j < NT; ++j) bfr[j] = wb[(g * NT + j) * 32];
            int kc = 2 * s + khalf;
            if ((KCH & 1) && kc >= KCH) kc = 0;  // padding chunk: its packed weights are zero
            const int t = kc / CC, cc = kc % CC;
            const int toff = tap_offset<MODE, H::HX, H::HY>(t);
#pragma unroll
            for (int i = 0; i < WM; ++i) {
                unsigned af[4];
                ldsm_x4(sbase + chunk_slot<CC, MODE>(hv0[i] + toff, cc) * 16, af);
#pragma unroll
                for (int j = 0; j < NT; ++j) mma_bf16(acc[i][j], af, bfr[j].x, bfr[j].y);
            }
        }
        __syncthreads();  // stage (c & 1) is refilled by the next iteration
    }

    // Epilogue: bf16 store (+ instance-norm statistics of the stored values).
    const int crow = lane >> 2, ccol = (lane & 3) * 2;
    float ssum[NT][2], ssq[NT][2];
#pragma unroll
    for (int j = 0; j < NT; ++j) ssum[j][0] = ssum[j][1] = ssq[j][0] = ssq[j][1] = 0.f;
#pragma unroll
    for (int i = 0; i < WM; ++i) {
        const int r = warp * WM + i;
        const int oy = oy0 + r % TY, oz = oz0 + r / TY;
#pragma unroll
        for (int hh = 0; hh < 2; ++hh) {
            const int ox = ox0 + crow + 8 * hh;
            if (ox >= a.ow || oy >= a.oh || oz >= a.od) continue;
            bf16 *dst = a.y + ((((size_t)nb * a.od + oz) * a.oh + oy) * a.ow + ox) * a.cout + 8 * j0 + ccol;
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                const __nv_bfloat162 v = __floats2bfloat162_rn(acc[i][j][2 * hh], acc[i][j][2 * hh + 1]);
                *reinterpret_cast<__nv_bfloat162 *>(dst + 8 * j) = v;
                const float f0 = __low2float(v), f1 = __high2float(v);
                ssum[j][0] += f0;
                ssum[j][1] += f1;
                ssq[j][0] += f0 * f0;
                ssq[j][1] += f1 * f1;
            }
        }
    }
    if (a.stats) {
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                float u = ssum[j][e], v = ssq[j][e];
#pragma unroll
                for (int o = 4; o < 32; o <<= 1) {
                    u += __shfl_xor_sync(0xffffffffu, u, o);
                    v += __shfl_xor_sync(0xffffffffu, v, o);
                }
                if (lane < 4) {
                    atomicAdd(&s_stat[8 * j + ccol + e], u);
                    atomicAdd(&s_stat[CG + 8 * j + ccol + e], v);
                }
            }
        __syncthreads();
        for (int q = tid; q < CG; q += kThreads) {
            const size_t c = (size_t)nb * a.cout + 8 * j0 + q;
            atomicAdd(&a.stats[c * 2 + 0], (double)s_stat[q]);
            atomicAdd(&a.stats[c * 2 + 1], (double)s_stat[CG + q]);
        }
    }
}

// ---------------------------------------------------------------------------
// Transposed 2x2x2 stride-2 convolution: out[2q + t] = W_t^T in[q] (+ addend).
// Forward of the decoder's up-sampling and backward-data of the down conv.
// ---------------------------------------------------------------------------
struct UpArgs {
    const bf16 *x;
    const uint2 *wt;
    const bf16 *addend;  // same shape as y, or null (may alias y)
    bf16 *y;
    int d, h, w;  // input (coarse) grid
    int tiles_x, tiles_y, tiles_z;
};

template <int CC, int NT, int TY, int TZ, int G>
__global__ void __launch_bounds__(kThreads) conv_up_kernel(UpArgs a) {
    constexpr int WM = TY * TZ / 4;
    constexpr int S = CC / 2;  // k16 steps per tap
    constexpr int COUT = NT * 8;
    static_assert(CC % 2 == 0, "transposed conv needs >= 16 input channels");
    extern __shared__ uint4 smem[];

    int b = blockIdx.x;
    const int tx = b % a.tiles_x;
    b /= a.tiles_x;
    const int ty = b % a.tiles_y;
    b /= a.tiles_y;
    const int tz = b % a.tiles_z;
    const int nb = b / a.tiles_z;
    const int ox0 = tx * 16, oy0 = ty * TY, oz0 = tz * TZ;
    const int tid = threadIdx.x;
    constexpr int WORDS = S * NT * 32;  // one tap's weights per stage
    uint2 *sw = reinterpret_cast<uint2 *>(smem + TZ * TY * 16 * CC);
    load_tile<CC, kConv3, 16, TY, TZ>(smem, a.x + (size_t)nb * a.d * a.h * a.w * (CC * 8), CC * 8, 0, a.d, a.h,
                                      a.w, oz0, oy0, ox0, a.x);
    // the CTA's taps: G groups of 8 / G taps over blockIdx.y (more CTAs on the
    // coarse grids, where one CTA per tile leaves SMs idle)
    constexpr int tpc = 8 / G;
    static_assert(tpc * G == 8, "tap groups divide the 8 taps");
    const int t0 = (int)blockIdx.y * tpc, t1 = t0 + tpc;
    stage_weights<S, NT>(sw, a.wt, t0 * S, 8 * S, NT, 0);
    cp_async_commit();

    const int warp = tid >> 5, lane = tid & 31;
    const int lrow = (lane & 7) + ((lane >> 3) & 1) * 8;
    const int khalf = lane >> 4;
    const int crow = lane >> 2, ccol = (lane & 3) * 2;
    const unsigned sbase = smem_u32(smem);
    const int fd = 2 * a.d, fh = 2 * a.h, fw = 2 * a.w;

#pragma unroll 1
    for (int t = t0; t < t1; ++t) {
        if (t + 1 < t1) {
            stage_weights<S, NT>(sw + ((t + 1 - t0) & 1) * WORDS, a.wt, (t + 1) * S, 8 * S, NT, 0);
            cp_async_commit();
            cp_async_wait_group<1>();
        } else {
            cp_async_wait_group<0>();
        }
        __syncthreads();
        const uint2 *wb = sw + ((t - t0) & 1) * WORDS + lane;
        float acc[WM][NT][4];
#pragma unroll
        for (int i = 0; i < WM; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            uint2 bfr[NT];
#pragma unroll
            for (int j = 0; j < NT; ++j) bfr[j] = wb[(s * NT + j) * 32];
            const int cc = 2 * s + khalf;
#pragma unroll
            for (int i = 0; i < WM; ++i) {
                unsigned af[4];
                ldsm_x4(sbase + chunk_slot<CC, kConv3>((warp * WM + i) * 16 + lrow, cc) * 16, af);
#pragma unroll
                for (int j = 0; j < NT; ++j) mma_bf16(acc[i][j], af, bfr[j].x, bfr[j].y);
            }
        }
        const int dz = t >> 2, dy = (t >> 1) & 1, dx = t & 1;
#pragma unroll
        for (int i = 0; i < WM; ++i) {
            const int r = warp * WM + i;
            const int cy = oy0 + r % TY, cz = oz0 + r / TY;
#pragma unroll
            for (int hh = 0; hh < 2; ++hh) {
                const int cx = ox0 + crow + 8 * hh;
                if (cx >= a.w || cy >= a.h || cz >= a.d) continue;
                const size_t o =
                    ((((size_t)nb * fd + 2 * cz + dz) * fh + 2 * cy + dy) * fw + 2 * cx + dx) * COUT + ccol;
#pragma unroll
                for (int j = 0; j < NT; ++j) {
                    float v0 = acc[i][j][2 * hh], v1 = acc[i][j][2 * hh + 1];
                    if (a.addend) {
                        const __nv_bfloat162 ad = *reinterpret_cast<const __nv_bfloat162 *>(a.addend + o + 8 * j);
                        v0 += __low2float(ad);
                        v1 += __high2float(ad);
                    }
                    *reinterpret_cast<__nv_bfloat162 *>(a.y + o + 8 * j) = __floats2bfloat162_rn(v0, v1);
                }
            }
        }
        __syncthreads();  // stage (t & 1) is refilled by the next iteration
    }
}

// ---------------------------------------------------------------------------
// Weight gradient: G[t][a][b] += sum_o P[g(o, t)][a] * Q[o][b], o over the Q
// grid.  Each CTA owns a group of taps and a range of b-chunks and reduces a
// contiguous run of Q tiles in registers before one fp32 atomicAdd per weight.
// ---------------------------------------------------------------------------
struct WgradArgs {
    const bf16 *p, *q;
    float *g;
    int d, h, w;     // Q grid
    int pd, ph, pw;  // P grid
    int tiles_x, tiles_y, tiles_z, n_tiles, tiles_per_split;
    int tg, b_groups;
    int cb;  // total Q channels
};

template <int MODE, int CCA, int NBT, int TY, int TZ>
__global__ void __launch_bounds__(kThreads) conv_wgrad_kernel(WgradArgs a) {
    using H = Halo<MODE, TY, TZ>;
    constexpr int MT = (CCA + 1) / 2;  // m16 tiles over P channels
    constexpr int PPW = 16 / NBT;      // (tap, m-tile) pairs per warp
    constexpr int CA = CCA * 8;
    constexpr int ROWS = TY * TZ;
    static_assert(NBT % 2 == 0, "b range is a whole number of 16-channel pairs");
    extern __shared__ uint4 smem[];
    uint4 *sp = smem;
    uint4 *sq = smem + H::N * CCA;

    const int bg = blockIdx.y % a.b_groups, tgi = blockIdx.y / a.b_groups;
    const int t0 = tgi * a.tg, t1 = min(H::T, t0 + a.tg);
    const int qc0 = bg * NBT;  // first Q chunk of this CTA
    const int npairs = (t1 - t0) * MT;
    const int tile_begin = blockIdx.x * a.tiles_per_split;
    const int tile_end = min(a.n_tiles, tile_begin + a.tiles_per_split);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mm = lane >> 3, rr = lane & 7;

    float acc[PPW][NBT][4];
#pragma unroll
    for (int k = 0; k < PPW; ++k)
#pragma unroll
        for (int j = 0; j < NBT; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[k][j][e] = 0.f;

    const unsigned spb = smem_u32(sp), sqb = smem_u32(sq);
    const int cq = a.cb / 8;  // Q chunks per voxel
#pragma unroll 1
    for (int tile = tile_begin; tile < tile_end; ++tile) {
        int b = tile;
        const int tx = b % a.tiles_x;
        b /= a.tiles_x;
        const int ty = b % a.tiles_y;
        b /= a.tiles_y;
        const int tz = b % a.tiles_z;
        const int nb = b / a.tiles_z;
        const int ox0 = tx * 16, oy0 = ty * TY, oz0 = tz * TZ;
        __syncthreads();  // the previous tile's reads are done
        {
            const bf16 *ps = a.p + (size_t)nb * a.pd * a.ph * a.pw * CA;
            if (MODE == kConv3)
                load_tile<CCA, MODE, H::HX, H::HY, H::HZ>(sp, ps, CA, 0, a.pd, a.ph, a.pw, oz0 - 1, oy0 - 1,
                                                          ox0 - 1, a.p);
            else
                load_tile<CCA, MODE, H::HX, H::HY, H::HZ>(sp, ps, CA, 0, a.pd, a.ph, a.pw, 2 * oz0, 2 * oy0,
                                                          2 * ox0, a.p);
            const bf16 *qs = a.q + (size_t)nb * a.d * a.h * a.w * a.cb;
            load_tile<NBT, kConv3, 16, TY, TZ>(sq, qs, a.cb, qc0 * 8, a.d, a.h, a.w, oz0, oy0, ox0, a.q);
        }
        cp_async_wait_all();
        __syncthreads();

#pragma unroll 1
        for (int r = 0; r < ROWS; ++r) {
            unsigned bfr[NBT][2];
#pragma unroll
            for (int jj = 0; jj < NBT / 2; ++jj) {
                unsigned q4[4];
                ldsm_x4_t(sqb + chunk_slot<NBT, kConv3>(r * 16 + rr + (mm & 1) * 8, 2 * jj + (mm >> 1)) * 16, q4);
                bfr[2 * jj][0] = q4[0];
                bfr[2 * jj][1] = q4[1];
                bfr[2 * jj + 1][0] = q4[2];
                bfr[2 * jj + 1][1] = q4[3];
            }
            const int hvb = H::base(r, rr + (mm >> 1) * 8);
#pragma unroll
            for (int k = 0; k < PPW; ++k) {
                const int pk = warp + 4 * k;
                if (pk >= npairs) break;  // warp-uniform
                const int t = t0 + pk / MT, mt = pk % MT;
                const int chunk = CCA == 1 ? 0 : 2 * mt + (mm & 1);
                unsigned af[4];
                ldsm_x4_t(spb + chunk_slot<CCA, MODE>(hvb + tap_offset<MODE, H::HX, H::HY>(t), chunk) * 16, af);
                if (CCA == 1) af[1] = af[3] = 0u;  // rows 8..15 of the m16 tile do not exist
#pragma unroll
                for (int j = 0; j < NBT; ++j) mma_bf16(acc[k][j], af, bfr[j][0], bfr[j][1]);
            }
        }
    }

#pragma unroll
    for (int k = 0; k < PPW; ++k) {
        const int pk = warp + 4 * k;
        if (pk >= npairs) break;
        const int t = t0 + pk / MT, mt = pk % MT;
#pragma unroll
        for (int j = 0; j < NBT; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int ar = 16 * mt + (lane >> 2) + (e >> 1) * 8;
                const int bc = 8 * (qc0 + j) + (lane & 3) * 2 + (e & 1);
                if (ar < CA) atomicAdd(&a.g[((size_t)t * CA + ar) * a.cb + bc], acc[k][j][e]);
            }
    }
    (void)cq;
}

// ---------------------------------------------------------------------------
// Weight packing into mma B-fragment order.
// ---------------------------------------------------------------------------
__global__ void pack_weights_kernel(const float *__restrict__ m, int T, int A, int B, int flip, int trans, int S,
                                    int NTt, uint2 *__restrict__ out) {
    const long long total = (long long)S * NTt * 32;
    const long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int lane = (int)(idx % 32);
    const int j = (int)((idx / 32) % NTt);
    const int s = (int)(idx / (32LL * NTt));
    const int Kc = trans ? B : A;
    const int K = T * Kc;
    const int n = 8 * j + lane / 4;
    float v[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const int k = 16 * s + 2 * (lane % 4) + (e & 1) + (e >> 1) * 8;
        if (k >= K) {
            v[e] = 0.f;
            continue;
        }
        const int t = k / Kc, kk = k % Kc;
        const int tt = flip ? T - 1 - t : t;
        v[e] = trans ? m[((size_t)tt * A + n) * B + kk] : m[((size_t)tt * A + kk) * B + n];
    }
    const __nv_bfloat162 lo = __floats2bfloat162_rn(v[0], v[1]);
    const __nv_bfloat162 hi = __floats2bfloat162_rn(v[2], v[3]);
    uint2 o;
    o.x = *reinterpret_cast<const unsigned *>(&lo);
    o.y = *reinterpret_cast<const unsigned *>(&hi);
    out[idx] = o;
}

// ---------------------------------------------------------------------------
// Instance norm + LeakyReLU.
// ---------------------------------------------------------------------------
__global__ void norm_finalize_kernel(const double *__restrict__ stats, int nc, int c, double count,
                                     const float *__restrict__ gamma, const float *__restrict__ beta, float eps,
                                     float4 *__restrict__ coef) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nc) return;
    const int ch = q % c;
    const double mean = stats[2 * q] / count;
    const double var = fmax(stats[2 * q + 1] / count - mean * mean, 0.0);
    const float rstd = (float)(1.0 / sqrt(var + (double)eps));
    const float alpha = gamma[ch] * rstd;
    coef[q] = make_float4(alpha, beta[ch] - (float)mean * alpha, (float)mean, rstd);
}

__device__ __forceinline__ void unpack8(const uint4 &u, float (&f)[8]) {
    const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        f[2 * i] = __low2float(h[i]);
        f[2 * i + 1] = __high2float(h[i]);
    }
}

__device__ __forceinline__ uint4 pack8(const float (&f)[8]) {
    uint4 u;
    __nv_bfloat162 *h = reinterpret_cast<__nv_bfloat162 *>(&u);
#pragma unroll
    for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
    return u;
}

// Instance-norm coefficients of (sample, channel) q from the convolution's
// statistics (see norm_finalize_kernel).
__device__ __forceinline__ float4 norm_coef(const double *stats, int q, int ch, double count, const float *gamma,
                                           const float *beta, float eps) {
    const double mean = stats[2 * q] / count;
    const double var = fmax(stats[2 * q + 1] / count - mean * mean, 0.0);
    const float rstd = (float)(1.0 / sqrt(var + (double)eps));
    const float alpha = gamma[ch] * rstd;
    return make_float4(alpha, beta[ch] - (float)mean * alpha, (float)mean, rstd);
}

// Finalize + apply in one pass: every block derives the coefficients of all
// (sample, channel) pairs into shared memory (block 0 also stores them for
// the backward pass), then a = lrelu(alpha*y + shift), 8 channels per thread.
__global__ void norm_stats_act_kernel(const uint4 *__restrict__ y, long long chunks, int cc_per_vox, long long vox,
                                      int n, int c, const double *__restrict__ stats, double count,
                                      const float *__restrict__ gamma, const float *__restrict__ beta, float eps,
                                      float slope, float4 *__restrict__ coef_out, uint4 *__restrict__ out) {
    extern __shared__ float4 s_coef[];
    for (int q = threadIdx.x; q < n * c; q += blockDim.x) {
        const float4 k = norm_coef(stats, q, q % c, count, gamma, beta, eps);
        s_coef[q] = k;
        if (blockIdx.x == 0 && coef_out) coef_out[q] = k;
    }
    __syncthreads();
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < chunks;
         q += (long long)gridDim.x * blockDim.x) {
        const long long v = q / cc_per_vox;
        const int cc = (int)(q - v * cc_per_vox);
        const int nb = (int)(v / vox);
        float f[8];
        unpack8(__ldg(y + q), f);
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const float4 k = s_coef[nb * c + cc * 8 + e];
            const float z = fmaf(f[e], k.x, k.y);
            f[e] = z > 0.f ? z : slope * z;
        }
        out[q] = pack8(f);
    }
}

// a = lrelu(alpha*y + shift), 8 channels per thread.
__global__ void norm_act_kernel(const uint4 *__restrict__ y, long long chunks, int cc_per_vox, long long vox,
                                int c, const float4 *__restrict__ coef, float slope, uint4 *__restrict__ out) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < chunks;
         q += (long long)gridDim.x * blockDim.x) {
        const long long v = q / cc_per_vox;
        const int cc = (int)(q - v * cc_per_vox);
        const int nb = (int)(v / vox);
        float f[8];
        unpack8(__ldg(y + q), f);
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const float4 k = __ldg(coef + (size_t)nb * c + cc * 8 + e);
            const float z = fmaf(f[e], k.x, k.y);
            f[e] = z > 0.f ? z : slope * z;
        }
        out[q] = pack8(f);
    }
}

// Pass 1 of the backward: per (n, c) sums of dz and dz*yhat, where
// dz = da * lrelu'(alpha*y + shift) and yhat = (y - mean)*rstd.
__global__ void __launch_bounds__(256) norm_bwd_reduce_kernel(const uint4 *__restrict__ y,
                                                              const uint4 *__restrict__ da, int cc_per_vox,
                                                              long long vox, int c, const float4 *__restrict__ coef,
                                                              float slope, double *__restrict__ red) {
    __shared__ float s_red[2 * 128];
    const int nb = blockIdx.y;
    const int cc = threadIdx.x % cc_per_vox;
    const int vpb = blockDim.x / cc_per_vox;
    for (int q = threadIdx.x; q < 2 * c; q += blockDim.x) s_red[q] = 0.f;
    __syncthreads();
    float s1[8], s2[8];
    float4 k[8];
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        s1[e] = s2[e] = 0.f;
        k[e] = __ldg(coef + (size_t)nb * c + cc * 8 + e);
    }
    const int vt = threadIdx.x / cc_per_vox;
    if (vt < vpb) {
        for (long long v = blockIdx.x * (long long)vpb + vt; v < vox; v += (long long)gridDim.x * vpb) {
            const size_t q = ((size_t)nb * vox + v) * cc_per_vox + cc;
            float fy[8], fd[8];
            unpack8(__ldg(y + q), fy);
            unpack8(__ldg(da + q), fd);
#pragma unroll
            for (int e = 0; e < 8; ++e) {
                const float z = fmaf(fy[e], k[e].x, k[e].y);
                const float dz = z > 0.f ? fd[e] : slope * fd[e];
                const float yh = (fy[e] - k[e].z) * k[e].w;
                s1[e] += dz;
                s2[e] += dz * yh;
            }
        }
    }
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        atomicAdd(&s_red[cc * 8 + e], s1[e]);
        atomicAdd(&s_red[c + cc * 8 + e], s2[e]);
    }
    __syncthreads();
    for (int q = threadIdx.x; q < c; q += blockDim.x) {
        atomicAdd(&red[((size_t)nb * c + q) * 2 + 0], (double)s_red[q]);
        atomicAdd(&red[((size_t)nb * c + q) * 2 + 1], (double)s_red[c + q]);
    }
}

// Pass 2: dy = gamma*rstd*(dz - mean(dz) - yhat*mean(dz*yhat)).
__global__ void norm_bwd_apply_kernel(const uint4 *__restrict__ y, const uint4 *__restrict__ da, long long chunks,
                                      int cc_per_vox, long long vox, int c, const float4 *__restrict__ coef,
                                      const float *__restrict__ gamma, float slope, const double *__restrict__ red,
                                      uint4 *__restrict__ dy) {
    const double inv = 1.0 / (double)vox;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < chunks;
         q += (long long)gridDim.x * blockDim.x) {
        const long long v = q / cc_per_vox;
        const int cc = (int)(q - v * cc_per_vox);
        const int nb = (int)(v / vox);
        float fy[8], fd[8];
        unpack8(__ldg(y + q), fy);
        unpack8(__ldg(da + q), fd);
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int ch = cc * 8 + e;
            const float4 k = __ldg(coef + (size_t)nb * c + ch);
            const float m1 = (float)(red[((size_t)nb * c + ch) * 2 + 0] * inv);
            const float m2 = (float)(red[((size_t)nb * c + ch) * 2 + 1] * inv);
            const float z = fmaf(fy[e], k.x, k.y);
            const float dz = z > 0.f ? fd[e] : slope * fd[e];
            const float yh = (fy[e] - k.z) * k.w;
            fd[e] = __ldg(gamma + ch) * k.w * (dz - m1 - yh * m2);
        }
        dy[q] = pack8(fd);
    }
}

__global__ void norm_param_grad_kernel(const double *__restrict__ red, int n, int c, float *__restrict__ dgamma,
                                       float *__restrict__ dbeta) {
    const int ch = blockIdx.x * blockDim.x + threadIdx.x;
    if (ch >= c) return;
    double g = 0.0, b = 0.0;
    for (int nb = 0; nb < n; ++nb) {
        b += red[((size_t)nb * c + ch) * 2 + 0];
        g += red[((size_t)nb * c + ch) * 2 + 1];
    }
    dgamma[ch] = (float)g;
    dbeta[ch] = (float)b;
}

// ---------------------------------------------------------------------------
// Network input and output head.
// ---------------------------------------------------------------------------
__global__ void pack_input_kernel(const float *__restrict__ terma, const float *__restrict__ density, long long vox,
                                  float terma_scale, uint4 *__restrict__ x8) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < vox;
         v += (long long)gridDim.x * blockDim.x) {
        float f[8] = {__ldg(terma + v) * terma_scale, __ldg(density + v), 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        x8[v] = pack8(f);
    }
}

// out = active ? scale*(w.g + bias) : 0 with active = mask > mask_thr (16 channels).
__global__ void head_fwd_kernel(const uint4 *__restrict__ g, long long vox, const float *__restrict__ w,
                                const float *__restrict__ bias, const float *__restrict__ mask, float mask_thr,
                                float scale, float *__restrict__ out) {
    __shared__ float s_w[17];
    if (threadIdx.x < 16) s_w[threadIdx.x] = w[threadIdx.x];
    if (threadIdx.x == 16) s_w[16] = bias[0];
    __syncthreads();
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < vox;
         v += (long long)gridDim.x * blockDim.x) {
        float r = 0.f;
        if (__ldg(mask + v) > mask_thr) {
            float f[8];
            float acc = s_w[16];
            unpack8(__ldg(g + 2 * v), f);
#pragma unroll
            for (int e = 0; e < 8; ++e) acc = fmaf(s_w[e], f[e], acc);
            unpack8(__ldg(g + 2 * v + 1), f);
#pragma unroll
            for (int e = 0; e < 8; ++e) acc = fmaf(s_w[8 + e], f[e], acc);
            r = scale * acc;
        }
        out[v] = r;
    }
}

// Squared-error loss over the voxels with target >= 0 (inactive voxels carry
// a negative sentinel), its gradient to the 16 head input channels and to the
// head's weights and bias.
__global__ void __launch_bounds__(256) head_loss_bwd_kernel(const uint4 *__restrict__ g, long long vox,
                                                            const float *__restrict__ w,
                                                            const float *__restrict__ pred,
                                                            const float *__restrict__ target, float inv_count_arg,
                                                            const float *__restrict__ inv_count_dev,
                                                            double *__restrict__ loss, uint4 *__restrict__ dg,
                                                            float *__restrict__ dw, float *__restrict__ dbias) {
    const float inv_count = inv_count_dev ? *inv_count_dev : inv_count_arg;
    __shared__ float s_w[16];
    __shared__ float s_acc[18];
    if (threadIdx.x < 16) s_w[threadIdx.x] = w[threadIdx.x];
    if (threadIdx.x < 18) s_acc[threadIdx.x] = 0.f;
    __syncthreads();
    float lw[16], lb = 0.f, ll = 0.f;
#pragma unroll
    for (int e = 0; e < 16; ++e) lw[e] = 0.f;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < vox;
         v += (long long)gridDim.x * blockDim.x) {
        const float t = __ldg(target + v);
        const float diff = t >= 0.f ? __ldg(pred + v) - t : 0.f;
        const float dp = 2.f * diff * inv_count;
        ll += diff * diff;
        lb += dp;
        float f[8], o[8];
        unpack8(__ldg(g + 2 * v), f);
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            lw[e] += f[e] * dp;
            o[e] = s_w[e] * dp;
        }
        dg[2 * v] = pack8(o);
        unpack8(__ldg(g + 2 * v + 1), f);
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            lw[8 + e] += f[e] * dp;
            o[e] = s_w[8 + e] * dp;
        }
        dg[2 * v + 1] = pack8(o);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lb += __shfl_xor_sync(0xffffffffu, lb, o);
        ll += __shfl_xor_sync(0xffffffffu, ll, o);
#pragma unroll
        for (int e = 0; e < 16; ++e) lw[e] += __shfl_xor_sync(0xffffffffu, lw[e], o);
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int e = 0; e < 16; ++e) atomicAdd(&s_acc[e], lw[e]);
        atomicAdd(&s_acc[16], lb);
        atomicAdd(&s_acc[17], ll * inv_count);
    }
    __syncthreads();
    if (threadIdx.x < 16) atomicAdd(&dw[threadIdx.x], s_acc[threadIdx.x]);
    if (threadIdx.x == 16) atomicAdd(dbias, s_acc[16]);
    if (threadIdx.x == 17) atomicAdd(loss, (double)s_acc[17]);
}

// ---------------------------------------------------------------------------
// Host helpers
// ---------------------------------------------------------------------------
void need(bool ok, const std::string &msg) {
    if (!ok) throw Error(DC_ERR_VALUE, msg);
}

// Device of the current C-ABI call; bound (cudaSetDevice) only after the
// arguments have been validated, so argument errors never touch a GPU.
thread_local int g_call_device = -1;

void bind_device() {
    if (g_call_device < 0) return;
    int n = 0;
    DC_CUDA(cudaGetDeviceCount(&n));
    if (g_call_device >= n) throw Error(DC_ERR_CUDA, "invalid device ordinal");
    DC_CUDA(cudaSetDevice(g_call_device));
}

bool gather_supported(int mode, int cin, int cout) {
    if (mode == kConv3)
        return (cin == 8 && cout == 16) || (cin == cout && (cin == 16 || cin == 32 || cin == 64 || cin == 128));
    if (mode == kDown2) return cout == 2 * cin && (cin == 16 || cin == 32 || cin == 64);
    return false;
}

int sm_count() {
    int dev = 0, n = 0;
    DC_CUDA(cudaGetDevice(&dev));
    DC_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    return n;
}

unsigned elementwise_blocks(long long work, int threads) {
    const long long want = (work + threads - 1) / threads;
    const long long cap = (long long)sm_count() * 16;
    return (unsigned)std::max(1LL, std::min(want, cap));
}

// Dynamic shared-memory opt-in, once per kernel instantiation and device
// (so that launches inside a CUDA-graph capture make no attribute calls).
template <class K>
void set_smem(K kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> done;  // (kernel, device) -> opted-in bytes
    int dev = 0;
    DC_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_pair(reinterpret_cast<const void *>(kernel), dev);
    std::lock_guard<std::mutex> lk(mu);
    auto it = done.find(key);
    if (it != done.end() && it->second >= bytes) return;
    DC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    done[key] = bytes;
}

template <int MODE, int CC, int NT, int TY, int TZ>
void launch_gather(const GatherArgs &a0, int n, cudaStream_t s) {
    using H = Halo<MODE, TY, TZ>;
    GatherArgs a = a0;
    a.tiles_x = (a.ow + 15) / 16;
    a.tiles_y = (a.oh + TY - 1) / TY;
    a.tiles_z = (a.od + TZ - 1) / TZ;
    constexpr int S = (H::T * CC + 1) / 2;
    const size_t smem = (size_t)H::N * CC * 16 + 2 * (size_t)WeightStages<S, NT>::WORDS * sizeof(uint2);
    auto k = conv_gather_kernel<MODE, CC, NT, TY, TZ>;
    set_smem(k, smem);
    const long long blocks = (long long)n * a.tiles_x * a.tiles_y * a.tiles_z;
    need(blocks < 0x7fffffffLL, "volume too large for the surrogate convolution");
    k<<<dim3((unsigned)blocks, (unsigned)(a.cout / (8 * NT))), kThreads, smem, s>>>(a);
    check_launch("conv_gather_kernel");
}

template <int CC, int NT, int TY, int TZ, int G>
void launch_up_groups(const UpArgs &a, long long blocks, cudaStream_t s) {
    const size_t smem = (size_t)TZ * TY * 16 * CC * 16 + 2 * (size_t)(CC / 2) * NT * 32 * sizeof(uint2);
    auto k = conv_up_kernel<CC, NT, TY, TZ, G>;
    set_smem(k, smem);
    k<<<dim3((unsigned)blocks, (unsigned)G), kThreads, smem, s>>>(a);
    check_launch("conv_up_kernel");
}

template <int CC, int NT, int TY, int TZ>
void launch_up(const UpArgs &a0, int n, cudaStream_t s) {
    UpArgs a = a0;
    a.tiles_x = (a.w + 15) / 16;
    a.tiles_y = (a.h + TY - 1) / TY;
    a.tiles_z = (a.d + TZ - 1) / TZ;
    const long long blocks = (long long)n * a.tiles_x * a.tiles_y * a.tiles_z;
    need(blocks < 0x7fffffffLL, "volume too large for the surrogate convolution");
    // tap groups: at least two waves of CTAs on the 148 SMs (measured: 16^3
    // -> 32^3 128 -> 64 channels 54.6 -> 11.5 us, 32^3 -> 64^3 52.8 -> 21.3 us)
    if (blocks >= 2 * 148) return launch_up_groups<CC, NT, TY, TZ, 1>(a, blocks, s);
    if (2 * blocks >= 2 * 148) return launch_up_groups<CC, NT, TY, TZ, 2>(a, blocks, s);
    if (4 * blocks >= 2 * 148) return launch_up_groups<CC, NT, TY, TZ, 4>(a, blocks, s);
    return launch_up_groups<CC, NT, TY, TZ, 8>(a, blocks, s);
}

template <int MODE, int CCA, int NBT, int TY, int TZ>
void launch_wgrad(const WgradArgs &a0, int n, cudaStream_t s) {
    using H = Halo<MODE, TY, TZ>;
    WgradArgs a = a0;
    a.tiles_x = (a.w + 15) / 16;
    a.tiles_y = (a.h + TY - 1) / TY;
    a.tiles_z = (a.d + TZ - 1) / TZ;
    a.n_tiles = n * a.tiles_x * a.tiles_y * a.tiles_z;
    constexpr int MT = (CCA + 1) / 2;
    constexpr int PPW = 16 / NBT;
    a.tg = std::max(1, std::min(H::T, 4 * PPW / MT));
    const int tap_groups = (H::T + a.tg - 1) / a.tg;
    a.b_groups = a.cb / (8 * NBT);
    const int groups = tap_groups * a.b_groups;
    const int target = 4 * sm_count();
    int splits = std::max(1, std::min(a.n_tiles, (target + groups - 1) / groups));
    a.tiles_per_split = (a.n_tiles + splits - 1) / splits;
    splits = (a.n_tiles + a.tiles_per_split - 1) / a.tiles_per_split;
    const size_t smem = ((size_t)H::N * CCA + (size_t)TZ * TY * 16 * NBT) * 16;
    auto k = conv_wgrad_kernel<MODE, CCA, NBT, TY, TZ>;
    set_smem(k, smem);
    k<<<dim3((unsigned)splits, (unsigned)groups), kThreads, smem, s>>>(a);
    check_launch("conv_wgrad_kernel");
}

}  // namespace

void set_call_device(int gpu_id) { g_call_device = gpu_id; }

long long packed_fragments(int taps, int k_per_tap, int n) {
    return (long long)((taps * k_per_tap + 15) / 16) * (n / 8) * 32;
}

void pack_weights(const float *master, int taps, int a, int b, int flip, int trans, uint2 *out, cudaStream_t s) {
    need(master && out, "weights must not be NULL");
    need(taps > 0 && a > 0 && b > 0, "weight shape must be positive");
    const int Kc = trans ? b : a, N = trans ? a : b;
    need(N % 8 == 0, "output channels must be a multiple of 8");
    bind_device();
    const int S = (taps * Kc + 15) / 16;
    const long long total = (long long)S * (N / 8) * 32;
    pack_weights_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(master, taps, a, b, flip, trans, S, N / 8,
                                                                          out);
    check_launch("pack_weights_kernel");
}

void conv_gather(int mode, const bf16 *x, int n, int d, int h, int w, int cin, const uint2 *wpk, long long wpk_frags,
                 int cout, bf16 *y, double *stats, cudaStream_t s) {
    need(x && wpk && y, "convolution buffers must not be NULL");
    need(n > 0 && d > 0 && h > 0 && w > 0, "convolution grid must be positive");
    need(mode == kConv3 || mode == kDown2, "unknown convolution mode");
    GatherArgs a{};
    a.x = x;
    a.wt = wpk;
    a.y = y;
    a.stats = stats;
    a.id = d;
    a.ih = h;
    a.iw = w;
    a.cout = cout;
    if (mode == kConv3) {
        a.od = d;
        a.oh = h;
        a.ow = w;
    } else {
        need(d % 2 == 0 && h % 2 == 0 && w % 2 == 0, "down-sampling needs even grid dimensions");
        a.od = d / 2;
        a.oh = h / 2;
        a.ow = w / 2;
    }
    need(gather_supported(mode, cin, cout), "unsupported convolution channels " + std::to_string(cin) + " -> " +
                                                std::to_string(cout));
    need(wpk_frags == packed_fragments(mode == kConv3 ? 27 : 8, cin, cout),
         "packed weights do not match the convolution's shape");
    bind_device();
    if (stats) DC_CUDA(cudaMemsetAsync(stats, 0, sizeof(double) * 2 * n * cout, s));
    if (mode == kConv3) {
        if (cin == 8 && cout == 16) return launch_gather<kConv3, 1, 2, 8, 2>(a, n, s);
        if (cin == 16 && cout == 16) return launch_gather<kConv3, 2, 2, 8, 2>(a, n, s);
        if (cin == 32 && cout == 32) return launch_gather<kConv3, 4, 4, 8, 2>(a, n, s);
        if (cin == 64 && cout == 64) return launch_gather<kConv3, 8, 4, 8, 2>(a, n, s);      // 2 channel groups
        if (cin == 128 && cout == 128) return launch_gather<kConv3, 16, 4, 4, 2>(a, n, s);  // 4 channel groups
    } else {
        if (cin == 16 && cout == 32) return launch_gather<kDown2, 2, 4, 8, 2>(a, n, s);
        if (cin == 32 && cout == 64) return launch_gather<kDown2, 4, 8, 4, 2>(a, n, s);
        if (cin == 64 && cout == 128) return launch_gather<kDown2, 8, 4, 4, 2>(a, n, s);  // 4 channel groups
    }
    throw Error(DC_ERR_VALUE, "unsupported convolution channels " + std::to_string(cin) + " -> " +
                                  std::to_string(cout));
}

void conv_up(const bf16 *x, int n, int d, int h, int w, int cin, const uint2 *wpk, long long wpk_frags, int cout,
             const bf16 *addend, bf16 *y, cudaStream_t s) {
    need(x && wpk && y, "convolution buffers must not be NULL");
    need(n > 0 && d > 0 && h > 0 && w > 0, "convolution grid must be positive");
    UpArgs a{};
    a.x = x;
    a.wt = wpk;
    a.addend = addend;
    a.y = y;
    a.d = d;
    a.h = h;
    a.w = w;
    need(cout * 2 == cin && (cin == 32 || cin == 64 || cin == 128),
         "unsupported transposed convolution channels " + std::to_string(cin) + " -> " + std::to_string(cout));
    need(wpk_frags == packed_fragments(8, cin, cout), "packed weights do not match the convolution's shape");
    bind_device();
    if (cin == 32 && cout == 16) return launch_up<4, 2, 8, 2>(a, n, s);
    if (cin == 64 && cout == 32) return launch_up<8, 4, 8, 2>(a, n, s);
    if (cin == 128 && cout == 64) return launch_up<16, 8, 4, 2>(a, n, s);
    throw Error(DC_ERR_VALUE, "unsupported transposed convolution channels " + std::to_string(cin) + " -> " +
                                  std::to_string(cout));
}

void conv_wgrad(int mode, const bf16 *p, const bf16 *q, int n, int d, int h, int w, int ca, int cb, float *grad,
                cudaStream_t s) {
    need(p && q && grad, "gradient buffers must not be NULL");
    need(n > 0 && d > 0 && h > 0 && w > 0, "convolution grid must be positive");
    WgradArgs a{};
    a.p = p;
    a.q = q;
    a.g = grad;
    a.d = d;
    a.h = h;
    a.w = w;
    a.cb = cb;
    const int T = mode == kConv3 ? 27 : 8;
    if (mode == kConv3) {
        a.pd = d;
        a.ph = h;
        a.pw = w;
    } else {
        a.pd = 2 * d;
        a.ph = 2 * h;
        a.pw = 2 * w;
    }
    need(gather_supported(mode, ca, cb), "unsupported weight-gradient channels " + std::to_string(ca) + " x " +
                                             std::to_string(cb));
    bind_device();
    DC_CUDA(cudaMemsetAsync(grad, 0, sizeof(float) * (size_t)T * ca * cb, s));
    if (mode == kConv3) {
        if (ca == 8 && cb == 16) return launch_wgrad<kConv3, 1, 2, 8, 4>(a, n, s);
        if (ca == 16 && cb == 16) return launch_wgrad<kConv3, 2, 2, 8, 4>(a, n, s);
        if (ca == 32 && cb == 32) return launch_wgrad<kConv3, 4, 4, 8, 2>(a, n, s);
        if (ca == 64 && cb == 64) return launch_wgrad<kConv3, 8, 8, 4, 2>(a, n, s);
        if (ca == 128 && cb == 128) return launch_wgrad<kConv3, 16, 8, 4, 2>(a, n, s);
    } else if (mode == kDown2) {
        if (ca == 16 && cb == 32) return launch_wgrad<kDown2, 2, 4, 8, 2>(a, n, s);
        if (ca == 32 && cb == 64) return launch_wgrad<kDown2, 4, 8, 4, 2>(a, n, s);
        if (ca == 64 && cb == 128) return launch_wgrad<kDown2, 8, 8, 4, 2>(a, n, s);
    }
    throw Error(DC_ERR_VALUE, "unsupported weight-gradient channels " + std::to_string(ca) + " x " +
                                  std::to_string(cb));
}

void norm_finalize(const double *stats, int n, int c, long long count, const float *gamma, const float *beta,
                   float eps, float *coef, cudaStream_t s) {
    need(stats && gamma && beta && coef, "norm buffers must not be NULL");
    need(count > 0 && n > 0 && c > 0, "norm count must be positive");
    bind_device();
    const int nc = n * c;
    norm_finalize_kernel<<<(nc + 127) / 128, 128, 0, s>>>(stats, nc, c, (double)count, gamma, beta, eps,
                                                          reinterpret_cast<float4 *>(coef));
    check_launch("norm_finalize_kernel");
}

void norm_act(const bf16 *y, int n, long long vox, int c, const float *coef, float slope, bf16 *out, cudaStream_t s) {
    need(y && coef && out, "norm buffers must not be NULL");
    need(c % 8 == 0 && c <= 128, "norm channels must be a multiple of 8, at most 128");
    need(n > 0 && vox > 0, "norm volume must be positive");
    bind_device();
    const long long chunks = (long long)n * vox * (c / 8);
    norm_act_kernel<<<elementwise_blocks(chunks, 256), 256, 0, s>>>(
        reinterpret_cast<const uint4 *>(y), chunks, c / 8, vox, c, reinterpret_cast<const float4 *>(coef), slope,
        reinterpret_cast<uint4 *>(out));
    check_launch("norm_act_kernel");
}

void norm_stats_act(const bf16 *y, int n, long long vox, int c, const double *stats, long long count,
                    const float *gamma, const float *beta, float eps, float slope, float *coef, bf16 *out,
                    cudaStream_t s) {
    need(y && stats && gamma && beta && out, "norm buffers must not be NULL");
    need(c % 8 == 0 && c <= 128, "norm channels must be a multiple of 8, at most 128");
    need(n > 0 && n <= 16 && vox > 0 && count > 0, "norm volume must be positive (at most 16 samples)");
    bind_device();
    const long long chunks = (long long)n * vox * (c / 8);
    norm_stats_act_kernel<<<elementwise_blocks(chunks, 256), 256, (size_t)n * c * sizeof(float4), s>>>(
        reinterpret_cast<const uint4 *>(y), chunks, c / 8, vox, n, c, stats, (double)count, gamma, beta, eps, slope,
        reinterpret_cast<float4 *>(coef), reinterpret_cast<uint4 *>(out));
    check_launch("norm_stats_act_kernel");
}

void norm_act_bwd(const bf16 *y, const bf16 *da, int n, long long vox, int c, const float *coef, const float *gamma,
                  float slope, double *red, bf16 *dy, float *dgamma, float *dbeta, cudaStream_t s) {
    need(y && da && coef && gamma && red && dy && dgamma && dbeta, "norm buffers must not be NULL");
    need(c % 8 == 0 && c <= 128, "norm channels must be a multiple of 8, at most 128");
    need(n > 0 && vox > 0, "norm volume must be positive");
    bind_device();
    DC_CUDA(cudaMemsetAsync(red, 0, sizeof(double) * 2 * n * c, s));
    const int cc = c / 8;
    const long long vpb = 256 / cc;
    const unsigned bx = (unsigned)std::max(1LL, std::min((vox + vpb - 1) / vpb, (long long)sm_count() * 8 / n + 1));
    norm_bwd_reduce_kernel<<<dim3(bx, (unsigned)n), 256, 0, s>>>(
        reinterpret_cast<const uint4 *>(y), reinterpret_cast<const uint4 *>(da), cc, vox, c,
        reinterpret_cast<const float4 *>(coef), slope, red);
    check_launch("norm_bwd_reduce_kernel");
    const long long chunks = (long long)n * vox * cc;
    norm_bwd_apply_kernel<<<elementwise_blocks(chunks, 256), 256, 0, s>>>(
        reinterpret_cast<const uint4 *>(y), reinterpret_cast<const uint4 *>(da), chunks, cc, vox, c,
        reinterpret_cast<const float4 *>(coef), gamma, slope, red, reinterpret_cast<uint4 *>(dy));
    check_launch("norm_bwd_apply_kernel");
    norm_param_grad_kernel<<<(c + 127) / 128, 128, 0, s>>>(red, n, c, dgamma, dbeta);
    check_launch("norm_param_grad_kernel");
}

void pack_input(const float *terma, const float *density, long long vox, float terma_scale, bf16 *x8,
                cudaStream_t s) {
    need(terma && density && x8, "input buffers must not be NULL");
    need(vox > 0, "input volume must be positive");
    bind_device();
    pack_input_kernel<<<elementwise_blocks(vox, 256), 256, 0, s>>>(terma, density, vox, terma_scale,
                                                                    reinterpret_cast<uint4 *>(x8));
    check_launch("pack_input_kernel");
}

void head_fwd(const bf16 *g, long long vox, int c, const float *w, const float *bias, const float *mask,
              float mask_thr, float scale, float *out, cudaStream_t s) {
    need(g && w && bias && mask && out, "head buffers must not be NULL");
    need(c == 16, "the output head takes 16 channels");
    need(vox > 0, "head volume must be positive");
    bind_device();
    head_fwd_kernel<<<elementwise_blocks(vox, 256), 256, 0, s>>>(reinterpret_cast<const uint4 *>(g), vox, w, bias,
                                                                  mask, mask_thr, scale, out);
    check_launch("head_fwd_kernel");
}

void head_loss_bwd(const bf16 *g, long long vox, int c, const float *w, const float *pred, const float *target,
                   float inv_count, const float *inv_count_dev, double *loss, bf16 *dg, float *dw, float *dbias,
                   cudaStream_t s) {
    need(g && w && pred && target && loss && dg && dw && dbias, "head buffers must not be NULL");
    need(c == 16, "the output head takes 16 channels");
    need(vox > 0, "head volume must be positive");
    bind_device();
    DC_CUDA(cudaMemsetAsync(loss, 0, sizeof(double), s));
    DC_CUDA(cudaMemsetAsync(dw, 0, sizeof(float) * 16, s));
    DC_CUDA(cudaMemsetAsync(dbias, 0, sizeof(float), s));
    head_loss_bwd_kernel<<<elementwise_blocks(vox, 256), 256, 0, s>>>(
        reinterpret_cast<const uint4 *>(g), vox, w, pred, target, inv_count, inv_count_dev, loss,
        reinterpret_cast<uint4 *>(dg), dw, dbias);
    check_launch("head_loss_bwd_kernel");
}

}  // namespace net
}  // namespace dc

// ---------------------------------------------------------------------------
// C ABI (include/dosecuda.h, "Surrogate network" section)
// ---------------------------------------------------------------------------
using namespace dc;
using dc::net::bf16;

namespace {
void select_device(int gpu_id) {
    if (gpu_id < 0) throw Error(DC_ERR_CUDA, "invalid device ordinal");
    net::set_call_device(gpu_id);
}
cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }
}  // namespace

extern "C" {

long long dc_net_packed_fragments(int taps, int k_per_tap, int n) {
    if (taps <= 0 || k_per_tap <= 0 || n <= 0 || n % 8) return -1;
    return net::packed_fragments(taps, k_per_tap, n);
}

int dc_net_pack_weights(int gpu_id, const float *master_dev, int taps, int a, int b, int flip, int trans,
                        void *packed_dev, void *stream) {
    return guarded([&] {
        select_device(gpu_id);
        net::pack_weights(master_dev, taps, a, b, flip, trans, static_cast<uint2 *>(packed_dev), as_stream(stream));
    });
}

int dc_net_conv(int gpu_id, int mode, const void *x_dev, int n, int d, int h, int w, int cin, const void *wpk_dev,
                long long wpk_frags, int cout, void *y_dev, double *stats_dev, void *stream) {
    return guarded([&] {
        select_device(gpu_id);
        net::conv_gather(mode, static_cast<const bf16 *>(x_dev), n, d, h, w, cin, static_cast<const uint2 *>(wpk_dev),
                         wpk_frags, cout, static_cast<bf16 *>(y_dev), stats_dev, as_stream(stream));
    });
}

int dc_net_conv_up(int gpu_id, const void *x_dev, int n, int d, int h, int w, int cin, const void *wpk_dev,
                   long long wpk_frags, int cout, const void *addend_dev, void *y_dev, void *stream) {
    return guarded([&] {
        select_device(gpu_id);
        net::conv_up(static_cast<const bf16 *>(x_dev), n, d, h, w, cin, static_cast<const uint2 *>(wpk_dev), wpk_frags,
                     cout,
                     static_cast<const bf16 *>(addend_dev), static_cast<bf16 *>(y_dev), as_stream(stream));
    });
}

int dc_net_wgrad(int gpu_id, int mode, const void *p_dev, const void *q_dev, int n, int d, int h, int w, int ca,
                 int cb, float *grad_dev, void *stream) {
    return guarded([&] {
        select_device(gpu_id);
        net::conv_wgrad(mode, static_cast<const bf16 *>(p_dev), static_cast<const bf16 *>(q_dev), n, d, h, w, ca, cb,
                        grad_dev, as_stream(stream));
    });
}

int dc_net_norm_finalize(int gpu_id, const double *stats_dev, int n, int c, long long count, const float *gamma_dev,
                         const float *beta_dev, float eps, float *coef_dev, void *stream) {
    return guarded([&] {
        select_device(gpu_id);
        net::norm_finalize(stats_dev, n, c, count, gamma_dev, beta_dev, eps, coef_dev, as_stream(stream));
    });
}

int dc_net_norm_act(int gpu_id, const void *y_dev, int n, long long vox, int c, const float *coef_dev, float slope,
                    void *a_dev, void *stream) {
    return guarded([&] {
        select_device(gpu_id);
        net::norm_act(static_cast<const bf16 *>(y_dev), n, vox, c, coef_dev, slope, static_cast<bf16 *>(a_dev),
                      as_stream(stream));
    });
}

int dc_net_norm_stats_act(int gpu_id, const void *y_dev, int n, long long vox, int c, const double *stats_dev,
                          long long count, const float *gamma_dev, const float *beta_dev, float eps, float slope,
                          float *coef_dev, void *a_dev, void *stream) {
    return guarded([&] {
        select_device(gpu_id);
        net::norm_stats_act(static_cast<const bf16 *>(y_dev), n, vox, c, stats_dev, count, gamma_dev, beta_dev, eps,
                            slope, coef_dev, static_cast<bf16 *>(a_dev), as_stream(stream));
    });
}

int dc_net_norm_act_bwd(int gpu_id, const void *y_dev, const void *da_dev, int n, long long vox, int c,
                        const float *coef_dev, const float *gamma_dev, float slope, double *red_dev, void *dy_dev,
                        float *dgamma_dev, float *dbeta_dev, void *stream) {
    return guarded([&] {
        select_device(gpu_id);
        net::norm_act_bwd(static_cast<const bf16 *>(y_dev), static_cast<const bf16 *>(da_dev), n, vox, c, coef_dev,
                          gamma_dev, slope, red_dev, static_cast<bf16 *>(dy_dev), dgamma_dev, dbeta_dev,
                          as_stream(stream));
    });
}

int dc_net_pack_input(int gpu_id, const float *terma_dev, const float *density_dev, long long vox, float terma_scale,
                      void *x8_dev, void *stream) {
    return guarded([&] {
        select_device(gpu_id);
        net::pack_input(terma_dev, density_dev, vox, terma_scale, static_cast<bf16 *>(x8_dev), as_stream(stream));
    });
}

int dc_net_head(int gpu_id, const void *g_dev, long long vox, int c, const float *w_dev, const float *bias_dev,
                const float *mask_dev, float mask_thr, float scale, float *out_dev, void *stream) {
    return guarded([&] {
        select_device(gpu_id);
        net::head_fwd(static_cast<const bf16 *>(g_dev), vox, c, w_dev, bias_dev, mask_dev, mask_thr, scale, out_dev,
                      as_stream(stream));
    });
}

int dc_net_head_loss_bwd(int gpu_id, const void *g_dev, long long vox, int c, const float *w_dev,
                         const float *pred_dev, const float *target_dev, float inv_count,
                         const float *inv_count_dev, double *loss_dev, void *dg_dev, float *dw_dev, float *dbias_dev,
                         void *stream) {
    return guarded([&] {
        select_device(gpu_id);
        net::head_loss_bwd(static_cast<const bf16 *>(g_dev), vox, c, w_dev, pred_dev, target_dev, inv_count,
                           inv_count_dev, loss_dev, static_cast<bf16 *>(dg_dev), dw_dev, dbias_dev,
                           as_stream(stream));
    });
}

}  // extern "C"
