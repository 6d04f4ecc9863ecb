// dc_net_tc.cu — the surrogate network's full-resolution 3x3x3 convolutions
// on the 5th-generation tensor cores (tcgen05.mma, accumulators in TMEM).
//
// Implicit GEMM over one output x-line per M=128 tile (the grid's x extent is
// 128): D[x][co] = sum_{tap, ci} A_tap[x][ci] * B_tap[ci][co].
//
// Shared-memory operands use the no-swizzle K-major canonical layout: a core
// matrix is 8 rows x 16 bytes stored contiguously, 8-row groups SBO = 128 B
// apart, the second 8-element K half LBO bytes away.
//  * A (activations): the CTA's input halo is stored as channel-chunk planes
//    plane[cc][line][LP] of 16-byte records (8 channels of one voxel), record
//    r of a line holding x = r - 1.  The 128 rows of tap (dz, dy, dx) are 128
//    consecutive records starting at x = dx - 1 of halo line (dz, dy), so a
//    tap is only a descriptor start address; LBO is the plane stride (the
//    next 8 channels).  With 8 input channels (one plane) two x-neighbouring
//    taps share one K=16 instruction: LBO = one record.
//  * B (weights): [step][k half][co][8] records, prepacked on the device.
// One thread issues all MMAs of the CTA (4 tiles x 27 or 18 steps), commits
// them to an mbarrier, and every warp reads its 32 TMEM lanes back
// (tcgen05.ld 32x32b.x16) for the bf16 store and the instance-norm sums.
// The wait on the mbarrier is bounded: on expiry the kernel records an error
// (dc_net_tc_error) and skips the epilogue instead of hanging.  It then frees
// its tensor memory although MMAs it issued may still be writing there, so a
// recorded expiry outside the self-test (which issues none) leaves the
// device's later results untrustworthy: callers treat it as a device error.
//
// Measured on B200: one tcgen05.mma of M=128, K=16 costs ~26 ns whatever N
// up to 64, so with 16 output channels the tensor cores top out near
// 370 TFLOP/s, below the legacy mma.sync ceiling (~540 TFLOP/s); they win
// at 64-128 channels (1.35-2.05 PFLOP/s).  The network therefore runs this
// kernel for its 8 -> 16 input layer (1.8x faster than the mma.sync kernel,
// which pads the 8-channel taps into k16 steps) and mma.sync elsewhere.
#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <utility>

#include <cuda_bf16.h>

#include "../../include/dosecuda.h"
#include "dc_net.cuh"
#include "dc_runtime.cuh"

namespace dc {
namespace net {
void need(bool ok, const std::string &msg);
namespace {

constexpr int kTcThreads = 128;
constexpr int kTcW = 128;           // grid x extent (= MMA M)
constexpr int kTcTY = 2, kTcTZ = 2; // output lines per CTA
constexpr int kTcTiles = kTcTY * kTcTZ;
constexpr int kTcLines = (kTcTY + 2) * (kTcTZ + 2);
constexpr int kTcLP = 136;          // records per halo line (130 used, the rest zero)
constexpr long long kTcSpinLimit = 1LL << 22;

__device__ int g_tc_error = 0;  // set when an mbarrier wait expired

__device__ __forceinline__ unsigned su32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void cp16(unsigned dst, const void *src, bool valid) {
    const int n = valid ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(n));
}

// no-swizzle K-major shared-memory matrix descriptor (sm_100 format: version 1)
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr, unsigned lbo, unsigned sbo) {
    unsigned long long d = 0;
    d |= (unsigned long long)((addr >> 4) & 0x3FFFu);
    d |= (unsigned long long)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (unsigned long long)((sbo >> 4) & 0x3FFFu) << 32;
    d |= 1ull << 46;  // descriptor version
    return d;         // base offset 0, lbo mode 0, layout type 0 (no swizzle)
}

// kind::f16 instruction descriptor: bf16 A and B (K-major), fp32 D, M=128.
template <int N>
__device__ __forceinline__ unsigned instr_desc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(N >> 3) << 17) | ((unsigned)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16_ss(unsigned tmem_d, unsigned long long a, unsigned long long b,
                                            unsigned idesc, unsigned accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

template <int CC, int N>
struct TcShape {
    static constexpr bool kPair = CC == 1;                       // 8 input channels: taps paired
    static constexpr int kSteps = kPair ? 18 : 27 * (CC / 2);   // K=16 instructions per tile
    static constexpr int kPlaneBytes = kTcLines * kTcLP * 16;
    static constexpr int kABytes = CC * kPlaneBytes;
    static constexpr int kBBytes = kSteps * 2 * N * 16;
    static constexpr int kSmem = kABytes + kBBytes + 64;        // + mbarrier, TMEM address
    static constexpr int kTmemCols = kTcTiles * N < 32 ? 32 : kTcTiles * N;
    static_assert((kTcTiles * N & (kTcTiles * N - 1)) == 0, "TMEM allocation is a power of two");
};

struct TcArgs {
    const bf16 *x;
    const uint4 *w;  // tc-packed weights, TcShape::kBBytes
    bf16 *y;
    double *stats;
    int d, h;  // grid (x extent is kTcW)
    int tiles_y, tiles_z, n_tiles;
    long long spin_limit;  // bound of the mbarrier wait
    int no_mma;            // self-test: issue nothing, so the wait must expire
};

// Bounded wait for phase `parity` of an mbarrier; false when it expired.
__device__ __forceinline__ bool wait_mbar(unsigned addr, unsigned parity, long long limit = kTcSpinLimit) {
    for (long long it = 0; it < limit; ++it) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        if (it > 64) __nanosleep(64);
    }
    return false;
}

// One CTA per tile of kTcTY x kTcTZ output x-lines: stage the halo and the
// weights, one thread issues the tile's MMAs (step-major, so the four
// accumulators are independent chains) and commits them to the mbarrier,
// every warp drains its 32 TMEM lanes.  Several CTAs per SM overlap one
// another's loads, MMAs and epilogues.
template <int CC, int N>
__global__ void __launch_bounds__(kTcThreads) conv3_tc_kernel(TcArgs a) {
    using S = TcShape<CC, N>;
    extern __shared__ __align__(128) unsigned char smem[];
    unsigned char *sa = smem;
    unsigned char *sb = smem + S::kABytes;
    unsigned long long *mbar = reinterpret_cast<unsigned long long *>(smem + S::kABytes + S::kBBytes);
    unsigned *tmem_slot = reinterpret_cast<unsigned *>(smem + S::kABytes + S::kBBytes + 16);
    __shared__ float s_stat[2 * N];

    int b = blockIdx.x;
    const int ty = b % a.tiles_y;
    b /= a.tiles_y;
    const int tz = b % a.tiles_z;
    const int nb = b / a.tiles_z;
    const int y0 = ty * kTcTY, z0 = tz * kTcTZ;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    {
        const bf16 *xs = a.x + (size_t)nb * a.d * a.h * kTcW * (CC * 8);
        constexpr int RECS = CC * kTcLines * kTcLP;
        for (int q = tid; q < RECS; q += kTcThreads) {
            const int r = q % kTcLP;
            const int line = (q / kTcLP) % kTcLines;
            const int cc = q / (kTcLP * kTcLines);
            const int gy = y0 - 1 + line % (kTcTY + 2);
            const int gz = z0 - 1 + line / (kTcTY + 2);
            const int gx = r - 1;
            const bool ok = gx >= 0 && gx < kTcW && gy >= 0 && gy < a.h && gz >= 0 && gz < a.d;
            const bf16 *src = ok ? xs + ((((size_t)gz * a.h + gy) * kTcW + gx) * CC + cc) * 8 : a.x;
            cp16(su32(sa + (size_t)q * 16), src, ok);
        }
        for (int q = tid; q < S::kBBytes / 16; q += kTcThreads) cp16(su32(sb + (size_t)q * 16), a.w + q, true);
    }
    if (a.stats)
        for (int q = tid; q < 2 * N; q += kTcThreads) s_stat[q] = 0.f;
    if (tid == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(su32(mbar)));
    if (warp == 0) {  // TMEM for the tiles' fp32 accumulators
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(su32(tmem_slot)),
                     "r"((unsigned)S::kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // generic writes -> tensor-core reads
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const unsigned tmem = *tmem_slot;

    if (tid == 0 && !a.no_mma) {
        const unsigned idesc = instr_desc<N>();
        const unsigned long long adesc0 = smem_desc(su32(sa), S::kPair ? 16u : (unsigned)S::kPlaneBytes, 128);
        const unsigned long long bdesc0 = smem_desc(su32(sb), N * 16, 128);
        for (int st = 0; st < S::kSteps; ++st)
            for (int m = 0; m < kTcTiles; ++m) {
                const int ry = m % kTcTY, rz = m / kTcTY;
                int line, rec, plane;
                if constexpr (S::kPair) {  // (dz, dy) x half: records x+2h and x+2h+1 of the one plane
                    const int dzdy = st >> 1, hh = st & 1;
                    line = (rz + dzdy / 3) * (kTcTY + 2) + (ry + dzdy % 3);
                    rec = 2 * hh;
                    plane = 0;
                } else {  // tap t, channel chunks 2s and 2s+1
                    const int t = st / (CC / 2), s2 = st % (CC / 2);
                    line = (rz + t / 9) * (kTcTY + 2) + (ry + (t / 3) % 3);
                    rec = t % 3;
                    plane = 2 * s2;
                }
                const unsigned off = (unsigned)((plane * S::kPlaneBytes + (line * kTcLP + rec) * 16) >> 4);
                mma_bf16_ss(tmem + m * N, adesc0 + off, bdesc0 + (unsigned long long)(st * (2 * N * 16) >> 4),
                            idesc, st > 0 ? 1u : 0u);
            }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         su32(mbar))
                     : "memory");
    }

    // bounded wait; every thread votes, so the epilogue decision is uniform
    const bool done = __syncthreads_and(wait_mbar(su32(mbar), 0, a.spin_limit) ? 1 : 0) != 0;
    if (!done && tid == 0) atomicExch(&g_tc_error, 1);
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");

    if (done) {
        float ssum[N], ssq[N];
#pragma unroll
        for (int c = 0; c < N; ++c) ssum[c] = ssq[c] = 0.f;
        const int x = warp * 32 + lane;  // the TMEM lane (row) this thread reads
#pragma unroll 1
        for (int m = 0; m < kTcTiles; ++m) {
            unsigned r[N];
#pragma unroll
            for (int c0 = 0; c0 < N; c0 += 16) {
                const unsigned addr = tmem + ((unsigned)(warp * 32) << 16) + m * N + c0;
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];\n"
                    : "=r"(r[c0 + 0]), "=r"(r[c0 + 1]), "=r"(r[c0 + 2]), "=r"(r[c0 + 3]), "=r"(r[c0 + 4]),
                      "=r"(r[c0 + 5]), "=r"(r[c0 + 6]), "=r"(r[c0 + 7]), "=r"(r[c0 + 8]), "=r"(r[c0 + 9]),
                      "=r"(r[c0 + 10]), "=r"(r[c0 + 11]), "=r"(r[c0 + 12]), "=r"(r[c0 + 13]), "=r"(r[c0 + 14]),
                      "=r"(r[c0 + 15])
                    : "r"(addr));
            }
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
            const int gy = y0 + m % kTcTY, gz = z0 + m / kTcTY;
            unsigned pk[N / 2];
#pragma unroll
            for (int c = 0; c < N; c += 2) {
                const __nv_bfloat162 o = __floats2bfloat162_rn(__uint_as_float(r[c]), __uint_as_float(r[c + 1]));
                pk[c / 2] = *reinterpret_cast<const unsigned *>(&o);
                const float f0 = __low2float(o), f1 = __high2float(o);
                ssum[c] += f0;
                ssum[c + 1] += f1;
                ssq[c] += f0 * f0;
                ssq[c + 1] += f1 * f1;
            }
            uint4 *dst = reinterpret_cast<uint4 *>(a.y + ((((size_t)nb * a.d + gz) * a.h + gy) * kTcW + x) * N);
#pragma unroll
            for (int c = 0; c < N / 8; ++c) dst[c] = make_uint4(pk[4 * c], pk[4 * c + 1], pk[4 * c + 2], pk[4 * c + 3]);
        }
        if (a.stats) {
#pragma unroll
            for (int c = 0; c < N; ++c) {
                float u = ssum[c], v = ssq[c];
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    u += __shfl_xor_sync(0xffffffffu, u, off);
                    v += __shfl_xor_sync(0xffffffffu, v, off);
                }
                if (lane == 0) {
                    atomicAdd(&s_stat[c], u);
                    atomicAdd(&s_stat[N + c], v);
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                     "r"((unsigned)S::kTmemCols));
    }
    if (done && a.stats)
        for (int q = tid; q < N; q += kTcThreads) {
            atomicAdd(&a.stats[((size_t)nb * N + q) * 2 + 0], (double)s_stat[q]);
            atomicAdd(&a.stats[((size_t)nb * N + q) * 2 + 1], (double)s_stat[N + q]);
        }
}

// tc weight packing: out[step][half][co][8 k] bf16 from master m[T][A][B]
// (flip/trans as in pack_weights).  Non-paired: step = tap*CC/2 + s, k =
// (2s + half)*8 + e.  Paired (8 input channels): step = (dz*3+dy)*2 + h, the
// half selects tap dx = 2h + half (zero for dx = 3).
__global__ void pack_weights_tc_kernel(const float *__restrict__ m, int T, int A, int B, int flip, int trans,
                                       int CC, int N, int steps, __nv_bfloat16 *__restrict__ out) {
    const int total = steps * 2 * N * 8;
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int e = idx % 8;
    const int n = (idx / 8) % N;
    const int half = (idx / (8 * N)) % 2;
    const int st = idx / (16 * N);
    const int Kc = trans ? B : A;
    int t, k;
    bool zero = false;
    if (CC == 1) {
        const int dzdy = st >> 1, hh = st & 1;
        const int dx = 2 * hh + half;
        zero = dx > 2;
        t = dzdy * 3 + (zero ? 0 : dx);
        k = e;
    } else {
        t = st / (CC / 2);
        k = (2 * (st % (CC / 2)) + half) * 8 + e;
    }
    float v = 0.f;
    if (!zero && k < Kc) {
        const int tt = flip ? T - 1 - t : t;
        v = trans ? m[((size_t)tt * A + n) * B + k] : m[((size_t)tt * A + k) * B + n];
    }
    out[idx] = __float2bfloat16_rn(v);
}

template <class K>
void set_smem_tc(K kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> done;
    int dev = 0;
    DC_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_pair(reinterpret_cast<const void *>(kernel), dev);
    std::lock_guard<std::mutex> lk(mu);
    auto it = done.find(key);
    if (it != done.end() && it->second >= bytes) return;
    DC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    done[key] = bytes;
}

template <int CC, int N>
void launch_tc(const TcArgs &a0, int n, cudaStream_t s) {
    using S = TcShape<CC, N>;
    TcArgs a = a0;
    a.tiles_y = a.h / kTcTY;
    a.tiles_z = a.d / kTcTZ;
    const long long tiles = (long long)n * a.tiles_y * a.tiles_z;
    need(tiles < 0x7fffffffLL, "volume too large for the surrogate convolution");
    a.n_tiles = (int)tiles;
    auto k = conv3_tc_kernel<CC, N>;
    set_smem_tc(k, S::kSmem);
    k<<<(unsigned)tiles, kTcThreads, S::kSmem, s>>>(a);
    check_launch("conv3_tc_kernel");
}

}  // namespace

void need(bool ok, const std::string &msg) {
    if (!ok) throw Error(DC_ERR_VALUE, msg);
}

long long packed_tc_bytes(int cin, int cout) {
    if (cout != 16) return -1;
    if (cin == 8) return (long long)TcShape<1, 16>::kBBytes;
    if (cin == 16) return (long long)TcShape<2, 16>::kBBytes;
    return -1;
}

void pack_weights_tc(const float *master, int taps, int a, int b, int flip, int trans, void *out, cudaStream_t s) {
    need(master && out, "weights must not be NULL");
    need(taps == 27, "tensor-core packing is for 3x3x3 weights");
    const int cin = trans ? b : a, cout = trans ? a : b;
    need(packed_tc_bytes(cin, cout) > 0, "tensor-core packing supports 8->16 and 16->16 channels");
    const int CC = cin / 8;
    const int steps = CC == 1 ? 18 : 27 * (CC / 2);
    const int total = steps * 2 * cout * 8;
    pack_weights_tc_kernel<<<(total + 255) / 256, 256, 0, s>>>(master, taps, a, b, flip, trans, CC, cout, steps,
                                                                static_cast<__nv_bfloat16 *>(out));
    check_launch("pack_weights_tc_kernel");
}

bool conv_tc_supported(int d, int h, int w, int cin, int cout) {
    return w == kTcW && d % kTcTZ == 0 && h % kTcTY == 0 && cout == 16 && (cin == 8 || cin == 16);
}

void conv_tc(const bf16 *x, int n, int d, int h, int w, int cin, const void *wtc, long long wtc_bytes, int cout,
             bf16 *y, double *stats, cudaStream_t s) {
    need(x && wtc && y, "convolution buffers must not be NULL");
    need(n > 0 && d > 0 && h > 0 && w > 0, "convolution grid must be positive");
    need(conv_tc_supported(d, h, w, cin, cout),
         "the tensor-core convolution takes x extent 128, even y and z extents, and 8->16 or 16->16 channels");
    need(wtc_bytes == packed_tc_bytes(cin, cout), "packed weights do not match the convolution's shape");
    if (stats) DC_CUDA(cudaMemsetAsync(stats, 0, sizeof(double) * 2 * n * cout, s));
    TcArgs a{};
    a.spin_limit = kTcSpinLimit;
    a.x = x;
    a.w = static_cast<const uint4 *>(wtc);
    a.y = y;
    a.stats = stats;
    a.d = d;
    a.h = h;
    if (cin == 8) return launch_tc<1, 16>(a, n, s);
    return launch_tc<2, 16>(a, n, s);
}

int take_tc_error();

// Launches one tile with its MMAs withheld and a short wait bound: nothing
// ever arrives on the CTA's mbarrier, so the bounded wait must expire, set the
// error flag and skip the epilogue.  Returns the flag (and clears it).
int tc_wait_selftest(cudaStream_t s) {
    using S = TcShape<2, 16>;
    const int d = kTcTZ, h = kTcTY;
    const size_t xbytes = (size_t)d * h * kTcW * 16 * sizeof(bf16);
    const size_t ybytes = xbytes;
    struct Owned {  // frees its allocations on every exit path
        void *p[3] = {nullptr, nullptr, nullptr};
        ~Owned() {
            for (void *q : p) cudaFree(q);
        }
    } mem;
    DC_CUDA(cudaMalloc(&mem.p[0], xbytes));
    DC_CUDA(cudaMalloc(&mem.p[1], ybytes));
    DC_CUDA(cudaMalloc(&mem.p[2], S::kBBytes));
    void *x = mem.p[0], *y = mem.p[1], *w = mem.p[2];
    DC_CUDA(cudaMemsetAsync(x, 0, xbytes, s));
    DC_CUDA(cudaMemsetAsync(w, 0, S::kBBytes, s));
    TcArgs a{};
    a.x = static_cast<const bf16 *>(x);
    a.w = static_cast<const uint4 *>(w);
    a.y = static_cast<bf16 *>(y);
    a.d = d;
    a.h = h;
    a.spin_limit = 256;
    a.no_mma = 1;
    launch_tc<2, 16>(a, 1, s);
    DC_CUDA(cudaStreamSynchronize(s));
    return take_tc_error();
}

int take_tc_error() {
    int v = 0, zero = 0;
    DC_CUDA(cudaMemcpyFromSymbol(&v, g_tc_error, sizeof(int)));
    DC_CUDA(cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int)));
    return v;
}

}  // namespace net
}  // namespace dc

// ---------------------------------------------------------------------------
// C ABI (include/dosecuda.h, "Surrogate network" section)
// ---------------------------------------------------------------------------
namespace {
void use_device(int gpu_id) {
    int n = 0;
    DC_CUDA(cudaGetDeviceCount(&n));
    if (gpu_id < 0 || gpu_id >= n) throw dc::Error(DC_ERR_CUDA, "invalid device ordinal");
    DC_CUDA(cudaSetDevice(gpu_id));
}
}  // namespace

extern "C" {

long long dc_net_packed_tc_bytes(int cin, int cout) { return dc::net::packed_tc_bytes(cin, cout); }

int dc_net_pack_weights_tc(int gpu_id, const float *master_dev, int taps, int a, int b, int flip, int trans,
                           void *packed_dev, void *stream) {
    return dc::guarded([&] {
        dc::net::need(master_dev && packed_dev, "weights must not be NULL");
        dc::net::need(taps == 27 && a > 0 && b > 0, "tensor-core packing is for 3x3x3 weights");
        const int cin = trans ? b : a, cout = trans ? a : b;
        dc::net::need(dc::net::packed_tc_bytes(cin, cout) > 0,
                      "tensor-core packing supports 8->16 and 16->16 channels");
        use_device(gpu_id);
        dc::net::pack_weights_tc(master_dev, taps, a, b, flip, trans, packed_dev,
                                 reinterpret_cast<cudaStream_t>(stream));
    });
}

int dc_net_conv_tc(int gpu_id, const void *x_dev, int n, int d, int h, int w, int cin, const void *wtc_dev,
                   long long wtc_bytes, int cout, void *y_dev, double *stats_dev, void *stream) {
    return dc::guarded([&] {
        dc::net::need(x_dev && wtc_dev && y_dev, "convolution buffers must not be NULL");
        dc::net::need(n > 0 && d > 0 && h > 0 && w > 0, "convolution grid must be positive");
        dc::net::need(dc::net::conv_tc_supported(d, h, w, cin, cout),
                      "the tensor-core convolution takes x extent 128, even y and z extents, and 8->16 or 16->16 "
                      "channels");
        dc::net::need(wtc_bytes == dc::net::packed_tc_bytes(cin, cout),
                      "packed weights do not match the convolution's shape");
        use_device(gpu_id);
        dc::net::conv_tc(static_cast<const dc::net::bf16 *>(x_dev), n, d, h, w, cin, wtc_dev, wtc_bytes, cout,
                         static_cast<dc::net::bf16 *>(y_dev), stats_dev, reinterpret_cast<cudaStream_t>(stream));
    });
}

int dc_net_tc_selftest(int gpu_id, int *wait_expired) {
    return dc::guarded([&] {
        dc::net::need(wait_expired != nullptr, "'wait_expired' must not be NULL");
        use_device(gpu_id);
        dc::net::take_tc_error();  // start from a clear flag
        *wait_expired = dc::net::tc_wait_selftest(nullptr);
    });
}

int dc_net_tc_error(int gpu_id, int *flag) {
    return dc::guarded([&] {
        dc::net::need(flag != nullptr, "'flag' must not be NULL");
        use_device(gpu_id);
        *flag = dc::net::take_tc_error();
    });
}

}  // extern "C"
