// dc_beam.cu — a proton beam kept resident on the device, for optimisation:
// dose from device-side spot weights, the adjoint (gradient of an objective
// with respect to the spot weights) and the dose-influence matrix in CSR.
//
// The reference offers the same reuse only at the Python level
// (computeIMPTWET / computeIMPTPlanFromWET, plan_impt.py:162-211: the WET is
// kept, every dose call re-uploads everything); there is no adjoint or
// influence matrix in the reference.  All members share the pencil-beam
// kernel family (dc_proton.cu), so dose, gradient and matrix are computed
// from identical per-pair influences:
//   dose(v)      = sum_s mu_s K_s(v)
//   grad_mu(s)   = sum_v g(v) K_s(v)           (D^T g)
//   A[v, s]      = K_s(v)  if K_s(v) >= cutoff * max_v K_s(v)
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/dosecuda.h"
#include "dc_common.cuh"
#include "dc_kernels.cuh"
#include "dc_runtime.cuh"

namespace dc {
const char *last_error_cstr();
}

using namespace dc;

struct dc_proton_beam {
    int device = 0;
    Grid g{};
    Frame f{};
    int n_spots = 0, n_layers = 0, n_energies = 0, lut_len = 0;
    long long n_vox = 0;
    DeviceBuffer tables;  // LayerRec[n_layers] | SpotRec[n_spots]
    DeviceBuffer luts;    // depths | sigmas | idds
    size_t spot_off = 0, lut_stride = 0;
    DeviceBuffer spot_max;  // unsigned[n_spots]
    DeviceBuffer thr;       // float[n_spots]
    DeviceBuffer counts;    // int[n_vox]
    DeviceBuffer block_sums;  // long long[ceil(n_vox / 1024) + 1]

    ~dc_proton_beam() {
        tables.release();
        luts.release();
        spot_max.release();
        thr.release();
        counts.release();
        block_sums.release();
    }

    ProtonTables view() const {
        ProtonTables t;
        t.layers = tables.as<const LayerRec>();
        t.spots = reinterpret_cast<const SpotRec *>(static_cast<const char *>(tables.ptr) + spot_off);
        t.lut_depths = luts.as<const float>();
        t.lut_sigmas = reinterpret_cast<const float *>(static_cast<const char *>(luts.ptr) + lut_stride);
        t.lut_idds = reinterpret_cast<const float *>(static_cast<const char *>(luts.ptr) + 2 * lut_stride);
        t.n_layers = n_layers;
        t.lut_len = lut_len;
        return t;
    }
};

namespace {

void need(bool ok, const std::string &m) {
    if (!ok) throw Error(DC_ERR_VALUE, m);
}

constexpr int kScanBlock = 1024;

// Exclusive scan of int counts into int64 row starts, in blocks of 1024;
// block totals go to sums[block].
__global__ void scan_blocks_kernel(const int *__restrict__ counts, long long n, long long *__restrict__ row_ptr,
                                   long long *__restrict__ sums) {
    __shared__ long long s[kScanBlock];
    const long long base = (long long)blockIdx.x * kScanBlock;
    const int t = threadIdx.x;
    const long long idx = base + t;
    long long v = idx < n ? (long long)counts[idx] : 0;
    s[t] = v;
    __syncthreads();
    for (int o = 1; o < kScanBlock; o <<= 1) {
        long long a = t >= o ? s[t - o] : 0;
        __syncthreads();
        s[t] += a;
        __syncthreads();
    }
    if (idx < n) row_ptr[idx] = s[t] - v;
    if (t == kScanBlock - 1) sums[blockIdx.x] = s[t];
}

// Exclusive scan of the block totals in place (one block, sequential chunks);
// sums[nb] receives the grand total.
__global__ void scan_sums_kernel(long long *__restrict__ sums, int nb) {
    __shared__ long long s[kScanBlock];
    __shared__ long long carry;
    const int t = threadIdx.x;
    if (t == 0) carry = 0;
    __syncthreads();
    for (int c0 = 0; c0 < nb; c0 += kScanBlock) {
        const int idx = c0 + t;
        long long v = idx < nb ? sums[idx] : 0;
        s[t] = v;
        __syncthreads();
        for (int o = 1; o < kScanBlock; o <<= 1) {
            long long a = t >= o ? s[t - o] : 0;
            __syncthreads();
            s[t] += a;
            __syncthreads();
        }
        if (idx < nb) sums[idx] = carry + s[t] - v;
        __syncthreads();
        if (t == kScanBlock - 1) carry += s[t];
        __syncthreads();
    }
    if (t == 0) sums[nb] = carry;
}

__global__ void scan_add_kernel(long long *__restrict__ row_ptr, long long n, const long long *__restrict__ sums,
                                int nb) {
    const long long idx = (long long)blockIdx.x * kScanBlock + threadIdx.x;
    if (idx < n) row_ptr[idx] += sums[blockIdx.x];
    if (idx == 0) row_ptr[n] = sums[nb];
}

__global__ void spot_thr_kernel(const unsigned *__restrict__ spot_max, float cutoff, float *__restrict__ thr, int n) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) thr[s] = cutoff * __uint_as_float(spot_max[s]);
}

}  // namespace

namespace dc {

void launch_scan_counts(const int *counts, long long n, long long *row_ptr, DeviceBuffer &scratch, cudaStream_t s) {
    const int nb = (int)((n + kScanBlock - 1) / kScanBlock);
    long long *sums = static_cast<long long *>(scratch.ensure(((size_t)nb + 1) * sizeof(long long)));
    scan_blocks_kernel<<<nb, kScanBlock, 0, s>>>(counts, n, row_ptr, sums);
    check_launch("scan_blocks_kernel");
    scan_sums_kernel<<<1, kScanBlock, 0, s>>>(sums, nb);
    check_launch("scan_sums_kernel");
    scan_add_kernel<<<nb, kScanBlock, 0, s>>>(row_ptr, n, sums, nb);
    check_launch("scan_add_kernel");
}

void launch_influence_count(DeviceContext &ctx, const Grid &g, const Frame &f, const ProtonTables &t, int n_spots,
                            const float *wet, float cutoff, unsigned *spot_max, float *thr, int *counts,
                            cudaStream_t s) {
    DC_CUDA(cudaMemsetAsync(spot_max, 0, (size_t)n_spots * sizeof(unsigned), s));
    PbExtra x;
    x.spot_max = spot_max;
    launch_pencil_beam_mode(ctx, kPbSpotMax, g, f, t, wet, x, s);
    spot_thr_kernel<<<(n_spots + 255) / 256, 256, 0, s>>>(spot_max, cutoff, thr, n_spots);
    check_launch("spot_thr_kernel");
    PbExtra y;
    y.thr = thr;
    y.counts = counts;
    launch_pencil_beam_mode(ctx, kPbCount, g, f, t, wet, y, s);
}

}  // namespace dc

namespace {

// counts -> row_ptr (n_vox + 1 entries) on stream s
void scan_counts(dc_proton_beam *b, long long *row_ptr, cudaStream_t s) {
    launch_scan_counts(b->counts.as<int>(), b->n_vox, row_ptr, b->block_sums, s);
}

// spot maxima -> thresholds -> per-voxel counts, on stream s
void count_pass(DeviceContext &ctx, dc_proton_beam *b, const float *wet, float cutoff, cudaStream_t s) {
    unsigned *sm = static_cast<unsigned *>(b->spot_max.ensure((size_t)b->n_spots * sizeof(unsigned)));
    float *thr = static_cast<float *>(b->thr.ensure((size_t)b->n_spots * sizeof(float)));
    int *counts = static_cast<int *>(b->counts.ensure((size_t)b->n_vox * sizeof(int)));
    launch_influence_count(ctx, b->g, b->f, b->view(), b->n_spots, wet, cutoff, sm, thr, counts, s);
}

DeviceContext &beam_ctx(dc_proton_beam *b) {
    need(b != nullptr, "beam handle must not be NULL.");
    return context(b->device);
}

}  // namespace

extern "C" {

int dc_proton_beam_create(int gpu_id, int nz, int ny, int nx, const float spacing[3], const float origin[3],
                          const float iso[3], double gantry_deg, float couch_deg, float vsadx, float vsady,
                          const float *divergence_params, int n_energies, int dvp_len, const float *lut_depths,
                          const float *lut_sigmas, const float *lut_idds, int lut_len, const float *spots,
                          int n_spots, dc_proton_beam **out) {
    return guarded([&] {
        need(out != nullptr, "output handle pointer must not be NULL.");
        *out = nullptr;
        need(nz > 0 && ny > 0 && nx > 0, "'voxel_data' must have positive dimensions.");
        need(spacing && origin && iso && spots && divergence_params && lut_depths && lut_sigmas && lut_idds,
             "NULL argument.");
        for (int a = 0; a < 3; ++a) need(std::isfinite(spacing[a]) && spacing[a] > 0.0f, "'spacing' must be positive.");
        need(std::isfinite(vsadx) && std::isfinite(vsady) && vsadx != 0.0f && vsady != 0.0f,
             "'VSADX' and 'VSADY' must be finite and non-zero.");
        need(lut_len >= 1 && lut_len <= 8192, "LUT length must be between 1 and 8192.");
        std::vector<LayerRec> layers;
        std::vector<SpotRec> recs;
        build_proton_tables(spots, n_spots, divergence_params, n_energies, dvp_len, vsadx, vsady, layers, recs);
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        std::unique_ptr<dc_proton_beam> b(new dc_proton_beam());
        b->device = gpu_id;
        b->g = make_grid(nz, ny, nx, spacing);
        b->f = make_frame(iso, origin, gantry_deg, couch_deg, 0.0, (vsadx + vsady) / 2.0f);
        b->n_spots = n_spots;
        b->n_layers = (int)layers.size();
        b->n_energies = n_energies;
        b->lut_len = lut_len;
        b->n_vox = (long long)nz * ny * nx;
        const size_t lb = layers.size() * sizeof(LayerRec);
        b->spot_off = (lb + 255) & ~(size_t)255;
        void *tp = b->tables.ensure(b->spot_off + recs.size() * sizeof(SpotRec));
        DC_CUDA(cudaMemcpy(tp, layers.data(), lb, cudaMemcpyHostToDevice));
        DC_CUDA(cudaMemcpy(static_cast<char *>(tp) + b->spot_off, recs.data(), recs.size() * sizeof(SpotRec),
                           cudaMemcpyHostToDevice));
        const size_t lbytes = (size_t)n_energies * lut_len * sizeof(float);
        b->lut_stride = (lbytes + 255) & ~(size_t)255;
        char *lp = static_cast<char *>(b->luts.ensure(3 * b->lut_stride));
        DC_CUDA(cudaMemcpy(lp, lut_depths, lbytes, cudaMemcpyHostToDevice));
        DC_CUDA(cudaMemcpy(lp + b->lut_stride, lut_sigmas, lbytes, cudaMemcpyHostToDevice));
        DC_CUDA(cudaMemcpy(lp + 2 * b->lut_stride, lut_idds, lbytes, cudaMemcpyHostToDevice));
        launch_layer_rcut(b->g, b->f, static_cast<LayerRec *>(tp), b->n_layers, reinterpret_cast<const float *>(lp),
                          reinterpret_cast<const float *>(lp + b->lut_stride), lut_len, nullptr);
        DC_CUDA(cudaDeviceSynchronize());
        *out = b.release();
    });
}

int dc_proton_beam_destroy(dc_proton_beam *b) {
    return guarded([&] {
        if (!b) return;
        cudaSetDevice(b->device);
        cudaDeviceSynchronize();
        delete b;
    });
}

int dc_proton_beam_info(const dc_proton_beam *b, int *n_spots, int *n_layers, long long *n_voxels) {
    return guarded([&] {
        need(b != nullptr, "beam handle must not be NULL.");
        if (n_spots) *n_spots = b->n_spots;
        if (n_layers) *n_layers = b->n_layers;
        if (n_voxels) *n_voxels = b->n_vox;
    });
}

int dc_proton_beam_dose(dc_proton_beam *b, const float *wet_dev, const float *mu_dev, float *dose_dev, void *stream) {
    return guarded([&] {
        DeviceContext &ctx = beam_ctx(b);
        need(wet_dev && dose_dev, "NULL device buffer.");
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        ctx.begin_call(s);
        launch_pencil_beam(ctx, b->g, b->f, b->view(), wet_dev, dose_dev, s, mu_dev);
        ctx.end_call(s);
    });
}

int dc_proton_beam_adjoint(dc_proton_beam *b, const float *wet_dev, const float *grad_dose_dev, double *grad_mu_dev,
                           void *stream) {
    return guarded([&] {
        DeviceContext &ctx = beam_ctx(b);
        need(wet_dev && grad_dose_dev && grad_mu_dev, "NULL device buffer.");
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        ctx.begin_call(s);
        DC_CUDA(cudaMemsetAsync(grad_mu_dev, 0, (size_t)b->n_spots * sizeof(double), s));
        PbExtra x;
        x.grad_dose = grad_dose_dev;
        x.grad_mu = grad_mu_dev;
        launch_pencil_beam_mode(ctx, kPbAdjoint, b->g, b->f, b->view(), wet_dev, x, s);
        ctx.end_call(s);
    });
}

int dc_proton_beam_dose_list(dc_proton_beam *b, const float *wet_dev, const float *mu_dev, const int *voxels_dev,
                             int n, float *out_dev, void *stream) {
    return guarded([&] {
        DeviceContext &ctx = beam_ctx(b);
        need(wet_dev && voxels_dev && out_dev, "NULL device buffer.");
        need(n >= 0, "'n' must not be negative.");
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        ctx.begin_call(s);
        PbExtra x;
        x.mu = mu_dev;
        x.list = voxels_dev;
        x.n_list = n;
        x.list_out = out_dev;
        launch_pencil_beam_list(ctx, kPbDose, b->g, b->f, b->view(), wet_dev, x, s);
        ctx.end_call(s);
    });
}

int dc_proton_beam_adjoint_list(dc_proton_beam *b, const float *wet_dev, const int *voxels_dev, int n,
                                const float *grad_dev, double *grad_mu_dev, void *stream) {
    return guarded([&] {
        DeviceContext &ctx = beam_ctx(b);
        need(wet_dev && voxels_dev && grad_dev && grad_mu_dev, "NULL device buffer.");
        need(n >= 0, "'n' must not be negative.");
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        ctx.begin_call(s);
        DC_CUDA(cudaMemsetAsync(grad_mu_dev, 0, (size_t)b->n_spots * sizeof(double), s));
        PbExtra x;
        x.grad_dose = grad_dev;
        x.grad_mu = grad_mu_dev;
        x.list = voxels_dev;
        x.n_list = n;
        launch_pencil_beam_list(ctx, kPbAdjoint, b->g, b->f, b->view(), wet_dev, x, s);
        ctx.end_call(s);
    });
}

int dc_proton_beam_influence_nnz(dc_proton_beam *b, const float *wet_dev, float cutoff, long long *nnz,
                                 void *stream) {
    return guarded([&] {
        DeviceContext &ctx = beam_ctx(b);
        need(wet_dev && nnz, "NULL argument.");
        need(std::isfinite(cutoff) && cutoff >= 0.0f && cutoff < 1.0f, "'cutoff' must be in [0, 1).");
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        ctx.begin_call(s);
        count_pass(ctx, b, wet_dev, cutoff, s);
        long long *rp = static_cast<long long *>(ctx.vol_c.ensure(((size_t)b->n_vox + 1) * sizeof(long long)));
        scan_counts(b, rp, s);
        DC_CUDA(cudaMemcpyAsync(nnz, rp + b->n_vox, sizeof(long long), cudaMemcpyDeviceToHost, s));
        ctx.end_call(s);
        DC_CUDA(cudaStreamSynchronize(s));
    });
}

int dc_proton_beam_influence_csr(dc_proton_beam *b, const float *wet_dev, float cutoff, long long *row_ptr_dev,
                                 int *col_dev, float *val_dev, long long capacity, void *stream) {
    return guarded([&] {
        DeviceContext &ctx = beam_ctx(b);
        need(wet_dev && row_ptr_dev && col_dev && val_dev, "NULL device buffer.");
        need(capacity >= 0, "'capacity' must be non-negative.");
        need(std::isfinite(cutoff) && cutoff >= 0.0f && cutoff < 1.0f, "'cutoff' must be in [0, 1).");
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        ctx.begin_call(s);
        count_pass(ctx, b, wet_dev, cutoff, s);
        scan_counts(b, row_ptr_dev, s);
        if (capacity > 0) {
            DC_CUDA(cudaMemsetAsync(col_dev, 0, (size_t)capacity * sizeof(int), s));
            DC_CUDA(cudaMemsetAsync(val_dev, 0, (size_t)capacity * sizeof(float), s));
        }
        PbExtra x;
        x.cap = capacity;
        x.thr = b->thr.as<const float>();
        x.row_ptr = row_ptr_dev;
        x.col = col_dev;
        x.val = val_dev;
        launch_pencil_beam_mode(ctx, kPbFill, b->g, b->f, b->view(), wet_dev, x, s);
        ctx.end_call(s);
    });
}

}  // extern "C"
