// dc_batch.cu — many IMPT plans in one persistent launch.
//
// The reference computes one beam per call, each call uploading its volumes
// and tables and synchronising (plan_impt.py:139-160 -> dosemodule.cu:243-374).
// A batch holds any number of plans (each with its own CT grid, RLSP volume
// and dose volume) and beams (each with its own geometry, spot list and WET
// volume) resident on one device.  Its dose call is a single persistent
// kernel whose CTAs take (plan, tile) work items from a device queue sorted
// by plan cost, so plans with uneven spot and beam counts share the GPU
// without a tail; each item sums its plan's beams layer by layer (energy
// order) in registers and writes each voxel once.  The WET call runs the ray
// march and smoothing of every beam.  Neither call touches host memory, so a
// caller can capture them into a CUDA graph and replay it.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/dosecuda.h"
#include "dc_common.cuh"
#include "dc_kernels.cuh"
#include "dc_runtime.cuh"

using namespace dc;

namespace {

struct HostPlan {
    Grid g;
    float origin[3];
    const float *rlsp;  // device
    float *dose;        // device
    std::vector<int> beams;
    long long cost = 0;
};

struct HostBeam {
    int plan;
    Frame f;
    float *wet;  // device
    std::vector<LayerRec> layers;
    std::vector<SpotRec> spots;
    size_t layer_off = 0, spot_off = 0;  // byte offsets in the table buffer
    int spot_base = 0;                   // offset in the batch's spot-weight vector
};

}  // namespace

struct dc_proton_batch {
    int device = 0;
    float vsadx = 0, vsady = 0;
    int n_energies = 0, dvp_len = 0, lut_len = 0;
    std::vector<float> dvp;
    std::vector<HostPlan> plans;
    std::vector<HostBeam> beams;
    bool committed = false;
    int n_spots_total = 0;
    DeviceBuffer luts;      // depths | sigmas | idds
    size_t lut_stride = 0;
    DeviceBuffer tables;    // per-beam LayerRec[] and SpotRec[]
    DeviceBuffer mu;        // float[n_spots_total]: the spot weights the dose uses
    DeviceBuffer d_plans;   // PbBatchPlan[]
    DeviceBuffer d_beams;   // PbBatchBeam[]
    DeviceBuffer d_items[8];
    int n_items[8] = {0};
    DeviceBuffer queue;     // unsigned queue head
    DeviceBuffer wet_raw;   // unsmoothed WET scratch (largest plan)
    std::vector<std::unique_ptr<VolumeArray>> arrays;  // per-plan RLSP texture
    std::vector<PbBatchBeam> hbeams;  // host copies of d_beams (beams grouped by plan)
    // influence-matrix scratch, one beam at a time: spot maxima, thresholds,
    // per-voxel counts, scan block sums; `inf_beam` is the beam (add order)
    // whose thresholds they hold and `inf_nnz` its entry count
    DeviceBuffer inf_spot_max, inf_thr, inf_counts, inf_sums;
    int inf_beam = -1;
    long long inf_nnz = 0;

    ~dc_proton_batch() {
        luts.release();
        tables.release();
        mu.release();
        d_plans.release();
        d_beams.release();
        for (auto &b : d_items) b.release();
        queue.release();
        wet_raw.release();
        for (auto &a : arrays) a->release();
        inf_spot_max.release();
        inf_thr.release();
        inf_counts.release();
        inf_sums.release();
    }
};

namespace {

void need(bool ok, const std::string &m) {
    if (!ok) throw Error(DC_ERR_VALUE, m);
}

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

// Position of beam `beam_id` (add order) among the committed beams, which
// are grouped by plan.
int committed_index(const dc_proton_batch *b, int beam_id) {
    need(beam_id >= 0 && beam_id < (int)b->beams.size(), "unknown beam id.");
    int seen = 0;
    for (auto &p : b->plans)
        for (int id : p.beams) {
            if (id == beam_id) return seen;
            ++seen;
        }
    throw Error(DC_ERR_VALUE, "unknown beam id.");
}

}  // namespace

extern "C" {

int dc_proton_batch_create(int gpu_id, const float *divergence_params, int n_energies, int dvp_len,
                           const float *lut_depths, const float *lut_sigmas, const float *lut_idds, int lut_len,
                           float vsadx, float vsady, dc_proton_batch **out) {
    return guarded([&] {
        need(out != nullptr, "output handle pointer must not be NULL.");
        *out = nullptr;
        need(divergence_params && lut_depths && lut_sigmas && lut_idds, "beam model tables must not be NULL.");
        need(n_energies > 0 && dvp_len >= 5, "'divergence_params' must hold energy, R80, A, B, C rows.");
        need(lut_len >= 1 && lut_len <= 8192, "LUT length must be between 1 and 8192.");
        need(std::isfinite(vsadx) && std::isfinite(vsady) && vsadx != 0.0f && vsady != 0.0f,
             "'VSADX' and 'VSADY' must be finite and non-zero.");
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        std::unique_ptr<dc_proton_batch> b(new dc_proton_batch());
        b->device = gpu_id;
        b->vsadx = vsadx;
        b->vsady = vsady;
        b->n_energies = n_energies;
        b->dvp_len = dvp_len;
        b->lut_len = lut_len;
        b->dvp.assign(divergence_params, divergence_params + (size_t)n_energies * dvp_len);
        const size_t lbytes = (size_t)n_energies * lut_len * sizeof(float);
        b->lut_stride = align256(lbytes);
        char *lp = static_cast<char *>(b->luts.ensure(3 * b->lut_stride));
        DC_CUDA(cudaMemcpy(lp, lut_depths, lbytes, cudaMemcpyHostToDevice));
        DC_CUDA(cudaMemcpy(lp + b->lut_stride, lut_sigmas, lbytes, cudaMemcpyHostToDevice));
        DC_CUDA(cudaMemcpy(lp + 2 * b->lut_stride, lut_idds, lbytes, cudaMemcpyHostToDevice));
        *out = b.release();
    });
}

int dc_proton_batch_add_plan(dc_proton_batch *b, int nz, int ny, int nx, const float spacing[3],
                             const float origin[3], const float *rlsp_dev, float *dose_dev, int *plan_id) {
    return guarded([&] {
        need(b != nullptr && !b->committed, "batch handle must be valid and not yet committed.");
        need(nz > 0 && ny > 0 && nx > 0, "'voxel_data' must have positive dimensions.");
        need(nx <= 16384 && ny <= 16384 && nz <= 16384, "volume dimensions above 16384 are not supported.");
        need(spacing && origin && rlsp_dev && dose_dev, "NULL argument.");
        for (int a = 0; a < 3; ++a) need(std::isfinite(spacing[a]) && spacing[a] > 0.0f, "'spacing' must be positive.");
        HostPlan p;
        p.g = make_grid(nz, ny, nx, spacing);
        std::memcpy(p.origin, origin, sizeof(p.origin));
        p.rlsp = rlsp_dev;
        p.dose = dose_dev;
        b->plans.push_back(p);
        if (plan_id) *plan_id = (int)b->plans.size() - 1;
    });
}

int dc_proton_batch_add_beam(dc_proton_batch *b, int plan_id, const float iso[3], double gantry_deg,
                             float couch_deg, const float *spots, int n_spots, float *wet_dev, int *beam_id) {
    return guarded([&] {
        need(b != nullptr && !b->committed, "batch handle must be valid and not yet committed.");
        need(plan_id >= 0 && plan_id < (int)b->plans.size(), "unknown plan id.");
        need(iso && spots && wet_dev, "NULL argument.");
        HostBeam hb;
        hb.plan = plan_id;
        hb.f = make_frame(iso, b->plans[plan_id].origin, gantry_deg, couch_deg, 0.0, (b->vsadx + b->vsady) / 2.0f);
        hb.wet = wet_dev;
        build_proton_tables(spots, n_spots, b->dvp.data(), b->n_energies, b->dvp_len, b->vsadx, b->vsady, hb.layers,
                            hb.spots);
        b->plans[plan_id].beams.push_back((int)b->beams.size());
        b->plans[plan_id].cost += (long long)n_spots;
        b->beams.push_back(std::move(hb));
        if (beam_id) *beam_id = (int)b->beams.size() - 1;
    });
}

int dc_proton_batch_commit(dc_proton_batch *b) {
    return guarded([&] {
        need(b != nullptr && !b->committed, "batch handle must be valid and not yet committed.");
        need(!b->plans.empty() && !b->beams.empty(), "a batch needs at least one plan with one beam.");
        DeviceContext &ctx = context(b->device);
        std::lock_guard<std::mutex> lk(ctx.mu);
        // beams grouped by plan (the kernel walks beam0 .. beam0 + n_beams)
        std::vector<int> order;
        for (auto &p : b->plans) order.insert(order.end(), p.beams.begin(), p.beams.end());
        std::vector<HostBeam> sorted;
        sorted.reserve(b->beams.size());
        for (int id : order) sorted.push_back(std::move(b->beams[id]));
        b->beams.swap(sorted);
        // table layout
        size_t off = 0;
        int spot_base = 0;
        for (auto &hb : b->beams) {
            hb.layer_off = off;
            off = align256(off + hb.layers.size() * sizeof(LayerRec));
            hb.spot_off = off;
            off = align256(off + hb.spots.size() * sizeof(SpotRec));
            hb.spot_base = spot_base;
            spot_base += (int)hb.spots.size();
        }
        b->n_spots_total = spot_base;
        char *tab = static_cast<char *>(b->tables.ensure(off));
        std::vector<float> mu0((size_t)spot_base);
        for (auto &hb : b->beams) {
            DC_CUDA(cudaMemcpy(tab + hb.layer_off, hb.layers.data(), hb.layers.size() * sizeof(LayerRec),
                               cudaMemcpyHostToDevice));
            DC_CUDA(cudaMemcpy(tab + hb.spot_off, hb.spots.data(), hb.spots.size() * sizeof(SpotRec),
                               cudaMemcpyHostToDevice));
            // MU in the caller's spot order (records are sorted by energy)
            for (const auto &r : hb.spots) mu0[hb.spot_base + r.orig] = r.mu;
        }
        float *mu = static_cast<float *>(b->mu.ensure((size_t)spot_base * sizeof(float)));
        DC_CUDA(cudaMemcpy(mu, mu0.data(), mu0.size() * sizeof(float), cudaMemcpyHostToDevice));
        const float *lut_d = b->luts.as<const float>();
        const float *lut_s = reinterpret_cast<const float *>(static_cast<const char *>(b->luts.ptr) + b->lut_stride);
        const float *lut_i = reinterpret_cast<const float *>(static_cast<const char *>(b->luts.ptr) + 2 * b->lut_stride);
        std::vector<PbBatchBeam> hbeams;
        int bi = 0;
        for (auto &p : b->plans) {
            for (size_t q = 0; q < p.beams.size(); ++q, ++bi) {
                HostBeam &hb = b->beams[bi];
                launch_layer_rcut(p.g, hb.f, reinterpret_cast<LayerRec *>(tab + hb.layer_off), (int)hb.layers.size(),
                                  lut_d, lut_s, b->lut_len, nullptr);
                PbBatchBeam B;
                B.f = hb.f;
                B.t.layers = reinterpret_cast<const LayerRec *>(tab + hb.layer_off);
                B.t.spots = reinterpret_cast<const SpotRec *>(tab + hb.spot_off);
                B.t.lut_depths = lut_d;
                B.t.lut_sigmas = lut_s;
                B.t.lut_idds = lut_i;
                B.t.n_layers = (int)hb.layers.size();
                B.t.lut_len = b->lut_len;
                B.wet = hb.wet;
                B.mu = mu + hb.spot_base;
                hbeams.push_back(B);
            }
        }
        std::vector<PbBatchPlan> hplans;
        int beam0 = 0;
        long long max_vox = 0;
        for (auto &p : b->plans) {
            PbBatchPlan P;
            P.g = p.g;
            P.dose = p.dose;
            P.beam0 = beam0;
            P.n_beams = (int)p.beams.size();
            beam0 += P.n_beams;
            hplans.push_back(P);
            max_vox = std::max(max_vox, p.g.n());
        }
        void *dp = b->d_plans.ensure(hplans.size() * sizeof(PbBatchPlan));
        DC_CUDA(cudaMemcpy(dp, hplans.data(), hplans.size() * sizeof(PbBatchPlan), cudaMemcpyHostToDevice));
        void *db = b->d_beams.ensure(hbeams.size() * sizeof(PbBatchBeam));
        DC_CUDA(cudaMemcpy(db, hbeams.data(), hbeams.size() * sizeof(PbBatchBeam), cudaMemcpyHostToDevice));
        b->hbeams = hbeams;
        // work queues, one per tile shape: plans by decreasing cost, tiles in order
        std::vector<int> plan_order(b->plans.size());
        std::iota(plan_order.begin(), plan_order.end(), 0);
        std::stable_sort(plan_order.begin(), plan_order.end(),
                         [&](int x, int y) { return b->plans[x].cost > b->plans[y].cost; });
        const int nv = pencil_beam_batch_variants();
        for (int v = 0; v < nv && v < 8; ++v) {
            std::vector<int2> items;
            for (int pi : plan_order) {
                const long long tiles = pencil_beam_batch_tiles(v, b->plans[pi].g);
                need(tiles < 0x7fffffffLL, "plan too large for the batch work queue.");
                for (long long t = 0; t < tiles; ++t) items.push_back(make_int2(pi, (int)t));
            }
            need(items.size() < 0x7fffffffULL, "batch too large for the work queue.");
            void *ip = b->d_items[v].ensure(items.size() * sizeof(int2));
            DC_CUDA(cudaMemcpy(ip, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice));
            b->n_items[v] = (int)items.size();
        }
        b->queue.ensure(sizeof(unsigned));
        b->wet_raw.ensure((size_t)max_vox * sizeof(float));
        for (auto &p : b->plans) {
            std::unique_ptr<VolumeArray> a(new VolumeArray());
            a->ensure(p.g.nx, p.g.ny, p.g.nz, false);
            a->texture(0.0f);
            b->arrays.push_back(std::move(a));
        }
        DC_CUDA(cudaDeviceSynchronize());
        b->committed = true;
    });
}

int dc_proton_batch_info(const dc_proton_batch *b, int *n_plans, int *n_beams, int *n_spots_total,
                         int *n_variants) {
    return guarded([&] {
        need(b != nullptr, "batch handle must not be NULL.");
        if (n_plans) *n_plans = (int)b->plans.size();
        if (n_beams) *n_beams = (int)b->beams.size();
        if (n_spots_total) *n_spots_total = b->n_spots_total;
        if (n_variants) *n_variants = pencil_beam_batch_variants();
    });
}

int dc_proton_batch_beam_spot_offset(const dc_proton_batch *b, int beam_id, int *offset) {
    return guarded([&] {
        need(b != nullptr && b->committed, "batch handle must be committed.");
        need(offset != nullptr, "NULL argument.");
        *offset = b->beams[committed_index(b, beam_id)].spot_base;
    });
}

int dc_proton_batch_wet(dc_proton_batch *b, void *stream) {
    return guarded([&] {
        need(b != nullptr && b->committed, "batch handle must be committed.");
        DeviceContext &ctx = context(b->device);
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        ctx.begin_call(s);
        int bi = 0;
        for (size_t pi = 0; pi < b->plans.size(); ++pi) {
            HostPlan &p = b->plans[pi];
            VolumeArray &a = *b->arrays[pi];
            cudaMemcpy3DParms cp{};
            cp.srcPtr = make_cudaPitchedPtr((void *)p.rlsp, (size_t)p.g.nx * sizeof(float), (size_t)p.g.nx,
                                            (size_t)p.g.ny);
            cp.dstArray = a.arr;
            cp.extent = make_cudaExtent((size_t)p.g.nx, (size_t)p.g.ny, (size_t)p.g.nz);
            cp.kind = cudaMemcpyDeviceToDevice;
            DC_CUDA(cudaMemcpy3DAsync(&cp, s));
            for (size_t q = 0; q < p.beams.size(); ++q, ++bi) {
                HostBeam &hb = b->beams[bi];
                launch_wet_march(ctx, p.g, hb.f, a.texture(0.0f), b->wet_raw.as<float>(), s);
                launch_wet_smooth(ctx, p.g, hb.f, b->wet_raw.as<float>(), hb.wet, s);
            }
        }
        ctx.end_call(s);
    });
}

int dc_proton_batch_dose(dc_proton_batch *b, const float *mu_dev, int variant, void *stream) {
    return guarded([&] {
        need(b != nullptr && b->committed, "batch handle must be committed.");
        need(variant >= 0 && variant < pencil_beam_batch_variants(), "unknown tile variant.");
        DeviceContext &ctx = context(b->device);
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        ctx.begin_call(s);
        if (mu_dev)
            DC_CUDA(cudaMemcpyAsync(b->mu.ptr, mu_dev, (size_t)b->n_spots_total * sizeof(float),
                                    cudaMemcpyDeviceToDevice, s));
        launch_pencil_beam_batch(ctx, variant, b->d_plans.as<const PbBatchPlan>(), b->d_beams.as<const PbBatchBeam>(),
                                 b->d_items[variant].as<const int2>(), b->n_items[variant], b->queue.as<unsigned>(),
                                 b->lut_len, s);
        ctx.end_call(s);
    });
}

int dc_proton_batch_influence_count(dc_proton_batch *b, int beam_id, float cutoff, long long *row_ptr_dev,
                                    long long *nnz, void *stream) {
    return guarded([&] {
        need(b != nullptr && b->committed, "batch handle must be committed.");
        need(row_ptr_dev != nullptr && nnz != nullptr, "NULL argument.");
        need(std::isfinite(cutoff) && cutoff >= 0.0f && cutoff < 1.0f, "'cutoff' must be in [0, 1).");
        const int bi = committed_index(b, beam_id);
        DeviceContext &ctx = context(b->device);
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        const HostBeam &hb = b->beams[bi];
        const Grid &g = b->plans[hb.plan].g;
        const int n_spots = (int)hb.spots.size();
        b->inf_beam = -1;
        ctx.begin_call(s);
        unsigned *sm = static_cast<unsigned *>(b->inf_spot_max.ensure((size_t)std::max(n_spots, 1) * sizeof(unsigned)));
        float *thr = static_cast<float *>(b->inf_thr.ensure((size_t)std::max(n_spots, 1) * sizeof(float)));
        int *counts = static_cast<int *>(b->inf_counts.ensure((size_t)g.n() * sizeof(int)));
        launch_influence_count(ctx, g, hb.f, b->hbeams[bi].t, n_spots, hb.wet, cutoff, sm, thr, counts, s);
        launch_scan_counts(counts, g.n(), row_ptr_dev, b->inf_sums, s);
        DC_CUDA(cudaMemcpyAsync(nnz, row_ptr_dev + g.n(), sizeof(long long), cudaMemcpyDeviceToHost, s));
        ctx.end_call(s);
        DC_CUDA(cudaStreamSynchronize(s));
        b->inf_beam = beam_id;
        b->inf_nnz = *nnz;
    });
}

int dc_proton_batch_influence_fill(dc_proton_batch *b, int beam_id, const long long *row_ptr_dev, int *col_dev,
                                   float *val_dev, long long capacity, void *stream) {
    return guarded([&] {
        need(b != nullptr && b->committed, "batch handle must be committed.");
        need(row_ptr_dev != nullptr && col_dev != nullptr && val_dev != nullptr, "NULL device buffer.");
        const int bi = committed_index(b, beam_id);
        need(b->inf_beam == beam_id, "dc_proton_batch_influence_count must run for this beam first.");
        need(capacity >= b->inf_nnz, "'capacity' is below the beam's entry count.");
        DeviceContext &ctx = context(b->device);
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
        const HostBeam &hb = b->beams[bi];
        ctx.begin_call(s);
        PbExtra x;
        x.cap = capacity;
        x.thr = b->inf_thr.as<const float>();
        x.row_ptr = row_ptr_dev;
        x.col = col_dev;
        x.val = val_dev;
        launch_pencil_beam_mode(ctx, kPbFill, b->plans[hb.plan].g, hb.f, b->hbeams[bi].t, hb.wet, x, s);
        ctx.end_call(s);
    });
}

int dc_proton_batch_destroy(dc_proton_batch *b) {
    return guarded([&] {
        if (!b) return;
        cudaSetDevice(b->device);
        cudaDeviceSynchronize();
        delete b;
    });
}

}  // extern "C"
