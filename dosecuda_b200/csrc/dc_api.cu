// dc_api.cu — extern "C" entry points (include/dosecuda.h).
//
// Host entry points mirror the reference's synchronous per-call flow
// (IMPTClasses.cu:274-340, IMRTClasses.cu:353-405): upload, run, download.
// They differ in what persists: device buffers, cudaArrays and texture
// objects live in the per-device context and are reused across calls.
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
const char *last_error_cstr();
}

using namespace dc;

namespace {

void need(bool ok, const std::string &msg) {
    if (!ok) throw Error(DC_ERR_VALUE, msg);
}

void check_volume(const void *p, int nz, int ny, int nx, const float spacing[3], const float origin[3],
                  const char *name) {
    need(p != nullptr, std::string("'") + name + "' must not be NULL.");
    need(nz > 0 && ny > 0 && nx > 0, std::string("'") + name + "' must have positive dimensions.");
    need(spacing && origin, "'spacing' and 'origin' must be given.");
    for (int a = 0; a < 3; ++a) {
        need(std::isfinite(spacing[a]) && spacing[a] > 0.0f, "'spacing' must be positive and finite.");
        need(std::isfinite(origin[a]), "'origin' must be finite.");
    }
    // 3D cudaArray extent limits for linear-filtered textures.
    need(nx <= 16384 && ny <= 16384 && nz <= 16384, "volume dimensions above 16384 are not supported.");
}

cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

void copy_host_to_array(VolumeArray &a, const float *src, int nz, int ny, int nx, cudaMemcpyKind kind,
                        cudaStream_t s) {
    cudaMemcpy3DParms p{};
    p.srcPtr = make_cudaPitchedPtr((void *)src, (size_t)nx * sizeof(float), (size_t)nx, (size_t)ny);
    p.dstArray = a.arr;
    p.extent = make_cudaExtent((size_t)nx, (size_t)ny, (size_t)nz);
    p.kind = kind;
    DC_CUDA(cudaMemcpy3DAsync(&p, s));
}

// WET march + smoothing with the RLSP volume already in ctx.density.
void proton_raytrace_core(DeviceContext &ctx, const Grid &g, const Frame &f, float *wet_s_dev, cudaStream_t s) {
    float *wet = static_cast<float *>(ctx.wet_raw.ensure((size_t)g.n() * sizeof(float)));
    // RLSP texture with border 0 (IMPTClasses.cu:292).
    launch_wet_march(ctx, g, f, ctx.density.texture(0.0f), wet, s);
    launch_wet_smooth(ctx, g, f, wet, wet_s_dev, s);
}

// Uploads the spot/layer tables (via pinned staging) and launches the pencil beam.
// Layer and spot tables on the device (through a pinned staging slot) and
// the layers' cut-off radii, enqueued on s.
ProtonTables proton_tables(DeviceContext &ctx, const Grid &g, const Frame &f, const std::vector<LayerRec> &layers,
                           const std::vector<SpotRec> &spots, const float *lut_d, const float *lut_s,
                           const float *lut_i, int lut_len, cudaStream_t s) {
    const size_t lb = layers.size() * sizeof(LayerRec);
    const size_t lb_al = (lb + 255) & ~(size_t)255;
    const size_t sb = spots.size() * sizeof(SpotRec);
    const int slot = ctx.pin_next;
    ctx.pin_next = (ctx.pin_next + 1) % DeviceContext::kPinSlots;
    // The copy that last used this staging slot must be done before it is rewritten.
    DC_CUDA(cudaEventSynchronize(ctx.pin_ev[slot]));
    char *pin = static_cast<char *>(ctx.pin_ring[slot].ensure(lb_al + sb));
    std::memcpy(pin, layers.data(), lb);
    std::memcpy(pin + lb_al, spots.data(), sb);
    char *dev = static_cast<char *>(ctx.tables.ensure(lb_al + sb));
    DC_CUDA(cudaMemcpyAsync(dev, pin, lb_al + sb, cudaMemcpyHostToDevice, s));
    DC_CUDA(cudaEventRecord(ctx.pin_ev[slot], s));
    launch_layer_rcut(g, f, reinterpret_cast<LayerRec *>(dev), (int)layers.size(), lut_d, lut_s, lut_len, s);
    ProtonTables t;
    t.layers = reinterpret_cast<const LayerRec *>(dev);
    t.spots = reinterpret_cast<const SpotRec *>(dev + lb_al);
    t.lut_depths = lut_d;
    t.lut_sigmas = lut_s;
    t.lut_idds = lut_i;
    t.n_layers = (int)layers.size();
    t.lut_len = lut_len;
    return t;
}

void proton_spot_core(DeviceContext &ctx, const Grid &g, const Frame &f, const std::vector<LayerRec> &layers,
                      const std::vector<SpotRec> &spots, const float *lut_d, const float *lut_s, const float *lut_i,
                      int lut_len, const float *wet_s_dev, float *dose_dev, cudaStream_t s) {
    const ProtonTables t = proton_tables(ctx, g, f, layers, spots, lut_d, lut_s, lut_i, lut_len, s);
    launch_pencil_beam(ctx, g, f, t, wet_s_dev, dose_dev, s);
}

void check_proton_model(float vsadx, float vsady) {
    need(std::isfinite(vsadx) && std::isfinite(vsady) && vsadx != 0.0f && vsady != 0.0f,
         "'VSADX' and 'VSADY' must be finite and non-zero.");
}

void check_luts(const void *dvp, int n_energies, int dvp_len, const void *d, const void *s, const void *i,
                int lut_len) {
    need(dvp != nullptr && d != nullptr && s != nullptr && i != nullptr, "beam model tables must not be NULL.");
    need(n_energies > 0, "'lut_depths' must hold at least one energy.");
    need(dvp_len >= 5, "'divergence_params' rows must hold energy, R80, A, B, C.");
    need(lut_len >= 1 && lut_len <= 8192, "LUT length must be between 1 and 8192.");
}

}  // namespace

extern "C" {

const char *dc_last_error(void) { return dc::last_error_cstr(); }

int dc_debug_bounds(int gpu_id, unsigned long long *violation, int *enabled) {
    return guarded([&] {
        need(violation != nullptr && enabled != nullptr, "output pointers must not be NULL.");
#ifdef DC_DEBUG_BOUNDS
        *enabled = 1;
#else
        *enabled = 0;
#endif
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        DC_CUDA(cudaDeviceSynchronize());
        unsigned long long v = 0;
        for (unsigned long long w : {take_bounds_wet(), take_bounds_photon(), take_bounds_proton(),
                                     take_bounds_basis(), take_bounds_noalloc(), take_bounds_xray(),
                                     take_bounds_fluence(), take_bounds_sweep()})
            if (v == 0) v = w;
        *violation = v;
    });
}

int dc_host_buffer_mapped(int gpu_id, const void *host, unsigned long long bytes, int *mapped) {
    return guarded([&] {
        need(mapped != nullptr, "'mapped' must not be NULL.");
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        *mapped = mapped_host_range(host, (size_t)bytes) != nullptr ? 1 : 0;
    });
}

int dc_version(void) { return 100; }

int dc_device_count(void) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) {
        cudaGetLastError();
        return 0;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    return n;
}

int dc_release_device(int gpu_id) {
    return guarded([&] { release_context(gpu_id); });
}

int dc_photon_set_depth_mode(int gpu_id, int mode) {
    return guarded([&] {
        need(mode == DC_DEPTH_MARCH || mode == DC_DEPTH_LATTICE, "depth mode must be 0 (march) or 1 (lattice).");
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        ctx.photon_depth_mode = mode;
    });
}

int dc_photon_get_depth_mode(int gpu_id, int *mode) {
    return guarded([&] {
        need(mode != nullptr, "'mode' must not be NULL.");
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        *mode = ctx.photon_depth_mode;
    });
}

int dc_photon_depth_stats(int gpu_id, long long *marched) {
    return guarded([&] {
        need(marched != nullptr, "'marched' must not be NULL.");
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        *marched = -1;
        if (ctx.xstat.ptr == nullptr) return;
        DC_CUDA(cudaDeviceSynchronize());
        unsigned v = 0;
        DC_CUDA(cudaMemcpy(&v, ctx.xstat.ptr, sizeof(v), cudaMemcpyDeviceToHost));
        *marched = v == 0xffffffffu ? -1 : (long long)v;
    });
}

int dc_photon_head_selftest(int gpu_id, float *largest_unsaturated, float *skip_bound) {
    return guarded([&] {
        need(largest_unsaturated != nullptr && skip_bound != nullptr, "output pointers must not be NULL.");
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        *largest_unsaturated = photon_erf_unsaturated(3.0f, 4.5f);
        *skip_bound = photon_erf_skip_bound();
    });
}

int dc_profile_enable(int gpu_id, int on) {
    return guarded([&] {
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        ctx.profiling = on != 0;
    });
}

int dc_profile_reset(int gpu_id) {
    return guarded([&] {
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        ctx.prof_collect();
        ctx.profile.clear();
    });
}

int dc_profile_read(int gpu_id, int max, const char **names, int *launches, double *total_ms) {
    int written = 0;
    int rc = guarded([&] {
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        ctx.prof_collect();
        for (auto &kv : ctx.profile) {
            if (written >= max) break;
            names[written] = kv.first.c_str();  // stable: map keys live until reset
            launches[written] = kv.second.launches;
            total_ms[written] = kv.second.total_ms;
            ++written;
        }
    });
    return rc == DC_OK ? written : -rc;
}

// ---------------------------------------------------------------------------
int dc_proton_raytrace(int gpu_id, const float *rlsp, int nz, int ny, int nx, const float spacing[3],
                       const float origin[3], const float iso[3], double gantry_deg, float couch_deg, float vsadx,
                       float vsady, float *wet_out) {
    return guarded([&] {
        check_volume(rlsp, nz, ny, nx, spacing, origin, "voxel_data");
        need(iso != nullptr && wet_out != nullptr, "'iso' and the output buffer must be given.");
        check_proton_model(vsadx, vsady);
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = ctx.stream;
        ctx.begin_call(s);
        const Grid g = make_grid(nz, ny, nx, spacing);
        const Frame f = make_frame(iso, origin, gantry_deg, couch_deg, 0.0, (vsadx + vsady) / 2.0f);
        ctx.density.ensure(nx, ny, nz, false);
        upload_host_volume(ctx, rlsp, nz, ny, nx, &ctx.density, nullptr, s);
        const size_t vb = (size_t)g.n() * sizeof(float);
        // page-locked output: the smoothing kernel stores into it directly
        float *direct = static_cast<float *>(mapped_host_range(wet_out, vb));
        float *wet_s = direct ? direct : static_cast<float *>(ctx.vol_b.ensure(vb));
        proton_raytrace_core(ctx, g, f, wet_s, s);
        if (!direct) DC_CUDA(cudaMemcpyAsync(wet_out, wet_s, vb, cudaMemcpyDeviceToHost, s));
        ctx.end_call(s);
        DC_CUDA(cudaStreamSynchronize(s));
    });
}

int dc_proton_raytrace_dev(int gpu_id, const float *rlsp_dev, int nz, int ny, int nx, const float spacing[3],
                           const float origin[3], const float iso[3], double gantry_deg, float couch_deg,
                           float vsadx, float vsady, float *wet_out_dev, void *stream) {
    return guarded([&] {
        check_volume(rlsp_dev, nz, ny, nx, spacing, origin, "voxel_data");
        need(iso != nullptr && wet_out_dev != nullptr, "'iso' and the output buffer must be given.");
        check_proton_model(vsadx, vsady);
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = as_stream(stream);
        ctx.begin_call(s);
        const Grid g = make_grid(nz, ny, nx, spacing);
        const Frame f = make_frame(iso, origin, gantry_deg, couch_deg, 0.0, (vsadx + vsady) / 2.0f);
        ctx.density.ensure(nx, ny, nz, false);
        copy_host_to_array(ctx.density, rlsp_dev, nz, ny, nx, cudaMemcpyDeviceToDevice, s);
        proton_raytrace_core(ctx, g, f, wet_out_dev, s);
        ctx.end_call(s);
    });
}

int dc_proton_spot(int gpu_id, const float *wet, int nz, int ny, int nx, const float spacing[3],
                   const float origin[3], const float iso[3], double gantry_deg, float couch_deg, float vsadx,
                   float vsady, const float *divergence_params, int n_energies, int dvp_len,
                   const float *lut_depths, const float *lut_sigmas, const float *lut_idds, int lut_len,
                   const float *spots, int n_spots, float *dose_out) {
    return guarded([&] {
        check_volume(wet, nz, ny, nx, spacing, origin, "voxel_data");
        need(iso != nullptr && dose_out != nullptr, "'iso' and the output buffer must be given.");
        need(spots != nullptr, "'spot_list' must not be NULL.");
        check_proton_model(vsadx, vsady);
        check_luts(divergence_params, n_energies, dvp_len, lut_depths, lut_sigmas, lut_idds, lut_len);
        std::vector<LayerRec> layers;
        std::vector<SpotRec> recs;
        build_proton_tables(spots, n_spots, divergence_params, n_energies, dvp_len, vsadx, vsady, layers, recs);
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = ctx.stream;
        ctx.begin_call(s);
        const Grid g = make_grid(nz, ny, nx, spacing);
        const Frame f = make_frame(iso, origin, gantry_deg, couch_deg, 0.0, (vsadx + vsady) / 2.0f);
        const size_t vb = (size_t)g.n() * sizeof(float);
        // Page-locked WET / dose buffers are read / written by the pencil beam
        // in place (each voxel's WET read once per tile, each dose written
        // once); other buffers go through device copies.
        const float *wet_direct = static_cast<const float *>(mapped_host_range(wet, vb));
        float *dose_direct = static_cast<float *>(mapped_host_range(dose_out, vb));
        float *wet_d = wet_direct ? nullptr : static_cast<float *>(ctx.vol_a.ensure(vb));
        float *dose_d = dose_direct ? dose_direct : static_cast<float *>(ctx.vol_b.ensure(vb));
        const size_t lb = (size_t)n_energies * lut_len * sizeof(float);
        const size_t lb_al = (lb + 255) & ~(size_t)255;
        char *lut = static_cast<char *>(ctx.lut.ensure(3 * lb_al));
        DC_CUDA(cudaMemcpyAsync(lut, lut_depths, lb, cudaMemcpyHostToDevice, s));
        DC_CUDA(cudaMemcpyAsync(lut + lb_al, lut_sigmas, lb, cudaMemcpyHostToDevice, s));
        DC_CUDA(cudaMemcpyAsync(lut + 2 * lb_al, lut_idds, lb, cudaMemcpyHostToDevice, s));
        const ProtonTables t = proton_tables(ctx, g, f, layers, recs, reinterpret_cast<const float *>(lut),
                                             reinterpret_cast<const float *>(lut + lb_al),
                                             reinterpret_cast<const float *>(lut + 2 * lb_al), lut_len, s);
        if (wet_direct) {
            launch_pencil_beam(ctx, g, f, t, wet_direct, dose_d, s);
        } else {
            // A voxel's dose needs only its own WET: the pencil beam runs on
            // the tiles whose planes have been uploaded, on the side stream,
            // while the next slab is copied on s.  Each launch waits on an
            // event recorded behind its slab's copy (a wait takes the event's
            // state when enqueued, so the one event is re-recorded per slab);
            // s joins the side stream at the end.
            const int depth = pencil_beam_tile_depth();
            int done = 0;
            upload_host_volume(ctx, wet, nz, ny, nx, nullptr, wet_d, s, [&](int planes) {
                const int ready = planes >= nz ? (nz + depth - 1) / depth : planes / depth;
                if (ready > done) {
                    DC_CUDA(cudaEventRecord(ctx.fork_ev, s));
                    DC_CUDA(cudaStreamWaitEvent(ctx.side, ctx.fork_ev, 0));
                    launch_pencil_beam(ctx, g, f, t, wet_d, dose_d, ctx.side, nullptr, done, ready);
                }
                done = std::max(done, ready);
            });
            DC_CUDA(cudaEventRecord(ctx.join_ev, ctx.side));
            DC_CUDA(cudaStreamWaitEvent(s, ctx.join_ev, 0));
        }
        if (!dose_direct) DC_CUDA(cudaMemcpyAsync(dose_out, dose_d, vb, cudaMemcpyDeviceToHost, s));
        ctx.end_call(s);
        DC_CUDA(cudaStreamSynchronize(s));
    });
}

int dc_proton_spot_dev(int gpu_id, const float *wet_dev, int nz, int ny, int nx, const float spacing[3],
                       const float origin[3], const float iso[3], double gantry_deg, float couch_deg, float vsadx,
                       float vsady, const float *divergence_params, int n_energies, int dvp_len,
                       const float *lut_depths_dev, const float *lut_sigmas_dev, const float *lut_idds_dev,
                       int lut_len, const float *spots, int n_spots, float *dose_out_dev, void *stream) {
    return guarded([&] {
        check_volume(wet_dev, nz, ny, nx, spacing, origin, "voxel_data");
        need(iso != nullptr && dose_out_dev != nullptr, "'iso' and the output buffer must be given.");
        need(spots != nullptr, "'spot_list' must not be NULL.");
        check_proton_model(vsadx, vsady);
        check_luts(divergence_params, n_energies, dvp_len, lut_depths_dev, lut_sigmas_dev, lut_idds_dev, lut_len);
        std::vector<LayerRec> layers;
        std::vector<SpotRec> recs;
        build_proton_tables(spots, n_spots, divergence_params, n_energies, dvp_len, vsadx, vsady, layers, recs);
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = as_stream(stream);
        ctx.begin_call(s);
        const Grid g = make_grid(nz, ny, nx, spacing);
        const Frame f = make_frame(iso, origin, gantry_deg, couch_deg, 0.0, (vsadx + vsady) / 2.0f);
        proton_spot_core(ctx, g, f, layers, recs, lut_depths_dev, lut_sigmas_dev, lut_idds_dev, lut_len, wet_dev,
                         dose_out_dev, s);
        ctx.end_call(s);
    });
}

// ---------------------------------------------------------------------------
namespace {
HuTable make_hu_table(const double *hu, const double *val, int n) {
    need(hu != nullptr && val != nullptr, "the HU table must not be NULL.");
    need(n >= 1 && n <= kMaxHuPoints, "the HU table must have between 1 and 64 points.");
    HuTable t;
    t.n = n;
    for (int i = 0; i < n; ++i) {
        need(std::isfinite(hu[i]) && std::isfinite(val[i]), "HU table entries must be finite.");
        if (i > 0) need(hu[i] > hu[i - 1], "the HU table must be strictly increasing.");
        t.hu[i] = hu[i];
        t.val[i] = val[i];
    }
    return t;
}

// acc = float32(double(acc) + double(d) * w): numpy's float32 += float32 *
// float64 (the reference's `beam_dose += dose * output_factor`).
__global__ void accumulate_weighted_kernel(float *__restrict__ acc, const float *__restrict__ d, long long n,
                                           double w) {
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < n; v += (long long)gridDim.x * blockDim.x)
        acc[v] = __double2float_rn(__dadd_rn((double)acc[v], __dmul_rn((double)d[v], w)));
}

void check_photon(const dc_photon_model *m, const dc_control_point *cp) {
    need(m != nullptr && cp != nullptr, "beam model and control point must be given.");
    need(cp->n_mlc_pairs == 0 ||
             (cp->mlc_x1 && cp->mlc_x2 && cp->mlc_y_offset && cp->mlc_y_width),
         "'mlc' columns must not be NULL.");
    need(m->profile_radius && m->profile_intensities && m->profile_softening, "profile arrays must not be NULL.");
    need(m->n_spectral_energies == 0 || (m->spectrum_attenuation_coefficients && m->spectrum_primary_weights &&
                                         m->spectrum_scatter_weights),
         "spectrum arrays must not be NULL.");
    need(m->kernel_theta_deg && m->kernel_Am && m->kernel_am && m->kernel_Bm && m->kernel_bm &&
             m->kernel_ray_length,
         "'kernel' columns must not be NULL.");
}
}  // namespace

int dc_photon_dose(int gpu_id, const float *density, int nz, int ny, int nx, const float spacing[3],
                   const float origin[3], const dc_photon_model *model, const dc_control_point *cp,
                   float *dose_out) {
    return guarded([&] {
        check_volume(density, nz, ny, nx, spacing, origin, "voxel_data");
        need(dose_out != nullptr, "the output buffer must be given.");
        check_photon(model, cp);
        static thread_local PhotonParams P;
        static thread_local CccsCones C;
        build_photon_params(*model, *cp, spacing[0] / 10.0f, P, C);
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = ctx.stream;
        ctx.begin_call(s);
        const Grid g = make_grid(nz, ny, nx, spacing);
        const Frame f = make_frame(cp->iso, origin, cp->gantry_deg, cp->couch_deg, cp->collimator_deg,
                                   model->primary_source_distance);
        photon_head_fork(ctx, g, f, P, s);  // the head factors need no density: they run during the upload
        ctx.density.ensure(nx, ny, nz, false);
        upload_host_volume(ctx, density, nz, ny, nx, &ctx.density, nullptr, s);
        const size_t vb = (size_t)g.n() * sizeof(float);
        // page-locked output: TERMA (masked zeros) and CCCS store into it directly
        float *direct = static_cast<float *>(mapped_host_range(dose_out, vb));
        float *dose_d = direct ? direct : static_cast<float *>(ctx.vol_b.ensure(vb));
        run_photon_pipeline(ctx, g, f, P, C, model->mu_calibration * cp->mu, dose_d, s);
        if (!direct) DC_CUDA(cudaMemcpyAsync(dose_out, dose_d, vb, cudaMemcpyDeviceToHost, s));
        ctx.end_call(s);
        DC_CUDA(cudaStreamSynchronize(s));
    });
}

int dc_photon_dose_dev(int gpu_id, const float *density_dev, int nz, int ny, int nx, const float spacing[3],
                       const float origin[3], const dc_photon_model *model, const dc_control_point *cp,
                       float *dose_out_dev, void *stream) {
    return guarded([&] {
        check_volume(density_dev, nz, ny, nx, spacing, origin, "voxel_data");
        need(dose_out_dev != nullptr, "the output buffer must be given.");
        check_photon(model, cp);
        static thread_local PhotonParams P;
        static thread_local CccsCones C;
        build_photon_params(*model, *cp, spacing[0] / 10.0f, P, C);
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = as_stream(stream);
        ctx.begin_call(s);
        const Grid g = make_grid(nz, ny, nx, spacing);
        const Frame f = make_frame(cp->iso, origin, cp->gantry_deg, cp->couch_deg, cp->collimator_deg,
                                   model->primary_source_distance);
        ctx.density.ensure(nx, ny, nz, false);
        copy_host_to_array(ctx.density, density_dev, nz, ny, nx, cudaMemcpyDeviceToDevice, s);
        run_photon_pipeline(ctx, g, f, P, C, model->mu_calibration * cp->mu, dose_out_dev, s);
        ctx.end_call(s);
    });
}

// ---------------------------------------------------------------------------
// HU conversion on the device, fused ray trace, multi-control-point photon
// plans (the next steps either side of the hot path; no reference counterpart
// beyond the host loops they replace, plan_impt.py:112-160,
// plan_imrt.py:114-158).
// ---------------------------------------------------------------------------
int dc_hu_convert_dev(int gpu_id, const float *hu_dev, int nz, int ny, int nx, const double *table_hu,
                      const double *table_val, int n_table, float *out_dev, void *stream) {
    return guarded([&] {
        need(hu_dev != nullptr && out_dev != nullptr, "'hu' and the output buffer must not be NULL.");
        need(nz > 0 && ny > 0 && nx > 0, "'hu' must have positive dimensions.");
        const HuTable t = make_hu_table(table_hu, table_val, n_table);
        DeviceContext &ctx = context(gpu_id);
        (void)ctx;
        launch_hu_convert(t, hu_dev, nx, ny, nz, out_dev, 0, as_stream(stream));
    });
}

int dc_proton_raytrace_hu_dev(int gpu_id, const float *hu_dev, int nz, int ny, int nx, const float spacing[3],
                              const float origin[3], const double *table_hu, const double *table_rlsp, int n_table,
                              const float iso[3], double gantry_deg, float couch_deg, float vsadx, float vsady,
                              float *wet_out_dev, void *stream) {
    return guarded([&] {
        check_volume(hu_dev, nz, ny, nx, spacing, origin, "voxel_data");
        need(iso != nullptr && wet_out_dev != nullptr, "'iso' and the output buffer must be given.");
        check_proton_model(vsadx, vsady);
        const HuTable t = make_hu_table(table_hu, table_rlsp, n_table);
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = as_stream(stream);
        ctx.begin_call(s);
        const Grid g = make_grid(nz, ny, nx, spacing);
        const Frame f = make_frame(iso, origin, gantry_deg, couch_deg, 0.0, (vsadx + vsady) / 2.0f);
        ctx.density.ensure(nx, ny, nz, true);  // RLSP written straight into the texture array
        launch_hu_convert(t, hu_dev, nx, ny, nz, nullptr, ctx.density.surf, s);
        proton_raytrace_core(ctx, g, f, wet_out_dev, s);
        ctx.end_call(s);
    });
}

int dc_photon_plan_dose_dev(int gpu_id, const float *volume_dev, int is_hu, const double *table_hu,
                            const double *table_density, int n_table, int nz, int ny, int nx, const float spacing[3],
                            const float origin[3], const dc_photon_model *model, const dc_control_point *cps,
                            int n_cps, const double *weights, float *dose_accum_dev, void *stream) {
    return guarded([&] {
        check_volume(volume_dev, nz, ny, nx, spacing, origin, "voxel_data");
        need(dose_accum_dev != nullptr, "the output buffer must be given.");
        need(n_cps >= 0 && (n_cps == 0 || (cps != nullptr && weights != nullptr)),
             "control points and weights must be given.");
        HuTable t{};
        if (is_hu) t = make_hu_table(table_hu, table_density, n_table);
        static thread_local PhotonParams P;
        static thread_local CccsCones Cn;
        for (int q = 0; q < n_cps; ++q) {  // validate every control point before any work
            check_photon(model, &cps[q]);
            need(std::isfinite(weights[q]), "control-point weights must be finite.");
            build_photon_params(*model, cps[q], spacing[0] / 10.0f, P, Cn);
        }
        DeviceContext &ctx = context(gpu_id);
        std::lock_guard<std::mutex> lk(ctx.mu);
        cudaStream_t s = as_stream(stream);
        ctx.begin_call(s);
        const Grid g = make_grid(nz, ny, nx, spacing);
        if (is_hu) {
            ctx.density.ensure(nx, ny, nz, true);
            launch_hu_convert(t, volume_dev, nx, ny, nz, nullptr, ctx.density.surf, s);
        } else {
            ctx.density.ensure(nx, ny, nz, false);
            copy_host_to_array(ctx.density, volume_dev, nz, ny, nx, cudaMemcpyDeviceToDevice, s);
        }
        const size_t vb = (size_t)g.n() * sizeof(float);
        float *cp_dose = static_cast<float *>(ctx.vol_b.ensure(vb));
        int sms = 0;
        DC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
        for (int q = 0; q < n_cps; ++q) {
            build_photon_params(*model, cps[q], spacing[0] / 10.0f, P, Cn);
            const Frame f = make_frame(cps[q].iso, origin, cps[q].gantry_deg, cps[q].couch_deg,
                                       cps[q].collimator_deg, model->primary_source_distance);
            run_photon_pipeline(ctx, g, f, P, Cn, model->mu_calibration * cps[q].mu, cp_dose, s);
            accumulate_weighted_kernel<<<(unsigned)std::min<long long>((g.n() + 255) / 256, (long long)sms * 8), 256,
                                         0, s>>>(dose_accum_dev, cp_dose, g.n(), weights[q]);
            check_launch("accumulate_weighted_kernel");
        }
        ctx.end_call(s);
    });
}

}  // extern "C"
