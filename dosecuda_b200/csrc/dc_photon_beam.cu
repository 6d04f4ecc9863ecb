// dc_photon_beam.cu — a photon beam kept on the device, for the learned
// surrogate path, and the gamma index used to accept or reject its output.
//
// A dc_photon_beam owns the work buffers of one grid (density texture, the
// (TERMA, density) surface array, radiological depth, electron term, CCCS
// voxel list, cone directions), so that one TERMA pass serves any number of
// CCCS evaluations: the full volume (dc_photon_beam_dose), or a sparse probe
// of voxels on a few lines through the field (dc_photon_beam_probe).  The
// kernels are the ones dc_photon_dose runs; the probe computes exactly the
// per-voxel CCCS sum of the full calculation at its voxels.
//
// dc_gamma evaluates the gamma index (distance-to-agreement dta_mm, dose
// difference dd_frac of a global normalisation) of an evaluated dose volume
// against reference points: one warp per reference point searches the
// evaluated volume, trilinearly interpolated, on a sub-voxel lattice of
// step dta/4 inside the dta sphere, which decides gamma <= 1 exactly up to
// that lattice.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <iterator>
#include <string>
#include <vector>

#include "../../include/dosecuda.h"
#include "dc_common.cuh"
#include "dc_kernels.cuh"
#include "dc_photon.cuh"
#include "dc_runtime.cuh"

using namespace dc;

struct dc_photon_beam {
    int device = 0;
    Grid g{};
    float origin[3] = {0, 0, 0};
    VolumeArray density;
    VolumeArray td;
    DeviceBuffer wet, electron, active, dirs, probe, xlat;
    // fluence mode: the unmodulated TERMA and electron term of the last
    // dc_photon_beam_terma, and the adjoint's scratch
    DeviceBuffer terma0, electron0, fl_h;
    DeviceBuffer sweep_lat, sweep_acc, sweep_box;  // cone-direction sweep mode
    bool have_e0 = false;
    PhotonParams P{};
    CccsCones C{};
    Frame f{};
    float dose_scale = 0.f;
    float src_dist = 0.f;
    float field[4] = {0, 0, 0, 0};  // open-field box at the isocentre plane: x1, x2, y1, y2 (mm)
    bool have_density = false, have_terma = false;
    std::vector<int> probe_host;
    int lattice = 4;                  // probe lattice stride (0: lines only)
    PinnedBuffer probe_pin;           // staging of the probe list
    cudaEvent_t probe_ev = nullptr;   // its last upload

    PhotonWork work() {
        PhotonWork w;
        const size_t n = (size_t)g.n();
        w.wet = static_cast<float *>(wet.ensure(n * sizeof(float)));
        w.electron = static_cast<float *>(electron.ensure(n * sizeof(float)));
        char *act = static_cast<char *>(active.ensure(256 + n * sizeof(int)));
        w.n_active = reinterpret_cast<unsigned *>(act);
        w.active = reinterpret_cast<int *>(act + 256);
        w.dirs = static_cast<float4 *>(dirs.ensure(kMaxCones * 12 * sizeof(float4)));
        w.dens_tex = density.texture(kAirDensity);
        w.td_surf = td.surf;
        w.td_tex = td.texture(0.0f, kAirDensity);
        w.xlat = &xlat;
        w.depth_mode = context(device).photon_depth_mode;
        return w;
    }
    ~dc_photon_beam() {
        cudaSetDevice(device);
        density.release();
        td.release();
        wet.release();
        xlat.release();
        terma0.release();
        electron0.release();
        fl_h.release();
        sweep_lat.release();
        sweep_acc.release();
        sweep_box.release();
        electron.release();
        active.release();
        dirs.release();
        probe.release();
        if (probe_ev) cudaEventSynchronize(probe_ev), cudaEventDestroy(probe_ev);
        probe_pin.release();
    }
};

namespace {

void need(bool ok, const std::string &m) {
    if (!ok) throw Error(DC_ERR_VALUE, m);
}

cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// ---------------------------------------------------------------------------
// gamma index
// ---------------------------------------------------------------------------
__global__ void volume_max_kernel(const float *__restrict__ v, long long n, unsigned *__restrict__ out_bits) {
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, __ldg(v + i));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    // non-negative floats order like their bit patterns
    if ((threadIdx.x & 31) == 0) atomicMax(out_bits, __float_as_uint(m));
}

__device__ __forceinline__ float trilinear(const float *__restrict__ vol, int nx, int ny, int nz, float x, float y,
                                           float z) {
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const int i0 = (int)fx, j0 = (int)fy, k0 = (int)fz;
    const float ax = x - fx, ay = y - fy, az = z - fz;
    const int i1 = min(i0 + 1, nx - 1), j1 = min(j0 + 1, ny - 1), k1 = min(k0 + 1, nz - 1);
    auto at = [&](int i, int j, int k) { return __ldg(vol + ((size_t)k * ny + j) * nx + i); };
    const float c00 = at(i0, j0, k0) + ax * (at(i1, j0, k0) - at(i0, j0, k0));
    const float c10 = at(i0, j1, k0) + ax * (at(i1, j1, k0) - at(i0, j1, k0));
    const float c01 = at(i0, j0, k1) + ax * (at(i1, j0, k1) - at(i0, j0, k1));
    const float c11 = at(i0, j1, k1) + ax * (at(i1, j1, k1) - at(i0, j1, k1));
    const float c0 = c00 + ay * (c10 - c00);
    const float c1 = c01 + ay * (c11 - c01);
    return c0 + az * (c1 - c0);
}

struct GammaArgs {
    const float *eval;
    const int *voxels;  // null: every voxel, ref is a volume
    const float *ref;
    long long n;
    int nx, ny, nz;
    float sx, sy, sz;
    float dta, dd_frac, cutoff_frac;
    float norm;                // > 0: the normalisation dose
    const unsigned *norm_bits; // else: max of eval
    int *counts;               // [0] evaluated, [1] passed, [2] max-of-eval scratch
};

constexpr int kGammaSteps = 4;  // lattice points per dta along each axis

__global__ void __launch_bounds__(256) gamma_kernel(GammaArgs a) {
    const int lane = threadIdx.x & 31;
    const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    const float norm = a.norm > 0.f ? a.norm : __uint_as_float(*a.norm_bits);
    const float dd = a.dd_frac * norm;
    const float inv_dd2 = dd > 0.f ? 1.0f / (dd * dd) : 0.f;
    const float inv_dta2 = 1.0f / (a.dta * a.dta);
    const float h = a.dta / kGammaSteps;
    constexpr int W = 2 * kGammaSteps + 1;
    int evaluated = 0, passed = 0;
    for (long long q = warp0; q < a.n; q += nwarps) {
        const long long v = a.voxels ? (long long)__ldg(a.voxels + q) : q;
        const float R = __ldg(a.ref + q);
        if (!(R >= a.cutoff_frac * norm) || !(norm > 0.f)) continue;  // warp-uniform
        if (v < 0 || v >= (long long)a.nx * a.ny * a.nz) continue;  // not a voxel of the grid
        const int k = (int)(v / ((long long)a.nx * a.ny));
        const int rem = (int)(v - (long long)k * a.nx * a.ny);
        const int j = rem / a.nx, i = rem - j * a.nx;
        float best = 3.0e38f;
        for (int c = lane; c < W * W * W; c += 32) {
            const int ix = c % W - kGammaSteps, iy = (c / W) % W - kGammaSteps, iz = c / (W * W) - kGammaSteps;
            const float r2 = (float)(ix * ix + iy * iy + iz * iz) * h * h;
            if (r2 > a.dta * a.dta * 1.0001f) continue;
            const float x = (float)i + ix * h / a.sx, y = (float)j + iy * h / a.sy, z = (float)k + iz * h / a.sz;
            if (x < 0.f || y < 0.f || z < 0.f || x > (float)(a.nx - 1) || y > (float)(a.ny - 1) ||
                z > (float)(a.nz - 1))
                continue;
            const float E = trilinear(a.eval, a.nx, a.ny, a.nz, x, y, z);
            const float g2 = r2 * inv_dta2 + (E - R) * (E - R) * inv_dd2;
            best = fminf(best, g2);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = fminf(best, __shfl_xor_sync(0xffffffffu, best, o));
        ++evaluated;
        passed += best <= 1.0f;
    }
    if (lane == 0 && evaluated) {
        atomicAdd(&a.counts[0], evaluated);
        atomicAdd(&a.counts[1], passed);
    }
}

// ---------------------------------------------------------------------------
// Probe voxels: rays from the source through points of the open field at the
// isocentre plane (centre, half-field and field-edge positions along both
// field axes), lateral profiles across the field at three depths, and a
// regular lattice of every `lattice`-th voxel along each axis (an unbiased
// sample of the whole volume; voxels outside the beam cost one texture
// fetch).  The CCCS of a probe costs about one voxel's march in latency
// whatever its size, so the lattice is nearly free.
// ---------------------------------------------------------------------------
void select_probe(dc_photon_beam &b) {
    const Grid &g = b.g;
    const Frame &f = b.f;
    std::vector<int> out;
    const float step = 0.5f * std::min(g.sx, std::min(g.sy, g.sz));
    const float ext[3] = {g.nx * g.sx, g.ny * g.sy, g.nz * g.sz};
    const float reach = 0.5f * std::sqrt(ext[0] * ext[0] + ext[1] * ext[1] + ext[2] * ext[2]) +
                        std::sqrt((f.isox - 0.5f * ext[0]) * (f.isox - 0.5f * ext[0]) +
                                  (f.isoy - 0.5f * ext[1]) * (f.isoy - 0.5f * ext[1]) +
                                  (f.isoz - 0.5f * ext[2]) * (f.isoz - 0.5f * ext[2]));
    auto add = [&](float3 h) {
        const float3 p = head_to_image<true>(f, h);
        const int i = (int)std::lround((p.x + f.isox) / g.sx);
        const int j = (int)std::lround((p.y + f.isoy) / g.sy);
        const int k = (int)std::lround((p.z + f.isoz) / g.sz);
        if (i < 0 || j < 0 || k < 0 || i >= g.nx || j >= g.ny || k >= g.nz) return;
        const int v = i + g.nx * (j + g.ny * k);
        if (out.empty() || out.back() != v) out.push_back(v);
    };
    const float cx = 0.5f * (b.field[0] + b.field[1]), cy = 0.5f * (b.field[2] + b.field[3]);
    const float hx = 0.5f * (b.field[1] - b.field[0]), hy = 0.5f * (b.field[3] - b.field[2]);
    const float sad = b.src_dist;
    const float fr[5][2] = {{0.f, 0.f}, {0.5f, 0.f}, {-0.5f, 0.f}, {0.f, 0.5f}, {0.f, -0.5f}};
    const float fe[4][2] = {{1.f, 0.f}, {-1.f, 0.f}, {0.f, 1.f}, {0.f, -1.f}};
    auto cone_line = [&](float qx, float qy) {
        // source (0, 0, sad) -> (qx, qy, 0), head frame
        const float dx = qx, dy = qy, dz = -sad;
        const float dn = std::sqrt(dx * dx + dy * dy + dz * dz);
        const float ux = dx / dn, uy = dy / dn, uz = dz / dn;
        for (float t = -reach; t <= reach; t += step) add(make_float3(qx + t * ux, qy + t * uy, t * uz));
    };
    for (auto &q : fr) cone_line(cx + q[0] * hx, cy + q[1] * hy);
    for (auto &q : fe) cone_line(cx + q[0] * hx, cy + q[1] * hy);
    const float depths[3] = {50.f, 0.f, -50.f};  // head z: upstream, isocentre, downstream (mm)
    for (float zz : depths) {
        const float div = (sad - zz) / sad;
        const float mx = (hx + 20.f) * div, my = (hy + 20.f) * div;
        for (float x = -mx; x <= mx; x += step) add(make_float3(cx * div + x, cy * div, zz));
        for (float y = -my; y <= my; y += step) add(make_float3(cx * div, cy * div + y, zz));
    }
    std::sort(out.begin(), out.end());
    out.erase(std::unique(out.begin(), out.end()), out.end());
    if (b.lattice > 0) {
        const int L = b.lattice, o = L / 2;
        std::vector<int> lat;
        lat.reserve((size_t)(g.nx / L + 1) * (g.ny / L + 1) * (g.nz / L + 1));
        for (int k = o; k < g.nz; k += L)
            for (int j = o; j < g.ny; j += L)
                for (int i = o; i < g.nx; i += L) lat.push_back(i + g.nx * (j + g.ny * k));
        std::vector<int> merged;
        merged.reserve(out.size() + lat.size());
        std::merge(out.begin(), out.end(), lat.begin(), lat.end(), std::back_inserter(merged));
        merged.erase(std::unique(merged.begin(), merged.end()), merged.end());
        out.swap(merged);
    }
    b.probe_host.swap(out);
}

// Selects the probe of the current control point and enqueues its upload on
// stream s (from pinned staging; no host synchronisation unless the previous
// upload is still in flight).
void select_and_upload_probe(dc_photon_beam &b, cudaStream_t s) {
    select_probe(b);
    const size_t bytes = b.probe_host.size() * sizeof(int);
    if (b.probe_ev) DC_CUDA(cudaEventSynchronize(b.probe_ev));
    else DC_CUDA(cudaEventCreateWithFlags(&b.probe_ev, cudaEventDisableTiming));
    void *dst = b.probe.ensure(std::max<size_t>(bytes, 256));
    if (bytes) {
        void *pin = b.probe_pin.ensure(bytes);
        std::memcpy(pin, b.probe_host.data(), bytes);
        DC_CUDA(cudaMemcpyAsync(dst, pin, bytes, cudaMemcpyHostToDevice, s));
    }
    DC_CUDA(cudaEventRecord(b.probe_ev, s));
}

}  // namespace

extern "C" {

int dc_photon_beam_create(int gpu_id, int nz, int ny, int nx, const float spacing[3], const float origin[3],
                          dc_photon_beam **out) {
    return guarded([&] {
        need(out != nullptr, "'out' must not be NULL.");
        *out = nullptr;
        need(nz > 0 && ny > 0 && nx > 0, "'voxel_data' must have positive dimensions.");
        need(spacing && origin, "'spacing' and 'origin' must be given.");
        for (int a = 0; a < 3; ++a) {
            need(std::isfinite(spacing[a]) && spacing[a] > 0.0f, "'spacing' must be positive and finite.");
            need(std::isfinite(origin[a]), "'origin' must be finite.");
        }
        need(nx <= 16384 && ny <= 16384 && nz <= 16384, "volume dimensions above 16384 are not supported.");
        need((long long)nx * ny * nz <= 0x7fffffffLL, "photon volumes are limited to 2^31 - 1 voxels.");
        context(gpu_id);  // validates the ordinal and makes the device current
        auto *b = new dc_photon_beam();
        try {
            b->device = gpu_id;
            b->g = make_grid(nz, ny, nx, spacing);
            for (int a = 0; a < 3; ++a) b->origin[a] = origin[a];
            b->density.ensure(nx, ny, nz, false);
            b->td.ensure(nx, ny, nz, true, 2);
            b->work();  // allocate the buffers now, not inside a timed or captured call
        } catch (...) {
            delete b;
            throw;
        }
        *out = b;
    });
}

int dc_photon_beam_destroy(dc_photon_beam *b) {
    return guarded([&] { delete b; });
}

int dc_photon_beam_set_density(dc_photon_beam *b, const float *density_dev, void *stream) {
    return guarded([&] {
        need(b != nullptr && density_dev != nullptr, "beam and density must not be NULL.");
        DC_CUDA(cudaSetDevice(b->device));
        cudaMemcpy3DParms p{};
        p.srcPtr = make_cudaPitchedPtr((void *)density_dev, (size_t)b->g.nx * sizeof(float), (size_t)b->g.nx,
                                       (size_t)b->g.ny);
        p.dstArray = b->density.arr;
        p.extent = make_cudaExtent((size_t)b->g.nx, (size_t)b->g.ny, (size_t)b->g.nz);
        p.kind = cudaMemcpyDeviceToDevice;
        DC_CUDA(cudaMemcpy3DAsync(&p, as_stream(stream)));
        b->have_density = true;
        b->have_terma = false;
    });
}

int dc_photon_beam_terma(dc_photon_beam *b, const dc_photon_model *model, const dc_control_point *cp,
                         float *terma_out_dev, void *stream) {
    return guarded([&] {
        need(b != nullptr && model != nullptr && cp != nullptr, "beam, model and control point must be given.");
        need(b->have_density, "the beam has no density volume (dc_photon_beam_set_density).");
        need(cp->n_mlc_pairs == 0 || (cp->mlc_x1 && cp->mlc_x2 && cp->mlc_y_offset && cp->mlc_y_width),
             "'mlc' columns must not be NULL.");
        need(model->profile_radius && model->profile_intensities && model->profile_softening && model->kernel_theta_deg &&
                 model->kernel_Am && model->kernel_am && model->kernel_Bm && model->kernel_bm &&
                 model->kernel_ray_length,
             "beam model arrays must not be NULL.");
        need(model->n_spectral_energies == 0 ||
                 (model->spectrum_attenuation_coefficients && model->spectrum_primary_weights &&
                  model->spectrum_scatter_weights),
             "spectrum arrays must not be NULL.");
        build_photon_params(*model, *cp, b->g.sx / 10.0f, b->P, b->C);
        b->f = make_frame(cp->iso, b->origin, cp->gantry_deg, cp->couch_deg, cp->collimator_deg,
                          model->primary_source_distance);
        b->dose_scale = model->mu_calibration * cp->mu;
        b->src_dist = model->primary_source_distance;
        float x1 = 0, x2 = 0, y1 = 0, y2 = 0;
        bool any = false;
        for (int q = 0; q < cp->n_mlc_pairs; ++q) {
            if (!(cp->mlc_x2[q] > cp->mlc_x1[q])) continue;
            const float yb = cp->mlc_y_offset[q] - 0.5f * cp->mlc_y_width[q];
            const float yt = cp->mlc_y_offset[q] + 0.5f * cp->mlc_y_width[q];
            if (!any) {
                x1 = cp->mlc_x1[q], x2 = cp->mlc_x2[q], y1 = yb, y2 = yt;
                any = true;
            } else {
                x1 = std::min(x1, cp->mlc_x1[q]), x2 = std::max(x2, cp->mlc_x2[q]);
                y1 = std::min(y1, yb), y2 = std::max(y2, yt);
            }
        }
        b->field[0] = x1, b->field[1] = x2, b->field[2] = y1, b->field[3] = y2;
        DC_CUDA(cudaSetDevice(b->device));
        DeviceContext &ctx = context(b->device);
        float *t0 = static_cast<float *>(b->terma0.ensure((size_t)b->g.n() * sizeof(float)));
        enqueue_terma(ctx, b->g, b->f, b->P, b->C, b->work(), nullptr, t0, as_stream(stream));
        if (terma_out_dev)
            DC_CUDA(cudaMemcpyAsync(terma_out_dev, t0, (size_t)b->g.n() * sizeof(float), cudaMemcpyDeviceToDevice,
                                    as_stream(stream)));
        b->have_terma = true;
        b->have_e0 = false;
        // the probe of this control point, selected on the host while the
        // TERMA kernels run
        select_and_upload_probe(*b, as_stream(stream));
    });
}

int dc_photon_beam_dose(dc_photon_beam *b, float *dose_out_dev, void *stream) {
    return guarded([&] {
        need(b != nullptr && dose_out_dev != nullptr, "beam and output must not be NULL.");
        need(b->have_terma, "dc_photon_beam_terma must run first.");
        DC_CUDA(cudaSetDevice(b->device));
        DeviceContext &ctx = context(b->device);
        cudaStream_t s = as_stream(stream);
        DC_CUDA(cudaMemsetAsync(dose_out_dev, 0, (size_t)b->g.n() * sizeof(float), s));
        enqueue_cccs(ctx, b->g, b->f, b->C, b->work(), b->dose_scale, dose_out_dev, s);
    });
}

namespace {

FluenceMap fluence_map(const dc_photon_beam &b, const dc_fluence_map *m) {
    need(m != nullptr, "fluence map must not be NULL.");
    need(m->na >= 1 && m->nb >= 1 && (long long)m->na * m->nb <= (1LL << 24), "fluence map size out of range.");
    need(std::isfinite(m->a0) && std::isfinite(m->b0) && std::isfinite(m->pitch) && m->pitch > 0.0f,
         "fluence map origin and pitch must be finite, the pitch positive.");
    FluenceMap M{};
    M.na = m->na;
    M.nb = m->nb;
    M.a0 = m->a0;
    M.b0 = m->b0;
    M.inv_pitch = 1.0f / m->pitch;
    M.sad = b.src_dist;
    return M;
}

// E0: the electron term of the last TERMA pass, kept before a fluence
// forward overwrites the work set's electron volume.
const float *electron0(dc_photon_beam &b, cudaStream_t s) {
    const size_t bytes = (size_t)b.g.n() * sizeof(float);
    float *e0 = static_cast<float *>(b.electron0.ensure(bytes));
    if (!b.have_e0) {
        DC_CUDA(cudaMemcpyAsync(e0, b.electron.ptr, bytes, cudaMemcpyDeviceToDevice, s));
        b.have_e0 = true;
    }
    return e0;
}

}  // namespace

int dc_photon_beam_fluence_dose(dc_photon_beam *b, const dc_fluence_map *map, const float *fluence_dev,
                                float *dose_out_dev, void *stream) {
    return guarded([&] {
        need(b != nullptr && fluence_dev != nullptr && dose_out_dev != nullptr,
             "beam, fluence and output must not be NULL.");
        need(b->have_terma, "dc_photon_beam_terma must run first.");
        const FluenceMap M = fluence_map(*b, map);
        DC_CUDA(cudaSetDevice(b->device));
        DeviceContext &ctx = context(b->device);
        cudaStream_t s = as_stream(stream);
        const PhotonWork w = b->work();
        const float *e0 = electron0(*b, s);
        enqueue_fluence_modulate(ctx, b->g, b->f, M, fluence_dev, b->terma0.as<float>(), e0, w, s);
        DC_CUDA(cudaMemsetAsync(dose_out_dev, 0, (size_t)b->g.n() * sizeof(float), s));
        enqueue_cccs(ctx, b->g, b->f, b->C, w, b->dose_scale, dose_out_dev, s);
    });
}

int dc_photon_beam_fluence_adjoint(dc_photon_beam *b, const dc_fluence_map *map, const float *grad_dose_dev,
                                   double *grad_fluence_dev, void *stream) {
    return guarded([&] {
        need(b != nullptr && grad_dose_dev != nullptr && grad_fluence_dev != nullptr,
             "beam, gradient and output must not be NULL.");
        need(b->have_terma, "dc_photon_beam_terma must run first.");
        const FluenceMap M = fluence_map(*b, map);
        DC_CUDA(cudaSetDevice(b->device));
        DeviceContext &ctx = context(b->device);
        cudaStream_t s = as_stream(stream);
        const PhotonWork w = b->work();
        const float *e0 = electron0(*b, s);
        float *h = static_cast<float *>(b->fl_h.ensure((size_t)b->g.n() * sizeof(float)));
        enqueue_fluence_adjoint(ctx, b->g, b->f, b->C, M, b->dose_scale, b->terma0.as<float>(), e0, w, grad_dose_dev,
                                h, grad_fluence_dev, s);
    });
}

int dc_photon_beam_dose_sweep(dc_photon_beam *b, float *dose_out_dev, void *stream) {
    return guarded([&] {
        need(b != nullptr && dose_out_dev != nullptr, "beam and output must not be NULL.");
        need(b->have_terma, "dc_photon_beam_terma must run first.");
        need(b->g.sx == b->g.sy && b->g.sx == b->g.sz, "the sweep needs isotropic voxels.");
        DC_CUDA(cudaSetDevice(b->device));
        DeviceContext &ctx = context(b->device);
        cudaStream_t s = as_stream(stream);
        DC_CUDA(cudaMemsetAsync(dose_out_dev, 0, (size_t)b->g.n() * sizeof(float), s));
        enqueue_cccs_sweep(ctx, b->g, b->f, b->C, b->work(), b->dose_scale, dose_out_dev, b->sweep_lat, b->sweep_acc,
                           b->sweep_box, s);
    });
}

int dc_photon_beam_probe_config(dc_photon_beam *b, int lattice_stride) {
    return guarded([&] {
        need(b != nullptr, "beam must not be NULL.");
        need(lattice_stride >= 0, "'lattice_stride' must not be negative.");
        b->lattice = lattice_stride;
    });
}

int dc_photon_beam_probe_select(dc_photon_beam *b, int *n_out, void *stream) {
    return guarded([&] {
        need(b != nullptr && n_out != nullptr, "beam and count must not be NULL.");
        need(b->have_terma, "dc_photon_beam_terma must run first.");
        DC_CUDA(cudaSetDevice(b->device));
        select_and_upload_probe(*b, as_stream(stream));
        *n_out = (int)b->probe_host.size();
    });
}

int dc_photon_beam_probe_list(const dc_photon_beam *b, const int **voxels_dev, int *n, int *voxels_host, int cap) {
    return guarded([&] {
        need(b != nullptr && voxels_dev != nullptr && n != nullptr, "arguments must not be NULL.");
        *voxels_dev = static_cast<const int *>(b->probe.ptr);
        *n = (int)b->probe_host.size();
        if (voxels_host)
            std::copy(b->probe_host.begin(), b->probe_host.begin() + std::min<size_t>(cap, b->probe_host.size()),
                      voxels_host);
    });
}

int dc_photon_beam_probe(dc_photon_beam *b, const int *voxels_dev, int n, float *dose_out_dev, void *stream) {
    return guarded([&] {
        need(b != nullptr && dose_out_dev != nullptr, "beam and output must not be NULL.");
        need(b->have_terma, "dc_photon_beam_terma must run first.");
        if (!voxels_dev) {
            voxels_dev = static_cast<const int *>(b->probe.ptr);
            n = (int)b->probe_host.size();
        }
        need(n >= 0, "'n' must not be negative.");
        DC_CUDA(cudaSetDevice(b->device));
        DeviceContext &ctx = context(b->device);
        enqueue_cccs_points(ctx, b->g, b->f, b->C, b->work(), b->dose_scale, voxels_dev, n, dose_out_dev,
                            as_stream(stream));
    });
}

int dc_gamma(int gpu_id, const float *eval_dev, int nz, int ny, int nx, const float spacing[3], const int *voxels_dev,
             const float *ref_dev, long long n, float dose_norm, float dta_mm, float dd_frac, float cutoff_frac,
             int *counts_dev, void *stream) {
    return guarded([&] {
        need(eval_dev && ref_dev && counts_dev && spacing, "gamma buffers must not be NULL.");
        need(nz > 0 && ny > 0 && nx > 0, "gamma volume must have positive dimensions.");
        need(dta_mm > 0.f && dd_frac > 0.f && cutoff_frac >= 0.f, "gamma criteria must be positive.");
        for (int a = 0; a < 3; ++a) need(spacing[a] > 0.f, "'spacing' must be positive.");
        const long long vox = (long long)nx * ny * nz;
        if (!voxels_dev) n = vox;
        need(n >= 0, "'n' must not be negative.");
        DeviceContext &ctx = context(gpu_id);
        cudaStream_t s = as_stream(stream);
        DC_CUDA(cudaMemsetAsync(counts_dev, 0, 2 * sizeof(int), s));
        GammaArgs a{};
        a.eval = eval_dev;
        a.voxels = voxels_dev;
        a.ref = ref_dev;
        a.n = n;
        a.nx = nx, a.ny = ny, a.nz = nz;
        a.sx = spacing[0], a.sy = spacing[1], a.sz = spacing[2];
        a.dta = dta_mm, a.dd_frac = dd_frac, a.cutoff_frac = cutoff_frac;
        a.norm = dose_norm;
        a.counts = counts_dev;
        int sms = 0;
        DC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx.device));
        if (!(dose_norm > 0.f)) {
            unsigned *bits = reinterpret_cast<unsigned *>(counts_dev + 2);  // caller-owned scratch word
            DC_CUDA(cudaMemsetAsync(bits, 0, sizeof(unsigned), s));
            volume_max_kernel<<<(unsigned)std::min<long long>((vox + 255) / 256, (long long)sms * 8), 256, 0, s>>>(
                eval_dev, vox, bits);
            check_launch("volume_max_kernel");
            a.norm_bits = bits;
        }
        if (n == 0) return;
        const long long warps = std::min<long long>(n, (long long)sms * 64);
        KernelTimer kt(ctx, "gamma", s);
        gamma_kernel<<<(unsigned)((warps * 32 + 255) / 256), 256, 0, s>>>(a);
        check_launch("gamma_kernel");
    });
}

}  // extern "C"
