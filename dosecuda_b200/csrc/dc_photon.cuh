// dc_photon.cuh — per-control-point parameter blocks of the photon engine.
// Both are passed to the kernels by value (kernel-parameter constant bank), so
// concurrent calls on different streams never share mutable device state.
#pragma once

#include "../../include/dosecuda.h"
#include "dc_common.cuh"
#include "dc_runtime.cuh"

namespace dc {

constexpr int kMaxPairs = 128;      // MLC leaf pairs
constexpr int kMaxProfile = 64;     // off-axis profile points
constexpr int kMaxSpectrum = 32;    // spectral energy bins
constexpr int kMaxCones = 8;        // zenith cones (kernel.csv rows)
constexpr int kMaxConeSteps = 512;  // summed samples per azimuth over all cones

struct PhotonParams {
    float psd, ssd, pss, sss, mlc_distance, ssw, ea, esw, efd;
    int n_pairs, n_prof, n_spec;
    int edges_sorted;  // y edges ascending (enables the leaf-pair range search)
    float mlc_xl[kMaxPairs], mlc_xr[kMaxPairs], mlc_yb[kMaxPairs], mlc_yt[kMaxPairs];
    float prof_r[kMaxProfile], prof_i[kMaxProfile], prof_s[kMaxProfile];
    float spec_mu[kMaxSpectrum], spec_pw[kMaxSpectrum], spec_sw[kMaxSpectrum];
};

struct CccsCones {
    int n_cones, total_steps;
    // directions (cone * 12 + azimuth) whose samples are interpolated in
    // software from the padded linear (TERMA, density) copy instead of the
    // texture unit, so that both the texture and the load/store paths work
    unsigned lsu_mask[3];
    float theta_deg[kMaxCones], Am[kMaxCones], am[kMaxCones], Bm[kMaxCones], bm[kMaxCones];
    int step_off[kMaxCones], n_steps[kMaxCones];
    float rl10[kMaxConeSteps];  // sample distance along the cone axis, mm
};

// Padded linear copy of the (TERMA, density) volume: one texel of border
// below and two above on every axis, so that software trilinear
// interpolation at any coordinate clamped to [-1, n] reads the border values
// (0, AIR_DENSITY) exactly where the texture unit would.
__host__ __device__ __forceinline__ long long td_pad_count(const Grid &g) {
    return (long long)(g.nx + 3) * (g.ny + 3) * (g.nz + 3);
}
__host__ __device__ __forceinline__ long long td_pad_index(const Grid &g, int i, int j, int k) {
    return (long long)(i + 1) + (long long)(g.nx + 3) * ((j + 1) + (long long)(g.ny + 3) * (k + 1));
}

// The texture unit's linear filtering of the (TERMA, density) volume at
// unnormalised coordinate tc, in software from the padded copy: coordinates
// shifted by half a texel, clamped into the border shell, fractions rounded
// to 1/256 as the texture unit stores its weights.
__device__ __forceinline__ float2 td_fetch_lin(const float2 *__restrict__ td, const Grid &g, float3 tc) {
    const float x = fminf(fmaxf(tc.x - 0.5f, -1.0f), (float)g.nx);
    const float y = fminf(fmaxf(tc.y - 0.5f, -1.0f), (float)g.ny);
    const float z = fminf(fmaxf(tc.z - 0.5f, -1.0f), (float)g.nz);
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const float a = rintf((x - fx) * 256.0f) * (1.0f / 256.0f);
    const float b = rintf((y - fy) * 256.0f) * (1.0f / 256.0f);
    const float c = rintf((z - fz) * 256.0f) * (1.0f / 256.0f);
    const int px = g.nx + 3;
    const long long pxy = (long long)px * (g.ny + 3);
    const long long base = td_pad_index(g, (int)fx, (int)fy, (int)fz);
    const float2 *p0 = td + base, *p1 = p0 + pxy;
    const float2 v000 = __ldg(p0), v100 = __ldg(p0 + 1), v010 = __ldg(p0 + px), v110 = __ldg(p0 + px + 1);
    const float2 v001 = __ldg(p1), v101 = __ldg(p1 + 1), v011 = __ldg(p1 + px), v111 = __ldg(p1 + px + 1);
    float2 r;
    {
        const float x00 = fmaf(a, v100.x - v000.x, v000.x), x10 = fmaf(a, v110.x - v010.x, v010.x);
        const float x01 = fmaf(a, v101.x - v001.x, v001.x), x11 = fmaf(a, v111.x - v011.x, v011.x);
        const float y0 = fmaf(b, x10 - x00, x00), y1 = fmaf(b, x11 - x01, x01);
        r.x = fmaf(c, y1 - y0, y0);
    }
    {
        const float x00 = fmaf(a, v100.y - v000.y, v000.y), x10 = fmaf(a, v110.y - v010.y, v010.y);
        const float x01 = fmaf(a, v101.y - v001.y, v001.y), x11 = fmaf(a, v111.y - v011.y, v011.y);
        const float y0 = fmaf(b, x10 - x00, x00), y1 = fmaf(b, x11 - x01, x01);
        r.y = fmaf(c, y1 - y0, y0);
    }
    return r;
}

// Beamlet fluence map on the head frame's isocentre plane (beam's eye view):
// beamlet (ia, ib) sits at (a0 + ia*pitch, b0 + ib*pitch); values are
// interpolated bilinearly at each voxel's ray and clamped to the map's edge.
struct FluenceMap {
    int na, nb;
    float a0, b0, inv_pitch;
    float sad;  // primary source distance (projection onto the isocentre plane)
};

// Validates the model/control point and fills the parameter blocks.
// spacing_cm is the CCCS step (the isotropic voxel spacing in cm).
void build_photon_params(const dc_photon_model &m, const dc_control_point &cp, float spacing_cm,
                         PhotonParams &P, CccsCones &C);

// Device work buffers of one photon calculation.
struct PhotonWork {
    float *wet = nullptr;          // radiological depth, n floats
    float *electron = nullptr;     // electron contamination, n floats
    unsigned *n_active = nullptr;  // number of CCCS voxels (device counter)
    int *active = nullptr;         // CCCS voxel list, n ints
    float4 *dirs = nullptr;        // kMaxCones*12 image-frame cone directions
    cudaTextureObject_t dens_tex = 0;  // density, border AIR_DENSITY
    cudaSurfaceObject_t td_surf = 0;   // (TERMA, density) float2 array
    cudaTextureObject_t td_tex = 0;    // its texture, border (0, AIR_DENSITY)
    DeviceBuffer *xlat = nullptr;      // ray-lattice storage of the depth pass (lattice mode)
    // (TERMA, density) on a linear grid padded by one texel below and two
    // above on every axis with the texture's border values, or null; written
    // by the TERMA kernel, read by the CCCS's software-interpolated samples
    DeviceBuffer *td_lin = nullptr;
    unsigned *depth_stats = nullptr;   // device word: voxels the depth pass marched (or null)
    int depth_mode = 0;                // 0: per-voxel march, 1: ray lattice (DeviceContext::photon_depth_mode)
};

// Ray trace + TERMA + cone directions.  dose_dev (or null) receives the zero
// of every masked voxel, terma_out (or null) a linear TERMA copy.
void enqueue_terma(DeviceContext &ctx, const Grid &g, const Frame &f, const PhotonParams &P, const CccsCones &C,
                   const PhotonWork &w, float *dose_dev, float *terma_out, cudaStream_t s);
// CCCS of every active voxel listed by the last enqueue_terma.
void enqueue_cccs(DeviceContext &ctx, const Grid &g, const Frame &f, const CccsCones &C, const PhotonWork &w,
                  float dose_scale, float *dose_dev, cudaStream_t s);
// CCCS at n listed voxels into out[0..n).
void enqueue_cccs_points(DeviceContext &ctx, const Grid &g, const Frame &f, const CccsCones &C, const PhotonWork &w,
                         float dose_scale, const int *voxels, int n, float *out, cudaStream_t s);

// Fluence-modulated TERMA (m*T0) and electron term (m*E0) of the photon
// beam's work set, for a following enqueue_cccs (dc_fluence.cu).
void enqueue_fluence_modulate(DeviceContext &ctx, const Grid &g, const Frame &f, const FluenceMap &M,
                              const float *F, const float *T0, const float *E0, const PhotonWork &w, cudaStream_t s);
// grad_F[beamlet] = d(sum_v grad_dose_v D_v)/dF (float64), with h (n floats)
// as scratch for s K^T grad_dose; the work set's active list, directions and
// density channel must be those of the TERMA pass that produced T0, E0.
void enqueue_fluence_adjoint(DeviceContext &ctx, const Grid &g, const Frame &f, const CccsCones &C,
                             const FluenceMap &M, float dose_scale, const float *T0, const float *E0,
                             const PhotonWork &w, const float *grad_dose, float *h, double *grad_F, cudaStream_t s);

// The CCCS by cone-direction sweeps over line lattices (dc_cccs_sweep.cu):
// an approximation of enqueue_cccs (no per-voxel kernel tilt, windows
// interpolated between lattice lines).  Synchronises the stream once (the
// active voxels' bounding box sizes the lattices).
void enqueue_cccs_sweep(DeviceContext &ctx, const Grid &g, const Frame &f, const CccsCones &C, const PhotonWork &w,
                        float dose_scale, float *dose_dev, DeviceBuffer &lattice, DeviceBuffer &acc_buf,
                        DeviceBuffer &box_buf, cudaStream_t s);

// Enqueues ray trace -> TERMA -> CCCS for one control point on stream s.
// The density volume must already be in ctx.density; dose_dev: device output.
void run_photon_pipeline(DeviceContext &ctx, const Grid &g, const Frame &f, const PhotonParams &P,
                         const CccsCones &C, float dose_scale, float *dose_dev, cudaStream_t s);

}  // namespace dc
