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
    float theta_deg[kMaxCones], Am[kMaxCones], am[kMaxCones], Bm[kMaxCones], bm[kMaxCones];
    int step_off[kMaxCones], n_steps[kMaxCones];
    float rl10[kMaxConeSteps];  // sample distance along the cone axis, mm
};

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
    unsigned *depth_stats = nullptr;   // device word: voxels the depth pass marched (or null)
    int depth_mode = 1;                // 0: per-voxel march, 1: ray lattice (DeviceContext::photon_depth_mode)
};

// Enqueues the density-independent head factors of every voxel (collimator
// transmission, off-axis factors) on the context's side stream, after the
// work enqueued on s so far.  The next enqueue_terma joins it; without this
// call enqueue_terma forks it itself, beside the depth pass.
// Head-transmission skip bound check: the largest float x in [lo, hi] whose
// device erff(+-x) is not exactly +-1 (0 when there is none; synchronous,
// current device), and the bound the head kernel skips leaf pairs beyond.
float photon_erf_unsaturated(float lo, float hi);
float photon_erf_skip_bound();
void photon_head_fork(DeviceContext &ctx, const Grid &g, const Frame &f, const PhotonParams &P, cudaStream_t s);
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
