// dc_kernels.cuh — launch wrappers of the DoseCUDA B200 kernels.
#pragma once

#include <vector>

#include "dc_common.cuh"
#include "dc_runtime.cuh"

namespace dc {

// ---- radiological depth (dc_wet.cu) --------------------------------------
void launch_wet_march(DeviceContext &ctx, const Grid &g, const Frame &f, cudaTextureObject_t density,
                      float *wet, cudaStream_t s);
void launch_wet_smooth(DeviceContext &ctx, const Grid &g, const Frame &f, const float *wet, float *wet_s,
                       cudaStream_t s);

// ---- photon radiological depth on a ray lattice (dc_xray.cu) -------------
// Rays from the source through (a0 + ia*pa, b0 + ib*pa) on the head frame's
// isocentre plane; nodes at distances (m0 + m) mm from the source.
struct XrayLattice {
    float a0, b0, pa, inv_pa;
    int na, nb, m0, nm;
    float sad;         // source distance (mm)
    float tau;         // largest spread of the four rays' sums interpolated (mm x density), ...
    float rho_floor;   // ... weighed by the voxel's own density, at least this
    float tau_big;     // largest weighed spread accepted where ...
    float tau_curv;    // ... the 4 x 4 rays' second-difference error estimate is below this
    float wet_exact;   // WET (cm) below which a voxel's depth is marched exactly ...
    float tau_shallow; // ... where its four lattice rays' sums spread by more than this (mm x density)
    float3 src;        // source, image frame relative to the isocentre
    float3 ex, ey, ez; // head-frame axes in the image frame
};
// Lattice geometry for this grid and beam; false when the lattice does not
// apply (source inside or next to the volume, lattice too large).
bool plan_xray_lattice(const Grid &g, const Frame &f, XrayLattice &L);
// Photon WET (cm) of every voxel through the lattice, with the reference's
// march for the voxels the lattice cannot serve (listed in list/n_list, which
// need room for every voxel); the plain march when the lattice does not apply.
// Voxels whose WET comes out below `wet_exact` (cm) are marched exactly too
// where their lattice rays disagree (+infinity: the plain march for every
// voxel).  `stats` (device word, or
// null) receives the number of voxels marched from the list (0xffffffff when
// the lattice did not apply).
void launch_xray_depth(DeviceContext &ctx, const Grid &g, const Frame &f, cudaTextureObject_t density, float *wet,
                       int *list, unsigned *n_list, DeviceBuffer &lattice, unsigned *stats, float wet_exact,
                       cudaStream_t s);

// ---- proton pencil beam (dc_proton.cu) -----------------------------------
// One energy layer: a run of spots with the same energy id
// (reference Layer, IMPTClasses.cuh:17-26; importLayers IMPTClasses.cu:37-67).
struct LayerRec {
    int spot_start;
    int n_spots;
    int energy_id;
    float r80;
    float A, B, C;  // sigma_air quadratic coefficients (divergence_params[2..4])
    float rcut;     // lateral cut-off radius (mm): 6 x the widest halo sigma of the layer
};

// Fills LayerRec::rcut on the device from the LUT rows (layer_rcut_kernel).
void launch_layer_rcut(const Grid &g, const Frame &f, LayerRec *layers, int n_layers, const float *lut_depths,
                       const float *lut_sigmas, int lut_len, cudaStream_t s);

// Spot record with the divergent-axis constants precomputed on the host:
// t = (x/VSADX, y/VSADY, -1), inv_t2 = 1/|t|^2 (IMPTClasses.cu:123-133).
// `orig` is the spot's row in the caller's spot list (records are sorted by
// energy id).
struct SpotRec {
    float x, y, mu;
    int orig;
    float tx, ty, inv_t2, pad1;
};

struct ProtonTables {
    const LayerRec *layers;
    const SpotRec *spots;
    const float *lut_depths;  // [n_energies][lut_len]
    const float *lut_sigmas;
    const float *lut_idds;
    int n_layers;
    int lut_len;
};

// Per-mode inputs/outputs of the pencil-beam kernel family (all device
// pointers; spot-indexed arrays are in the caller's spot order).
struct PbExtra {
    const float *mu = nullptr;         // dose/adjoint: MU per spot (nullptr: the table's MU)
    const float *grad_dose = nullptr;  // adjoint: dObjective/dDose per voxel
    double *grad_mu = nullptr;         // adjoint: += sum_v grad_dose(v) * K_s(v)
    unsigned *spot_max = nullptr;      // spot-max: max_v K_s(v) as float bits
    const float *thr = nullptr;        // count/fill: keep K_s(v) >= thr[s]
    int *counts = nullptr;             // count: entries per voxel row
    const long long *row_ptr = nullptr;  // fill: CSR row starts (voxel rows)
    int *col = nullptr;                // fill: spot index
    float *val = nullptr;              // fill: dose per MU
    long long cap = 0;                 // fill: capacity of col/val
    // voxel-list mode (dose / adjoint only): the CTA's voxels are entries of
    // `list` (flat voxel indices) instead of an image tile; `list_out` (dose)
    // and grad_dose (adjoint) are then compact arrays indexed like `list`.
    const int *list = nullptr;
    int n_list = 0;
    float *list_out = nullptr;
    // image-tile modes: the tiles along z launched, [tile_z0, tile_z1) (tile_z1
    // < 0: to the last)
    int tile_z0 = 0, tile_z1 = -1;
};

enum PbMode { kPbDose = 0, kPbAdjoint = 1, kPbSpotMax = 2, kPbCount = 3, kPbFill = 4 };

// First bounds violation recorded by each translation unit's checked
// accesses since the last call, and cleared (debug builds; 0 otherwise).
unsigned long long take_bounds_wet();
unsigned long long take_bounds_photon();
unsigned long long take_bounds_proton();
unsigned long long take_bounds_basis();
unsigned long long take_bounds_noalloc();
unsigned long long take_bounds_xray();
unsigned long long take_bounds_fluence();
unsigned long long take_bounds_sweep();

// Builds the sorted spot table and the layer table on the host.  Throws
// Error(DC_ERR_VALUE) for malformed input.
void build_proton_tables(const float *spots, int n_spots, const float *dvp, int n_energies, int dvp_len,
                         float vsadx, float vsady, std::vector<LayerRec> &layers,
                         std::vector<SpotRec> &spot_recs);

void launch_pencil_beam(DeviceContext &ctx, const Grid &g, const Frame &f, const ProtonTables &t,
                        const float *wet_s, float *dose, cudaStream_t s, const float *mu_dev = nullptr,
                        int tile_z0 = 0, int tile_z1 = -1);
// Voxels along z per tile of the single-beam pencil-beam kernel: tiles
// [z0, z1) cover planes [z0 * depth, z1 * depth).
int pencil_beam_tile_depth();
// Dose (x.list_out) or adjoint (x.grad_dose compact, x.grad_mu) of the voxels
// in x.list only; mode kPbDose or kPbAdjoint.
void launch_pencil_beam_list(DeviceContext &ctx, int mode, const Grid &g, const Frame &f, const ProtonTables &t,
                             const float *wet_s, const PbExtra &x, cudaStream_t s);

// The other members of the family (see PbMode); `name` labels the profiler entry.
void launch_pencil_beam_mode(DeviceContext &ctx, int mode, const Grid &g, const Frame &f, const ProtonTables &t,
                             const float *wet_s, const PbExtra &x, cudaStream_t s);

// ---- dose-influence matrix, count-then-fill (dc_beam.cu) -------------------
// Count pass of one beam: spot_max[s] = max_v K_s(v) (float bits), thr[s] =
// cutoff * spot_max[s], counts[v] = #{s : K_s(v) >= thr[s]}.  The fill pass is
// launch_pencil_beam_mode(kPbFill) with the same thresholds and the row starts.
void launch_influence_count(DeviceContext &ctx, const Grid &g, const Frame &f, const ProtonTables &t, int n_spots,
                            const float *wet, float cutoff, unsigned *spot_max, float *thr, int *counts,
                            cudaStream_t s);
// Exclusive scan of n int counts into n + 1 int64 row starts (row_ptr[n] =
// the total); `scratch` grows to ceil(n / 1024) + 1 int64 block sums.
void launch_scan_counts(const int *counts, long long n, long long *row_ptr, DeviceBuffer &scratch, cudaStream_t s);

// ---- batched pencil beam (persistent, many plans) -------------------------
struct PbBatchBeam {
    Frame f;
    ProtonTables t;
    const float *wet;  // smoothed WET of this beam (cm)
    const float *mu;   // spot weights (nullptr: the table's MU)
};

struct PbBatchPlan {
    Grid g;
    float *dose;  // sum over the plan's beams
    int beam0, n_beams;
};

// Work items are (plan, tile) pairs; tile = bz * tiles_x * tiles_y + by * tiles_x + bx
// for the variant's tile shape.  `next` is the device queue head (reset here).
int pencil_beam_batch_variants();
void pencil_beam_batch_tile(int variant, int *threads_y, int *voxels_per_thread);
long long pencil_beam_batch_tiles(int variant, const Grid &g);  // tiles of grid g
void launch_pencil_beam_batch(DeviceContext &ctx, int variant, const PbBatchPlan *plans, const PbBatchBeam *beams,
                              const int2 *items, int n_items, unsigned *next, int lut_len, cudaStream_t s);

// Piecewise-linear HU table (strictly increasing HU), kernel parameter.
constexpr int kMaxHuPoints = 64;
struct HuTable {
    int n;
    double hu[kMaxHuPoints];
    double val[kMaxHuPoints];
};
// HU -> table value for every voxel: into out (linear, or null) and/or the
// float cudaArray behind surf (or 0).
void launch_hu_convert(const HuTable &t, const float *hu, int nx, int ny, int nz, float *out, cudaSurfaceObject_t surf,
                       cudaStream_t s);

}  // namespace dc
