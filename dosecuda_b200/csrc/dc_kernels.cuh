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

// ---- proton pencil beam (dc_proton.cu) -----------------------------------
// One energy layer: a run of spots with the same energy id
// (reference Layer, IMPTClasses.cuh:17-26; importLayers IMPTClasses.cu:37-67).
struct LayerRec {
    int spot_start;
    int n_spots;
    int energy_id;
    float r80;
    float A, B, C;  // sigma_air quadratic coefficients (divergence_params[2..4])
    float pad;
};

// Spot record with the divergent-axis constants precomputed on the host:
// t = (x/VSADX, y/VSADY, -1), inv_t2 = 1/|t|^2 (IMPTClasses.cu:123-133).
struct SpotRec {
    float x, y, mu, pad0;
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

// Builds the sorted spot table and the layer table on the host.  Throws
// Error(DC_ERR_VALUE) for malformed input.
void build_proton_tables(const float *spots, int n_spots, const float *dvp, int n_energies, int dvp_len,
                         float vsadx, float vsady, std::vector<LayerRec> &layers,
                         std::vector<SpotRec> &spot_recs);

void launch_pencil_beam(DeviceContext &ctx, const Grid &g, const Frame &f, const ProtonTables &t,
                        const float *wet_s, float *dose, cudaStream_t s);

}  // namespace dc
