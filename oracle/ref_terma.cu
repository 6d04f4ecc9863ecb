// ref_terma.cu — CHECKER ONLY: runs the reference's own photon ray trace and
// TERMA kernels (rayTraceKernel, CudaClasses.cu:180-228; termaKernel,
// IMRTClasses.cu:209-250), compiled from the reference sources by
// oracle/build_ref.sh, and hands back their intermediate volumes (WET, TERMA,
// electron term), which the reference's photon_dose_cuda
// (IMRTClasses.cu:356-405) keeps on the device and frees.
//
// The reference's beam and dose objects are built here the way its extension
// builds them for one control point (dosemodule.cu:471-534: gantry + 180,
// isocentre relative to the origin, spacing[0] as the isotropic spacing), and
// the two kernels are launched with the reference's own TILE_WIDTH^3 blocks.
// Used by tests that pin where the reference's TERMA departs from the
// algorithm; never by the engine.
#include <cstdio>
#include <cstring>
#include <vector>

#include "CudaClasses.cuh"
#include "IMRTClasses.cuh"
#include "TextureClasses.cuh"

namespace {

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

template <class T>
T *upload(DevBuf &b, const T *h, size_t n) {
    if (cudaMalloc(&b.p, n * sizeof(T) > 0 ? n * sizeof(T) : 4) != cudaSuccess) return nullptr;
    if (n && cudaMemcpy(b.p, h, n * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
    return static_cast<T *>(b.p);
}

int report(char *err, int len, const char *what, cudaError_t e) {
    if (err && len > 0) std::snprintf(err, (size_t)len, "%s: %s", what, cudaGetErrorString(e));
    return 1;
}

}  // namespace

// scalars: mu_cal, primary/scatter source distance, primary/scatter source
// size, mlc_distance, scatter weight, electron attenuation, electron source
// weight, electron fitted dmax (the model attributes dosemodule.cu:400-411
// reads, in that order, without the two unused transmissions).
extern "C" int ref_photon_terma(int gpu_id, const float *density, int nz, int ny, int nx, float spacing,
                                const float origin[3], const float iso[3], float gantry, float collimator,
                                float couch, const float scalars[10], int n_prof, const float *prof_r,
                                const float *prof_i, const float *prof_s, int n_spec, const float *spec_mu,
                                const float *spec_pw, const float *spec_sw, int n_pairs, const float *x1,
                                const float *x2, const float *yoff, const float *yw, float mu, float *wet_out,
                                float *terma_out, float *electron_out, char *err, int err_len) {
    try {
        cudaError_t e = cudaSetDevice(gpu_id);
        if (e != cudaSuccess) return report(err, err_len, "cudaSetDevice", e);
        size_t dims[3] = {(size_t)nz, (size_t)ny, (size_t)nx};
        const size_t n = dims[0] * dims[1] * dims[2];

        IMRTBeam::Model model{};
        model.n_profile_points = n_prof;
        model.n_spectral_energies = n_spec;
        model.mu_cal = scalars[0];
        model.primary_src_dist = scalars[1];
        model.scatter_src_dist = scalars[2];
        model.primary_src_size = scalars[3];
        model.scatter_src_size = scalars[4];
        model.mlc_distance = scalars[5];
        model.scatter_src_weight = scalars[6];
        model.electron_attenuation = scalars[7];
        model.electron_src_weight = scalars[8];
        model.electron_fitted_dmax = scalars[9];

        float rel_iso[3] = {iso[0] - origin[0], iso[1] - origin[1], iso[2] - origin[2]};
        IMRTDose h_dose(dims, spacing);
        IMRTBeam h_beam(rel_iso, fmodf(gantry + 180.0f, 360.0f), couch, collimator, &model);
        h_beam.n_mlc_pairs = n_pairs;
        h_beam.mu = mu;

        IMRTDose d_dose(&h_dose);
        IMRTBeam d_beam(&h_beam);
        std::vector<MLCPair> pairs((size_t)n_pairs);
        for (int q = 0; q < n_pairs; ++q) pairs[(size_t)q] = MLCPair{x1[q], x2[q], yoff[q], yw[q]};
        DevBuf b_mlc, b_pr, b_pi, b_ps, b_sm, b_pw, b_sw, b_wet, b_terma, b_elec, b_dose, b_beam, b_dosep;
        d_beam.mlc = upload(b_mlc, pairs.data(), pairs.size());
        d_beam.model.profile_radius = upload(b_pr, prof_r, (size_t)n_prof);
        d_beam.model.profile_intensities = upload(b_pi, prof_i, (size_t)n_prof);
        d_beam.model.profile_softening = upload(b_ps, prof_s, (size_t)n_prof);
        d_beam.model.spectrum_attenuation_coefficients = upload(b_sm, spec_mu, (size_t)n_spec);
        d_beam.model.spectrum_primary_weights = upload(b_pw, spec_pw, (size_t)n_spec);
        d_beam.model.spectrum_scatter_weights = upload(b_sw, spec_sw, (size_t)n_spec);
        d_beam.model.kernel = nullptr;  // not read by the ray trace or TERMA
        float *wet = nullptr, *terma = nullptr, *elec = nullptr, *dose = nullptr;
        for (auto *pp : {&b_wet, &b_terma, &b_elec, &b_dose}) {
            e = cudaMalloc(&pp->p, n * sizeof(float));
            if (e != cudaSuccess) return report(err, err_len, "cudaMalloc", e);
            cudaMemset(pp->p, 0, n * sizeof(float));
        }
        wet = static_cast<float *>(b_wet.p);
        terma = static_cast<float *>(b_terma.p);
        elec = static_cast<float *>(b_elec.p);
        dose = static_cast<float *>(b_dose.p);
        d_dose.WETArray = wet;
        d_dose.DoseArray = dose;
        IMRTBeam *beam_dev = upload(b_beam, &d_beam, 1);
        IMRTDose *dose_dev = upload(b_dosep, &d_dose, 1);
        if (!beam_dev || !dose_dev || !d_beam.mlc) return report(err, err_len, "upload", cudaGetLastError());

        auto density_tex = Texture3D::fromHostData(density, h_dose.img_sz, cudaFilterModeLinear, AIR_DENSITY);
        dim3 block(TILE_WIDTH, TILE_WIDTH, TILE_WIDTH);
        dim3 grid((d_dose.img_sz.k + TILE_WIDTH - 1) / TILE_WIDTH, (d_dose.img_sz.j + TILE_WIDTH - 1) / TILE_WIDTH,
                  (d_dose.img_sz.i + TILE_WIDTH - 1) / TILE_WIDTH);
        rayTraceKernel<<<grid, block>>>(dose_dev, beam_dev, density_tex);
        termaKernel<<<grid, block>>>(dose_dev, beam_dev, terma, elec);
        e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return report(err, err_len, "kernels", e);
        if (wet_out) cudaMemcpy(wet_out, wet, n * sizeof(float), cudaMemcpyDeviceToHost);
        if (terma_out) cudaMemcpy(terma_out, terma, n * sizeof(float), cudaMemcpyDeviceToHost);
        if (electron_out) cudaMemcpy(electron_out, elec, n * sizeof(float), cudaMemcpyDeviceToHost);
        e = cudaGetLastError();
        if (e != cudaSuccess) return report(err, err_len, "copy back", e);
        return 0;
    } catch (const std::exception &ex) {
        if (err && err_len > 0) std::snprintf(err, (size_t)err_len, "%s", ex.what());
        return 1;
    }
}
